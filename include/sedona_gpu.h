/* sedona_gpu.h -- C ABI of the B200 implementation of Sedona's implicit
 * Monte Carlo transport step (packet propagation + per-zone opacity build).
 *
 * The boundary is the reference `transport` class (src/transport/transport.h:45-320).
 * A host `transport` keeps owning its std::vectors; it flattens zone data to
 * the structure-of-arrays structs below, calls these entry points, and copies
 * results back into the same vectors it already writes out
 * (J_nu_, zone e_abs/e_rad/f*_rad, spectrum_array flux/click, opacity tables).
 *
 * Conventions
 *  - Every entry point returns 0 (SED_OK) or a positive sed_status code and
 *    never exits the process; sed_last_error() gives the message.
 *  - All pointers in the structs are HOST pointers unless a name ends in
 *    `_dev`.  Nothing passed in is retained after a call returns.
 *  - One context = one CUDA stream on one device; calls on a context are
 *    synchronous with respect to the caller and not re-entrant.
 *  - Arrays over (zone, frequency) are zone-major: a[zone * n_nu + bin].
 */
#ifndef SEDONA_GPU_H
#define SEDONA_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum sed_status {
  SED_OK = 0,
  SED_ERR_ARG = 1,       /* invalid argument or inconsistent sizes */
  SED_ERR_CUDA = 2,      /* CUDA runtime error (message has the CUDA string) */
  SED_ERR_CAPACITY = 3,  /* packet capacity (particles_max_total) exceeded */
  SED_ERR_STATE = 4,     /* call out of order (e.g. step before set_grid) */
  SED_ERR_LIMIT = 5,     /* a packet hit the per-packet segment limit */
  SED_ERR_NOMEM = 6      /* device allocation failed */
};

/* Warnings of a step (sed_step_stats.warnings): conditions the reference
 * reports on stderr and carries on from. */
enum sed_warning {
  /* the core packets did not fit next to the census and the radioactive
   * packets (particles_max_total): none were emitted this step and the step
   * propagated the others, as emit_inner_source does after printing
   * "# Not enough particle space" (src/transport/emission.cpp:391-392) */
  SED_WARN_NO_PARTICLE_SPACE = 1
};

/* Bin-edge array with the semantics of locate_array
 * (src/utils/locate_array.h:15-217): n bins, `right[i]` is the right wall of
 * bin i, `min` the left wall of bin 0; bins are closed on the left. */
enum sed_locate_type { SED_LOC_FLEX = 0, SED_LOC_LIN = 1, SED_LOC_LOG = 2, SED_LOC_NONE = 3 };
typedef struct sed_locate_grid {
  int32_t n;
  int32_t type;          /* enum sed_locate_type */
  double min;
  double del;            /* lin: bin width; log: fractional width (1+del ratio) */
  const double* right;   /* n right walls */
} sed_locate_grid;

enum sed_grid_type { SED_GRID_1D_SPHERE = 0, SED_GRID_3D_CART = 1 };
enum sed_precision { SED_PREC_FP64 = 0, SED_PREC_MIXED = 1 };

/* Transport-step parameters: the Lua parameters transport::init reads
 * (src/transport/transport_init.cpp:82-363) that the step depends on. */
typedef struct sed_transport_params {
  int32_t steady_state;          /* transport_steady_iterate > 0 */
  int32_t radiative_eq;          /* transport_radiative_equilibrium */
  int32_t boundary_in_reflect;   /* transport_boundary_in_reflect */
  int32_t boundary_out_reflect;  /* transport_boundary_out_reflect */
  int32_t store_Jnu;             /* transport_store_Jnu */
  int32_t omit_scattering;       /* opacity_no_scattering */
  int32_t core_fix_luminosity;   /* core_fix_luminosity */
  int32_t tally_forces;          /* 1: tally fx/fy/fz/fr_rad as the reference does */
  int32_t precision;             /* enum sed_precision: opacity tables FP64 or FP32 */
  uint32_t rng_seed;             /* transport_rng_seed (Philox key) */
  int64_t max_particles;         /* particles_max_total */
  int64_t core_n_emit;           /* core_n_emit */
  double core_radius;            /* core_radius */
  double core_luminosity;        /* L_core used for this step (core_luminosity(t)) */
  double core_temperature;       /* core_temperature */
  double core_photon_frequency;  /* core_photon_frequency */
  double fleck_alpha;            /* transport_fleck_alpha */
  int32_t max_segments;          /* per-packet segment limit; 0 = default (10^7) */
  int32_t reserved;
  int64_t first_packet_id;       /* Philox stream id of this context's first packet:
                                    rank r of N replicas uses r * core_n_emit, so
                                    the N emissions form one packet ensemble */
  sed_locate_grid nu_grid;       /* transport_nu_grid */
  sed_locate_grid spec_time;     /* spectrum_time_grid */
  sed_locate_grid spec_nu;       /* spectrum_nu_grid */
  sed_locate_grid spec_mu;       /* mu grid: init(-1, 1, spectrum_n_mu) */
  sed_locate_grid spec_phi;      /* phi grid: init(0, 2*pi, spectrum_n_phi) */
  /* radioactive source (transport::emit_radioactive, src/transport/emission.cpp:163-243);
   * zero-initialised fields leave it off */
  int64_t n_emit_radioactive;    /* particles_n_emit_radioactive */
  int32_t force_rprocess_heating;/* force_rprocess_heating */
  int32_t reserved3;
  sed_locate_grid gamma_nu;      /* frequency grid of the gamma-ray spectrum (which shares
                                    spec_time, spec_mu, spec_phi); n = 0: one catch-all bin.
                                    The reference passes spectrum_nu_grid here
                                    (transport_init.cpp:170-173), not gamma_nu_grid */
  /* discrete diffusion in optically thick zones (1D spheres):
   * transport_use_ddmc (0 off; 1 IMD, Gentile 2001, discrete_diffuse_IMD
   * with the per-step hop probabilities of compute_diffusion_probabilities,
   * src/transport/discrete_diffusion.cpp:18-110, 687-756; 2 DDMC, Densmore
   * et al. 2007, src/transport/discrete_diffusion.cpp:114-404) and
   * transport_ddmc_tau_threshold: a zone is diffusive for a photon when its
   * total opacity at the photon's comoving frequency times the zone width
   * exceeds it */
  int32_t use_ddmc;
  int32_t reserved4;
  double ddmc_tau;
} sed_transport_params;

/* Zone geometry and gas state (grid_general + zone, src/grid/grid_general.h:34-147,
 * src/grid/zone.h:9-50), flattened to structure-of-arrays. */
typedef struct sed_grid {
  int32_t type;                  /* enum sed_grid_type */
  int32_t n_zones;
  int32_t homologous;            /* hydro_module == "homologous" (v = x/t) */
  int32_t n_elems;
  double t_now;                  /* grid time: homologous v = x / t_now */
  /* 1D sphere: r_out[n_zones] right walls, r_min left wall of zone 0 */
  double r_min;
  const double* r_out;
  const double* v_r;             /* zone outer-edge radial velocity (non-homologous only) */
  /* 3D Cartesian: nx*ny*nz zones, index i*ny*nz + j*nz + k; each axis is a
   * locate_array (flex when read from x_out/y_out/z_out, lin when from dr),
   * src/grid/grid_3D_cart.cpp:120-166 */
  int32_t nx, ny, nz;
  sed_locate_grid x_axis, y_axis, z_axis;
  /* per-zone state */
  const double* vol;             /* zone volume */
  const double* rho;
  const double* T_gas;
  const double* e_gas;           /* only for the Fleck factor when fleck_alpha != 0 */
  const double* total_grey_opacity; /* zone total_grey_opacity (cm^2/g); 0 = use microphysics */
  const double* X;               /* mass fractions [n_zones * n_elems] */
  const int32_t* elem_Z;         /* [n_elems] */
  const int32_t* elem_A;         /* [n_elems] */
} sed_grid;

/* Opacity switches: the opacity_* Lua parameters GasState reads
 * (src/transport/transport_init.cpp:206-249). */
typedef struct sed_opacity_params {
  int32_t use_electron_scattering;
  int32_t use_free_free;
  int32_t use_bound_free;
  int32_t use_line_expansion;
  int32_t use_fuzz_expansion;
  int32_t n_atom_zero_epsilon;
  const int32_t* atom_zero_epsilon;  /* atomic numbers with epsilon = 0 */
  double epsilon;                /* opacity_epsilon */
  double maximum_opacity;        /* opacity_maximum_opacity (cm^2/g) */
  double temp_min, temp_max;     /* limits_temp_min / limits_temp_max */
  double line_velocity_width;    /* line_velocity_width */
} sed_opacity_params;

/* Atomic data for the elements of the grid, in elem order (LTE subset of
 * IndividualAtomData, src/opacity/AtomicData.h:12-158, after the loader's
 * own post-processing: extra fully-ionized stage appended, E_ion and ic set,
 * photoionisation tables filled).  Offsets are prefix sums of length n+1. */
typedef struct sed_atomic_data {
  int32_t n_atoms;               /* must equal sed_grid.n_elems */
  const int32_t* ion_off;        /* [n_atoms+1] into ion arrays */
  const double* ion_chi;         /* ionisation energy (eV) */
  const int32_t* lev_off;        /* [n_atoms+1] into level arrays */
  const int32_t* lev_ion;
  const int32_t* lev_g;
  const int32_t* lev_ic;         /* level index (within the atom) it ionizes to, -1 none */
  const double* lev_E;           /* excitation energy (eV) */
  const double* lev_Eion;        /* ionisation threshold (eV) */
  const int32_t* photo_off;      /* [total levels + 1] into photo tables */
  const double* photo_E;         /* photoionisation table abscissae (eV) */
  const double* photo_s;         /* cross-section (cm^2) */
  const int32_t* line_off;       /* [n_atoms+1] level-to-level lines */
  const int32_t* line_l;
  const int32_t* line_u;
  const double* line_nu;
  const double* line_f;
  const int32_t* fuzz_off;       /* [n_atoms+1] fuzz lines */
  const double* fuzz_nu;
  const double* fuzz_gf;
  const double* fuzz_El;         /* lower-level energy (eV) */
  const int32_t* fuzz_ion;
} sed_atomic_data;

typedef struct sed_step_stats {
  int64_t n_packets;             /* packets propagated this step */
  int64_t n_escaped;
  int64_t n_absorbed;
  int64_t n_stopped;             /* still alive at the end of the step */
  int64_t n_segments;            /* propagate_monte_carlo loop iterations */
  int64_t n_scatters;            /* interaction events */
  int64_t n_limit;               /* packets stopped by the segment limit */
  int32_t kernel_launches;       /* kernels launched by the call */
  int32_t warnings;              /* sed_warning bits of the step */
  float ms_opacity;              /* device time of the opacity build */
  float ms_transport;            /* device time of emission + propagation */
  float ms_total;                /* device time of the whole call */
  float ms_propagate_kernel;     /* device time of the packet kernel alone */
} sed_step_stats;

typedef struct sed_ctx sed_ctx;

/* Creates a context on `device` (-1: current device).  Replaces the
 * allocations of transport::init (src/transport/transport_init.cpp:44-427). */
int sed_ctx_create(const sed_transport_params* params, int device, sed_ctx** out);

/* Copies zone geometry/state to the device.  Replaces grid->z[] reads on the
 * hot path (src/grid/grid_1D_sphere.cpp:494-590, grid_3D_cart.cpp:363-469). */
int sed_set_grid(sed_ctx* ctx, const sed_grid* grid);

/* Copies atomic data and computes line bins with locate_within_bounds
 * (AtomicData.cpp:851-852).  Replaces AtomicData/GasState::initialize. */
int sed_set_atomic_data(sed_ctx* ctx, const sed_atomic_data* atoms);
int sed_set_opacity_params(sed_ctx* ctx, const sed_opacity_params* op);

/* Builds abs/scat opacity, emissivity CDF, n_e, Planck/Rosseland means and
 * eps_imc for every zone.  Replaces transport::set_opacity
 * (src/transport/transport_opacity.cpp:21-260) incl. GasState::solve_state and
 * GasState::computeOpacity. */
int sed_set_opacity(sed_ctx* ctx, double dt);

/* Loads caller-computed tables instead of sed_set_opacity (abs, scat,
 * emissivity CDF are [n_zones * n_nu]; eps_imc is [n_zones]; scat may be NULL
 * when opacity_no_scattering). */
int sed_load_opacity(sed_ctx* ctx, const double* abs, const double* scat,
                     const double* emis_cdf, const double* eps_imc);

/* Wipes tallies, emits the core packets, propagates every packet, tallies
 * escapes and normalises J/e_abs/e_rad.  Replaces transport.cpp:46-124
 * (wipe_radiation, emit_particles, the propagate loop, spectrum count,
 * clean_up_particle_vector, steady-state rescale, reduce_radiation).
 * Core packets that would not fit next to the census and the radioactive
 * packets are not emitted: the step runs without them and sets
 * SED_WARN_NO_PARTICLE_SPACE in stats->warnings (emission.cpp:391-392). */
int sed_transport(sed_ctx* ctx, double dt, sed_step_stats* stats);

/* sed_set_opacity followed by sed_transport: transport::step
 * (src/transport/transport.cpp:26-140) without the temperature solve. */
int sed_step(sed_ctx* ctx, double dt, sed_step_stats* stats);

/* Results.  Sizes: spectrum n_t*n_nu*n_mu*n_phi (spectrum_array flux/click,
 * src/transport/spectrum_array.h:28-31); J_nu n_zones*n_nu (or n_zones when
 * store_Jnu = 0); zone arrays n_zones.  NULL pointers are skipped. */
int sed_get_spectrum(sed_ctx* ctx, double* flux, double* click);
int sed_get_zone_tallies(sed_ctx* ctx, double* J_nu, double* e_abs, double* e_rad,
                         double* fx, double* fy, double* fz, double* fr);
/* The opacity tables the packet kernel reads (transport::abs_opacity_,
 * scat_opacity_, emissivity_ after set_opacity, transport.h), n_zones*n_nu
 * each, widened to double from FP32 in the mixed-precision form; emis_cdf is
 * the normalised emissivity CDF.  Zone arrays n_zones. */
int sed_get_opacity(sed_ctx* ctx, double* abs, double* scat, double* emis_cdf,
                    double* n_elec, double* eps_imc, double* planck_mean,
                    double* rosseland_mean, double* L_thermal);

/* Per-packet outcome records of the last sed_transport (replay parity):
 * fate (ParticleFate enum, particle.h:9), final zone, number of deviates
 * drawn after emission, and state {x,y,z,Dx,Dy,Dz,t,e,nu} (t = t_obs for
 * escaped packets).  Recording costs memory traffic; enable it only for
 * checks.  Arrays hold n entries. */
int sed_record_packets(sed_ctx* ctx, int32_t enable);
int sed_get_packet_records(sed_ctx* ctx, int64_t n, int32_t* fate, int32_t* ind,
                           int32_t* draws, double* state9);

/* Number of packets carried to the next step: transport::n_particles, the
 * particle vector after clean_up_particle_vector (transport.cpp:91, 164-194).
 * A time-dependent step keeps its stopped packets, in the reference's vector
 * order, and propagates them first in the next step; a steady-state step
 * keeps none. */
int64_t sed_n_particles(sed_ctx* ctx);
/* The carried packets: zone, type (enum PType: 0 photon, 1 gamma-ray) and
 * {x, D, t, e, nu} of the first n (n <= sed_n_particles). */
int sed_get_particles(sed_ctx* ctx, int64_t n, int32_t* ind, int32_t* type, double* state9);
/* The inner source's luminosity and, when weights is not NULL, its spectrum:
 * weights[i] = L_nu dnu of frequency bin i (core_spectrum_file, read by
 * transport::setup_core_emission, src/transport/transport_init.cpp:486-537),
 * summed in bin order into the emission CDF and normalised as cdf_array
 * does.  The luminosity is what emit_inner_source divides among the packets
 * (emission.cpp:386-389); the host sets it each step from core_luminosity at
 * the transport clock when that is a function of time.  At context creation
 * the spectrum is a blackbody at core_temperature. */
int sed_set_core_source(sed_ctx* ctx, double luminosity, const double* weights);
/* transport::wipe_spectra (src/transport/transport_output.cpp:63-67): empties
 * the optical and gamma-ray spectra.  A steady-state step starts from empty
 * spectra (the driver wipes them every iteration, SedonaClass.cpp:349); a
 * time-dependent step adds to them. */
int sed_wipe_spectra(sed_ctx* ctx);
/* The transport clock (transport::t_now_): the first grid's t_now; a
 * time-dependent step advances it by dt (transport.cpp:136) while the grid's
 * time is the caller's (the hydro step moves it, hydro_homologous.cpp:27-45).
 * Emission times, the end of the step, decay rates and the Sobolev time of
 * the opacity build use it; velocities use the grid's time. */
int sed_set_time(sed_ctx* ctx, double t_now);
double sed_get_time(sed_ctx* ctx);
/* transport::initialize_particles (src/transport/emission.cpp:112-159): n
 * photons drawn in proportion to e_rad[zone] * vol (erg/cm^3, per zone), each
 * with a blackbody spectrum at the zone's gas temperature, isotropic in the
 * comoving frame, at the transport clock's time; they join the carried
 * packets.  Packet k draws from Philox stream first_packet_id + (carried
 * packets) + k at step number 0xFFFFFFFF.  SED_ERR_CAPACITY when n exceeds
 * particles_max_total. */
int sed_initialize_particles(sed_ctx* ctx, int64_t n, const double* e_rad);
const char* sed_last_error(sed_ctx* ctx);
void sed_ctx_destroy(sed_ctx* ctx);

/* Library version / build string (never NULL). */
const char* sed_version(void);

/* Packet counts of the following steps: core_n_emit (emit_inner_source) and
 * particles_n_emit_radioactive (emit_radioactive), as the host's time loop
 * changes them (particles_last_iter_pump on the last iteration,
 * emission.cpp:180-184 and 377-382; multiply_particles_n_emit_by_dt_over_dtmax,
 * :170-173).  SED_ERR_ARG for a negative count. */
int sed_set_emission(sed_ctx* ctx, double core_n_emit, int64_t n_emit_radioactive);

/* Radioactive source results of the last step (n_emit_radioactive > 0): the
 * escaping gamma-ray spectrum (gamma_spectrum, n_t*n_gamma_nu*n_mu*n_phi) and
 * per zone the decay luminosity per volume L_radio_emit and the deposited
 * luminosity per volume L_radio_dep (zone.h:41-42, normalised as
 * transport_mpi.cpp:419-420).  NULL pointers are skipped. */
int sed_get_gamma_spectrum(sed_ctx* ctx, double* flux, double* click);
int sed_get_radioactive_tallies(sed_ctx* ctx, double* L_radio_emit, double* L_radio_dep);

/* Radiative-equilibrium gas temperature of every zone after a transport step:
 * transport::solve_eq_temperature (src/transport/solve_equilibrium.cpp:66-96)
 * for LTE, i.e. per zone Brent's method (temp_brent_method, :227-320) on
 * sum_i 4 pi kappa_abs B_nu(T) dnu - e_abs over [limits_temp_min,
 * limits_temp_max] with the absorption opacities of the last opacity build;
 * with set_Tgas_to_Trad, T = (e_rad / a)^(1/4).  The new temperatures replace
 * the context's zone temperatures (the next sed_set_opacity uses them) and are
 * copied to T_gas when it is not NULL.  A zone where Brent exhausts its 100
 * iterations gets T = 0 as in the reference; their number goes to
 * *n_unsolved (may be NULL). */
int sed_solve_temperature(sed_ctx* ctx, int32_t set_Tgas_to_Trad, double* T_gas, int32_t* n_unsolved);

/* Sets the Philox step number the next transport (or weighted forward) of
 * the context draws with; each step advances it by one.  Runs given the same
 * step number consume the same deviates (common random numbers), as
 * transport_fix_rng_seed does for the reference's GSL streams
 * (src/transport/transport_init.cpp:93-104). */
int sed_set_rng_step(sed_ctx* ctx, uint32_t step);

/* ------------------------------------------------------------ differentiation
 * Gradient of the binned emergent spectrum with respect to the absorption
 * opacity, per zone and frequency band, by path replay.  No counterpart in
 * the reference (it has no adjoint); the checks are central finite
 * differences of the weighted forward itself with common random numbers.
 *
 * The weighted forward is the same transport step (homologous 1D sphere or
 * 3D Cartesian grid, after sed_set_opacity or sed_load_opacity) with one change of estimator:
 * interactions are sampled from the scattering opacity alone and absorption
 * is a continuous weight exp(-a dshift l) on each segment.  Its expected
 * spectrum is the reference's (radiative_eq = 0, fleck_alpha = 0, no
 * steady-state luminosity rescale are required), and for fixed deviates it
 * is a smooth function of the absorption opacity.  The absorption of zone z
 * in bin i is multiplied by abs_scale[z * n_bands + band], band = i * n_bands
 * / n_nu (NULL = all ones); gradients are with respect to those factors.
 * Spectrum and tallies are read with sed_get_spectrum / sed_get_zone_tallies
 * (tallies use each segment's average weight). */
int sed_diff_forward(sed_ctx* ctx, double dt, const double* abs_scale, int32_t n_bands, sed_step_stats* stats);
/* Vector-Jacobian product of the last weighted forward: grad_scale[z * n_bands
 * + k] = sum_s grad_flux[s] d flux[s] / d abs_scale[z, k].  Replays every
 * escaped packet from its Philox stream (nothing of its path was stored). */
int sed_diff_vjp(sed_ctx* ctx, const double* grad_flux, double* grad_scale, sed_step_stats* stats);
/* Vector-Jacobian product with respect to the density of each zone, the
 * opacity per unit mass held (absorption and scattering extinction of the
 * zone scale together): grad_rho[z] = sum_s grad_flux[s] d E[flux[s]] /
 * d ln rho_z.  Per escaped packet of weight w: the absorption weight's
 * pathwise derivative -w sum (a dshift l), and, because the scattering
 * opacity decides where the path goes, the score of the sampled path
 * w (n_scatterings - sum s dshift l) over the packet's segments in zone z
 * (a likelihood-ratio estimator: unbiased, noisier than the pathwise one). */
int sed_diff_vjp_density(sed_ctx* ctx, const double* grad_flux, double* grad_rho, sed_step_stats* stats);
/* Full Jacobian of the last weighted forward: jac[(s * n_zones + z) * n_bands
 * + k] = d flux[s] / d abs_scale[z, k], s over the n_spec spectrum bins.
 * The three replays need the context as the forward left it: any call of
 * sed_set_grid, sed_set_opacity, sed_load_opacity, sed_step, sed_transport,
 * sed_set_time, sed_initialize_particles, sed_set_core_source or
 * sed_set_emission in between makes them return SED_ERR_STATE. */
int sed_diff_jacobian(sed_ctx* ctx, double* jac, sed_step_stats* stats);

/* Device-pointer forms for callers whose data already lives on the GPU (a
 * torch tensor, another library's buffer): the same computations with every
 * array argument a device pointer of this context's device.  The caller's
 * work that writes those arrays must be complete before the call (the
 * library reads them on its own stream); the results are complete when the
 * call returns.  sed_diff_forward_dev also copies the binned spectrum
 * (n_spec doubles) into flux_dev when flux_dev is not NULL. */
int sed_diff_forward_dev(sed_ctx* ctx, double dt, const double* abs_scale_dev, int32_t n_bands, double* flux_dev,
                         sed_step_stats* stats);
int sed_diff_vjp_dev(sed_ctx* ctx, const double* grad_flux_dev, double* grad_scale_dev, sed_step_stats* stats);
int sed_diff_vjp_density_dev(sed_ctx* ctx, const double* grad_flux_dev, double* grad_rho_dev,
                             sed_step_stats* stats);

/* Per-zone density factors for the differentiable transport: both
 * extinctions of zone z in the tables of the last opacity build (or load)
 * are multiplied by rho_scale[z] (n_zones entries; the opacity per unit mass
 * held), in place of the tables the packet kernels read, until the next call
 * or build.  NULL puts the built tables back.  The built tables are kept on
 * the device, so repeated calls scale the build, never an earlier scaling.
 * The _dev form takes a device pointer.  No reference counterpart. */
int sed_diff_scale_extinction(sed_ctx* ctx, const double* rho_scale);
int sed_diff_scale_extinction_dev(sed_ctx* ctx, const double* rho_scale_dev);

/* ------------------------------------------------------------------ batches
 * Many independent 1D spherical ejecta models (grid_1D_sphere, homologous)
 * stepped together: one opacity build over all their zones and ONE packet
 * launch over all their packets, captured into CUDA graphs (opacity build,
 * packet kernel, normalisation) that are replayed every step.  Each model is what one reference run (one `transport` object,
 * src/transport/transport.h:45-320) would hold: its own zones, core source,
 * packet count, spectrum and zone tallies.  The batch shares the
 * frequency/spectrum grids, the transport switches, the opacity parameters,
 * the atomic data, the element list and the grid time t_now.  A model's
 * packets use that model's Philox key and stream ids, so its results are
 * those of a separate context with the same rng_seed and first_packet_id
 * (tallies up to summation order). */
typedef struct sed_batch sed_batch;

/* One model: the sed_grid fields of a 1D sphere plus the core_* parameters
 * and the Philox key/stream ids of sed_transport_params. */
typedef struct sed_batch_model {
  int32_t n_zones;
  int32_t reserved;
  double r_min;
  const double* r_out;               /* [n_zones] */
  const double* vol;                 /* [n_zones] */
  const double* rho;
  const double* T_gas;
  const double* e_gas;               /* may be NULL (zeros) */
  const double* total_grey_opacity;  /* may be NULL (zeros: microphysics) */
  const double* X;                   /* [n_zones * n_elems] mass fractions */
  int64_t core_n_emit;
  double core_radius;
  double core_luminosity;
  double core_temperature;
  uint32_t rng_seed;
  int32_t reserved2;
  int64_t first_packet_id;
} sed_batch_model;

/* Launch shape of the batched packet kernel: one of the compiled shapes
 * (variant -> threads per block / minimum blocks per SM), how many blocks
 * per SM to launch (0 = as many as fit) and how many consecutive packets a
 * thread claims per pop of the packet queue. */
typedef struct sed_batch_tuning {
  int32_t variant;
  int32_t threads;          /* output: threads per block of the variant */
  int32_t blocks_per_sm;
  int32_t queue_chunk;
  float ms;                 /* autotune: kernel time of the sample with this shape */
  int32_t n_tried;          /* autotune: shapes timed */
} sed_batch_tuning;

/* Creates a batch on `device`.  `common` supplies everything but the core_*
 * fields, rng_seed and first_packet_id, which come per model.  Replaces one
 * transport::init per model (transport_init.cpp:44-427). */
int sed_batch_create(const sed_transport_params* common, double t_now, int32_t n_elems, const int32_t* elem_Z,
                     const int32_t* elem_A, int32_t n_models, const sed_batch_model* models, int device,
                     sed_batch** out);
int sed_batch_set_opacity_params(sed_batch* b, const sed_opacity_params* op);
int sed_batch_set_atomic_data(sed_batch* b, const sed_atomic_data* atoms);

/* Times the batched packet kernel on a sample of every model's packets
 * (`sample_fraction` of each, at least one) for each compiled shape and
 * queue chunk, keeps the fastest and returns it.  Runs an opacity build
 * first if none exists.  Per-packet results do not depend on the choice. */
int sed_batch_autotune(sed_batch* b, double sample_fraction, sed_batch_tuning* best);
/* Uses the given shape instead (variant, blocks_per_sm, queue_chunk). */
int sed_batch_set_tuning(sed_batch* b, const sed_batch_tuning* t);
/* 1 (default): steps after the first are replays of captured CUDA graphs;
 * 0: every step is launched kernel by kernel. */
int sed_batch_use_graph(sed_batch* b, int32_t enable);

/* transport::step of every model: opacity build, emission, propagation,
 * spectrum and zone tallies, steady-state rescale and normalisation.
 * `total` sums the counters over the models. */
int sed_batch_step(sed_batch* b, double dt, sed_step_stats* total);

/* Replaces the density and gas temperature of one model's zones (what the
 * next step's opacity build reads; the reference's hydro and temperature
 * solve update grid->z[i].rho / T_gas between steps).  NULL skips an array. */
int sed_batch_set_zone_state(sed_batch* b, int32_t model, const double* rho, const double* T_gas);

/* Per-model results, laid out as the single-context getters lay them out. */
int sed_batch_get_escaped(sed_batch* b, int64_t* n_escaped /* [n_models] */);
int sed_batch_get_spectrum(sed_batch* b, int32_t model, double* flux, double* click);
int sed_batch_get_zone_tallies(sed_batch* b, int32_t model, double* J_nu, double* e_abs, double* e_rad,
                               double* fx, double* fy, double* fz, double* fr);
int sed_batch_get_opacity(sed_batch* b, int32_t model, double* abs, double* scat, double* emis_cdf,
                          double* n_elec, double* eps_imc);
int sed_batch_record_packets(sed_batch* b, int32_t enable);
/* Records of the model's first n packets; `ind` is the model's own zone index. */
int sed_batch_get_packet_records(sed_batch* b, int32_t model, int64_t n, int32_t* fate, int32_t* ind,
                                 int32_t* draws, double* state9);
const char* sed_batch_last_error(sed_batch* b);
void sed_batch_destroy(sed_batch* b);

/* LTE electron density of every zone (the Saha-Boltzmann / Brent solve that
 * sed_set_opacity runs first), for callers that cannot allocate device memory
 * when they need it -- e.g. a host code whose device memory is all handed out
 * by its own pool allocator, or a per-step loop that cannot afford the
 * synchronisation cudaMalloc/cudaFree bring.  No counterpart in the
 * reference: it has no GPU and no allocation constraints.
 *
 * Every pointer is a DEVICE pointer owned by the caller, including the arrays
 * inside *atoms_dev (only ion_off, ion_chi, lev_off, lev_ion, lev_g, lev_E are
 * read; the struct itself is in host memory).  rho, T_gas: [n_zones];
 * X: [n_zones * n_elems] mass fractions; elem_A: [n_elems]; outputs
 * n_elec: [n_zones] (cm^-3) and solve_err: [n_zones] (0 ok, 1 root not
 * bracketed, 2 iteration limit).  The work is queued on `stream`
 * (cudaStream_t, NULL = legacy default stream); the call returns without
 * waiting for it.
 *
 * The per-zone working set lives in a fixed 4 MiB array inside the library
 * (every GPU that loads the library holds it until exit).  The call returns
 * SED_ERR_CAPACITY when n_zones * (2 n_elems + 2 + 2 n_ions_total +
 * 2 n_levels_total) exceeds 524288.  All calls on a device share that array,
 * so calls whose work overlaps on the GPU (different streams, or other
 * threads) race; serialise them.  The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress); make that first call before
 * any stream capture. */
int sed_lte_electron_density_noalloc(int32_t n_zones, const double* rho, const double* T_gas,
                                     const double* X, int32_t n_elems, const int32_t* elem_A,
                                     const sed_atomic_data* atoms_dev, int32_t n_ions_total,
                                     int32_t n_levels_total, double temp_min, double temp_max,
                                     double* n_elec, int32_t* solve_err, void* stream);

#ifdef __cplusplus
}
#endif
#endif
