// sed_internal.h -- device-side argument blocks and kernel launchers shared
// between the C-ABI layer (sed_abi.cu) and the kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "sed_common.cuh"

namespace sed {

// Zone geometry on the device (1D sphere or 3D Cartesian).
struct GridDev {
  int32_t type;       // 0 = 1D sphere, 1 = 3D Cartesian
  int32_t nzones;
  int32_t homologous;
  int32_t nx, ny, nz;
  double t_grid;      // homologous velocity v = x / t_grid
  DevLoc r_out;       // 1D: zone right walls (flex), min = r_min
  const double* v_r;  // 1D non-homologous zone velocities
  DevLoc ax[3];       // 3D axes
};

struct BatchModel;

// counters[] slots written by the packet kernel
enum Counter { C_QUEUE = 0, C_ESCAPED, C_ABSORBED, C_STOPPED, C_SEGMENTS, C_SCATTERS, C_LIMIT, C_DDMC_CAP, C_IMD_CAP,
               C_COUNT };

struct StepArgs {
  int32_t steady, radiative_eq, bound_in_reflect, bound_out_reflect;
  int32_t store_Jnu, omit_scat, tally_forces, precision;  // precision: 0 fp64 tables, 1 fp32
  uint32_t seed, step;
  int64_t n_packets;
  int64_t first_pid;          // Philox stream id of queue entry 0
  double Ep, t_now, dt, tstop;
  double inv_t, ct, inv_ct, inv_ct2;  // 1/t_grid, c t_grid, 1/(c t_grid), its square (homologous flow)
  double core_radius, core_freq;
  const double* core_cdf;     // [n_nu] normalised core emission CDF
  int32_t max_segments;
  int32_t use_ddmc;           // 1: IMD, 2: DDMC in diffusive zones (1D)
  double ddmc_tau;            // transport_ddmc_tau_threshold
  const double* imd_p;        // IMD: [4][nz] hop up, hop down, stay, absorb probabilities of the step
  int32_t smem_zones;         // 1: per-block shared-memory zone tallies
  int32_t n_rep;              // >0 (and smem_zones 0): zone-scalar tallies in n_rep global copies
  double* zone_rep;           // [n_rep][5][nz] e_abs, fx, fy, fz, fr copies, summed by the finish kernel
  DevLoc nu, st, sn, sm, sp;  // frequency grid and spectrum grids
  int64_t a1, a2, a3;         // spectrum strides
  const void* opac;           // [nz*n_nu] double2 {abs, scat} or float2
  const void* cdf;            // [nz*n_nu] double or float emissivity CDF
  const void* cdf_coarse;     // [nz*n_coarse] every CDF_STRIDE-th CDF value (last of each block)
  int32_t n_coarse;           // blocks per zone row = ceil(n_nu / CDF_STRIDE)
  const uint16_t* cdf_guide;  // [nz*(guide_n+1)] guide[k] = upper_bound(CDF row, k / guide_n), or null
  int32_t guide_n;            // power of two >= n_nu (0: no guide table, n_nu > 65535)
  const double* eps_imc;      // [nz]
  int32_t rescale_lum;        // core_fix_luminosity (steady-state rescale)
  int32_t pad_;
  double* J;                  // [nz * (store_Jnu ? n_nu : 1)]
  double *e_abs, *e_rad, *fx, *fy, *fz, *fr;
  double *flux, *click;
  unsigned long long* counters;  // [C_COUNT]
  int32_t *rec_fate, *rec_ind, *rec_draws;  // optional per-packet records
  double* rec_state;
  int32_t* rec_type;                         // PType of the record (with the records of a time-dependent step)
  // ---- batch of independent 1D models (batched kernels only) ----
  const BatchModel* models;         // [n_models], ordered by pkt_off
  int32_t n_models;
  int32_t queue_chunk;               // packets a thread claims per queue pop
  const int4* zone_nbr;              // [zones] {inner neighbour or -1, outer or -2, no-inner flag, model}
  const double* zone_rin;            // [zones] inner wall after the core substitution
  // [zones] {outer wall, inner wall after the core substitution} with the
  // neighbours in the signs: the outer wall negative where the outer
  // neighbour is the model's edge (-2), the inner wall negative (-0.0 for a
  // wall at r = 0) where the inner neighbour is -1
  const double2* zone_wall;
  unsigned long long* model_escaped; // [n_models] escaped packets per model
  uint32_t* step_dev;                // step counter on the device (advanced by the finish kernel)
  // ---- queued packets: the census, then the radioactive packets (single-context kernels) ----
  int64_t n_core;                    // queue entries [0, n_core) are core packets, the rest queued packets
  int64_t radio_first_pid;           // Philox stream id of queued packet 0
  const double* q_state;             // [n_q * 9] {x, D, t, e, nu} of queued photons
  const int32_t* q_ind;              // [n_q] their zone (or -1 / -2)
  const uint32_t* q_n;               // [n_q] next deviate index; RADIO_NO_PHOTON: none
  double *L_dep, *L_emit;            // [nz] radioactive tallies normalised by the finish kernel, or null
  // ---- packets emitted ahead of the mixed-form 1D kernel (emit_mixed_kernel) ----
  double* em_state;                  // [9][n] {x, D, t, e, nu} of core packet q at em_state[k * n + q]
  int32_t* em_ind;                   // [n] its zone (or -1 / -2)
  float* em_tau;                     // [n] optical depth of its first flight
  int32_t* em_model;                 // [n] its model (batches)
  int64_t em_n;                      // core packets emitted there (the stride of em_state)
  // ---- differentiable transport (weighted forward and adjoint replay kernels only) ----
  const double* abs_scale;           // [nz * n_bands] factor on the absorption opacity, or null
  int32_t n_bands;                   // band of bin i = i * n_bands / n_nu
  int32_t adj_jacobian;              // adjoint: 1 = full Jacobian rows, 0 = vector-Jacobian product
  int32_t adj_density;               // adjoint: 1 = d / d ln rho per zone (likelihood-ratio score + absorption)
  int32_t* esc_bin;                  // [n_packets] spectrum index of an escaped, counted packet; -1 otherwise
  double* esc_e;                     // [n_packets] its energy at escape
  const double* adj_g;               // [nspec] d(loss)/d(flux) for the vector-Jacobian product
  double* adj_out;                   // VJP [nz * n_bands]; Jacobian [nspec * nz * n_bands]
};

constexpr uint32_t RADIO_NO_PHOTON = 0xFFFFFFFFu;
// particle types (enum PType, src/transport/particle.h:8)
constexpr int32_t TYPE_PHOTON = 0, TYPE_GAMMA = 1;
// Philox step number of the deviates transport::initialize_particles draws
constexpr uint32_t INIT_STEP = 0xFFFFFFFFu;

// Radioactive gamma-ray source (transport::emit_radioactive, src/transport/
// emission.cpp:163-243) and gamma-ray transport (Compton scattering and
// photo-absorption, scatter.cpp:45-133, transport_opacity.cpp:290-313).
struct RadioArgs {
  int32_t nz, n_elems, force_rproc, pad_;
  int64_t n_census;                // queued packets [0, n_census) come from the census
  int64_t n_radio;                 // radioactive packets of the step: queued packets [n_census, n_census + n_radio)
  int64_t first_pid;               // Philox stream id of queued packet 0
  const int32_t* q_type;           // [n_census] census packet types
  double t_now, dt;
  const double *rho, *vol, *X;     // zone state; X the zone's composition (not decayed)
  const int32_t *eZ, *eA;
  double *L_emit, *gamma_frac, *compton, *photoion;  // [nz] per-zone results
  double* cdf;                     // [nz] zone emission CDF
  double* L_tot;                   // device scalar: decay luminosity of the grid
  double* L_dep;                   // [nz] deposition tally
  double* q_state;                 // [n_q * 9] {x, D, t, e, nu} of queued optical photons
  int32_t* q_ind;                  // [n_q] their zone
  uint32_t* q_n;                   // [n_q] their next deviate index, RADIO_NO_PHOTON if none
  int32_t* n_reject_cap;           // Compton rejection loops that hit their cap
};
// per-zone decay luminosity, gamma fraction and gamma opacities, then the
// zone emission CDF and the grid total (two launches)
int launch_radio_zones(const RadioArgs& a, cudaStream_t s);
// emission of the radioactive packets and transport of the gamma-rays; the
// optical photons they become are queued for the packet kernel
int launch_gamma(const StepArgs& a, const StepArgs& ag, const RadioArgs& r, const GridDev& g, int num_sms,
                 cudaStream_t s);

// Packets carried between time-dependent steps: transport::step leaves
// the stopped packets in its particle vector (transport.cpp:91, 164-194).
struct CensusArgs {
  int64_t n_census;                // census packets loaded at the start of the step
  int64_t n_core, n_q;             // record slots: [0, n_core) core packets, then the n_q queued packets
  double* census_state;            // [n * 9] {x, D, t, e, nu}: read at the start, rewritten at the end
  int32_t *census_ind, *census_type;
  double* q_state;                 // queue of the step
  int32_t *q_ind, *q_type;
  uint32_t* q_n;
  const int32_t *rec_fate, *rec_ind, *rec_type;  // end states of the step's packets
  const double* rec_state;
  int32_t *flag_e, *flag_a;        // [n + 1] packet exists / is stopped, in the reference's vector order
  int32_t *scan_e, *scan_a;        // their exclusive sums
  int32_t* front_dead;             // [n]
  unsigned long long* n_gamma;     // gamma-rays in the new census
};
// loads the census into the front of the step's queue (2 launches at most)
int launch_census_load(const CensusArgs& a, const GridDev& g, cudaStream_t s);
// existence / stopped flags of the step's packets in vector order
int launch_census_flags(const CensusArgs& a, int64_t n, cudaStream_t s);
// the reference's swap-from-the-back compaction (clean_up_particle_vector)
// of the stopped packets into the census, from the flags' exclusive sums
int launch_census_compact(const CensusArgs& a, int64_t n, cudaStream_t s);

// transport::initialize_particles (src/transport/emission.cpp:112-159):
// photons emitted in proportion to e_rad * vol with a blackbody spectrum at
// the gas temperature, appended to the census
struct InitArgs {
  int64_t n, census_off;           // packets; first census slot
  uint32_t seed;
  int64_t first_pid;
  double t_now;
  int32_t nz;
  const double *e_rad, *vol, *T;   // [nz]
  double* zone_cdf;                // [nz] scratch
  double* E_sum;                   // device scalar
  double* bb_cdf;                  // [nz * n_nu] scratch: blackbody emissivity CDF per zone
  DevLoc nu;
  double* census_state;
  int32_t *census_ind, *census_type;
};
int launch_init_particles(const InitArgs& a, const GridDev& g, cudaStream_t s);

// One model of a batch: its packets are global queue entries
// [pkt_off, pkt_off + n_packets), its zones [zone_off, zone_off + n_zones)
// of the concatenated zone arrays, its spectrum at flux + spec_off.
struct BatchModel {
  int64_t pkt_off, n_packets, first_pid, spec_off;
  int32_t zone_off, n_zones;
  uint32_t seed, emit_draws;         // Philox key; deviates drawn by the emission
  double r_min, core_radius, Ep;
  const double* core_cdf;            // [n_nu] normalised core emission CDF
};

// launches the persistent packet kernel; returns the number of launches
int launch_propagate(const StepArgs& a, const GridDev& g, int num_sms, cudaStream_t s);
// whether launch_propagate runs the mixed-form 1D kernel for these
// arguments: its core packets are then emitted ahead into the em_* buffers
// (A.em_n of them), which the caller provides
bool mixed_1d_path(const StepArgs& a, const GridDev& g);
// IMD probabilities of the step (transport::compute_diffusion_probabilities)
// from the zone Planck means into out[4][nz]
int launch_imd_probabilities(const GridDev& g, const double* planck, double dt, double* out, cudaStream_t s);
// zone-scalar tally normalisation (reduce_radiation) and steady-state rescale
int launch_finish(const StepArgs& a, const GridDev& g, const double* vol, int64_t nspec, cudaStream_t s);

// Differentiable transport on a 1D grid: mode 1 = forward with absorption as
// a continuous weight (interactions sampled from scattering only), mode 2 =
// adjoint replay of the escaped packets of the last mode-1 launch.
int launch_propagate_diff(const StepArgs& a, const GridDev& g, int mode, int num_sms, cudaStream_t s);

// Batched packet kernel: compiled shapes {threads per block, min blocks per
// SM} selectable at run time (the autotuner times each).  `blocks_per_sm`
// 0 = as many as fit.
constexpr int BATCH_VARIANTS = 4;
void batch_variant_shape(int variant, int* threads, int* min_blocks);
int launch_propagate_batch(const StepArgs& a, const GridDev& g, int variant, int blocks_per_sm, int num_sms,
                           int64_t total_packets, cudaStream_t s);
// per-model steady-state rescale of the spectra, per-zone normalisation with
// the zone's model factor, then the device step counter advances
int launch_finish_batch(const StepArgs& a, const double* vol, int nz_total, int64_t nspec, cudaStream_t s);

// ---------------------------------------------------------------- temperature
struct TemperatureArgs {
  int32_t nz, precision, set_Tgas_to_Trad, pad_;
  DevLoc nu;
  const void* opac;            // {abs, scat} pairs, double2 or float2 [nz * n_nu]
  const double *e_abs, *e_rad; // normalised zone tallies of the last step
  double temp_min, temp_max;   // limits_temp_min / limits_temp_max
  double* T;                   // [nz] zone temperature, replaced
  int32_t* n_unsolved;         // zones where Brent hit its iteration limit
};
// radiative-equilibrium temperature of every zone (one thread per zone)
int launch_temperature(const TemperatureArgs& a, cudaStream_t s);

// ---------------------------------------------------------------- opacity
struct OpacityArgs {
  int32_t nzones, n_nu, nelem;
  int32_t seq_cdf;   // FP64 emissivity CDF summed in the reference's order (grids up to 65536 zones)
  int32_t use_es, use_ff, use_bf, use_line, use_fuzz;
  int32_t radiative_eq, omit_scat, precision;
  double epsilon, max_opacity, temp_min, temp_max, fleck_alpha, dt, time;
  DevLoc nu;
  const double *rho, *T, *e_gas, *grey, *X;  // zone state
  const int32_t *eZ, *eA;
  const int32_t* zero_eps_atom;  // [nelem] 1 when the atom's epsilon is 0
  // atomic data (device)
  int32_t natoms;
  const int32_t *ion_off, *lev_off, *lev_ion, *lev_g, *lev_ic, *photo_off;
  const double *ion_chi, *lev_E, *lev_Eion, *photo_E, *photo_s;
  const int32_t* ion_atom;      // [n_ions_total] atom of each ion
  const int32_t* lev_atom;      // [n_lev_total] atom of each level
  const int32_t* ln_order;      // [n_nu] bins by decreasing level-line count
  const int32_t* fz_order;      // [n_nu] bins by decreasing fuzz-line count
  // level-to-level lines sorted by (bin, atom): bin j holds [ln_seg[j], ln_seg[j+1])
  const int32_t* ln_seg;       // [n_nu + 1]
  const int4* ln_lv;           // {lower level, upper level (absolute indices), bin, atom}
  const double2* ln_c;         // {sigma_tot f lambda, g_l / g_u}
  const float2* ln_c32;        // FP32 copy of ln_c
  // fuzz lines sorted by (bin, atom)
  const int32_t* fz_seg;       // [n_nu + 1]
  const int4* fz_ia;           // {absolute ion index, bin, atom, 0}
  const double2* fz_c;         // {sigma_tot lambda gf, E_l / k_ev}
  const double* fz_h;          // h nu / k
  const float4* fz_c32;        // FP32 {sigma_tot lambda gf, E_l / k_ev, h nu / k, 0}
  int32_t uniform_eps;         // every atom has epsilon = A.epsilon
  int32_t smem_rows;           // FP64 rows of the zone in shared memory
  // per-zone LTE state (device scratch written by the LTE kernel)
  double *ion_part, *ion_frac, *lev_n;  // [nzones * n_ions_total] etc.
  int32_t n_ions_total, n_lev_total;
  double* n_elec;                        // [nz]
  double* n_dens;                        // [nz * natoms]
  double* mass_frac;                     // [nz * natoms]
  double* temp_c;                        // [nz] clamped temperature
  int32_t* solve_err;                    // [nz]
  double* boltz;                         // [n_lev_total * nz] exp(-E/kT) per level
  // outputs
  double *abs64, *scat64, *emis64;       // [nz*n_nu] FP64 rows when they do not fit in shared memory
  double *epsl64, *epsf64;               // [nz*n_nu] epsilon-weighted line / fuzz sums (same condition)
  void* opac_out;                        // double2 / float2 [nz*n_nu]
  void* cdf_out;                         // double / float [nz*n_nu]
  void* cdf_coarse_out;                  // double / float [nz*n_coarse]
  int32_t n_coarse;
  uint16_t* cdf_guide_out;               // [nz*(guide_n+1)] or null
  int32_t guide_n;
  double *eps_imc, *planck, *ross, *L_th;
};

// dynamic shared memory of the per-zone opacity kernel for these arguments
size_t opacity_smem_bytes(const OpacityArgs& a);
// dynamic shared memory of the line-sum kernel (n_pop levels or ions per zone)
size_t line_sum_smem_bytes(int precision, int natoms, int n_pop);
int launch_opacity(const OpacityArgs& a, int num_sms, cudaStream_t s);

}  // namespace sed
