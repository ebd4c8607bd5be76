// transport_gpu.cpp -- see transport_gpu.h.
//
// Compiled against the reference's headers (src/transport, src/opacity,
// src/grid, src/utils, src/main); the members it reads are private there,
// hence the opened access below.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#define private public
#define protected public
#include "transport.h"
#include "grid_1D_sphere.h"
#include "grid_3D_cart.h"
#include "ParameterReader.h"  // (AtomicData.h comes with transport.h; its include guard does not guard it twice)
#undef private
#undef protected

#include "transport_gpu.h"

namespace sed_binding {

struct GpuTransport {
  sed_ctx* ctx = nullptr;
  std::vector<double> walls[9];  // nu, spectrum t/nu/mu/phi, gamma nu, 3D axes
  std::string err;
};

namespace {

std::string g_err;

// locate_array -> sed_locate_grid (the LAType order flex, do_lin, do_log,
// none is sed_locate_type's)
sed_locate_grid flat(const locate_array& a, std::vector<double>& w)
{
  w.assign(a.x_.begin(), a.x_.end());
  sed_locate_grid g{};
  g.n = a.size();
  g.type = (int32_t)a.locate_type_;
  g.min = a.min_;
  g.del = a.del_;
  g.right = w.data();
  return g;
}

int fail(GpuTransport* g, int rc, const char* what)
{
  std::string m = std::string(what) + ": " + (g && g->ctx ? sed_last_error(g->ctx) : "");
  if (g) g->err = m;
  g_err = m;
  return rc;
}

// zone state of the grid, flattened (grid_general::z, the 1D walls or 3D axes)
struct GridArrays {
  std::vector<double> r_out, v_r, vol, rho, T, e_gas, grey, X;
  std::vector<int32_t> Z, A;
};

sed_grid fill_grid(transport& t, GpuTransport* b, GridArrays& a)
{
  grid_general* gr = t.grid;
  const int nz = gr->n_zones, ne = gr->n_elems;
  sed_grid g{};
  g.n_zones = nz;
  g.homologous = gr->use_homologous_velocities_;
  g.n_elems = ne;
  g.t_now = gr->t_now;
  a.vol.resize(nz); a.rho.resize(nz); a.T.resize(nz); a.e_gas.resize(nz); a.grey.resize(nz);
  a.X.resize((size_t)nz * ne); a.v_r.resize(nz);
  for (int i = 0; i < nz; ++i) {
    const zone& z = gr->z[i];
    a.vol[i] = gr->zone_volume(i);
    a.rho[i] = z.rho;
    a.T[i] = z.T_gas;
    a.e_gas[i] = z.e_gas;
    a.grey[i] = z.total_grey_opacity;
    a.v_r[i] = z.v[0];
    for (int k = 0; k < ne; ++k) a.X[(size_t)i * ne + k] = z.X_gas[k];
  }
  a.Z.assign(gr->elems_Z.begin(), gr->elems_Z.end());
  a.A.assign(gr->elems_A.begin(), gr->elems_A.end());
  if (grid_1D_sphere* s = dynamic_cast<grid_1D_sphere*>(gr)) {
    g.type = SED_GRID_1D_SPHERE;
    a.r_out.assign(s->r_out.x_.begin(), s->r_out.x_.end());
    g.r_min = s->r_out.min_;
    g.r_out = a.r_out.data();
    g.v_r = a.v_r.data();
  } else if (grid_3D_cart* c = dynamic_cast<grid_3D_cart*>(gr)) {
    g.type = SED_GRID_3D_CART;
    g.nx = c->nx_; g.ny = c->ny_; g.nz = c->nz_;
    g.x_axis = flat(c->x_out_, b->walls[6]);
    g.y_axis = flat(c->y_out_, b->walls[7]);
    g.z_axis = flat(c->z_out_, b->walls[8]);
  } else {
    g.type = -1;
  }
  g.vol = a.vol.data(); g.rho = a.rho.data(); g.T_gas = a.T.data(); g.e_gas = a.e_gas.data();
  g.total_grey_opacity = a.grey.data(); g.X = a.X.data();
  g.elem_Z = a.Z.data(); g.elem_A = a.A.data();
  return g;
}

// the atomic data the transport loaded (IndividualAtomData per element, after
// the loader's own post-processing), in the grid's element order; false when
// an element has none (grey opacities)
struct AtomArrays {
  std::vector<int32_t> ion_off{0}, lev_off{0}, line_off{0}, fuzz_off{0}, photo_off{0};
  std::vector<double> ion_chi, lev_E, lev_Eion, photo_E, photo_s, line_nu, line_f, fuzz_nu, fuzz_gf, fuzz_El;
  std::vector<int32_t> lev_ion, lev_g, lev_ic, line_l, line_u, fuzz_ion;
};

bool fill_atoms(transport& t, AtomArrays& a, sed_atomic_data& s)
{
  if (!t.atomic_data_) return false;
  for (int Z : t.grid->elems_Z) {
    IndividualAtomData* d = t.atomic_data_->get_pointer_to_individual_atom(Z);
    if (!d || !d->data_exists_) return false;
    for (int i = 0; i < d->n_ions_; ++i) a.ion_chi.push_back(d->ions_[i].chi);
    for (int l = 0; l < d->n_levels_; ++l) {
      const AtomicLevel& L = d->levels_[l];
      a.lev_ion.push_back(L.ion); a.lev_g.push_back(L.g); a.lev_ic.push_back(L.ic);
      a.lev_E.push_back(L.E); a.lev_Eion.push_back(L.E_ion);
      a.photo_E.insert(a.photo_E.end(), L.s_photo.x.begin(), L.s_photo.x.end());
      a.photo_s.insert(a.photo_s.end(), L.s_photo.y.begin(), L.s_photo.y.end());
      a.photo_off.push_back((int32_t)a.photo_E.size());
    }
    for (int k = 0; k < d->n_lines_; ++k) {
      const AtomicLine& L = d->lines_[k];
      a.line_l.push_back(L.ll); a.line_u.push_back(L.lu); a.line_nu.push_back(L.nu); a.line_f.push_back(L.f_lu);
    }
    const fuzz_line_structure& f = d->fuzz_lines_;
    for (int k = 0; k < f.n_lines; ++k) {
      a.fuzz_nu.push_back(f.nu[k]); a.fuzz_gf.push_back(f.gf[k]);
      a.fuzz_El.push_back(f.El[k]); a.fuzz_ion.push_back(f.ion[k]);
    }
    a.ion_off.push_back((int32_t)a.ion_chi.size());
    a.lev_off.push_back((int32_t)a.lev_ion.size());
    a.line_off.push_back((int32_t)a.line_l.size());
    a.fuzz_off.push_back((int32_t)a.fuzz_nu.size());
  }
  s = sed_atomic_data{};
  s.n_atoms = (int32_t)t.grid->elems_Z.size();
  s.ion_off = a.ion_off.data(); s.ion_chi = a.ion_chi.data();
  s.lev_off = a.lev_off.data(); s.lev_ion = a.lev_ion.data(); s.lev_g = a.lev_g.data(); s.lev_ic = a.lev_ic.data();
  s.lev_E = a.lev_E.data(); s.lev_Eion = a.lev_Eion.data();
  s.photo_off = a.photo_off.data(); s.photo_E = a.photo_E.data(); s.photo_s = a.photo_s.data();
  s.line_off = a.line_off.data(); s.line_l = a.line_l.data(); s.line_u = a.line_u.data();
  s.line_nu = a.line_nu.data(); s.line_f = a.line_f.data();
  s.fuzz_off = a.fuzz_off.data(); s.fuzz_nu = a.fuzz_nu.data(); s.fuzz_gf = a.fuzz_gf.data();
  s.fuzz_El = a.fuzz_El.data(); s.fuzz_ion = a.fuzz_ion.data();
  return true;
}

}  // namespace

GpuTransport* attach(transport& t, ParameterReader* params, int precision, int device)
{
  GpuTransport* b = new GpuTransport;
  sed_transport_params p{};
  p.steady_state = t.steady_state;
  p.radiative_eq = t.radiative_eq;
  p.boundary_in_reflect = t.boundary_in_reflect_;
  p.boundary_out_reflect = t.boundary_out_reflect_;
  p.store_Jnu = t.store_Jnu_;
  p.omit_scattering = t.omit_scattering_;
  p.core_fix_luminosity = t.core_fix_luminosity_;
  p.tally_forces = 1;
  p.precision = precision;
  p.rng_seed = (uint32_t)params->getScalar<int>("transport_rng_seed");
  p.max_particles = t.max_total_particles;
  p.core_n_emit = params->getScalar<int>("core_n_emit");
  p.core_radius = t.r_core_;
  p.core_luminosity = t.L_core_;
  p.core_temperature = t.T_core_;
  p.core_photon_frequency = t.core_frequency_;
  p.fleck_alpha = t.fleck_alpha_;
  p.first_packet_id = (int64_t)t.MPI_myID * p.core_n_emit;  // ranks draw disjoint packets
  p.nu_grid = flat(t.nu_grid_, b->walls[0]);
  p.spec_time = flat(t.optical_spectrum.time_grid, b->walls[1]);
  p.spec_nu = flat(t.optical_spectrum.wave_grid, b->walls[2]);
  p.spec_mu = flat(t.optical_spectrum.mu_grid, b->walls[3]);
  p.spec_phi = flat(t.optical_spectrum.phi_grid, b->walls[4]);
  p.n_emit_radioactive = params->getScalar<int>("particles_n_emit_radioactive");
  p.force_rprocess_heating = params->getScalar<int>("force_rprocess_heating");
  p.gamma_nu = flat(t.gamma_spectrum.wave_grid, b->walls[5]);
  p.use_ddmc = t.use_ddmc_;
  p.ddmc_tau = t.ddmc_tau_;
  if (sed_ctx_create(&p, device, &b->ctx)) {
    fail(b, SED_ERR_ARG, "sed_ctx_create");
    detach(b);
    return nullptr;
  }
  // an inner source read from core_spectrum_file: its per-bin weights are
  // the steps of the CDF setup_core_emission built (transport_init.cpp:495-537)
  if (params->getScalar<std::string>("core_spectrum_file") != "") {
    const int nn = t.nu_grid_.size();
    std::vector<double> w(nn);
    for (int j = 0; j < nn; ++j) w[j] = t.core_emission_spectrum_.get(j) - (j ? t.core_emission_spectrum_.get(j - 1) : 0.0);
    if (sed_set_core_source(b->ctx, t.L_core_, w.data())) { fail(b, SED_ERR_ARG, "sed_set_core_source"); }
  }
  GridArrays ga;
  sed_grid g = fill_grid(t, b, ga);
  if (sed_set_grid(b->ctx, &g)) { fail(b, SED_ERR_ARG, "sed_set_grid"); detach(b); return nullptr; }
  sed_opacity_params op{};
  op.use_electron_scattering = params->getScalar<int>("opacity_electron_scattering");
  op.use_free_free = params->getScalar<int>("opacity_free_free");
  op.use_bound_free = params->getScalar<int>("opacity_bound_free");
  op.use_line_expansion = params->getScalar<int>("opacity_line_expansion");
  op.use_fuzz_expansion = params->getScalar<int>("opacity_fuzz_expansion");
  std::vector<int> ze = params->getVector<int>("opacity_atom_zero_epsilon");
  std::vector<int32_t> ze32(ze.begin(), ze.end());
  op.n_atom_zero_epsilon = (int32_t)ze32.size();
  op.atom_zero_epsilon = ze32.empty() ? nullptr : ze32.data();
  op.epsilon = params->getScalar<double>("opacity_epsilon");
  op.maximum_opacity = params->getScalar<double>("opacity_maximum_opacity");
  op.temp_min = params->getScalar<double>("limits_temp_min");
  op.temp_max = params->getScalar<double>("limits_temp_max");
  op.line_velocity_width = params->getScalar<double>("line_velocity_width");
  if (sed_set_opacity_params(b->ctx, &op)) { fail(b, SED_ERR_ARG, "sed_set_opacity_params"); detach(b); return nullptr; }
  AtomArrays aa;
  sed_atomic_data ad;
  if (fill_atoms(t, aa, ad) && sed_set_atomic_data(b->ctx, &ad)) {
    fail(b, SED_ERR_ARG, "sed_set_atomic_data");
    detach(b);
    return nullptr;
  }
  return b;
}

int step(transport& t, GpuTransport* b, double dt, sed_step_stats* stats)
{
  if (!b || !b->ctx) return SED_ERR_STATE;
  ParameterReader* params = t.params_;
  if (t.steady_state) dt = 1;
  // zone state of this step (the hydro step may have moved it)
  GridArrays ga;
  sed_grid g = fill_grid(t, b, ga);
  int rc = sed_set_grid(b->ctx, &g);
  if (rc) return fail(b, rc, "sed_set_grid");
  // emit_inner_source's luminosity at the transport clock (emission.cpp:386-389)
  // and the emission count rules (emission.cpp:170-184, 377-382)
  const double L_current = params->getFunction("core_luminosity", t.t_now_);
  if (L_current != 0) t.L_core_ = L_current;
  rc = sed_set_core_source(b->ctx, t.L_core_, nullptr);
  if (rc) return fail(b, rc, "sed_set_core_source");
  double n_core = params->getScalar<int>("core_n_emit");
  double n_radio = params->getScalar<int>("particles_n_emit_radioactive");
  if (params->getScalar<int>("multiply_particles_n_emit_by_dt_over_dtmax"))
    n_radio = (int)(n_radio * (dt / params->getScalar<double>("tstep_max_dt")));
  if (t.last_iteration_) {
    const int pump = params->getScalar<int>("particles_last_iter_pump");
    if (pump != 0) { n_radio *= pump; n_core *= pump; }
  }
  rc = sed_set_emission(b->ctx, n_core, (int64_t)n_radio);
  if (rc) return fail(b, rc, "sed_set_emission");
  sed_step_stats st{};
  rc = sed_step(b->ctx, dt, &st);
  if (stats) *stats = st;
  if (rc) return fail(b, rc, "sed_step");
  if (st.warnings & SED_WARN_NO_PARTICLE_SPACE) std::fprintf(stderr, "# Not enough particle space\n");

  // results back into the transport's own containers
  grid_general* gr = t.grid;
  const int nz = gr->n_zones, nn = t.nu_grid_.size();
  const int nj = t.store_Jnu_ ? nn : 1;
  std::vector<double> J((size_t)nz * nj), e_abs(nz), e_rad(nz), fx(nz), fy(nz), fz(nz), fr(nz);
  rc = sed_get_zone_tallies(b->ctx, J.data(), e_abs.data(), e_rad.data(), fx.data(), fy.data(), fz.data(), fr.data());
  if (rc) return fail(b, rc, "sed_get_zone_tallies");
  std::vector<double> ab((size_t)nz * nn), sc((size_t)nz * nn), cdf((size_t)nz * nn), ne(nz), eps(nz), pm(nz),
      rm(nz), lt(nz);
  rc = sed_get_opacity(b->ctx, ab.data(), sc.data(), cdf.data(), ne.data(), eps.data(), pm.data(), rm.data(),
                       lt.data());
  if (rc) return fail(b, rc, "sed_get_opacity");
  for (int i = 0; i < nz; ++i) {
    zone& z = gr->z[i];
    z.e_abs = e_abs[i]; z.e_rad = e_rad[i];
    z.fx_rad = fx[i]; z.fy_rad = fy[i]; z.fz_rad = fz[i]; z.fr_rad = fr[i];
    z.n_elec = ne[i]; z.eps_imc = eps[i]; z.L_thermal = lt[i];
    t.planck_mean_opacity_[i] = pm[i];
    t.rosseland_mean_opacity_[i] = rm[i];
    for (int j = 0; j < nj && j < (int)t.J_nu_[i].size(); ++j) t.J_nu_[i][j] = J[(size_t)i * nj + j];
    for (int j = 0; j < nn; ++j) {
      t.abs_opacity_[i][j] = ab[(size_t)i * nn + j];
      if (!t.omit_scattering_) t.scat_opacity_[i][j] = sc[(size_t)i * nn + j];
      t.emissivity_[i].set(j, cdf[(size_t)i * nn + j]);
    }
  }
  rc = sed_get_spectrum(b->ctx, t.optical_spectrum.flux.data(), t.optical_spectrum.click.data());
  if (rc) return fail(b, rc, "sed_get_spectrum");
  if (n_radio > 0) {
    std::vector<double> Le(nz), Ld(nz);
    rc = sed_get_radioactive_tallies(b->ctx, Le.data(), Ld.data());
    if (rc) return fail(b, rc, "sed_get_radioactive_tallies");
    for (int i = 0; i < nz; ++i) { gr->z[i].L_radio_emit = Le[i]; gr->z[i].L_radio_dep = Ld[i]; }
    rc = sed_get_gamma_spectrum(b->ctx, t.gamma_spectrum.flux.data(), t.gamma_spectrum.click.data());
    if (rc) return fail(b, rc, "sed_get_gamma_spectrum");
  }
  // solve_eq_temperature on the device, as transport::step calls it
  // (transport.cpp:125-131)
  if (t.radiative_eq == 1 && t.fix_Tgas_during_transport_ == 0 && t.solve_Tgas_with_updated_opacities_ == 0) {
    std::vector<double> T(nz);
    int32_t unsolved = 0;
    rc = sed_solve_temperature(b->ctx, t.set_Tgas_to_Trad_, T.data(), &unsolved);
    if (rc) return fail(b, rc, "sed_solve_temperature");
    for (int i = 0; i < nz; ++i) gr->z[i].T_gas = T[i];
  }
  if (!t.steady_state) t.t_now_ += dt;
  return SED_OK;
}

const char* last_error(GpuTransport* g) { return g ? g->err.c_str() : g_err.c_str(); }

void detach(GpuTransport* g)
{
  if (!g) return;
  if (g->ctx) sed_ctx_destroy(g->ctx);
  delete g;
}

}  // namespace sed_binding
