// sed_abi.cu -- host side of the C ABI declared in include/sedona_gpu.h.
//
// A sed_ctx owns one CUDA stream and every device buffer of the transport
// step: zone state, atomic data, opacity tables, tallies.  Host-side work is
// limited to set-up (copies, the core emission CDF, sorting line lists by
// frequency bin); a transport step is a short sequence of kernel launches on
// the context's stream followed by one synchronisation.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include <cub/cub.cuh>
#include "sed_ctx.h"

using namespace sed;

namespace {

int alloc_tallies(sed_ctx* c)
{
  const size_t nz = (size_t)c->nz, nn = (size_t)c->nu.n();
  const size_t nj = c->tp.store_Jnu ? nn : 1;
  CK(c->d_J.resize(nz * nj));
  CK(c->d_e_abs.resize(nz)); CK(c->d_e_rad.resize(nz));
  CK(c->d_fx.resize(nz)); CK(c->d_fy.resize(nz)); CK(c->d_fz.resize(nz)); CK(c->d_fr.resize(nz));
  const size_t esz = c->tp.precision ? sizeof(float) : sizeof(double);
  CK(c->d_opac.resize(nz * nn * 2 * esz));
  CK(c->d_cdf.resize(nz * nn * esz));
  c->n_coarse = (int)((nn + CDF_STRIDE - 1) / CDF_STRIDE);
  CK(c->d_cdf_coarse.resize(nz * (size_t)c->n_coarse * esz));
  // guide tables: G = the power of two >= n_nu (uint16 bin indices)
  c->guide_n = 0;
  if (nn > 1 && nn <= 65535) {
    c->guide_n = 1;
    while ((size_t)c->guide_n < nn) c->guide_n <<= 1;
    CK(c->d_cdf_guide.resize(nz * (size_t)(c->guide_n + 1)));
  }
  CK(c->d_eps_imc.resize(nz)); CK(c->d_planck.resize(nz)); CK(c->d_ross.resize(nz)); CK(c->d_L.resize(nz));
  CK(c->d_n_elec.resize(nz)); CK(c->d_temp_c.resize(nz)); CK(c->d_solve_err.resize(nz));
  CK(cudaMemsetAsync(c->d_n_elec.p, 0, nz * sizeof(double), c->stream));
  return SED_OK;
}

// Scratch of the opacity build, sized for one pass over `chunk_zones` zones:
// FP64 abs/scat/emissivity rows and the LTE state (mass fractions, number
// densities, partition functions, ion fractions, level populations and
// Boltzmann factors).  Passes of at most OPACITY_SCRATCH_BYTES keep this
// bounded whatever the grid size, so the resident memory of a step is the
// packed transport tables plus the tallies.  The environment variable
// SEDONA_GPU_OPACITY_SCRATCH_BYTES lowers or raises the bound.
constexpr size_t OPACITY_SCRATCH_BYTES = size_t(8) << 30;

size_t opacity_scratch_bytes()
{
  const char* e = std::getenv("SEDONA_GPU_OPACITY_SCRATCH_BYTES");
  if (e && *e) {
    const unsigned long long v = std::strtoull(e, nullptr, 10);
    if (v > 0) return (size_t)v;
  }
  return OPACITY_SCRATCH_BYTES;
}

// Shared memory per CTA: the per-zone opacity kernel keeps its three FP64
// rows (abs, scat, emissivity) there when they take at most SMEM_ZONE_BYTES,
// else in the chunk scratch; the line-sum kernel stages the populations of a
// tile of zones and must fit in SMEM_ZONE_BYTES.
constexpr size_t SMEM_ZONE_BYTES = 200 * 1024;

bool rows_in_smem(size_t na, size_t nn) { return (na + 3 * nn) * sizeof(double) <= SMEM_ZONE_BYTES; }

// Chunk scratch: per zone the line and fuzz Sobolev sums (overwritten by the
// abs and scat rows), the emissivity row when the rows are not in shared
// memory, two epsilon-weighted sums when atoms differ in epsilon, and the LTE
// state.
int alloc_lte(sed_ctx* c)
{
  const size_t nz = (size_t)c->nz, nn = (size_t)c->nu.n();
  const size_t na = (size_t)std::max(c->nelem, 1);
  const size_t ni = (size_t)std::max(c->n_ions_total, 1), nl = (size_t)std::max(c->n_lev_total, 1);
  const bool smem_rows = rows_in_smem(na, nn);
  const size_t rows = (smem_rows ? 2 : 3) * nn + (c->any_zero_eps ? 2 * nn : 0);
  const size_t per_zone = (rows + 2 * na + 2 * ni + 2 * nl) * sizeof(double);
  const size_t cz = std::max<size_t>(1, std::min(nz, opacity_scratch_bytes() / per_zone));
  c->chunk_zones = (int)cz;
  CK(c->d_abs64.resize(cz * nn)); CK(c->d_scat64.resize(cz * nn));
  CK(c->d_emis64.resize(smem_rows ? 1 : cz * nn));
  CK(c->d_epsl64.resize(c->any_zero_eps ? cz * nn : 1)); CK(c->d_epsf64.resize(c->any_zero_eps ? cz * nn : 1));
  CK(c->d_n_dens.resize(cz * na));
  CK(c->d_mass_frac.resize(cz * na));
  CK(c->d_ion_part.resize(cz * ni));
  CK(c->d_ion_frac.resize(cz * ni));
  CK(c->d_lev_n.resize(cz * nl));
  CK(c->d_boltz.resize(cz * nl));
  return SED_OK;
}

}  // namespace


// Kernel arguments of a transport step of this context (transport.cpp:46-124):
// switches, packet count and energy (emission.cpp:383-392), grids, tables
// and tallies; per-packet records are left off.
StepArgs sed::make_step_args(sed_ctx* c, double dt, int64_t n_emit)
{
  const size_t nz = (size_t)c->nz;
  StepArgs A{};
  A.steady = c->tp.steady_state; A.radiative_eq = c->tp.radiative_eq;
  A.bound_in_reflect = c->tp.boundary_in_reflect; A.bound_out_reflect = c->tp.boundary_out_reflect;
  A.store_Jnu = c->tp.store_Jnu; A.omit_scat = c->tp.omit_scattering; A.tally_forces = c->tp.tally_forces;
  A.precision = c->tp.precision; A.seed = c->tp.rng_seed; A.step = c->step;
  A.n_packets = n_emit;
  A.first_pid = c->tp.first_packet_id;
  A.Ep = n_emit > 0 ? c->tp.core_luminosity * dt / n_emit : 0.0;
  A.t_now = c->t_now; A.dt = dt; A.tstop = c->t_now + dt;
  if (c->t_grid > 0) {
    A.inv_t = 1.0 / c->t_grid;
    A.ct = C_LIGHT * c->t_grid;
    A.inv_ct = 1.0 / A.ct;
    A.inv_ct2 = A.inv_ct * A.inv_ct;
  }
  A.core_radius = c->tp.core_radius; A.core_freq = c->tp.core_photon_frequency; A.core_cdf = c->d_core_cdf.p;
  A.max_segments = c->tp.max_segments;
  A.use_ddmc = c->tp.use_ddmc; A.ddmc_tau = c->tp.ddmc_tau;
  const size_t zone_smem = (size_t)5 * nz * sizeof(double);
  A.smem_zones = (zone_smem <= 64 * 1024) ? 1 : 0;
  A.nu = dev_loc(c->nu, c->d_nu); A.st = dev_loc(c->st, c->d_st); A.sn = dev_loc(c->sn, c->d_sn);
  A.sm = dev_loc(c->sm, c->d_sm); A.sp = dev_loc(c->sp, c->d_sp);
  A.a3 = c->sp.n(); A.a2 = (int64_t)c->sm.n() * A.a3; A.a1 = (int64_t)c->sn.n() * A.a2;
  A.opac = c->d_opac.p; A.cdf = c->d_cdf.p; A.eps_imc = c->d_eps_imc.p;
  A.cdf_coarse = c->d_cdf_coarse.p; A.n_coarse = c->n_coarse;
  A.cdf_guide = c->guide_n ? c->d_cdf_guide.p : nullptr; A.guide_n = c->guide_n;
  A.rescale_lum = c->tp.core_fix_luminosity;
  A.J = c->d_J.p; A.e_abs = c->d_e_abs.p; A.e_rad = c->d_e_rad.p;
  A.fx = c->d_fx.p; A.fy = c->d_fy.p; A.fz = c->d_fz.p; A.fr = c->d_fr.p;
  A.flux = c->d_flux.p; A.click = c->d_click.p; A.counters = c->d_counters.p;
  return A;
}

GridDev sed::make_grid_dev(sed_ctx* c)
{
  GridDev G{};
  G.type = c->gtype; G.nzones = c->nz; G.homologous = c->homologous; G.t_grid = c->t_grid;
  if (c->gtype == SED_GRID_1D_SPHERE) {
    G.r_out = dev_loc(c->r_out, c->d_r_out);
    G.v_r = c->d_v_r.p;
  } else {
    G.nx = c->nx; G.ny = c->ny; G.nz = c->nzz;
    for (int a = 0; a < 3; ++a) G.ax[a] = dev_loc(c->ax[a], c->d_ax[a]);
  }
  return G;
}

// core emission CDF, transport::setup_core_emission (src/transport/transport_init.cpp:465-556)
std::vector<double> sed::core_emission_cdf(const HostLoc& nug, double T)
{
  const int nn = nug.n();
  std::vector<double> cdf(nn);
  for (int j = 0; j < nn; ++j) {
    const double nu = nug.center(j), dnu = nug.delta(j);
    double bb;
    if (T <= 0) bb = 1;
    else {
      const double zeta = H_PLANCK * nu / K_BOLTZ / T;
      bb = 2.0 * nu * nu * nu * H_PLANCK / C_LIGHT / C_LIGHT / (std::exp(zeta) - 1);
    }
    const double w = bb * dnu * 1.0;
    cdf[j] = (j == 0) ? w : cdf[j - 1] + w;
  }
  for (int j = 0; j < nn; ++j) if (std::isnan(cdf[j])) cdf[j] = 0;
  if (cdf[nn - 1] == 0) for (int j = 0; j < nn; ++j) cdf[j] = 1.0;
  const double N = cdf[nn - 1];
  for (int j = 0; j < nn; ++j) cdf[j] /= N;
  return cdf;
}

extern "C" {

const char* sed_version(void) { return "sedona-b200 transport 0.1 (sm_100a)"; }

// gamma-ray spectrum and the radioactive scalars, once per context
static int alloc_gamma_spectrum(sed_ctx* c)
{
  if (c->nspec_g > 0) return SED_OK;
  CK(upload(c, c->d_gn, c->gn.x.data(), c->gn.x.size()));
  c->nspec_g = (int64_t)c->st.n() * c->gn.n() * c->sm.n() * c->sp.n();
  CK(c->d_gflux.resize(c->nspec_g));
  CK(c->d_gclick.resize(c->nspec_g));
  CK(cudaMemsetAsync(c->d_gflux.p, 0, c->nspec_g * sizeof(double), c->stream));
  CK(cudaMemsetAsync(c->d_gclick.p, 0, c->nspec_g * sizeof(double), c->stream));
  CK(c->d_L_tot.resize(1));
  CK(c->d_reject.resize(1));
  return SED_OK;
}

int sed_ctx_create(const sed_transport_params* p, int device, sed_ctx** out)
{
  if (!p || !out) return SED_ERR_ARG;
  *out = nullptr;
  if (!valid_grid(p->nu_grid) || !valid_grid(p->spec_time) || !valid_grid(p->spec_nu) || !valid_grid(p->spec_mu) ||
      !valid_grid(p->spec_phi))
    return SED_ERR_ARG;
  sed_ctx* c = new sed_ctx();
  if (device < 0) cudaGetDevice(&c->device);
  else c->device = device;
  cudaError_t e = cudaSetDevice(c->device);
  if (e != cudaSuccess) { delete c; return SED_ERR_CUDA; }
  cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, c->device);
  e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) { delete c; return SED_ERR_CUDA; }
  for (auto& ev : c->ev) cudaEventCreate(&ev);
  c->tp = *p;
  c->nu = host_loc(p->nu_grid);
  c->st = host_loc(p->spec_time);
  c->sn = host_loc(p->spec_nu);
  c->sm = host_loc(p->spec_mu);
  c->sp = host_loc(p->spec_phi);
  if (valid_grid(p->gamma_nu)) c->gn = host_loc(p->gamma_nu);
  else {  // one catch-all bin, as locate_array builds for an empty range
    c->gn.type = LOC_NONE; c->gn.min = -INFINITY; c->gn.del = 0; c->gn.x.assign(1, INFINITY);
  }
  // grid pointers in the copy are not retained
  c->tp.nu_grid.right = c->tp.spec_time.right = c->tp.spec_nu.right = c->tp.spec_mu.right = c->tp.spec_phi.right = nullptr;
  c->tp.gamma_nu.right = nullptr;
  CK(upload(c, c->d_nu, c->nu.x.data(), c->nu.x.size()));
  CK(upload(c, c->d_st, c->st.x.data(), c->st.x.size()));
  CK(upload(c, c->d_sn, c->sn.x.data(), c->sn.x.size()));
  CK(upload(c, c->d_sm, c->sm.x.data(), c->sm.x.size()));
  CK(upload(c, c->d_sp, c->sp.x.data(), c->sp.x.size()));
  const std::vector<double> cdf = core_emission_cdf(c->nu, p->core_temperature);
  CK(upload(c, c->d_core_cdf, cdf.data(), cdf.size()));
  c->nspec = (int64_t)c->st.n() * c->sn.n() * c->sm.n() * c->sp.n();
  CK(c->d_flux.resize(c->nspec));
  CK(c->d_click.resize(c->nspec));
  CK(c->d_counters.resize(C_COUNT + 1));
  CK(cudaMemsetAsync(c->d_flux.p, 0, c->nspec * sizeof(double), c->stream));
  CK(cudaMemsetAsync(c->d_click.p, 0, c->nspec * sizeof(double), c->stream));
  if (p->n_emit_radioactive > 0) {
    const int rc = alloc_gamma_spectrum(c);
    if (rc) return rc;
  }
  CK(cudaStreamSynchronize(c->stream));
  c->op.epsilon = 1.0;
  c->op.maximum_opacity = 1e40;
  c->op.temp_min = 1000;
  c->op.temp_max = 1e8;
  *out = c;
  return SED_OK;
}

int sed_set_grid(sed_ctx* c, const sed_grid* g)
{
  if (!c) return SED_ERR_ARG;
  c->have_diff = false;  // the last weighted forward no longer matches the context
  if (!g || g->n_zones <= 0 || !g->vol || !g->rho || !g->T_gas) return set_err(c, SED_ERR_ARG, "sed_set_grid: missing zone arrays");
  if (g->n_elems < 0 || (g->n_elems > 0 && (!g->X || !g->elem_A || !g->elem_Z)))
    return set_err(c, SED_ERR_ARG, "sed_set_grid: missing composition");
  const bool resized = (g->n_zones != c->nz) || !c->have_grid;
  c->gtype = g->type;
  c->nz = g->n_zones;
  c->nelem = g->n_elems;
  c->homologous = g->homologous;
  c->t_grid = g->t_now;
  // transport::init takes the grid's time (transport_init.cpp:371); a
  // time-dependent run then keeps its own clock, a steady-state run never
  // advances either
  if (!c->have_t_now || c->tp.steady_state) { c->t_now = g->t_now; c->have_t_now = true; }
  const size_t nz = (size_t)g->n_zones;
  if (g->type == SED_GRID_1D_SPHERE) {
    if (!g->r_out) return set_err(c, SED_ERR_ARG, "sed_set_grid: 1D sphere needs r_out");
    sed_locate_grid rg{g->n_zones, SED_LOC_FLEX, g->r_min, 0.0, g->r_out};
    c->r_out = host_loc(rg);
    CK(upload(c, c->d_r_out, g->r_out, nz));
    CK(upload_or_zero(c, c->d_v_r, g->v_r, nz));
  } else if (g->type == SED_GRID_3D_CART) {
    if ((int64_t)g->nx * g->ny * g->nz != g->n_zones) return set_err(c, SED_ERR_ARG, "sed_set_grid: nx*ny*nz != n_zones");
    if (!valid_grid(g->x_axis) || !valid_grid(g->y_axis) || !valid_grid(g->z_axis) || g->x_axis.n != g->nx ||
        g->y_axis.n != g->ny || g->z_axis.n != g->nz)
      return set_err(c, SED_ERR_ARG, "sed_set_grid: bad 3D axes");
    c->nx = g->nx; c->ny = g->ny; c->nzz = g->nz;
    const sed_locate_grid* axes[3] = {&g->x_axis, &g->y_axis, &g->z_axis};
    for (int a = 0; a < 3; ++a) {
      c->ax[a] = host_loc(*axes[a]);
      CK(upload(c, c->d_ax[a], c->ax[a].x.data(), c->ax[a].x.size()));
    }
  } else {
    return set_err(c, SED_ERR_ARG, "sed_set_grid: unknown grid type %d", g->type);
  }
  CK(upload(c, c->d_vol, g->vol, nz));
  CK(upload(c, c->d_rho, g->rho, nz));
  CK(upload(c, c->d_T, g->T_gas, nz));
  CK(upload_or_zero(c, c->d_egas, g->e_gas, nz));
  CK(upload_or_zero(c, c->d_grey, g->total_grey_opacity, nz));
  CK(upload(c, c->d_X, g->X, nz * (size_t)g->n_elems));
  CK(upload(c, c->d_eZ, g->elem_Z, (size_t)g->n_elems));
  CK(upload(c, c->d_eA, g->elem_A, (size_t)g->n_elems));
  c->h_eZ.assign(g->elem_Z, g->elem_Z + g->n_elems);
  if (resized) {
    int rc = alloc_tallies(c);
    if (rc) return rc;
    c->have_opacity = false;
  }
  int rc = alloc_lte(c);
  if (rc) return rc;
  // per-atom epsilon switch
  std::vector<int32_t> ze(std::max(c->nelem, 1), 0);
  c->any_zero_eps = false;
  for (int a = 0; a < c->nelem; ++a)
    for (int z : c->zero_eps) if (z == c->h_eZ[a]) { ze[a] = 1; c->any_zero_eps = true; }
  CK(upload(c, c->d_zero_eps_atom, ze.data(), ze.size()));
  c->have_grid = true;
  CK(cudaStreamSynchronize(c->stream));
  return SED_OK;
}

int sed_set_opacity_params(sed_ctx* c, const sed_opacity_params* op)
{
  if (!c || !op) return SED_ERR_ARG;
  c->op = *op;
  c->zero_eps.assign(op->atom_zero_epsilon, op->atom_zero_epsilon + std::max(op->n_atom_zero_epsilon, 0));
  c->op.atom_zero_epsilon = nullptr;
  if (c->have_grid) {
    std::vector<int32_t> ze(std::max(c->nelem, 1), 0);
    c->any_zero_eps = false;
    for (int a = 0; a < c->nelem; ++a)
      for (int z : c->zero_eps) if (z == c->h_eZ[a]) { ze[a] = 1; c->any_zero_eps = true; }
    CK(upload(c, c->d_zero_eps_atom, ze.data(), ze.size()));
    CK(cudaStreamSynchronize(c->stream));
  }
  return SED_OK;
}

int sed_set_atomic_data(sed_ctx* c, const sed_atomic_data* a)
{
  if (!c || !a || a->n_atoms < 0) return SED_ERR_ARG;
  if (!c->have_grid) return set_err(c, SED_ERR_STATE, "sed_set_atomic_data: call sed_set_grid first");
  if (a->n_atoms != c->nelem) return set_err(c, SED_ERR_ARG, "sed_set_atomic_data: %d atoms for %d elements", a->n_atoms, c->nelem);
  const int na = a->n_atoms;
  const int nn = c->nu.n();
  c->natoms = na;
  c->n_ions_total = a->ion_off[na];
  c->n_lev_total = a->lev_off[na];
  CK(upload(c, c->d_ion_off, a->ion_off, (size_t)na + 1));
  CK(upload(c, c->d_ion_chi, a->ion_chi, (size_t)c->n_ions_total));
  CK(upload(c, c->d_lev_off, a->lev_off, (size_t)na + 1));
  const size_t nl = (size_t)c->n_lev_total;
  CK(upload(c, c->d_lev_ion, a->lev_ion, nl));
  CK(upload(c, c->d_lev_g, a->lev_g, nl));
  CK(upload(c, c->d_lev_ic, a->lev_ic, nl));
  CK(upload(c, c->d_lev_E, a->lev_E, nl));
  CK(upload(c, c->d_lev_Eion, a->lev_Eion, nl));
  CK(upload(c, c->d_photo_off, a->photo_off, nl + 1));
  const size_t np = (size_t)a->photo_off[nl];
  CK(upload(c, c->d_photo_E, a->photo_E, np));
  CK(upload(c, c->d_photo_s, a->photo_s, np));
  {
    std::vector<int32_t> ia((size_t)std::max(c->n_ions_total, 1), 0), la(std::max(nl, (size_t)1), 0);
    for (int at = 0; at < na; ++at) {
      for (int i = a->ion_off[at]; i < a->ion_off[at + 1]; ++i) ia[i] = at;
      for (int l = a->lev_off[at]; l < a->lev_off[at + 1]; ++l) la[l] = at;
    }
    CK(upload(c, c->d_ion_atom, ia.data(), ia.size()));
    CK(upload(c, c->d_lev_atom, la.data(), la.size()));
  }
  // bins by decreasing line count (ties by bin): the line-sum kernel deals
  // them to threads in this order so the lanes of a warp get similar counts
  auto bin_order = [&](const std::vector<int32_t>& seg) {
    std::vector<int32_t> o(nn);
    std::iota(o.begin(), o.end(), 0);
    std::stable_sort(o.begin(), o.end(), [&](int x, int y) { return seg[x + 1] - seg[x] > seg[y + 1] - seg[y]; });
    return o;
  };
  // level-to-level lines: bin (AtomicData.cpp:680), stable sort by (bin, atom)
  // so each bin is one contiguous run in the atoms' list order; per line the
  // absolute level indices, sigma_tot f lambda and g_l/g_u
  {
    const int n = a->line_off[na];
    std::vector<int> order(n);
    std::vector<int64_t> key(n);
    std::vector<int> atom_of(n);
    for (int at = 0; at < na; ++at)
      for (int k = a->line_off[at]; k < a->line_off[at + 1]; ++k) {
        key[k] = (int64_t)c->nu.within(a->line_nu[k]) * na + at;
        atom_of[k] = at;
      }
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return key[x] < key[y]; });
    std::vector<int4> lv(std::max(n, 1));
    std::vector<double2> lc(std::max(n, 1));
    std::vector<float2> lc32(std::max(n, 1));
    std::vector<int32_t> seg((size_t)nn + 1, 0);
    for (int k = 0; k < n; ++k) {
      const int s = order[k], at = atom_of[s], l0 = a->lev_off[at];
      const int ll = l0 + a->line_l[s], lu = l0 + a->line_u[s];
      lv[k] = make_int4(ll, lu, (int)(key[s] / na), at);
      const double lam = C_LIGHT / a->line_nu[s];
      const double gr = (1.0 * a->lev_g[ll]) / (1.0 * a->lev_g[lu]);
      lc[k] = make_double2(SIGMA_TOT * a->line_f[s] * lam, gr);
      lc32[k] = make_float2((float)lc[k].x, (float)gr);
      seg[key[s] / na + 1]++;
    }
    for (size_t q = 1; q < seg.size(); ++q) seg[q] += seg[q - 1];
    c->nlines = n;
    const std::vector<int32_t> ord = bin_order(seg);
    CK(upload(c, c->d_ln_order, ord.data(), ord.size()));
    CK(upload(c, c->d_ln_seg, seg.data(), seg.size()));
    CK(upload(c, c->d_ln_lv, lv.data(), lv.size()));
    CK(upload(c, c->d_ln_c, lc.data(), lc.size()));
    CK(upload(c, c->d_ln_c32, lc32.data(), lc32.size()));
    CK(cudaStreamSynchronize(c->stream));
  }
  // fuzz lines: bin (AtomicData.cpp:851), stable sort by (bin, atom); per line
  // the absolute ion index, sigma_tot lambda gf, E_l/k_ev, h nu/k
  {
    const int n = a->fuzz_off[na];
    std::vector<int64_t> key(n);
    std::vector<int> order(n), atom_of(n);
    for (int at = 0; at < na; ++at)
      for (int k = a->fuzz_off[at]; k < a->fuzz_off[at + 1]; ++k) {
        key[k] = (int64_t)c->nu.within(a->fuzz_nu[k]) * na + at;
        atom_of[k] = at;
      }
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return key[x] < key[y]; });
    std::vector<int4> fia(std::max(n, 1));
    std::vector<double2> fc(std::max(n, 1));
    std::vector<double> fh(std::max(n, 1));
    std::vector<float4> fc32(std::max(n, 1));
    std::vector<int32_t> seg((size_t)nn + 1, 0);
    for (int k = 0; k < n; ++k) {
      const int s = order[k], at = atom_of[s];
      const double fnu = a->fuzz_nu[s];
      fia[k] = make_int4(a->ion_off[at] + a->fuzz_ion[s], (int)(key[s] / na), at, 0);
      fc[k] = make_double2(SIGMA_TOT * (C_LIGHT / fnu) * a->fuzz_gf[s], a->fuzz_El[s] / K_EV);
      fh[k] = H_PLANCK * fnu / K_BOLTZ;
      fc32[k] = make_float4((float)fc[k].x, (float)fc[k].y, (float)fh[k], 0.f);
      seg[key[s] / na + 1]++;
    }
    for (size_t q = 1; q < seg.size(); ++q) seg[q] += seg[q - 1];
    c->nfuzz = n;
    const std::vector<int32_t> ord = bin_order(seg);
    CK(upload(c, c->d_fz_order, ord.data(), ord.size()));
    CK(upload(c, c->d_fz_seg, seg.data(), seg.size()));
    CK(upload(c, c->d_fz_ia, fia.data(), fia.size()));
    CK(upload(c, c->d_fz_c, fc.data(), fc.size()));
    CK(upload(c, c->d_fz_h, fh.data(), fh.size()));
    CK(upload(c, c->d_fz_c32, fc32.data(), fc32.size()));
    CK(cudaStreamSynchronize(c->stream));
  }
  c->have_atoms = true;
  int rc = alloc_lte(c);
  if (rc) return rc;
  CK(cudaStreamSynchronize(c->stream));
  return SED_OK;
}

}  // extern "C"

int sed::enqueue_opacity(sed_ctx* c, double dt)
{
  if (!c) return SED_ERR_ARG;
  c->have_diff = false;  // the last weighted forward no longer matches the context
  if (!c->have_grid) return set_err(c, SED_ERR_STATE, "sed_set_opacity: no grid");
  if (c->tp.steady_state) dt = 1;
  OpacityArgs A{};
  A.nzones = c->nz; A.n_nu = c->nu.n(); A.nelem = c->nelem;
  A.seq_cdf = (c->nz <= 65536) ? 1 : 0;
  A.use_es = c->op.use_electron_scattering; A.use_ff = c->op.use_free_free; A.use_bf = c->op.use_bound_free;
  A.use_line = c->op.use_line_expansion; A.use_fuzz = c->op.use_fuzz_expansion;
  A.radiative_eq = c->tp.radiative_eq; A.omit_scat = c->tp.omit_scattering; A.precision = c->tp.precision;
  A.epsilon = c->op.epsilon; A.max_opacity = c->op.maximum_opacity; A.temp_min = c->op.temp_min;
  A.temp_max = c->op.temp_max; A.fleck_alpha = c->tp.fleck_alpha; A.dt = dt; A.time = c->t_now;
  A.nu = dev_loc(c->nu, c->d_nu);
  A.rho = c->d_rho.p; A.T = c->d_T.p; A.e_gas = c->d_egas.p; A.grey = c->d_grey.p; A.X = c->d_X.p;
  A.eZ = c->d_eZ.p; A.eA = c->d_eA.p; A.zero_eps_atom = c->d_zero_eps_atom.p;
  A.natoms = c->have_atoms ? c->natoms : 0;
  A.ion_off = c->d_ion_off.p; A.lev_off = c->d_lev_off.p; A.lev_ion = c->d_lev_ion.p; A.lev_g = c->d_lev_g.p;
  A.lev_ic = c->d_lev_ic.p; A.photo_off = c->d_photo_off.p; A.ion_chi = c->d_ion_chi.p; A.lev_E = c->d_lev_E.p;
  A.lev_Eion = c->d_lev_Eion.p; A.photo_E = c->d_photo_E.p; A.photo_s = c->d_photo_s.p;
  A.ion_atom = c->d_ion_atom.p; A.lev_atom = c->d_lev_atom.p;
  A.ln_order = c->d_ln_order.p; A.fz_order = c->d_fz_order.p;
  A.ln_seg = c->d_ln_seg.p; A.ln_lv = c->d_ln_lv.p; A.ln_c = c->d_ln_c.p; A.ln_c32 = c->d_ln_c32.p;
  A.fz_seg = c->d_fz_seg.p; A.fz_ia = c->d_fz_ia.p; A.fz_c = c->d_fz_c.p; A.fz_h = c->d_fz_h.p;
  A.fz_c32 = c->d_fz_c32.p;
  A.uniform_eps = c->any_zero_eps ? 0 : 1;
  A.smem_rows = rows_in_smem((size_t)std::max(c->nelem, 1), (size_t)c->nu.n());
  if (!A.uniform_eps && c->d_epsl64.n < (size_t)c->chunk_zones * c->nu.n()) {
    int rc = alloc_lte(c);  // epsilon-weighted sums appear with the first atom of epsilon 0
    if (rc) return rc;
  }
  A.epsl64 = c->d_epsl64.p; A.epsf64 = c->d_epsf64.p;
  if (A.natoms > 0 && (A.use_line || A.use_fuzz)) {
    const int npop = std::max(A.use_line ? c->n_lev_total : 0, A.use_fuzz ? c->n_ions_total : 0);
    if (line_sum_smem_bytes(c->tp.precision, c->natoms, npop) > SMEM_ZONE_BYTES)
      return set_err(c, SED_ERR_CAPACITY, "sed_set_opacity: %d populations per zone exceed the line-sum kernel's "
                     "shared memory", npop);
  }
  if (A.natoms > 0 && ((A.use_line && c->nlines > 0 && !c->d_ln_seg.p) || (A.use_fuzz && !c->d_fz_seg.p)))
    return set_err(c, SED_ERR_STATE, "sed_set_opacity: line lists not set");
  if (A.natoms == 0) { A.use_line = 0; A.use_fuzz = 0; }
  A.ion_part = c->d_ion_part.p; A.ion_frac = c->d_ion_frac.p; A.lev_n = c->d_lev_n.p;
  A.n_ions_total = c->n_ions_total; A.n_lev_total = c->n_lev_total;
  A.n_elec = c->d_n_elec.p; A.n_dens = c->d_n_dens.p; A.mass_frac = c->d_mass_frac.p; A.temp_c = c->d_temp_c.p;
  A.solve_err = c->d_solve_err.p; A.boltz = c->d_boltz.p;
  A.abs64 = c->d_abs64.p; A.scat64 = c->d_scat64.p; A.emis64 = c->d_emis64.p;
  A.opac_out = c->d_opac.p; A.cdf_out = c->d_cdf.p;
  A.cdf_coarse_out = c->d_cdf_coarse.p; A.n_coarse = c->n_coarse;
  A.cdf_guide_out = c->guide_n ? c->d_cdf_guide.p : nullptr; A.guide_n = c->guide_n;
  A.eps_imc = c->d_eps_imc.p; A.planck = c->d_planck.p; A.ross = c->d_ross.p; A.L_th = c->d_L.p;
  // passes over chunks of zones: per-zone inputs and outputs are offset to
  // the chunk, the scratch is reused with the chunk's zone count as stride
  const size_t nn = (size_t)c->nu.n(), esz = c->tp.precision ? sizeof(float) : sizeof(double);
  CK(cudaEventRecord(c->ev[0], c->stream));
  c->opacity_launches = 0;
  for (int z0 = 0; z0 < c->nz; z0 += c->chunk_zones) {
    const size_t o = (size_t)z0;
    OpacityArgs B = A;
    B.nzones = std::min(c->chunk_zones, c->nz - z0);
    B.rho += o; B.T += o; B.e_gas += o; B.grey += o; B.X += o * (size_t)c->nelem;
    B.n_elec += o; B.temp_c += o; B.solve_err += o;
    B.eps_imc += o; B.planck += o; B.ross += o; B.L_th += o;
    B.opac_out = static_cast<unsigned char*>(A.opac_out) + o * nn * 2 * esz;
    B.cdf_out = static_cast<unsigned char*>(A.cdf_out) + o * nn * esz;
    B.cdf_coarse_out = static_cast<unsigned char*>(A.cdf_coarse_out) + o * (size_t)c->n_coarse * esz;
    if (A.cdf_guide_out) B.cdf_guide_out = A.cdf_guide_out + o * (size_t)(c->guide_n + 1);
    const int nl = launch_opacity(B, c->num_sms, c->stream);
    CK(cudaGetLastError());
    if (nl < 0) return set_err(c, SED_ERR_CUDA, "sed_set_opacity: opacity kernel configuration rejected");
    c->opacity_launches += nl;
  }
  return SED_OK;
}

extern "C" {

int sed_set_opacity(sed_ctx* c, double dt)
{
  if (!c) return SED_ERR_ARG;
  int rc = enqueue_opacity(c, dt);
  if (rc) return rc;
  CK(cudaEventRecord(c->ev[1], c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->have_opacity = true;
  c->opac_base_valid = false;
  c->opac_scaled = false;
  return SED_OK;
}

int sed_load_opacity(sed_ctx* c, const double* abs, const double* scat, const double* emis_cdf, const double* eps_imc)
{
  if (!c || !abs || !emis_cdf || !eps_imc) return SED_ERR_ARG;
  c->have_diff = false;  // the last weighted forward no longer matches the context
  if (!c->have_grid) return set_err(c, SED_ERR_STATE, "sed_load_opacity: no grid");
  const size_t n = (size_t)c->nz * c->nu.n();
  // guide tables of the stored rows (value(i) = stored CDF entry i as a double)
  auto upload_guide = [&](auto value) -> int {
    if (!c->guide_n) return SED_OK;
    const int G = c->guide_n, nn = c->nu.n();
    std::vector<uint16_t> g((size_t)c->nz * (G + 1));
    for (int z = 0; z < c->nz; ++z)
      for (int k = 0; k <= G; ++k) {
        const double t = (double)k / (double)G;
        int lo = 0, hi = nn;
        while (lo < hi) {
          const int m = (lo + hi) >> 1;
          if (value((size_t)z * nn + m) <= t) lo = m + 1; else hi = m;
        }
        g[(size_t)z * (G + 1) + k] = (uint16_t)lo;
      }
    CK(cudaMemcpyAsync(c->d_cdf_guide.p, g.data(), g.size() * sizeof(uint16_t), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return SED_OK;
  };
  int rc = SED_OK;
  if (c->tp.precision) {
    std::vector<float> o(2 * n), cd(n);
    for (size_t i = 0; i < n; ++i) { o[2 * i] = (float)abs[i]; o[2 * i + 1] = scat ? (float)scat[i] : 0.f; cd[i] = (float)emis_cdf[i]; }
    CK(cudaMemcpyAsync(c->d_opac.p, o.data(), o.size() * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->d_cdf.p, cd.data(), cd.size() * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    std::vector<float> co((size_t)c->nz * c->n_coarse);
    for (int z = 0; z < c->nz; ++z)
      for (int k = 0; k < c->n_coarse; ++k)
        co[(size_t)z * c->n_coarse + k] = cd[(size_t)z * c->nu.n() + std::min((k + 1) * CDF_STRIDE - 1, c->nu.n() - 1)];
    CK(cudaMemcpyAsync(c->d_cdf_coarse.p, co.data(), co.size() * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    rc = upload_guide([&](size_t i) { return (double)cd[i]; });
  } else {
    std::vector<double> o(2 * n);
    for (size_t i = 0; i < n; ++i) { o[2 * i] = abs[i]; o[2 * i + 1] = scat ? scat[i] : 0.0; }
    CK(cudaMemcpyAsync(c->d_opac.p, o.data(), o.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->d_cdf.p, emis_cdf, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    std::vector<double> co((size_t)c->nz * c->n_coarse);
    for (int z = 0; z < c->nz; ++z)
      for (int k = 0; k < c->n_coarse; ++k)
        co[(size_t)z * c->n_coarse + k] = emis_cdf[(size_t)z * c->nu.n() + std::min((k + 1) * CDF_STRIDE - 1, c->nu.n() - 1)];
    CK(cudaMemcpyAsync(c->d_cdf_coarse.p, co.data(), co.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    rc = upload_guide([&](size_t i) { return emis_cdf[i]; });
  }
  if (rc) return rc;
  CK(cudaMemcpyAsync(c->d_eps_imc.p, eps_imc, (size_t)c->nz * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->have_opacity = true;
  c->opac_base_valid = false;
  c->opac_scaled = false;
  return SED_OK;
}

// The stopped packets of the step, in the reference's vector order, become
// the census (clean_up_particle_vector, transport.cpp:164-194).
static int build_census(sed_ctx* c, CensusArgs& C, int64_t n_all, int64_t* n_alive)
{
  const size_t m = (size_t)n_all + 1;
  CK(c->d_cmp.resize(5 * m));
  C.flag_e = c->d_cmp.p; C.flag_a = C.flag_e + m; C.scan_e = C.flag_a + m; C.scan_a = C.scan_e + m;
  C.front_dead = C.scan_a + m;
  CK(c->d_cmp_count.resize(1));
  C.n_gamma = c->d_cmp_count.p;
  CK(cudaMemsetAsync(C.n_gamma, 0, sizeof(unsigned long long), c->stream));
  CK(c->d_census_state.resize(std::max<size_t>(m - 1, 1) * 9));
  CK(c->d_census_ind.resize(std::max<size_t>(m - 1, 1)));
  CK(c->d_census_type.resize(std::max<size_t>(m - 1, 1)));
  C.census_state = c->d_census_state.p; C.census_ind = c->d_census_ind.p; C.census_type = c->d_census_type.p;
  launch_census_flags(C, n_all, c->stream);
  size_t tmp = 0;
  CK(cub::DeviceScan::ExclusiveSum(nullptr, tmp, C.flag_e, C.scan_e, (int)m, c->stream));
  CK(c->d_scan_tmp.resize(std::max<size_t>(tmp, 1)));
  CK(cub::DeviceScan::ExclusiveSum(c->d_scan_tmp.p, tmp, C.flag_e, C.scan_e, (int)m, c->stream));
  CK(cub::DeviceScan::ExclusiveSum(c->d_scan_tmp.p, tmp, C.flag_a, C.scan_a, (int)m, c->stream));
  launch_census_compact(C, n_all, c->stream);
  CK(cudaGetLastError());
  int32_t na = 0;
  unsigned long long ng = 0;
  CK(cudaMemcpyAsync(&na, C.scan_a + n_all, sizeof na, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(&ng, C.n_gamma, sizeof ng, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  *n_alive = na;
  c->n_census_gamma = (int64_t)ng;
  return SED_OK;
}

static int transport_impl(sed_ctx* c, double dt, sed_step_stats* stats, float ms_opacity)
{
  if (!c) return SED_ERR_ARG;
  c->have_diff = false;  // the last weighted forward no longer matches the context
  if (!c->have_grid) return set_err(c, SED_ERR_STATE, "sed_transport: no grid");
  if (!c->have_opacity) return set_err(c, SED_ERR_STATE, "sed_transport: opacity tables not set");
  if (c->tp.steady_state) dt = 1;
  const bool timedep = !c->tp.steady_state;
  // emit_inner_source packet count and energy (src/transport/emission.cpp:383-392)
  int64_t n_emit = (int64_t)(c->tp.core_n_emit / 1.0);
  // The packet list of the step (transport.cpp:46-54): the census the last
  // step left, then emit_radioactive (emission.cpp:163-243: it adds nothing
  // when its packets would not fit next to the census), then the core
  // packets.  When those would not fit next to both, emit_inner_source
  // prints "# Not enough particle space" and emits nothing
  // (emission.cpp:391-392), and the step goes on with the others: so here,
  // flagged in the step's warnings.  Census and radioactive packets are the
  // queue; their Philox streams come first, the core packets' after.
  const int64_t n_census = c->n_census;
  int64_t n_radio = c->tp.n_emit_radioactive > 0 ? c->tp.n_emit_radioactive : 0;
  if (n_census + n_radio > c->tp.max_particles) n_radio = 0;
  int32_t warnings = 0;
  if (n_census + n_radio + n_emit > c->tp.max_particles) {
    n_emit = 0;
    warnings |= SED_WARN_NO_PARTICLE_SPACE;
  }
  if (c->tp.use_ddmc != 0 && ((c->tp.use_ddmc != 1 && c->tp.use_ddmc != 2) || c->gtype != SED_GRID_1D_SPHERE))
    return set_err(c, SED_ERR_ARG,
                   "transport_use_ddmc %d: discrete diffusion is built for methods 1 (IMD) and 2 (DDMC) on 1D spheres",
                   (int)c->tp.use_ddmc);
  const int64_t n_q = n_census + n_radio;
  const int64_t n_all = n_emit + n_q;
  const bool gamma_phase = n_radio > 0 || (n_census > 0 && c->n_census_gamma > 0);
  const bool keep = c->record || timedep;  // end states: records, and the next census
  const size_t nz = (size_t)c->nz, nn = (size_t)c->nu.n();
  const size_t nj = c->tp.store_Jnu ? nn : 1;
  if (keep) {
    CK(c->d_rec_fate.resize(std::max<int64_t>(n_all, 1)));
    CK(c->d_rec_ind.resize(std::max<int64_t>(n_all, 1)));
    CK(c->d_rec_draws.resize(std::max<int64_t>(n_all, 1)));
    CK(c->d_rec_type.resize(std::max<int64_t>(n_all, 1)));
    CK(c->d_rec_state.resize(std::max<int64_t>(n_all, 1) * 9));
  }
  if (c->record) c->n_rec = n_all;
  if (n_q > 0) {
    CK(c->d_q_state.resize((size_t)n_q * 9));
    CK(c->d_q_ind.resize((size_t)n_q));
    CK(c->d_q_n.resize((size_t)n_q));
    CK(c->d_q_type.resize((size_t)n_q));
  }
  if (gamma_phase) {
    if (c->nspec_g == 0) {
      const int rc = alloc_gamma_spectrum(c);
      if (rc) return rc;
    }
    CK(c->d_radio_cdf.resize(nz)); CK(c->d_gamma_frac.resize(nz)); CK(c->d_compton.resize(nz));
    CK(c->d_photoion.resize(nz)); CK(c->d_L_emit.resize(nz)); CK(c->d_L_dep.resize(nz));
  }
  CK(cudaEventRecord(c->ev[2], c->stream));
  if (gamma_phase) {
    CK(cudaMemsetAsync(c->d_L_dep.p, 0, nz * sizeof(double), c->stream));
    CK(cudaMemsetAsync(c->d_L_emit.p, 0, nz * sizeof(double), c->stream));
    CK(cudaMemsetAsync(c->d_reject.p, 0, sizeof(int32_t), c->stream));
  }
  // spectra: a steady-state iteration starts from empty ones (the driver's
  // wipe_spectra, SedonaClass.cpp:349); a time-dependent run accumulates
  // them over its steps
  if (!timedep) {
    CK(cudaMemsetAsync(c->d_flux.p, 0, c->nspec * sizeof(double), c->stream));
    CK(cudaMemsetAsync(c->d_click.p, 0, c->nspec * sizeof(double), c->stream));
    if (c->nspec_g > 0) {
      CK(cudaMemsetAsync(c->d_gflux.p, 0, c->nspec_g * sizeof(double), c->stream));
      CK(cudaMemsetAsync(c->d_gclick.p, 0, c->nspec_g * sizeof(double), c->stream));
    }
  }
  // wipe_radiation (src/transport/transport_mpi.cpp:18-34) and the spectrum
  CK(cudaMemsetAsync(c->d_J.p, 0, nz * nj * sizeof(double), c->stream));
  CK(cudaMemsetAsync(c->d_e_abs.p, 0, nz * sizeof(double), c->stream));
  CK(cudaMemsetAsync(c->d_e_rad.p, 0, nz * sizeof(double), c->stream));
  CK(cudaMemsetAsync(c->d_fx.p, 0, nz * sizeof(double), c->stream));
  CK(cudaMemsetAsync(c->d_fy.p, 0, nz * sizeof(double), c->stream));
  CK(cudaMemsetAsync(c->d_fz.p, 0, nz * sizeof(double), c->stream));
  CK(cudaMemsetAsync(c->d_fr.p, 0, nz * sizeof(double), c->stream));
  CK(cudaMemsetAsync(c->d_counters.p, 0, (C_COUNT + 1) * sizeof(unsigned long long), c->stream));

  StepArgs A = make_step_args(c, dt, n_emit);
  if (keep) {
    A.rec_fate = c->d_rec_fate.p; A.rec_ind = c->d_rec_ind.p; A.rec_draws = c->d_rec_draws.p;
    A.rec_state = c->d_rec_state.p; A.rec_type = c->d_rec_type.p;
  }
  A.n_core = n_emit;
  const GridDev G = make_grid_dev(c);
  int launches = 0;
  CensusArgs C{};
  C.n_census = n_census; C.n_core = n_emit; C.n_q = n_q;
  if (n_q > 0) {
    C.q_state = c->d_q_state.p; C.q_ind = c->d_q_ind.p; C.q_type = c->d_q_type.p; C.q_n = c->d_q_n.p;
  }
  if (n_census > 0) {
    C.census_state = c->d_census_state.p; C.census_ind = c->d_census_ind.p; C.census_type = c->d_census_type.p;
    launches += launch_census_load(C, G, c->stream);
  }
  if (gamma_phase) {
    // decay luminosity and gamma-ray opacity per zone, then the census
    // gamma-rays and the radioactive packets; the optical photons they
    // become join the packet kernel's queue
    RadioArgs R{};
    R.nz = c->nz; R.n_elems = c->nelem; R.force_rproc = c->tp.force_rprocess_heating;
    R.n_census = n_census; R.n_radio = n_radio; R.first_pid = c->tp.first_packet_id;
    R.q_type = c->d_q_type.p;
    R.t_now = c->t_now; R.dt = dt;
    R.rho = c->d_rho.p; R.vol = c->d_vol.p; R.X = c->d_X.p; R.eZ = c->d_eZ.p; R.eA = c->d_eA.p;
    R.L_emit = c->d_L_emit.p; R.gamma_frac = c->d_gamma_frac.p; R.compton = c->d_compton.p;
    R.photoion = c->d_photoion.p; R.cdf = c->d_radio_cdf.p; R.L_tot = c->d_L_tot.p; R.L_dep = c->d_L_dep.p;
    R.q_state = c->d_q_state.p; R.q_ind = c->d_q_ind.p; R.q_n = c->d_q_n.p; R.n_reject_cap = c->d_reject.p;
    StepArgs AG = A;  // the gamma-ray spectrum
    AG.sn = dev_loc(c->gn, c->d_gn);
    AG.a3 = c->sp.n(); AG.a2 = (int64_t)c->sm.n() * AG.a3; AG.a1 = (int64_t)c->gn.n() * AG.a2;
    AG.flux = c->d_gflux.p; AG.click = c->d_gclick.p;
    launches += launch_radio_zones(R, c->stream);
    // emit_radioactive sets L_radio_emit only when it emits (emission.cpp:176, 205)
    if (n_radio == 0) CK(cudaMemsetAsync(c->d_L_emit.p, 0, nz * sizeof(double), c->stream));
    launches += launch_gamma(A, AG, R, G, c->num_sms, c->stream);
    CK(cudaGetLastError());
    A.L_dep = c->d_L_dep.p; A.L_emit = c->d_L_emit.p;
  }
  if (n_q > 0) {
    A.n_packets = n_all;
    A.first_pid = c->tp.first_packet_id + n_q;
    A.radio_first_pid = c->tp.first_packet_id;
    A.q_state = c->d_q_state.p; A.q_ind = c->d_q_ind.p; A.q_n = c->d_q_n.p;
  }
  if (c->tp.use_ddmc == 1) {  // compute_diffusion_probabilities(dt) (transport.cpp:44)
    CK(c->d_imd_p.resize(4 * nz));
    launches += launch_imd_probabilities(G, c->d_planck.p, dt, c->d_imd_p.p, c->stream);
    A.imd_p = c->d_imd_p.p;
  }
  if (mixed_1d_path(A, G) && n_emit > 0) {  // core packets emitted ahead of the packet kernel
    CK(c->d_em_state.resize((size_t)n_emit * 9));
    CK(c->d_em_ind.resize((size_t)n_emit));
    CK(c->d_em_tau.resize((size_t)n_emit));
    A.em_state = c->d_em_state.p; A.em_ind = c->d_em_ind.p; A.em_tau = c->d_em_tau.p; A.em_n = n_emit;
  }
  if (mixed_1d_path(A, G)) {
    // the 1D mixed kernel adds each zone visit's tallies to one of n_rep
    // global copies (block b to copy b % n_rep, fire-and-forget reductions),
    // which the finish kernel sums: against the per-block shared-memory
    // copies, whose atomic adds hold the warp, the Type Ia packet kernel ran
    // 563 ms against 587 ms
    const int n_rep = (int)std::min<size_t>(32, std::max<size_t>(1, (size_t(256) << 20) / (5 * sizeof(double) * nz)));
    CK(c->d_zone_rep.resize((size_t)n_rep * 5 * nz));
    CK(cudaMemsetAsync(c->d_zone_rep.p, 0, (size_t)n_rep * 5 * nz * sizeof(double), c->stream));
    A.smem_zones = 0; A.n_rep = n_rep; A.zone_rep = c->d_zone_rep.p;
  }
  CK(cudaEventRecord(c->ev[3], c->stream));
  if (A.n_packets > 0) launches += launch_propagate(A, G, c->num_sms, c->stream);
  CK(cudaGetLastError());
  CK(cudaEventRecord(c->ev[4], c->stream));
  launches += launch_finish(A, G, c->d_vol.p, c->nspec, c->stream);
  CK(cudaGetLastError());
  CK(cudaEventRecord(c->ev[5], c->stream));
  unsigned long long cnt[C_COUNT + 1];
  CK(cudaMemcpyAsync(cnt, c->d_counters.p, sizeof cnt, cudaMemcpyDeviceToHost, c->stream));
  int32_t n_reject_cap = 0;
  if (gamma_phase)
    CK(cudaMemcpyAsync(&n_reject_cap, c->d_reject.p, sizeof n_reject_cap, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  // the stopped packets stay for the next step; a steady-state step leaves
  // none (its packets never reach the end of the step)
  int64_t n_next = 0;
  if (timedep && n_all > 0) {
    C.rec_fate = c->d_rec_fate.p; C.rec_ind = c->d_rec_ind.p; C.rec_type = c->d_rec_type.p;
    C.rec_state = c->d_rec_state.p;
    const int rc = build_census(c, C, n_all, &n_next);
    if (rc) return rc;
    launches += 4;
  }
  c->n_census = n_next;
  if (n_next == 0) c->n_census_gamma = 0;
  c->step++;
  if (timedep) c->t_now += dt;
  if (stats) {
    std::memset(stats, 0, sizeof *stats);
    stats->n_packets = n_all;
    stats->n_escaped = (int64_t)cnt[C_ESCAPED];
    stats->n_absorbed = (int64_t)cnt[C_ABSORBED];
    stats->n_stopped = (int64_t)cnt[C_STOPPED];
    stats->n_segments = (int64_t)cnt[C_SEGMENTS];
    stats->n_scatters = (int64_t)cnt[C_SCATTERS];
    stats->n_limit = (int64_t)cnt[C_LIMIT];
    stats->kernel_launches = launches;
    stats->warnings = warnings;
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev[3], c->ev[4]);
    stats->ms_propagate_kernel = ms;
    cudaEventElapsedTime(&ms, c->ev[2], c->ev[5]);
    stats->ms_transport = ms;
    stats->ms_opacity = ms_opacity;
    stats->ms_total = ms + ms_opacity;
  }
  if (cnt[C_LIMIT] > 0) return set_err(c, SED_ERR_LIMIT, "%llu packets hit the segment limit", cnt[C_LIMIT]);
  if (cnt[C_DDMC_CAP] > 0)
    return set_err(c, SED_ERR_LIMIT, "%llu diffusion scatters found no new frequency bin", cnt[C_DDMC_CAP]);
  if (cnt[C_IMD_CAP] > 0) return set_err(c, SED_ERR_LIMIT, "%llu IMD calls hit the hop bound", cnt[C_IMD_CAP]);
  if (n_reject_cap > 0)
    return set_err(c, SED_ERR_LIMIT, "%d Compton scatters hit the rejection-sampling bound", (int)n_reject_cap);
  return SED_OK;
}

int sed_transport(sed_ctx* c, double dt, sed_step_stats* stats) { return transport_impl(c, dt, stats, 0.f); }

int sed_set_emission(sed_ctx* c, double core_n_emit, int64_t n_emit_radioactive)
{
  if (!c) return SED_ERR_ARG;
  c->have_diff = false;  // the last weighted forward no longer matches the context
  if (!(core_n_emit >= 0) || n_emit_radioactive < 0)
    return set_err(c, SED_ERR_ARG, "sed_set_emission: negative packet count");
  c->tp.core_n_emit = core_n_emit;
  c->tp.n_emit_radioactive = n_emit_radioactive;
  if (n_emit_radioactive > 0) {
    const int rc = alloc_gamma_spectrum(c);
    if (rc) return rc;
  }
  CK(cudaStreamSynchronize(c->stream));
  return SED_OK;
}

int sed_step(sed_ctx* c, double dt, sed_step_stats* stats)
{
  int rc = sed_set_opacity(c, dt);
  if (rc) return rc;
  float ms = 0;
  cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]);
  rc = transport_impl(c, dt, stats, ms);
  if (stats && rc == SED_OK) stats->kernel_launches += c->opacity_launches;
  return rc;
}

int sed_get_gamma_spectrum(sed_ctx* c, double* flux, double* click)
{
  if (!c) return SED_ERR_ARG;
  if (c->nspec_g == 0) return set_err(c, SED_ERR_STATE, "no radioactive source in this context");
  if (flux) CK(cudaMemcpyAsync(flux, c->d_gflux.p, c->nspec_g * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  if (click) CK(cudaMemcpyAsync(click, c->d_gclick.p, c->nspec_g * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return SED_OK;
}

int sed_get_radioactive_tallies(sed_ctx* c, double* L_radio_emit, double* L_radio_dep)
{
  if (!c) return SED_ERR_ARG;
  if (!c->d_L_dep.p) return set_err(c, SED_ERR_STATE, "no radioactive step yet");
  const size_t nz = (size_t)c->nz;
  if (L_radio_emit) CK(cudaMemcpyAsync(L_radio_emit, c->d_L_emit.p, nz * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  if (L_radio_dep) CK(cudaMemcpyAsync(L_radio_dep, c->d_L_dep.p, nz * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return SED_OK;
}

int sed_solve_temperature(sed_ctx* c, int32_t set_Tgas_to_Trad, double* T_gas, int32_t* n_unsolved)
{
  if (!c) return SED_ERR_ARG;
  if (!c->have_grid) return set_err(c, SED_ERR_STATE, "sed_solve_temperature: no grid");
  if (!c->have_opacity) return set_err(c, SED_ERR_STATE, "sed_solve_temperature: no opacity tables");
  TemperatureArgs A{};
  A.nz = c->nz; A.precision = c->tp.precision; A.set_Tgas_to_Trad = set_Tgas_to_Trad ? 1 : 0;
  A.nu = dev_loc(c->nu, c->d_nu);
  A.opac = c->d_opac.p; A.e_abs = c->d_e_abs.p; A.e_rad = c->d_e_rad.p;
  A.temp_min = c->op.temp_min; A.temp_max = c->op.temp_max;
  A.T = c->d_T.p;
  CK(c->d_temp_bad.resize(1));
  A.n_unsolved = c->d_temp_bad.p;
  CK(cudaMemsetAsync(c->d_temp_bad.p, 0, sizeof(int32_t), c->stream));
  launch_temperature(A, c->stream);
  CK(cudaGetLastError());
  int32_t bad = 0;
  CK(cudaMemcpyAsync(&bad, c->d_temp_bad.p, sizeof bad, cudaMemcpyDeviceToHost, c->stream));
  if (T_gas) CK(cudaMemcpyAsync(T_gas, c->d_T.p, (size_t)c->nz * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (n_unsolved) *n_unsolved = bad;
  return SED_OK;
}

int sed_get_spectrum(sed_ctx* c, double* flux, double* click)
{
  if (!c) return SED_ERR_ARG;
  if (flux) CK(cudaMemcpyAsync(flux, c->d_flux.p, c->nspec * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  if (click) CK(cudaMemcpyAsync(click, c->d_click.p, c->nspec * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return SED_OK;
}

int sed_get_zone_tallies(sed_ctx* c, double* J, double* e_abs, double* e_rad, double* fx, double* fy, double* fz,
                         double* fr)
{
  if (!c) return SED_ERR_ARG;
  if (!c->have_grid) return set_err(c, SED_ERR_STATE, "no grid");
  const size_t nz = (size_t)c->nz, nj = c->tp.store_Jnu ? (size_t)c->nu.n() : 1;
  if (J) CK(cudaMemcpyAsync(J, c->d_J.p, nz * nj * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  struct { double* h; double* d; } z[6] = {{e_abs, c->d_e_abs.p}, {e_rad, c->d_e_rad.p}, {fx, c->d_fx.p},
                                           {fy, c->d_fy.p}, {fz, c->d_fz.p}, {fr, c->d_fr.p}};
  for (auto& q : z) if (q.h) CK(cudaMemcpyAsync(q.h, q.d, nz * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return SED_OK;
}

int sed_get_opacity(sed_ctx* c, double* abs, double* scat, double* cdf, double* n_elec, double* eps_imc,
                    double* planck, double* ross, double* L_th)
{
  if (!c) return SED_ERR_ARG;
  if (!c->have_opacity) return set_err(c, SED_ERR_STATE, "no opacity tables");
  const size_t nz = (size_t)c->nz, n = nz * c->nu.n();
  // the tables the packet kernel reads: {abs, scat} pairs and the CDF, in
  // FP64 or FP32 by the context's precision, returned widened to double
  if (abs || scat) {
    if (c->tp.precision) {
      std::vector<float> o(2 * n);
      CK(cudaMemcpyAsync(o.data(), c->d_opac.p, 2 * n * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
      CK(cudaStreamSynchronize(c->stream));
      for (size_t i = 0; i < n; ++i) { if (abs) abs[i] = o[2 * i]; if (scat) scat[i] = o[2 * i + 1]; }
    } else {
      std::vector<double> o(2 * n);
      CK(cudaMemcpyAsync(o.data(), c->d_opac.p, 2 * n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
      CK(cudaStreamSynchronize(c->stream));
      for (size_t i = 0; i < n; ++i) { if (abs) abs[i] = o[2 * i]; if (scat) scat[i] = o[2 * i + 1]; }
    }
  }
  if (cdf) {
    if (c->tp.precision) {
      std::vector<float> o(n);
      CK(cudaMemcpyAsync(o.data(), c->d_cdf.p, n * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
      CK(cudaStreamSynchronize(c->stream));
      for (size_t i = 0; i < n; ++i) cdf[i] = o[i];
    } else {
      CK(cudaMemcpyAsync(cdf, c->d_cdf.p, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    }
  }
  struct { double* h; double* d; } z[5] = {{n_elec, c->d_n_elec.p}, {eps_imc, c->d_eps_imc.p}, {planck, c->d_planck.p},
                                           {ross, c->d_ross.p}, {L_th, c->d_L.p}};
  for (auto& q : z) if (q.h) CK(cudaMemcpyAsync(q.h, q.d, nz * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return SED_OK;
}

int sed_record_packets(sed_ctx* c, int32_t enable)
{
  if (!c) return SED_ERR_ARG;
  c->record = enable ? 1 : 0;
  return SED_OK;
}

int sed_get_packet_records(sed_ctx* c, int64_t n, int32_t* fate, int32_t* ind, int32_t* draws, double* state9)
{
  if (!c) return SED_ERR_ARG;
  if (!c->record || n > c->n_rec) return set_err(c, SED_ERR_STATE, "no packet records for %lld packets", (long long)n);
  if (fate) CK(cudaMemcpyAsync(fate, c->d_rec_fate.p, n * 4, cudaMemcpyDeviceToHost, c->stream));
  if (ind) CK(cudaMemcpyAsync(ind, c->d_rec_ind.p, n * 4, cudaMemcpyDeviceToHost, c->stream));
  if (draws) CK(cudaMemcpyAsync(draws, c->d_rec_draws.p, n * 4, cudaMemcpyDeviceToHost, c->stream));
  if (state9) CK(cudaMemcpyAsync(state9, c->d_rec_state.p, n * 9 * 8, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return SED_OK;
}

int64_t sed_n_particles(sed_ctx* c) { return c ? c->n_census : 0; }

int sed_set_core_source(sed_ctx* c, double luminosity, const double* weights)
{
  if (!c) return SED_ERR_ARG;
  c->have_diff = false;  // the last weighted forward no longer matches the context
  if (!(luminosity >= 0)) return set_err(c, SED_ERR_ARG, "sed_set_core_source: luminosity %g", luminosity);
  c->tp.core_luminosity = luminosity;
  if (weights) {
    // core_emission_spectrum_: cdf_array::set_value in bin order, then normalize
    const int nn = c->nu.n();
    std::vector<double> cdf(nn);
    for (int j = 0; j < nn; ++j) cdf[j] = (j == 0) ? weights[0] : cdf[j - 1] + weights[j];
    for (int j = 0; j < nn; ++j) if (std::isnan(cdf[j])) cdf[j] = 0;
    if (cdf[nn - 1] == 0) for (int j = 0; j < nn; ++j) cdf[j] = 1.0;
    const double N = cdf[nn - 1];
    for (int j = 0; j < nn; ++j) cdf[j] /= N;
    CK(upload(c, c->d_core_cdf, cdf.data(), cdf.size()));
    CK(cudaStreamSynchronize(c->stream));
  }
  return SED_OK;
}

int sed_wipe_spectra(sed_ctx* c)
{
  if (!c) return SED_ERR_ARG;
  CK(cudaMemsetAsync(c->d_flux.p, 0, c->nspec * sizeof(double), c->stream));
  CK(cudaMemsetAsync(c->d_click.p, 0, c->nspec * sizeof(double), c->stream));
  if (c->nspec_g > 0) {
    CK(cudaMemsetAsync(c->d_gflux.p, 0, c->nspec_g * sizeof(double), c->stream));
    CK(cudaMemsetAsync(c->d_gclick.p, 0, c->nspec_g * sizeof(double), c->stream));
  }
  CK(cudaStreamSynchronize(c->stream));
  return SED_OK;
}

int sed_set_time(sed_ctx* c, double t_now)
{
  if (!c) return SED_ERR_ARG;
  c->have_diff = false;  // the last weighted forward no longer matches the context
  c->t_now = t_now;
  c->have_t_now = true;
  return SED_OK;
}

double sed_get_time(sed_ctx* c) { return c ? c->t_now : 0.0; }

int sed_get_particles(sed_ctx* c, int64_t n, int32_t* ind, int32_t* type, double* state9)
{
  if (!c) return SED_ERR_ARG;
  if (n < 0 || n > c->n_census) return set_err(c, SED_ERR_ARG, "sed_get_particles: %lld of %lld packets",
                                               (long long)n, (long long)c->n_census);
  if (n == 0) return SED_OK;
  if (ind) CK(cudaMemcpyAsync(ind, c->d_census_ind.p, n * 4, cudaMemcpyDeviceToHost, c->stream));
  if (type) CK(cudaMemcpyAsync(type, c->d_census_type.p, n * 4, cudaMemcpyDeviceToHost, c->stream));
  if (state9) CK(cudaMemcpyAsync(state9, c->d_census_state.p, n * 72, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return SED_OK;
}

int sed_initialize_particles(sed_ctx* c, int64_t n, const double* e_rad)
{
  if (!c) return SED_ERR_ARG;
  c->have_diff = false;  // the last weighted forward no longer matches the context
  if (!c->have_grid) return set_err(c, SED_ERR_STATE, "sed_initialize_particles: no grid");
  if (n < 0 || (n > 0 && !e_rad)) return set_err(c, SED_ERR_ARG, "sed_initialize_particles: bad arguments");
  if (n == 0) return SED_OK;
  // emission.cpp:122-125: the packets must fit on their own
  if (n > c->tp.max_particles)
    return set_err(c, SED_ERR_CAPACITY, "Not enough particle space to initialize %lld packets", (long long)n);
  const int64_t off = c->n_census;
  const size_t nz = (size_t)c->nz, nn = (size_t)c->nu.n();
  // the census grows to off + n packets; what it held is kept
  DevBuf<double> st;
  DevBuf<int32_t> ind, typ;
  CK(st.resize((size_t)(off + n) * 9)); CK(ind.resize((size_t)(off + n))); CK(typ.resize((size_t)(off + n)));
  if (off > 0) {
    CK(cudaMemcpyAsync(st.p, c->d_census_state.p, (size_t)off * 72, cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(ind.p, c->d_census_ind.p, (size_t)off * 4, cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(typ.p, c->d_census_type.p, (size_t)off * 4, cudaMemcpyDeviceToDevice, c->stream));
  }
  DevBuf<double> erad, zcdf, esum, bb;
  CK(upload(c, erad, e_rad, nz));
  CK(zcdf.resize(nz)); CK(esum.resize(1)); CK(bb.resize(nz * nn));
  InitArgs I{};
  I.n = n; I.census_off = off; I.seed = c->tp.rng_seed; I.first_pid = c->tp.first_packet_id + off;
  I.t_now = c->t_now; I.nz = c->nz;
  I.e_rad = erad.p; I.vol = c->d_vol.p; I.T = c->d_T.p;
  I.zone_cdf = zcdf.p; I.E_sum = esum.p; I.bb_cdf = bb.p;
  I.nu = dev_loc(c->nu, c->d_nu);
  I.census_state = st.p; I.census_ind = ind.p; I.census_type = typ.p;
  launch_init_particles(I, make_grid_dev(c), c->stream);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));
  std::swap(c->d_census_state, st); std::swap(c->d_census_ind, ind); std::swap(c->d_census_type, typ);
  st.release(); ind.release(); typ.release(); erad.release(); zcdf.release(); esum.release(); bb.release();
  c->n_census = off + n;
  return SED_OK;
}

const char* sed_last_error(sed_ctx* c) { return c ? c->err.c_str() : "null context"; }

void sed_ctx_destroy(sed_ctx* c)
{
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (auto& ev : c->ev) if (ev) cudaEventDestroy(ev);
  DevBuf<double>* dbl[] = {&c->d_nu, &c->d_st, &c->d_sn, &c->d_sm, &c->d_sp, &c->d_core_cdf, &c->d_r_out, &c->d_v_r,
                           &c->d_ax[0], &c->d_ax[1], &c->d_ax[2], &c->d_vol, &c->d_rho, &c->d_T, &c->d_egas,
                           &c->d_grey, &c->d_X, &c->d_ion_chi, &c->d_lev_E, &c->d_lev_Eion, &c->d_photo_E,
                           &c->d_photo_s, &c->d_fz_h,
                           &c->d_eps_imc, &c->d_abs64, &c->d_scat64, &c->d_emis64, &c->d_epsl64, &c->d_epsf64, &c->d_planck, &c->d_ross, &c->d_L,
                           &c->d_n_elec, &c->d_n_dens, &c->d_mass_frac, &c->d_temp_c, &c->d_ion_part, &c->d_ion_frac,
                           &c->d_lev_n, &c->d_boltz, &c->d_J, &c->d_e_abs, &c->d_e_rad, &c->d_fx, &c->d_fy,
                           &c->d_fz, &c->d_fr, &c->d_flux, &c->d_click, &c->d_rec_state,
                           &c->d_esc_e, &c->d_abs_scale, &c->d_adj_g, &c->d_adj_out};
  for (auto* b : dbl) b->release();
  DevBuf<int32_t>* ints[] = {&c->d_eZ, &c->d_eA, &c->d_zero_eps_atom, &c->d_ion_off, &c->d_lev_off, &c->d_lev_ion,
                             &c->d_lev_g, &c->d_lev_ic, &c->d_photo_off, &c->d_ion_atom, &c->d_ln_seg,
                             &c->d_fz_seg, &c->d_lev_atom, &c->d_ln_order, &c->d_fz_order, &c->d_solve_err, &c->d_rec_fate, &c->d_rec_ind, &c->d_rec_draws,
                             &c->d_esc_bin};
  for (auto* b : ints) b->release();
  c->d_ln_lv.release(); c->d_ln_c.release(); c->d_ln_c32.release(); c->d_fz_ia.release(); c->d_fz_c.release();
  c->d_fz_c32.release();
  c->d_opac.release(); c->d_cdf.release(); c->d_cdf_coarse.release(); c->d_counters.release();
  c->d_cdf_guide.release();
  c->d_temp_bad.release();
  DevBuf<double>* rad[] = {&c->d_gn, &c->d_gflux, &c->d_gclick, &c->d_radio_cdf, &c->d_gamma_frac, &c->d_compton,
                           &c->d_photoion, &c->d_L_emit, &c->d_L_dep, &c->d_L_tot, &c->d_q_state};
  for (auto* b : rad) b->release();
  c->d_q_ind.release(); c->d_reject.release(); c->d_q_n.release();
  c->d_rec_type.release(); c->d_census_state.release(); c->d_census_ind.release(); c->d_census_type.release();
  c->d_q_type.release(); c->d_cmp.release(); c->d_scan_tmp.release(); c->d_cmp_count.release();
  c->d_rho_scale.release(); c->d_opac_base.release(); c->d_imd_p.release(); c->d_zone_rep.release();
  c->d_em_state.release(); c->d_em_ind.release(); c->d_em_tau.release();
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

}  // extern "C"
