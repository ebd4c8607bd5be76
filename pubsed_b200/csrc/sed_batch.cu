// sed_batch.cu -- many independent 1D models stepped as one (sed_batch_* in
// include/sedona_gpu.h).
//
// The zones of all models are concatenated into one inner sed_ctx, so the
// opacity build (LTE solve, line sums, tables) runs once over every zone of
// the batch, and the zone tallies (J_nu, e_abs, ...) live in that context's
// arrays.  The packet queue spans every packet of every model: one launch of
// the batched packet kernel propagates them all, each thread finding its
// packet's model from the queue index.  The whole step is captured once
// into three CUDA graphs replayed back to back -- tally wipes + opacity
// build, the packet kernel, rescale + normalisation -- with the timing events
// recorded between them; the Philox step number lives on the device and is
// advanced by the last kernel, so replays need no parameter updates.  Launch shape and queue chunk come from a small autotuner that
// times the kernel on a sample of every model's packets.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "sed_ctx.h"

using namespace sed;

struct sed_batch {
  sed_ctx* inner = nullptr;  // concatenated zones
  std::string err;
  int n_models = 0;
  std::vector<BatchModel> models;       // host copy (Ep for the current dt)
  std::vector<double> L_core;           // per-model core luminosity
  int64_t total_packets = 0;
  int64_t nspec = 0;
  DevBuf<BatchModel> d_models, d_sample_models;
  DevBuf<int4> d_nbr;
  DevBuf<double> d_rin, d_core_cdf, d_flux, d_click;
  DevBuf<double2> d_wall;
  DevBuf<unsigned long long> d_model_esc;
  DevBuf<uint32_t> d_step;
  DevBuf<double> d_zone_rep;            // copies of the zone-scalar tallies (many zones)
  int n_rep = 0;
  double models_dt = -1;                // dt the device model table was written for
  // launch shape
  int variant = 0, blocks_per_sm = 0, queue_chunk = 1;
  // graph
  bool use_graph = true;
  bool stepped = false;                 // a step has run eagerly (kernel attributes set, buffers sized)
  cudaGraphExec_t exec[3] = {};         // wipe + opacity, packet kernel, finish
  double graph_dt = -1;
  cudaEvent_t ev[5] = {};
  // records
  int record = 0;
  DevBuf<int32_t> d_rec_fate, d_rec_ind, d_rec_draws;
  DevBuf<double> d_rec_state;
  // packets emitted ahead of the mixed-form kernel (state [9][n], zone, first depth, model)
  DevBuf<double> d_em_state;
  DevBuf<int32_t> d_em_ind, d_em_model;
  DevBuf<float> d_em_tau;
};

namespace {

int bset_err(sed_batch* b, int code, const char* fmt, ...)
{
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (b) b->err = buf;
  return code;
}

#define BCK(call)                                                                                       \
  do {                                                                                                  \
    cudaError_t e_ = (call);                                                                            \
    if (e_ != cudaSuccess)                                                                              \
      return bset_err(b, e_ == cudaErrorMemoryAllocation ? SED_ERR_NOMEM : SED_ERR_CUDA, "%s: %s (%s:%d)", \
                      #call, cudaGetErrorString(e_), __FILE__, __LINE__);                               \
  } while (0)

// inner-context failures carry their message into the batch
int from_inner(sed_batch* b, int rc)
{
  if (rc != SED_OK) b->err = b->inner->err;
  return rc;
}

// milliseconds between two completed events, -1 when they cannot be timed
float elapsed(cudaEvent_t a, cudaEvent_t z)
{
  float ms = 0;
  if (cudaEventElapsedTime(&ms, a, z) != cudaSuccess) {
    (void)cudaGetLastError();
    return -1.f;
  }
  return ms;
}

void drop_graph(sed_batch* b)
{
  for (auto& x : b->exec) {
    if (x) cudaGraphExecDestroy(x);
    x = nullptr;
  }
  b->graph_dt = -1;
}

// packet energy of each model for this dt (emission.cpp:383-392) and the
// device copy of the model table
int write_models(sed_batch* b, double dt)
{
  if (dt == b->models_dt) return SED_OK;
  for (int m = 0; m < b->n_models; ++m) {
    const int64_t n = b->models[m].n_packets;
    b->models[m].Ep = n > 0 ? b->L_core[m] * dt / n : 0.0;
  }
  sed_ctx* c = b->inner;
  BCK(cudaMemcpyAsync(b->d_models.p, b->models.data(), b->models.size() * sizeof(BatchModel), cudaMemcpyHostToDevice,
                      c->stream));
  BCK(cudaStreamSynchronize(c->stream));
  b->models_dt = dt;
  return SED_OK;
}

StepArgs step_args(sed_batch* b, double dt, const BatchModel* models, int64_t total)
{
  sed_ctx* c = b->inner;
  StepArgs A{};
  A.steady = c->tp.steady_state; A.radiative_eq = c->tp.radiative_eq;
  A.bound_in_reflect = c->tp.boundary_in_reflect; A.bound_out_reflect = c->tp.boundary_out_reflect;
  A.store_Jnu = c->tp.store_Jnu; A.omit_scat = c->tp.omit_scattering; A.tally_forces = c->tp.tally_forces;
  A.precision = c->tp.precision;
  A.n_packets = total;
  A.t_now = c->t_grid; A.dt = dt; A.tstop = c->t_grid + dt;
  if (c->t_grid > 0) {
    A.inv_t = 1.0 / c->t_grid;
    A.ct = C_LIGHT * c->t_grid;
    A.inv_ct = 1.0 / A.ct;
    A.inv_ct2 = A.inv_ct * A.inv_ct;
  }
  A.core_freq = c->tp.core_photon_frequency;
  A.max_segments = c->tp.max_segments;
  A.smem_zones = ((size_t)5 * c->nz * sizeof(double) <= 64 * 1024) ? 1 : 0;
  A.nu = dev_loc(c->nu, c->d_nu); A.st = dev_loc(c->st, c->d_st); A.sn = dev_loc(c->sn, c->d_sn);
  A.sm = dev_loc(c->sm, c->d_sm); A.sp = dev_loc(c->sp, c->d_sp);
  A.a3 = c->sp.n(); A.a2 = (int64_t)c->sm.n() * A.a3; A.a1 = (int64_t)c->sn.n() * A.a2;
  A.opac = c->d_opac.p; A.cdf = c->d_cdf.p; A.eps_imc = c->d_eps_imc.p;
  A.cdf_coarse = c->d_cdf_coarse.p; A.n_coarse = c->n_coarse;
  A.cdf_guide = c->guide_n ? c->d_cdf_guide.p : nullptr; A.guide_n = c->guide_n;
  A.rescale_lum = c->tp.core_fix_luminosity;
  A.J = c->d_J.p; A.e_abs = c->d_e_abs.p; A.e_rad = c->d_e_rad.p;
  A.fx = c->d_fx.p; A.fy = c->d_fy.p; A.fz = c->d_fz.p; A.fr = c->d_fr.p;
  A.flux = b->d_flux.p; A.click = b->d_click.p; A.counters = c->d_counters.p;
  A.models = models; A.n_models = b->n_models; A.queue_chunk = std::max(1, b->queue_chunk);
  A.zone_nbr = b->d_nbr.p; A.zone_rin = b->d_rin.p; A.zone_wall = b->d_wall.p;
  A.model_escaped = b->d_model_esc.p; A.step_dev = b->d_step.p;
  A.n_rep = A.smem_zones ? 0 : b->n_rep;
  A.zone_rep = b->d_zone_rep.p;
  if (b->d_em_state.p) {  // the mixed form emits every queue entry ahead of the packet kernel
    A.em_state = b->d_em_state.p; A.em_ind = b->d_em_ind.p; A.em_tau = b->d_em_tau.p;
    A.em_model = b->d_em_model.p; A.em_n = total;
  }
  return A;
}

GridDev grid_dev(sed_batch* b)
{
  sed_ctx* c = b->inner;
  GridDev G{};
  G.type = SED_GRID_1D_SPHERE; G.nzones = c->nz; G.homologous = 1; G.t_grid = c->t_grid;
  G.r_out = dev_loc(c->r_out, c->d_r_out);
  G.v_r = nullptr;
  return G;
}

int wipe(sed_batch* b)
{
  sed_ctx* c = b->inner;
  const size_t nz = (size_t)c->nz, nj = c->tp.store_Jnu ? (size_t)c->nu.n() : 1;
  cudaStream_t s = c->stream;
  // wipe_radiation (src/transport/transport_mpi.cpp:18-34) of every model
  BCK(cudaMemsetAsync(c->d_J.p, 0, nz * nj * sizeof(double), s));
  double* z[6] = {c->d_e_abs.p, c->d_e_rad.p, c->d_fx.p, c->d_fy.p, c->d_fz.p, c->d_fr.p};
  for (double* p : z) BCK(cudaMemsetAsync(p, 0, nz * sizeof(double), s));
  BCK(cudaMemsetAsync(b->d_flux.p, 0, b->d_flux.n * sizeof(double), s));
  BCK(cudaMemsetAsync(b->d_click.p, 0, b->d_click.n * sizeof(double), s));
  BCK(cudaMemsetAsync(c->d_counters.p, 0, (C_COUNT + 1) * sizeof(unsigned long long), s));
  BCK(cudaMemsetAsync(b->d_model_esc.p, 0, b->d_model_esc.n * sizeof(unsigned long long), s));
  if (b->n_rep) BCK(cudaMemsetAsync(b->d_zone_rep.p, 0, b->d_zone_rep.n * sizeof(double), s));
  return SED_OK;
}

// Queues one part of a step on the inner stream with no host
// synchronisation, so it can be captured: 0 = wipe + opacity build,
// 1 = packet kernel, 2 = rescale / normalisation / step counter.
int enqueue_part(sed_batch* b, double dt, int part)
{
  sed_ctx* c = b->inner;
  cudaStream_t s = c->stream;
  if (part == 0) {
    int rc = wipe(b);
    if (rc) return rc;
    rc = enqueue_opacity(c, dt);
    return rc ? from_inner(b, rc) : SED_OK;
  }
  StepArgs A = step_args(b, dt, b->d_models.p, b->total_packets);
  if (b->record) {
    A.rec_fate = b->d_rec_fate.p; A.rec_ind = b->d_rec_ind.p; A.rec_draws = b->d_rec_draws.p;
    A.rec_state = b->d_rec_state.p;
  }
  if (part == 1) {
    if (b->total_packets > 0)
      launch_propagate_batch(A, grid_dev(b), b->variant, b->blocks_per_sm, c->num_sms, b->total_packets, s);
  } else {
    launch_finish_batch(A, c->d_vol.p, c->nz, b->nspec, s);
  }
  BCK(cudaGetLastError());
  return SED_OK;
}

int check_model(const sed_batch_model& m, int n_elems)
{
  if (m.n_zones <= 0 || !m.r_out || !m.vol || !m.rho || !m.T_gas) return 1;
  if (n_elems > 0 && !m.X) return 1;
  if (m.core_n_emit < 0) return 1;
  for (int i = 0; i < m.n_zones; ++i)
    if (!(m.r_out[i] > (i ? m.r_out[i - 1] : m.r_min))) return 2;
  return 0;
}

}  // namespace

extern "C" {

int sed_batch_create(const sed_transport_params* common, double t_now, int32_t n_elems, const int32_t* elem_Z,
                     const int32_t* elem_A, int32_t n_models, const sed_batch_model* models, int device,
                     sed_batch** out)
{
  if (!common || !out || n_models <= 0 || !models || n_elems < 0 || (n_elems > 0 && (!elem_Z || !elem_A)))
    return SED_ERR_ARG;
  *out = nullptr;
  for (int m = 0; m < n_models; ++m)
    if (check_model(models[m], n_elems)) return SED_ERR_ARG;
  sed_batch* b = new sed_batch();
  b->n_models = n_models;
  int rc = sed_ctx_create(common, device, &b->inner);
  if (rc) { delete b; return rc; }
  sed_ctx* c = b->inner;
  // concatenated zone arrays: the inner context's grid
  std::vector<double> r_out, vol, rho, T, eg, grey, X;
  std::vector<int4> nbr;
  std::vector<double> rin;
  std::vector<double2> wall;
  int64_t nz_tot = 0;
  for (int m = 0; m < n_models; ++m) nz_tot += models[m].n_zones;
  if (nz_tot > INT32_MAX / 2) { sed_ctx_destroy(b->inner); delete b; return SED_ERR_ARG; }
  r_out.reserve(nz_tot); nbr.reserve(nz_tot); rin.reserve(nz_tot); wall.reserve(nz_tot);
  b->models.resize(n_models);
  b->L_core.resize(n_models);
  const int nn = c->nu.n();
  std::vector<double> core_cdf((size_t)n_models * nn);
  int64_t pkt = 0;
  int zo = 0;
  const int64_t nspec = (int64_t)c->st.n() * c->sn.n() * c->sm.n() * c->sp.n();
  b->nspec = nspec;
  for (int m = 0; m < n_models; ++m) {
    const sed_batch_model& M = models[m];
    const int nz = M.n_zones;
    // emit_inner_source packet count (emission.cpp:383-392), one rank
    const int64_t n_emit = (int64_t)(M.core_n_emit / 1.0);
    if (n_emit > common->max_particles) {
      b->err = "Not enough particle space";
      sed_ctx_destroy(b->inner); delete b;
      return SED_ERR_CAPACITY;
    }
    for (int i = 0; i < nz; ++i) {
      const int g = zo + i;
      r_out.push_back(M.r_out[i]);
      vol.push_back(M.vol[i]);
      rho.push_back(M.rho[i]);
      T.push_back(M.T_gas[i]);
      eg.push_back(M.e_gas ? M.e_gas[i] : 0.0);
      grey.push_back(M.total_grey_opacity ? M.total_grey_opacity[i] : 0.0);
      for (int k = 0; k < n_elems; ++k) X.push_back(M.X[(size_t)i * n_elems + k]);
      // grid_1D_sphere::get_next_zone's inner wall and neighbours
      // (grid_1D_sphere.cpp:527-546) with this model's r_min and core
      double r_in = (i != 0) ? M.r_out[i - 1] : M.r_min;
      int ind_in = (i != 0) ? g - 1 : -1;
      if (M.core_radius >= r_in) { r_in = M.core_radius; ind_in = -1; }
      const int no_inner = ((i == 0) && (r_in == 0)) ? 1 : 0;
      const int outer = (i + 1 == nz) ? -2 : g + 1;
      nbr.push_back(make_int4(ind_in, outer, no_inner, m));
      rin.push_back(r_in);
      wall.push_back(make_double2(outer == -2 ? -M.r_out[i] : M.r_out[i], ind_in == -1 ? -r_in : r_in));
    }
    BatchModel& D = b->models[m];
    D.pkt_off = pkt;
    D.n_packets = n_emit;
    D.first_pid = M.first_packet_id;
    D.spec_off = (int64_t)m * nspec;
    D.zone_off = zo;
    D.n_zones = nz;
    D.seed = M.rng_seed;
    D.emit_draws = (M.core_radius == 0 ? 2u : 4u) + (common->core_photon_frequency > 0 ? 0u : 2u) + 1u;
    D.r_min = M.r_min;
    D.core_radius = M.core_radius;
    D.Ep = 0;
    b->L_core[m] = M.core_luminosity;
    const std::vector<double> cd = core_emission_cdf(c->nu, M.core_temperature);
    std::copy(cd.begin(), cd.end(), core_cdf.begin() + (size_t)m * nn);
    pkt += n_emit;
    zo += nz;
  }
  b->total_packets = pkt;
  sed_grid g{};
  g.type = SED_GRID_1D_SPHERE;
  g.n_zones = (int32_t)nz_tot;
  g.homologous = 1;
  g.n_elems = n_elems;
  g.t_now = t_now;
  g.r_min = models[0].r_min;
  g.r_out = r_out.data();
  g.vol = vol.data(); g.rho = rho.data(); g.T_gas = T.data(); g.e_gas = eg.data();
  g.total_grey_opacity = grey.data(); g.X = X.empty() ? nullptr : X.data();
  g.elem_Z = elem_Z; g.elem_A = elem_A;
  rc = sed_set_grid(c, &g);
  if (rc) { b->err = c->err; sed_ctx_destroy(c); delete b; return rc; }
  auto fail = [&](cudaError_t e) {
    sed_ctx_destroy(b->inner);
    delete b;
    return e == cudaErrorMemoryAllocation ? SED_ERR_NOMEM : SED_ERR_CUDA;
  };
  cudaError_t e;
  if ((e = upload(c, b->d_nbr, nbr.data(), nbr.size())) != cudaSuccess) return fail(e);
  if ((e = upload(c, b->d_rin, rin.data(), rin.size())) != cudaSuccess) return fail(e);
  if ((e = upload(c, b->d_wall, wall.data(), wall.size())) != cudaSuccess) return fail(e);
  if ((e = upload(c, b->d_core_cdf, core_cdf.data(), core_cdf.size())) != cudaSuccess) return fail(e);
  for (int m = 0; m < n_models; ++m) b->models[m].core_cdf = b->d_core_cdf.p + (size_t)m * nn;
  if ((e = b->d_models.resize(n_models)) != cudaSuccess) return fail(e);
  if ((e = b->d_flux.resize((size_t)n_models * nspec)) != cudaSuccess) return fail(e);
  if ((e = b->d_click.resize((size_t)n_models * nspec)) != cudaSuccess) return fail(e);
  if ((e = b->d_model_esc.resize(n_models)) != cudaSuccess) return fail(e);
  if ((e = b->d_step.resize(1)) != cudaSuccess) return fail(e);
  if (c->tp.precision != 0 && pkt > 0) {  // the mixed form emits its packets ahead of the packet kernel
    if ((e = b->d_em_state.resize((size_t)pkt * 9)) != cudaSuccess) return fail(e);
    if ((e = b->d_em_ind.resize((size_t)pkt)) != cudaSuccess) return fail(e);
    if ((e = b->d_em_tau.resize((size_t)pkt)) != cudaSuccess) return fail(e);
    if ((e = b->d_em_model.resize((size_t)pkt)) != cudaSuccess) return fail(e);
  }
  // zones beyond the per-block shared-memory tallies: 128 copies of the
  // zone-scalar tallies (fewer if that would pass 256 MiB).  A batch's
  // packets are drawn model by model, so the lanes in flight crowd onto the
  // few hundred zones of one or two models and visit each for ~1.2 segments;
  // with 32 copies their reductions queued on the same addresses (64-model
  // batch at half its packets: packet kernel 723 ms with 32 copies, 640 ms
  // with 128, 640 ms with 256 or 512)
  if ((size_t)5 * nz_tot * sizeof(double) > 64 * 1024) {
    b->n_rep = (int)std::min<size_t>(128, std::max<size_t>(1, (size_t(256) << 20) / (5 * sizeof(double) * nz_tot)));
    if ((e = b->d_zone_rep.resize((size_t)b->n_rep * 5 * nz_tot)) != cudaSuccess) return fail(e);
  }
  if ((e = cudaMemsetAsync(b->d_step.p, 0, sizeof(uint32_t), c->stream)) != cudaSuccess) return fail(e);
  if ((e = cudaMemsetAsync(b->d_flux.p, 0, b->d_flux.n * sizeof(double), c->stream)) != cudaSuccess) return fail(e);
  if ((e = cudaMemsetAsync(b->d_click.p, 0, b->d_click.n * sizeof(double), c->stream)) != cudaSuccess) return fail(e);
  for (auto& ev : b->ev)
    if ((e = cudaEventCreate(&ev)) != cudaSuccess) return fail(e);
  if ((e = cudaStreamSynchronize(c->stream)) != cudaSuccess) return fail(e);
  *out = b;
  return SED_OK;
}

int sed_batch_set_opacity_params(sed_batch* b, const sed_opacity_params* op)
{
  if (!b) return SED_ERR_ARG;
  drop_graph(b);
  b->stepped = false;
  return from_inner(b, sed_set_opacity_params(b->inner, op));
}

int sed_batch_set_atomic_data(sed_batch* b, const sed_atomic_data* atoms)
{
  if (!b) return SED_ERR_ARG;
  drop_graph(b);
  b->stepped = false;
  return from_inner(b, sed_set_atomic_data(b->inner, atoms));
}

int sed_batch_set_tuning(sed_batch* b, const sed_batch_tuning* t)
{
  if (!b || !t || t->variant < 0 || t->variant >= BATCH_VARIANTS || t->blocks_per_sm < 0 || t->queue_chunk < 1)
    return SED_ERR_ARG;
  b->variant = t->variant;
  b->blocks_per_sm = t->blocks_per_sm;
  b->queue_chunk = t->queue_chunk;
  drop_graph(b);
  return SED_OK;
}

int sed_batch_use_graph(sed_batch* b, int32_t enable)
{
  if (!b) return SED_ERR_ARG;
  b->use_graph = enable != 0;
  if (!b->use_graph) drop_graph(b);
  return SED_OK;
}

int sed_batch_autotune(sed_batch* b, double frac, sed_batch_tuning* best)
{
  if (!b || !(frac > 0) || frac > 1) return SED_ERR_ARG;
  sed_ctx* c = b->inner;
  const double dt = (c->tp.steady_state || !(b->models_dt > 0)) ? 1.0 : b->models_dt;
  if (!c->have_opacity) {
    int rc = sed_set_opacity(c, dt);
    if (rc) return from_inner(b, rc);
  }
  int rc = write_models(b, dt);
  if (rc) return rc;
  // the sample: the first ceil(frac * n) packets of every model, same
  // sources, keys and stream ids
  std::vector<BatchModel> sm = b->models;
  int64_t tot = 0;
  for (auto& m : sm) {
    const int64_t n = m.n_packets > 0 ? std::max<int64_t>(1, (int64_t)std::ceil(frac * (double)m.n_packets)) : 0;
    m.pkt_off = tot;
    m.n_packets = n;
    tot += n;
  }
  BCK(b->d_sample_models.resize(sm.size()));
  BCK(cudaMemcpyAsync(b->d_sample_models.p, sm.data(), sm.size() * sizeof(BatchModel), cudaMemcpyHostToDevice,
                      c->stream));
  const int chunks[3] = {1, 4, 16};
  float best_ms = 1e30f;
  int bv = 0, bc = 1, tried = 0;
  const GridDev G = grid_dev(b);
  for (int warm = 1; warm >= 0; --warm) {
    for (int v = 0; v < BATCH_VARIANTS; ++v) {
      for (int q : chunks) {
        if (warm && (v > 0 || q != 1)) continue;
        const int save_chunk = b->queue_chunk;
        b->queue_chunk = q;
        StepArgs A = step_args(b, b->models_dt, b->d_sample_models.p, tot);
        b->queue_chunk = save_chunk;
        BCK(cudaMemsetAsync(c->d_counters.p, 0, (C_COUNT + 1) * sizeof(unsigned long long), c->stream));
        BCK(cudaMemsetAsync(b->d_model_esc.p, 0, b->d_model_esc.n * sizeof(unsigned long long), c->stream));
        BCK(cudaEventRecord(b->ev[2], c->stream));
        launch_propagate_batch(A, G, v, 0, c->num_sms, tot, c->stream);
        BCK(cudaGetLastError());
        BCK(cudaEventRecord(b->ev[3], c->stream));
        BCK(cudaStreamSynchronize(c->stream));
        float ms = 0;
        BCK(cudaEventElapsedTime(&ms, b->ev[2], b->ev[3]));
        if (warm) continue;
        ++tried;
        if (ms < best_ms) { best_ms = ms; bv = v; bc = q; }
      }
    }
  }
  b->variant = bv;
  b->blocks_per_sm = 0;
  b->queue_chunk = bc;
  drop_graph(b);
  if (best) {
    best->variant = bv;
    int th = 0, mb = 0;
    batch_variant_shape(bv, &th, &mb);
    best->threads = th;
    best->blocks_per_sm = 0;
    best->queue_chunk = bc;
    best->ms = best_ms;
    best->n_tried = tried;
  }
  return SED_OK;
}

int sed_batch_step(sed_batch* b, double dt, sed_step_stats* st)
{
  if (!b) return SED_ERR_ARG;
  sed_ctx* c = b->inner;
  if (c->tp.steady_state) dt = 1;
  int rc = write_models(b, dt);
  if (rc) return rc;
  if (b->record) {
    const size_t n = (size_t)std::max<int64_t>(b->total_packets, 1);
    BCK(b->d_rec_fate.resize(n)); BCK(b->d_rec_ind.resize(n)); BCK(b->d_rec_draws.resize(n));
    BCK(b->d_rec_state.resize(n * 9));
  }
  // One graph per part, so the timing events sit between graph launches
  // (events recorded inside a capture cannot be timed).
  const bool graph = b->use_graph && b->stepped;
  if (graph && (!b->exec[0] || b->graph_dt != dt)) {
    drop_graph(b);
    for (int part = 0; part < 3; ++part) {
      cudaGraph_t g = nullptr;
      BCK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
      rc = enqueue_part(b, dt, part);
      cudaError_t e = cudaStreamEndCapture(c->stream, &g);
      if (rc) { if (g) cudaGraphDestroy(g); drop_graph(b); return rc; }
      if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec[part], g, 0);
      if (g) cudaGraphDestroy(g);
      if (e != cudaSuccess) { drop_graph(b); BCK(e); }
    }
    b->graph_dt = dt;
  }
  const int ev_at[3][2] = {{0, 1}, {2, 3}, {3, 4}};
  for (int part = 0; part < 3; ++part) {
    if (part != 2) BCK(cudaEventRecord(b->ev[ev_at[part][0]], c->stream));
    if (graph) BCK(cudaGraphLaunch(b->exec[part], c->stream));
    else {
      rc = enqueue_part(b, dt, part);
      if (rc) return rc;
    }
    BCK(cudaEventRecord(b->ev[ev_at[part][1]], c->stream));
  }
  unsigned long long cnt[C_COUNT + 1];
  BCK(cudaMemcpyAsync(cnt, c->d_counters.p, sizeof cnt, cudaMemcpyDeviceToHost, c->stream));
  BCK(cudaStreamSynchronize(c->stream));
  b->stepped = true;
  c->have_opacity = true;
  if (st) {
    std::memset(st, 0, sizeof *st);
    st->n_packets = b->total_packets;
    st->n_escaped = (int64_t)cnt[C_ESCAPED];
    st->n_absorbed = (int64_t)cnt[C_ABSORBED];
    st->n_stopped = (int64_t)cnt[C_STOPPED];
    st->n_segments = (int64_t)cnt[C_SEGMENTS];
    st->n_scatters = (int64_t)cnt[C_SCATTERS];
    st->n_limit = (int64_t)cnt[C_LIMIT];
    st->kernel_launches = c->opacity_launches + (b->total_packets > 0 ? 1 : 0) +
                          ((c->tp.steady_state && c->tp.core_fix_luminosity) ? 2 : 1);
    st->ms_opacity = elapsed(b->ev[0], b->ev[1]);
    st->ms_propagate_kernel = elapsed(b->ev[2], b->ev[3]);
    st->ms_transport = elapsed(b->ev[1], b->ev[4]);
    st->ms_total = elapsed(b->ev[0], b->ev[4]);
  }
  if (cnt[C_LIMIT] > 0) return bset_err(b, SED_ERR_LIMIT, "%llu packets hit the segment limit", cnt[C_LIMIT]);
  return SED_OK;
}

int sed_batch_set_zone_state(sed_batch* b, int32_t m, const double* rho, const double* T)
{
  if (!b) return SED_ERR_ARG;
  if (m < 0 || m >= b->n_models) return bset_err(b, SED_ERR_ARG, "model %d out of range", m);
  sed_ctx* c = b->inner;
  const size_t zo = (size_t)b->models[m].zone_off, nz = (size_t)b->models[m].n_zones;
  if (rho) BCK(cudaMemcpyAsync(c->d_rho.p + zo, rho, nz * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  if (T) BCK(cudaMemcpyAsync(c->d_T.p + zo, T, nz * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  BCK(cudaStreamSynchronize(c->stream));
  return SED_OK;
}

int sed_batch_get_escaped(sed_batch* b, int64_t* n_escaped)
{
  if (!b || !n_escaped) return SED_ERR_ARG;
  std::vector<unsigned long long> v(b->n_models);
  BCK(cudaMemcpyAsync(v.data(), b->d_model_esc.p, v.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                      b->inner->stream));
  BCK(cudaStreamSynchronize(b->inner->stream));
  for (int m = 0; m < b->n_models; ++m) n_escaped[m] = (int64_t)v[m];
  return SED_OK;
}

int sed_batch_get_spectrum(sed_batch* b, int32_t m, double* flux, double* click)
{
  if (!b) return SED_ERR_ARG;
  if (m < 0 || m >= b->n_models) return bset_err(b, SED_ERR_ARG, "model %d out of range", m);
  cudaStream_t s = b->inner->stream;
  const size_t o = (size_t)m * b->nspec, n = (size_t)b->nspec * sizeof(double);
  if (flux) BCK(cudaMemcpyAsync(flux, b->d_flux.p + o, n, cudaMemcpyDeviceToHost, s));
  if (click) BCK(cudaMemcpyAsync(click, b->d_click.p + o, n, cudaMemcpyDeviceToHost, s));
  BCK(cudaStreamSynchronize(s));
  return SED_OK;
}

int sed_batch_get_zone_tallies(sed_batch* b, int32_t m, double* J, double* e_abs, double* e_rad, double* fx,
                               double* fy, double* fz, double* fr)
{
  if (!b) return SED_ERR_ARG;
  if (m < 0 || m >= b->n_models) return bset_err(b, SED_ERR_ARG, "model %d out of range", m);
  sed_ctx* c = b->inner;
  const size_t zo = (size_t)b->models[m].zone_off, nz = (size_t)b->models[m].n_zones;
  const size_t nj = c->tp.store_Jnu ? (size_t)c->nu.n() : 1;
  if (J) BCK(cudaMemcpyAsync(J, c->d_J.p + zo * nj, nz * nj * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  struct { double* h; double* d; } z[6] = {{e_abs, c->d_e_abs.p}, {e_rad, c->d_e_rad.p}, {fx, c->d_fx.p},
                                           {fy, c->d_fy.p}, {fz, c->d_fz.p}, {fr, c->d_fr.p}};
  for (auto& q : z)
    if (q.h) BCK(cudaMemcpyAsync(q.h, q.d + zo, nz * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  BCK(cudaStreamSynchronize(c->stream));
  return SED_OK;
}

int sed_batch_get_opacity(sed_batch* b, int32_t m, double* abs, double* scat, double* cdf, double* n_elec,
                          double* eps_imc)
{
  if (!b) return SED_ERR_ARG;
  if (m < 0 || m >= b->n_models) return bset_err(b, SED_ERR_ARG, "model %d out of range", m);
  sed_ctx* c = b->inner;
  if (!c->have_opacity) return bset_err(b, SED_ERR_STATE, "no opacity tables");
  const size_t zo = (size_t)b->models[m].zone_off, nz = (size_t)b->models[m].n_zones, nn = (size_t)c->nu.n();
  const size_t n = nz * nn, esz = c->tp.precision ? sizeof(float) : sizeof(double);
  std::vector<unsigned char> o(2 * n * esz), cd(n * esz);
  BCK(cudaMemcpyAsync(o.data(), c->d_opac.p + zo * nn * 2 * esz, o.size(), cudaMemcpyDeviceToHost, c->stream));
  BCK(cudaMemcpyAsync(cd.data(), c->d_cdf.p + zo * nn * esz, cd.size(), cudaMemcpyDeviceToHost, c->stream));
  if (n_elec) BCK(cudaMemcpyAsync(n_elec, c->d_n_elec.p + zo, nz * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  if (eps_imc)
    BCK(cudaMemcpyAsync(eps_imc, c->d_eps_imc.p + zo, nz * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  BCK(cudaStreamSynchronize(c->stream));
  for (size_t i = 0; i < n; ++i) {
    double a, s, q;
    if (c->tp.precision) {
      const float* f = reinterpret_cast<const float*>(o.data());
      a = f[2 * i]; s = f[2 * i + 1]; q = reinterpret_cast<const float*>(cd.data())[i];
    } else {
      const double* f = reinterpret_cast<const double*>(o.data());
      a = f[2 * i]; s = f[2 * i + 1]; q = reinterpret_cast<const double*>(cd.data())[i];
    }
    if (abs) abs[i] = a;
    if (scat) scat[i] = s;
    if (cdf) cdf[i] = q;
  }
  return SED_OK;
}

int sed_batch_record_packets(sed_batch* b, int32_t enable)
{
  if (!b) return SED_ERR_ARG;
  if ((enable != 0) != (b->record != 0)) drop_graph(b);
  b->record = enable ? 1 : 0;
  return SED_OK;
}

int sed_batch_get_packet_records(sed_batch* b, int32_t m, int64_t n, int32_t* fate, int32_t* ind, int32_t* draws,
                                 double* state9)
{
  if (!b) return SED_ERR_ARG;
  if (m < 0 || m >= b->n_models) return bset_err(b, SED_ERR_ARG, "model %d out of range", m);
  const BatchModel& M = b->models[m];
  if (!b->record || !b->d_rec_fate.p || n < 0 || n > M.n_packets)
    return bset_err(b, SED_ERR_STATE, "no packet records for %lld packets of model %d", (long long)n, m);
  cudaStream_t s = b->inner->stream;
  const size_t o = (size_t)M.pkt_off;
  if (fate) BCK(cudaMemcpyAsync(fate, b->d_rec_fate.p + o, n * 4, cudaMemcpyDeviceToHost, s));
  if (ind) BCK(cudaMemcpyAsync(ind, b->d_rec_ind.p + o, n * 4, cudaMemcpyDeviceToHost, s));
  if (draws) BCK(cudaMemcpyAsync(draws, b->d_rec_draws.p + o, n * 4, cudaMemcpyDeviceToHost, s));
  if (state9) BCK(cudaMemcpyAsync(state9, b->d_rec_state.p + o * 9, n * 9 * 8, cudaMemcpyDeviceToHost, s));
  BCK(cudaStreamSynchronize(s));
  if (ind)
    for (int64_t k = 0; k < n; ++k)
      if (ind[k] >= 0) ind[k] -= M.zone_off;
  return SED_OK;
}

const char* sed_batch_last_error(sed_batch* b) { return b ? b->err.c_str() : "null batch"; }

void sed_batch_destroy(sed_batch* b)
{
  if (!b) return;
  if (b->inner) {
    cudaSetDevice(b->inner->device);
    cudaStreamSynchronize(b->inner->stream);
  }
  drop_graph(b);
  for (auto& ev : b->ev) if (ev) cudaEventDestroy(ev);
  b->d_models.release(); b->d_sample_models.release(); b->d_nbr.release(); b->d_rin.release(); b->d_wall.release();
  b->d_core_cdf.release(); b->d_flux.release(); b->d_click.release(); b->d_model_esc.release(); b->d_step.release();
  b->d_em_state.release(); b->d_em_ind.release(); b->d_em_tau.release(); b->d_em_model.release();
  b->d_zone_rep.release();
  b->d_rec_fate.release(); b->d_rec_ind.release(); b->d_rec_draws.release(); b->d_rec_state.release();
  if (b->inner) sed_ctx_destroy(b->inner);
  delete b;
}

}  // extern "C"
