// sed_diff.cu -- differentiable transport (sed_diff_* in include/sedona_gpu.h).
//
// sed_diff_forward runs the weighted-forward packet kernel and keeps, per
// packet, only the spectrum index it escaped into and its escaping energy.
// sed_diff_vjp / sed_diff_jacobian then launch the adjoint replay kernel:
// each escaped packet is emitted and walked again from its Philox stream
// (same step number, same deviates, same path) and every segment adds
// -w a0 dshift l to the (zone, band) entry it crossed.  sed_diff_vjp_density
// replays the same way into one entry per zone: -w ((a + s) dshift l) per
// segment and +w per scattering (the score of the scattering path, a
// likelihood-ratio term, since the scattering opacity decides where the
// path goes).  Nothing of a path is stored between the two launches.
#include <cstring>
#include <vector>

#include "sed_ctx.h"

using namespace sed;

namespace {

int diff_args_ok(sed_ctx* c)
{
  if (!c->have_grid) return set_err(c, SED_ERR_STATE, "differentiable transport: no grid");
  if (!c->have_opacity) return set_err(c, SED_ERR_STATE, "differentiable transport: opacity tables not set");
  if (!c->homologous)
    return set_err(c, SED_ERR_ARG, "differentiable transport: homologous velocity fields only");
  if (c->tp.radiative_eq)
    return set_err(c, SED_ERR_ARG, "differentiable transport: needs transport_radiative_equilibrium = 0 "
                                   "(absorbed energy leaves the packet)");
  if (c->tp.fleck_alpha != 0)
    return set_err(c, SED_ERR_ARG, "differentiable transport: needs transport_fleck_alpha = 0");
  if (c->tp.steady_state && c->tp.core_fix_luminosity)
    return set_err(c, SED_ERR_ARG, "differentiable transport: no steady-state luminosity rescale");
  return SED_OK;
}

void fill_stats(sed_step_stats* st, const unsigned long long* cnt, int64_t n, float ms_kernel, float ms_total,
                int launches)
{
  if (!st) return;
  std::memset(st, 0, sizeof *st);
  st->n_packets = n;
  st->n_escaped = (int64_t)cnt[C_ESCAPED];
  st->n_absorbed = (int64_t)cnt[C_ABSORBED];
  st->n_stopped = (int64_t)cnt[C_STOPPED];
  st->n_segments = (int64_t)cnt[C_SEGMENTS];
  st->n_scatters = (int64_t)cnt[C_SCATTERS];
  st->n_limit = (int64_t)cnt[C_LIMIT];
  st->kernel_launches = launches;
  st->ms_propagate_kernel = ms_kernel;
  st->ms_transport = ms_total;
  st->ms_total = ms_total;
}

// the adjoint replay of the last weighted forward into c->d_adj_out
int replay(sed_ctx* c, bool jacobian, sed_step_stats* st, bool density = false)
{
  if (!c->have_diff) return set_err(c, SED_ERR_STATE, "sed_diff_vjp/jacobian: no weighted forward to replay");
  StepArgs A = make_step_args(c, c->diff_dt, c->diff_n);
  A.step = c->diff_step;
  A.n_bands = c->diff_bands;
  A.abs_scale = c->diff_scaled ? c->d_abs_scale.p : nullptr;
  A.esc_bin = c->d_esc_bin.p;
  A.esc_e = c->d_esc_e.p;
  A.adj_g = c->d_adj_g.p;
  A.adj_out = c->d_adj_out.p;
  A.adj_jacobian = jacobian ? 1 : 0;
  A.adj_density = density ? 1 : 0;
  CK(cudaMemsetAsync(c->d_counters.p, 0, (C_COUNT + 1) * sizeof(unsigned long long), c->stream));
  CK(cudaEventRecord(c->ev[3], c->stream));
  if (c->diff_n > 0 && launch_propagate_diff(A, make_grid_dev(c), 2, c->num_sms, c->stream) < 0)
    return set_err(c, SED_ERR_ARG, "adjoint replay: unsupported grid");
  CK(cudaGetLastError());
  CK(cudaEventRecord(c->ev[4], c->stream));
  unsigned long long cnt[C_COUNT + 1];
  CK(cudaMemcpyAsync(cnt, c->d_counters.p, sizeof cnt, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  float ms = 0;
  cudaEventElapsedTime(&ms, c->ev[3], c->ev[4]);
  fill_stats(st, cnt, c->diff_n, ms, ms, c->diff_n > 0 ? 1 : 0);
  if (cnt[C_LIMIT] > 0) return set_err(c, SED_ERR_LIMIT, "%llu packets hit the segment limit", cnt[C_LIMIT]);
  return SED_OK;
}

}  // namespace

extern "C" {

int sed_set_rng_step(sed_ctx* c, uint32_t step)
{
  if (!c) return SED_ERR_ARG;
  c->step = step;
  return SED_OK;
}

int sed_diff_forward(sed_ctx* c, double dt, const double* abs_scale, int32_t n_bands, sed_step_stats* st)
{
  if (!c) return SED_ERR_ARG;
  int rc = diff_args_ok(c);
  if (rc) return rc;
  if (n_bands < 1 || n_bands > c->nu.n()) return set_err(c, SED_ERR_ARG, "sed_diff_forward: %d bands", n_bands);
  if (c->tp.steady_state) dt = 1;
  const int64_t n_emit = (int64_t)(c->tp.core_n_emit / 1.0);
  if (n_emit > c->tp.max_particles)
    return set_err(c, SED_ERR_CAPACITY, "Not enough particle space: %lld packets > particles_max_total %lld",
                   (long long)n_emit, (long long)c->tp.max_particles);
  const size_t nz = (size_t)c->nz, nn = (size_t)c->nu.n(), nj = c->tp.store_Jnu ? nn : 1;
  CK(c->d_esc_bin.resize((size_t)std::max<int64_t>(n_emit, 1)));
  CK(c->d_esc_e.resize((size_t)std::max<int64_t>(n_emit, 1)));
  if (abs_scale) CK(upload(c, c->d_abs_scale, abs_scale, nz * (size_t)n_bands));
  if (c->record) {
    CK(c->d_rec_fate.resize(std::max<int64_t>(n_emit, 1)));
    CK(c->d_rec_ind.resize(std::max<int64_t>(n_emit, 1)));
    CK(c->d_rec_draws.resize(std::max<int64_t>(n_emit, 1)));
    CK(c->d_rec_state.resize(std::max<int64_t>(n_emit, 1) * 9));
    c->n_rec = n_emit;
  }
  CK(cudaEventRecord(c->ev[2], c->stream));
  CK(cudaMemsetAsync(c->d_J.p, 0, nz * nj * sizeof(double), c->stream));
  double* z[6] = {c->d_e_abs.p, c->d_e_rad.p, c->d_fx.p, c->d_fy.p, c->d_fz.p, c->d_fr.p};
  for (double* p : z) CK(cudaMemsetAsync(p, 0, nz * sizeof(double), c->stream));
  CK(cudaMemsetAsync(c->d_flux.p, 0, c->nspec * sizeof(double), c->stream));
  CK(cudaMemsetAsync(c->d_click.p, 0, c->nspec * sizeof(double), c->stream));
  CK(cudaMemsetAsync(c->d_counters.p, 0, (C_COUNT + 1) * sizeof(unsigned long long), c->stream));
  StepArgs A = make_step_args(c, dt, n_emit);
  A.n_bands = n_bands;
  A.abs_scale = abs_scale ? c->d_abs_scale.p : nullptr;
  A.esc_bin = c->d_esc_bin.p;
  A.esc_e = c->d_esc_e.p;
  if (c->record) {
    A.rec_fate = c->d_rec_fate.p; A.rec_ind = c->d_rec_ind.p; A.rec_draws = c->d_rec_draws.p; A.rec_state = c->d_rec_state.p;
  }
  const GridDev G = make_grid_dev(c);
  int launches = 0;
  CK(cudaEventRecord(c->ev[3], c->stream));
  if (n_emit > 0) {
    if (launch_propagate_diff(A, G, 1, c->num_sms, c->stream) < 0)
      return set_err(c, SED_ERR_ARG, "weighted forward: unsupported grid");
    ++launches;
  }
  CK(cudaGetLastError());
  CK(cudaEventRecord(c->ev[4], c->stream));
  launches += launch_finish(A, G, c->d_vol.p, c->nspec, c->stream);
  CK(cudaGetLastError());
  CK(cudaEventRecord(c->ev[5], c->stream));
  unsigned long long cnt[C_COUNT + 1];
  CK(cudaMemcpyAsync(cnt, c->d_counters.p, sizeof cnt, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->have_diff = true;
  c->diff_step = c->step;
  c->diff_dt = dt;
  c->diff_bands = n_bands;
  c->diff_scaled = abs_scale != nullptr;
  c->diff_n = n_emit;
  c->step++;
  float mk = 0, mt = 0;
  cudaEventElapsedTime(&mk, c->ev[3], c->ev[4]);
  cudaEventElapsedTime(&mt, c->ev[2], c->ev[5]);
  fill_stats(st, cnt, n_emit, mk, mt, launches);
  if (cnt[C_LIMIT] > 0) return set_err(c, SED_ERR_LIMIT, "%llu packets hit the segment limit", cnt[C_LIMIT]);
  return SED_OK;
}

int sed_diff_vjp(sed_ctx* c, const double* grad_flux, double* grad_scale, sed_step_stats* st)
{
  if (!c || !grad_flux || !grad_scale) return SED_ERR_ARG;
  const size_t n_out = (size_t)c->nz * (size_t)std::max(c->diff_bands, 1);
  CK(upload(c, c->d_adj_g, grad_flux, (size_t)c->nspec));
  CK(c->d_adj_out.resize(n_out));
  CK(cudaMemsetAsync(c->d_adj_out.p, 0, n_out * sizeof(double), c->stream));
  int rc = replay(c, false, st);
  if (rc) return rc;
  CK(cudaMemcpyAsync(grad_scale, c->d_adj_out.p, n_out * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return SED_OK;
}

int sed_diff_vjp_density(sed_ctx* c, const double* grad_flux, double* grad_rho, sed_step_stats* st)
{
  if (!c || !grad_flux || !grad_rho) return SED_ERR_ARG;
  const size_t n_out = (size_t)c->nz;
  CK(upload(c, c->d_adj_g, grad_flux, (size_t)c->nspec));
  CK(c->d_adj_out.resize(n_out));
  CK(cudaMemsetAsync(c->d_adj_out.p, 0, n_out * sizeof(double), c->stream));
  int rc = replay(c, false, st, true);
  if (rc) return rc;
  CK(cudaMemcpyAsync(grad_rho, c->d_adj_out.p, n_out * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return SED_OK;
}

int sed_diff_jacobian(sed_ctx* c, double* jac, sed_step_stats* st)
{
  if (!c || !jac) return SED_ERR_ARG;
  const size_t n_out = (size_t)c->nspec * (size_t)c->nz * (size_t)std::max(c->diff_bands, 1);
  CK(c->d_adj_g.resize(1));
  CK(c->d_adj_out.resize(n_out));
  CK(cudaMemsetAsync(c->d_adj_out.p, 0, n_out * sizeof(double), c->stream));
  int rc = replay(c, true, st);
  if (rc) return rc;
  CK(cudaMemcpyAsync(jac, c->d_adj_out.p, n_out * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return SED_OK;
}

}  // extern "C"
