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

// out[z][j] = base[z][j] * r[z] for both members of the {abs, scat} pair;
// in FP64, then rounded to the table's type (what scaling the widened tables
// on the host and loading them again rounds to)
template <typename P>
__global__ void scale_rows_kernel(const P* __restrict__ base, P* __restrict__ out, const double* __restrict__ r,
                                  size_t nz, size_t nn)
{
  using T = decltype(P::x);
  const size_t n = nz * nn;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double f = r[i / nn];
    const P b = base[i];
    P o;
    o.x = (T)((double)b.x * f);
    o.y = (T)((double)b.y * f);
    out[i] = o;
  }
}

}  // namespace

extern "C" {

int sed_set_rng_step(sed_ctx* c, uint32_t step)
{
  if (!c) return SED_ERR_ARG;
  c->step = step;
  return SED_OK;
}

// the weighted forward; abs_scale (or null) is read with copy kind `in`
int diff_forward(sed_ctx* c, double dt, const double* abs_scale, cudaMemcpyKind in, int32_t n_bands,
                 sed_step_stats* st)
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
  if (abs_scale) {
    CK(c->d_abs_scale.resize(nz * (size_t)n_bands));
    CK(cudaMemcpyAsync(c->d_abs_scale.p, abs_scale, nz * (size_t)n_bands * sizeof(double), in, c->stream));
  }
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

int sed_diff_forward(sed_ctx* c, double dt, const double* abs_scale, int32_t n_bands, sed_step_stats* st)
{
  return diff_forward(c, dt, abs_scale, cudaMemcpyHostToDevice, n_bands, st);
}

int sed_diff_forward_dev(sed_ctx* c, double dt, const double* abs_scale_dev, int32_t n_bands, double* flux_dev,
                         sed_step_stats* st)
{
  int rc = diff_forward(c, dt, abs_scale_dev, cudaMemcpyDeviceToDevice, n_bands, st);
  if (rc) return rc;
  if (flux_dev) {
    CK(cudaMemcpyAsync(flux_dev, c->d_flux.p, c->nspec * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  }
  return SED_OK;
}

// vector-Jacobian product of the last forward (per (zone, band) or, with
// density, per zone): grad_flux read and the result written with the given
// copy kinds
int diff_vjp(sed_ctx* c, const double* grad_flux, cudaMemcpyKind in, double* out, cudaMemcpyKind out_kind,
             bool density, sed_step_stats* st)
{
  if (!c || !grad_flux || !out) return SED_ERR_ARG;
  const size_t n_out = density ? (size_t)c->nz : (size_t)c->nz * (size_t)std::max(c->diff_bands, 1);
  CK(c->d_adj_g.resize((size_t)c->nspec));
  CK(cudaMemcpyAsync(c->d_adj_g.p, grad_flux, (size_t)c->nspec * sizeof(double), in, c->stream));
  CK(c->d_adj_out.resize(n_out));
  CK(cudaMemsetAsync(c->d_adj_out.p, 0, n_out * sizeof(double), c->stream));
  int rc = replay(c, false, st, density);
  if (rc) return rc;
  CK(cudaMemcpyAsync(out, c->d_adj_out.p, n_out * sizeof(double), out_kind, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return SED_OK;
}

int sed_diff_vjp(sed_ctx* c, const double* grad_flux, double* grad_scale, sed_step_stats* st)
{
  return diff_vjp(c, grad_flux, cudaMemcpyHostToDevice, grad_scale, cudaMemcpyDeviceToHost, false, st);
}

int sed_diff_vjp_dev(sed_ctx* c, const double* grad_flux_dev, double* grad_scale_dev, sed_step_stats* st)
{
  return diff_vjp(c, grad_flux_dev, cudaMemcpyDeviceToDevice, grad_scale_dev, cudaMemcpyDeviceToDevice, false, st);
}

int sed_diff_vjp_density(sed_ctx* c, const double* grad_flux, double* grad_rho, sed_step_stats* st)
{
  return diff_vjp(c, grad_flux, cudaMemcpyHostToDevice, grad_rho, cudaMemcpyDeviceToHost, true, st);
}

int sed_diff_vjp_density_dev(sed_ctx* c, const double* grad_flux_dev, double* grad_rho_dev, sed_step_stats* st)
{
  return diff_vjp(c, grad_flux_dev, cudaMemcpyDeviceToDevice, grad_rho_dev, cudaMemcpyDeviceToDevice, true, st);
}

// both extinctions of zone z of the built tables times r[z], in place of the
// tables the packet kernels read; r null: the built tables back
int scale_extinction(sed_ctx* c, const double* r, cudaMemcpyKind in)
{
  if (!c) return SED_ERR_ARG;
  if (!c->have_opacity) return set_err(c, SED_ERR_STATE, "sed_diff_scale_extinction: opacity tables not set");
  c->have_diff = false;  // the last weighted forward no longer matches the context
  const size_t nz = (size_t)c->nz, nn = (size_t)c->nu.n();
  const size_t bytes = c->d_opac.n;
  if (!c->opac_base_valid) {
    CK(c->d_opac_base.resize(bytes));
    CK(cudaMemcpyAsync(c->d_opac_base.p, c->d_opac.p, bytes, cudaMemcpyDeviceToDevice, c->stream));
    c->opac_base_valid = true;
  }
  if (!r) {
    if (c->opac_scaled) CK(cudaMemcpyAsync(c->d_opac.p, c->d_opac_base.p, bytes, cudaMemcpyDeviceToDevice, c->stream));
    c->opac_scaled = false;
  } else {
    CK(c->d_rho_scale.resize(nz));
    CK(cudaMemcpyAsync(c->d_rho_scale.p, r, nz * sizeof(double), in, c->stream));
    if (c->tp.precision)
      scale_rows_kernel<float2><<<c->num_sms * 4, 256, 0, c->stream>>>(
          reinterpret_cast<const float2*>(c->d_opac_base.p), reinterpret_cast<float2*>(c->d_opac.p),
          c->d_rho_scale.p, nz, nn);
    else
      scale_rows_kernel<double2><<<c->num_sms * 4, 256, 0, c->stream>>>(
          reinterpret_cast<const double2*>(c->d_opac_base.p), reinterpret_cast<double2*>(c->d_opac.p),
          c->d_rho_scale.p, nz, nn);
    CK(cudaGetLastError());
    c->opac_scaled = true;
  }
  CK(cudaStreamSynchronize(c->stream));
  return SED_OK;
}

int sed_diff_scale_extinction(sed_ctx* c, const double* rho_scale)
{
  return scale_extinction(c, rho_scale, cudaMemcpyHostToDevice);
}

int sed_diff_scale_extinction_dev(sed_ctx* c, const double* rho_scale_dev)
{
  return scale_extinction(c, rho_scale_dev, cudaMemcpyDeviceToDevice);
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
