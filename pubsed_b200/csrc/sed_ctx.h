// sed_ctx.h -- the transport context behind the C ABI (struct sed_ctx) and
// the host helpers shared by the single-model entry points (sed_abi.cu) and
// the batched ones (sed_batch.cu).
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/sedona_gpu.h"
#include "sed_internal.h"

namespace sed {


template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  cudaError_t resize(size_t m)
  {
    if (m == n && p) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
    if (m == 0) return cudaSuccess;
    cudaError_t e = cudaMalloc(&p, m * sizeof(T));
    if (e == cudaSuccess) n = m;
    return e;
  }
  void release()
  {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
};

// host copy of a locate_array with the same lookup rules as the device
struct HostLoc {
  int type = 0;
  double min = 0, del = 0;
  std::vector<double> x;
  int n() const { return (int)x.size(); }
  double left(int i) const { return i == 0 ? min : x[i - 1]; }
  double delta(int i) const { return i == 0 ? x[0] - min : x[i] - x[i - 1]; }
  double center(int i) const { return i == 0 ? 0.5 * (min + x[0]) : 0.5 * (x[i - 1] + x[i]); }
  int upper(double v) const { return (int)(std::upper_bound(x.begin(), x.end(), v) - x.begin()); }
  int locate(double v) const  // locate_array::locate (src/utils/locate_array.cpp:191-218)
  {
    const int nn = n();
    if (nn == 1) return 0;
    if (v >= x[nn - 1]) return nn;
    if (v < min) return 0;
    int ind;
    if (type == LOC_FLEX) return upper(v);
    else if (type == LOC_LIN) ind = (int)std::floor((v - min) / del);
    else if (type == LOC_LOG) ind = (int)std::floor(std::log(v / min) / std::log(1 + del));
    else return 0;
    if (ind != 0 && ind != nn && (left(ind) > v || x[ind] <= v)) ind = upper(v);
    return ind;
  }
  int within(double v) const { const int i = locate(v); return i == n() ? n() - 1 : i; }
};

inline HostLoc host_loc(const sed_locate_grid& g)
{
  HostLoc h;
  h.type = g.type;
  h.min = g.min;
  h.del = g.del;
  h.x.assign(g.right, g.right + g.n);
  return h;
}


}  // namespace sed

using sed::DevBuf;
using sed::HostLoc;

struct sed_ctx {
  int device = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev[6] = {};
  std::string err;
  sed_transport_params tp{};
  HostLoc nu, st, sn, sm, sp;
  DevBuf<double> d_nu, d_st, d_sn, d_sm, d_sp, d_core_cdf;
  uint32_t step = 0;

  // grid
  bool have_grid = false;
  int gtype = 0, nz = 0, nelem = 0, homologous = 1, nx = 0, ny = 0, nzz = 0;
  double t_grid = 0;
  HostLoc r_out, ax[3];
  DevBuf<double> d_r_out, d_v_r, d_ax[3], d_vol, d_rho, d_T, d_egas, d_grey, d_X;
  DevBuf<int32_t> d_eZ, d_eA;
  std::vector<int32_t> h_eZ;

  // opacity parameters and atomic data
  sed_opacity_params op{};
  std::vector<int32_t> zero_eps;
  DevBuf<int32_t> d_zero_eps_atom;
  bool have_atoms = false;
  bool any_zero_eps = false;
  int natoms = 0, n_ions_total = 0, n_lev_total = 0, nfuzz = 0, nlines = 0;
  DevBuf<int32_t> d_ion_off, d_lev_off, d_lev_ion, d_lev_g, d_lev_ic, d_photo_off, d_ion_atom, d_lev_atom, d_ln_seg,
      d_fz_seg, d_ln_order, d_fz_order;
  DevBuf<double> d_ion_chi, d_lev_E, d_lev_Eion, d_photo_E, d_photo_s, d_fz_h;
  DevBuf<int4> d_ln_lv;
  DevBuf<double2> d_ln_c, d_fz_c;
  DevBuf<float2> d_ln_c32;
  DevBuf<int4> d_fz_ia;
  DevBuf<float4> d_fz_c32;

  // tables
  bool have_opacity = false;
  DevBuf<unsigned char> d_opac, d_cdf, d_cdf_coarse;
  DevBuf<double> d_zone_rep;          // [n_rep][5][nz] zone-scalar tally copies of the 1D mixed kernel
  DevBuf<double> d_rho_scale;         // per-zone extinction factors of the last scaling
  DevBuf<unsigned char> d_opac_base;  // the built {abs, scat} tables while scaled ones are in d_opac
  bool opac_base_valid = false;       // d_opac_base holds the tables of the last build or load
  bool opac_scaled = false;           // d_opac holds density-scaled tables
  int n_coarse = 0;
  DevBuf<uint16_t> d_cdf_guide;  // CDF guide tables, guide_n + 1 entries per zone
  int guide_n = 0;
  int chunk_zones = 0;  // zones per opacity-build pass (bounds the FP64/LTE scratch)
  int opacity_launches = 0;
  DevBuf<double> d_imd_p;  // IMD probabilities of the step [4][nz]
  // core packets emitted ahead of the mixed-form 1D kernel: state [9][n], zone, first optical depth
  DevBuf<double> d_em_state;
  DevBuf<int32_t> d_em_ind;
  DevBuf<float> d_em_tau;
  DevBuf<double> d_eps_imc, d_abs64, d_scat64, d_emis64, d_epsl64, d_epsf64, d_planck, d_ross, d_L, d_n_elec, d_n_dens, d_mass_frac,
      d_temp_c, d_ion_part, d_ion_frac, d_lev_n, d_boltz;
  DevBuf<int32_t> d_solve_err;
  DevBuf<int32_t> d_temp_bad;     // zones the temperature solve left unsolved

  // tallies
  DevBuf<double> d_J, d_e_abs, d_e_rad, d_fx, d_fy, d_fz, d_fr, d_flux, d_click;

  // radioactive source: gamma-ray spectrum grid and tallies, per-zone decay
  // quantities, and the queue of optical photons it hands to the packet kernel
  HostLoc gn;
  int64_t nspec_g = 0;
  DevBuf<double> d_gn, d_gflux, d_gclick, d_radio_cdf, d_gamma_frac, d_compton, d_photoion, d_L_emit, d_L_dep,
      d_L_tot, d_q_state;
  DevBuf<int32_t> d_q_ind, d_reject;
  DevBuf<uint32_t> d_q_n;
  DevBuf<unsigned long long> d_counters;
  int64_t nspec = 0;

  // differentiable transport: escape records of the last weighted forward
  // (its Philox step, band count, whether a scale array was applied)
  bool have_diff = false;
  uint32_t diff_step = 0;
  double diff_dt = 1;
  int diff_bands = 0;
  bool diff_scaled = false;
  int64_t diff_n = 0;
  DevBuf<int32_t> d_esc_bin;
  DevBuf<double> d_esc_e, d_abs_scale, d_adj_g, d_adj_out;

  // per-packet records (also the end states a time-dependent step builds
  // its census from)
  int record = 0;
  int64_t n_rec = 0;
  DevBuf<int32_t> d_rec_fate, d_rec_ind, d_rec_draws, d_rec_type;
  DevBuf<double> d_rec_state;

  // transport clock (transport::t_now_): the first grid's time, then
  // advanced by dt after each time-dependent step (transport.cpp:136)
  double t_now = 0;
  bool have_t_now = false;
  // packets carried to the next step, in the reference's vector order:
  // {x, D, t, e, nu}, zone, type; and the queue entries they load into
  int64_t n_census = 0, n_census_gamma = 0;
  DevBuf<double> d_census_state;
  DevBuf<int32_t> d_census_ind, d_census_type, d_q_type;
  DevBuf<int32_t> d_cmp;                  // flags, sums and front list of the compaction
  DevBuf<unsigned char> d_scan_tmp;       // scan scratch
  DevBuf<unsigned long long> d_cmp_count;
};

namespace sed {


inline int set_err(sed_ctx* c, int code, const char* fmt, ...)
{
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (c) c->err = buf;
  return code;
}

#define CK(call)                                                                                       \
  do {                                                                                                 \
    cudaError_t e_ = (call);                                                                           \
    if (e_ != cudaSuccess)                                                                             \
      return set_err(c, e_ == cudaErrorMemoryAllocation ? SED_ERR_NOMEM : SED_ERR_CUDA, "%s: %s (%s:%d)", \
                     #call, cudaGetErrorString(e_), __FILE__, __LINE__);                               \
  } while (0)

template <typename T>
cudaError_t upload(sed_ctx* c, DevBuf<T>& b, const T* src, size_t n)
{
  cudaError_t e = b.resize(n ? n : 1);
  if (e != cudaSuccess) return e;
  if (n && src) return cudaMemcpyAsync(b.p, src, n * sizeof(T), cudaMemcpyHostToDevice, c->stream);
  return cudaMemsetAsync(b.p, 0, (n ? n : 1) * sizeof(T), c->stream);
}

// n elements from src, or n zeros when the caller passed no array
template <typename T>
cudaError_t upload_or_zero(sed_ctx* c, DevBuf<T>& b, const T* src, size_t n)
{
  cudaError_t e = b.resize(n ? n : 1);
  if (e != cudaSuccess) return e;
  if (src) return cudaMemcpyAsync(b.p, src, n * sizeof(T), cudaMemcpyHostToDevice, c->stream);
  return cudaMemsetAsync(b.p, 0, (n ? n : 1) * sizeof(T), c->stream);
}

inline DevLoc dev_loc(const HostLoc& h, const DevBuf<double>& d)
{
  DevLoc g;
  g.n = h.n();
  g.type = h.type;
  g.min = h.min;
  g.del = h.del;
  g.right = d.p;
  g.inv_step = 0.f;
  if (h.type == LOC_LOG && h.del > 0) g.inv_step = (float)(1.0 / std::log2(1.0 + h.del));
  else if (h.type == LOC_LIN && h.del > 0) g.inv_step = (float)(1.0 / h.del);
  g.lmin_step = (h.type == LOC_LOG && h.min > 0) ? (float)(std::log2(h.min) * g.inv_step) : 0.f;
  g.inv_min = (h.type == LOC_LOG && h.min > 0) ? (float)(1.0 / h.min) : 0.f;
  return g;
}

inline bool valid_grid(const sed_locate_grid& g) { return g.n > 0 && g.right != nullptr; }

// Queues the opacity build of every zone of the context on its stream
// (transport::set_opacity) without synchronising; used directly by the
// batched step, which captures it into a CUDA graph.
int enqueue_opacity(sed_ctx* c, double dt);

// kernel arguments and device grid of a transport step of this context
StepArgs make_step_args(sed_ctx* c, double dt, int64_t n_emit);
GridDev make_grid_dev(sed_ctx* c);

// normalised core emission CDF of a blackbody at T over the bins of `nu`
// (transport::setup_core_emission, src/transport/transport_init.cpp:465-556)
std::vector<double> core_emission_cdf(const HostLoc& nu, double T);

}  // namespace sed
