// opacity_kernel.cu -- per-zone opacity/emissivity build on the device
// (transport::set_opacity, src/transport/transport_opacity.cpp:21-260).
//
//   zone_state_kernel   one thread per zone: temperature clamp, mass
//                       fractions, then the LTE electron-density solve
//                       (GasState::solve_state / ne_brent_method,
//                       src/opacity/GasState.cpp:208-337) with
//                       AtomicSpecies::solve_lte (AtomicSpecies_state.cpp:56-123).
//                       Boltzmann factors depend on T only and are computed
//                       once per zone instead of once per Brent iteration
//                       (same values, same rounding).
//   zone_opacity_kernel one CTA per zone: electron scattering, free-free,
//                       bound-free, Sobolev line and fuzz-line expansion
//                       opacity per frequency bin in the reference's order
//                       (GasState::computeOpacity, GasState_opacities.cpp:11-136),
//                       then the opacity cap, Planck/Rosseland means,
//                       emissivity CDF (cdf_array::set_value prefix sum, in
//                       the reference's order for FP64 grids up to 65536
//                       zones), L_thermal, Fleck factor and
//                       the packed tables the packet kernel reads.  The
//                       zone's level populations are staged in shared memory
//                       with their reciprocals, so a line costs two
//                       shared-memory reads, one 16 B and one 16 B (8 B in
//                       FP32) global load and no division.  Line lists are
//                       sorted by (bin, atom) with a stable sort, so each bin
//                       is one contiguous run in the reference's list order.
//                       In the mixed-precision form the per-line Sobolev sums
//                       run in FP32 with Kahan compensation; everything else
//                       stays FP64.
//
// The host runs the kernels once per chunk of zones: per-zone inputs and
// outputs are passed offset to the chunk, and every scratch array
// (index * nzones + zone) is sized for one chunk, so a 128^3-zone grid with
// thousands of bins builds its tables through a bounded working set.
#include <cfloat>
#include <cmath>
#include <mutex>
#include <type_traits>
#include "../../include/sedona_gpu.h"
#include "sed_internal.h"

namespace sed {
namespace {

// ------------------------------------------------------------ LTE
// Per-zone scratch is stored level-major / ion-major (index * nz + zone) so
// neighbouring threads (zones) touch neighbouring addresses.

// AtomicSpecies::solve_lte for atom a at electron density ne; partition
// functions `part` (ion-major scratch) and Boltzmann factors are cached.
__device__ void solve_lte_atom(const OpacityArgs& A, int z, int a, double ne, double T, const double* boltz_e,
                               double* part, double* frac, double* lev, int write_lev, double* net)
{
  const int nz = A.nzones;
  const int i0 = A.ion_off[a], ni = A.ion_off[a + 1] - i0;
  const int l0 = A.lev_off[a], nl = A.lev_off[a + 1] - l0;
  const double lt = H_PLANCK * H_PLANCK / (2.0 * PI * MASS_E * K_BOLTZ * T);
  const double fac = 2 / ne / pow(lt, 1.5);
  frac[(size_t)i0 * nz + z] = 1.;
  for (int i = 1; i < ni; ++i) {
    const double chi = A.ion_chi[i0 + i - 1];
    double saha = exp(-1.0 * chi / K_EV / T);
    saha = saha * (part[(size_t)(i0 + i) * nz + z] / part[(size_t)(i0 + i - 1) * nz + z]) * fac;
    double fi = saha * frac[(size_t)(i0 + i - 1) * nz + z];
    if (ne < 1e-50) fi = 0;
    frac[(size_t)(i0 + i) * nz + z] = fi;
    double norm = 0;
    for (int j = 0; j <= i; j++) norm += frac[(size_t)(i0 + j) * nz + z];
    for (int j = 0; j <= i; j++) frac[(size_t)(i0 + j) * nz + z] = frac[(size_t)(i0 + j) * nz + z] / norm;
  }
  double x = 0;
  for (int i = 0; i < nl; ++i) {
    const int ion = A.lev_ion[l0 + i];
    const double Z = part[(size_t)(i0 + ion) * nz + z];
    const double f = frac[(size_t)(i0 + ion) * nz + z];
    double v = f * A.lev_g[l0 + i] * boltz_e[(size_t)(l0 + i) * nz + z] / Z;
    if (v < 1e-30) v = 1e-30;
    if (write_lev) lev[(size_t)(l0 + i) * nz + z] = v;
    x += v * A.lev_ion[l0 + i];
  }
  *net = x;
}

__device__ double charge_conservation(const OpacityArgs& A, int z, double ne, double T, double dens,
                                      const double* boltz_e, int write_lev)
{
  double f = 0;
  for (int a = 0; a < A.natoms; ++a) {
    double net;
    solve_lte_atom(A, z, a, ne, T, boltz_e, A.ion_part, A.ion_frac, A.lev_n, write_lev, &net);
    f += dens * A.mass_frac[(size_t)a * A.nzones + z] / (A.eA[a] * MASS_P) * net;
  }
  return f - ne;
}

// GasState::ne_brent_method (GasState.cpp:270-337); *last = last point evaluated
__device__ double ne_brent(const OpacityArgs& A, int z, double T, double dens, const double* boltz_e, double x1,
                           double x2, double tol, double* last, int* err)
{
  const int ITMAX = 100;
  const double EPS = 3.0e-8;
  double a = x1, b = x2, c = x2, d = 0, e = 0, min1, min2;
  double fa = charge_conservation(A, z, a, T, dens, boltz_e, 0);
  double fb = charge_conservation(A, z, b, T, dens, boltz_e, 0);
  *last = b;
  double fc, p, q, r, s, tol1, xm;
  if ((fa > 0.0 && fb > 0.0) || (fa < 0.0 && fb < 0.0)) *err = 1;
  fc = fb;
  for (int iter = 1; iter <= ITMAX; iter++) {
    if ((fb > 0.0 && fc > 0.0) || (fb < 0.0 && fc < 0.0)) { c = a; fc = fa; e = d = b - a; }
    if (fabs(fc) < fabs(fb)) { a = b; b = c; c = a; fa = fb; fb = fc; fc = fa; }
    tol1 = 2.0 * EPS * fabs(b) + 0.5 * tol;
    xm = 0.5 * (c - b);
    if (fabs(xm) <= tol1 || fb == 0.0) return b;
    if (fabs(e) >= tol1 && fabs(fa) > fabs(fb)) {
      s = fb / fa;
      if (a == c) { p = 2.0 * xm * s; q = 1.0 - s; }
      else {
        q = fa / fc;
        r = fb / fc;
        p = s * (2.0 * xm * q * (q - r) - (b - a) * (r - 1.0));
        q = (q - 1.0) * (r - 1.0) * (s - 1.0);
      }
      if (p > 0.0) q = -q;
      p = fabs(p);
      min1 = 3.0 * xm * q - fabs(tol1 * q);
      min2 = fabs(e * q);
      if (2.0 * p < (min1 < min2 ? min1 : min2)) { e = d; d = p / q; }
      else { d = xm; e = d; }
    } else { d = xm; e = d; }
    a = b;
    fa = fb;
    b += (fabs(d) > tol1) ? d : (xm >= 0.0 ? fabs(tol1) : -fabs(tol1));
    fb = charge_conservation(A, z, b, T, dens, boltz_e, 0);
    *last = b;
  }
  *err = 2;
  return 0.0;
}

__global__ void zone_state_kernel(const OpacityArgs A, double* boltz_e)
{
  const int z = blockIdx.x * blockDim.x + threadIdx.x;
  const int nz = A.nzones;
  if (z >= nz) return;
  double T = A.T[z];
  if (T < A.temp_min) T = A.temp_min;
  if (T > A.temp_max) T = A.temp_max;
  A.temp_c[z] = T;
  const double dens = A.rho[z];
  // GasState::set_mass_fractions (GasState.cpp:137-156)
  double norm = 0.0;
  for (int a = 0; a < A.nelem; ++a) norm += A.X[(size_t)z * A.nelem + a];
  double inv = 0.;
  for (int a = 0; a < A.nelem; ++a) {
    const double mf = A.X[(size_t)z * A.nelem + a] / norm;
    A.mass_frac[(size_t)a * nz + z] = mf;
    inv += mf / A.eA[a];
  }
  const double mu_I = 1. / inv;
  A.solve_err[z] = 0;
  if (A.grey[z] != 0 || A.natoms == 0) { A.n_elec[z] = 0; return; }
  for (int a = 0; a < A.natoms; ++a)
    A.n_dens[(size_t)a * nz + z] = dens * A.mass_frac[(size_t)a * nz + z] / (A.eA[a] * MASS_P);
  // Boltzmann factors exp(-E/kT) and partition functions: T only
  for (int a = 0; a < A.natoms; ++a) {
    const int i0 = A.ion_off[a], ni = A.ion_off[a + 1] - i0;
    const int l0 = A.lev_off[a], nl = A.lev_off[a + 1] - l0;
    for (int i = 0; i < ni; ++i) A.ion_part[(size_t)(i0 + i) * nz + z] = 0;
    for (int i = 0; i < nl; ++i) {
      const double eb = exp(-A.lev_E[l0 + i] / K_EV / T);
      boltz_e[(size_t)(l0 + i) * nz + z] = eb;
      const int ion = A.lev_ion[l0 + i];
      A.ion_part[(size_t)(i0 + ion) * nz + z] += A.lev_g[l0 + i] * eb;
    }
  }
  const double max_ne = 100 * dens / (mu_I * MASS_P);
  const double min_ne = 1e-10 * dens / (mu_I * MASS_P);
  double last = 0;
  int err = 0;
  const double ne = ne_brent(A, z, T, dens, boltz_e, min_ne, max_ne, 1e-3, &last, &err);
  charge_conservation(A, z, last, T, dens, boltz_e, 1);  // populations of the last evaluation
  A.n_elec[z] = ne;
  A.solve_err[z] = err;
}

// ------------------------------------------------------------ per zone
// xy_array::value_at_with_zero_edges (src/utils/xy_array.cpp:42-104)
__device__ double photo_cs(const OpacityArgs& A, int lev, double zv)
{
  const int p0 = A.photo_off[lev], n = A.photo_off[lev + 1] - p0;
  const double* x = A.photo_E + p0;
  const double* y = A.photo_s + p0;
  if (n <= 0) return 0;
  if (zv < x[0]) return 0;
  if (zv > x[n - 1]) return 0;
  if (n == 1) return y[0];
  int ind;
  if (zv >= x[n - 1]) ind = n;
  else if (zv <= x[0]) ind = 0;
  else {
    int bl = 0, bu = n - 1;
    while (bu - bl > 1) { const int bm = (bu + bl) / 2; if (x[bm] <= zv) bl = bm; else bu = bm; }
    ind = bl;
  }
  int i1, i2;
  if (ind < n - 1) { i1 = ind; i2 = ind + 1; }
  else { i2 = ind < n ? ind : n - 1; i1 = i2 - 1; }
  const double slope = (y[i2] - y[i1]) / (x[i2] - x[i1]);
  return y[ind < n ? ind : n - 1] + slope * (zv - x[i1]);
}

// 1 - exp(-tau), the Sobolev escape factor of one line, as the reference
// writes it: for tau below ~1e-16 it is exactly 0 and for small tau it
// carries the cancellation of 1 - exp(-tau), which the FP64 tables reproduce.
__device__ __forceinline__ double sobolev_term(double tau) { return 1 - exp(-tau); }

// FP32 form of 1 - exp(-x) for x >= 0, branch-free: below x = 0.1 the
// Taylor series to x^7 (truncation below x^8/8! < 3e-12 relative), above it
// 1 - __expf(-x), whose ~2^-22 relative error in exp(-x) stays below 3e-6
// relative in 1 - exp(-x) for x >= 0.1.  Neither has the cancellation of
// 1 - expf(-x) at small x.
__device__ __forceinline__ float one_minus_exp32(float x)
{
  const float p = x * (1.f - x * 0.5f * (1.f - x * (1.f / 3) * (1.f - x * 0.25f * (1.f - x * 0.2f *
                 (1.f - x * (1.f / 6) * (1.f - x * (1.f / 7)))))));
  const float e = 1.f - __expf(-x);
  return (x < 0.1f) ? p : e;
}

__device__ __forceinline__ float sobolev_term32(float tau) { return one_minus_exp32(tau); }

// Level populations of one zone in the chunk scratch (level-major).
struct LevView {
  const double* p;
  int64_t stride;
  __device__ __forceinline__ double n(int l) const { return p[l * stride]; }
};

// Per-bin Sobolev sums of one line list (level-to-level lines, or fuzz lines
// when FUZZ) for a tile of ZT zones: S[z][bin] = sum of (1 - exp(-tau)) over
// the bin's lines, Se[z][bin] the same weighted by the line's atom epsilon
// when atoms differ in epsilon (AtomicSpecies_opacities.cpp:292-375,
// GasState_opacities.cpp:424-494).  The tile's level populations times the
// atom's number density, n_l n_atom, and their reciprocals (or the ion
// populations for fuzz lines) are staged in shared memory level-major, ZT
// zones contiguous; the ratio n_u g_l / (n_l g_u) is formed from them (the
// atom density cancels).  A warp takes one bin at a time (warp w the bins
// order[w], order[w + 8], ..., `order` listing the bins by decreasing line
// count): its lanes are ZT zones x 32/ZT line slots, slot s summing the
// bin's lines s, s + 32/ZT, ... (sorted by bin, atom), and the slots of a
// zone are then added in FP64 in a fixed butterfly order, so the sums are
// the same from run to run.  The FP64 form sums in FP64; the mixed form
// computes its terms in FP32 and sums them in FP32 with Kahan compensation
// (measured on the Type Ia and 3D builds: the same time and the same
// largest error against the FP64 oracle as FP64 sums of the FP32 terms,
// 1.6e-6 relative, which the FP32 tables' rounding sets).
// Level populations come from the LTE solve, floored at 1e-30, so they are
// normal FP32 numbers and the reference's n_l < DBL_MIN skip never applies
// to them; a NaN term is skipped as in the reference.
constexpr int LINE_SUM_WARPS = 8;  // line_sum_kernel runs 256 threads per CTA

template <bool MIXED, bool FUZZ, int ZT>
__global__ void __launch_bounds__(32 * LINE_SUM_WARPS) line_sum_kernel(const OpacityArgs A, double* S, double* Se)
{
  using V = typename std::conditional<MIXED, float, double>::type;
  extern __shared__ double lsm[];
  const int nn = A.n_nu, nz = A.nzones, na = A.natoms, tid = threadIdx.x, bd = blockDim.x;
  const int z0 = blockIdx.x * ZT;
  const int nzt = min(ZT, nz - z0);
  if (nzt <= 0) return;
  // shared: ndv[na][ZT], epsv[na], invT[ZT], pop[np][ZT], ipop[np][ZT] (V)
  const int np = FUZZ ? A.n_ions_total : A.n_lev_total;
  V* ndv = reinterpret_cast<V*>(lsm);
  V* epsv = ndv + na * ZT;
  V* invT = epsv + na;
  V* pop = invT + ZT;
  V* ipop = pop + (size_t)np * ZT;
  for (int i = tid; i < na * ZT; i += bd) {
    const int a = i / ZT, zi = i % ZT;
    ndv[i] = (zi < nzt) ? (V)A.n_dens[(size_t)a * nz + z0 + zi] : (V)0;
  }
  for (int a = tid; a < na; a += bd) epsv[a] = A.zero_eps_atom[a] ? (V)0 : (V)A.epsilon;
  for (int zi = tid; zi < ZT; zi += bd) invT[zi] = (zi < nzt) ? (V)(1.0 / A.temp_c[z0 + zi]) : (V)0;
  for (int i = tid; i < np * ZT; i += bd) {
    const int l = i / ZT, zi = i % ZT;
    double v = 0;
    if (zi < nzt) {
      if constexpr (FUZZ) {
        const int a = A.ion_atom[l];
        v = A.n_dens[(size_t)a * nz + z0 + zi] * A.ion_frac[(size_t)l * nz + z0 + zi] /
            A.ion_part[(size_t)l * nz + z0 + zi];
      } else {
        v = A.lev_n[(size_t)l * nz + z0 + zi] * A.n_dens[(size_t)A.lev_atom[l] * nz + z0 + zi];
      }
    }
    pop[i] = (V)v;
    if constexpr (!FUZZ) ipop[i] = (zi < nzt) ? (V)(1.0 / v) : (V)0;
  }
  __syncthreads();
  const bool want_e = !A.uniform_eps;
  const int32_t* seg = FUZZ ? A.fz_seg : A.ln_seg;
  const int32_t* order = FUZZ ? A.fz_order : A.ln_order;
  const double time = A.time;
  // a warp per bin: its 32 lanes are ZT zones x LS line slots; slot s takes
  // the bin's lines s, s + LS, ..., so the lanes of a warp run the same
  // number of lines (up to one) and read the same few line records.  The
  // warp stages the bin's records 32 at a time in its shared-memory buffer,
  // one coalesced load per lane, and the slots read them from there: one
  // memory round trip per 32 records instead of one per LS (48^3 level-line
  // build 61.2 -> 48.5 ms, Type Ia fuzz-line build 5.2 -> 5.0 ms).  The
  // line loop is unrolled by two (Type Ia 6.9 -> 5.4 ms before the staging).
  constexpr int LS = 32 / ZT;
  static_assert(32 % LS == 0, "a slot keeps its lines across the 32-record chunks");
  const int lane = tid & 31, warp = tid >> 5, nwarps = bd >> 5;
  const int zi = lane % ZT, slot = lane / ZT;
  using CRec = typename std::conditional<MIXED, typename std::conditional<FUZZ, float4, float2>::type, double2>::type;
  __shared__ int4 s_ix[LINE_SUM_WARPS][32];
  __shared__ CRec s_cr[LINE_SUM_WARPS][32];
  __shared__ double s_h[(FUZZ && !MIXED) ? LINE_SUM_WARPS : 1][32];
  const int4* __restrict__ ix_g = FUZZ ? A.fz_ia : A.ln_lv;
  const CRec* __restrict__ cr_g;
  if constexpr (MIXED) {
    if constexpr (FUZZ) cr_g = A.fz_c32; else cr_g = A.ln_c32;
  } else {
    cr_g = FUZZ ? A.fz_c : A.ln_c;
  }
  for (int jj = warp; jj < nn; jj += nwarps) {
    const int j = __ldg(order + jj);
    double acc = 0, acce = 0;
    float ks = 0.f, kc = 0.f, kse = 0.f, kce = 0.f;  // the mixed form's FP32 Kahan sums
    const int k0 = seg[j], k1 = seg[j + 1];
    for (int kb = k0; kb < k1; kb += 32) {
      const int nk = min(32, k1 - kb);
      __syncwarp();
      if (lane < nk) {
        s_ix[warp][lane] = __ldg(ix_g + kb + lane);
        s_cr[warp][lane] = __ldg(cr_g + kb + lane);
        if constexpr (FUZZ && !MIXED) s_h[warp][lane] = __ldg(A.fz_h + kb + lane);
      }
      __syncwarp();
#pragma unroll 2
      for (int kk = slot; kk < nk; kk += LS) {
        int atom;
        V term;
        if constexpr (!FUZZ) {
          // tau = n_l n_atom sigma_tot f lambda t (1 - n_u g_l / (n_l g_u)), 0 past the laser limit
          const int4 lv = s_ix[warp][kk];
          atom = lv.w;
          const V pl = pop[(size_t)lv.x * ZT + zi];   // n_l n_atom
          const V il = ipop[(size_t)lv.x * ZT + zi];  // 1 / (n_l n_atom)
          const V pu = pop[(size_t)lv.y * ZT + zi];   // n_u n_atom
          if constexpr (MIXED) {
            const float2 c = s_cr[warp][kk];
            const float r = pu * il * c.y;
            const float tau = (r > 1.f) ? 0.f : pl * (c.x * (float)time) * (1.f - r);
            const float t = sobolev_term32(tau);
            term = (t == t) ? t : 0.f;
          } else {
            const double2 c = s_cr[warp][kk];
            double t = 0;
            if (!(pl < DBL_MIN)) {
              const double r = pu * il * c.y;
              const double tau = (r > 1) ? 0.0 : pl * c.x * time * (1 - r);
              t = sobolev_term(tau);
              if (isnan(t)) t = 0;
            }
            term = t;
          }
        } else {
          // n_l = n_ion exp(-E_l/kT) / Z_ion, tau = sigma_tot lambda n_l gf (1 - exp(-h nu/kT)) t
          const int4 ia = s_ix[warp][kk];
          atom = ia.z;
          const V pi = pop[(size_t)ia.x * ZT + zi];
          if constexpr (MIXED) {
            const float4 c = s_cr[warp][kk];
            const float stim = one_minus_exp32(c.z * invT[zi]);
            const float tau = (c.x * (float)time) * pi * __expf(-c.y * invT[zi]) * stim;
            term = sobolev_term32(tau);
          } else {
            const double2 c = s_cr[warp][kk];
            const double h = s_h[warp][kk];
            if (zi < nzt) {
              const double temp = A.temp_c[z0 + zi];
              const double nl = pi * exp(-c.y / temp);
              const double stim_cor = (1 - exp(-h / temp));
              const double tau = c.x * nl * stim_cor * time;
              term = sobolev_term(tau);
            } else {
              term = 0;
            }
          }
        }
        if constexpr (MIXED) {
          // Kahan (compensated) summation in FP32: the rounding error of each
          // addition is carried into the next term
          { const float y = term - kc; const float t = ks + y; kc = (t - ks) - y; ks = t; }
          if (want_e) {
            const float y = term * epsv[atom] - kce;
            const float t = kse + y;
            kce = (t - kse) - y;
            kse = t;
          }
        } else {
          acc += (double)term;
          if (want_e) acce += (double)(term * epsv[atom]);
        }
      }
    }
    if constexpr (MIXED) { acc = (double)ks; acce = (double)kse; }
    // the LS slots of each zone, summed in a fixed butterfly order
#pragma unroll
    for (int off = ZT; off < 32; off <<= 1) {
      acc += __shfl_xor_sync(0xffffffffu, acc, off);
      acce += __shfl_xor_sync(0xffffffffu, acce, off);
    }
    if (slot == 0 && zi < nzt) {
      S[(size_t)(z0 + zi) * nn + j] = acc;
      if (want_e) Se[(size_t)(z0 + zi) * nn + j] = acce;
    }
  }
}

// Opacity, scattering and emissivity of bin j of zone z (GasState::
// computeOpacity, GasState_opacities.cpp:11-136, with its terms in the
// reference's order: electron scattering, free-free, bound-free, Sobolev
// lines, fuzz lines).  The line terms arrive as the bin's Sobolev sums
// (ls, lse, fs, fse; the epsilon-weighted sums only when atoms differ in
// epsilon); nu and ez = exp(h nu/kT) are shared with the caller, which reuses
// ez for the mean opacities.
__device__ void bin_opacity(const OpacityArgs& A, int zc, int j, double nu, double ez, double temp, double grey,
                            double ne, double es, double ff_fac, const double* nd, const LevView& L, double ls,
                            double lse, double fs, double fse, double& ab_o, double& sc_o, double& em_o)
{
  double ab = 0, sc = 0, em = 0;
  if (grey != 0) {  // GasState_opacities.cpp:29-41
    const double gopac = A.rho[zc] * grey;
    ab = gopac * A.epsilon;
    sc = gopac * (1 - A.epsilon);
    const double bb = 2.0 * nu * nu * nu * H_PLANCK / C_LIGHT / C_LIGHT / (ez - 1);
    em += bb * ab;
  } else if (A.natoms > 0) {
    if (A.use_es) {  // :49-58
      sc += es;
      ab += 1e-20 * A.epsilon * es;
    }
    if (A.use_ff) {  // GasState::free_free_opacity :152-183
      const double ezeta = exp(-1.0 * H_PLANCK * nu / K_BOLTZ / temp);
      const double bb = 2.0 * nu * nu * nu * H_PLANCK / C_LIGHT / C_LIGHT / (1.0 / ezeta - 1);
      const double op = ff_fac / nu / nu / nu * (1 - ezeta);
      ab += op;
      em += op * bb;
    }
    if (A.use_bf) {  // GasState::bound_free_opacity + AtomicSpecies_opacities.cpp:58-151
      const double kt_ev = K_EV * temp;
      const double lam_t = sqrt(H_PLANCK * H_PLANCK / (2 * PI * MASS_E * K_BOLTZ * temp));
      const double E = H_PLANCK * nu * ERGS_TO_EV;
      const double emis_fac = 2. * H_PLANCK * nu * nu * nu / C_LIGHT / C_LIGHT;
      double so = 0, se = 0;
      for (int a = 0; a < A.natoms; ++a) {
        const int l0 = A.lev_off[a], nl = A.lev_off[a + 1] - l0;
        double ao = 0, ae = 0;
        for (int q = 0; q < nl; ++q) {
          const int ic = A.lev_ic[l0 + q];
          if (ic == -1) continue;
          const double Eion = A.lev_Eion[l0 + q];
          if (E < Eion) continue;
          const double nc = nd[a] * L.n(l0 + ic);
          const double gl_o_gc = (1.0 * A.lev_g[l0 + q]) / (1.0 * A.lev_g[l0 + ic]);
          const double ncp = nc * gl_o_gc / 2. * lam_t * lam_t * lam_t;
          const double zeta_net = (Eion - E) / kt_ev;
          const double ezeta_net = exp(zeta_net);
          const double sigma = photo_cs(A, l0 + q, E);
          double opac_fac = nd[a] * L.n(l0 + q) - ncp * ne * ezeta_net;
          if (opac_fac < 0) opac_fac = 0.;
          ao += sigma * opac_fac;
          ae += emis_fac * sigma * ncp * ezeta_net;
        }
        so += ao;
        se += ae;
      }
      ab += so;
      em += se * ne;
    }
    const double bb = 2.0 * nu * nu * nu * H_PLANCK / C_LIGHT / C_LIGHT / (ez - 1);
    const double fac = nu / loc_delta(A.nu, j) / C_LIGHT / A.time;
    if (A.use_line) {  // GasState::line_expansion_opacity :424-454
      const double opac = ls * fac;
      const double aopac = (A.uniform_eps ? ls * A.epsilon : lse) * fac;
      ab += aopac;
      sc += opac - aopac;
      em += bb * aopac;
    }
    if (A.use_fuzz) {  // GasState::fuzz_expansion_opacity :464-494
      const double opac = fs * fac;
      const double aopac = (A.uniform_eps ? fs * A.epsilon : fse) * fac;
      ab += aopac;
      sc += opac - aopac;
      em += bb * aopac;
    }
  }
  ab_o = ab;
  sc_o = sc;
  em_o = em;
}

// One CTA per zone of the chunk, after line_sum_kernel: each thread builds
// bins j = tid, tid + 256, ... from the continuum terms and the bin's
// Sobolev sums (GasState::computeOpacity), caps them and accumulates the
// Planck/Rosseland partial sums (GasState_opacities.cpp:564-666); then the
// CTA forms the emissivity CDF, L_thermal and eps_imc
// (transport_opacity.cpp:152-252) and writes the packed tables the packet
// kernel reads.  The FP64 rows (abs, scat, emissivity) live in shared memory
// when they fit (A.smem_rows); otherwise abs and scat overwrite the line and
// fuzz sums of the zone in the chunk scratch (each bin is read, then written,
// by the same thread) and the emissivity row is scratch too.
template <bool MIXED>
__global__ void __launch_bounds__(256) zone_opacity_kernel(const OpacityArgs A)
{
  extern __shared__ double dsm[];
  __shared__ double red[4][256];
  __shared__ double zs[2];  // electron scattering, free-free factor
  const int z = blockIdx.x;
  if (z >= A.nzones) return;
  const int nn = A.n_nu, nz = A.nzones, na = A.natoms, tid = threadIdx.x, bd = blockDim.x;
  const double temp = A.temp_c[z];
  const double grey = A.grey[z];
  const double ne = A.n_elec[z];
  const bool want_e = !A.uniform_eps;

  // shared layout: nd[na] rows[3 nn]
  double* nd = dsm;
  double* rows = nd + na;
  const size_t zo = (size_t)z * nn;
  const double* LS = A.abs64 + zo;
  const double* FS = A.scat64 + zo;
  const double* LSe = A.epsl64 + zo;
  const double* FSe = A.epsf64 + zo;
  double* R0 = A.smem_rows ? rows : A.abs64 + zo;
  double* R1 = A.smem_rows ? rows + nn : A.scat64 + zo;
  double* R2 = A.smem_rows ? rows + 2 * nn : A.emis64 + zo;

  const bool micro = (grey == 0 && na > 0);
  if (micro) {
    for (int a = tid; a < na; a += bd) nd[a] = A.n_dens[(size_t)a * nz + z];
    if (tid == 0) {
      zs[0] = THOMSON * ne;
      double ff = 0;
      if (A.use_ff) {  // GasState::free_free_opacity :152-183 (zone factor)
        const double dens = A.rho[z];
        for (int a = 0; a < na; ++a) {
          const int i0 = A.ion_off[a], ni = A.ion_off[a + 1] - i0;
          double zsq = 0;
          for (int q = 0; q < ni; q++) zsq += A.ion_frac[(size_t)(i0 + q) * nz + z] * q * q;
          const double n_ion = A.mass_frac[(size_t)a * nz + z] * dens / (A.eA[a] * MASS_P);
          ff += n_ion * zsq;
        }
        ff *= 3.7e8 * pow(temp, -0.5) * ne;
      }
      zs[1] = ff;
    }
  }
  __syncthreads();
  LevView L;
  L.p = A.lev_n + z;
  L.stride = nz;
  const double es = micro ? zs[0] : 0.0, ff_fac = micro ? zs[1] : 0.0;
  const bool lines = micro && A.use_line, fuzz = micro && A.use_fuzz;

  // bins, cap (transport_opacity.cpp:189-200) and mean-opacity partial sums
  const double max_ext = A.max_opacity * A.rho[z];
  double pm = 0, pn = 0, rm = 0, rn = 0;
  for (int j = tid; j < nn; j += bd) {
    const double nu = loc_center(A.nu, j);
    const double zeta = H_PLANCK * nu / K_BOLTZ / temp;
    const double ez = exp(zeta);
    double ab, sc, em;
    bin_opacity(A, z, j, nu, ez, temp, grey, ne, es, ff_fac, nd, L, lines ? LS[j] : 0.0,
                (lines && want_e) ? LSe[j] : 0.0, fuzz ? FS[j] : 0.0, (fuzz && want_e) ? FSe[j] : 0.0, ab, sc, em);
    if (A.omit_scat) sc = 0;
    else if (sc > max_ext) sc = max_ext;
    if (ab > max_ext) ab = max_ext;
    R0[j] = ab;
    R1[j] = sc;
    R2[j] = em;
    double Bnu = 2.0 * nu * nu * nu * H_PLANCK / C_LIGHT / C_LIGHT / (ez - 1);
    if (isnan(Bnu)) Bnu = 0;
    const double d = loc_delta(A.nu, j);
    const double W = Bnu * d;
    pm += W * ab;
    pn += W;
    double dBdT = pow(nu, 4) * ez / (ez - 1) / (ez - 1);
    if (isnan(dBdT)) dBdT = 0;
    const double Wr = dBdT * d;
    rm += Wr / (ab + sc);
    rn += Wr;
  }
  double* ab_r = R0;
  double* sc_r = R1;
  red[0][tid] = pm; red[1][tid] = pn; red[2][tid] = rm; red[3][tid] = rn;
  __syncthreads();
  for (int st = bd / 2; st > 0; st >>= 1) {
    if (tid < st)
      for (int q = 0; q < 4; ++q) red[q][tid] += red[q][tid + st];
    __syncthreads();
  }
  const double pm_tot = red[0][0], pn_tot = red[1][0], rm_tot = red[2][0], rn_tot = red[3][0];
  __syncthreads();

  // emissivity CDF: cdf_array::set_value prefix sum of emis*dnu (cdf_array.h:
  // 53-75) and L_thermal = 4 pi sum(emis*dnu).  FP64 tables of grids up to
  // 65536 zones: in the reference's order, so the CDF is the reference's sum
  // to the bit (and a bin's share of it, the difference of two neighbouring
  // values, too): the terms in parallel, the running sums by one thread, a
  // few microseconds per zone.  Otherwise (FP32 tables, or millions of zones
  // where a serial row per CTA would dominate the build) a blocked scan in a
  // fixed order: each thread sums a contiguous run of bins, thread 0 scans
  // the run totals, each run adds its offset; non-negative terms, so every
  // prefix is within a few ulp of the sequential sum, and a NaN term
  // propagates to the end as in the sequential sum.
  double* em = R2;
  double Lth = 0;
  if (nn == 1) {
    if (tid == 0) {
      const double bb_int = SB * pow(A.T[z], 4) / PI;
      Lth += 4 * PI * ab_r[0] * bb_int;
      em[0] = 1;
    }
  } else if (!MIXED && A.seq_cdf) {
    for (int j = tid; j < nn; j += bd) em[j] = em[j] * loc_delta(A.nu, j);
    __syncthreads();
    if (tid == 0) {
      double run = 0, L = 0;
      for (int j = 0; j < nn; ++j) {
        const double ednu = em[j];
        run = (j == 0) ? ednu : run + ednu;
        em[j] = run;
        L += 4 * PI * ednu;
      }
      red[2][0] = L;
    }
    __syncthreads();
    Lth = red[2][0];
  } else {
    const int per = (nn + bd - 1) / bd;
    const int j0 = min(nn, tid * per), j1 = min(nn, j0 + per);
    double run = 0, Lp = 0;
    for (int j = j0; j < j1; ++j) {
      const double ednu = em[j] * loc_delta(A.nu, j);
      run = (j == j0) ? ednu : run + ednu;
      em[j] = run;
      Lp += 4 * PI * ednu;
    }
    red[0][tid] = run;
    red[1][tid] = Lp;
    __syncthreads();
    if (tid == 0) {
      double acc = 0, Lacc = 0;
      for (int t = 0; t < bd; ++t) {
        const double v = red[0][t];
        red[0][t] = acc;
        acc = (t == 0) ? v : acc + v;
        Lacc += red[1][t];
      }
      red[2][0] = Lacc;
    }
    __syncthreads();
    const double off = red[0][tid];
    if (tid > 0)
      for (int j = j0; j < j1; ++j) em[j] = off + em[j];
    Lth = red[2][0];
  }
  __syncthreads();
  for (int j = tid; j < nn; j += bd) if (isnan(em[j])) em[j] = 0;
  __syncthreads();
  const bool all_zero = (em[nn - 1] == 0);
  __syncthreads();
  if (all_zero) for (int j = tid; j < nn; j += bd) em[j] = 1.0;
  __syncthreads();
  if (tid == 0) {
    A.L_th[z] = Lth;
    if (nn == 1) {
      A.planck[z] = ab_r[0];
      A.ross[z] = ab_r[0] + sc_r[0];
    } else {
      A.planck[z] = pm_tot / pn_tot;
      A.ross[z] = rn_tot / rm_tot;
    }
    if (A.radiative_eq) A.eps_imc[z] = 1.;
    else {
      const double fleck_beta = 4.0 * A_RAD * pow(A.T[z], 4) / (A.e_gas[z] * A.rho[z]);
      const double tfac = C_LIGHT * A.planck[z] * A.dt;
      double f_imc = A.fleck_alpha * fleck_beta * tfac;
      if (A.fleck_alpha == 0) f_imc = 0.;
      A.eps_imc[z] = 1.0 / (1.0 + f_imc);
    }
  }
  const double N = em[nn - 1];
  __syncthreads();  // every thread has N before em[] is overwritten below
  // normalised CDF, packed tables and the coarse CDF index for the packet kernel
  for (int j = tid; j < nn; j += bd) {
    const size_t k = (size_t)z * nn + j;
    const double c = em[j] / N;
    if constexpr (MIXED) {
      reinterpret_cast<float2*>(A.opac_out)[k] = make_float2((float)ab_r[j], (float)sc_r[j]);
      reinterpret_cast<float*>(A.cdf_out)[k] = (float)c;
    } else {
      reinterpret_cast<double2*>(A.opac_out)[k] = make_double2(ab_r[j], sc_r[j]);
      reinterpret_cast<double*>(A.cdf_out)[k] = c;
    }
    if ((j % CDF_STRIDE) == CDF_STRIDE - 1 || j == nn - 1) {
      const size_t kc = (size_t)z * A.n_coarse + j / CDF_STRIDE;
      if constexpr (MIXED) reinterpret_cast<float*>(A.cdf_coarse_out)[kc] = (float)c;
      else reinterpret_cast<double*>(A.cdf_coarse_out)[kc] = c;
    }
    // the value the packet kernel compares against, as a double
    em[j] = MIXED ? (double)(float)c : c;
  }
  // guide table of the stored row: guide[k] = upper_bound(row, k / G)
  if (A.cdf_guide_out) {
    __syncthreads();
    const int G = A.guide_n;
    uint16_t* gz = A.cdf_guide_out + (size_t)z * (G + 1);
    for (int k = tid; k <= G; k += bd) {
      const double t = (double)k / (double)G;
      int lo = 0, hi = nn;
      while (lo < hi) {
        const int m = (lo + hi) >> 1;
        if (em[m] <= t) lo = m + 1; else hi = m;
      }
      gz[k] = (uint16_t)lo;
    }
  }
}

// zone tiles of the line-sum kernel: 8 zones per CTA in FP32, 4 in FP64
constexpr int LINE_TILE_MIXED = 8;
constexpr int LINE_TILE_FP64 = 4;

template <bool MIXED, bool FUZZ>
int launch_line_sums(const OpacityArgs& a, double* S, double* Se, cudaStream_t s)
{
  constexpr int ZT = MIXED ? LINE_TILE_MIXED : LINE_TILE_FP64;
  const size_t vs = MIXED ? sizeof(float) : sizeof(double);
  const size_t np = FUZZ ? (size_t)a.n_ions_total : (size_t)a.n_lev_total;
  const size_t smem = vs * ((size_t)a.natoms * ZT + a.natoms + ZT + 2 * np * ZT);
  auto k = line_sum_kernel<MIXED, FUZZ, ZT>;
  if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return -1;
  k<<<(a.nzones + ZT - 1) / ZT, 256, smem, s>>>(a, S, Se);
  return 1;
}

}  // namespace

size_t opacity_smem_bytes(const OpacityArgs& a)
{
  size_t d = (size_t)a.natoms;
  if (a.smem_rows) d += 3 * (size_t)a.n_nu;
  return d * sizeof(double);
}

size_t line_sum_smem_bytes(int precision, int natoms, int n_pop)
{
  const int ZT = precision ? LINE_TILE_MIXED : LINE_TILE_FP64;
  const size_t vs = precision ? sizeof(float) : sizeof(double);
  return vs * ((size_t)natoms * ZT + natoms + ZT + 2 * (size_t)n_pop * ZT);
}

int launch_opacity(const OpacityArgs& a, int num_sms, cudaStream_t s)
{
  (void)num_sms;
  const int nz = a.nzones;
  int n = 0;
  zone_state_kernel<<<(nz + 127) / 128, 128, 0, s>>>(a, a.boltz);
  ++n;
  const bool micro = a.natoms > 0;
  int r = 0;
  if (micro && a.use_line)
    r = a.precision ? launch_line_sums<true, false>(a, a.abs64, a.epsl64, s)
                    : launch_line_sums<false, false>(a, a.abs64, a.epsl64, s);
  if (r < 0) return -1;
  n += r;
  r = 0;
  if (micro && a.use_fuzz)
    r = a.precision ? launch_line_sums<true, true>(a, a.scat64, a.epsf64, s)
                    : launch_line_sums<false, true>(a, a.scat64, a.epsf64, s);
  if (r < 0) return -1;
  n += r;
  const size_t smem = opacity_smem_bytes(a);
  if (a.precision) {
    if (cudaFuncSetAttribute(zone_opacity_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
      return -1;
    zone_opacity_kernel<true><<<nz, 256, smem, s>>>(a);
  } else {
    if (cudaFuncSetAttribute(zone_opacity_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
      return -1;
    zone_opacity_kernel<false><<<nz, 256, smem, s>>>(a);
  }
  return n + 1;
}

}  // namespace sed

// ---------------------------------------------------------------------------
// LTE electron densities without any device allocation.
//
// Some callers cannot allocate device memory at the point where they need
// this result: a host code whose device memory is entirely handed out by its
// own pool allocator, or one that runs the solve inside a per-step loop where
// the implicit synchronisation of cudaMalloc/cudaFree is not acceptable.
// They own the inputs and the outputs.  The per-zone working set of the
// solve (mass fractions, number densities, clamped temperature, partition
// functions, ion fractions, level populations, Boltzmann factors) lives in
// the fixed array below, which is part of the library image: every GPU that
// loads the library holds it until the process exits.
namespace {
constexpr size_t NOALLOC_SCRATCH_DOUBLES = size_t(1) << 19;  // 4 MiB per device
__device__ __align__(256) double g_lte_scratch[NOALLOC_SCRATCH_DOUBLES];

constexpr int NOALLOC_MAX_DEVICES = 64;
std::mutex g_scratch_mutex;
double* g_scratch_addr[NOALLOC_MAX_DEVICES] = {};
}  // namespace

extern "C" int sed_lte_electron_density_noalloc(int32_t n_zones, const double* rho, const double* T_gas,
                                                const double* X, int32_t n_elems, const int32_t* elem_A,
                                                const sed_atomic_data* atoms_dev, int32_t n_ions_total,
                                                int32_t n_levels_total, double temp_min, double temp_max,
                                                double* n_elec, int32_t* solve_err, void* stream)
{
  using namespace sed;
  if (n_zones <= 0 || n_elems <= 0 || n_ions_total <= 0 || n_levels_total <= 0) return SED_ERR_ARG;
  if (!rho || !T_gas || !X || !elem_A || !atoms_dev || !n_elec || !solve_err) return SED_ERR_ARG;
  if (atoms_dev->n_atoms != n_elems || !atoms_dev->ion_off || !atoms_dev->ion_chi || !atoms_dev->lev_off ||
      !atoms_dev->lev_ion || !atoms_dev->lev_g || !atoms_dev->lev_E)
    return SED_ERR_ARG;
  const size_t nz = (size_t)n_zones, na = (size_t)n_elems;
  const size_t ni = (size_t)n_ions_total, nl = (size_t)n_levels_total;
  // doubles per zone, then zones: the limit is checked as a quotient so that
  // no product of the caller's counts can wrap around
  const size_t per_zone = 2 * na + 2 + 2 * ni + 2 * nl;
  if (per_zone > NOALLOC_SCRATCH_DOUBLES || nz > NOALLOC_SCRATCH_DOUBLES / per_zone)
    return SED_ERR_CAPACITY;  // limit stated in include/sedona_gpu.h

  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NOALLOC_MAX_DEVICES) return SED_ERR_CUDA;
  double* base = nullptr;
  {
    // first call on this device: look up the array's device address with
    // this device current (the host-side symbol is only a stand-in)
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_addr[dev]) {
      void* p = nullptr;
      if (cudaGetSymbolAddress(&p, g_lte_scratch) != cudaSuccess || !p) return SED_ERR_CUDA;
      g_scratch_addr[dev] = static_cast<double*>(p);
    }
    base = g_scratch_addr[dev];
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  OpacityArgs A{};
  A.nzones = n_zones;
  A.nelem = n_elems;
  A.natoms = n_elems;
  A.temp_min = temp_min;
  A.temp_max = temp_max;
  A.rho = rho;
  A.T = T_gas;
  A.X = X;
  A.eA = elem_A;
  A.ion_off = atoms_dev->ion_off;
  A.ion_chi = atoms_dev->ion_chi;
  A.lev_off = atoms_dev->lev_off;
  A.lev_ion = atoms_dev->lev_ion;
  A.lev_g = atoms_dev->lev_g;
  A.lev_E = atoms_dev->lev_E;
  A.n_ions_total = n_ions_total;
  A.n_lev_total = n_levels_total;
  // carve the scratch array
  double* q = base;
  A.mass_frac = q;  q += na * nz;
  A.n_dens = q;     q += na * nz;
  A.temp_c = q;     q += nz;
  double* grey = q; q += nz;  // all zones take the microphysical path: zero grey opacity
  A.ion_part = q;   q += ni * nz;
  A.ion_frac = q;   q += ni * nz;
  A.lev_n = q;      q += nl * nz;
  A.boltz = q;      q += nl * nz;
  A.grey = grey;
  A.n_elec = n_elec;
  A.solve_err = solve_err;
  // the array keeps the previous call's contents; only the grey-opacity
  // column must start at zero (every other entry is written before it is read)
  if (cudaMemsetAsync(grey, 0, nz * sizeof(double), s) != cudaSuccess) return SED_ERR_CUDA;
  zone_state_kernel<<<(unsigned)((nz + 127) / 128), 128, 0, s>>>(A, A.boltz);
  return cudaGetLastError() == cudaSuccess ? SED_OK : SED_ERR_CUDA;
}
