// sed_common.cuh -- device-side building blocks shared by the kernels:
// physical constants, the Philox4x32-10 packet streams, and the bin-edge
// search with locate_array semantics.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace sed {

// physical_constants (src/utils/physical_constants.h:9-31); pi is 3.14159 there
constexpr double PI = 3.14159;
constexpr double C_LIGHT = 2.99792458e10;
constexpr double H_PLANCK = 6.6260755e-27;
constexpr double K_BOLTZ = 1.380658e-16;
constexpr double K_EV = 8.6173324e-5;
constexpr double MASS_P = 1.67262158e-24;
constexpr double MASS_E = 9.10938188e-28;
constexpr double SB = 5.6704e-5;
constexpr double A_RAD = 7.5657e-15;
constexpr double THOMSON = 0.66523e-24;
constexpr double SIGMA_TOT = 0.0265400193567;
constexpr double ERGS_TO_EV = 624150975230.2815;
constexpr double M_E_MEV = 0.510998910511;  // electron rest energy (MeV)
constexpr double MEV_TO_ERGS = 1.60217646e-6;
constexpr double ALPHA_FS = 0.007;          // fine-structure constant as the reference has it

enum Fate : int32_t { MOVING = 0, STOPPED = 1, ESCAPED = 2, ABSORBED = 3 };
enum LocType : int32_t { LOC_FLEX = 0, LOC_LIN = 1, LOC_LOG = 2, LOC_NONE = 3 };

// ---------------------------------------------------------------- Philox
// Philox4x32-10 (Salmon et al., SC'11).  A packet's deviates form the stream
// key = {seed, 0}, counter = {n >> 1, pid.lo, pid.hi, step}; draw n uses
// output words 0,1 (n even) or 2,3 (n odd) as a 53-bit double in [0, 1).
struct PhiloxOut { uint32_t w[4]; };

__host__ __device__ inline PhiloxOut philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                                   uint32_t k0, uint32_t k1)
{
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    if (r) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
#ifdef __CUDA_ARCH__
    const uint32_t lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
    const uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
#else
    const uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
    const uint32_t lo0 = (uint32_t)p0, hi0 = (uint32_t)(p0 >> 32);
    const uint32_t lo1 = (uint32_t)p1, hi1 = (uint32_t)(p1 >> 32);
#endif
    const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
  }
  return PhiloxOut{{c0, c1, c2, c3}};
}

__host__ __device__ inline double u01(uint32_t a, uint32_t b)
{
  return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6)) * (1.0 / 9007199254740992.0);
}

// one 32-bit word as a deviate in [0, 1)
__host__ __device__ inline double w01(uint32_t a) { return (double)a * (1.0 / 4294967296.0); }

// Per-packet stream.  Each draw evaluates its Philox block: lanes of a warp
// sit at different draw parities, so keeping the odd half of a block for the
// next draw would only make half the lanes compute while the others wait.
#ifndef SED_RNG_CACHE
#define SED_RNG_CACHE 0
#endif
struct PacketRng {
  uint32_t seed, step;
  uint64_t pid;
  uint32_t n;
#if SED_RNG_CACHE
  uint32_t cached_ctr;
  uint32_t cw2, cw3;
  bool have;
#endif

  __device__ void init(uint32_t seed_, uint64_t pid_, uint32_t step_, uint32_t n0)
  {
    seed = seed_; pid = pid_; step = step_; n = n0;
#if SED_RNG_CACHE
    have = false;
#endif
  }
  // Word layout of the mixed form: one Philox block per call, four 32-bit
  // words each used as one deviate, counter {k, pid.lo, pid.hi, step}, key
  // {seed, 1} (streams independent of the per-draw layout's key {seed, 0}).
  __device__ uint4 block()
  {
    const PhiloxOut o = philox4x32_10(n++, (uint32_t)pid, (uint32_t)(pid >> 32), step, seed, 1u);
    return make_uint4(o.w[0], o.w[1], o.w[2], o.w[3]);
  }
  __device__ double next()
  {
    const uint32_t k = n++;
    const uint32_t ctr = k >> 1;
#if SED_RNG_CACHE
    if ((k & 1u) && have && cached_ctr == ctr) return u01(cw2, cw3);
#endif
    PhiloxOut o = philox4x32_10(ctr, (uint32_t)pid, (uint32_t)(pid >> 32), step, seed, 0u);
#if SED_RNG_CACHE
    cached_ctr = ctr; cw2 = o.w[2]; cw3 = o.w[3]; have = true;
#endif
    return (k & 1u) ? u01(o.w[2], o.w[3]) : u01(o.w[0], o.w[1]);
  }
};

// ------------------------------------------- FP64 approximations (mixed form)
// Mixed-form FP64 square roots, reciprocal square roots and reciprocals
// start from the hardware's FP64 approximations (PTX rsqrt.approx.ftz.f64 and
// rcp.approx.ftz.f64, about 20 correct bits: measured on B200 over 2^20
// log-uniform inputs in [1e-30, 2e30], largest relative error 2^-20.1 and
// 2^-20.0) and take one Newton-Raphson step with its second-order term
// (Markstein, IA-64 and Elementary Functions, 2000), which cubes the error:
// measured largest relative error of the results 2^-52.7 and 2^-53.0.  Not
// correctly rounded, which the mixed form does not need (the FP64 form uses
// the IEEE operations).  The approximations take the FP64 operand whole (no
// FP32 conversion, so no range limit short of subnormals, which they flush
// to zero).

// 1/sqrt(a), a > 0 normal
__device__ __forceinline__ double rsqrt_nr(double a)
{
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(a));
  const double h = fma(-a * y, y, 1.0);        // 1 - a y^2
  return fma(y * h, fma(0.375, h, 0.5), y);    // y (1 + h/2 + 3 h^2/8)
}

// sqrt(a), a >= 0 (0 for 0, NaN for a < 0)
__device__ __forceinline__ double sqrt_nr(double a)
{
  const double r = a * rsqrt_nr(a);
  return (a == 0.0) ? a : r;
}

// 1/a, a normal
__device__ __forceinline__ double rcp_nr(double a)
{
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(a));
  const double e = fma(-a, y, 1.0);            // 1 - a y
  return fma(y, fma(e, e, e), y);              // y (1 + e + e^2)
}

// ---------------------------------------------------------------- locate
struct DevLoc {
  int32_t n, type;
  double min, del;
  const double* right;  // device pointer, n walls
  float inv_step;       // log grids: 1/log2(1+del); lin grids: 1/del (index estimate only)
  float lmin_step;      // log grids: log2(min) * inv_step (index estimate without a division)
  float inv_min;        // log grids: 1/min (the mixed form's estimate, without cancellation)
};

__device__ __forceinline__ int upper_bound_dev(const double* __restrict__ a, int n, double v)
{
  int lo = 0, hi = n;
  while (lo < hi) {
    const int m = (lo + hi) >> 1;
    if (__ldg(a + m) <= v) lo = m + 1; else hi = m;
  }
  return lo;
}

template <typename T>
__device__ __forceinline__ int upper_bound_t(const T* __restrict__ a, int n, double v)
{
  int lo = 0, hi = n;
  while (lo < hi) {
    const int m = (lo + hi) >> 1;
    if ((double)__ldg(a + m) <= v) lo = m + 1; else hi = m;
  }
  return lo;
}

// Two-level upper_bound over a CDF row: `coarse[k]` holds row[min(k*S+S-1,
// n-1)], the last value of block k.  The first block whose last value
// exceeds v holds the first element > v, so the result equals
// upper_bound(row, row+n, v) exactly, with log2(n/S) searches in a table
// small enough to stay in L1 and one short scan within a single block.
constexpr int CDF_STRIDE = 32;

template <typename T>
__device__ __forceinline__ int upper_bound_2level(const T* __restrict__ row, const T* __restrict__ coarse, int n,
                                                  int nblk, double v)
{
  const int k = upper_bound_t<T>(coarse, nblk, v);
  if (k >= nblk) return n;
  const int lo = k * CDF_STRIDE;
  const int hi = min(lo + CDF_STRIDE, n);
  return lo + upper_bound_t<T>(row + lo, hi - lo, v);
}

// upper_bound over a CDF row through its guide table: with guide[k] =
// upper_bound(row, k / G) for a power of two G, the answer for u lies in
// [guide[k], guide[k+1]] where k = floor(u G) (exact: u G is a scaling by a
// power of two), so a binary search over that short range returns exactly
// upper_bound(row, row + n, u).
template <typename T>
__device__ __forceinline__ int upper_bound_guided(const T* __restrict__ row, const uint16_t* __restrict__ guide, int G,
                                                  double u)
{
  const int k = (int)(u * (double)G);
  int lo = __ldg(guide + k), hi = __ldg(guide + k + 1);
  while (lo < hi) {
    const int m = (lo + hi) >> 1;
    if ((double)__ldg(row + m) <= u) lo = m + 1; else hi = m;
  }
  return lo;
}

// locate_array::locate (src/utils/locate_array.cpp:191-218): fast lin/log
// index corrected by a binary search unless it is 0 or n
__device__ __forceinline__ int loc_locate(const DevLoc& g, double x)
{
  if (g.n == 1) return 0;
  if (x >= __ldg(g.right + g.n - 1)) return g.n;
  if (x < g.min) return 0;
  int ind;
  if (g.type == LOC_FLEX) return upper_bound_dev(g.right, g.n, x);
  else if (g.type == LOC_LIN) ind = (int)floor((x - g.min) / g.del);
  else if (g.type == LOC_LOG) ind = (int)floor(log(x / g.min) / log(1 + g.del));
  else return 0;
  if (ind != 0 && ind != g.n) {
    const double left = __ldg(g.right + ind - 1), right = __ldg(g.right + ind);
    if (left > x || right <= x) ind = upper_bound_dev(g.right, g.n, x);
  }
  return ind;
}

__device__ __forceinline__ int loc_within(const DevLoc& g, double x)
{
  const int i = loc_locate(g, x);
  return i == g.n ? g.n - 1 : i;
}

// locate_within_bounds on a lin/log grid without the FP64 logarithm.  For
// a result of 2 or more the reference's answer is the exact upper_bound bin
// (its fast index is corrected by a binary search unless it is 0 or n, and
// n maps to n-1), found here from a float estimate and a wall check.  For
// bins 0 and 1 the reference's own fast index is evaluated, because an
// uncorrected fast index of 0 is what it returns.
// NODIV: the log-grid estimate log2(x) * inv_step - lmin_step instead of
// log2(x / min) * inv_step (no FP64 division; the wall checks below make
// the result the same).
template <bool NODIV = false>
__device__ __forceinline__ int loc_within_fast(const DevLoc& g, double x)
{
  if (g.n == 1) return 0;
  if (x >= __ldg(g.right + g.n - 1)) return g.n - 1;
  if (x < g.min) return 0;
  if (g.type != LOC_LOG && g.type != LOC_LIN) return loc_within(g, x);
  float est;
  if (g.type == LOC_LOG) est = NODIV ? __log2f((float)x) * g.inv_step - g.lmin_step
                                     : __log2f((float)(x / g.min)) * g.inv_step;
  else est = (float)(x - g.min) * g.inv_step;
  int i = (int)est;
  i = max(0, min(i, g.n - 1));
  while (i < g.n - 1 && x >= __ldg(g.right + i)) ++i;
  while (i > 0 && x < __ldg(g.right + i - 1)) --i;
  if (i <= 1) {
    const int fast = (g.type == LOC_LOG) ? (int)floor(log(x / g.min) / log(1 + g.del))
                                         : (int)floor((x - g.min) / g.del);
    if (fast == 0) return 0;
  }
  return i;
}

// The mixed form's bin lookup on log and linear grids: the FP32 index
// estimate (log2(x/min)/log2(1+del), or (x-min)/del) is the bin unless it
// lies within a margin of a wall, where the walls decide (loc_within_fast).
// The estimate's error is below ~4e-7 n bins for an n-bin grid (__log2f's
// 2 ulp, the FP32 roundings of x/min, 1/log2(1+del) and an index below n):
// 1.5e-3 of a bin on the 4096-bin Type Ia grid, against a margin of
// max(1/64, n 2^-18) of a bin, ten times larger.  The answer is the bin the
// walls give, and the wall loads, two dependent memory round trips, are
// left out for ~97% of the Type Ia lookups.
__device__ __forceinline__ int loc_within_mixed(const DevLoc& g, double x)
{
  if (g.n == 1) return 0;
  if (g.type != LOC_LOG && g.type != LOC_LIN) return loc_within_fast<true>(g, x);
  float est = (g.type == LOC_LOG) ? __log2f((float)x * g.inv_min) * g.inv_step : (float)(x - g.min) * g.inv_step;
  est = fminf(fmaxf(est, 0.0f), (float)g.n - 0.5f);  // below the grid: bin 0; above: bin n-1
  const int i = (int)est;
  const float fr = est - (float)i;
  const float margin = fmaxf(0.015625f, (float)g.n * 3.814697265625e-6f);
  if (fr > margin && fr < 1.0f - margin) return i;
  return loc_within_fast<true>(g, x);
}

__device__ __forceinline__ double loc_left(const DevLoc& g, int i) { return i == 0 ? g.min : __ldg(g.right + i - 1); }
__device__ __forceinline__ double loc_delta(const DevLoc& g, int i)
{
  return i == 0 ? __ldg(g.right) - g.min : __ldg(g.right + i) - __ldg(g.right + i - 1);
}
__device__ __forceinline__ double loc_center(const DevLoc& g, int i)
{
  return i == 0 ? 0.5 * (g.min + __ldg(g.right)) : 0.5 * (__ldg(g.right + i - 1) + __ldg(g.right + i));
}
// locate_array::sample (locate_array.cpp:237-242)
__device__ __forceinline__ double loc_sample(const DevLoc& g, int i, double r)
{
  if (g.n == 1) return 0;
  if (i == 0) return g.min + (__ldg(g.right) - g.min) * r;
  const double l = __ldg(g.right + i - 1);
  return l + (__ldg(g.right + i) - l) * r;
}

}  // namespace sed
