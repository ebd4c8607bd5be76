// transport_kernel.cu -- the persistent Monte Carlo packet kernel.
//
// One thread owns one packet at a time and pulls the next packet index from
// a global counter when its packet escapes, is absorbed or stops, so every
// lane stays busy no matter how uneven packet histories are.  Emission is
// fused in: a packet is created in registers from its first Philox draws
// (emit_inner_source, src/transport/emission.cpp:370-485) and never stored.
// Each loop iteration is one segment of propagate_monte_carlo
// (src/transport/transport.cpp:260-484).  Packet state stays in registers;
// the opacity table is a zone-major array of {abs, scat} pairs (one 16 B or
// 8 B load per segment); zone-scalar tallies go to per-block shared memory
// when the grid has few zones, J_nu goes straight to global FP64 atomics.
//
// Arithmetic follows the reference expression by expression; this file is
// compiled without FMA contraction so products and sums round as written.
#include <cfloat>
#include <cmath>
#include "sed_internal.h"

namespace sed {

namespace {

struct Pkt {
  double x[3], D[3];
  double t, e, nu, dvds;
  int32_t ind;
};

// ----------------------------------------------------------- geometry
// grid_1D_sphere::get_zone (src/grid/grid_1D_sphere.cpp:494-505) and
// grid_3D_cart::get_zone (src/grid/grid_3D_cart.cpp:363-390)
template <int GRID>
__device__ __forceinline__ int get_zone(const GridDev& G, const double* x)
{
  if constexpr (GRID == 0) {
    const double r = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
    if (r < G.r_out.min) return -1;
    if (r >= __ldg(G.r_out.right + G.r_out.n - 1)) return -2;
    return loc_within(G.r_out, r);
  } else {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      if (x[a] < G.ax[a].min) return -2;
      if (x[a] > __ldg(G.ax[a].right + G.ax[a].n - 1)) return -2;
    }
    const int i = loc_within(G.ax[0], x[0]);
    const int j = loc_within(G.ax[1], x[1]);
    const int k = loc_within(G.ax[2], x[2]);
    return i * G.ny * G.nz + j * G.nz + k;
  }
}

// grid_1D_sphere::get_next_zone (grid_1D_sphere.cpp:510-590) and
// grid_3D_cart::get_next_zone (grid_3D_cart.cpp:396-469)
// (1D: rsq = x.x and xdotD = D.x come from the caller; FAST, the mixed
// form: the 3D wall distances from the FP64 reciprocal approximation)
template <int GRID, bool FAST = false>
__device__ __forceinline__ int get_next_zone(const GridDev& G, const double* x, const double* D, int i,
                                             double r_core, double rsq, double xdotD, double* l)
{
  if constexpr (GRID == 0) {
    const double r_o = __ldg(G.r_out.right + i);
    const double l_out = -1 * xdotD + sqrt(xdotD * xdotD + r_o * r_o - rsq);
    double r_in;
    int ind_in;
    if (i != 0) { r_in = __ldg(G.r_out.right + i - 1); ind_in = i - 1; }
    else { r_in = G.r_out.min; ind_in = -1; }
    if (r_core >= r_in) { r_in = r_core; ind_in = -1; }
    double l_in;
    if ((i == 0) && (r_in == 0)) l_in = -1;
    // moving outward the reference's -x.D - sqrt(rad) is negative, and only
    // its sign is used below: the square root is skipped, the branch is the same
    else if (xdotD > 0) l_in = -1;
    else {
      const double rad = xdotD * xdotD + r_in * r_in - rsq;
      l_in = (rad < 0) ? -1 : -1 * xdotD - sqrt(rad);
    }
    constexpr double tiny_offset = 1 + 1e-6;
    int ind;
    if ((l_out < l_in) || (l_in < 0)) {
      ind = i + 1;
      if (ind == G.nzones) { ind = -2; *l = l_out / tiny_offset; }
      else *l = l_out * tiny_offset;
    } else {
      ind = ind_in;
      *l = (ind_in == -1) ? l_in / tiny_offset : l_in * tiny_offset;
    }
    return ind;
  } else {
    const int nyz = G.ny * G.nz;
    const int idx3[3] = {i / nyz, (i / G.nz) % G.ny, i % G.nz};
    const double tiny = 1e-10;
    double len[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const double dd = loc_delta(G.ax[a], idx3[a]);
      const double bn = (D[a] > 0) ? __ldg(G.ax[a].right + idx3[a]) + dd * tiny : loc_left(G.ax[a], idx3[a]) - dd * tiny;
      if constexpr (FAST) len[a] = (D[a] != 0.0) ? (bn - x[a]) * rcp_nr(D[a]) : (double)INFINITY;
      else len[a] = (bn - x[a]) / D[a];
    }
    int d[3] = {0, 0, 0};
    if ((len[0] < len[1]) && (len[0] < len[2])) { d[0] = (D[0] < 0) ? -1 : 1; *l = len[0]; }
    else if (len[1] < len[2]) { d[1] = (D[1] < 0) ? -1 : 1; *l = len[1]; }
    else { d[2] = (D[2] < 0) ? -1 : 1; *l = len[2]; }
    const int nx_ = idx3[0] + d[0], ny_ = idx3[1] + d[1], nz_ = idx3[2] + d[2];
    if (nx_ < 0 || nx_ > G.nx - 1) return -2;
    if (ny_ < 0 || ny_ > G.ny - 1) return -2;
    if (nz_ < 0 || nz_ > G.nz - 1) return -2;
    return nx_ * nyz + ny_ * G.nz + nz_;
  }
}

// get_velocity (grid_1D_sphere.cpp:707-748, grid_3D_cart.cpp:513-521)
template <int GRID>
__device__ __forceinline__ void get_velocity(const GridDev& G, int i, const double* x, const double* D, double* v,
                                             double* dvds)
{
  if (G.homologous) {
    v[0] = x[0] / G.t_grid;
    v[1] = x[1] / G.t_grid;
    v[2] = x[2] / G.t_grid;
    *dvds = 1.0 / G.t_grid;
    return;
  }
  if constexpr (GRID == 0) {
    // a diffusion leak past the outer wall leaves the zone index one past
    // the grid (discrete_diffusion.cpp:324-328), where the reference reads
    // past its zone array; the last zone's velocity field is used instead
    if (i >= G.nzones) i = G.nzones - 1;
    const double rr = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
    double v_0, r_0;
    if (i == 0) { v_0 = 0; r_0 = G.r_out.min; }
    else { v_0 = __ldg(G.v_r + i - 1); r_0 = __ldg(G.r_out.right + i - 1); }
    const double dr = rr - r_0;
    const double dv_dr = (__ldg(G.v_r + i) - v_0) / (__ldg(G.r_out.right + i) - r_0);
    const double vv = v_0 + dv_dr * dr;
    const double Ddr = (D[0] * x[0] + D[1] * x[1] + D[2] * x[2]) / rr;
    v[0] = x[0] / rr * vv;
    v[1] = x[1] / rr * vv;
    v[2] = x[2] / rr * vv;
    *dvds = Ddr * Ddr * (dv_dr - vv / rr) + vv / rr;
    if (rr == 0) { v[0] = v[1] = v[2] = 0; *dvds = dv_dr; }
  } else {
    v[0] = v[1] = v[2] = 0;
    *dvds = 0;
  }
}

// transport::do_dshift lab -> comoving (src/transport/relativity.cpp:14-43)
template <int GRID>
__device__ __forceinline__ double dshift_lab_to_comoving(const GridDev& G, Pkt& p)
{
  double v[3], dvds;
  get_velocity<GRID>(G, p.ind, p.x, p.D, v, &dvds);
  const double beta2 = (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) / C_LIGHT / C_LIGHT;
  const double vdd = v[0] * p.D[0] + v[1] * p.D[1] + v[2] * p.D[2];
  const double gamma = 1.0 / sqrt(1 - beta2);
  p.dvds = dvds;
  return gamma * (1 - vdd / C_LIGHT);
}

// transport::lorentz_transform(p, 1) (relativity.cpp:84-127)
template <int GRID>
__device__ __forceinline__ void comoving_to_lab(const GridDev& G, Pkt& p)
{
  double v[3], dvds;
  get_velocity<GRID>(G, p.ind, p.x, p.D, v, &dvds);
  v[0] *= -1; v[1] *= -1; v[2] *= -1;
  const double beta2 = (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) / C_LIGHT / C_LIGHT;
  const double vdd = v[0] * p.D[0] + v[1] * p.D[1] + v[2] * p.D[2];
  const double gamma = 1.0 / sqrt(1 - beta2);
  const double dshift = gamma * (1 - vdd / C_LIGHT);
  p.dvds = dvds;
  p.e *= dshift;
  p.nu *= dshift;
  const double f = (1 - gamma * vdd / C_LIGHT / (gamma + 1));
  p.D[0] = 1.0 / dshift * (p.D[0] - gamma * v[0] / C_LIGHT * f);
  p.D[1] = 1.0 / dshift * (p.D[1] - gamma * v[1] / C_LIGHT * f);
  p.D[2] = 1.0 / dshift * (p.D[2] - gamma * v[2] / C_LIGHT * f);
  const double norm = p.D[0] * p.D[0] + p.D[1] * p.D[1] + p.D[2] * p.D[2];
  p.D[0] /= norm;
  p.D[1] /= norm;
  p.D[2] /= norm;
}

// ----------------------------------------------------------- batches
// get_next_zone of grid_1D_sphere for a zone of one model of a batch.  The
// model's walls sit in the concatenated r_out array; per zone the host has
// precomputed what the reference derives from the zone index, r_min and the
// core radius (grid_1D_sphere.cpp:527-546): the inner wall after the core
// substitution, the inner neighbour (-1 at the core or the model's first
// zone), the outer neighbour (-2 past the model's last zone) and whether
// zone 0 starts at r = 0.  Values and branches are the single-model ones.
__device__ __forceinline__ int get_next_zone_batch(const StepArgs& A, const GridDev& G, int i, double rsq,
                                                   double xdotD, double* l)
{
  const double r_o = __ldg(G.r_out.right + i);
  const double l_out = -1 * xdotD + sqrt(xdotD * xdotD + r_o * r_o - rsq);
  const int4 nb = __ldg(A.zone_nbr + i);
  const double r_in = __ldg(A.zone_rin + i);
  double l_in;
  if (nb.z) l_in = -1;
  else if (xdotD > 0) l_in = -1;  // outward: negative in the reference too, only its sign is used
  else {
    const double rad = xdotD * xdotD + r_in * r_in - rsq;
    l_in = (rad < 0) ? -1 : -1 * xdotD - sqrt(rad);
  }
  const double tiny_offset = 1 + 1e-6;
  int ind;
  if ((l_out < l_in) || (l_in < 0)) {
    ind = nb.y;
    *l = (ind == -2) ? l_out / tiny_offset : l_out * tiny_offset;
  } else {
    ind = nb.x;
    *l = (ind == -1) ? l_in / tiny_offset : l_in * tiny_offset;
  }
  return ind;
}

// model holding global queue entry `q`: the last model whose first entry is
// at or before q (models without packets share their successor's offset)
__device__ __forceinline__ int find_model(const BatchModel* __restrict__ M, int n, int64_t q)
{
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if ((int64_t)__ldg(reinterpret_cast<const long long*>(&M[mid].pkt_off)) <= q) lo = mid + 1;
    else hi = mid;
  }
  return lo - 1;
}

// grid_1D_sphere::get_zone over one model's slice of the walls
struct BatchZoneOf {
  DevLoc slice;  // n = model zones, min = r_min, right = first wall of the model
  int zone_off;
  __device__ int operator()(const double* x) const
  {
    const double r = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
    if (r < slice.min) return -1;
    if (r >= __ldg(slice.right + slice.n - 1)) return -2;
    return zone_off + loc_within(slice, r);
  }
};

template <int GRID>
struct GridZoneOf {
  const GridDev& G;
  __device__ int operator()(const double* x) const { return get_zone<GRID>(G, x); }
};

// upper_bound(CDF row of zone iz, u): through the guide table when there is
// one, else the two-level search over the coarse table
template <typename CT>
__device__ __forceinline__ int cdf_row_sample(const StepArgs& A, int iz, double u)
{
  const int nn = A.nu.n;
  const CT* row = reinterpret_cast<const CT*>(A.cdf) + (size_t)iz * nn;
  if (A.cdf_guide) return upper_bound_guided<CT>(row, A.cdf_guide + (size_t)iz * (A.guide_n + 1), A.guide_n, u);
  const CT* crow = reinterpret_cast<const CT*>(A.cdf_coarse) + (size_t)iz * A.n_coarse;
  return upper_bound_2level<CT>(row, crow, nn, A.n_coarse, u);
}

template <typename CT>
__device__ __forceinline__ int cdf_sample(const CT* __restrict__ y, int n, double u)
{
  if (n == 1) return 0;
  return upper_bound_t<CT>(y, n, u);
}

// transport::isotropic_scatter (src/transport/scatter.cpp:303-351)
template <int GRID, typename CT>
__device__ __forceinline__ void isotropic_scatter(const StepArgs& A, const GridDev& G, Pkt& p, PacketRng& rng,
                                                  int redist)
{
  double V[3], dvds;
  get_velocity<GRID>(G, p.ind, p.x, p.D, V, &dvds);
  const double vdotD = V[0] * p.D[0] + V[1] * p.D[1] + V[2] * p.D[2];
  const double beta2 = (V[0] * V[0] + V[1] * V[1] + V[2] * V[2]) / C_LIGHT / C_LIGHT;
  const double gamma = 1.0 / sqrt(1 - beta2);
  const double dshift_in = gamma * (1 - vdotD / C_LIGHT);
  p.e = p.e * dshift_in;
  p.nu = p.nu * dshift_in;
  const double mu = 1 - 2.0 * rng.next();
  const double phi = 2.0 * PI * rng.next();
  const double smu = sqrt(1 - mu * mu);
  double s, c;
  sincos(phi, &s, &c);
  const double Dn[3] = {smu * c, smu * s, mu};
  if (redist) {  // transport::sample_photon_frequency (emission.cpp:27-46)
    const int nn = A.nu.n;
    const double u = rng.next();
    // cdf_array::sample (src/transport/cdf_array.h:84-89): upper_bound
    const int inu = (nn == 1) ? 0 : cdf_row_sample<CT>(A, p.ind, u);
    p.nu = loc_sample(A.nu, inu, rng.next());
  }
  V[0] = -1 * V[0]; V[1] = -1 * V[1]; V[2] = -1 * V[2];
  const double vdp = (Dn[0] * V[0] + Dn[1] * V[1] + Dn[2] * V[2]);
  const double vd_out = gamma * (1 - vdp / C_LIGHT);
  const double f = (1 - gamma * vdp / C_LIGHT / (gamma + 1));
  p.D[0] = 1.0 / vd_out * (Dn[0] - gamma * V[0] / C_LIGHT * f);
  p.D[1] = 1.0 / vd_out * (Dn[1] - gamma * V[1] / C_LIGHT * f);
  p.D[2] = 1.0 / vd_out * (Dn[2] - gamma * V[2] / C_LIGHT * f);
  const double norm = sqrt(p.D[0] * p.D[0] + p.D[1] * p.D[1] + p.D[2] * p.D[2]);
  p.D[0] = p.D[0] / norm;
  p.D[1] = p.D[1] / norm;
  p.D[2] = p.D[2] / norm;
  p.e = p.e * vd_out;
  p.nu = p.nu * vd_out;
}

// ------------------------------------------------ mixed form, homologous flow
// The mixed form is held to the reference's spectra within Monte Carlo
// noise, not to its bits, so with homologous velocities v = x / t it
// evaluates the same FP64 transforms without divisions: beta = x / (c t),
// gamma = rsqrt(1 - beta^2), reciprocals and rsqrt for the normalisations.
// Position, time, frequency and the Lorentz transforms stay FP64.

// transport::do_dshift, lab -> comoving, from rsq = x.x and xdotD = D.x
__device__ __forceinline__ double dshift_fast(const StepArgs& A, double rsq, double xdotD)
{
  const double gamma = rsqrt_nr(fma(-rsq, A.inv_ct2, 1.0));
  return gamma * fma(-xdotD, A.inv_ct, 1.0);
}

// transport::isotropic_scatter (scatter.cpp:303-351), homologous flow
// Its deviates are the four words of one Philox block: mu, phi, the
// emissivity-CDF deviate and the position within the bin.
template <typename CT>
__device__ __forceinline__ void isotropic_scatter_fast(const StepArgs& A, Pkt& p, const uint4 w, int redist)
{
  const double b0 = p.x[0] * A.inv_ct, b1 = p.x[1] * A.inv_ct, b2 = p.x[2] * A.inv_ct;  // v / c
  const double bdotD = fma(b0, p.D[0], fma(b1, p.D[1], b2 * p.D[2]));
  const double gamma = rsqrt_nr(1 - fma(b0, b0, fma(b1, b1, b2 * b2)));
  const double dshift_in = gamma * (1 - bdotD);
  p.e = p.e * dshift_in;
  p.nu = p.nu * dshift_in;
  const double mu = 1 - 2.0 * w01(w.x);
  // the azimuth's sine and cosine in FP32 from the hardware's sincos on
  // [-pi, pi): phi - pi has sine -sin(phi) and cosine -cos(phi) (a direction
  // sample, not a frame transform; the transforms below and the
  // normalisation are FP64)
  const float phi = (float)(2.0 * PI * w01(w.y));
  const double smu = sqrt_nr(fma(-mu, mu, 1.0));
  float sf, cf;
  __sincosf(phi - (float)PI, &sf, &cf);
  sf = -sf;
  cf = -cf;
  const double Dn[3] = {smu * (double)cf, smu * (double)sf, mu};
  if (redist) {  // transport::sample_photon_frequency (emission.cpp:27-46)
    const int nn = A.nu.n;
    const double u = w01(w.z);
    const int inu = (nn == 1) ? 0 : cdf_row_sample<CT>(A, p.ind, u);
    p.nu = loc_sample(A.nu, inu, w01(w.w));
  }
  // comoving -> lab with the velocity reversed: beta' = -beta
  const double bdp = -fma(b0, Dn[0], fma(b1, Dn[1], b2 * Dn[2]));
  const double vd_out = gamma * (1 - bdp);
  const double f = fma(-gamma * bdp, rcp_nr(gamma + 1), 1.0);
  const double gf = gamma * f;
  const double inv_vd = rcp_nr(vd_out);
  p.D[0] = inv_vd * fma(gf, b0, Dn[0]);
  p.D[1] = inv_vd * fma(gf, b1, Dn[1]);
  p.D[2] = inv_vd * fma(gf, b2, Dn[2]);
  const double inv_norm = rsqrt_nr(fma(p.D[0], p.D[0], fma(p.D[1], p.D[1], p.D[2] * p.D[2])));
  p.D[0] *= inv_norm;
  p.D[1] *= inv_norm;
  p.D[2] *= inv_norm;
  p.e = p.e * vd_out;
  p.nu = p.nu * vd_out;
}

// transport::emit_inner_source for one packet (emission.cpp:395-480).  The
// source (core radius, packet energy, core CDF) and the zone lookup are
// arguments so one model of a batch can supply its own.
// Deviates of the emission: one per draw (the reference's layout), or the
// 32-bit words of consecutive Philox blocks (the mixed form's layout).
struct DrawNext {
  PacketRng& r;
  __device__ double operator()() { return r.next(); }
};
struct DrawWords {
  PacketRng& r;
  uint4 b;
  int used = 4;
  __device__ uint32_t word()
  {
    if (used == 4) { b = r.block(); used = 0; }
    const uint32_t w = (used == 0) ? b.x : (used == 1) ? b.y : (used == 2) ? b.z : b.w;
    ++used;
    return w;
  }
  __device__ double operator()() { return w01(word()); }
};

template <int GRID, class ZoneOf, class Draw>
__device__ __forceinline__ void emit_core(const StepArgs& A, const GridDev& G, Pkt& p, Draw& rng, double rc,
                                          double Ep, const double* core_cdf, const ZoneOf& zone_of)
{
  if (rc == 0) {
    p.x[0] = p.x[1] = p.x[2] = 0;
    const double mu = 1 - 2.0 * rng();
    const double phi = 2.0 * PI * rng();
    const double smu = sqrt(1 - mu * mu);
    double s, c;
    sincos(phi, &s, &c);
    p.D[0] = smu * c;
    p.D[1] = smu * s;
    p.D[2] = mu;
  } else {
    const double phi_core = 2 * PI * rng();
    double sinp, cosp;
    sincos(phi_core, &sinp, &cosp);
    const double cost = 1 - 2.0 * rng();
    const double sint = sqrt(1 - cost * cost);
    const double a_phot = rc + rc * 1e-10;
    p.x[0] = a_phot * sint * cosp;
    p.x[1] = a_phot * sint * sinp;
    p.x[2] = a_phot * cost;
    const double phi_loc = 2 * PI * rng();
    const double cost_loc = sqrt(rng());
    const double sint_loc = sqrt(1 - cost_loc * cost_loc);
    double sl, cl;
    sincos(phi_loc, &sl, &cl);
    const double D_xl = sint_loc * cl, D_yl = sint_loc * sl, D_zl = cost_loc;
    p.D[0] = cost * cosp * D_xl - sinp * D_yl + sint * cosp * D_zl;
    p.D[1] = cost * sinp * D_xl + cosp * D_yl + sint * sinp * D_zl;
    p.D[2] = -sint * D_xl + cost * D_zl;
  }
  p.e = Ep;
  if (A.core_freq > 0) p.nu = A.core_freq;
  else {
    const int inu = cdf_sample<double>(core_cdf, A.nu.n, rng());
    p.nu = loc_sample(A.nu, inu, rng());
    p.e /= 1.0;  // emissivity_weight_ is 1 (transport_init.cpp:322-332)
  }
  p.ind = zone_of(p.x);
  // the reference asserts p.ind >= 0 here (relativity.cpp:86); homologous
  // velocities do not depend on the zone, other velocity fields need one
  if (G.homologous || p.ind >= 0) comoving_to_lab<GRID>(G, p);
  p.t = A.t_now + rng() * A.dt;
}

// spectrum_array::count (src/transport/spectrum_array.cpp:215-246)
// Returns the spectrum index the packet was counted in, -1 when dropped.
__device__ __forceinline__ int64_t spectrum_count(const StepArgs& A, double* flux, double* click, double t, double w,
                                                  double E, const double* D)
{
  const double mu = D[2];
  double phi = atan2(D[1], D[0]);
  if (phi < 0) phi += 2. * PI;
  const int t_bin = loc_locate(A.st, t);
  int l_bin = loc_locate(A.sn, w);
  const int m_bin = loc_locate(A.sm, mu);
  const int p_bin = loc_locate(A.sp, phi);
  if (l_bin < 0) l_bin = 0;
  if (l_bin >= A.sn.n) l_bin = 0;
  if ((t_bin < 0) || (m_bin < 0) || (p_bin < 0)) return -1;
  if (t_bin >= A.st.n || m_bin >= A.sm.n || p_bin >= A.sp.n) return -1;
  const int64_t ind = t_bin * A.a1 + l_bin * A.a2 + m_bin * A.a3 + p_bin;
  atomicAdd(flux + ind, E);
  atomicAdd(click + ind, 1.0);
  return ind;
}

__device__ __forceinline__ unsigned long long warp_sum(unsigned long long v)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Block size and minimum resident blocks per SM of the differentiable-
// transport kernels.  The packet kernel is latency bound (dependent FP64
// chains, L2 table loads): 24-32 warps per SM at 64-80 registers beat fewer
// warps with more registers (2 blocks of 256 at 120 registers ran the Type
// Ia step 19% slower), despite a small register spill.
#ifndef SED_PROP_THREADS
#define SED_PROP_THREADS 128
#endif
// launch shape of the mixed-form 1D kernel (propagate_mixed_kernel):
// 128 x 8 at 64 registers without spills, 32 warps per SM (Type Ia packet
// kernel 623 ms; 128 x 7 at 70 registers 638 ms; 128 x 9 at 56 registers
// spills 40 B and ran 676 ms)
#ifndef SED_MIXED_THREADS
#define SED_MIXED_THREADS 128
#endif
#ifndef SED_MIXED_MINB
#define SED_MIXED_MINB 8
#endif
#ifndef SED_PROP_MINB
#define SED_PROP_MINB 8
#endif

// BATCH = 1: the queue spans every packet of a batch of 1D models; a thread
// claims `queue_chunk` consecutive entries per pop, finds each entry's model
// and emits the packet from that model's source, Philox key and stream id;
// zone walks use the per-zone neighbour tables.  The step number is read
// from device memory so a captured graph can be replayed step after step.
// MODE 0 follows the reference's estimator.  MODE 1 (differentiable
// forward) samples interactions from the scattering opacity only and carries
// absorption as a continuous weight exp(-a dshift l) per segment, so for
// fixed deviates the path does not depend on the absorption opacity and the
// spectrum is a smooth function of it; tallies use the segment-averaged
// weight.  MODE 2 replays the escaped packets of a MODE-1 launch (same
// deviates, same path) and adds -w a0 dshift l per segment into the
// gradient with respect to the (zone, band) absorption factors, where w is
// the packet's escaping energy times d(loss)/d(its spectrum bin).
// FAST (mixed form on a homologous grid): the division-free transforms above.
// discrete diffusion (1D spheres, FP64 expressions), defined with the
// gamma-ray helpers below
template <typename OT>
__device__ bool ddmc_zone(const StepArgs& A, const GridDev& G, const OT* __restrict__ opac, Pkt& p);
template <typename OT, typename CT>
__device__ int ddmc_event(const StepArgs& A, const GridDev& G, const OT* __restrict__ opac, Pkt& p, PacketRng& rng,
                          double& dt_remaining, double& acc_eabs, unsigned long long& n_scat,
                          unsigned long long& n_cap);
__device__ void ddmc_move_across(const StepArgs& A, const GridDev& G, Pkt& p, PacketRng& rng, int new_ind,
                                 double sigma_i, double dr);
template <typename OT>
__device__ __forceinline__ int ddmc_opacity(const StepArgs& A, const OT* __restrict__ opac, int iz, double nu_cmf,
                                            double* op, double* eps);

template <typename OT>
__device__ int imd_event(const StepArgs& A, const GridDev& G, Pkt& p, PacketRng& rng, double* t_eabs,
                         unsigned long long& n_cap);
// DD: discrete diffusion on (transport_use_ddmc = 1 IMD or 2 DDMC; 1D, FP64 expressions)
template <int GRID, typename OT, typename CT, int BATCH, int MODE, bool FAST, int THREADS, int MINB, bool DD = false>
__global__ void __launch_bounds__(THREADS, MINB) propagate_kernel(const StepArgs A, const GridDev G)
{
  extern __shared__ double s_tal[];  // [5][nz] when A.smem_zones
  const int nz = G.nzones;
  const int nn = A.nu.n;
  const int nj = A.store_Jnu ? nn : 1;
  if (A.smem_zones) {
    for (int i = threadIdx.x; i < 5 * nz; i += blockDim.x) s_tal[i] = 0.0;
    __syncthreads();
  }
  double* t_eabs = A.smem_zones ? s_tal : A.e_abs;
  double* t_fx = A.smem_zones ? s_tal + nz : A.fx;
  double* t_fy = A.smem_zones ? s_tal + 2 * nz : A.fy;
  double* t_fz = A.smem_zones ? s_tal + 3 * nz : A.fz;
  double* t_fr = A.smem_zones ? s_tal + 4 * nz : A.fr;
  if (!A.smem_zones && A.n_rep > 0) {
    // the zones of the one or two models in flight take the atomics of
    // every block: blocks spread them over n_rep copies
    double* base = A.zone_rep + (size_t)(blockIdx.x % A.n_rep) * 5 * nz;
    t_eabs = base; t_fx = base + nz; t_fy = base + 2 * nz; t_fz = base + 3 * nz; t_fr = base + 4 * nz;
  }
  const OT* __restrict__ opac = reinterpret_cast<const OT*>(A.opac);
  // the mixed form takes the division-free transforms on homologous grids;
  // the FP64 form keeps the reference's expressions
  constexpr bool fast = FAST;
  const int64_t limit = A.max_segments > 0 ? A.max_segments : 10000000;
  // deviates (per-draw layout) or Philox blocks (word layout) the emission uses
  uint32_t K = (A.core_radius == 0 ? 2u : 4u) + (A.core_freq > 0 ? 0u : 2u) + 1u;
  if (FAST) K = (K + 3u) / 4u;
  uint32_t step = A.step;
  if constexpr (BATCH) step = *A.step_dev;
  // batch: claimed queue entries [q_next, q_end), the current packet's model,
  // and escapes counted per model until the model changes
  int64_t q_next = 0, q_end = 0;
  int m = 0, esc_model = -1;
  unsigned long long esc_count = 0;
  // adjoint replay: the packet's weight and Jacobian row, and the sum over
  // consecutive segments in one (zone, band) before its atomic add
  double adj_w = 0, acc_g = 0;
  int64_t adj_row = 0, acc_key = -1;

  unsigned long long n_esc = 0, n_abs = 0, n_stop = 0, n_seg = 0, n_scat = 0, n_lim = 0;
  // One loop iteration is either one segment of the lane's packet or, when
  // that packet has finished, its bookkeeping and the emission of the next
  // packet.  A lane therefore refills as soon as its packet ends instead of
  // idling until the longest packet of its warp is done.
  Pkt p;
  PacketRng rng;
  int fate = ABSORBED;  // no packet yet
  bool have = false;    // a finished packet awaits its bookkeeping
  unsigned long long pid = 0;
  int64_t seg = 0;
  // zone-scalar tallies of the packet's current zone, kept in registers
  // while the packet stays in that zone and added to the shared/global
  // tally when it leaves (the same terms, summed per visit first)
  int acc_zone = -1;
  double acc_eabs = 0, acc_fx = 0, acc_fy = 0, acc_fz = 0, acc_fr = 0;
  // discrete diffusion: whether the last pass was a diffusion event (one
  // call of discrete_diffuse_DDMC) and the time that call has left
  bool dd_call = false;
  double dd_rem = 0;
  unsigned long long n_ddcap = 0, n_imdcap = 0;
  for (;;) {
    if (fate != MOVING) {
      if (have && MODE == 2) {
        if (acc_key >= 0) atomicAdd(A.adj_out + acc_key, -adj_w * acc_g);
        n_seg += seg;
        have = false;
      }
      if (have) {
        if (acc_zone >= 0) {
          atomicAdd(t_eabs + acc_zone, acc_eabs);
          if (A.tally_forces) {
            atomicAdd(t_fx + acc_zone, acc_fx);
            atomicAdd(t_fy + acc_zone, acc_fy);
            atomicAdd(t_fz + acc_zone, acc_fz);
            atomicAdd(t_fr + acc_zone, acc_fr);
          }
        }
        n_seg += seg;
        if (fate == ESCAPED) {
          const double t_obs = p.t - (p.x[0] * p.D[0] + p.x[1] * p.D[1] + p.x[2] * p.D[2]) / C_LIGHT;
          if constexpr (BATCH) {
            const int64_t so = A.models[m].spec_off;
            spectrum_count(A, A.flux + so, A.click + so, t_obs, p.nu, p.e, p.D);
            if (m != esc_model) {
              if (esc_model >= 0) atomicAdd(A.model_escaped + esc_model, esc_count);
              esc_model = m;
              esc_count = 0;
            }
            ++esc_count;
          } else {
            const int64_t si = spectrum_count(A, A.flux, A.click, t_obs, p.nu, p.e, p.D);
            if constexpr (MODE == 1) {
              A.esc_bin[pid] = (int32_t)si;
              A.esc_e[pid] = p.e;
            }
          }
          p.t = t_obs;
          ++n_esc;
        } else if (fate == ABSORBED) {
          ++n_abs;
        } else {
          ++n_stop;
        }
        if constexpr (MODE == 1) {
          if (fate != ESCAPED) A.esc_bin[pid] = -1;
        }
        if (A.rec_fate) {
          A.rec_fate[pid] = fate;
          A.rec_ind[pid] = p.ind;
          A.rec_draws[pid] = (int32_t)(rng.n - K);
          if (A.rec_type) A.rec_type[pid] = TYPE_PHOTON;
          double* s = A.rec_state + pid * 9;
          s[0] = p.x[0]; s[1] = p.x[1]; s[2] = p.x[2];
          s[3] = p.D[0]; s[4] = p.D[1]; s[5] = p.D[2];
          s[6] = p.t; s[7] = p.e; s[8] = p.nu;
        }
        have = false;
      }
      if constexpr (BATCH) {
        if (q_next >= q_end) {
          q_next = (int64_t)atomicAdd(A.counters + C_QUEUE, (unsigned long long)A.queue_chunk);
          q_end = q_next + A.queue_chunk;
          if (q_end > A.n_packets) q_end = A.n_packets;
        }
        if (q_next >= A.n_packets) break;
        pid = (unsigned long long)q_next++;
        m = find_model(A.models, A.n_models, (int64_t)pid);
        const BatchModel& M = A.models[m];
        K = FAST ? (M.emit_draws + 3u) / 4u : M.emit_draws;
        rng.init(M.seed, (uint64_t)(M.first_pid + ((int64_t)pid - M.pkt_off)), step, 0);
        BatchZoneOf zf;
        zf.slice = G.r_out;
        zf.slice.n = M.n_zones;
        zf.slice.min = M.r_min;
        zf.slice.right = G.r_out.right + M.zone_off;
        zf.zone_off = M.zone_off;
        if constexpr (FAST) {
          DrawWords d{rng};
          emit_core<GRID>(A, G, p, d, M.core_radius, M.Ep, M.core_cdf, zf);
        } else {
          DrawNext d{rng};
          emit_core<GRID>(A, G, p, d, M.core_radius, M.Ep, M.core_cdf, zf);
        }
      } else {
        pid = atomicAdd(A.counters + C_QUEUE, 1ULL);
        if (pid >= (unsigned long long)A.n_packets) break;
        if (!BATCH && MODE == 0 && A.q_n != nullptr && (int64_t)pid >= A.n_core) {
          // a queued photon: a census photon (stream position 0), or an
          // optical photon of the radioactive source handed over by the
          // gamma-ray kernel with its position in its Philox stream
          const int64_t k = (int64_t)pid - A.n_core;
          const uint32_t qn = A.q_n[k];
          if (qn == RADIO_NO_PHOTON) continue;  // ended as a gamma-ray
          const double* q = A.q_state + (size_t)k * 9;
          p.x[0] = q[0]; p.x[1] = q[1]; p.x[2] = q[2];
          p.D[0] = q[3]; p.D[1] = q[4]; p.D[2] = q[5];
          p.t = q[6]; p.e = q[7]; p.nu = q[8];
          p.ind = A.q_ind[k];
          rng.init(A.seed, (uint64_t)(A.radio_first_pid + k), step, qn);
          K = 0;  // a radioactive packet records every deviate of its stream
          fate = MOVING;
          if (p.ind == -1) fate = ABSORBED;
          else if (p.ind == -2) fate = ESCAPED;
          seg = 0;
          dd_call = false;
          acc_zone = -1;
          acc_eabs = acc_fx = acc_fy = acc_fz = acc_fr = 0;
          have = true;
          if (fate != MOVING) continue;
          goto segment;
        }
        if constexpr (MODE == 2) {
          // only packets that reached the spectrum carry a gradient
          const int32_t sb = A.esc_bin[pid];
          adj_w = 0;
          if (sb >= 0) adj_w = A.adj_jacobian ? A.esc_e[pid] : A.adj_g[sb] * A.esc_e[pid];
          if (adj_w == 0) continue;  // fate is not MOVING: pull the next packet
          adj_row = A.adj_jacobian ? (int64_t)sb * nz * A.n_bands : 0;
          acc_key = -1;
          acc_g = 0;
        }
        rng.init(A.seed, (uint64_t)A.first_pid + pid, step, 0);
        if constexpr (FAST) {
          DrawWords d{rng};
          emit_core<GRID>(A, G, p, d, A.core_radius, A.Ep, A.core_cdf, GridZoneOf<GRID>{G});
        } else {
          DrawNext d{rng};
          emit_core<GRID>(A, G, p, d, A.core_radius, A.Ep, A.core_cdf, GridZoneOf<GRID>{G});
        }
      }
      // transport::propagate (transport.cpp:202-254): its get_zone of the
      // emitted position is the p.ind emit_core set (x has not moved since)
      fate = MOVING;
      if (p.ind == -1) fate = ABSORBED;
      else if (p.ind == -2) fate = ESCAPED;
      seg = 0;
      dd_call = false;
      acc_zone = -1;
      acc_eabs = acc_fx = acc_fy = acc_fz = acc_fr = 0;
      have = true;
      if (fate != MOVING) continue;
    }
  segment:
    {
      if (seg >= limit) { fate = STOPPED; ++n_lim; continue; }
      ++seg;
      const int iz = p.ind;
      if (MODE != 2 && iz != acc_zone) {
        if (acc_zone >= 0) {
          atomicAdd(t_eabs + acc_zone, acc_eabs);
          if (A.tally_forces) {
            atomicAdd(t_fx + acc_zone, acc_fx);
            atomicAdd(t_fy + acc_zone, acc_fy);
            atomicAdd(t_fz + acc_zone, acc_fz);
            atomicAdd(t_fr + acc_zone, acc_fr);
          }
        }
        acc_zone = iz;
        acc_eabs = acc_fx = acc_fy = acc_fz = acc_fr = 0;
      }
      if constexpr (DD) {
        // transport::propagate's zone test (transport.cpp:216-246): a photon
        // in a diffusive zone takes a diffusion event instead of a segment
        if (ddmc_zone<OT>(A, G, opac, p)) {
          if (A.use_ddmc == 1) {  // one IMD call (transport.cpp:236-237)
            fate = imd_event<OT>(A, G, p, rng, t_eabs, n_imdcap);
            continue;
          }
          if (!dd_call) { dd_rem = A.tstop - p.t; dd_call = true; }
          fate = ddmc_event<OT, CT>(A, G, opac, p, rng, dd_rem, acc_eabs, n_scat, n_ddcap);
          continue;
        }
        dd_call = false;
      }
      double d_bn = 0;
      double rsq, xdotD;
      if (fast) {
        rsq = fma(p.x[0], p.x[0], fma(p.x[1], p.x[1], p.x[2] * p.x[2]));
        xdotD = fma(p.D[0], p.x[0], fma(p.D[1], p.x[1], p.D[2] * p.x[2]));
      } else {
        rsq = (p.x[0] * p.x[0] + p.x[1] * p.x[1] + p.x[2] * p.x[2]);
        xdotD = (p.D[0] * p.x[0] + p.D[1] * p.x[1] + p.D[2] * p.x[2]);
      }
      int new_ind;
      if constexpr (BATCH) new_ind = get_next_zone_batch(A, G, iz, rsq, xdotD, &d_bn);
      else new_ind = get_next_zone<GRID, FAST>(G, p.x, p.D, iz, A.core_radius, rsq, xdotD, &d_bn);
      double dshift;
      if (fast) {
        dshift = dshift_fast(A, rsq, xdotD);
        p.dvds = A.inv_t;
      } else {
        dshift = dshift_lab_to_comoving<GRID>(G, p);
      }
      // a diffusive neighbour (transport.cpp:295-309)
      bool new_cell_ddmc = false;
      double sigma_new = 0, dr_new = 0;
      if constexpr (DD) {
        if (new_ind >= 0) {
          double e_new;
          ddmc_opacity<OT>(A, opac, new_ind, p.nu * dshift, &sigma_new, &e_new);
          dr_new = loc_delta(G.r_out, new_ind);
          new_cell_ddmc = sigma_new * dr_new > A.ddmc_tau;
        }
      }
      // transport::get_opacity (transport_opacity.cpp:268-299)
      const double nu_cmf = p.nu * dshift;
      const int i_nu = (fast) ? loc_within_fast<true>(A.nu, nu_cmf) : loc_within_fast<false>(A.nu, nu_cmf);
      const OT ab = opac[(size_t)iz * nn + i_nu];
      double a_opac = (double)ab.x;
      const double s_opac = A.omit_scat ? 0.0 : (double)ab.y;
      int band = 0;
      if constexpr (MODE != 0) {
        band = (int)(((int64_t)i_nu * A.n_bands) / nn);
        if (A.abs_scale) a_opac *= __ldg(A.abs_scale + (size_t)iz * A.n_bands + band);
      }
      const double op = a_opac + s_opac;
      double eps = 0;
      if (!(fast)) eps = (op == 0) ? 0 : a_opac / op;
      double d_nu;
      // distance to the bin's edge: only where the segment stops to look up
      // the next bin, so FP32 in the mixed form
      if (fast) d_nu = (double)__fdividef((float)(loc_delta(A.nu, i_nu) * A.ct), (float)p.nu);
      else {
        d_nu = loc_delta(A.nu, i_nu) / p.nu * C_LIGHT / p.dvds;
        if (p.dvds == 0) d_nu = INFINITY;
      }
      if (d_nu < 0) d_nu = -1 * d_nu;
      if (d_nu < d_bn) { d_bn = d_nu; new_ind = p.ind; }
      const double tot_lab = (MODE == 0 ? op : s_opac) * dshift;
      // mixed form: the segment's Philox block gives tau (53 bits) and the
      // two interaction tests
      uint4 blk = make_uint4(0u, 0u, 0u, 0u);
      double tau_r;
      if constexpr (FAST) {
        blk = rng.block();
        // -log(1 - u) in FP32: log1pf for u < 1/2, logf of the exact FP64
        // 1 - u above, so the relative error stays ~1e-7 over the whole range
        const double u = u01(blk.x, blk.y);
        tau_r = (double)((u < 0.5) ? -log1pf(-(float)u) : -logf((float)(1.0 - u)));
      } else {
        tau_r = -1.0 * log(1 - rng.next());
      }
      // mixed form: tau is an FP32 deviate, so its distance is formed in FP32
      // (the hardware's FP32 division, off the FP64 pipe); position and time
      // stay FP64
      double d_sc;
      if constexpr (FAST) d_sc = (double)__fdividef((float)tau_r, (float)tot_lab);
      else d_sc = tau_r / tot_lab;
      if (tot_lab == 0) d_sc = INFINITY;
      double d_tm = (A.tstop - p.t) * C_LIGHT;
      if (A.steady) d_tm = INFINITY;
      int event;
      double this_d;
      if ((d_sc < d_bn) && (d_sc < d_tm)) { event = 0; this_d = d_sc; }
      else if (d_bn < d_tm) { event = 1; this_d = d_bn; }
      else { event = 2; this_d = d_tm; }
      // tallies (transport.cpp:361-392)
      double this_E = p.e * this_d;
      double att = 1.0;
      if constexpr (MODE == 1) {
        // absorption over the segment: the weight falls by exp(-tau_a); the
        // tallies use its segment average e (1 - exp(-tau_a)) / tau_a
        const double tau_a = a_opac * dshift * this_d;
        att = exp(-tau_a);
        const double em1 = expm1(-tau_a);
        this_E = (tau_a > 0 ? p.e * (-em1 / tau_a) : p.e) * this_d;
      }
      if constexpr (MODE == 2) {
        if (A.adj_density) {
          // d / d ln rho of zone iz, opacity per mass held: the weight's log
          // falls by a dshift l, the sampled path's log-likelihood by
          // s dshift l per segment and rises by one per scattering
          const int64_t key = iz;
          if (key != acc_key) {
            if (acc_key >= 0) atomicAdd(A.adj_out + acc_key, -adj_w * acc_g);
            acc_key = key;
            acc_g = 0;
          }
          acc_g += (a_opac + s_opac) * dshift * this_d;
          if (event == 0) acc_g -= 1.0;
        } else {
          const int64_t key = adj_row + (int64_t)iz * A.n_bands + band;
          if (key != acc_key) {
            if (acc_key >= 0) atomicAdd(A.adj_out + acc_key, -adj_w * acc_g);
            acc_key = key;
            acc_g = 0;
          }
          acc_g += (double)ab.x * dshift * this_d;  // d(theta a0 dshift l) / d theta
        }
      }
      const double eps_imc = __ldg(A.eps_imc + iz);
      if constexpr (MODE == 0) {
        if (fast) acc_eabs += this_E * dshift * dshift * a_opac * eps_imc;
        else acc_eabs += this_E * dshift * (op) * eps * dshift * eps_imc;
      }
      if constexpr (MODE == 1) acc_eabs += this_E * dshift * a_opac * dshift * eps_imc;
      if constexpr (MODE != 2) atomicAdd(A.J + (size_t)iz * nj + (A.store_Jnu ? i_nu : 0), this_E);
      if (MODE != 2 && A.tally_forces) {
        const double w = this_E * dshift * op;
        acc_fx += w * p.D[0] * dshift;
        acc_fy += w * p.D[1] * dshift;
        acc_fz += w * p.D[2] * dshift;
        // |x| and x.D before the move: the segment's rsq and xdotD
        if (fast) acc_fr += w * xdotD * rsqrt(rsq) * dshift;
        else acc_fr += w * xdotD / sqrt(rsq) * dshift;
      }
      p.x[0] += this_d * p.D[0];
      p.x[1] += this_d * p.D[1];
      p.x[2] += this_d * p.D[2];
      constexpr double INV_C = 1.0 / C_LIGHT;
      if (fast) p.t = p.t + this_d * INV_C;
      else p.t = p.t + this_d / C_LIGHT;
      if constexpr (MODE == 1) p.e *= att;
      if (event == 1) {
        if (new_ind == -1) {
          if (A.bound_in_reflect) { p.D[0] *= -1; p.D[1] *= -1; p.D[2] *= -1; }
          else { p.ind = new_ind; fate = ABSORBED; }
        } else if (new_ind == -2) {
          if (A.bound_out_reflect) { p.D[0] *= -1; p.D[1] *= -1; p.D[2] *= -1; }
          else { p.ind = new_ind; fate = ESCAPED; }
        } else if (DD && new_cell_ddmc && new_ind != p.ind) {
          ddmc_move_across(A, G, p, rng, new_ind, sigma_new, dr_new);
        } else {
          p.ind = new_ind;
        }
      } else if (event == 0) {
        // transport::do_scatter (scatter.cpp:12-70): coherent scatter
        // (redist 0) or absorption with effective re-emission (redist 1);
        // one call site keeps a single inlined copy of isotropic_scatter
        ++n_scat;
        int redist = 0;
        if constexpr (MODE == 0) {
          if (fast) eps = (op == 0) ? 0 : a_opac / op;
          if (!((FAST ? w01(blk.z) : rng.next()) > eps)) {
            const double z2 = FAST ? w01(blk.w) : rng.next();
            if ((z2 > eps_imc) || A.radiative_eq) redist = 1;
            else fate = ABSORBED;
          }
        }
        if (fate == MOVING) {
          if (fast) isotropic_scatter_fast<CT>(A, p, rng.block(), redist);
          else isotropic_scatter<GRID, CT>(A, G, p, rng, redist);
        }
      } else {
        fate = STOPPED;
      }
    }
  }
  if constexpr (BATCH) {
    if (esc_model >= 0 && esc_count) atomicAdd(A.model_escaped + esc_model, esc_count);
  }
  // counters: warp reduction, one atomic per warp
  n_esc = warp_sum(n_esc); n_abs = warp_sum(n_abs); n_stop = warp_sum(n_stop);
  n_seg = warp_sum(n_seg); n_scat = warp_sum(n_scat); n_lim = warp_sum(n_lim);
  if constexpr (DD) { n_ddcap = warp_sum(n_ddcap); n_imdcap = warp_sum(n_imdcap); }
  if ((threadIdx.x & 31) == 0) {
    if (n_esc) atomicAdd(A.counters + C_ESCAPED, n_esc);
    if (n_abs) atomicAdd(A.counters + C_ABSORBED, n_abs);
    if (n_stop) atomicAdd(A.counters + C_STOPPED, n_stop);
    if (n_seg) atomicAdd(A.counters + C_SEGMENTS, n_seg);
    if (n_scat) atomicAdd(A.counters + C_SCATTERS, n_scat);
    if (n_lim) atomicAdd(A.counters + C_LIMIT, n_lim);
    if (n_ddcap) atomicAdd(A.counters + C_DDMC_CAP, n_ddcap);
    if (n_imdcap) atomicAdd(A.counters + C_IMD_CAP, n_imdcap);
  }
  if (MODE != 2 && A.smem_zones) {
    __syncthreads();
    double* g[5] = {A.e_abs, A.fx, A.fy, A.fz, A.fr};
    for (int i = threadIdx.x; i < 5 * nz; i += blockDim.x) {
      const double v = s_tal[i];
      if (v != 0.0 || isnan(v)) atomicAdd(g[i / nz] + (i % nz), v);
    }
  }
}

// reduce_radiation normalisation (src/transport/transport_mpi.cpp:415-441)
// of zone iz, after the steady-state luminosity rescale (transport.cpp:94-115)
// by `fac` when do_rescale.  Run by one block per zone.
__device__ __forceinline__ void finish_zone(const StepArgs& A, const double* __restrict__ vol, int iz, double fac,
                                            int do_rescale)
{
  const int nn = A.nu.n;
  const double dt = A.dt;
  const double v = vol[iz];
  __shared__ double red[256];
  if (A.store_Jnu && nn > 1) {
    double* J = A.J + (size_t)iz * nn;
    double esum = 0;
    for (int j = threadIdx.x; j < nn; j += blockDim.x) {
      double x = J[j];
      if (do_rescale) x *= fac;
      const double d = loc_delta(A.nu, j);
      x /= v * dt * 4 * PI * d;
      J[j] = x;
      esum += x * d * 4 * PI / C_LIGHT;
    }
    red[threadIdx.x] = esum;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
      if (threadIdx.x < (unsigned)s) red[threadIdx.x] += red[threadIdx.x + s];
      __syncthreads();
    }
  }
  if (threadIdx.x == 0) {
    A.e_abs[iz] /= v * dt;
    A.fr[iz] /= v * C_LIGHT * dt;
    if (A.L_dep) {  // transport_mpi.cpp:419-420
      A.L_dep[iz] /= v * dt;
      A.L_emit[iz] /= v;
    }
    if ((nn == 1) || (!A.store_Jnu)) {
      double j0 = A.J[(size_t)iz * (A.store_Jnu ? nn : 1)];
      if (do_rescale && A.store_Jnu) { j0 *= fac; A.J[(size_t)iz * nn] = j0; }
      A.e_rad[iz] = j0 / (v * dt * C_LIGHT);
    } else {
      A.e_rad[iz] = red[0];
    }
  }
}

// steady-state rescale factor L / (escaped energy fraction): transport.cpp:94-115
__device__ __forceinline__ double rescale_factor(unsigned long long escaped, int64_t n_active)
{
  const double per_esc = (1.0 * (double)escaped) / (1.0 * (double)n_active);
  return 1.0 / per_esc;
}

// The factor is formed on the device from the escape counter.
__global__ void finish_zones_kernel(const StepArgs A, const double* __restrict__ vol, int nz, int64_t n_active,
                                    int do_rescale)
{
  const int iz = blockIdx.x;
  if (iz >= nz) return;
  if (!A.smem_zones && A.n_rep > 0) {  // add the zone-scalar tally copies
    if (threadIdx.x < 5) {
      double sum = 0;
      for (int r = 0; r < A.n_rep; ++r) sum += A.zone_rep[((size_t)r * 5 + threadIdx.x) * nz + iz];
      double* dst[5] = {A.e_abs, A.fx, A.fy, A.fz, A.fr};
      dst[threadIdx.x][iz] += sum;
    }
    __syncthreads();
  }
  const double fac = do_rescale ? rescale_factor(A.counters[C_ESCAPED], n_active) : 1.0;
  finish_zone(A, vol, iz, fac, do_rescale);
}

__global__ void rescale_spectrum_kernel(const StepArgs A, int64_t nspec, int64_t n_active)
{
  const double fac = rescale_factor(A.counters[C_ESCAPED], n_active);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nspec; i += (int64_t)gridDim.x * blockDim.x)
    A.flux[i] *= fac;
}

// Batch: each zone and each spectrum is rescaled with its own model's factor
// (a model without packets keeps factor 1); the last block to finish is not
// needed for the step counter, block 0 advances it once everything of the
// step has been queued before this kernel.
__global__ void finish_zones_batch_kernel(const StepArgs A, const double* __restrict__ vol, int nz, int do_rescale)
{
  const int iz = blockIdx.x;
  if (iz >= nz) return;
  if (!A.smem_zones && A.n_rep > 0) {  // sum the zone-scalar tally copies
    if (threadIdx.x < 5) {
      double sum = 0;
      for (int r = 0; r < A.n_rep; ++r) sum += A.zone_rep[((size_t)r * 5 + threadIdx.x) * nz + iz];
      double* dst[5] = {A.e_abs, A.fx, A.fy, A.fz, A.fr};
      dst[threadIdx.x][iz] = sum;
    }
    __syncthreads();
  }
  double fac = 1.0;
  if (do_rescale) {
    const int m = __ldg(A.zone_nbr + iz).w;
    const int64_t n = A.models[m].n_packets;
    if (n > 0) fac = rescale_factor(A.model_escaped[m], n);
  }
  finish_zone(A, vol, iz, fac, do_rescale);
  if (iz == 0 && threadIdx.x == 0) *A.step_dev += 1u;
}

__global__ void rescale_spectrum_batch_kernel(const StepArgs A, int64_t nspec)
{
  const int64_t total = nspec * A.n_models;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int m = (int)(i / nspec);
    const int64_t n = A.models[m].n_packets;
    if (n > 0) A.flux[i] *= rescale_factor(A.model_escaped[m], n);
  }
}

// ------------------------------------------------------------ gamma-rays
// transport::lorentz_transform (relativity.cpp:84-127) in either direction:
// tolab = 1 flips the velocity (comoving -> lab), tolab = 0 does not
template <int GRID>
__device__ __forceinline__ void lorentz_transform(const GridDev& G, Pkt& p, int tolab)
{
  double v[3], dvds;
  get_velocity<GRID>(G, p.ind, p.x, p.D, v, &dvds);
  if (tolab) { v[0] *= -1; v[1] *= -1; v[2] *= -1; }
  const double beta2 = (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) / C_LIGHT / C_LIGHT;
  const double vdd = v[0] * p.D[0] + v[1] * p.D[1] + v[2] * p.D[2];
  const double gamma = 1.0 / sqrt(1 - beta2);
  const double dshift = gamma * (1 - vdd / C_LIGHT);
  p.dvds = dvds;
  p.e *= dshift;
  p.nu *= dshift;
  const double f = (1 - gamma * vdd / C_LIGHT / (gamma + 1));
  p.D[0] = 1.0 / dshift * (p.D[0] - gamma * v[0] / C_LIGHT * f);
  p.D[1] = 1.0 / dshift * (p.D[1] - gamma * v[1] / C_LIGHT * f);
  p.D[2] = 1.0 / dshift * (p.D[2] - gamma * v[2] / C_LIGHT * f);
  const double norm = p.D[0] * p.D[0] + p.D[1] * p.D[1] + p.D[2] * p.D[2];
  p.D[0] /= norm;
  p.D[1] /= norm;
  p.D[2] /= norm;
}

// transport::klein_nishina (transport_opacity.cpp:302-313), x in MeV
__device__ __forceinline__ double klein_nishina(double x)
{
  x = x / M_E_MEV;
  const double logfac = log(1 + 2 * x);
  const double term1 = (1 + x) / x / x / x * (2 * x * (1 + x) / (1 + 2 * x) - logfac);
  const double term2 = 1.0 / 2.0 / x * logfac;
  const double term3 = -1.0 * (1 + 3 * x) / (1 + 2 * x) / (1 + 2 * x);
  return .75 * (term1 + term2 + term3);
}

// grid::sample_in_zone: uniform in the shell volume (grid_1D_sphere.cpp:
// 681-700) or in the Cartesian cell (grid_3D_cart.cpp:484-494)
template <int GRID>
__device__ __forceinline__ void sample_in_zone(const GridDev& G, int i, double u0, double u1, double u2, double* r)
{
  if constexpr (GRID == 0) {
    const double r_0 = (i == 0) ? G.r_out.min : __ldg(G.r_out.right + i - 1);
    const double ro = __ldg(G.r_out.right + i);
    const double r_samp = pow(r_0 * r_0 * r_0 + u0 * (ro * ro * ro - r_0 * r_0 * r_0), 1.0 / 3.0);
    const double mu = 1 - 2.0 * u1;
    const double phi = 2.0 * PI * u2;
    const double sin_theta = sqrt(1 - mu * mu);
    r[0] = r_samp * sin_theta * cos(phi);
    r[1] = r_samp * sin_theta * sin(phi);
    r[2] = r_samp * mu;
  } else {
    const int nyz = G.ny * G.nz;
    const int idx[3] = {i / nyz, (i / G.nz) % G.ny, i % G.nz};
    const double u[3] = {u0, u1, u2};
#pragma unroll
    for (int a = 0; a < 3; ++a) r[a] = loc_left(G.ax[a], idx[a]) + u[a] * loc_delta(G.ax[a], idx[a]);
  }
}

// isotropic direction in the comoving frame (mu, phi: two deviates)
__device__ __forceinline__ void isotropic_direction(PacketRng& rng, double* D)
{
  const double mu = 1 - 2.0 * rng.next();
  const double phi = 2.0 * PI * rng.next();
  const double smu = sqrt(1 - mu * mu);
  D[0] = smu * cos(phi);
  D[1] = smu * sin(phi);
  D[2] = mu;
}

// transport::sample_photon_frequency for an optical photon (emission.cpp:27-46)
template <typename CT>
__device__ __forceinline__ void sample_optical_nu(const StepArgs& A, Pkt& p, PacketRng& rng)
{
  const int inu = (A.nu.n == 1) ? 0 : cdf_row_sample<CT>(A, p.ind, rng.next());
  p.nu = loc_sample(A.nu, inu, rng.next());
}

// ------------------------------------------------------------ discrete diffusion
// transport_use_ddmc = 2 (src/transport/discrete_diffusion.cpp:114-510), on
// 1D spheres with the reference's FP64 expressions.

// transport::get_opacity of zone iz at comoving frequency nu_cmf
template <typename OT>
__device__ __forceinline__ int ddmc_opacity(const StepArgs& A, const OT* __restrict__ opac, int iz, double nu_cmf,
                                            double* op, double* eps)
{
  const int nn = A.nu.n;
  const int i_nu = loc_within_fast<false>(A.nu, nu_cmf);
  const OT ab = opac[(size_t)iz * nn + i_nu];
  const double a_opac = (double)ab.x;
  const double s_opac = A.omit_scat ? 0.0 : (double)ab.y;
  *op = a_opac + s_opac;
  *eps = (*op == 0) ? 0 : a_opac / *op;
  return i_nu;
}

__device__ __forceinline__ double pkt_r(const Pkt& p)
{
  return sqrt(p.x[0] * p.x[0] + p.x[1] * p.x[1] + p.x[2] * p.x[2]);
}

// the zone test of transport::propagate (transport.cpp:219-231)
template <typename OT>
__device__ bool ddmc_zone(const StepArgs& A, const GridDev& G, const OT* __restrict__ opac, Pkt& p)
{
  const double dshift = dshift_lab_to_comoving<0>(G, p);
  double sigma, eps;
  ddmc_opacity<OT>(A, opac, p.ind, p.nu * dshift, &sigma, &eps);
  return sigma * loc_delta(G.r_out, p.ind) > A.ddmc_tau;
}

// transport::sample_dir_from_blackbody_surface (discrete_diffusion.cpp:753-794)
__device__ void bb_surface_dir(PacketRng& rng, Pkt& p)
{
  const double mu = sqrt(rng.next());
  const double phi = 2.0 * PI * rng.next();
  const double smu = sqrt(1.0 - mu * mu);
  const double v1 = smu * cos(phi), v2 = smu * sin(phi), v3 = mu;
  const double r1 = p.x[0] / pkt_r(p), r2 = p.x[1] / pkt_r(p), r3 = p.x[2] / pkt_r(p);
  const double costheta = r3, sintheta = sqrt(1 - costheta * costheta);
  const double v1p = v1 * costheta + r1 * v3 * sintheta - r2 * (1.0 - costheta) * (-r2 * v1 + r1 * v2);
  const double v2p = v2 * costheta + r2 * v3 * sintheta - r1 * (1.0 - costheta) * (-r2 * v1 + r1 * v2);
  const double v3p = v3 * costheta - (r1 * v1 + r2 * v2) * sintheta;
  const double norm = sqrt(v1p * v1p + v2p * v2p + v3p * v3p);
  p.D[0] = v1p / norm;
  p.D[1] = v2p / norm;
  p.D[2] = v3p / norm;
}

// transport::move_across_DDMC_interface (discrete_diffusion.cpp:413-510):
// the photon converts to the diffusive zone new_ind (and stays in the
// comoving frame, as the reference leaves it) or is put back next to the
// interface with a direction away from it
__device__ void ddmc_move_across(const StepArgs& A, const GridDev& G, Pkt& p, PacketRng& rng, int new_ind,
                                 double sigma_i, double dr)
{
  const int nz = G.nzones;
  int ip = p.ind + 1, im = p.ind - 1;
  if (ip == nz) ip = p.ind;
  if (im < 0) im = 0;
  const double r_p = __ldg(G.r_out.right + p.ind);
  double r_m = __ldg(G.r_out.right + im);
  if (p.ind == 0) r_m = G.r_out.min;
  double r_interface = 0;
  if (new_ind == ip) r_interface = r_p;
  else if (new_ind == im) r_interface = r_m;
  lorentz_transform<0>(G, p, 0);
  const double rr = pkt_r(p);
  double mu = (p.x[0] * p.D[0] + p.x[1] * p.D[1] + p.x[2] * p.D[2]) / rr;
  mu = fabs(mu);
  const double p_convert = 4.0 * (1.0 + 1.5 * mu) / (3.0 * sigma_i * dr + 6.0 * 0.7104);
  const double xi = rng.next();
  const double u0 = rng.next(), u1 = rng.next(), u2 = rng.next();
  const double push = 1.0e-8;
  if (xi <= p_convert) {
    p.ind = new_ind;
    sample_in_zone<0>(G, p.ind, u0, u1, u2, p.x);
    return;
  }
  sample_in_zone<0>(G, p.ind, u0, u1, u2, p.x);
  if (new_ind == ip) {
    double d = r_interface - pkt_r(p);
    d *= (1.0 - push);
    p.x[0] += p.x[0] / pkt_r(p) * d;  // the radius is taken again after each coordinate moves
    p.x[1] += p.x[1] / pkt_r(p) * d;
    p.x[2] += p.x[2] / pkt_r(p) * d;
  } else if (new_ind == im) {
    double d = pkt_r(p) - r_interface;
    d *= (1.0 - push);
    p.x[0] -= p.x[0] / pkt_r(p) * d;
    p.x[1] -= p.x[1] / pkt_r(p) * d;
    p.x[2] -= p.x[2] / pkt_r(p) * d;
  }
  bb_surface_dir(rng, p);
  const double mu2 = (p.x[0] * p.D[0] + p.x[1] * p.D[1] + p.x[2] * p.D[2]) / pkt_r(p);
  if ((new_ind == ip && mu2 > 0.0) || (new_ind == im && mu2 < 0.0)) {
    p.D[0] = -p.D[0]; p.D[1] = -p.D[1]; p.D[2] = -p.D[2];
  }
  lorentz_transform<0>(G, p, 1);
}

// ------------------------------------------------------------ IMD
// transport::discrete_diffuse_IMD (discrete_diffusion.cpp:18-110), IMD
// (Gentile 2001) as the reference has it: propagate calls it with the end
// time of the step where the function means the step (transport.cpp:237), so
// the photon's time advances by tstop and the J tally and the advection take
// tstop as the interval.  The photon hops one zone up or down (a radial move
// by its starting zone's width) until it stays, is then advected, loses
// energy adiabatically and stops.  J goes to bin 0 of the zone, as in the
// reference; the hop loop, unbounded there, gives up after 2^24 hops
// (counted, SED_ERR_LIMIT).
template <typename OT>
__device__ int imd_event(const StepArgs& A, const GridDev& G, Pkt& p, PacketRng& rng, double* t_eabs,
                         unsigned long long& n_cap)
{
  const int nz = G.nzones, nn = A.nu.n;
  const int nj = A.store_Jnu ? nn : 1;
  const double* P_up = A.imd_p;
  const double* P_dn = A.imd_p + nz;
  const double* P_st = A.imd_p + 2 * nz;
  const double* P_ab = A.imd_p + 3 * nz;
  const double dt = A.tstop;
  const double dx = loc_delta(G.r_out, p.ind);
  p.t += dt;
  for (int hops = 0;; ++hops) {
    if (hops >= (1 << 24)) { ++n_cap; break; }
    p.ind = get_zone<0>(G, p.x);
    if (p.ind == -1) return ABSORBED;
    if (p.ind == -2) return ESCAPED;
    const int i = p.ind;
    atomicAdd(t_eabs + i, p.e * __ldg(P_ab + i));
    atomicAdd(A.J + (size_t)i * nj, p.e * __ldg(P_st + i) * dt * C_LIGHT);
    const double P_diff = __ldg(P_up + i) + __ldg(P_dn + i);
    const double P_stay = __ldg(P_ab + i) + __ldg(P_st + i);
    const double r1 = rng.next();
    if (r1 < P_diff) {
      const double r2 = rng.next();
      if (r2 < __ldg(P_up + i) / P_diff) {
        p.ind++;
        const double rr = sqrt(p.x[0] * p.x[0] + p.x[1] * p.x[1] + p.x[2] * p.x[2]);
        p.x[0] += p.x[0] / rr * dx;
        p.x[1] += p.x[1] / rr * dx;
        p.x[2] += p.x[2] / rr * dx;
      } else {
        p.ind--;
        const double rr = sqrt(p.x[0] * p.x[0] + p.x[1] * p.x[1] + p.x[2] * p.x[2]);
        p.x[0] -= p.x[0] / rr * dx;
        p.x[1] -= p.x[1] / rr * dx;
        p.x[2] -= p.x[2] / rr * dx;
      }
    } else {
      const double r2 = rng.next();
      const double f_abs = __ldg(P_ab + i) / P_stay;
      if (r2 < f_abs) return ABSORBED;
      double v[3], dvds;
      get_velocity<0>(G, p.ind, p.x, p.D, v, &dvds);
      p.x[0] += v[0] * dt;
      p.x[1] += v[1] * dt;
      p.x[2] += v[2] * dt;
      p.e *= (1 - dvds * dt);
      break;
    }
  }
  p.ind = get_zone<0>(G, p.x);
  if (p.ind == -1) return ABSORBED;
  if (p.ind == -2) return ESCAPED;
  return STOPPED;
}

// transport::compute_diffusion_probabilities (discrete_diffusion.cpp:687-756)
// for zone i: hop probabilities from the Planck-mean diffusion coefficients
// of the zone and its neighbours, normalised with the (zero) advection and
// absorption probabilities; the rest is "stay"
__global__ void imd_probabilities_kernel(const GridDev G, const double* __restrict__ planck, double dt,
                                         double* __restrict__ out)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int nz = G.nzones;
  if (i >= nz) return;
  const double dx = loc_delta(G.r_out, i);
  int ip = i + 1;
  if (ip == nz) ip = i;
  int im = i - 1;
  if (im < 0) im = 0;
  const double Dj0 = C_LIGHT / (3.0 * planck[i]);
  const double Djp = C_LIGHT / (3.0 * planck[ip]);
  const double Djm = C_LIGHT / (3.0 * planck[im]);
  const double Dh_up = 2 * dx * (Dj0 * Djp) / (Dj0 * dx + Djp * dx);
  const double Dh_dn = 2 * dx * (Dj0 * Djm) / (Dj0 * dx + Djm * dx);
  const double r_p = __ldg(G.r_out.right + i);  // grid_1D_sphere::coordinates: r_out[i]
  double r_m = __ldg(G.r_out.right + im);
  if (i == 0) r_m = 0;
  const double r_0 = 0.5 * (r_p + r_m);
  double up = (dt / dx) * (Dh_up / dx) * r_p * r_p / r_0 / r_0;
  double dn = (dt / dx) * (Dh_dn / dx) * r_m * r_m / r_0 / r_0;
  if (i == 0) dn = 0;
  double adv = 0.0, ab = 0.0;
  double norm = 1 + adv + ab;
  norm += up + dn;
  ab /= norm;
  up /= norm;
  dn /= norm;
  out[i] = up;
  out[nz + i] = dn;
  out[2 * nz + i] = 1.0 / norm;
  out[3 * nz + i] = ab;
}

// One pass of the event loop of transport::discrete_diffuse_DDMC
// (discrete_diffusion.cpp:136-404): leakage to a neighbour, effective
// (inelastic) scattering, or the end of the step, then advection and the
// adiabatic loss.  dt_remaining carries over the passes of one call; the
// zone's J (bin 0, as the reference tallies it) and e_abs are tallied.  The
// effective-scattering loop, unbounded in the reference, gives up after
// 65536 re-emissions that stay in the same bin (counted).
template <typename OT, typename CT>
__device__ int ddmc_event(const StepArgs& A, const GridDev& G, const OT* __restrict__ opac, Pkt& p, PacketRng& rng,
                          double& dt_remaining, double& acc_eabs, unsigned long long& n_scat,
                          unsigned long long& n_cap)
{
  const int nz = G.nzones, nn = A.nu.n;
  const int nj = A.store_Jnu ? nn : 1;
  const double lambda_ddmc = 0.7104, push = 1.0e-8;
  int fate = MOVING;
  const int ii = p.ind;
  int ip = ii + 1, im = ii - 1;
  if (ip == nz) ip = ii;
  if (im < 0) im = 0;
  const double dx = loc_delta(G.r_out, ii), dxp1 = loc_delta(G.r_out, ip), dxm1 = loc_delta(G.r_out, im);
  double dshift = dshift_lab_to_comoving<0>(G, p);
  double sigma_i, eps_i, sigma_ip1, eps_ip1, sigma_im1, eps_im1;
  int i_nu = ddmc_opacity<OT>(A, opac, ii, p.nu * dshift, &sigma_i, &eps_i);
  ddmc_opacity<OT>(A, opac, ip, p.nu * dshift, &sigma_ip1, &eps_ip1);
  ddmc_opacity<OT>(A, opac, im, p.nu * dshift, &sigma_im1, &eps_im1);
  const double r_p = __ldg(G.r_out.right + ii);
  double r_m = __ldg(G.r_out.right + im);
  if (ii == 0) r_m = G.r_out.min;
  const double r_0 = 0.5 * (r_p + r_m);
  const double Xi = 1.0 + dx * dx / (12.0 * r_0 * r_0);
  double geo_factor = r_m * r_m / r_0 / r_0 / Xi;
  const double tau_im1 = sigma_im1 * dxm1;
  const bool ddmc_on_im1 = !(tau_im1 <= A.ddmc_tau);
  double sigma_leak_left;
  if (ddmc_on_im1) sigma_leak_left = (2.0 / 3.0 / dx) * (1.0 / (sigma_i * dx + sigma_im1 * dxm1)) * geo_factor;
  else sigma_leak_left = (2.0 / 3.0 / dx) * (1.0 / (sigma_i * dx + 2.0 * lambda_ddmc)) * geo_factor;
  geo_factor = r_p * r_p / r_0 / r_0 / Xi;
  const double tau_ip1 = sigma_ip1 * dxp1;
  const bool ddmc_on_ip1 = !(tau_ip1 <= A.ddmc_tau);
  double sigma_leak_right;
  if (ddmc_on_ip1) sigma_leak_right = (2.0 / 3.0 / dx) * (1.0 / (sigma_i * dx + sigma_ip1 * dxp1)) * geo_factor;
  else sigma_leak_right = (2.0 / 3.0 / dx) * (1.0 / (sigma_i * dx + 2.0 * lambda_ddmc)) * geo_factor;
  if (ip == ii) sigma_leak_right = (2.0 / 3.0 / dx) * (1.0 / (sigma_i * dx + 2.0 * lambda_ddmc)) * geo_factor;
  if (ii == 0) sigma_leak_left = 0.0;
  const double sigma_leak_tot = sigma_leak_left + sigma_leak_right;
  const double xi = rng.next();
  bool leaked2imc = false;
  const double d_stay = C_LIGHT * dt_remaining;
  const double d_leak = -log(xi) / (sigma_leak_left + sigma_leak_right);
  double d_sc;
  if (nn == 1) d_sc = INFINITY;
  else {
    const double tau_r = -1.0 * log(rng.next());
    if (eps_i > 0.0) {
      double k_es_inelastic = sigma_i * eps_i;
      dshift = dshift_lab_to_comoving<0>(G, p);
      i_nu = ddmc_opacity<OT>(A, opac, p.ind, p.nu * dshift, &sigma_i, &eps_i);
      // emissivity_[zone].get_value(i_nu): the bin's share of the CDF
      const CT* row = reinterpret_cast<const CT*>(A.cdf) + (size_t)p.ind * nn;
      const double elastic_frac = (i_nu == 0) ? (double)row[0] : (double)(row[i_nu] - row[i_nu - 1]);
      k_es_inelastic *= 1.0 - elastic_frac;
      d_sc = tau_r / k_es_inelastic;
    } else {
      d_sc = INFINITY;
    }
  }
  int event;
  double this_d;
  if ((d_sc < d_leak) && (d_sc < d_stay)) { event = 0; this_d = d_sc; }
  else if (d_leak < d_stay) { event = 1; this_d = d_leak; }
  else { event = 2; this_d = d_stay; }
  const double this_dt = this_d / C_LIGHT;
  p.t += this_dt;
  dt_remaining -= this_dt;
  atomicAdd(A.J + (size_t)p.ind * nj, p.e * this_d);
  acc_eabs += (p.e * dshift) * this_d * sigma_i * eps_i;
  if (event == 0) {
    ++n_scat;
    int now_i_nu = i_nu;
    for (int tries = 0; now_i_nu == i_nu; ++tries) {
      if (tries >= (1 << 16)) { ++n_cap; break; }
      // do_scatter(p, 1.0) (scatter.cpp:12-41): never coherent
      fate = MOVING;
      if (rng.next() > 1.0) {
        isotropic_scatter<0, CT>(A, G, p, rng, 0);
      } else {
        const double z2 = rng.next();
        if ((z2 > __ldg(A.eps_imc + p.ind)) || A.radiative_eq) isotropic_scatter<0, CT>(A, G, p, rng, 1);
        else fate = ABSORBED;
      }
      dshift = dshift_lab_to_comoving<0>(G, p);
      double s2, e2;
      now_i_nu = ddmc_opacity<OT>(A, opac, p.ind, p.nu * dshift, &s2, &e2);
    }
  } else if (event == 2) {
    dt_remaining = -1.0;
    fate = STOPPED;
  } else {
    const double P_leak_left = sigma_leak_left / sigma_leak_tot;
    const double xi2 = rng.next();
    if (xi2 <= P_leak_left) {
      p.ind--;
      const double rr = pkt_r(p);
      double dr = rr - r_m;
      if (ddmc_on_im1) dr += rng.next() * dxm1;
      else dr *= (1.0 + push);
      p.x[0] -= p.x[0] / rr * dr;
      p.x[1] -= p.x[1] / rr * dr;
      p.x[2] -= p.x[2] / rr * dr;
      if (!ddmc_on_im1) {
        leaked2imc = true;
        lorentz_transform<0>(G, p, 0);
        bb_surface_dir(rng, p);
        const double mu = (p.x[0] * p.D[0] + p.x[1] * p.D[1] + p.x[2] * p.D[2]) / pkt_r(p);
        if (mu > 0.0) { p.D[0] = -p.D[0]; p.D[1] = -p.D[1]; p.D[2] = -p.D[2]; }
        lorentz_transform<0>(G, p, 1);
      }
    } else {
      p.ind++;
      const double rr = pkt_r(p);
      double dr = r_p - rr;
      if (ddmc_on_ip1) dr += rng.next() * dxp1;
      else dr *= (1.0 + push);
      p.x[0] += p.x[0] / rr * dr;
      p.x[1] += p.x[1] / rr * dr;
      p.x[2] += p.x[2] / rr * dr;
      if (!ddmc_on_ip1) {
        leaked2imc = true;
        lorentz_transform<0>(G, p, 0);
        bb_surface_dir(rng, p);
        const double mu = (p.x[0] * p.D[0] + p.x[1] * p.D[1] + p.x[2] * p.D[2]) / pkt_r(p);
        if (mu < 0.0) { p.D[0] = -p.D[0]; p.D[1] = -p.D[1]; p.D[2] = -p.D[2]; }
        lorentz_transform<0>(G, p, 1);
      }
    }
  }
  // advection and the adiabatic loss (discrete_diffusion.cpp:371-397)
  double zone_vel[3], dvds;
  get_velocity<0>(G, p.ind, p.x, p.D, zone_vel, &dvds);
  const double vel = sqrt(zone_vel[0] * zone_vel[0] + zone_vel[1] * zone_vel[1] + zone_vel[2] * zone_vel[2]);
  const double v_over_r = vel / pkt_r(p);
  const double dlnrhodt = dvds + 2.0 * v_over_r;
  const double doppler_shift_ddmc = (1.0 - dlnrhodt * this_dt / 3.0);
  lorentz_transform<0>(G, p, 0);
  p.e *= doppler_shift_ddmc;
  p.nu *= doppler_shift_ddmc;
  lorentz_transform<0>(G, p, 1);
  if (!leaked2imc) {
    p.x[0] += zone_vel[0] * this_dt;
    p.x[1] += zone_vel[1] * this_dt;
    p.x[2] += zone_vel[2] * this_dt;
  }
  p.ind = get_zone<0>(G, p.x);
  if (p.ind == -1) fate = ABSORBED;
  if (p.ind == -2) fate = ESCAPED;
  return fate;
}

// Radioactive packets: emission (transport::emit_radioactive, emission.cpp:
// 212-236, and create_isotropic_particle, :57-107) and, for the gamma-rays,
// the segment loop of propagate_monte_carlo with the gamma-ray opacity
// (transport_opacity.cpp:290-296) and do_scatter / compton_scatter
// (scatter.cpp:45-133).  Deviates come from the packet's own stream in the
// reference's order.  A packet that is or becomes an optical photon is
// queued, with its stream position, for the packet kernel.
template <int GRID, typename CT>
__global__ void __launch_bounds__(128, 8) gamma_kernel(const StepArgs A, const StepArgs AG, const RadioArgs R,
                                                       const GridDev G)
{
  unsigned long long n_esc = 0, n_abs = 0, n_stop = 0, n_seg = 0, n_scat = 0, n_lim = 0;
  const int64_t limit = A.max_segments > 0 ? A.max_segments : 10000000;
  constexpr int COMPTON_TRIES = 1 << 16;
  const double L_tot = *R.L_tot;
  const double Ep = L_tot * R.dt / (1.0 * R.n_radio);
  const int64_t n_q = R.n_census + R.n_radio;
  for (;;) {
    const int64_t k = (int64_t)atomicAdd(A.counters + C_COUNT, 1ULL);
    if (k >= n_q) break;
    PacketRng rng;
    Pkt p;
    bool photon;
    if (k < R.n_census) {
      // a gamma-ray of the census continues on its stream of this step;
      // census photons are the packet kernel's
      if (R.q_type[k] != TYPE_GAMMA) continue;
      R.q_n[k] = RADIO_NO_PHOTON;
      rng.init(A.seed, (uint64_t)(R.first_pid + k), A.step, 0);
      const double* q = R.q_state + (size_t)k * 9;
      p.x[0] = q[0]; p.x[1] = q[1]; p.x[2] = q[2];
      p.D[0] = q[3]; p.D[1] = q[4]; p.D[2] = q[5];
      p.t = q[6]; p.e = q[7]; p.nu = q[8];
      p.dvds = 0;
      photon = false;
    } else {
      R.q_n[k] = RADIO_NO_PHOTON;
      if (L_tot == 0) {  // the reference emits nothing then
        if (A.rec_fate) {
          const int64_t r = A.n_core + k;
          A.rec_fate[r] = -1; A.rec_ind[r] = 0; A.rec_draws[r] = 0;
          for (int j = 0; j < 9; ++j) A.rec_state[r * 9 + j] = 0;
        }
        continue;
      }
      rng.init(A.seed, (uint64_t)(R.first_pid + k), A.step, 0);
      // zone_emission_cdf_.sample: upper_bound over the zones
      const int i = (R.nz == 1) ? 0 : upper_bound_dev(R.cdf, R.nz, rng.next());
      const double t = R.t_now + R.dt * rng.next();
      const bool is_gamma = rng.next() < __ldg(R.gamma_frac + i);
      if (!is_gamma) atomicAdd(R.L_dep + i, Ep);  // positrons deposit and become photons
      const double u0 = rng.next(), u1 = rng.next(), u2 = rng.next();
      sample_in_zone<GRID>(G, i, u0, u1, u2, p.x);
      isotropic_direction(rng, p.D);
      p.ind = i;
      if (is_gamma) p.nu = 1;  // sample_photon_frequency for gamma-rays (emission.cpp:35-38)
      else sample_optical_nu<CT>(A, p, rng);
      p.e = Ep;
      lorentz_transform<GRID>(G, p, 1);
      p.t = t;
      photon = !is_gamma;
    }
    // transport::propagate: the zone of the packet's position
    p.ind = get_zone<GRID>(G, p.x);
    int fate = MOVING;
    if (!photon) {
      if (p.ind == -1) fate = ABSORBED;
      else if (p.ind == -2) fate = ESCAPED;
    }
    int64_t seg = 0;
    while (!photon && fate == MOVING) {
      if (seg >= limit) { fate = STOPPED; ++n_lim; break; }
      ++seg;
      const int iz = p.ind;
      double d_bn = 0;
      const double rsq = (p.x[0] * p.x[0] + p.x[1] * p.x[1] + p.x[2] * p.x[2]);
      const double xdotD = (p.D[0] * p.x[0] + p.D[1] * p.x[1] + p.D[2] * p.x[2]);
      int new_ind = get_next_zone<GRID>(G, p.x, p.D, iz, A.core_radius, rsq, xdotD, &d_bn);
      const double dshift = dshift_lab_to_comoving<GRID>(G, p);
      const double c_opac = __ldg(R.compton + iz) * klein_nishina(p.nu);
      const double p_opac = __ldg(R.photoion + iz) * pow(p.nu, -3.5);
      const double op = c_opac + p_opac;
      const double eps = p_opac / (c_opac + p_opac);
      double d_nu = loc_delta(A.nu, 0) / p.nu * C_LIGHT / p.dvds;  // i_nu = 0 for gamma-rays
      if (p.dvds == 0) d_nu = INFINITY;
      if (d_nu < 0) d_nu = -1 * d_nu;
      if (d_nu < d_bn) { d_bn = d_nu; new_ind = p.ind; }
      const double tot_lab = op * dshift;
      const double tau_r = -1.0 * log(1 - rng.next());
      double d_sc = tau_r / tot_lab;
      if (tot_lab == 0) d_sc = INFINITY;
      double d_tm = (A.tstop - p.t) * C_LIGHT;
      if (A.steady) d_tm = INFINITY;
      int event;
      double this_d;
      if ((d_sc < d_bn) && (d_sc < d_tm)) { event = 0; this_d = d_sc; }
      else if (d_bn < d_tm) { event = 1; this_d = d_bn; }
      else { event = 2; this_d = d_tm; }
      // radiation force tallies (gamma-rays add nothing to e_abs and J)
      const double this_E = p.e * this_d;
      if (A.tally_forces) {
        atomicAdd(A.fx + iz, this_E * dshift * op * p.D[0] * dshift);
        atomicAdd(A.fy + iz, this_E * dshift * op * p.D[1] * dshift);
        atomicAdd(A.fz + iz, this_E * dshift * op * p.D[2] * dshift);
        const double rr = sqrt(p.x[0] * p.x[0] + p.x[1] * p.x[1] + p.x[2] * p.x[2]);
        const double xd = p.x[0] * p.D[0] + p.x[1] * p.D[1] + p.x[2] * p.D[2];
        atomicAdd(A.fr + iz, this_E * dshift * op * xd / rr * dshift);
      }
      p.x[0] += this_d * p.D[0];
      p.x[1] += this_d * p.D[1];
      p.x[2] += this_d * p.D[2];
      p.t = p.t + this_d / C_LIGHT;
      if (event == 1) {
        if (new_ind == -1) {
          if (A.bound_in_reflect) { p.D[0] *= -1; p.D[1] *= -1; p.D[2] *= -1; }
          else { p.ind = new_ind; fate = ABSORBED; }
        } else if (new_ind == -2) {
          if (A.bound_out_reflect) { p.D[0] *= -1; p.D[1] *= -1; p.D[2] *= -1; }
          else { p.ind = new_ind; fate = ESCAPED; }
        } else {
          p.ind = new_ind;
        }
      } else if (event == 0) {
        ++n_scat;
        if (rng.next() > eps) {
          // transport::compton_scatter (scatter.cpp:76-133)
          lorentz_transform<GRID>(G, p, 0);
          double E_ratio = 1, Dn[3];
          for (int tries = 0;; ++tries) {
            isotropic_direction(rng, Dn);
            const double cost = p.D[0] * Dn[0] + p.D[1] * Dn[1] + p.D[2] * Dn[2];
            E_ratio = 1 / (1 + p.nu / M_E_MEV * (1 - cost));
            const double diff_cs = 0.5 * (E_ratio * E_ratio * (1 / E_ratio + E_ratio - 1 + cost * cost));
            if (rng.next() < diff_cs) break;
            if (tries + 1 >= COMPTON_TRIES) { atomicAdd(R.n_reject_cap, 1); break; }
          }
          p.nu = p.nu * E_ratio;
          if (rng.next() > E_ratio) {
            atomicAdd(R.L_dep + p.ind, p.e);
            photon = true;
            isotropic_direction(rng, Dn);
            sample_optical_nu<CT>(A, p, rng);
          }
          p.D[0] = Dn[0];
          p.D[1] = Dn[1];
          p.D[2] = Dn[2];
          lorentz_transform<GRID>(G, p, 1);
        } else {
          // photo-absorbed: deposited, re-emitted as an optical photon
          atomicAdd(R.L_dep + p.ind, p.e);
          photon = true;
          isotropic_direction(rng, p.D);
          sample_optical_nu<CT>(A, p, rng);
          lorentz_transform<GRID>(G, p, 1);
        }
      } else {
        fate = STOPPED;
      }
    }
    n_seg += seg;
    if (photon) {
      double* q = R.q_state + (size_t)k * 9;
      q[0] = p.x[0]; q[1] = p.x[1]; q[2] = p.x[2];
      q[3] = p.D[0]; q[4] = p.D[1]; q[5] = p.D[2];
      q[6] = p.t; q[7] = p.e; q[8] = p.nu;
      R.q_ind[k] = p.ind;
      R.q_n[k] = rng.n;
      continue;
    }
    if (fate == ESCAPED) {
      const double t_obs = p.t - (p.x[0] * p.D[0] + p.x[1] * p.D[1] + p.x[2] * p.D[2]) / C_LIGHT;
      spectrum_count(AG, AG.flux, AG.click, t_obs, p.nu, p.e, p.D);
      p.t = t_obs;
      ++n_esc;
    } else if (fate == ABSORBED) {
      ++n_abs;
    } else {
      ++n_stop;
    }
    if (A.rec_fate) {  // slots after the core packets'
      const int64_t r = A.n_core + k;
      A.rec_fate[r] = fate;
      A.rec_ind[r] = p.ind;
      A.rec_draws[r] = (int32_t)rng.n;
      if (A.rec_type) A.rec_type[r] = TYPE_GAMMA;
      double* s = A.rec_state + r * 9;
      s[0] = p.x[0]; s[1] = p.x[1]; s[2] = p.x[2];
      s[3] = p.D[0]; s[4] = p.D[1]; s[5] = p.D[2];
      s[6] = p.t; s[7] = p.e; s[8] = p.nu;
    }
  }
  n_esc = warp_sum(n_esc); n_abs = warp_sum(n_abs); n_stop = warp_sum(n_stop);
  n_seg = warp_sum(n_seg); n_scat = warp_sum(n_scat); n_lim = warp_sum(n_lim);
  if ((threadIdx.x & 31) == 0) {
    if (n_esc) atomicAdd(A.counters + C_ESCAPED, n_esc);
    if (n_abs) atomicAdd(A.counters + C_ABSORBED, n_abs);
    if (n_stop) atomicAdd(A.counters + C_STOPPED, n_stop);
    if (n_seg) atomicAdd(A.counters + C_SEGMENTS, n_seg);
    if (n_scat) atomicAdd(A.counters + C_SCATTERS, n_scat);
    if (n_lim) atomicAdd(A.counters + C_LIMIT, n_lim);
  }
}

// ------------------------------------------------------------ census
// The census opens the step's queue.  transport::propagate starts with
// get_zone (transport.cpp:205-209), so each packet is located again on the
// grid of this step.
template <int GRID>
__global__ void census_load_kernel(const CensusArgs C, const GridDev G)
{
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < C.n_census; k += stride) {
    const double* s = C.census_state + k * 9;
    double* q = C.q_state + k * 9;
#pragma unroll
    for (int j = 0; j < 9; ++j) q[j] = s[j];
    C.q_type[k] = C.census_type[k];
    C.q_ind[k] = get_zone<GRID>(G, s);
    C.q_n[k] = 0;
  }
}

// Record slot of the packet at position r of the reference's vector
// (census, then radioactive, then core packets).
__device__ __forceinline__ int64_t census_slot(const CensusArgs& C, int64_t r)
{
  return r < C.n_q ? C.n_core + r : r - C.n_q;
}

__global__ void census_flags_kernel(const CensusArgs C, int64_t n)
{
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r <= n; r += stride) {
    if (r == n) { C.flag_e[r] = 0; C.flag_a[r] = 0; continue; }
    const int32_t f = C.rec_fate[census_slot(C, r)];
    C.flag_e[r] = (f != -1);  // -1: a radioactive packet that was never emitted
    C.flag_a[r] = (f == STOPPED);
  }
}

// clean_up_particle_vector keeps the n_alive stopped packets: a stopped
// packet at vector position s < n_alive stays there, and the j-th removed
// position below n_alive (counted from the front) takes the j-th stopped
// packet counted from the back.
__global__ void census_front_kernel(const CensusArgs C, int64_t n)
{
  const int64_t n_alive = C.scan_a[n];
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += stride) {
    if (!C.flag_e[r] || C.flag_a[r]) continue;
    const int64_t s = C.scan_e[r];
    if (s < n_alive) C.front_dead[s - C.scan_a[r]] = (int32_t)s;
  }
}

__global__ void census_scatter_kernel(const CensusArgs C, int64_t n)
{
  const int64_t n_alive = C.scan_a[n];
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  unsigned long long ng = 0;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += stride) {
    if (!C.flag_a[r]) continue;
    const int64_t s = C.scan_e[r];
    const int64_t dest = s < n_alive ? s : C.front_dead[n_alive - 1 - C.scan_a[r]];
    const int64_t slot = census_slot(C, r);
    const double* src = C.rec_state + slot * 9;
    double* d = C.census_state + dest * 9;
#pragma unroll
    for (int j = 0; j < 9; ++j) d[j] = src[j];
    C.census_ind[dest] = C.rec_ind[slot];
    C.census_type[dest] = C.rec_type[slot];
    if (C.rec_type[slot] == TYPE_GAMMA) ++ng;
  }
  if (ng) atomicAdd(C.n_gamma, ng);
}

// ------------------------------------------------------------ initialisation
// transport::blackbody_nu (transport_opacity.cpp:322-326)
__device__ __forceinline__ double blackbody_nu(double T, double nu)
{
  const double zeta = H_PLANCK * nu / K_BOLTZ / T;
  return 2.0 * nu * nu * nu * H_PLANCK / C_LIGHT / C_LIGHT / (exp(zeta) - 1);
}

// cdf_array::normalize (src/transport/cdf_array.h:62-74), in order
__device__ void cdf_normalize_seq(double* y, int n)
{
  for (int i = 0; i < n; ++i) if (isnan(y[i])) y[i] = 0;
  if (y[n - 1] == 0) for (int i = 0; i < n; ++i) y[i] = 1.0;
  const double N = y[n - 1];
  for (int i = 0; i < n; ++i) y[i] /= N;
}

// the zone CDF of e_rad * vol and its sum, in the reference's order
// (emission.cpp:128-150); one thread
__global__ void init_zone_cdf_kernel(const InitArgs I)
{
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double E_sum = 0;
  for (int i = 0; i < I.nz; ++i) {
    const double E_zone = I.e_rad[i] * I.vol[i];
    I.zone_cdf[i] = (i == 0) ? E_zone : I.zone_cdf[i - 1] + E_zone;
    E_sum += E_zone;
  }
  cdf_normalize_seq(I.zone_cdf, I.nz);
  *I.E_sum = E_sum;
}

// the blackbody emissivity CDF of each zone at its gas temperature
// (emission.cpp:137-146); one thread per zone, bins in order
__global__ void init_bb_cdf_kernel(const InitArgs I)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= I.nz) return;
  const int ng = I.nu.n;
  double* row = I.bb_cdf + (size_t)i * ng;
  const double T = I.T[i];
  for (int j = 0; j < ng; ++j) {
    const double emis = blackbody_nu(T, loc_center(I.nu, j)) * loc_delta(I.nu, j);
    row[j] = (j == 0) ? emis : row[j - 1] + emis;
  }
  cdf_normalize_seq(row, ng);
}

// the packets: zone, then create_isotropic_particle (emission.cpp:57-107)
// with the blackbody emissivity, at time t_now
template <int GRID>
__global__ void init_particles_kernel(const InitArgs I, const GridDev G)
{
  const double Ep = *I.E_sum / (1.0 * I.n);
  const int ng = I.nu.n;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < I.n; k += stride) {
    PacketRng rng;
    rng.init(I.seed, (uint64_t)(I.first_pid + k), INIT_STEP, 0);
    Pkt p;
    const int i = (I.nz == 1) ? 0 : upper_bound_dev(I.zone_cdf, I.nz, rng.next());
    p.ind = i;
    const double u0 = rng.next(), u1 = rng.next(), u2 = rng.next();
    sample_in_zone<GRID>(G, i, u0, u1, u2, p.x);
    isotropic_direction(rng, p.D);
    const int inu = (ng == 1) ? 0 : upper_bound_dev(I.bb_cdf + (size_t)i * ng, ng, rng.next());
    p.nu = loc_sample(I.nu, inu, rng.next());
    p.e = Ep;
    lorentz_transform<GRID>(G, p, 1);
    p.t = I.t_now;
    const int64_t c = I.census_off + k;
    double* d = I.census_state + c * 9;
    d[0] = p.x[0]; d[1] = p.x[1]; d[2] = p.x[2];
    d[3] = p.D[0]; d[4] = p.D[1]; d[5] = p.D[2];
    d[6] = p.t; d[7] = p.e; d[8] = p.nu;
    I.census_ind[c] = i;
    I.census_type[c] = TYPE_PHOTON;
  }
}

#include "mixed_kernel.cuh"

// the mixed-form 1D kernel (propagate_mixed_kernel) in one compiled shape
// (zone-scalar tallies go to global memory when MINB blocks' shared-memory
// copies, next to the kernel's static per-thread slots and the block's 1 KB,
// would not fit in an SM's 228 KB)
template <int BATCH, int THREADS, int MINB>
int launch_mixed_t(const StepArgs& a0, const GridDev& g, int blocks_per_sm, int num_sms, int64_t total,
                   cudaStream_t s)
{
  StepArgs a = a0;
  auto kern = propagate_mixed_kernel<BATCH, THREADS, MINB>;
  cudaFuncAttributes fa{};
  cudaFuncGetAttributes(&fa, kern);
  const size_t per_block = (size_t)5 * g.nzones * sizeof(double) + fa.sharedSizeBytes + 1024;
  if (a.smem_zones && (size_t)MINB * per_block > (size_t)228 * 1024) a.smem_zones = 0;
  const size_t smem = a.smem_zones ? (size_t)5 * g.nzones * sizeof(double) : 0;
  if (a.em_n > 0) {  // the core packets, emitted ahead
    int64_t eb = (a.em_n + 255) / 256;
    if (eb > (int64_t)num_sms * 16) eb = (int64_t)num_sms * 16;
    emit_mixed_kernel<BATCH><<<(unsigned)eb, 256, 0, s>>>(a, g);
  }
  if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, THREADS, smem);
  if (per_sm < 1) per_sm = 1;
  if (blocks_per_sm > 0 && blocks_per_sm < per_sm) per_sm = blocks_per_sm;
  int64_t blocks = (int64_t)num_sms * per_sm;
  const int64_t need = (total + THREADS - 1) / THREADS;
  if (blocks > need) blocks = need;
  if (blocks < 1) blocks = 1;
  kern<<<(unsigned)blocks, THREADS, smem, s>>>(a, g);
  return a.em_n > 0 ? 2 : 1;
}

template <int GRID, typename OT, typename CT, int BATCH, int THREADS, int MINB, int MODE = 0,
          bool FAST = (sizeof(OT) == sizeof(float2)), bool DD = false>
int launch_kernel_t(const StepArgs& a, const GridDev& g, int blocks_per_sm, int num_sms, int64_t total,
                    cudaStream_t s)
{
  const size_t smem = a.smem_zones ? (size_t)5 * g.nzones * sizeof(double) : 0;
  auto kern = propagate_kernel<GRID, OT, CT, BATCH, MODE, FAST, THREADS, MINB, DD>;
  if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, THREADS, smem);
  if (per_sm < 1) per_sm = 1;
  if (blocks_per_sm > 0 && blocks_per_sm < per_sm) per_sm = blocks_per_sm;
  int64_t blocks = (int64_t)num_sms * per_sm;
  const int64_t need = (total + THREADS - 1) / THREADS;
  if (blocks > need) blocks = need;
  if (blocks < 1) blocks = 1;
  kern<<<(unsigned)blocks, THREADS, smem, s>>>(a, g);
  return 1;
}

// Single-context shapes: the FP64 form runs best with 256 x 4 (64
// registers; Type Ia step 1753 ms vs 1788 ms at 128 x 8); the mixed form on
// 1D grids is propagate_mixed_kernel (SED_MIXED_THREADS x SED_MIXED_MINB);
// on 3D grids the mixed form runs 128 x 7 (64^3 cells, 2e7 packets: packet
// kernel 572 ms vs 583 ms at 256 x 3).
template <int GRID, typename OT, typename CT>
int launch_propagate_t(const StepArgs& a, const GridDev& g, int num_sms, cudaStream_t s)
{
  // discrete diffusion (1D): the reference's expressions in both forms
  if constexpr (GRID == 0) {
    if (a.use_ddmc == 1 || a.use_ddmc == 2)
      return launch_kernel_t<0, OT, CT, 0, 256, 4, 0, false, true>(a, g, 0, num_sms, a.n_packets, s);
  }
  // mixed tables on a grid with a tabulated velocity field: the reference's
  // expressions (the division-free transforms assume v = x / t)
  if (sizeof(OT) == sizeof(float2) && !g.homologous)
    return launch_kernel_t<GRID, OT, CT, 0, 256, 4, 0, false>(a, g, 0, num_sms, a.n_packets, s);
  if constexpr (sizeof(OT) == sizeof(float2)) {
    if constexpr (GRID == 0) return launch_mixed_t<0, SED_MIXED_THREADS, SED_MIXED_MINB>(a, g, 0, num_sms, a.n_packets, s);
    else return launch_kernel_t<GRID, OT, CT, 0, 128, 7>(a, g, 0, num_sms, a.n_packets, s);
  } else {
    return launch_kernel_t<GRID, OT, CT, 0, 256, 4>(a, g, 0, num_sms, a.n_packets, s);
  }
}

// batched kernel shapes {threads, min blocks per SM}: 32, 28 or 24 warps per
// SM (64, 72 or 80 registers per thread) in blocks of 4 or 8 warps
constexpr int BATCH_SHAPES[BATCH_VARIANTS][2] = {{128, 8}, {256, 4}, {128, 7}, {256, 3}};

template <typename OT, typename CT>
int launch_batch_t(const StepArgs& a, const GridDev& g, int variant, int bps, int num_sms, int64_t total,
                   cudaStream_t s)
{
  if constexpr (sizeof(OT) == sizeof(float2)) {  // mixed form: propagate_mixed_kernel
    switch (variant) {
      case 1: return launch_mixed_t<1, BATCH_SHAPES[1][0], BATCH_SHAPES[1][1]>(a, g, bps, num_sms, total, s);
      case 2: return launch_mixed_t<1, BATCH_SHAPES[2][0], BATCH_SHAPES[2][1]>(a, g, bps, num_sms, total, s);
      case 3: return launch_mixed_t<1, BATCH_SHAPES[3][0], BATCH_SHAPES[3][1]>(a, g, bps, num_sms, total, s);
      default: return launch_mixed_t<1, BATCH_SHAPES[0][0], BATCH_SHAPES[0][1]>(a, g, bps, num_sms, total, s);
    }
  } else {
    switch (variant) {
      case 1: return launch_kernel_t<0, OT, CT, 1, BATCH_SHAPES[1][0], BATCH_SHAPES[1][1]>(a, g, bps, num_sms, total, s);
      case 2: return launch_kernel_t<0, OT, CT, 1, BATCH_SHAPES[2][0], BATCH_SHAPES[2][1]>(a, g, bps, num_sms, total, s);
      case 3: return launch_kernel_t<0, OT, CT, 1, BATCH_SHAPES[3][0], BATCH_SHAPES[3][1]>(a, g, bps, num_sms, total, s);
      default: return launch_kernel_t<0, OT, CT, 1, BATCH_SHAPES[0][0], BATCH_SHAPES[0][1]>(a, g, bps, num_sms, total, s);
    }
  }
}

}  // namespace

bool mixed_1d_path(const StepArgs& a, const GridDev& g)
{
  return a.precision != 0 && g.type == 0 && g.homologous && a.use_ddmc == 0;
}

int launch_propagate(const StepArgs& a, const GridDev& g, int num_sms, cudaStream_t s)
{
  if (g.type == 0) {
    if (a.precision == 0) return launch_propagate_t<0, double2, double>(a, g, num_sms, s);
    return launch_propagate_t<0, float2, float>(a, g, num_sms, s);
  }
  if (a.precision == 0) return launch_propagate_t<1, double2, double>(a, g, num_sms, s);
  return launch_propagate_t<1, float2, float>(a, g, num_sms, s);
}

int launch_imd_probabilities(const GridDev& g, const double* planck, double dt, double* out, cudaStream_t s)
{
  imd_probabilities_kernel<<<(g.nzones + 127) / 128, 128, 0, s>>>(g, planck, dt, out);
  return 1;
}

int launch_finish(const StepArgs& a, const GridDev& g, const double* vol, int64_t nspec, cudaStream_t s)
{
  const int rescale = (a.steady && a.rescale_lum) ? 1 : 0;
  int n = 0;
  if (rescale) {
    rescale_spectrum_kernel<<<64, 256, 0, s>>>(a, nspec, a.n_packets);
    ++n;
  }
  finish_zones_kernel<<<g.nzones, 256, 0, s>>>(a, vol, g.nzones, a.n_packets, rescale);
  return n + 1;
}

template <int GRID>
int launch_diff_t(const StepArgs& b, const GridDev& g, int mode, int num_sms, cudaStream_t s)
{
  constexpr int T = SED_PROP_THREADS, B = SED_PROP_MINB;
  if (b.precision == 0)
    return mode == 1 ? launch_kernel_t<GRID, double2, double, 0, T, B, 1>(b, g, 0, num_sms, b.n_packets, s)
                     : launch_kernel_t<GRID, double2, double, 0, T, B, 2>(b, g, 0, num_sms, b.n_packets, s);
  return mode == 1 ? launch_kernel_t<GRID, float2, float, 0, T, B, 1>(b, g, 0, num_sms, b.n_packets, s)
                   : launch_kernel_t<GRID, float2, float, 0, T, B, 2>(b, g, 0, num_sms, b.n_packets, s);
}

int launch_propagate_diff(const StepArgs& a, const GridDev& g, int mode, int num_sms, cudaStream_t s)
{
  if (!g.homologous || (mode != 1 && mode != 2)) return -1;
  StepArgs b = a;
  if (mode == 2) b.smem_zones = 0;  // the replay tallies nothing per zone
  return g.type == 0 ? launch_diff_t<0>(b, g, mode, num_sms, s) : launch_diff_t<1>(b, g, mode, num_sms, s);
}

int launch_gamma(const StepArgs& a, const StepArgs& ag, const RadioArgs& r, const GridDev& g, int num_sms,
                 cudaStream_t s)
{
  if (r.n_radio <= 0) return 0;
  int64_t blocks = (int64_t)num_sms * 8;
  const int64_t need = (r.n_radio + 127) / 128;
  if (blocks > need) blocks = need;
  if (g.type == 0) {
    if (a.precision == 0) gamma_kernel<0, double><<<(unsigned)blocks, 128, 0, s>>>(a, ag, r, g);
    else gamma_kernel<0, float><<<(unsigned)blocks, 128, 0, s>>>(a, ag, r, g);
  } else {
    if (a.precision == 0) gamma_kernel<1, double><<<(unsigned)blocks, 128, 0, s>>>(a, ag, r, g);
    else gamma_kernel<1, float><<<(unsigned)blocks, 128, 0, s>>>(a, ag, r, g);
  }
  return 1;
}

static unsigned grid_for(int64_t n, int threads, int num_blocks_max)
{
  int64_t b = (n + threads - 1) / threads;
  if (b > num_blocks_max) b = num_blocks_max;
  if (b < 1) b = 1;
  return (unsigned)b;
}

int launch_census_load(const CensusArgs& a, const GridDev& g, cudaStream_t s)
{
  if (a.n_census <= 0) return 0;
  const unsigned b = grid_for(a.n_census, 256, 148 * 16);
  if (g.type == 0) census_load_kernel<0><<<b, 256, 0, s>>>(a, g);
  else census_load_kernel<1><<<b, 256, 0, s>>>(a, g);
  return 1;
}

int launch_census_flags(const CensusArgs& a, int64_t n, cudaStream_t s)
{
  census_flags_kernel<<<grid_for(n + 1, 256, 148 * 16), 256, 0, s>>>(a, n);
  return 1;
}

int launch_census_compact(const CensusArgs& a, int64_t n, cudaStream_t s)
{
  if (n <= 0) return 0;
  census_front_kernel<<<grid_for(n, 256, 148 * 16), 256, 0, s>>>(a, n);
  census_scatter_kernel<<<grid_for(n, 256, 148 * 16), 256, 0, s>>>(a, n);
  return 2;
}

int launch_init_particles(const InitArgs& a, const GridDev& g, cudaStream_t s)
{
  if (a.n <= 0) return 0;
  init_zone_cdf_kernel<<<1, 32, 0, s>>>(a);
  init_bb_cdf_kernel<<<(a.nz + 127) / 128, 128, 0, s>>>(a);
  const unsigned b = grid_for(a.n, 128, 148 * 8);
  if (g.type == 0) init_particles_kernel<0><<<b, 128, 0, s>>>(a, g);
  else init_particles_kernel<1><<<b, 128, 0, s>>>(a, g);
  return 3;
}

void batch_variant_shape(int variant, int* threads, int* min_blocks)
{
  if (variant < 0 || variant >= BATCH_VARIANTS) variant = 0;
  *threads = BATCH_SHAPES[variant][0];
  *min_blocks = BATCH_SHAPES[variant][1];
}

int launch_propagate_batch(const StepArgs& a, const GridDev& g, int variant, int blocks_per_sm, int num_sms,
                           int64_t total_packets, cudaStream_t s)
{
  if (a.precision == 0) return launch_batch_t<double2, double>(a, g, variant, blocks_per_sm, num_sms, total_packets, s);
  return launch_batch_t<float2, float>(a, g, variant, blocks_per_sm, num_sms, total_packets, s);
}

int launch_finish_batch(const StepArgs& a, const double* vol, int nz_total, int64_t nspec, cudaStream_t s)
{
  const int rescale = (a.steady && a.rescale_lum) ? 1 : 0;
  int n = 0;
  if (rescale) {
    rescale_spectrum_batch_kernel<<<148, 256, 0, s>>>(a, nspec);
    ++n;
  }
  finish_zones_batch_kernel<<<nz_total, 256, 0, s>>>(a, vol, nz_total, rescale);
  return n + 1;
}

}  // namespace sed
