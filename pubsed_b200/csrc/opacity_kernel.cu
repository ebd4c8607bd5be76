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
//   bin_opacity_kernel  one thread per (zone, frequency bin): electron
//                       scattering, free-free, bound-free, Sobolev line and
//                       fuzz-line expansion opacity summed in the reference
//                       order (GasState::computeOpacity, GasState_opacities.cpp:11-136).
//                       Line lists are stored sorted by (atom, bin) with a
//                       stable sort, so the lines of one bin are summed in
//                       the reference's list order.  In the mixed-precision
//                       mode the per-line Sobolev sum runs in FP32 with Kahan
//                       compensation; everything else stays FP64.
//   zone_finish_kernel  one block per zone: emissivity CDF (blocked prefix
//                       sum in a fixed order, cdf_array::set_value), opacity
//                       cap, L_thermal, Planck/Rosseland means, Fleck factor,
//                       and the packed tables the packet kernel reads.
//
// The host runs the three kernels once per chunk of zones: per-zone inputs
// and outputs are passed offset to the chunk, and every scratch array
// (index * nzones + zone) is sized for one chunk, so a 128^3-zone grid with
// thousands of bins builds its tables through a bounded working set.
#include <cfloat>
#include <cmath>
#include <mutex>
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

// ------------------------------------------------------------ per bin
__device__ __forceinline__ double bb_nu(double nu, double temp)
{
  const double ezeta = exp(1.0 * H_PLANCK * nu / K_BOLTZ / temp);
  return 2.0 * nu * nu * nu * H_PLANCK / C_LIGHT / C_LIGHT / (ezeta - 1);
}

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

template <bool MIXED>
__global__ void bin_opacity_kernel(const OpacityArgs A)
{
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int nn = A.n_nu, nz = A.nzones;
  if (t >= (int64_t)nz * nn) return;
  const int z = (int)(t / nn), i = (int)(t % nn);
  const double temp = A.temp_c[z];
  const double nu = loc_center(A.nu, i);
  double ab = 0, sc = 0, em = 0;
  const double grey = A.grey[z];
  if (grey != 0) {  // GasState_opacities.cpp:29-41
    const double gopac = A.rho[z] * grey;
    ab = gopac * A.epsilon;
    sc = gopac * (1 - A.epsilon);
    em += bb_nu(nu, temp) * ab;
  } else if (A.natoms > 0) {
    const double ne = A.n_elec[z];
    const double dens = A.rho[z];
    if (A.use_es) {  // :49-58
      const double es = THOMSON * ne;
      sc += es;
      ab += 1e-20 * A.epsilon * es;
    }
    if (A.use_ff) {  // GasState::free_free_opacity :152-183
      double fac = 0;
      for (int a = 0; a < A.natoms; ++a) {
        const int i0 = A.ion_off[a], ni = A.ion_off[a + 1] - i0;
        double zsq = 0;
        for (int j = 0; j < ni; j++) zsq += A.ion_frac[(size_t)(i0 + j) * nz + z] * j * j;
        const double n_ion = A.mass_frac[(size_t)a * nz + z] * dens / (A.eA[a] * MASS_P);
        fac += n_ion * zsq;
      }
      fac *= 3.7e8 * pow(temp, -0.5) * ne;
      const double ezeta = exp(-1.0 * H_PLANCK * nu / K_BOLTZ / temp);
      const double bb = 2.0 * nu * nu * nu * H_PLANCK / C_LIGHT / C_LIGHT / (1.0 / ezeta - 1);
      const double op = fac / nu / nu / nu * (1 - ezeta);
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
        const double nd = A.n_dens[(size_t)a * nz + z];
        double ao = 0, ae = 0;
        for (int j = 0; j < nl; ++j) {
          const int ic = A.lev_ic[l0 + j];
          if (ic == -1) continue;
          const double Eion = A.lev_Eion[l0 + j];
          if (E < Eion) continue;
          const double nc = nd * A.lev_n[(size_t)(l0 + ic) * nz + z];
          const double gl_o_gc = (1.0 * A.lev_g[l0 + j]) / (1.0 * A.lev_g[l0 + ic]);
          const double ncp = nc * gl_o_gc / 2. * lam_t * lam_t * lam_t;
          const double zeta_net = (Eion - E) / kt_ev;
          const double ezeta_net = exp(zeta_net);
          const double sigma = photo_cs(A, l0 + j, E);
          double opac_fac = nd * A.lev_n[(size_t)(l0 + j) * nz + z] - ncp * ne * ezeta_net;
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
    if (A.use_line) {  // GasState::line_expansion_opacity :424-454, AtomicSpecies_opacities.cpp:331-375
      double opac = 0, aopac = 0;
      for (int a = 0; a < A.natoms; ++a) {
        const double this_eps = A.zero_eps_atom[a] ? 0.0 : A.epsilon;
        const int l0 = A.lev_off[a];
        const double nd = A.n_dens[(size_t)a * nz + z];
        double s = 0;
        const int k0 = A.line_seg[(size_t)a * nn + i], k1 = A.line_seg[(size_t)a * nn + i + 1];
        for (int k = k0; k < k1; ++k) {
          const int ll = A.line_l[k], lu = A.line_u[k];
          const double nl = A.lev_n[(size_t)(l0 + ll) * nz + z];
          const double nup = A.lev_n[(size_t)(l0 + lu) * nz + z];
          const double gl = 1.0 * A.lev_g[l0 + ll], gu = 1.0 * A.lev_g[l0 + lu];
          if (nl < DBL_MIN) continue;
          const double lam = C_LIGHT / A.line_nu[k];
          double tau = nl * nd * SIGMA_TOT * A.line_f[k] * A.time * lam;
          tau = tau * (1 - nup * gl / (nl * gu));
          if (nup * gl > nl * gu) tau = 0;
          const double etau = exp(-tau);
          if (!isnan(etau)) s += (1 - etau);
        }
        s = s * nu / loc_delta(A.nu, i) / C_LIGHT / A.time;
        opac += s;
        aopac += s * this_eps;
      }
      ab += aopac;
      sc += opac - aopac;
      em += bb_nu(nu, temp) * aopac;
    }
    if (A.use_fuzz) {  // GasState::fuzz_expansion_opacity :464-494, AtomicSpecies_opacities.cpp:292-324
      double opac = 0, aopac = 0;
      for (int a = 0; a < A.natoms; ++a) {
        const double this_eps = A.zero_eps_atom[a] ? 0.0 : A.epsilon;
        const int i0 = A.ion_off[a];
        const double nd = A.n_dens[(size_t)a * nz + z];
        const int k0 = A.fuzz_seg[(size_t)a * nn + i], k1 = A.fuzz_seg[(size_t)a * nn + i + 1];
        double s;
        if constexpr (MIXED) {
          // FP32 Sobolev sum with Kahan compensation; per-line constants
          // A32 = sigma_tot*lambda*gf, El32 = El/k_ev, hnu32 = h nu/k
          const float invT = (float)(1.0 / temp);
          const float tm = (float)A.time;
          float sum = 0.f, comp = 0.f;
          for (int k = k0; k < k1; ++k) {
            const int ion = A.fz_ion[k];
            const float pop = (float)(nd * A.ion_frac[(size_t)(i0 + ion) * nz + z] / A.ion_part[(size_t)(i0 + ion) * nz + z]);
            const float stim = -expm1f(-__ldg(A.fz_hnu32 + k) * invT);
            const float tau = __ldg(A.fz_A32 + k) * pop * expf(-__ldg(A.fz_El32 + k) * invT) * stim * tm;
            const float term = -expm1f(-tau);
            const float y = term - comp;
            const float tt = sum + y;
            comp = (tt - sum) - y;
            sum = tt;
          }
          s = (double)sum;
        } else {
          s = 0;
          for (int k = k0; k < k1; ++k) {
            const double fnu = A.fz_nu[k], gf = A.fz_gf[k], El = A.fz_El[k];
            const int ion = A.fz_ion[k];
            const double nion = nd * A.ion_frac[(size_t)(i0 + ion) * nz + z];
            const double nl = nion * exp(-1.0 * El / K_EV / temp) / A.ion_part[(size_t)(i0 + ion) * nz + z];
            const double lam = C_LIGHT / fnu;
            const double stim_cor = (1 - exp(-H_PLANCK * fnu / K_BOLTZ / temp));
            const double tau = SIGMA_TOT * lam * nl * gf * stim_cor * A.time;
            const double etau = exp(-tau);
            s += (1 - etau);
          }
        }
        s = s * nu / loc_delta(A.nu, i) / C_LIGHT / A.time;
        opac += s;
        aopac += s * this_eps;
      }
      ab += aopac;
      sc += opac - aopac;
      em += bb_nu(nu, temp) * aopac;
    }
  }
  A.abs64[t] = ab;
  A.scat64[t] = sc;
  A.emis64[t] = em;
}

// emissivity CDF, cap, L_thermal, means, eps_imc (transport_opacity.cpp:152-252)
// The CDF prefix sum and L_thermal are sequential (cdf_array::set_value
// order); the Planck and Rosseland means are block reductions in a fixed
// order (strided partial sums, then a tree).
template <bool MIXED>
__global__ void __launch_bounds__(256) zone_finish_kernel(const OpacityArgs A)
{
  __shared__ double red[4][256];
  const int z = blockIdx.x;
  if (z >= A.nzones) return;
  const int nn = A.n_nu;
  double* ab = A.abs64 + (size_t)z * nn;
  double* sc = A.scat64 + (size_t)z * nn;
  double* em = A.emis64 + (size_t)z * nn;
  const double max_ext = A.max_opacity * A.rho[z];
  const double temp = A.temp_c[z];
  // cap (element-wise) and the mean-opacity partial sums
  double pm = 0, pn = 0, rm = 0, rn = 0;
  for (int j = threadIdx.x; j < nn; j += blockDim.x) {
    double s = sc[j];
    if (A.omit_scat) s = 0;
    else if (s > max_ext) s = max_ext;
    sc[j] = s;
    double a = ab[j];
    if (a > max_ext) a = max_ext;
    ab[j] = a;
    // GasState::get_planck_mean / get_rosseland_mean (GasState_opacities.cpp:564-666)
    const double nu = loc_center(A.nu, j);
    const double zeta = H_PLANCK * nu / K_BOLTZ / temp;
    double Bnu = 2.0 * nu * nu * nu * H_PLANCK / C_LIGHT / C_LIGHT / (exp(zeta) - 1);
    if (isnan(Bnu)) Bnu = 0;
    const double d = loc_delta(A.nu, j);
    const double W = Bnu * d;
    pm += W * a;
    pn += W;
    const double ezeta = exp(zeta);
    double dBdT = pow(nu, 4) * ezeta / (ezeta - 1) / (ezeta - 1);
    if (isnan(dBdT)) dBdT = 0;
    const double Wr = dBdT * d;
    rm += Wr / (a + s);
    rn += Wr;
  }
  red[0][threadIdx.x] = pm; red[1][threadIdx.x] = pn; red[2][threadIdx.x] = rm; red[3][threadIdx.x] = rn;
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if (threadIdx.x < (unsigned)st)
      for (int q = 0; q < 4; ++q) red[q][threadIdx.x] += red[q][threadIdx.x + st];
    __syncthreads();
  }
  const double pm_tot = red[0][0], pn_tot = red[1][0], rm_tot = red[2][0], rn_tot = red[3][0];
  __syncthreads();
  // emissivity CDF: cdf_array::set_value prefix sum of emis*dnu (cdf_array.h:53-75)
  // and L_thermal = 4 pi sum(emis*dnu).  Blocked scan in a fixed order: each
  // thread sums a contiguous run of bins, thread 0 scans the 256 run totals,
  // each run then adds its offset.  Non-negative terms, so every prefix is
  // within a few ulp of the sequential sum; a NaN term propagates to the end
  // of the CDF exactly as in the sequential sum.
  double L = 0;
  if (nn == 1) {
    if (threadIdx.x == 0) {
      const double bb_int = SB * pow(A.T[z], 4) / PI;
      L += 4 * PI * ab[0] * bb_int;
      em[0] = 1;
    }
  } else {
    const int per = (nn + blockDim.x - 1) / blockDim.x;
    const int j0 = min(nn, (int)threadIdx.x * per), j1 = min(nn, j0 + per);
    double run = 0, Lp = 0;
    for (int j = j0; j < j1; ++j) {
      const double ednu = em[j] * loc_delta(A.nu, j);
      run = (j == j0) ? ednu : run + ednu;
      em[j] = run;
      Lp += 4 * PI * ednu;
    }
    red[0][threadIdx.x] = run;
    red[1][threadIdx.x] = Lp;
    __syncthreads();
    if (threadIdx.x == 0) {
      double acc = 0, Lacc = 0;
      for (int t = 0; t < (int)blockDim.x; ++t) {
        const double v = red[0][t];
        red[0][t] = acc;
        acc = (t == 0) ? v : acc + v;
        Lacc += red[1][t];
      }
      red[2][0] = Lacc;
    }
    __syncthreads();
    const double off = red[0][threadIdx.x];
    if (threadIdx.x > 0)
      for (int j = j0; j < j1; ++j) em[j] = off + em[j];
    L = red[2][0];
  }
  __syncthreads();
  for (int j = threadIdx.x; j < nn; j += blockDim.x) if (isnan(em[j])) em[j] = 0;
  __syncthreads();
  const bool all_zero = (em[nn - 1] == 0);
  __syncthreads();
  if (all_zero) for (int j = threadIdx.x; j < nn; j += blockDim.x) em[j] = 1.0;
  __syncthreads();
  if (threadIdx.x == 0) {
    A.L_th[z] = L;
    if (nn == 1) {
      A.planck[z] = ab[0];
      A.ross[z] = ab[0] + sc[0];
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
  __syncthreads();
  const double N = em[nn - 1];
  // normalised CDF, packed tables and the coarse CDF index for the packet kernel
  for (int j = threadIdx.x; j < nn; j += blockDim.x) {
    const size_t k = (size_t)z * nn + j;
    const double c = em[j] / N;
    if constexpr (MIXED) {
      reinterpret_cast<float2*>(A.opac_out)[k] = make_float2((float)ab[j], (float)sc[j]);
      reinterpret_cast<float*>(A.cdf_out)[k] = (float)c;
    } else {
      reinterpret_cast<double2*>(A.opac_out)[k] = make_double2(ab[j], sc[j]);
      reinterpret_cast<double*>(A.cdf_out)[k] = c;
    }
    if ((j % CDF_STRIDE) == CDF_STRIDE - 1 || j == nn - 1) {
      const size_t kc = (size_t)z * A.n_coarse + j / CDF_STRIDE;
      if constexpr (MIXED) reinterpret_cast<float*>(A.cdf_coarse_out)[kc] = (float)c;
      else reinterpret_cast<double*>(A.cdf_coarse_out)[kc] = c;
    }
  }
  __syncthreads();
  for (int j = threadIdx.x; j < nn; j += blockDim.x) em[j] = em[j] / N;
}

}  // namespace

int launch_opacity(const OpacityArgs& a, int num_sms, cudaStream_t s)
{
  (void)num_sms;
  const int nz = a.nzones;
  zone_state_kernel<<<(nz + 127) / 128, 128, 0, s>>>(a, a.boltz);
  const int64_t nt = (int64_t)nz * a.n_nu;
  const int threads = 256;
  const unsigned blocks = (unsigned)((nt + threads - 1) / threads);
  if (a.precision) bin_opacity_kernel<true><<<blocks, threads, 0, s>>>(a);
  else bin_opacity_kernel<false><<<blocks, threads, 0, s>>>(a);
  if (a.precision) zone_finish_kernel<true><<<nz, 256, 0, s>>>(a);
  else zone_finish_kernel<false><<<nz, 256, 0, s>>>(a);
  return 3;
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
  const size_t need = nz * (2 * na + 2 + 2 * ni + 2 * nl);
  if (need > NOALLOC_SCRATCH_DOUBLES) return SED_ERR_CAPACITY;  // limit stated in include/sedona_gpu.h

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
