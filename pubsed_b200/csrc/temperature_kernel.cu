// temperature_kernel.cu -- the radiative-equilibrium gas temperature that
// ends transport::step (src/transport/solve_equilibrium.cpp:66-96, LTE).
//
// One thread per zone runs temp_brent_method (:227-320) on
// rad_eq_function_LTE with solve_flag 0 (:113-170): the zone's emission
// sum_i 4 pi kappa_abs,i B_nu(T) dnu_i, with the absorption opacities of
// the last opacity build, minus its normalised absorbed-energy tally e_abs.
// The sum runs over the bins in order, as in the reference, so the iterates
// are the reference's.  Compiled without FMA contraction like the rest.
#include <cmath>
#include "sed_internal.h"

namespace sed {

namespace {

// transport::blackbody_nu (src/transport/transport_opacity.cpp:322-326)
__device__ __forceinline__ double blackbody_nu(double T, double nu)
{
  const double zeta = H_PLANCK * nu / K_BOLTZ / T;
  return 2.0 * nu * nu * nu * H_PLANCK / C_LIGHT / C_LIGHT / (exp(zeta) - 1);
}

template <typename OT>
__device__ double rad_eq_lte(const OT* __restrict__ row, const DevLoc& nu, double e_abs, double T)
{
  double E_emitted = 0.;
  const double E_absorbed = e_abs;
  if (nu.n == 1) {
    E_emitted = 4.0 * PI * (double)row[0].x * SB / PI * pow(T, 4);
  } else {
    for (int i = 0; i < nu.n; i++) {
      const double dnu = loc_delta(nu, i);
      const double nc = loc_center(nu, i);
      const double B_nu = blackbody_nu(T, nc);
      const double kappa_abs = (double)__ldg(&row[i].x);
      E_emitted += 4.0 * PI * kappa_abs * B_nu * dnu;
    }
  }
  return (E_emitted - E_absorbed);
}

template <typename OT>
__global__ void temperature_kernel(const TemperatureArgs A)
{
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= A.nz) return;
  if (A.set_Tgas_to_Trad) {
    A.T[c] = pow(A.e_rad[c] / A_RAD, 0.25);
    return;
  }
  const OT* row = reinterpret_cast<const OT*>(A.opac) + (size_t)c * A.nu.n;
  const double e_abs = A.e_abs[c];
  const double brent_solve_tolerance = 1.0e-2;
  const int ITMAX = 100;
  const double EPS = 3.0e-8;
  double a = A.temp_min, b = A.temp_max, cc = b, d = 0, e = 0, min1, min2;
  double fa = rad_eq_lte<OT>(row, A.nu, e_abs, a), fb = rad_eq_lte<OT>(row, A.nu, e_abs, b);
  double fc, p, q, r, s, tol1, xm;
  fc = fb;
  for (int iter = 1; iter <= ITMAX; iter++) {
    if ((fb > 0.0 && fc > 0.0) || (fb < 0.0 && fc < 0.0)) { cc = a; fc = fa; e = d = b - a; }
    if (fabs(fc) < fabs(fb)) { a = b; b = cc; cc = a; fa = fb; fb = fc; fc = fa; }
    tol1 = 2.0 * EPS * fabs(b) + 0.5 * brent_solve_tolerance;
    xm = 0.5 * (cc - b);
    if (fabs(xm) <= tol1 || fb == 0.0) {
      A.T[c] = b;
      return;
    }
    if (fabs(e) >= tol1 && fabs(fa) > fabs(fb)) {
      s = fb / fa;
      if (a == cc) { p = 2.0 * xm * s; q = 1.0 - s; }
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
    if (fabs(d) > tol1) b += d;
    else b += (xm >= 0.0 ? fabs(tol1) : -fabs(tol1));
    fb = rad_eq_lte<OT>(row, A.nu, e_abs, b);
  }
  // the reference prints "Maximum number of iterations exceeded" and uses 0
  A.T[c] = 0.0;
  atomicAdd(A.n_unsolved, 1);
}

}  // namespace

int launch_temperature(const TemperatureArgs& a, cudaStream_t s)
{
  const int threads = 128;
  const int blocks = (a.nz + threads - 1) / threads;
  if (blocks == 0) return 0;
  if (a.precision) temperature_kernel<float2><<<blocks, threads, 0, s>>>(a);
  else temperature_kernel<double2><<<blocks, threads, 0, s>>>(a);
  return 1;
}

}  // namespace sed
