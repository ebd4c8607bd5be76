// radioactive_kernel.cu -- per-zone quantities of the radioactive source:
// decay luminosity and its gamma-ray fraction (radioactive::decay,
// src/transport/radioactive.cpp:144-275), the gamma-ray Compton and
// photo-electric opacity coefficients (transport_opacity.cpp:187-203), and
// the zone emission CDF of transport::emit_radioactive
// (src/transport/emission.cpp:189-205).
#include <cmath>
#include "sed_internal.h"

namespace sed {

namespace {

// decay data and timescales (src/transport/radioactive.h:11-35)
constexpr double TAU_56NI = 757241.8;
constexpr double TAU_56CO = 9627379.;
constexpr double AVERAGE_56NI_ENERGY = 1.725;
constexpr double AVERAGE_56CO_ENERGY = 3.730;
constexpr double CO_POSITRON_FRACTION = 0.0324;
constexpr double TAU_48CR = 111976.;
constexpr double TAU_48V = 1.99107843e6;
constexpr double AVERAGE_48CR_ENERGY = 0.442;
constexpr double AVERAGE_48V_ENERGY = 3.066;

// fit of the r-process heating rate in log10 t (radioactive.cpp:46-48)
__constant__ double R_PROC_FIT[11] = {17.608179, -2.0442059, -0.42565322, 0.39830095, -0.0059089906,
                                      -0.054805836, 0.014068697, -0.00086706160, -5.7056758e-05, 2.6401842e-06,
                                      3.7186979e-07};

// radioactive::rprocess_heating_rate (radioactive.cpp:118-142): Lippuner &
// Roberts fit times the Barnes et al. thermalisation efficiency
__device__ double rprocess_heating_rate(double t, double* gfrac)
{
  const double td = t / 3600.0 / 24.0;
  const double A1 = 8.4939E+09, alpha = 1.3642E+00, B1 = 8.3425E+09, beta1 = 3.6280E+00;
  const double B2 = 8.8616E+08, beta2 = 1.0847E+01;
  const double eps = A1 * pow(td, -1.0 * alpha) + B1 * exp(-1.0 * td / beta1) + B2 * exp(-1.0 * td / beta2);
  const double af = 0.56, bf = 0.17, df = 0.74;
  const double x = 2 * bf * pow(td, df);
  const double f = 0.36 * (exp(-af * td) + log(1 + x) / x);
  *gfrac = 0;
  return eps * f;
}

// radioactive::decay_energy_rate (radioactive.cpp:178-275)
__device__ double decay_energy_rate(int Z, int A, double t, double* gfrac)
{
  double total = 0, gtotal = 0;
  if ((Z == 28) && (A == 56)) {
    const double e_ni = exp(-t / TAU_56NI), e_co = exp(-t / TAU_56CO);
    const double ni56 = (e_ni / TAU_56NI);
    const double co56 = 1.0 / (TAU_56NI - TAU_56CO) * (e_ni - e_co);
    const double ni_E = ni56 * (AVERAGE_56NI_ENERGY * MEV_TO_ERGS);
    const double co_E = co56 * (AVERAGE_56CO_ENERGY * MEV_TO_ERGS);
    gtotal = ni_E + (1 - CO_POSITRON_FRACTION) * co_E;
    total = ni_E + co_E;
  }
  if ((Z == 27) && (A == 56)) {
    const double e_co = exp(-t / TAU_56CO);
    const double co56 = 1.0 / (TAU_56CO)*e_co;
    const double co_E = co56 * (AVERAGE_56CO_ENERGY * MEV_TO_ERGS);
    gtotal = (1 - CO_POSITRON_FRACTION) * co_E;
    total = co_E;
  }
  if ((Z == 24) && (A == 48)) {
    const double e_cr = exp(-t / TAU_48CR), e_vn = exp(-t / TAU_48V);
    const double cr48 = (e_cr / TAU_48CR);
    const double vn48 = 1.0 / (TAU_48CR - TAU_48V) * (e_cr - e_vn);
    const double cr_E = cr48 * (AVERAGE_48CR_ENERGY * MEV_TO_ERGS);
    const double vn_E = vn48 * (AVERAGE_48V_ENERGY * MEV_TO_ERGS);
    gtotal += cr_E + vn_E;
    total += cr_E + vn_E;
  }
  if ((Z >= 58)) {
    const double at = log10(t);
    double rproc = 0;
    for (int j = 0; j < 11; j++) rproc += R_PROC_FIT[j] * pow(at, j);
    rproc = pow(10.0, rproc) * (A * MASS_P);
    const double fission_E = 0.1 * rproc;
    double beta_E = 0.9 * rproc;
    beta_E = 0.75 * beta_E;
    total += (fission_E + beta_E);
    gtotal += 0.5 * beta_E;
  }
  *gfrac = gtotal / total;
  if (total == 0) *gfrac = 0;
  return total;
}

// One thread per zone: radioactive::decay (radioactive.cpp:144-176) times
// rho vol (emission.cpp:196-198), and the gamma opacity coefficients.
__global__ void radio_zone_kernel(const RadioArgs A)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.nz) return;
  const int ne = A.n_elems;
  const double* X = A.X + (size_t)i * ne;
  int rprocess_heat = 0;
  for (int k = 0; k < ne; ++k)
    if (((A.eZ[k] > 57) && (A.eA[k] > 0)) || A.force_rproc) rprocess_heat = 1;
  double L_decay, gfrac;
  if (rprocess_heat) {
    L_decay = rprocess_heating_rate(A.t_now, &gfrac);
  } else {
    double total = 0, gtotal = 0, gf;
    for (int k = 0; k < ne; ++k) {
      const int el_Z = A.eZ[k], el_A = A.eA[k];
      double val = decay_energy_rate(el_Z, el_A, A.t_now, &gf);
      val = val * X[k] / (el_A * MASS_P);
      total += val;
      gtotal += val * gf;
    }
    gfrac = gtotal / total;
    if (total == 0) gfrac = 0;
    L_decay = total;
  }
  L_decay = A.rho[i] * L_decay * A.vol[i];
  A.L_emit[i] = L_decay;
  A.gamma_frac[i] = gfrac;
  A.cdf[i] = L_decay;
  // gamma-ray opacity: Compton (Thomson per electron) and photo-electric
  double comp = 0, phot = 0;
  for (int k = 0; k < ne; ++k) {
    const double dens = X[k] * A.rho[i];
    const double ndens = dens / (MASS_P * A.eA[k]);
    comp += ndens * THOMSON * A.eZ[k];
    double photo = pow(ALPHA_FS, 4.0) * 4.0 * sqrt(2.0);
    photo *= pow(1.0 * A.eZ[k], 5.0);
    photo *= pow(M_E_MEV, 3.5);
    phot += ndens * 2.0 * THOMSON * photo;
  }
  A.compton[i] = comp;
  A.photoion[i] = phot;
}

// cdf_array::set_value / normalize (src/transport/cdf_array.h:53-75) over the
// zones: a blocked prefix sum in a fixed order (per-thread contiguous runs,
// then the run totals), the grid total, NaN -> 0, an all-zero CDF -> all 1,
// then the division by the last value.  One CTA.
__global__ void radio_cdf_kernel(const RadioArgs A)
{
  __shared__ double run_sum[1024];
  const int nz = A.nz, tid = threadIdx.x, bd = blockDim.x;
  const int per = (nz + bd - 1) / bd;
  const int j0 = min(nz, tid * per), j1 = min(nz, j0 + per);
  double run = 0;
  for (int j = j0; j < j1; ++j) {
    run = (j == j0) ? A.cdf[j] : run + A.cdf[j];
    A.cdf[j] = run;
  }
  run_sum[tid] = (j1 > j0) ? run : 0.0;
  __syncthreads();
  if (tid == 0) {
    double acc = 0;
    for (int t = 0; t < bd; ++t) {
      const double v = run_sum[t];
      run_sum[t] = acc;
      acc = (t == 0) ? v : acc + v;
    }
    *A.L_tot = acc;
  }
  __syncthreads();
  const double off = run_sum[tid];
  if (tid > 0)
    for (int j = j0; j < j1; ++j) A.cdf[j] = off + A.cdf[j];
  __syncthreads();
  for (int j = tid; j < nz; j += bd) if (isnan(A.cdf[j])) A.cdf[j] = 0;
  __syncthreads();
  const bool all_zero = (A.cdf[nz - 1] == 0);
  __syncthreads();
  if (all_zero) for (int j = tid; j < nz; j += bd) A.cdf[j] = 1.0;
  __syncthreads();
  const double N = A.cdf[nz - 1];
  __syncthreads();
  for (int j = tid; j < nz; j += bd) A.cdf[j] /= N;
}

}  // namespace

int launch_radio_zones(const RadioArgs& a, cudaStream_t s)
{
  if (a.nz <= 0) return 0;
  radio_zone_kernel<<<(a.nz + 127) / 128, 128, 0, s>>>(a);
  radio_cdf_kernel<<<1, 1024, 0, s>>>(a);
  return 2;
}

}  // namespace sed
