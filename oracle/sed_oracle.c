/* oracle/sed_oracle.c -- TEST INFRASTRUCTURE (the oracle; never shipped).
 *
 * Plain-C restatement of the reference's implicit Monte Carlo transport step
 * for the functions on the GPU hot path.  Every function names the reference
 * file:line it follows (paths relative to the reference checkout).  The
 * arithmetic is written in the same order as the reference so that, compiled
 * without floating-point contraction, results match the reference bit for bit
 * up to the last-ulp behaviour of libm (log, exp, pow, sin, cos, atan2).
 *
 * Random numbers: the reference draws from per-thread GSL generators
 * (src/transport/thread_RNG.cpp:91-99); here draw n of packet p comes from the
 * Philox4x32-10 stream (seed, p, step) defined in oracle/philox.h, which the
 * reference harness (oracle/ref) also installs in place of GSL.
 */
#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "sed_oracle.h"
#include "philox.h"

/* physical constants, src/utils/physical_constants.h:9-31 (pi is 3.14159 there) */
#define PC_PI 3.14159
#define PC_C 2.99792458e10
#define PC_H 6.6260755e-27
#define PC_K 1.380658e-16
#define PC_K_EV 8.6173324e-5
#define PC_M_P 1.67262158e-24
#define PC_M_E 9.10938188e-28
#define PC_SB 5.6704e-5
#define PC_A 7.5657e-15
#define PC_THOMSON 0.66523e-24
#define PC_SIGMA_TOT 0.0265400193567
#define PC_ERGS_TO_EV 624150975230.2815

enum { F_MOVING = 0, F_STOPPED = 1, F_ESCAPED = 2, F_ABSORBED = 3 };

typedef struct {
  int n, type;
  double min, del;
  double* x;
} lgrid;

typedef struct {
  double x[3], D[3], t, e, nu, dvds;
  int ind;
  int fate;
  uint64_t pid;
  uint32_t n;  /* next deviate index */
} packet;

struct oracle_ctx {
  sed_transport_params tp;
  lgrid nu, st, sn, sm, sp;
  /* grid */
  int have_grid, gtype, nzones, homologous, nelem;
  double t_grid, r_min;
  lgrid r_out;
  double* v_r;
  int nx, ny, nz;
  lgrid ax[3];
  double *vol, *rho, *T, *e_gas, *grey, *X;
  int *eZ, *eA;
  /* atomic data */
  int have_atoms;
  int natoms;
  int *ion_off, *lev_off, *lev_ion, *lev_g, *lev_ic, *photo_off, *line_off, *line_l, *line_u, *line_bin;
  double *ion_chi, *lev_E, *lev_Eion, *photo_E, *photo_s, *line_nu, *line_f;
  int *fuzz_off, *fuzz_ion, *fuzz_bin;
  double *fuzz_nu, *fuzz_gf, *fuzz_El;
  sed_opacity_params op;
  int* zero_eps;
  /* tables */
  int have_opacity;
  double *abs, *scat, *cdf, *eps_imc, *n_elec, *planck, *ross, *L_th;
  double core_cdf_dummy;
  double* core_cdf;
  /* tallies */
  double *J, *e_abs, *e_rad, *fx, *fy, *fz, *fr;
  double *flux, *click;
  int64_t nspec;
  int64_t n_escaped_acc, n_active_acc;
  /* records */
  int record;
  int64_t nrec;
  int32_t *r_fate, *r_ind, *r_draws;
  double* r_state;
  uint32_t step;
  /* radioactive source: gamma-ray spectrum and per-zone decay quantities */
  lgrid gn;
  int64_t nspec_g;
  double *gflux, *gclick;
  int64_t n_reject_cap;  /* Compton scatters that hit the rejection bound */
  int64_t n_limit;       /* packets of the step stopped by the segment limit */
  /* the built {abs, scat} tables while density-scaled ones are in abs/scat */
  double *abs_base, *scat_base;
  int base_valid;
  /* IMD (transport_use_ddmc = 1): per-zone hop / stay / absorption
   * probabilities of the step (compute_diffusion_probabilities) */
  double *imd_up, *imd_dn, *imd_stay, *imd_abs;
  int64_t n_imd_cap;     /* IMD calls that hit the hop bound */
  /* transport clock (transport::t_now_) and the packets carried to the next
   * step, in the reference's vector order */
  double t_now;
  int have_t_now;
  int64_t n_census;
  double* c_state;
  int32_t *c_ind, *c_type;
  int32_t* r_type;
  double *L_emit, *L_dep, *radio_cdf, *gamma_frac, *compton, *photoion;
  /* differentiable transport: exact Jacobian of the last weighted forward,
   * accumulated forward-mode per packet ([nspec][nzones][bands]) */
  double* jac;
  double* jac_rho;  /* [nspec][nzones] d flux / d ln rho of the last weighted forward */
  int64_t jac_n;
  int diff_bands;
  char err[256];
};

static int fail(oracle_ctx* o, int code, const char* msg)
{
  snprintf(o->err, sizeof o->err, "%s", msg);
  return code;
}

/* ---------------------------------------------------------------- locate_array */
static void lgrid_copy(lgrid* g, const sed_locate_grid* s)
{
  free(g->x);
  g->n = s->n; g->type = s->type; g->min = s->min; g->del = s->del;
  g->x = (double*)malloc(sizeof(double) * (size_t)(s->n > 0 ? s->n : 1));
  for (int i = 0; i < s->n; ++i) g->x[i] = s->right[i];
}
static double lg_left(const lgrid* g, int i) { return i == 0 ? g->min : g->x[i - 1]; } /* locate_array.h:60-62 */
static double lg_delta(const lgrid* g, int i) { return i == 0 ? g->x[0] - g->min : g->x[i] - g->x[i - 1]; } /* :69-72 */
static double lg_center(const lgrid* g, int i) { return i == 0 ? 0.5 * (g->min + g->x[0]) : 0.5 * (g->x[i - 1] + g->x[i]); } /* :54-57 */
static int upper_bound_d(const double* a, int n, double v)
{
  int lo = 0, hi = n;
  while (lo < hi) { int m = lo + (hi - lo) / 2; if (a[m] <= v) lo = m + 1; else hi = m; }
  return lo;
}
/* locate_array::locate, src/utils/locate_array.cpp:191-218 */
static int lg_locate(const lgrid* g, double xv)
{
  if (g->n == 1) return 0;
  if (xv >= g->x[g->n - 1]) return g->n;
  if (xv < g->min) return 0;
  int ind;
  if (g->type == SED_LOC_FLEX) ind = upper_bound_d(g->x, g->n, xv);
  else if (g->type == SED_LOC_LIN) ind = (int)floor((xv - g->min) / g->del);
  else if (g->type == SED_LOC_LOG) ind = (int)floor(log(xv / g->min) / log(1 + g->del));
  else ind = 0;
  if (g->type != SED_LOC_NONE && ind != 0 && ind != g->n && (lg_left(g, ind) > xv || g->x[ind] <= xv))
    ind = upper_bound_d(g->x, g->n, xv);
  return ind;
}
/* locate_array::locate_within_bounds, locate_array.cpp:225-230 */
static int lg_locate_wb(const lgrid* g, double xv)
{
  int ind = lg_locate(g, xv);
  if (ind == g->n) return g->n - 1;
  return ind;
}
/* locate_array::sample, locate_array.cpp:237-242 */
static double lg_sample(const lgrid* g, int i, double r)
{
  if (g->n == 1) return 0;
  if (i == 0) return g->min + (g->x[0] - g->min) * r;
  return g->x[i - 1] + (g->x[i] - g->x[i - 1]) * r;
}
int oracle_locate(const sed_locate_grid* s, double x)
{
  lgrid g = {0};
  lgrid_copy(&g, s);
  int r = lg_locate(&g, x);
  free(g.x);
  return r;
}

/* cdf_array::sample, src/transport/cdf_array.h:84-89 */
static int cdf_sample(const double* y, int n, double u)
{
  if (n == 1) return 0;
  return upper_bound_d(y, n, u);
}
/* cdf_array::normalize, cdf_array.h:62-75 */
static void cdf_normalize(double* y, int n)
{
  for (int i = 0; i < n; ++i) if (isnan(y[i])) y[i] = 0;
  if (y[n - 1] == 0) for (int i = 0; i < n; ++i) y[i] = 1.0;
  double N = y[n - 1];
  for (int i = 0; i < n; ++i) y[i] /= N;
}

/* ---------------------------------------------------------------- context */
static void alloc_gamma_spectrum(oracle_ctx* o)
{
  if (o->gflux) return;
  o->nspec_g = (int64_t)o->st.n * o->gn.n * o->sm.n * o->sp.n;
  o->gflux = (double*)calloc((size_t)o->nspec_g, sizeof(double));
  o->gclick = (double*)calloc((size_t)o->nspec_g, sizeof(double));
}

int oracle_ctx_create(const sed_transport_params* p, oracle_ctx** out)
{
  if (!p || !out) return SED_ERR_ARG;
  oracle_ctx* o = (oracle_ctx*)calloc(1, sizeof(oracle_ctx));
  o->tp = *p;
  lgrid_copy(&o->nu, &p->nu_grid);
  lgrid_copy(&o->st, &p->spec_time);
  lgrid_copy(&o->sn, &p->spec_nu);
  lgrid_copy(&o->sm, &p->spec_mu);
  lgrid_copy(&o->sp, &p->spec_phi);
  o->nspec = (int64_t)o->st.n * o->sn.n * o->sm.n * o->sp.n;
  o->flux = (double*)calloc((size_t)o->nspec, sizeof(double));
  o->click = (double*)calloc((size_t)o->nspec, sizeof(double));
  /* core emission spectrum, transport::setup_core_emission
   * (src/transport/transport_init.cpp:465-556), blackbody branch */
  int nn = o->nu.n;
  o->core_cdf = (double*)calloc((size_t)nn, sizeof(double));
  for (int j = 0; j < nn; ++j) {
    double nu = lg_center(&o->nu, j), dnu = lg_delta(&o->nu, j);
    double bb;
    if (p->core_temperature <= 0) bb = 1;
    else {
      double zeta = PC_H * nu / PC_K / p->core_temperature;  /* blackbody_nu, transport_opacity.cpp:322-326 */
      bb = 2.0 * nu * nu * nu * PC_H / PC_C / PC_C / (exp(zeta) - 1);
    }
    double w = bb * dnu * 1.0;  /* emissivity_weight_ = 1 (transport_init.cpp:322-332) */
    o->core_cdf[j] = (j == 0) ? w : o->core_cdf[j - 1] + w;
  }
  cdf_normalize(o->core_cdf, nn);
  /* the gamma-ray spectrum (used once a step emits radioactive packets) */
  if (p->gamma_nu.n > 0 && p->gamma_nu.right) lgrid_copy(&o->gn, &p->gamma_nu);
  else {  /* one catch-all bin */
    o->gn.n = 1; o->gn.type = SED_LOC_NONE; o->gn.min = -INFINITY; o->gn.del = 0;
    o->gn.x = (double*)malloc(sizeof(double)); o->gn.x[0] = INFINITY;
  }
  if (p->n_emit_radioactive > 0) alloc_gamma_spectrum(o);
  *out = o;
  return SED_OK;
}

static void free_grid(oracle_ctx* o)
{
  free(o->r_out.x); o->r_out.x = NULL;
  for (int a = 0; a < 3; ++a) { free(o->ax[a].x); o->ax[a].x = NULL; }
  free(o->v_r); free(o->vol); free(o->rho); free(o->T); free(o->e_gas); free(o->grey); free(o->X);
  free(o->eZ); free(o->eA);
  free(o->J); free(o->e_abs); free(o->e_rad); free(o->fx); free(o->fy); free(o->fz); free(o->fr);
  free(o->abs); free(o->scat); free(o->cdf); free(o->eps_imc); free(o->n_elec); free(o->planck); free(o->ross); free(o->L_th);
  free(o->imd_up); free(o->imd_dn); free(o->imd_stay); free(o->imd_abs);
  o->imd_up = o->imd_dn = o->imd_stay = o->imd_abs = NULL;
  free(o->abs_base); free(o->scat_base);
  o->abs_base = o->scat_base = NULL;
  o->base_valid = 0;
  o->v_r = o->vol = o->rho = o->T = o->e_gas = o->grey = o->X = NULL;
  o->eZ = o->eA = NULL;
}

static double* dup_d(const double* s, size_t n, double fill)
{
  double* d = (double*)malloc(sizeof(double) * (n ? n : 1));
  for (size_t i = 0; i < n; ++i) d[i] = s ? s[i] : fill;
  return d;
}
static int* dup_i(const int32_t* s, size_t n)
{
  int* d = (int*)malloc(sizeof(int) * (n ? n : 1));
  for (size_t i = 0; i < n; ++i) d[i] = s ? s[i] : 0;
  return d;
}

int oracle_set_grid(oracle_ctx* o, const sed_grid* g)
{
  if (!o || !g || g->n_zones <= 0) return SED_ERR_ARG;
  free_grid(o);
  o->gtype = g->type;
  o->nzones = g->n_zones;
  o->homologous = g->homologous;
  o->nelem = g->n_elems;
  o->t_grid = g->t_now;
  /* transport::init takes the grid's time; a time-dependent run keeps its
   * own clock afterwards */
  if (!o->have_t_now || o->tp.steady_state) { o->t_now = g->t_now; o->have_t_now = 1; }
  size_t nz = (size_t)g->n_zones;
  if (g->type == SED_GRID_1D_SPHERE) {
    sed_locate_grid rg = {g->n_zones, SED_LOC_FLEX, g->r_min, 0.0, g->r_out};
    memset(&o->r_out, 0, sizeof o->r_out);
    lgrid_copy(&o->r_out, &rg);
    o->r_min = g->r_min;
    o->v_r = dup_d(g->v_r, nz, 0.0);
  } else if (g->type == SED_GRID_3D_CART) {
    if ((int64_t)g->nx * g->ny * g->nz != g->n_zones) return fail(o, SED_ERR_ARG, "nx*ny*nz != n_zones");
    o->nx = g->nx; o->ny = g->ny; o->nz = g->nz;
    memset(o->ax, 0, sizeof o->ax);
    lgrid_copy(&o->ax[0], &g->x_axis);
    lgrid_copy(&o->ax[1], &g->y_axis);
    lgrid_copy(&o->ax[2], &g->z_axis);
  } else {
    return fail(o, SED_ERR_ARG, "unsupported grid type");
  }
  o->vol = dup_d(g->vol, nz, 0.0);
  o->rho = dup_d(g->rho, nz, 0.0);
  o->T = dup_d(g->T_gas, nz, 0.0);
  o->e_gas = dup_d(g->e_gas, nz, 0.0);
  o->grey = dup_d(g->total_grey_opacity, nz, 0.0);
  o->X = dup_d(g->X, nz * (size_t)(g->n_elems > 0 ? g->n_elems : 0), 0.0);
  o->eZ = dup_i(g->elem_Z, (size_t)g->n_elems);
  o->eA = dup_i(g->elem_A, (size_t)g->n_elems);
  size_t nn = (size_t)o->nu.n;
  size_t nj = o->tp.store_Jnu ? nn : 1;
  o->J = (double*)calloc(nz * nj, sizeof(double));
  o->e_abs = (double*)calloc(nz, sizeof(double));
  o->e_rad = (double*)calloc(nz, sizeof(double));
  o->fx = (double*)calloc(nz, sizeof(double));
  o->fy = (double*)calloc(nz, sizeof(double));
  o->fz = (double*)calloc(nz, sizeof(double));
  o->fr = (double*)calloc(nz, sizeof(double));
  o->abs = (double*)calloc(nz * nn, sizeof(double));
  o->scat = (double*)calloc(nz * nn, sizeof(double));
  o->cdf = (double*)calloc(nz * nn, sizeof(double));
  o->eps_imc = (double*)calloc(nz, sizeof(double));
  o->n_elec = (double*)calloc(nz, sizeof(double));
  o->planck = (double*)calloc(nz, sizeof(double));
  o->ross = (double*)calloc(nz, sizeof(double));
  o->L_th = (double*)calloc(nz, sizeof(double));
  o->have_grid = 1;
  o->have_opacity = 0;
  return SED_OK;
}

int oracle_set_opacity_params(oracle_ctx* o, const sed_opacity_params* op)
{
  if (!o || !op) return SED_ERR_ARG;
  o->op = *op;
  free(o->zero_eps);
  o->zero_eps = dup_i(op->atom_zero_epsilon, (size_t)op->n_atom_zero_epsilon);
  o->op.atom_zero_epsilon = o->zero_eps;
  return SED_OK;
}

int oracle_set_atomic_data(oracle_ctx* o, const sed_atomic_data* a)
{
  if (!o || !a || a->n_atoms < 0) return SED_ERR_ARG;
  int na = a->n_atoms;
  o->natoms = na;
  o->ion_off = dup_i(a->ion_off, (size_t)na + 1);
  o->lev_off = dup_i(a->lev_off, (size_t)na + 1);
  o->line_off = dup_i(a->line_off, (size_t)na + 1);
  o->fuzz_off = dup_i(a->fuzz_off, (size_t)na + 1);
  size_t ni = (size_t)o->ion_off[na], nl = (size_t)o->lev_off[na];
  size_t nli = (size_t)o->line_off[na], nf = (size_t)o->fuzz_off[na];
  o->ion_chi = dup_d(a->ion_chi, ni, 0.0);
  o->lev_ion = dup_i(a->lev_ion, nl);
  o->lev_g = dup_i(a->lev_g, nl);
  o->lev_ic = dup_i(a->lev_ic, nl);
  o->lev_E = dup_d(a->lev_E, nl, 0.0);
  o->lev_Eion = dup_d(a->lev_Eion, nl, 0.0);
  o->photo_off = dup_i(a->photo_off, nl + 1);
  size_t np = (size_t)o->photo_off[nl];
  o->photo_E = dup_d(a->photo_E, np, 0.0);
  o->photo_s = dup_d(a->photo_s, np, 0.0);
  o->line_l = dup_i(a->line_l, nli);
  o->line_u = dup_i(a->line_u, nli);
  o->line_nu = dup_d(a->line_nu, nli, 0.0);
  o->line_f = dup_d(a->line_f, nli, 0.0);
  o->line_bin = (int*)malloc(sizeof(int) * (nli ? nli : 1));
  for (size_t i = 0; i < nli; ++i) o->line_bin[i] = lg_locate_wb(&o->nu, o->line_nu[i]); /* AtomicData.cpp:680 */
  o->fuzz_nu = dup_d(a->fuzz_nu, nf, 0.0);
  o->fuzz_gf = dup_d(a->fuzz_gf, nf, 0.0);
  o->fuzz_El = dup_d(a->fuzz_El, nf, 0.0);
  o->fuzz_ion = dup_i(a->fuzz_ion, nf);
  o->fuzz_bin = (int*)malloc(sizeof(int) * (nf ? nf : 1));
  for (size_t i = 0; i < nf; ++i) o->fuzz_bin[i] = lg_locate_wb(&o->nu, o->fuzz_nu[i]); /* AtomicData.cpp:851 */
  o->have_atoms = 1;
  return SED_OK;
}

int oracle_get_fuzz_bins(oracle_ctx* o, int32_t* bins)
{
  if (!o || !o->have_atoms) return SED_ERR_STATE;
  for (int i = 0; i < o->fuzz_off[o->natoms]; ++i) bins[i] = o->fuzz_bin[i];
  return SED_OK;
}

/* ---------------------------------------------------------------- LTE gas state */
typedef struct {
  double* ion_part;  /* per atom ions */
  double* ion_frac;
  double* lev_n;
  double* n_dens;    /* per atom */
  double* mass_frac;
  double dens, temp, mu_I, n_elec, time;
  int solve_error;
} gas;

/* AtomicSpecies::solve_lte, src/opacity/AtomicSpecies_state.cpp:56-123 */
static void solve_lte(oracle_ctx* o, gas* g, int a, double ne)
{
  int i0 = o->ion_off[a], ni = o->ion_off[a + 1] - i0;
  int l0 = o->lev_off[a], nl = o->lev_off[a + 1] - l0;
  double T = g->temp;
  double* part = g->ion_part + i0;
  double* frac = g->ion_frac + i0;
  double* lev = g->lev_n + l0;
  for (int i = 0; i < ni; ++i) part[i] = 0;
  for (int i = 0; i < nl; ++i) {
    double E = o->lev_E[l0 + i];
    int gg = o->lev_g[l0 + i];
    int ion = o->lev_ion[l0 + i];
    lev[i] = gg * exp(-E / PC_K_EV / T);
    part[ion] += lev[i];
  }
  double lt = PC_H * PC_H / (2.0 * PC_PI * PC_M_E * PC_K * T);
  double fac = 2 / ne / pow(lt, 1.5);
  frac[0] = 1.;
  double norm = 1.;
  for (int i = 1; i < ni; ++i) {
    double chi = o->ion_chi[i0 + i - 1];
    double saha = exp(-1.0 * chi / PC_K_EV / T);
    saha = saha * (part[i] / part[i - 1]) * fac;
    frac[i] = saha * frac[i - 1];
    if (ne < 1e-50) frac[i] = 0;
    norm = 0;
    for (int j = 0; j <= i; j++) norm += frac[j];
    for (int j = 0; j <= i; j++) frac[j] = frac[j] / norm;
  }
  for (int i = 0; i < nl; ++i) {
    double E = o->lev_E[l0 + i];
    int gg = o->lev_g[l0 + i];
    int ion = o->lev_ion[l0 + i];
    double Z = part[ion];
    double f = frac[ion];
    lev[i] = f * gg * exp(-E / PC_K_EV / T) / Z;
    if (lev[i] < 1e-30) lev[i] = 1e-30; /* min_level_pop_, AtomicSpecies_init.cpp:36 */
  }
}

/* GasState::charge_conservation, src/opacity/GasState.cpp:242-263 */
static double charge_conservation(oracle_ctx* o, gas* g, double ne)
{
  double f = 0;
  for (int a = 0; a < o->natoms; ++a) {
    solve_lte(o, g, a, ne);
    int l0 = o->lev_off[a], nl = o->lev_off[a + 1] - l0;
    double x = 0; /* AtomicSpecies::get_net_ion_fraction, AtomicSpecies.h:125-131 */
    for (int i = 0; i < nl; ++i) x += g->lev_n[l0 + i] * o->lev_ion[l0 + i];
    f += g->dens * g->mass_frac[a] / (o->eA[a] * PC_M_P) * x;
  }
  return f - ne;
}

#define SIGN(a, b) ((b) >= 0.0 ? fabs(a) : -fabs(a))
/* GasState::ne_brent_method, src/opacity/GasState.cpp:270-337.  Also returns
 * the last electron density the charge function was evaluated at: the atoms'
 * populations the opacities use are those of that last evaluation. */
static double ne_brent(oracle_ctx* o, gas* g, double x1, double x2, double tol, double* last)
{
  int ITMAX = 100;
  double EPS = 3.0e-8;
  double a = x1, b = x2, c = x2, d = 0, e = 0, min1, min2;
  double fa = charge_conservation(o, g, a);
  double fb = charge_conservation(o, g, b);
  *last = b;
  double fc, p, q, r, s, tol1, xm;
  if ((fa > 0.0 && fb > 0.0) || (fa < 0.0 && fb < 0.0)) g->solve_error = 1;
  fc = fb;
  for (int iter = 1; iter <= ITMAX; iter++) {
    if ((fb > 0.0 && fc > 0.0) || (fb < 0.0 && fc < 0.0)) {
      c = a; fc = fa; e = d = b - a;
    }
    if (fabs(fc) < fabs(fb)) {
      a = b; b = c; c = a;
      fa = fb; fb = fc; fc = fa;
    }
    tol1 = 2.0 * EPS * fabs(b) + 0.5 * tol;
    xm = 0.5 * (c - b);
    if (fabs(xm) <= tol1 || fb == 0.0) return b;
    if (fabs(e) >= tol1 && fabs(fa) > fabs(fb)) {
      s = fb / fa;
      if (a == c) {
        p = 2.0 * xm * s;
        q = 1.0 - s;
      } else {
        q = fa / fc;
        r = fb / fc;
        p = s * (2.0 * xm * q * (q - r) - (b - a) * (r - 1.0));
        q = (q - 1.0) * (r - 1.0) * (s - 1.0);
      }
      if (p > 0.0) q = -q;
      p = fabs(p);
      min1 = 3.0 * xm * q - fabs(tol1 * q);
      min2 = fabs(e * q);
      if (2.0 * p < (min1 < min2 ? min1 : min2)) {
        e = d;
        d = p / q;
      } else {
        d = xm;
        e = d;
      }
    } else {
      d = xm;
      e = d;
    }
    a = b;
    fa = fb;
    if (fabs(d) > tol1) b += d;
    else b += SIGN(tol1, xm);
    fb = charge_conservation(o, g, b);
    *last = b;
  }
  g->solve_error = 2;
  return 0.0;
}

/* AtomicSpecies::ionization_fraction, AtomicSpecies.h:118-123 (stage == index) */
static double ion_fraction(oracle_ctx* o, gas* g, int a, int stage)
{
  int i0 = o->ion_off[a], ni = o->ion_off[a + 1] - i0;
  if (stage < 0 || stage >= ni) return 0;
  return g->ion_frac[i0 + stage];
}

/* xy_array::value_at_with_zero_edges, src/utils/xy_array.cpp:42-104 */
static double photo_cs(oracle_ctx* o, int lev, double z)
{
  int p0 = o->photo_off[lev], n = o->photo_off[lev + 1] - p0;
  const double* x = o->photo_E + p0;
  const double* y = o->photo_s + p0;
  if (n <= 0) return 0;
  if (z < x[0]) return 0;
  if (z > x[n - 1]) return 0;
  int ind;
  if (n == 1) ind = 0;
  else if (z >= x[n - 1]) ind = n;
  else if (z <= x[0]) ind = 0;
  else {
    int bl = 0, bu = n - 1;
    while (bu - bl > 1) { int bm = (bu + bl) / 2; if (x[bm] <= z) bl = bm; else bu = bm; }
    ind = bl;
  }
  if (n == 1) return y[0];
  int i1, i2;
  if (ind < n - 1) { i1 = ind; i2 = ind + 1; }
  else { i2 = ind < n ? ind : n - 1; i1 = i2 - 1; } /* ind == n only at z == x[n-1] exactly */
  double slope = (y[i2] - y[i1]) / (x[i2] - x[i1]);
  return y[ind < n ? ind : n - 1] + slope * (z - x[i1]);
}

/* transport::set_opacity, src/transport/transport_opacity.cpp:21-260, for one
 * zone: GasState::solve_state (GasState.cpp:208-233) + computeOpacity
 * (GasState_opacities.cpp:11-136) + the emissivity CDF, cap and means. */
static void zone_opacity(oracle_ctx* o, int iz, double dt, gas* g, double* opac, double* aopac, double* emis,
                         double* tmp_o, double* tmp_e)
{
  int nn = o->nu.n;
  double* ab = o->abs + (size_t)iz * nn;
  double* sc = o->scat + (size_t)iz * nn;
  double* cdf = o->cdf + (size_t)iz * nn;
  g->dens = o->rho[iz];
  g->temp = o->T[iz];
  if (g->temp < o->op.temp_min) g->temp = o->op.temp_min;
  if (g->temp > o->op.temp_max) g->temp = o->op.temp_max;
  /* GasState::set_mass_fractions, GasState.cpp:137-156 */
  double norm = 0.0;
  for (int a = 0; a < o->nelem; ++a) { g->mass_frac[a] = o->X[(size_t)iz * o->nelem + a]; norm += g->mass_frac[a]; }
  for (int a = 0; a < o->nelem; ++a) g->mass_frac[a] /= norm;
  double inv = 0.;
  for (int a = 0; a < o->nelem; ++a) inv += g->mass_frac[a] / o->eA[a];
  g->mu_I = 1. / inv;
  double grey = o->grey[iz];
  double temp = g->temp;
  for (int i = 0; i < nn; ++i) { ab[i] = 0; sc[i] = 0; emis[i] = 0; }

  if (grey != 0) {
    /* grey branch, GasState_opacities.cpp:29-41 */
    double gopac = g->dens * grey;
    for (int i = 0; i < nn; ++i) {
      ab[i] = gopac * o->op.epsilon;
      sc[i] = gopac * (1 - o->op.epsilon);
      double nu = lg_center(&o->nu, i);
      double ezeta = exp(1.0 * PC_H * nu / PC_K / temp);
      double bb = 2.0 * nu * nu * nu * PC_H / PC_C / PC_C / (ezeta - 1);
      emis[i] += bb * ab[i];
    }
  } else {
    if (!o->have_atoms) return;
    /* GasState::solve_state (LTE) */
    for (int a = 0; a < o->natoms; ++a) g->n_dens[a] = g->dens * g->mass_frac[a] / (o->eA[a] * PC_M_P);
    double max_ne = 100 * g->dens / (g->mu_I * PC_M_P);
    double min_ne = 1e-10 * g->dens / (g->mu_I * PC_M_P);
    g->solve_error = 0;
    double last = 0;
    g->n_elec = ne_brent(o, g, min_ne, max_ne, 1e-3, &last);
    for (int a = 0; a < o->natoms; ++a) solve_lte(o, g, a, last);
    o->n_elec[iz] = g->n_elec;
    double ne = g->n_elec;

    if (o->op.use_electron_scattering) { /* :49-58 */
      double es = PC_THOMSON * ne;
      for (int i = 0; i < nn; ++i) { sc[i] += es; ab[i] += 1e-20 * o->op.epsilon * es; }
    }
    if (o->op.use_free_free) { /* GasState::free_free_opacity, :152-183 */
      double fac = 0;
      for (int a = 0; a < o->natoms; ++a) {
        int ni = o->ion_off[a + 1] - o->ion_off[a];
        double zsq = 0;
        for (int j = 0; j < ni; j++) zsq += ion_fraction(o, g, a, j) * j * j;
        double n_ion = g->mass_frac[a] * g->dens / (o->eA[a] * PC_M_P);
        fac += n_ion * zsq;
      }
      fac *= 3.7e8 * pow(temp, -0.5) * ne;
      for (int i = 0; i < nn; ++i) {
        double nu = lg_center(&o->nu, i);
        double ezeta = exp(-1.0 * PC_H * nu / PC_K / temp);
        double bb = 2.0 * nu * nu * nu * PC_H / PC_C / PC_C / (1.0 / ezeta - 1);
        double op_ = fac / nu / nu / nu * (1 - ezeta);
        ab[i] += op_;
        emis[i] += op_ * bb;
      }
    }
    if (o->op.use_bound_free) { /* GasState::bound_free_opacity :352-371 + AtomicSpecies_opacities.cpp:58-151 */
      for (int i = 0; i < nn; ++i) { tmp_o[i] = 0; tmp_e[i] = 0; }
      double kt_ev = PC_K_EV * temp;
      double lam_t = sqrt(PC_H * PC_H / (2 * PC_PI * PC_M_E * PC_K * temp));
      for (int a = 0; a < o->natoms; ++a) {
        int l0 = o->lev_off[a], nl = o->lev_off[a + 1] - l0;
        double nd = g->n_dens[a];
        double* ncp = (double*)calloc((size_t)(nl ? nl : 1), sizeof(double));
        for (int j = 0; j < nl; ++j) {
          int ic = o->lev_ic[l0 + j];
          if (ic == -1) continue;
          double nc = nd * g->lev_n[l0 + ic];
          int gl = o->lev_g[l0 + j], gc = o->lev_g[l0 + ic];
          double gl_o_gc = (1.0 * gl) / (1.0 * gc);
          ncp[j] = nc * gl_o_gc / 2. * lam_t * lam_t * lam_t;
        }
        for (int i = 0; i < nn; ++i) {
          double nu = lg_center(&o->nu, i);
          double E = PC_H * nu * PC_ERGS_TO_EV;
          double emis_fac = 2. * PC_H * nu * nu * nu / PC_C / PC_C;
          double ao = 0, ae = 0;
          for (int j = 0; j < nl; ++j) {
            double Eion = o->lev_Eion[l0 + j];
            int ic = o->lev_ic[l0 + j];
            if (ic == -1) continue;
            if (E < Eion) continue;
            double zeta_net = (Eion - E) / kt_ev;
            double ezeta_net = exp(zeta_net);
            double sigma = photo_cs(o, l0 + j, E);
            double opac_fac = nd * g->lev_n[l0 + j] - ncp[j] * ne * ezeta_net;
            if (opac_fac < 0) opac_fac = 0.;
            ao += sigma * opac_fac;
            ae += emis_fac * sigma * ncp[j] * ezeta_net;
          }
          tmp_o[i] += ao;
          tmp_e[i] += ae;
        }
        free(ncp);
      }
      for (int i = 0; i < nn; ++i) { ab[i] += tmp_o[i]; emis[i] += tmp_e[i] * ne; }
    }
    if (o->op.use_line_expansion) { /* GasState::line_expansion_opacity :424-454 + AtomicSpecies_opacities.cpp:331-375 */
      for (int i = 0; i < nn; ++i) { opac[i] = 0; aopac[i] = 0; }
      for (int a = 0; a < o->natoms; ++a) {
        double this_eps = o->op.epsilon;
        for (int k = 0; k < o->op.n_atom_zero_epsilon; k++) if (o->zero_eps[k] == o->eZ[a]) this_eps = 0;
        for (int i = 0; i < nn; ++i) tmp_o[i] = 0;
        int l0 = o->lev_off[a];
        for (int k = o->line_off[a]; k < o->line_off[a + 1]; ++k) {
          int ll = o->line_l[k], lu = o->line_u[k];
          double nl = g->lev_n[l0 + ll], nup = g->lev_n[l0 + lu];
          double gl = 1.0 * o->lev_g[l0 + ll], gu = 1.0 * o->lev_g[l0 + lu];
          if (nl < DBL_MIN) continue;
          double nu0 = o->line_nu[k];
          double lam = PC_C / nu0;
          double tau = nl * g->n_dens[a] * PC_SIGMA_TOT * o->line_f[k] * g->time * lam;
          tau = tau * (1 - nup * gl / (nl * gu));
          if (nup * gl > nl * gu) tau = 0;
          double etau = exp(-tau);
          if (!isnan(etau)) tmp_o[o->line_bin[k]] += (1 - etau);
        }
        for (int i = 0; i < nn; ++i) {
          tmp_o[i] = tmp_o[i] * lg_center(&o->nu, i) / lg_delta(&o->nu, i) / PC_C / g->time;
          opac[i] += tmp_o[i];
          aopac[i] += tmp_o[i] * this_eps;
        }
      }
      for (int i = 0; i < nn; ++i) {
        ab[i] += aopac[i];
        sc[i] += opac[i] - aopac[i];
        double nu = lg_center(&o->nu, i);
        double ezeta = exp(1.0 * PC_H * nu / PC_K / temp);
        double bb = 2.0 * nu * nu * nu * PC_H / PC_C / PC_C / (ezeta - 1);
        emis[i] += bb * aopac[i];
      }
    }
    if (o->op.use_fuzz_expansion) { /* GasState::fuzz_expansion_opacity :464-494 + AtomicSpecies_opacities.cpp:292-324 */
      for (int i = 0; i < nn; ++i) { opac[i] = 0; aopac[i] = 0; }
      for (int a = 0; a < o->natoms; ++a) {
        double this_eps = o->op.epsilon;
        for (int k = 0; k < o->op.n_atom_zero_epsilon; k++) if (o->zero_eps[k] == o->eZ[a]) this_eps = 0;
        for (int i = 0; i < nn; ++i) tmp_o[i] = 0;
        int i0 = o->ion_off[a];
        for (int k = o->fuzz_off[a]; k < o->fuzz_off[a + 1]; ++k) {
          double nu = o->fuzz_nu[k], gf = o->fuzz_gf[k], El = o->fuzz_El[k];
          int ion = o->fuzz_ion[k];
          double nion = g->n_dens[a] * g->ion_frac[i0 + ion];
          double nl = nion * exp(-1.0 * El / PC_K_EV / temp) / g->ion_part[i0 + ion];
          double lam = PC_C / nu;
          double stim_cor = (1 - exp(-PC_H * nu / PC_K / temp));
          double tau = PC_SIGMA_TOT * lam * nl * gf * stim_cor * g->time;
          double etau = exp(-tau);
          tmp_o[o->fuzz_bin[k]] += (1 - etau);
        }
        for (int i = 0; i < nn; ++i) {
          tmp_o[i] = tmp_o[i] * lg_center(&o->nu, i) / lg_delta(&o->nu, i) / PC_C / g->time;
          opac[i] += tmp_o[i];
          aopac[i] += tmp_o[i] * this_eps;
        }
      }
      for (int i = 0; i < nn; ++i) {
        ab[i] += aopac[i];
        sc[i] += opac[i] - aopac[i];
        double nu = lg_center(&o->nu, i);
        double ezeta = exp(1.0 * PC_H * nu / PC_K / temp);
        double bb = 2.0 * nu * nu * nu * PC_H / PC_C / PC_C / (ezeta - 1);
        emis[i] += bb * aopac[i];
      }
    }
  }

  /* emissivity CDF, L_thermal and the opacity cap, transport_opacity.cpp:152-179 */
  double max_ext = o->op.maximum_opacity * o->rho[iz];
  double L = 0;
  if (nn == 1) {
    double bb_int = PC_SB * pow(o->T[iz], 4) / PC_PI;
    L += 4 * PC_PI * ab[0] * bb_int;
    cdf[0] = 1;
    if (o->tp.omit_scattering) sc[0] = 0;
  } else {
    for (int j = 0; j < nn; ++j) {
      double ednu = emis[j] * lg_delta(&o->nu, j);
      cdf[j] = (j == 0) ? ednu : cdf[j - 1] + ednu;
      L += 4 * PC_PI * ednu;
      if (o->tp.omit_scattering) sc[j] = 0;
      if (!o->tp.omit_scattering) { if (sc[j] > max_ext) sc[j] = max_ext; }
      if (ab[j] > max_ext) ab[j] = max_ext;
    }
  }
  o->L_th[iz] = L;
  cdf_normalize(cdf, nn);
  /* GasState::get_planck_mean / get_rosseland_mean, GasState_opacities.cpp:564-666 */
  if (nn == 1) {
    o->planck[iz] = ab[0];
    o->ross[iz] = ab[0] + sc[0];
  } else {
    double mean = 0, norm2 = 0, rmean = 0, rnorm = 0;
    for (int i = 0; i < nn; ++i) {
      double nu = lg_center(&o->nu, i);
      double zeta = PC_H * nu / PC_K / temp;
      double Bnu = 2.0 * nu * nu * nu * PC_H / PC_C / PC_C / (exp(zeta) - 1);
      if (isnan(Bnu)) Bnu = 0;
      double W = Bnu * lg_delta(&o->nu, i);
      mean += W * (ab[i]);
      norm2 += W;
      double ezeta = exp(zeta);
      double dBdT = pow(nu, 4) * ezeta / (ezeta - 1) / (ezeta - 1);
      if (isnan(dBdT)) dBdT = 0;
      double Wr = dBdT * lg_delta(&o->nu, i);
      rmean += Wr / (ab[i] + sc[i]);
      rnorm += Wr;
    }
    o->planck[iz] = mean / norm2;
    o->ross[iz] = rnorm / rmean;
  }
  /* eps_imc, transport_opacity.cpp:231-252 */
  if (o->tp.radiative_eq) o->eps_imc[iz] = 1.;
  else {
    double fleck_beta = 4.0 * PC_A * pow(o->T[iz], 4) / (o->e_gas[iz] * o->rho[iz]);
    double tfac = PC_C * o->planck[iz] * dt;
    double f_imc = o->tp.fleck_alpha * fleck_beta * tfac;
    if (o->tp.fleck_alpha == 0) f_imc = 0.;
    o->eps_imc[iz] = 1.0 / (1.0 + f_imc);
  }
}

int oracle_set_opacity(oracle_ctx* o, double dt)
{
  if (!o || !o->have_grid) return SED_ERR_STATE;
  if (o->tp.steady_state) dt = 1;
  int nn = o->nu.n;
  size_t ni = o->have_atoms ? (size_t)o->ion_off[o->natoms] : 1;
  size_t nl = o->have_atoms ? (size_t)o->lev_off[o->natoms] : 1;
  gas g;
  memset(&g, 0, sizeof g);
  g.ion_part = (double*)calloc(ni ? ni : 1, sizeof(double));
  g.ion_frac = (double*)calloc(ni ? ni : 1, sizeof(double));
  g.lev_n = (double*)calloc(nl ? nl : 1, sizeof(double));
  g.n_dens = (double*)calloc((size_t)(o->nelem > 0 ? o->nelem : 1), sizeof(double));
  g.mass_frac = (double*)calloc((size_t)(o->nelem > 0 ? o->nelem : 1), sizeof(double));
  g.time = o->t_now;
  double* opac = (double*)calloc((size_t)nn, sizeof(double));
  double* aopac = (double*)calloc((size_t)nn, sizeof(double));
  double* emis = (double*)calloc((size_t)nn, sizeof(double));
  double* t1 = (double*)calloc((size_t)nn, sizeof(double));
  double* t2 = (double*)calloc((size_t)nn, sizeof(double));
  for (int iz = 0; iz < o->nzones; ++iz) zone_opacity(o, iz, dt, &g, opac, aopac, emis, t1, t2);
  free(opac); free(aopac); free(emis); free(t1); free(t2);
  free(g.ion_part); free(g.ion_frac); free(g.lev_n); free(g.n_dens); free(g.mass_frac);
  o->have_opacity = 1;
  o->base_valid = 0;
  return SED_OK;
}

int oracle_load_opacity(oracle_ctx* o, const double* abs, const double* scat, const double* emis_cdf, const double* eps_imc)
{
  if (!o || !o->have_grid || !abs || !emis_cdf || !eps_imc) return SED_ERR_ARG;
  size_t n = (size_t)o->nzones * o->nu.n;
  for (size_t i = 0; i < n; ++i) {
    o->abs[i] = abs[i];
    o->scat[i] = scat ? scat[i] : 0.0;
    o->cdf[i] = emis_cdf[i];
  }
  for (int i = 0; i < o->nzones; ++i) o->eps_imc[i] = eps_imc[i];
  o->have_opacity = 1;
  o->base_valid = 0;
  return SED_OK;
}

/* sed_diff_scale_extinction: both extinctions of zone z of the built tables
 * times r[z]; r NULL puts the built tables back (no reference counterpart) */
int oracle_diff_scale_extinction(oracle_ctx* o, const double* r)
{
  if (!o || !o->have_opacity) return SED_ERR_STATE;
  size_t nn = (size_t)o->nu.n, n = (size_t)o->nzones * nn;
  if (!o->base_valid) {
    free(o->abs_base); free(o->scat_base);
    o->abs_base = (double*)malloc(n * sizeof(double));
    o->scat_base = (double*)malloc(n * sizeof(double));
    memcpy(o->abs_base, o->abs, n * sizeof(double));
    memcpy(o->scat_base, o->scat, n * sizeof(double));
    o->base_valid = 1;
  }
  for (size_t i = 0; i < n; ++i) {
    double f = r ? r[i / nn] : 1.0;
    o->abs[i] = r ? o->abs_base[i] * f : o->abs_base[i];
    o->scat[i] = r ? o->scat_base[i] * f : o->scat_base[i];
  }
  return SED_OK;
}

/* ---------------------------------------------------------------- geometry */
/* grid_1D_sphere::get_zone, src/grid/grid_1D_sphere.cpp:494-505;
 * grid_3D_cart::get_zone, src/grid/grid_3D_cart.cpp:363-390 */
static int get_zone(const oracle_ctx* o, const double* x)
{
  if (o->gtype == SED_GRID_1D_SPHERE) {
    double r = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
    if (r < o->r_out.min) return -1;
    if (r >= o->r_out.x[o->r_out.n - 1]) return -2;
    return lg_locate_wb(&o->r_out, r);
  }
  for (int a = 0; a < 3; ++a) {
    if (x[a] < o->ax[a].min) return -2;
    if (x[a] > o->ax[a].x[o->ax[a].n - 1]) return -2;
  }
  int i = lg_locate_wb(&o->ax[0], x[0]);
  int j = lg_locate_wb(&o->ax[1], x[1]);
  int k = lg_locate_wb(&o->ax[2], x[2]);
  return i * o->ny * o->nz + j * o->nz + k;
}

/* grid_1D_sphere::get_next_zone, grid_1D_sphere.cpp:510-590;
 * grid_3D_cart::get_next_zone, grid_3D_cart.cpp:396-469 */
static int get_next_zone(const oracle_ctx* o, const double* x, const double* D, int i, double r_core, double* l)
{
  if (o->gtype == SED_GRID_1D_SPHERE) {
    double rsq = (x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
    double xdotD = (D[0] * x[0] + D[1] * x[1] + D[2] * x[2]);
    double r_o = o->r_out.x[i];
    double l_out = -1 * xdotD + sqrt(xdotD * xdotD + r_o * r_o - rsq);
    double r_in;
    int ind_in;
    if (i != 0) { r_in = o->r_out.x[i - 1]; ind_in = i - 1; }
    else { r_in = o->r_out.min; ind_in = -1; }
    if (r_core >= r_in) { r_in = r_core; ind_in = -1; }
    double l_in;
    if ((i == 0) && (r_in == 0)) l_in = -1;
    else {
      double rad = xdotD * xdotD + r_in * r_in - rsq;
      if (rad < 0) l_in = -1;
      else l_in = -1 * xdotD - sqrt(rad);
    }
    int ind;
    double tiny_offset = 1 + 1e-6;
    if ((l_out < l_in) || (l_in < 0)) {
      ind = i + 1;
      if (ind == o->nzones) { ind = -2; *l = l_out / tiny_offset; }
      else *l = l_out * tiny_offset;
    } else {
      ind = ind_in;
      if (ind_in == -1) *l = l_in / tiny_offset;
      else *l = l_in * tiny_offset;
    }
    return ind;
  }
  int nyz = o->ny * o->nz;
  int ix = i / nyz, iy = (i / o->nz) % o->ny, iz = i % o->nz;
  int idx3[3] = {ix, iy, iz};
  double tiny = 1e-10;
  double len[3];
  for (int a = 0; a < 3; ++a) {
    const lgrid* g = &o->ax[a];
    double dd = lg_delta(g, idx3[a]);
    double bn = (D[a] > 0) ? g->x[idx3[a]] + dd * tiny : lg_left(g, idx3[a]) - dd * tiny;
    len[a] = (bn - x[a]) / D[a];
  }
  int idx = 0, idy = 0, idz = 0;
  if ((len[0] < len[1]) && (len[0] < len[2])) { idx = (D[0] < 0) ? -1 : 1; *l = len[0]; }
  else if (len[1] < len[2]) { idy = (D[1] < 0) ? -1 : 1; *l = len[1]; }
  else { idz = (D[2] < 0) ? -1 : 1; *l = len[2]; }
  int nx_ = ix + idx, ny_ = iy + idy, nz_ = iz + idz;
  if (nx_ < 0 || nx_ > o->nx - 1) return -2;
  if (ny_ < 0 || ny_ > o->ny - 1) return -2;
  if (nz_ < 0 || nz_ > o->nz - 1) return -2;
  return nx_ * nyz + ny_ * o->nz + nz_;
}

/* get_velocity, grid_1D_sphere.cpp:707-748 / grid_3D_cart.cpp:513-521 (homologous) */
static void get_velocity(const oracle_ctx* o, int i, const double* x, const double* D, double* v, double* dvds)
{
  if (o->homologous) {
    v[0] = x[0] / o->t_grid;
    v[1] = x[1] / o->t_grid;
    v[2] = x[2] / o->t_grid;
    *dvds = 1.0 / o->t_grid;
    return;
  }
  if (o->gtype == SED_GRID_1D_SPHERE) {
    /* a diffusion leak past the outer wall leaves the index one past the
     * grid; the last zone's velocity field is used there */
    if (i >= o->nzones) i = o->nzones - 1;
    double rr = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
    double v_0, r_0;
    if (i == 0) { v_0 = 0; r_0 = o->r_out.min; }
    else { v_0 = o->v_r[i - 1]; r_0 = o->r_out.x[i - 1]; }
    double dr = rr - r_0;
    double dv_dr = (o->v_r[i] - v_0) / (o->r_out.x[i] - r_0);
    double vv = v_0 + dv_dr * dr;
    double D_dot_rhat = (D[0] * x[0] + D[1] * x[1] + D[2] * x[2]) / rr;
    v[0] = x[0] / rr * vv;
    v[1] = x[1] / rr * vv;
    v[2] = x[2] / rr * vv;
    *dvds = D_dot_rhat * D_dot_rhat * (dv_dr - vv / rr) + vv / rr;
    if (rr == 0) { v[0] = v[1] = v[2] = 0; *dvds = dv_dr; }
    return;
  }
  v[0] = v[1] = v[2] = 0; /* non-homologous 3D velocities are not on this path */
  *dvds = 0;
}

/* transport::do_dshift, src/transport/relativity.cpp:14-43 (lab -> comoving) */
static double dshift_lab_to_comoving(const oracle_ctx* o, packet* p)
{
  double v[3], dvds;
  get_velocity(o, p->ind, p->x, p->D, v, &dvds);
  double beta2 = (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) / PC_C / PC_C;
  double vdd = v[0] * p->D[0] + v[1] * p->D[1] + v[2] * p->D[2];
  double gamma = 1.0 / sqrt(1 - beta2);
  double dshift = gamma * (1 - vdd / PC_C);
  p->dvds = dvds;
  return dshift;
}

/* transport::lorentz_transform(p, tolab=1), relativity.cpp:84-127 */
static void transform_comoving_to_lab(const oracle_ctx* o, packet* p)
{
  double v[3], dvds;
  get_velocity(o, p->ind, p->x, p->D, v, &dvds);
  v[0] *= -1; v[1] *= -1; v[2] *= -1;
  double beta2 = (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) / PC_C / PC_C;
  double vdd = v[0] * p->D[0] + v[1] * p->D[1] + v[2] * p->D[2];
  double gamma = 1.0 / sqrt(1 - beta2);
  double dshift = gamma * (1 - vdd / PC_C);
  p->dvds = dvds;
  p->e *= dshift;
  p->nu *= dshift;
  p->D[0] = 1.0 / dshift * (p->D[0] - gamma * v[0] / PC_C * (1 - gamma * vdd / PC_C / (gamma + 1)));
  p->D[1] = 1.0 / dshift * (p->D[1] - gamma * v[1] / PC_C * (1 - gamma * vdd / PC_C / (gamma + 1)));
  p->D[2] = 1.0 / dshift * (p->D[2] - gamma * v[2] / PC_C * (1 - gamma * vdd / PC_C / (gamma + 1)));
  double norm = p->D[0] * p->D[0] + p->D[1] * p->D[1] + p->D[2] * p->D[2];
  p->D[0] /= norm;
  p->D[1] /= norm;
  p->D[2] /= norm;
}

static double draw(const oracle_ctx* o, packet* p)
{
  return oracle_packet_uniform(o->tp.rng_seed, p->pid, o->step, p->n++);
}

/* transport::isotropic_scatter, src/transport/scatter.cpp:303-351 */
static void isotropic_scatter(const oracle_ctx* o, packet* p, int redist)
{
  double V[3], dvds;
  get_velocity(o, p->ind, p->x, p->D, V, &dvds);
  double vdotD = V[0] * p->D[0] + V[1] * p->D[1] + V[2] * p->D[2];
  double beta2 = (V[0] * V[0] + V[1] * V[1] + V[2] * V[2]) / PC_C / PC_C;
  double gamma = 1.0 / sqrt(1 - beta2);
  double dshift_in = gamma * (1 - vdotD / PC_C);
  p->e = p->e * dshift_in;
  p->nu = p->nu * dshift_in;
  double mu = 1 - 2.0 * draw(o, p);
  double phi = 2.0 * PC_PI * draw(o, p);
  double smu = sqrt(1 - mu * mu);
  double Dn[3] = {smu * cos(phi), smu * sin(phi), mu};
  if (redist) { /* sample_photon_frequency, emission.cpp:27-46 */
    int nn = o->nu.n;
    int inu = cdf_sample(o->cdf + (size_t)p->ind * nn, nn, draw(o, p));
    p->nu = lg_sample(&o->nu, inu, draw(o, p));
  }
  for (int i = 0; i < 3; i++) V[i] = -1 * V[i];
  double vdp = (Dn[0] * V[0] + Dn[1] * V[1] + Dn[2] * V[2]);
  double vd_out = gamma * (1 - vdp / PC_C);
  p->D[0] = 1.0 / vd_out * (Dn[0] - gamma * V[0] / PC_C * (1 - gamma * vdp / PC_C / (gamma + 1)));
  p->D[1] = 1.0 / vd_out * (Dn[1] - gamma * V[1] / PC_C * (1 - gamma * vdp / PC_C / (gamma + 1)));
  p->D[2] = 1.0 / vd_out * (Dn[2] - gamma * V[2] / PC_C * (1 - gamma * vdp / PC_C / (gamma + 1)));
  double norm = sqrt(p->D[0] * p->D[0] + p->D[1] * p->D[1] + p->D[2] * p->D[2]);
  p->D[0] = p->D[0] / norm;
  p->D[1] = p->D[1] / norm;
  p->D[2] = p->D[2] / norm;
  p->e = p->e * vd_out;
  p->nu = p->nu * vd_out;
}

/* transport::emit_inner_source, src/transport/emission.cpp:370-485 (one packet) */
static void emit_core_packet(const oracle_ctx* o, packet* p, double Ep, double t_now, double dt)
{
  double rc = o->tp.core_radius;
  if (rc == 0) {
    p->x[0] = p->x[1] = p->x[2] = 0;
    double mu = 1 - 2.0 * draw(o, p);
    double phi = 2.0 * PC_PI * draw(o, p);
    double smu = sqrt(1 - mu * mu);
    p->D[0] = smu * cos(phi);
    p->D[1] = smu * sin(phi);
    p->D[2] = mu;
  } else {
    double phi_core = 2 * PC_PI * draw(o, p);
    double cosp_core = cos(phi_core);
    double sinp_core = sin(phi_core);
    double cost_core = 1 - 2.0 * draw(o, p);
    double sint_core = sqrt(1 - cost_core * cost_core);
    double a_phot = rc + rc * 1e-10;
    p->x[0] = a_phot * sint_core * cosp_core;
    p->x[1] = a_phot * sint_core * sinp_core;
    p->x[2] = a_phot * cost_core;
    double phi_loc = 2 * PC_PI * draw(o, p);
    double cost_loc = sqrt(draw(o, p));
    double sint_loc = sqrt(1 - cost_loc * cost_loc);
    double D_xl = sint_loc * cos(phi_loc);
    double D_yl = sint_loc * sin(phi_loc);
    double D_zl = cost_loc;
    p->D[0] = cost_core * cosp_core * D_xl - sinp_core * D_yl + sint_core * cosp_core * D_zl;
    p->D[1] = cost_core * sinp_core * D_xl + cosp_core * D_yl + sint_core * sinp_core * D_zl;
    p->D[2] = -sint_core * D_xl + cost_core * D_zl;
  }
  p->e = Ep;
  if (o->tp.core_photon_frequency > 0) p->nu = o->tp.core_photon_frequency;
  else {
    int inu = cdf_sample(o->core_cdf, o->nu.n, draw(o, p));
    p->nu = lg_sample(&o->nu, inu, draw(o, p));
    p->e /= 1.0;  /* emissivity_weight_[inu] */
  }
  p->ind = get_zone(o, p->x);
  transform_comoving_to_lab(o, p);
  p->t = t_now + draw(o, p) * dt;
}

/* spectrum_array::count, src/transport/spectrum_array.cpp:215-246, on the
 * frequency grid `sn` into flux/click; returns the index, -1 when dropped */
static int64_t spectrum_count_on(oracle_ctx* o, const lgrid* sn, double* flux, double* click, double t, double w,
                                 double E, const double* D);
static int64_t spectrum_count(oracle_ctx* o, double t, double w, double E, const double* D)
{
  return spectrum_count_on(o, &o->sn, o->flux, o->click, t, w, E, D);
}
static int64_t spectrum_count_on(oracle_ctx* o, const lgrid* sn, double* flux, double* click, double t, double w,
                                 double E, const double* D)
{
  double mu = D[2];
  double phi = atan2(D[1], D[0]);
  if (phi < 0) phi += 2. * PC_PI;
  int t_bin = lg_locate(&o->st, t);
  int l_bin = lg_locate(sn, w);
  int m_bin = lg_locate(&o->sm, mu);
  int p_bin = lg_locate(&o->sp, phi);
  if (l_bin < 0) l_bin = 0;
  if (l_bin >= sn->n) l_bin = 0;
  if ((t_bin < 0) || (l_bin < 0) || (m_bin < 0) || (p_bin < 0)) return -1;
  if (t_bin >= o->st.n) return -1;
  if (m_bin >= o->sm.n) return -1;
  if (p_bin >= o->sp.n) return -1;
  int64_t a3 = o->sp.n, a2 = (int64_t)o->sm.n * a3, a1 = (int64_t)sn->n * a2;
  int64_t ind = t_bin * a1 + l_bin * a2 + m_bin * a3 + p_bin;
  flux[ind] += E;
  click[ind] += 1;
  return ind;
}

/* transport::propagate + propagate_monte_carlo, src/transport/transport.cpp:202-484;
 * relocate = 0 continues a packet whose zone is current (a gamma-ray that
 * became an optical photon inside propagate_monte_carlo) */
static int propagate_from(oracle_ctx* o, packet* p, double t_now, double dt, int64_t* nseg, int64_t* nscat,
                          int relocate);
static int propagate(oracle_ctx* o, packet* p, double t_now, double dt, int64_t* nseg, int64_t* nscat)
{
  return propagate_from(o, p, t_now, dt, nseg, nscat, 1);
}
/* ---------------------------------------------------------------- discrete diffusion
 * transport_use_ddmc = 2 (src/transport/discrete_diffusion.cpp:114-510), 1D
 * spheres.  A photon in a zone whose total opacity times the zone width
 * exceeds transport_ddmc_tau_threshold makes discrete diffusion events
 * (leakage to a neighbour, effective scattering, end of step) instead of
 * Monte Carlo segments; it enters such a zone through
 * move_across_DDMC_interface. */
static void lorentz(const oracle_ctx* o, packet* p, int tolab);
static void sample_in_zone(const oracle_ctx* o, int i, double u0, double u1, double u2, double* r);
static double zone_size(const oracle_ctx* o, int i) { return lg_delta(&o->r_out, i); }  /* grid_1D_sphere.h:65-68 */

static int opacity_of(const oracle_ctx* o, int iz, double nu_cmf, double* opac, double* eps)
{
  int nn = o->nu.n;
  int i_nu = lg_locate_wb(&o->nu, nu_cmf);
  double a_opac = o->abs[(size_t)iz * nn + i_nu];
  double s_opac = o->tp.omit_scattering ? 0 : o->scat[(size_t)iz * nn + i_nu];
  *opac = a_opac + s_opac;
  *eps = (*opac == 0) ? 0 : a_opac / *opac;
  return i_nu;
}

static double pr(const packet* p) { return sqrt(p->x[0] * p->x[0] + p->x[1] * p->x[1] + p->x[2] * p->x[2]); }

/* the zone test of transport::propagate (transport.cpp:219-231) */
static int in_ddmc_zone(const oracle_ctx* o, packet* p)
{
  double dshift = dshift_lab_to_comoving(o, p);
  double sigma, eps;
  opacity_of(o, p->ind, p->nu * dshift, &sigma, &eps);
  return sigma * zone_size(o, p->ind) > o->tp.ddmc_tau;
}

/* transport::sample_dir_from_blackbody_surface (discrete_diffusion.cpp:753-794) */
static void bb_surface_dir(const oracle_ctx* o, packet* p)
{
  double mu = sqrt(draw(o, p));
  double phi = 2.0 * PC_PI * draw(o, p);
  double smu = sqrt(1.0 - mu * mu);
  double v1 = smu * cos(phi), v2 = smu * sin(phi), v3 = mu;
  double r1 = p->x[0] / pr(p), r2 = p->x[1] / pr(p), r3 = p->x[2] / pr(p);
  double costheta = r3, sintheta = sqrt(1 - costheta * costheta);
  double v1p = v1 * costheta + r1 * v3 * sintheta - r2 * (1.0 - costheta) * (-r2 * v1 + r1 * v2);
  double v2p = v2 * costheta + r2 * v3 * sintheta - r1 * (1.0 - costheta) * (-r2 * v1 + r1 * v2);
  double v3p = v3 * costheta - (r1 * v1 + r2 * v2) * sintheta;
  double norm = sqrt(v1p * v1p + v2p * v2p + v3p * v3p);
  p->D[0] = v1p / norm; p->D[1] = v2p / norm; p->D[2] = v3p / norm;
}

/* transport::move_across_DDMC_interface (discrete_diffusion.cpp:413-510):
 * returns 1 when the photon converts to the diffusive zone new_ind (left in
 * the comoving frame, as the reference leaves it) */
static int move_across(const oracle_ctx* o, packet* p, int new_ind, double sigma_i, double dr)
{
  int nz = o->nzones;
  int ip = p->ind + 1, im = p->ind - 1;
  if (ip == nz) ip = p->ind;
  if (im < 0) im = 0;
  double r_p = o->r_out.x[p->ind];
  double r_m = o->r_out.x[im];
  if (p->ind == 0) r_m = o->r_out.min;
  double r_interface = 0, r_0 = 0;
  if (new_ind == ip) { r_interface = r_p; r_0 = r_interface + 0.5 * dr; }
  else if (new_ind == im) { r_interface = r_m; r_0 = r_interface - 0.5 * dr; }
  (void)r_0;
  lorentz(o, p, 0);
  double rr = pr(p);
  double mu = (p->x[0] * p->D[0] + p->x[1] * p->D[1] + p->x[2] * p->D[2]) / rr;
  mu = fabs(mu);
  double p_convert = 4.0 * (1.0 + 1.5 * mu) / (3.0 * sigma_i * dr + 6.0 * 0.7104);
  double xi = draw(o, p);
  double u0 = draw(o, p), u1 = draw(o, p), u2 = draw(o, p);
  double push = 1.0e-8;
  if (xi <= p_convert) {
    p->ind = new_ind;
    sample_in_zone(o, p->ind, u0, u1, u2, p->x);
    return 1;
  }
  sample_in_zone(o, p->ind, u0, u1, u2, p->x);
  if (new_ind == ip) {
    double d = r_interface - pr(p);
    d *= (1.0 - push);
    p->x[0] += p->x[0] / pr(p) * d;
    p->x[1] += p->x[1] / pr(p) * d;
    p->x[2] += p->x[2] / pr(p) * d;
  } else if (new_ind == im) {
    double d = pr(p) - r_interface;
    d *= (1.0 - push);
    p->x[0] -= p->x[0] / pr(p) * d;
    p->x[1] -= p->x[1] / pr(p) * d;
    p->x[2] -= p->x[2] / pr(p) * d;
  }
  bb_surface_dir(o, p);
  double mu2 = (p->x[0] * p->D[0] + p->x[1] * p->D[1] + p->x[2] * p->D[2]) / pr(p);
  if (new_ind == ip) {
    if (mu2 > 0.0) { p->D[0] = -p->D[0]; p->D[1] = -p->D[1]; p->D[2] = -p->D[2]; }
  } else if (new_ind == im) {
    if (mu2 < 0.0) { p->D[0] = -p->D[0]; p->D[1] = -p->D[1]; p->D[2] = -p->D[2]; }
  }
  lorentz(o, p, 1);
  return 0;
}

/* ---------------------------------------------------------------- IMD
 * transport_use_ddmc = 1: Implicit Monte Carlo Diffusion (Gentile 2001) as
 * the reference has it, 1D spheres.  The Monte Carlo side (the diffusive-
 * zone test of every pass, the interface into a diffusive zone) is the
 * DDMC one; inside a diffusive zone a photon makes one IMD call. */

/* transport::compute_diffusion_probabilities (discrete_diffusion.cpp:
 * 687-756): hop up / down probabilities from the Planck-mean diffusion
 * coefficients of the zone and its neighbours, normalised together with the
 * (zero) advection and absorption probabilities; the rest is "stay" */
static void imd_probabilities(oracle_ctx* o, double dt)
{
  int nz = o->nzones;
  double* arr[4] = {o->imd_up, o->imd_dn, o->imd_stay, o->imd_abs};
  for (int k = 0; k < 4; k++) free(arr[k]);
  o->imd_up = (double*)calloc((size_t)nz, sizeof(double));
  o->imd_dn = (double*)calloc((size_t)nz, sizeof(double));
  o->imd_stay = (double*)calloc((size_t)nz, sizeof(double));
  o->imd_abs = (double*)calloc((size_t)nz, sizeof(double));
  for (int i = 0; i < nz; i++) {
    double dx = zone_size(o, i);
    int ip = i + 1;
    if (ip == nz) ip = i;
    int im = i - 1;
    if (im < 0) im = 0;
    double Dj0 = PC_C / (3.0 * o->planck[i]);
    double Djp = PC_C / (3.0 * o->planck[ip]);
    double Djm = PC_C / (3.0 * o->planck[im]);
    double Dh_up = 2 * dx * (Dj0 * Djp) / (Dj0 * dx + Djp * dx);
    double Dh_dn = 2 * dx * (Dj0 * Djm) / (Dj0 * dx + Djm * dx);
    double r_p = o->r_out.x[i];     /* grid_1D_sphere::coordinates: r_out[i] */
    double r_m = o->r_out.x[im];
    if (i == 0) r_m = 0;
    double r_0 = 0.5 * (r_p + r_m);
    double up = (dt / dx) * (Dh_up / dx) * r_p * r_p / r_0 / r_0;
    double dn = (dt / dx) * (Dh_dn / dx) * r_m * r_m / r_0 / r_0;
    if (i == 0) dn = 0;
    double adv = 0.0, ab = 0.0;
    double norm = 1 + adv + ab;
    norm += up + dn;
    ab /= norm;
    up /= norm;
    dn /= norm;
    o->imd_up[i] = up; o->imd_dn[i] = dn; o->imd_abs[i] = ab; o->imd_stay[i] = 1.0 / norm;
  }
}

#define IMD_HOPS (1 << 24)
/* transport::discrete_diffuse_IMD (discrete_diffusion.cpp:18-110), called
 * with the end time of the step where the function means the step
 * (transport.cpp:237): the photon's time advances by tstop, the J tally and
 * the advection take tstop as the interval.  Hops one zone up or down (a
 * radial move by the starting zone's width) until it stays, then is
 * advected, loses energy adiabatically and stops.  The hop loop, unbounded
 * in the reference, gives up after 2^24 hops (counted). */
static int imd_event(oracle_ctx* o, packet* p, double dt)
{
  int nn = o->nu.n, nj = o->tp.store_Jnu ? nn : 1;
  double dx = zone_size(o, p->ind);
  p->t += dt;
  for (int hops = 0;; hops++) {
    if (hops >= IMD_HOPS) { o->n_imd_cap++; break; }
    p->ind = get_zone(o, p->x);
    if (p->ind == -1) return F_ABSORBED;
    if (p->ind == -2) return F_ESCAPED;
    o->e_abs[p->ind] += p->e * o->imd_abs[p->ind];
    o->J[(size_t)p->ind * nj] += p->e * o->imd_stay[p->ind] * dt * PC_C;
    double P_diff = o->imd_up[p->ind] + o->imd_dn[p->ind];
    double P_stay = o->imd_abs[p->ind] + o->imd_stay[p->ind];
    double r1 = draw(o, p);
    if (r1 < P_diff) {
      double r2 = draw(o, p);
      if (r2 < o->imd_up[p->ind] / P_diff) {
        p->ind++;
        double rr = pr(p);
        p->x[0] += p->x[0] / rr * dx;
        p->x[1] += p->x[1] / rr * dx;
        p->x[2] += p->x[2] / rr * dx;
      } else {
        p->ind--;
        double rr = pr(p);
        p->x[0] -= p->x[0] / rr * dx;
        p->x[1] -= p->x[1] / rr * dx;
        p->x[2] -= p->x[2] / rr * dx;
      }
    } else {
      double r2 = draw(o, p);
      double f_abs = o->imd_abs[p->ind] / P_stay;
      if (r2 < f_abs) return F_ABSORBED;
      double v[3], dvds;
      get_velocity(o, p->ind, p->x, p->D, v, &dvds);
      p->x[0] += v[0] * dt;
      p->x[1] += v[1] * dt;
      p->x[2] += v[2] * dt;
      p->e *= (1 - dvds * dt);
      break;
    }
  }
  p->ind = get_zone(o, p->x);
  if (p->ind == -1) return F_ABSORBED;
  if (p->ind == -2) return F_ESCAPED;
  return F_STOPPED;
}

#define DDMC_SCATTER_TRIES (1 << 16)
/* one pass of the event loop of transport::discrete_diffuse_DDMC
 * (discrete_diffusion.cpp:136-404); *dt_remaining carries over the passes of
 * one call */
static int ddmc_event(oracle_ctx* o, packet* p, double* dt_remaining, int64_t* nscat)
{
  int nz = o->nzones, nn = o->nu.n, nj = o->tp.store_Jnu ? nn : 1;
  double lambda_ddmc = 0.7104, push = 1.0e-8;
  int fate = F_MOVING;
  int ii = p->ind, ip = ii + 1, im = ii - 1;
  if (ip == nz) ip = ii;
  if (im < 0) im = 0;
  double dx = zone_size(o, ii), dxp1 = zone_size(o, ip), dxm1 = zone_size(o, im);
  double sigma_i, sigma_im1, sigma_ip1, eps_i, eps_ip1, eps_im1;
  double dshift = dshift_lab_to_comoving(o, p);
  int i_nu = opacity_of(o, ii, p->nu * dshift, &sigma_i, &eps_i);
  opacity_of(o, ip, p->nu * dshift, &sigma_ip1, &eps_ip1);
  opacity_of(o, im, p->nu * dshift, &sigma_im1, &eps_im1);
  double r_p = o->r_out.x[ii];
  double r_m = o->r_out.x[im];
  if (ii == 0) r_m = o->r_out.min;
  double r_0 = 0.5 * (r_p + r_m);
  double Xi = 1.0 + dx * dx / (12.0 * r_0 * r_0);
  double geo_factor = r_m * r_m / r_0 / r_0 / Xi;
  double tau_im1 = sigma_im1 * dxm1;
  int ddmc_on_im1 = !(tau_im1 <= o->tp.ddmc_tau);
  double sigma_leak_left;
  if (ddmc_on_im1) sigma_leak_left = (2.0 / 3.0 / dx) * (1.0 / (sigma_i * dx + sigma_im1 * dxm1)) * geo_factor;
  else sigma_leak_left = (2.0 / 3.0 / dx) * (1.0 / (sigma_i * dx + 2.0 * lambda_ddmc)) * geo_factor;
  geo_factor = r_p * r_p / r_0 / r_0 / Xi;
  double tau_ip1 = sigma_ip1 * dxp1;
  int ddmc_on_ip1 = !(tau_ip1 <= o->tp.ddmc_tau);
  double sigma_leak_right;
  if (ddmc_on_ip1) sigma_leak_right = (2.0 / 3.0 / dx) * (1.0 / (sigma_i * dx + sigma_ip1 * dxp1)) * geo_factor;
  else sigma_leak_right = (2.0 / 3.0 / dx) * (1.0 / (sigma_i * dx + 2.0 * lambda_ddmc)) * geo_factor;
  if (ip == ii) sigma_leak_right = (2.0 / 3.0 / dx) * (1.0 / (sigma_i * dx + 2.0 * lambda_ddmc)) * geo_factor;
  if (ii == 0) sigma_leak_left = 0.0;
  double sigma_leak_tot = sigma_leak_left + sigma_leak_right;
  double xi = draw(o, p);
  int leaked2imc = 0;
  double d_stay = PC_C * *dt_remaining;
  double d_leak = -log(xi) / (sigma_leak_left + sigma_leak_right);
  double d_sc;
  if (nn == 1) d_sc = INFINITY;
  else {
    double tau_r = -1.0 * log(draw(o, p));
    if (eps_i > 0.0) {
      double k_es_inelastic = sigma_i * eps_i;
      dshift = dshift_lab_to_comoving(o, p);
      i_nu = opacity_of(o, p->ind, p->nu * dshift, &sigma_i, &eps_i);
      const double* cdf = o->cdf + (size_t)p->ind * nn;
      double elastic_frac = (i_nu == 0) ? cdf[0] : (cdf[i_nu] - cdf[i_nu - 1]);
      k_es_inelastic *= 1.0 - elastic_frac;
      d_sc = tau_r / k_es_inelastic;
    } else d_sc = INFINITY;
  }
  int event;
  double this_d;
  if ((d_sc < d_leak) && (d_sc < d_stay)) { event = 0; this_d = d_sc; }
  else if (d_leak < d_stay) { event = 1; this_d = d_leak; }
  else { event = 2; this_d = d_stay; }
  double this_dt = this_d / PC_C;
  p->t += this_dt;
  *dt_remaining -= this_dt;
  o->J[(size_t)p->ind * nj] += p->e * this_d;
  o->e_abs[p->ind] += (p->e * dshift) * this_d * sigma_i * eps_i;
  if (event == 0) {
    (*nscat)++;
    int now_i_nu = i_nu;
    for (int tries = 0; now_i_nu == i_nu; ++tries) {
      if (tries >= DDMC_SCATTER_TRIES) { o->n_reject_cap++; break; }
      /* do_scatter(p, 1.0) (scatter.cpp:12-41) */
      fate = F_MOVING;
      if (draw(o, p) > 1.0) isotropic_scatter(o, p, 0);
      else {
        double z2 = draw(o, p);
        if ((z2 > o->eps_imc[p->ind]) || o->tp.radiative_eq) isotropic_scatter(o, p, 1);
        else fate = F_ABSORBED;
      }
      dshift = dshift_lab_to_comoving(o, p);
      double s2, e2;
      now_i_nu = opacity_of(o, p->ind, p->nu * dshift, &s2, &e2);
    }
  } else if (event == 2) {
    *dt_remaining = -1.0;
    fate = F_STOPPED;
  } else {
    double P_leak_left = sigma_leak_left / sigma_leak_tot;
    double xi2 = draw(o, p);
    if (xi2 <= P_leak_left) {
      p->ind--;
      double rr = pr(p);
      double dr = rr - r_m;
      if (ddmc_on_im1) dr += draw(o, p) * dxm1;
      else dr *= (1.0 + push);
      p->x[0] -= p->x[0] / rr * dr;
      p->x[1] -= p->x[1] / rr * dr;
      p->x[2] -= p->x[2] / rr * dr;
      if (!ddmc_on_im1) {
        leaked2imc = 1;
        lorentz(o, p, 0);
        bb_surface_dir(o, p);
        double mu = (p->x[0] * p->D[0] + p->x[1] * p->D[1] + p->x[2] * p->D[2]) / pr(p);
        if (mu > 0.0) { p->D[0] = -p->D[0]; p->D[1] = -p->D[1]; p->D[2] = -p->D[2]; }
        lorentz(o, p, 1);
      }
    } else {
      p->ind++;
      double rr = pr(p);
      double dr = r_p - rr;
      if (ddmc_on_ip1) dr += draw(o, p) * dxp1;
      else dr *= (1.0 + push);
      p->x[0] += p->x[0] / rr * dr;
      p->x[1] += p->x[1] / rr * dr;
      p->x[2] += p->x[2] / rr * dr;
      if (!ddmc_on_ip1) {
        leaked2imc = 1;
        lorentz(o, p, 0);
        bb_surface_dir(o, p);
        double mu = (p->x[0] * p->D[0] + p->x[1] * p->D[1] + p->x[2] * p->D[2]) / pr(p);
        if (mu < 0.0) { p->D[0] = -p->D[0]; p->D[1] = -p->D[1]; p->D[2] = -p->D[2]; }
        lorentz(o, p, 1);
      }
    }
  }
  /* advection and adiabatic loss (discrete_diffusion.cpp:371-397) */
  double zone_vel[3], dvds;
  get_velocity(o, p->ind, p->x, p->D, zone_vel, &dvds);
  double vel = sqrt(zone_vel[0] * zone_vel[0] + zone_vel[1] * zone_vel[1] + zone_vel[2] * zone_vel[2]);
  double v_over_r = vel / pr(p);
  double dlnrhodt = dvds + 2.0 * v_over_r;
  double doppler_shift_ddmc = (1.0 - dlnrhodt * this_dt / 3.0);
  lorentz(o, p, 0);
  p->e *= doppler_shift_ddmc;
  p->nu *= doppler_shift_ddmc;
  lorentz(o, p, 1);
  if (!leaked2imc) {
    p->x[0] += zone_vel[0] * this_dt;
    p->x[1] += zone_vel[1] * this_dt;
    p->x[2] += zone_vel[2] * this_dt;
  }
  p->ind = get_zone(o, p->x);
  if (p->ind == -1) fate = F_ABSORBED;
  if (p->ind == -2) fate = F_ESCAPED;
  return fate;
}

static int propagate_from(oracle_ctx* o, packet* p, double t_now, double dt, int64_t* nseg, int64_t* nscat,
                          int relocate)
{
  int nn = o->nu.n;
  int nj = o->tp.store_Jnu ? nn : 1;
  if (relocate) p->ind = get_zone(o, p->x);
  if (p->ind == -1) return F_ABSORBED;
  if (p->ind == -2) return F_ESCAPED;
  double tstop = t_now + dt;
  int fate = F_MOVING;
  int64_t limit = o->tp.max_segments > 0 ? o->tp.max_segments : 10000000;
  int64_t seg = 0;
  /* discrete diffusion: the zone test before every pass (transport.cpp:
   * 216-246, 272-286); the remaining time of one diffusion call */
  int dd = (o->tp.use_ddmc == 2 || o->tp.use_ddmc == 1) && (o->gtype == SED_GRID_1D_SPHERE);
  int in_call = 0;
  double dt_remaining = 0;
  while (fate == F_MOVING) {
    if (seg >= limit) { fate = F_STOPPED; o->n_limit++; break; }
    seg++;
    if (dd && o->tp.use_ddmc == 1 && in_ddmc_zone(o, p)) {
      fate = imd_event(o, p, tstop);
      continue;
    }
    if (dd && in_ddmc_zone(o, p)) {
      if (!in_call) { dt_remaining = tstop - p->t; in_call = 1; }
      fate = ddmc_event(o, p, &dt_remaining, nscat);
      continue;
    }
    in_call = 0;
    int iz = p->ind;
    double d_bn = 0;
    int new_ind = get_next_zone(o, p->x, p->D, iz, o->tp.core_radius, &d_bn);
    double dshift = dshift_lab_to_comoving(o, p);
    /* a diffusive neighbour (transport.cpp:295-309) */
    int new_cell_ddmc = 0;
    double sigma_new = 0, dr_new = 0;
    if (dd && new_ind >= 0) {
      double e_new;
      opacity_of(o, new_ind, p->nu * dshift, &sigma_new, &e_new);
      dr_new = zone_size(o, new_ind);
      new_cell_ddmc = sigma_new * dr_new > o->tp.ddmc_tau;
    }
    /* transport::get_opacity, transport_opacity.cpp:268-299 */
    double nu_cmf = p->nu * dshift;
    int i_nu = lg_locate_wb(&o->nu, nu_cmf);
    double a_opac = o->abs[(size_t)iz * nn + i_nu];
    double s_opac = 0;
    if (!o->tp.omit_scattering) s_opac = o->scat[(size_t)iz * nn + i_nu];
    double opac = a_opac + s_opac;
    double eps = (opac == 0) ? 0 : a_opac / opac;
    double d_nu = lg_delta(&o->nu, i_nu) / p->nu * PC_C / p->dvds;
    if (p->dvds == 0) d_nu = INFINITY;
    if (d_nu < 0) d_nu = -1 * d_nu;
    if (d_nu < d_bn) { d_bn = d_nu; new_ind = p->ind; }
    double tot_lab = opac * dshift;
    double tau_r = -1.0 * log(1 - draw(o, p));
    double d_sc = tau_r / tot_lab;
    if (tot_lab == 0) d_sc = INFINITY;
    double d_tm = (tstop - p->t) * PC_C;
    if (o->tp.steady_state) d_tm = INFINITY;
    int event;
    double this_d;
    if ((d_sc < d_bn) && (d_sc < d_tm)) { event = 0; this_d = d_sc; }
    else if (d_bn < d_tm) { event = 1; this_d = d_bn; }
    else { event = 2; this_d = d_tm; }
    double this_E = p->e * this_d;
    o->e_abs[iz] += this_E * dshift * (opac) * eps * dshift * o->eps_imc[iz];
    if (o->tp.store_Jnu) o->J[(size_t)iz * nj + i_nu] += this_E;
    else o->J[(size_t)iz * nj] += this_E;
    if (o->tp.tally_forces) {
      o->fx[iz] += this_E * dshift * opac * p->D[0] * dshift;
      o->fy[iz] += this_E * dshift * opac * p->D[1] * dshift;
      o->fz[iz] += this_E * dshift * opac * p->D[2] * dshift;
      double rr = sqrt(p->x[0] * p->x[0] + p->x[1] * p->x[1] + p->x[2] * p->x[2]);
      double xdotD = p->x[0] * p->D[0] + p->x[1] * p->D[1] + p->x[2] * p->D[2];
      o->fr[iz] += this_E * dshift * opac * xdotD / rr * dshift;
    }
    p->x[0] += this_d * p->D[0];
    p->x[1] += this_d * p->D[1];
    p->x[2] += this_d * p->D[2];
    p->t = p->t + this_d / PC_C;
    if (event == 1) {
      if (new_ind == -1) {
        if (o->tp.boundary_in_reflect) { p->D[0] *= -1; p->D[1] *= -1; p->D[2] *= -1; }
        else { p->ind = new_ind; fate = F_ABSORBED; }
      } else if (new_ind == -2) {
        if (o->tp.boundary_out_reflect) { p->D[0] *= -1; p->D[1] *= -1; p->D[2] *= -1; }
        else { p->ind = new_ind; fate = F_ESCAPED; }
      } else if (dd && new_cell_ddmc && (new_ind != p->ind)) {
        move_across(o, p, new_ind, sigma_new, dr_new);
      } else {
        p->ind = new_ind;
      }
    } else if (event == 0) {
      /* transport::do_scatter, scatter.cpp:12-70 (photons) */
      (*nscat)++;
      if (draw(o, p) > eps) isotropic_scatter(o, p, 0);
      else {
        double z2 = draw(o, p);
        if ((z2 > o->eps_imc[iz]) || o->tp.radiative_eq) isotropic_scatter(o, p, 1);
        else fate = F_ABSORBED;
      }
    } else {
      fate = F_STOPPED;
    }
  }
  *nseg += seg;
  return fate;
}

static uint32_t draws_per_emission(const oracle_ctx* o)
{
  uint32_t k = (o->tp.core_radius == 0) ? 2 : 4;
  if (!(o->tp.core_photon_frequency > 0)) k += 2;
  return k + 1;
}

static void wipe_tallies(oracle_ctx* o)
{
  size_t nz = (size_t)o->nzones;
  size_t nj = o->tp.store_Jnu ? (size_t)o->nu.n : 1;
  memset(o->J, 0, nz * nj * sizeof(double));
  memset(o->e_abs, 0, nz * sizeof(double));
  memset(o->e_rad, 0, nz * sizeof(double));
  memset(o->fx, 0, nz * sizeof(double));
  memset(o->fy, 0, nz * sizeof(double));
  memset(o->fz, 0, nz * sizeof(double));
  memset(o->fr, 0, nz * sizeof(double));
}

/* normalisation of transport::reduce_radiation, src/transport/transport_mpi.cpp:415-441,
 * preceded by the steady-state rescale of transport.cpp:94-115 */
static void finish_step(oracle_ctx* o, double dt, int64_t n_active, int64_t n_escaped)
{
  int nn = o->nu.n;
  int nj = o->tp.store_Jnu ? nn : 1;
  if (o->tp.steady_state && o->tp.core_fix_luminosity) {
    double per_esc = (1.0 * n_escaped) / (1.0 * n_active);
    double fac = 1.0 / per_esc;
    for (int64_t i = 0; i < o->nspec; ++i) o->flux[i] *= fac;
    for (int i = 0; i < o->nzones; ++i) {
      o->e_rad[i] *= fac;
      if (o->tp.store_Jnu) for (int j = 0; j < nn; ++j) o->J[(size_t)i * nj + j] *= fac;
    }
  }
  for (int i = 0; i < o->nzones; ++i) {
    double vol = o->vol[i];
    o->e_abs[i] /= vol * dt;
    o->fr[i] /= vol * PC_C * dt;
    if ((nn == 1) || (!o->tp.store_Jnu)) {
      o->e_rad[i] = o->J[(size_t)i * nj] / (vol * dt * PC_C);
    } else {
      double esum = 0;
      for (int j = 0; j < nn; ++j) {
        double d = lg_delta(&o->nu, j);
        o->J[(size_t)i * nj + j] /= vol * dt * 4 * PC_PI * d;
        esum += o->J[(size_t)i * nj + j] * d * 4 * PC_PI / PC_C;
      }
      o->e_rad[i] = esum;
    }
  }
}

int oracle_transport_range(oracle_ctx* o, double dt, int64_t first, int64_t count, int finish, sed_step_stats* st)
{
  if (!o || !o->have_grid) return SED_ERR_STATE;
  if (!o->have_opacity) return fail(o, SED_ERR_STATE, "opacity tables not set");
  if (o->tp.steady_state) dt = 1;
  double t_now = o->t_now;
  int64_t n_emit = (int64_t)(o->tp.core_n_emit / 1.0);
  if (n_emit > o->tp.max_particles) return fail(o, SED_ERR_CAPACITY, "Not enough particle space");
  if (first == 0) {
    if (o->tp.use_ddmc == 1) imd_probabilities(o, dt);  /* transport.cpp:44 */
    o->n_imd_cap = 0;
    wipe_tallies(o);
    memset(o->flux, 0, (size_t)o->nspec * sizeof(double));
    memset(o->click, 0, (size_t)o->nspec * sizeof(double));
    o->n_escaped_acc = 0;
    o->n_active_acc = 0;
  }
  if (first < 0 || first + count > n_emit) return fail(o, SED_ERR_ARG, "packet range outside the emission");
  o->n_limit = 0;
  double Ep = o->tp.core_luminosity * dt / n_emit;
  uint32_t K = draws_per_emission(o);
  if (o->record) {
    free(o->r_fate); free(o->r_ind); free(o->r_draws); free(o->r_state);
    o->nrec = count;
    o->r_fate = (int32_t*)calloc((size_t)count + 1, 4);
    o->r_ind = (int32_t*)calloc((size_t)count + 1, 4);
    o->r_draws = (int32_t*)calloc((size_t)count + 1, 4);
    o->r_state = (double*)calloc((size_t)count * 9 + 1, 8);
  }
  int64_t nseg = 0, nscat = 0, nesc = 0, nabs = 0, nstop = 0;
  for (int64_t k = 0; k < count; ++k) {
    packet p;
    memset(&p, 0, sizeof p);
    p.pid = (uint64_t)(o->tp.first_packet_id + first + k);
    p.n = 0;
    emit_core_packet(o, &p, Ep, t_now, dt);
    p.n = K;
    int fate = propagate(o, &p, t_now, dt, &nseg, &nscat);
    if (fate == F_ESCAPED) {
      double t_obs = p.t - (p.x[0] * p.D[0] + p.x[1] * p.D[1] + p.x[2] * p.D[2]) / PC_C;
      spectrum_count(o, t_obs, p.nu, p.e, p.D);
      p.t = t_obs;
      nesc++;
    } else if (fate == F_ABSORBED) nabs++;
    else nstop++;
    if (o->record) {
      o->r_fate[k] = fate; o->r_ind[k] = p.ind; o->r_draws[k] = (int32_t)(p.n - K);
      double* s = o->r_state + (size_t)k * 9;
      s[0] = p.x[0]; s[1] = p.x[1]; s[2] = p.x[2]; s[3] = p.D[0]; s[4] = p.D[1]; s[5] = p.D[2];
      s[6] = p.t; s[7] = p.e; s[8] = p.nu;
    }
  }
  o->n_escaped_acc += nesc;
  o->n_active_acc += count;
  if (finish) {
    finish_step(o, dt, n_emit, o->n_escaped_acc);
    o->step++;  /* the next step draws from fresh streams */
  }
  if (st) {
    memset(st, 0, sizeof *st);
    st->n_packets = count; st->n_escaped = nesc; st->n_absorbed = nabs; st->n_stopped = nstop;
    st->n_segments = nseg; st->n_scatters = nscat; st->n_limit = o->n_limit;
  }
  if (o->n_limit > 0) return fail(o, SED_ERR_LIMIT, "packets hit the segment limit");
  if (o->n_imd_cap > 0) return fail(o, SED_ERR_LIMIT, "IMD calls hit the hop bound");
  return SED_OK;
}

/* ---------------------------------------------------------------- radioactive source
 * transport::emit_radioactive (src/transport/emission.cpp:163-243) with
 * radioactive::decay (src/transport/radioactive.cpp:144-275), and gamma-ray
 * transport: opacity (transport_opacity.cpp:187-203, 290-313), do_scatter
 * and compton_scatter (scatter.cpp:45-133).  Radioactive packets take the
 * stream ids before the core packets (the reference emits them first);
 * each draws from its own stream in the reference's order. */
#define TAU_56NI 757241.8
#define TAU_56CO 9627379.
#define AVERAGE_56NI_ENERGY 1.725
#define AVERAGE_56CO_ENERGY 3.730
#define CO_POSITRON_FRACTION 0.0324
#define TAU_48CR 111976.
#define TAU_48V 1.99107843e6
#define AVERAGE_48CR_ENERGY 0.442
#define AVERAGE_48V_ENERGY 3.066
#define PC_M_E_MEV 0.510998910511
#define PC_MEV_TO_ERGS 1.60217646e-6
#define PC_ALPHA_FS 0.007
static const double R_PROC_FIT[11] = {17.608179, -2.0442059, -0.42565322, 0.39830095, -0.0059089906,
                                      -0.054805836, 0.014068697, -0.00086706160, -5.7056758e-05, 2.6401842e-06,
                                      3.7186979e-07};

static double rprocess_heating_rate(double t, double* gfrac)  /* radioactive.cpp:118-142 */
{
  double td = t / 3600.0 / 24.0;
  double A1 = 8.4939E+09, alpha = 1.3642E+00, B1 = 8.3425E+09, beta1 = 3.6280E+00;
  double B2 = 8.8616E+08, beta2 = 1.0847E+01;
  double eps = A1 * pow(td, -1.0 * alpha) + B1 * exp(-1.0 * td / beta1) + B2 * exp(-1.0 * td / beta2);
  double af = 0.56, bf = 0.17, df = 0.74;
  double x = 2 * bf * pow(td, df);
  double f = 0.36 * (exp(-af * td) + log(1 + x) / x);
  *gfrac = 0;
  return eps * f;
}

static double decay_energy_rate(int Z, int A, double t, double* gfrac)  /* radioactive.cpp:178-275 */
{
  double total = 0, gtotal = 0;
  if ((Z == 28) && (A == 56)) {
    double e_ni = exp(-t / TAU_56NI), e_co = exp(-t / TAU_56CO);
    double ni56 = (e_ni / TAU_56NI);
    double co56 = 1.0 / (TAU_56NI - TAU_56CO) * (e_ni - e_co);
    double ni_E = ni56 * (AVERAGE_56NI_ENERGY * PC_MEV_TO_ERGS);
    double co_E = co56 * (AVERAGE_56CO_ENERGY * PC_MEV_TO_ERGS);
    gtotal = ni_E + (1 - CO_POSITRON_FRACTION) * co_E;
    total = ni_E + co_E;
  }
  if ((Z == 27) && (A == 56)) {
    double e_co = exp(-t / TAU_56CO);
    double co56 = 1.0 / (TAU_56CO)*e_co;
    double co_E = co56 * (AVERAGE_56CO_ENERGY * PC_MEV_TO_ERGS);
    gtotal = (1 - CO_POSITRON_FRACTION) * co_E;
    total = co_E;
  }
  if ((Z == 24) && (A == 48)) {
    double e_cr = exp(-t / TAU_48CR), e_vn = exp(-t / TAU_48V);
    double cr48 = (e_cr / TAU_48CR);
    double vn48 = 1.0 / (TAU_48CR - TAU_48V) * (e_cr - e_vn);
    double cr_E = cr48 * (AVERAGE_48CR_ENERGY * PC_MEV_TO_ERGS);
    double vn_E = vn48 * (AVERAGE_48V_ENERGY * PC_MEV_TO_ERGS);
    gtotal += cr_E + vn_E;
    total += cr_E + vn_E;
  }
  if ((Z >= 58)) {
    double at = log10(t);
    double rproc = 0;
    for (int j = 0; j < 11; j++) rproc += R_PROC_FIT[j] * pow(at, j);
    rproc = pow(10.0, rproc) * (A * PC_M_P);
    double fission_E = 0.1 * rproc;
    double beta_E = 0.9 * rproc;
    beta_E = 0.75 * beta_E;
    total += (fission_E + beta_E);
    gtotal += 0.5 * beta_E;
  }
  *gfrac = gtotal / total;
  if (total == 0) *gfrac = 0;
  return total;
}

/* per-zone decay luminosity (emission.cpp:189-205), gamma opacity
 * coefficients, zone emission CDF; returns the grid total */
static double radio_zones(oracle_ctx* o, double t)
{
  int nz = o->nzones, ne = o->nelem;
  double L_tot = 0;
  for (int i = 0; i < nz; i++) {
    const double* X = o->X + (size_t)i * ne;
    int rprocess_heat = 0;
    for (int k = 0; k < ne; k++)
      if (((o->eZ[k] > 57) && (o->eA[k] > 0)) || o->tp.force_rprocess_heating) rprocess_heat = 1;
    double L_decay, gfrac;
    if (rprocess_heat) L_decay = rprocess_heating_rate(t, &gfrac);
    else {
      double total = 0, gtotal = 0, gf;
      for (int k = 0; k < ne; k++) {
        double val = decay_energy_rate(o->eZ[k], o->eA[k], t, &gf);
        val = val * X[k] / (o->eA[k] * PC_M_P);
        total += val;
        gtotal += val * gf;
      }
      gfrac = gtotal / total;
      if (total == 0) gfrac = 0;
      L_decay = total;
    }
    L_decay = o->rho[i] * L_decay * o->vol[i];
    o->L_emit[i] = L_decay;
    o->gamma_frac[i] = gfrac;
    L_tot += L_decay;
    o->radio_cdf[i] = (i == 0) ? L_decay : o->radio_cdf[i - 1] + L_decay;  /* cdf_array::set_value */
    double comp = 0, phot = 0;
    for (int k = 0; k < ne; k++) {
      double dens = X[k] * o->rho[i];
      double ndens = dens / (PC_M_P * o->eA[k]);
      comp += ndens * PC_THOMSON * o->eZ[k];
      double photo = pow(PC_ALPHA_FS, 4.0) * 4.0 * sqrt(2.0);
      photo *= pow(1.0 * o->eZ[k], 5.0);
      photo *= pow(PC_M_E_MEV, 3.5);
      phot += ndens * 2.0 * PC_THOMSON * photo;
    }
    o->compton[i] = comp;
    o->photoion[i] = phot;
  }
  cdf_normalize(o->radio_cdf, nz);
  return L_tot;
}

static double klein_nishina(double x)  /* transport_opacity.cpp:302-313 */
{
  x = x / PC_M_E_MEV;
  double logfac = log(1 + 2 * x);
  double term1 = (1 + x) / x / x / x * (2 * x * (1 + x) / (1 + 2 * x) - logfac);
  double term2 = 1.0 / 2.0 / x * logfac;
  double term3 = -1.0 * (1 + 3 * x) / (1 + 2 * x) / (1 + 2 * x);
  return .75 * (term1 + term2 + term3);
}

/* transport::lorentz_transform (relativity.cpp:84-127), either direction */
static void lorentz(const oracle_ctx* o, packet* p, int tolab)
{
  double v[3], dvds;
  get_velocity(o, p->ind, p->x, p->D, v, &dvds);
  if (tolab) { v[0] *= -1; v[1] *= -1; v[2] *= -1; }
  double beta2 = (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) / PC_C / PC_C;
  double vdd = v[0] * p->D[0] + v[1] * p->D[1] + v[2] * p->D[2];
  double gamma = 1.0 / sqrt(1 - beta2);
  double dshift = gamma * (1 - vdd / PC_C);
  p->dvds = dvds;
  p->e *= dshift;
  p->nu *= dshift;
  double f = (1 - gamma * vdd / PC_C / (gamma + 1));
  p->D[0] = 1.0 / dshift * (p->D[0] - gamma * v[0] / PC_C * f);
  p->D[1] = 1.0 / dshift * (p->D[1] - gamma * v[1] / PC_C * f);
  p->D[2] = 1.0 / dshift * (p->D[2] - gamma * v[2] / PC_C * f);
  double norm = p->D[0] * p->D[0] + p->D[1] * p->D[1] + p->D[2] * p->D[2];
  p->D[0] /= norm;
  p->D[1] /= norm;
  p->D[2] /= norm;
}

/* grid::sample_in_zone (grid_1D_sphere.cpp:681-700, grid_3D_cart.cpp:484-494) */
static void sample_in_zone(const oracle_ctx* o, int i, double u0, double u1, double u2, double* r)
{
  if (o->gtype == SED_GRID_1D_SPHERE) {
    double r_0 = (i == 0) ? o->r_out.min : o->r_out.x[i - 1];
    double ro = o->r_out.x[i];
    double r_samp = pow(r_0 * r_0 * r_0 + u0 * (ro * ro * ro - r_0 * r_0 * r_0), 1.0 / 3.0);
    double mu = 1 - 2.0 * u1;
    double phi = 2.0 * PC_PI * u2;
    double sin_theta = sqrt(1 - mu * mu);
    r[0] = r_samp * sin_theta * cos(phi);
    r[1] = r_samp * sin_theta * sin(phi);
    r[2] = r_samp * mu;
  } else {
    int nyz = o->ny * o->nz;
    int idx[3] = {i / nyz, (i / o->nz) % o->ny, i % o->nz};
    double u[3] = {u0, u1, u2};
    for (int a = 0; a < 3; a++) r[a] = lg_left(&o->ax[a], idx[a]) + u[a] * lg_delta(&o->ax[a], idx[a]);
  }
}

static void iso_dir(const oracle_ctx* o, packet* p, double* D)
{
  double mu = 1 - 2.0 * draw(o, p);
  double phi = 2.0 * PC_PI * draw(o, p);
  double smu = sqrt(1 - mu * mu);
  D[0] = smu * cos(phi);
  D[1] = smu * sin(phi);
  D[2] = mu;
}

static void sample_optical_nu(const oracle_ctx* o, packet* p)  /* sample_photon_frequency, emission.cpp:27-46 */
{
  int nn = o->nu.n;
  int inu = cdf_sample(o->cdf + (size_t)p->ind * nn, nn, draw(o, p));
  p->nu = lg_sample(&o->nu, inu, draw(o, p));
}

#define COMPTON_TRIES (1 << 16)
/* propagate + propagate_monte_carlo for a gamma-ray; *photon is set when it
 * becomes an optical photon (its state is then the photon's) */
static int propagate_gamma(oracle_ctx* o, packet* p, double t_now, double dt, int* photon, int64_t* nseg,
                           int64_t* nscat)
{
  *photon = 0;
  p->ind = get_zone(o, p->x);
  if (p->ind == -1) return F_ABSORBED;
  if (p->ind == -2) return F_ESCAPED;
  double tstop = t_now + dt;
  int fate = F_MOVING;
  int64_t limit = o->tp.max_segments > 0 ? o->tp.max_segments : 10000000;
  int64_t seg = 0;
  while (fate == F_MOVING && !*photon) {
    if (seg >= limit) { fate = F_STOPPED; o->n_limit++; break; }
    seg++;
    int iz = p->ind;
    double d_bn = 0;
    int new_ind = get_next_zone(o, p->x, p->D, iz, o->tp.core_radius, &d_bn);
    double dshift = dshift_lab_to_comoving(o, p);
    double c_opac = o->compton[iz] * klein_nishina(p->nu);
    double p_opac = o->photoion[iz] * pow(p->nu, -3.5);
    double opac = c_opac + p_opac;
    double eps = p_opac / (c_opac + p_opac);
    double d_nu = lg_delta(&o->nu, 0) / p->nu * PC_C / p->dvds;
    if (p->dvds == 0) d_nu = INFINITY;
    if (d_nu < 0) d_nu = -1 * d_nu;
    if (d_nu < d_bn) { d_bn = d_nu; new_ind = p->ind; }
    double tot_lab = opac * dshift;
    double tau_r = -1.0 * log(1 - draw(o, p));
    double d_sc = tau_r / tot_lab;
    if (tot_lab == 0) d_sc = INFINITY;
    double d_tm = (tstop - p->t) * PC_C;
    if (o->tp.steady_state) d_tm = INFINITY;
    int event;
    double this_d;
    if ((d_sc < d_bn) && (d_sc < d_tm)) { event = 0; this_d = d_sc; }
    else if (d_bn < d_tm) { event = 1; this_d = d_bn; }
    else { event = 2; this_d = d_tm; }
    double this_E = p->e * this_d;
    if (o->tp.tally_forces) {
      o->fx[iz] += this_E * dshift * opac * p->D[0] * dshift;
      o->fy[iz] += this_E * dshift * opac * p->D[1] * dshift;
      o->fz[iz] += this_E * dshift * opac * p->D[2] * dshift;
      double rr = sqrt(p->x[0] * p->x[0] + p->x[1] * p->x[1] + p->x[2] * p->x[2]);
      double xdotD = p->x[0] * p->D[0] + p->x[1] * p->D[1] + p->x[2] * p->D[2];
      o->fr[iz] += this_E * dshift * opac * xdotD / rr * dshift;
    }
    p->x[0] += this_d * p->D[0];
    p->x[1] += this_d * p->D[1];
    p->x[2] += this_d * p->D[2];
    p->t = p->t + this_d / PC_C;
    if (event == 1) {
      if (new_ind == -1) {
        if (o->tp.boundary_in_reflect) { p->D[0] *= -1; p->D[1] *= -1; p->D[2] *= -1; }
        else { p->ind = new_ind; fate = F_ABSORBED; }
      } else if (new_ind == -2) {
        if (o->tp.boundary_out_reflect) { p->D[0] *= -1; p->D[1] *= -1; p->D[2] *= -1; }
        else { p->ind = new_ind; fate = F_ESCAPED; }
      } else {
        p->ind = new_ind;
      }
    } else if (event == 0) {
      (*nscat)++;
      if (draw(o, p) > eps) {
        lorentz(o, p, 0);
        double E_ratio = 1, Dn[3];
        for (int tries = 0;; ++tries) {
          iso_dir(o, p, Dn);
          double cost = p->D[0] * Dn[0] + p->D[1] * Dn[1] + p->D[2] * Dn[2];
          E_ratio = 1 / (1 + p->nu / PC_M_E_MEV * (1 - cost));
          double diff_cs = 0.5 * (E_ratio * E_ratio * (1 / E_ratio + E_ratio - 1 + cost * cost));
          if (draw(o, p) < diff_cs) break;
          if (tries + 1 >= COMPTON_TRIES) { o->n_reject_cap++; break; }
        }
        p->nu = p->nu * E_ratio;
        if (draw(o, p) > E_ratio) {
          o->L_dep[p->ind] += p->e;
          *photon = 1;
          iso_dir(o, p, Dn);
          sample_optical_nu(o, p);
        }
        p->D[0] = Dn[0]; p->D[1] = Dn[1]; p->D[2] = Dn[2];
        lorentz(o, p, 1);
      } else {
        o->L_dep[p->ind] += p->e;
        *photon = 1;
        iso_dir(o, p, p->D);
        sample_optical_nu(o, p);
        lorentz(o, p, 1);
      }
    } else {
      fate = F_STOPPED;
    }
  }
  *nseg += seg;
  return fate;
}

/* the record of a packet: fate, zone, deviates, end state and type */
static void record_at(oracle_ctx* o, int64_t r, int fate, const packet* p, int32_t draws, int type)
{
  o->r_fate[r] = fate; o->r_ind[r] = p->ind; o->r_draws[r] = draws; o->r_type[r] = type;
  double* sv = o->r_state + (size_t)r * 9;
  sv[0] = p->x[0]; sv[1] = p->x[1]; sv[2] = p->x[2]; sv[3] = p->D[0]; sv[4] = p->D[1]; sv[5] = p->D[2];
  sv[6] = p->t; sv[7] = p->e; sv[8] = p->nu;
}

#define T_PHOTON 0
#define T_GAMMA 1

/* transport::clean_up_particle_vector (transport.cpp:164-194), literally, on
 * the step's packet vector (queued packets, then core packets; radioactive
 * packets that were never emitted are not in it): the stopped packets that
 * remain become the census */
static void build_census(oracle_ctx* o, int64_t n_core, int64_t n_q)
{
  int64_t n_all = n_core + n_q, m = 0;
  int64_t* v = (int64_t*)malloc((size_t)(n_all + 1) * sizeof(int64_t));
  for (int64_t r = 0; r < n_all; ++r) {
    int64_t slot = r < n_q ? n_core + r : r - n_q;
    if (o->r_fate[slot] != -1) v[m++] = slot;
  }
#define DEAD(k) (o->r_fate[v[k]] == F_ESCAPED || o->r_fate[v[k]] == F_ABSORBED)
  int64_t size = m, i = 0;
  for (;;) {
    while (size > 0 && DEAD(size - 1)) size--;
    if (i >= size) break;
    if (DEAD(i)) { v[i] = v[size - 1]; size--; }
    i++;
  }
#undef DEAD
  free(o->c_state); free(o->c_ind); free(o->c_type);
  o->c_state = (double*)malloc((size_t)(size + 1) * 9 * sizeof(double));
  o->c_ind = (int32_t*)malloc((size_t)(size + 1) * sizeof(int32_t));
  o->c_type = (int32_t*)malloc((size_t)(size + 1) * sizeof(int32_t));
  for (int64_t k = 0; k < size; ++k) {
    memcpy(o->c_state + (size_t)k * 9, o->r_state + (size_t)v[k] * 9, 9 * sizeof(double));
    o->c_ind[k] = o->r_ind[v[k]];
    o->c_type[k] = o->r_type[v[k]];
  }
  o->n_census = size;
  free(v);
}

/* transport::step with every source this restatement has (transport.cpp:
 * 26-140): the census the last step left, then the radioactive packets,
 * then the core packets, each on its own Philox stream (census and
 * radioactive packets first).  Records list the core packets, then the
 * queued ones (as gamma-rays, or as the optical photons they became). */
int oracle_wipe_spectra(oracle_ctx* o);

static int transport_general(oracle_ctx* o, double dt, sed_step_stats* st)
{
  if (o->tp.steady_state) dt = 1;
  int timedep = !o->tp.steady_state;
  double t_now = o->t_now;
  int64_t n_emit = (int64_t)(o->tp.core_n_emit / 1.0);
  int64_t n_census = o->n_census;
  int64_t n_radio = o->tp.n_emit_radioactive > 0 ? o->tp.n_emit_radioactive : 0;
  if (n_census + n_radio > o->tp.max_particles) n_radio = 0;
  /* emit_inner_source: "# Not enough particle space", nothing emitted, and
   * the step goes on with the census and radioactive packets
   * (emission.cpp:391-392) */
  int32_t warnings = 0;
  if (n_census + n_radio + n_emit > o->tp.max_particles) { n_emit = 0; warnings |= SED_WARN_NO_PARTICLE_SPACE; }
  int64_t n_q = n_census + n_radio, n_all = n_emit + n_q;
  int census_gammas = 0;
  for (int64_t k = 0; k < n_census; ++k) census_gammas += (o->c_type[k] == T_GAMMA);
  int gamma_phase = n_radio > 0 || census_gammas > 0;
  int nz = o->nzones;
  if (o->tp.use_ddmc == 1) imd_probabilities(o, dt);  /* transport.cpp:44 */
  o->n_imd_cap = 0;
  wipe_tallies(o);
  /* spectra accumulate over time-dependent steps; a steady-state iteration
   * starts from empty ones (SedonaClass.cpp:349) */
  if (gamma_phase) alloc_gamma_spectrum(o);
  if (!timedep) oracle_wipe_spectra(o);
  double L_tot = 0;
  if (gamma_phase) {
    double** zarr[6] = {&o->L_emit, &o->L_dep, &o->radio_cdf, &o->gamma_frac, &o->compton, &o->photoion};
    for (int q = 0; q < 6; q++) { free(*zarr[q]); *zarr[q] = (double*)calloc((size_t)nz, sizeof(double)); }
    L_tot = radio_zones(o, t_now);
    /* emit_radioactive sets L_radio_emit only when it emits */
    if (n_radio == 0) memset(o->L_emit, 0, (size_t)nz * sizeof(double));
  }
  o->n_reject_cap = 0;
  o->n_limit = 0;
  double Ep_r = L_tot * dt / (1.0 * n_radio);
  if (o->record || timedep) {
    free(o->r_fate); free(o->r_ind); free(o->r_draws); free(o->r_state); free(o->r_type);
    o->nrec = n_all;
    o->r_fate = (int32_t*)calloc((size_t)n_all + 1, 4);
    o->r_ind = (int32_t*)calloc((size_t)n_all + 1, 4);
    o->r_draws = (int32_t*)calloc((size_t)n_all + 1, 4);
    o->r_type = (int32_t*)calloc((size_t)n_all + 1, 4);
    o->r_state = (double*)calloc((size_t)n_all * 9 + 1, 8);
    for (int64_t k = n_emit; k < n_all; ++k) o->r_fate[k] = -1;  /* stays when nothing is emitted */
  }
  int keep = o->record || timedep;
  int64_t nseg = 0, nscat = 0, nesc = 0, nabs = 0, nstop = 0;
  for (int64_t k = 0; k < n_q; ++k) {
    packet p;
    memset(&p, 0, sizeof p);
    p.pid = (uint64_t)(o->tp.first_packet_id + k);
    p.n = 0;
    int is_gamma, relocate = 1;
    if (k < n_census) {
      const double* c = o->c_state + (size_t)k * 9;
      p.x[0] = c[0]; p.x[1] = c[1]; p.x[2] = c[2]; p.D[0] = c[3]; p.D[1] = c[4]; p.D[2] = c[5];
      p.t = c[6]; p.e = c[7]; p.nu = c[8];
      p.ind = o->c_ind[k];
      is_gamma = (o->c_type[k] == T_GAMMA);
    } else {
      if (L_tot == 0) continue;
      int i = cdf_sample(o->radio_cdf, nz, draw(o, &p));
      double t = t_now + dt * draw(o, &p);
      is_gamma = draw(o, &p) < o->gamma_frac[i];
      if (!is_gamma) o->L_dep[i] += Ep_r;
      double u0 = draw(o, &p), u1 = draw(o, &p), u2 = draw(o, &p);
      sample_in_zone(o, i, u0, u1, u2, p.x);
      iso_dir(o, &p, p.D);
      p.ind = i;
      if (is_gamma) p.nu = 1;
      else sample_optical_nu(o, &p);
      p.e = Ep_r;
      lorentz(o, &p, 1);
      p.t = t;
    }
    int fate;
    if (is_gamma) {
      int photon = 0;
      fate = propagate_gamma(o, &p, t_now, dt, &photon, &nseg, &nscat);
      if (!photon) {
        if (fate == F_ESCAPED) {
          double t_obs = p.t - (p.x[0] * p.D[0] + p.x[1] * p.D[1] + p.x[2] * p.D[2]) / PC_C;
          spectrum_count_on(o, &o->gn, o->gflux, o->gclick, t_obs, p.nu, p.e, p.D);
          p.t = t_obs;
          nesc++;
        } else if (fate == F_ABSORBED) nabs++;
        else nstop++;
        if (keep) record_at(o, n_emit + k, fate, &p, (int32_t)p.n, T_GAMMA);
        continue;
      }
      relocate = 0;
    }
    fate = propagate_from(o, &p, t_now, dt, &nseg, &nscat, relocate);
    if (fate == F_ESCAPED) {
      double t_obs = p.t - (p.x[0] * p.D[0] + p.x[1] * p.D[1] + p.x[2] * p.D[2]) / PC_C;
      spectrum_count(o, t_obs, p.nu, p.e, p.D);
      p.t = t_obs;
      nesc++;
    } else if (fate == F_ABSORBED) nabs++;
    else nstop++;
    if (keep) record_at(o, n_emit + k, fate, &p, (int32_t)p.n, T_PHOTON);
  }
  double Ep = o->tp.core_luminosity * dt / n_emit;
  uint32_t K = draws_per_emission(o);
  for (int64_t j = 0; j < n_emit; ++j) {
    packet p;
    memset(&p, 0, sizeof p);
    p.pid = (uint64_t)(o->tp.first_packet_id + n_q + j);
    p.n = 0;
    emit_core_packet(o, &p, Ep, t_now, dt);
    p.n = K;
    int fate = propagate(o, &p, t_now, dt, &nseg, &nscat);
    if (fate == F_ESCAPED) {
      double t_obs = p.t - (p.x[0] * p.D[0] + p.x[1] * p.D[1] + p.x[2] * p.D[2]) / PC_C;
      spectrum_count(o, t_obs, p.nu, p.e, p.D);
      p.t = t_obs;
      nesc++;
    } else if (fate == F_ABSORBED) nabs++;
    else nstop++;
    if (keep) record_at(o, j, fate, &p, (int32_t)(p.n - K), T_PHOTON);
  }
  finish_step(o, dt, n_all, nesc);
  if (gamma_phase)
    for (int i = 0; i < nz; i++) {  /* transport_mpi.cpp:419-420 */
      o->L_dep[i] /= o->vol[i] * dt;
      o->L_emit[i] /= o->vol[i];
    }
  if (timedep) build_census(o, n_emit, n_q);
  else o->n_census = 0;
  o->step++;
  if (timedep) o->t_now += dt;
  if (st) {
    memset(st, 0, sizeof *st);
    st->n_packets = n_all; st->n_escaped = nesc; st->n_absorbed = nabs; st->n_stopped = nstop;
    st->n_segments = nseg; st->n_scatters = nscat; st->warnings = warnings; st->n_limit = o->n_limit;
  }
  if (o->n_limit > 0) return fail(o, SED_ERR_LIMIT, "packets hit the segment limit");
  if (o->n_imd_cap > 0) return fail(o, SED_ERR_LIMIT, "IMD calls hit the hop bound");
  if (o->n_reject_cap > 0)
    return fail(o, SED_ERR_LIMIT, "Compton rejection or diffusion effective-scattering loops hit their bound");
  return SED_OK;
}

int64_t oracle_n_particles(oracle_ctx* o) { return o ? o->n_census : 0; }

int oracle_set_core_source(oracle_ctx* o, double luminosity, const double* weights)
{
  if (!o) return SED_ERR_ARG;
  if (!(luminosity >= 0)) return fail(o, SED_ERR_ARG, "negative luminosity");
  o->tp.core_luminosity = luminosity;
  if (weights) {  /* transport_init.cpp:509-537: set_value per bin, then normalize */
    int nn = o->nu.n;
    for (int j = 0; j < nn; ++j) o->core_cdf[j] = (j == 0) ? weights[0] : o->core_cdf[j - 1] + weights[j];
    cdf_normalize(o->core_cdf, nn);
  }
  return SED_OK;
}

int oracle_wipe_spectra(oracle_ctx* o)  /* transport::wipe_spectra (transport_output.cpp:63-67) */
{
  if (!o) return SED_ERR_ARG;
  memset(o->flux, 0, (size_t)o->nspec * sizeof(double));
  memset(o->click, 0, (size_t)o->nspec * sizeof(double));
  if (o->gflux) {
    memset(o->gflux, 0, (size_t)o->nspec_g * sizeof(double));
    memset(o->gclick, 0, (size_t)o->nspec_g * sizeof(double));
  }
  return SED_OK;
}

int oracle_get_particles(oracle_ctx* o, int64_t n, int32_t* ind, int32_t* type, double* state9)
{
  if (!o) return SED_ERR_ARG;
  if (n < 0 || n > o->n_census) return fail(o, SED_ERR_ARG, "more packets than carried");
  if (n == 0) return SED_OK;
  if (ind) memcpy(ind, o->c_ind, (size_t)n * 4);
  if (type) memcpy(type, o->c_type, (size_t)n * 4);
  if (state9) memcpy(state9, o->c_state, (size_t)n * 72);
  return SED_OK;
}

int oracle_set_time(oracle_ctx* o, double t_now)
{
  if (!o) return SED_ERR_ARG;
  o->t_now = t_now;
  o->have_t_now = 1;
  return SED_OK;
}

double oracle_get_time(oracle_ctx* o) { return o ? o->t_now : 0.0; }

static double blackbody_nu(double T, double nu);

/* transport::initialize_particles (emission.cpp:112-159): zone from e_rad *
 * vol, then create_isotropic_particle with a blackbody emissivity at the
 * gas temperature, at the transport clock's time.  The deviates of packet k
 * come from stream first_packet_id + (carried packets) + k at step number
 * 0xFFFFFFFF. */
int oracle_initialize_particles(oracle_ctx* o, int64_t n, const double* e_rad)
{
  if (!o) return SED_ERR_ARG;
  if (!o->have_grid) return SED_ERR_STATE;
  if (n < 0 || (n > 0 && !e_rad)) return fail(o, SED_ERR_ARG, "bad arguments");
  if (n == 0) return SED_OK;
  if (n > o->tp.max_particles) return fail(o, SED_ERR_CAPACITY, "Not enough particle space to initialize");
  int nz = o->nzones, ng = o->nu.n;
  double* zc = (double*)malloc((size_t)nz * sizeof(double));
  double* bb = (double*)malloc((size_t)nz * ng * sizeof(double));
  double E_sum = 0;
  for (int i = 0; i < nz; ++i) {
    double E_zone = e_rad[i] * o->vol[i];
    zc[i] = (i == 0) ? E_zone : zc[i - 1] + E_zone;
    E_sum += E_zone;
    double* row = bb + (size_t)i * ng;
    for (int j = 0; j < ng; ++j) {
      double emis = blackbody_nu(o->T[i], lg_center(&o->nu, j)) * lg_delta(&o->nu, j);
      row[j] = (j == 0) ? emis : row[j - 1] + emis;
    }
    cdf_normalize(row, ng);
  }
  cdf_normalize(zc, nz);
  int64_t off = o->n_census;
  o->c_state = (double*)realloc(o->c_state, (size_t)(off + n) * 9 * sizeof(double));
  o->c_ind = (int32_t*)realloc(o->c_ind, (size_t)(off + n) * sizeof(int32_t));
  o->c_type = (int32_t*)realloc(o->c_type, (size_t)(off + n) * sizeof(int32_t));
  double Ep = E_sum / (1.0 * n);
  uint32_t saved = o->step;
  o->step = 0xFFFFFFFFu;
  for (int64_t k = 0; k < n; ++k) {
    packet p;
    memset(&p, 0, sizeof p);
    p.pid = (uint64_t)(o->tp.first_packet_id + off + k);
    int i = cdf_sample(zc, nz, draw(o, &p));
    p.ind = i;
    double u0 = draw(o, &p), u1 = draw(o, &p), u2 = draw(o, &p);
    sample_in_zone(o, i, u0, u1, u2, p.x);
    iso_dir(o, &p, p.D);
    int inu = cdf_sample(bb + (size_t)i * ng, ng, draw(o, &p));
    p.nu = lg_sample(&o->nu, inu, draw(o, &p));
    p.e = Ep;
    lorentz(o, &p, 1);
    p.t = o->t_now;
    double* c = o->c_state + (size_t)(off + k) * 9;
    c[0] = p.x[0]; c[1] = p.x[1]; c[2] = p.x[2]; c[3] = p.D[0]; c[4] = p.D[1]; c[5] = p.D[2];
    c[6] = p.t; c[7] = p.e; c[8] = p.nu;
    o->c_ind[off + k] = i;
    o->c_type[off + k] = T_PHOTON;
  }
  o->step = saved;
  o->n_census = off + n;
  free(zc); free(bb);
  return SED_OK;
}

int oracle_get_gamma_spectrum(oracle_ctx* o, double* flux, double* click)
{
  if (!o || !o->gflux) return SED_ERR_STATE;
  if (flux) memcpy(flux, o->gflux, (size_t)o->nspec_g * sizeof(double));
  if (click) memcpy(click, o->gclick, (size_t)o->nspec_g * sizeof(double));
  return SED_OK;
}

int oracle_get_radioactive_tallies(oracle_ctx* o, double* L_emit, double* L_dep)
{
  if (!o || !o->L_dep) return SED_ERR_STATE;
  if (L_emit) memcpy(L_emit, o->L_emit, (size_t)o->nzones * sizeof(double));
  if (L_dep) memcpy(L_dep, o->L_dep, (size_t)o->nzones * sizeof(double));
  return SED_OK;
}

int oracle_transport(oracle_ctx* o, double dt, sed_step_stats* st)
{
  if (!o) return SED_ERR_ARG;
  if (o->tp.use_ddmc != 0 && ((o->tp.use_ddmc != 1 && o->tp.use_ddmc != 2) || o->gtype != SED_GRID_1D_SPHERE))
    return fail(o, SED_ERR_ARG, "discrete diffusion is built for methods 1 and 2 on 1D spheres");
  if (o->tp.n_emit_radioactive > 0 || o->n_census > 0 || !o->tp.steady_state ||
      (int64_t)(o->tp.core_n_emit / 1.0) > o->tp.max_particles) {
    if (!o->have_grid) return SED_ERR_STATE;
    if (!o->have_opacity) return fail(o, SED_ERR_STATE, "opacity tables not set");
    return transport_general(o, dt, st);
  }
  return oracle_transport_range(o, dt, 0, (int64_t)(o->tp.core_n_emit / 1.0), 1, st);
}

/* ---------------------------------------------------------------- differentiation
 * No reference counterpart.  The weighted forward is propagate() with one
 * change of estimator: interactions are sampled from the scattering opacity
 * alone and the absorption a (times abs_scale of the zone's band) is a
 * continuous weight exp(-a dshift l) on every segment; tallies use the
 * segment-averaged weight e (1 - exp(-tau_a)) / tau_a.  The derivative of the
 * escaping energy W with respect to the band factor theta of (zone, band) is
 * -W sum a0 dshift l over the packet's segments in that (zone, band); here it
 * is accumulated forward, per packet, into the dense Jacobian. */
typedef struct {
  double* acc;     /* [nzones * bands] sum of a0 dshift l of the current packet */
  int64_t* touched;
  int64_t n_touched;
  double* rho;     /* [nzones] sum of (a + s) dshift l minus the scatters, per zone */
  unsigned char* rmark;  /* [nzones] zone touched by the current packet */
  int64_t* rtouched;
  int64_t n_rtouched;
} diff_acc;

static int propagate_weighted(oracle_ctx* o, packet* p, double t_now, double dt, const double* abs_scale,
                              int n_bands, diff_acc* da, int64_t* nseg, int64_t* nscat)
{
  int nn = o->nu.n;
  int nj = o->tp.store_Jnu ? nn : 1;
  p->ind = get_zone(o, p->x);
  if (p->ind == -1) return F_ABSORBED;
  if (p->ind == -2) return F_ESCAPED;
  double tstop = t_now + dt;
  int fate = F_MOVING;
  int64_t limit = o->tp.max_segments > 0 ? o->tp.max_segments : 10000000;
  int64_t seg = 0;
  while (fate == F_MOVING) {
    if (seg >= limit) { fate = F_STOPPED; o->n_limit++; break; }
    seg++;
    int iz = p->ind;
    double d_bn = 0;
    int new_ind = get_next_zone(o, p->x, p->D, iz, o->tp.core_radius, &d_bn);
    double dshift = dshift_lab_to_comoving(o, p);
    double nu_cmf = p->nu * dshift;
    int i_nu = lg_locate_wb(&o->nu, nu_cmf);
    double a0 = o->abs[(size_t)iz * nn + i_nu];
    double a_opac = a0;
    double s_opac = 0;
    if (!o->tp.omit_scattering) s_opac = o->scat[(size_t)iz * nn + i_nu];
    int band = (int)(((int64_t)i_nu * n_bands) / nn);
    if (abs_scale) a_opac *= abs_scale[(size_t)iz * n_bands + band];
    double opac = a_opac + s_opac;
    double d_nu = lg_delta(&o->nu, i_nu) / p->nu * PC_C / p->dvds;
    if (p->dvds == 0) d_nu = INFINITY;
    if (d_nu < 0) d_nu = -1 * d_nu;
    if (d_nu < d_bn) { d_bn = d_nu; new_ind = p->ind; }
    double tot_lab = s_opac * dshift;
    double tau_r = -1.0 * log(1 - draw(o, p));
    double d_sc = tau_r / tot_lab;
    if (tot_lab == 0) d_sc = INFINITY;
    double d_tm = (tstop - p->t) * PC_C;
    if (o->tp.steady_state) d_tm = INFINITY;
    int event;
    double this_d;
    if ((d_sc < d_bn) && (d_sc < d_tm)) { event = 0; this_d = d_sc; }
    else if (d_bn < d_tm) { event = 1; this_d = d_bn; }
    else { event = 2; this_d = d_tm; }
    double tau_a = a_opac * dshift * this_d;
    double att = exp(-tau_a);
    double em1 = expm1(-tau_a);
    double this_E = (tau_a > 0 ? p->e * (-em1 / tau_a) : p->e) * this_d;
    if (da) {
      int64_t key = (int64_t)iz * n_bands + band;
      if (da->acc[key] == 0) da->touched[da->n_touched++] = key;
      da->acc[key] += a0 * dshift * this_d;
      /* density of zone iz scales a and s alike: the weight's log falls by
       * (a dshift l), the path's log-likelihood by (s dshift l) per segment
       * and rises by one per scattering (score of the sampled path) */
      if (!da->rmark[iz]) { da->rmark[iz] = 1; da->rtouched[da->n_rtouched++] = iz; }
      da->rho[iz] += (a_opac + s_opac) * dshift * this_d;
      if (event == 0) da->rho[iz] -= 1.0;
    }
    o->e_abs[iz] += this_E * dshift * a_opac * dshift * o->eps_imc[iz];
    if (o->tp.store_Jnu) o->J[(size_t)iz * nj + i_nu] += this_E;
    else o->J[(size_t)iz * nj] += this_E;
    if (o->tp.tally_forces) {
      o->fx[iz] += this_E * dshift * opac * p->D[0] * dshift;
      o->fy[iz] += this_E * dshift * opac * p->D[1] * dshift;
      o->fz[iz] += this_E * dshift * opac * p->D[2] * dshift;
      double rr = sqrt(p->x[0] * p->x[0] + p->x[1] * p->x[1] + p->x[2] * p->x[2]);
      double xdotD = p->x[0] * p->D[0] + p->x[1] * p->D[1] + p->x[2] * p->D[2];
      o->fr[iz] += this_E * dshift * opac * xdotD / rr * dshift;
    }
    p->x[0] += this_d * p->D[0];
    p->x[1] += this_d * p->D[1];
    p->x[2] += this_d * p->D[2];
    p->t = p->t + this_d / PC_C;
    p->e *= att;
    if (event == 1) {
      if (new_ind == -1) {
        if (o->tp.boundary_in_reflect) { p->D[0] *= -1; p->D[1] *= -1; p->D[2] *= -1; }
        else { p->ind = new_ind; fate = F_ABSORBED; }
      } else if (new_ind == -2) {
        if (o->tp.boundary_out_reflect) { p->D[0] *= -1; p->D[1] *= -1; p->D[2] *= -1; }
        else { p->ind = new_ind; fate = F_ESCAPED; }
      } else {
        p->ind = new_ind;
      }
    } else if (event == 0) {
      (*nscat)++;
      isotropic_scatter(o, p, 0);
    } else {
      fate = F_STOPPED;
    }
  }
  *nseg += seg;
  return fate;
}

int oracle_set_emission(oracle_ctx* o, double core_n_emit, int64_t n_emit_radioactive)
{
  if (!o) return SED_ERR_ARG;
  if (!(core_n_emit >= 0) || n_emit_radioactive < 0) return fail(o, SED_ERR_ARG, "negative packet count");
  o->tp.core_n_emit = core_n_emit;
  o->tp.n_emit_radioactive = n_emit_radioactive;
  if (n_emit_radioactive > 0) alloc_gamma_spectrum(o);
  return SED_OK;
}

int oracle_set_rng_step(oracle_ctx* o, uint32_t step)
{
  if (!o) return SED_ERR_ARG;
  o->step = step;
  return SED_OK;
}

int oracle_diff_forward(oracle_ctx* o, double dt, const double* abs_scale, int32_t n_bands, sed_step_stats* st)
{
  if (!o || !o->have_grid) return SED_ERR_STATE;
  if (!o->have_opacity) return fail(o, SED_ERR_STATE, "opacity tables not set");
  if (!o->homologous || o->tp.radiative_eq || o->tp.fleck_alpha != 0 ||
      (o->tp.steady_state && o->tp.core_fix_luminosity))
    return fail(o, SED_ERR_ARG, "differentiable transport: unsupported configuration");
  if (n_bands < 1 || n_bands > o->nu.n) return fail(o, SED_ERR_ARG, "bad band count");
  if (o->tp.steady_state) dt = 1;
  double t_now = o->t_now;
  int64_t n_emit = (int64_t)(o->tp.core_n_emit / 1.0);
  if (n_emit > o->tp.max_particles) return fail(o, SED_ERR_CAPACITY, "Not enough particle space");
  wipe_tallies(o);
  memset(o->flux, 0, (size_t)o->nspec * sizeof(double));
  memset(o->click, 0, (size_t)o->nspec * sizeof(double));
  size_t nzb = (size_t)o->nzones * (size_t)n_bands;
  free(o->jac);
  o->jac_n = o->nspec * (int64_t)nzb;
  o->jac = (double*)calloc((size_t)o->jac_n, sizeof(double));
  o->diff_bands = n_bands;
  free(o->jac_rho);
  o->jac_rho = (double*)calloc((size_t)o->nspec * (size_t)o->nzones, sizeof(double));
  diff_acc da;
  da.acc = (double*)calloc(nzb, sizeof(double));
  da.touched = (int64_t*)malloc(nzb * sizeof(int64_t));
  da.rho = (double*)calloc((size_t)o->nzones, sizeof(double));
  da.rmark = (unsigned char*)calloc((size_t)o->nzones, 1);
  da.rtouched = (int64_t*)malloc((size_t)o->nzones * sizeof(int64_t));
  if (!o->jac || !o->jac_rho || !da.acc || !da.touched || !da.rho || !da.rmark || !da.rtouched) {
    free(da.acc); free(da.touched); free(da.rho); free(da.rmark); free(da.rtouched);
    return fail(o, SED_ERR_NOMEM, "out of memory");
  }
  double Ep = o->tp.core_luminosity * dt / n_emit;
  uint32_t K = draws_per_emission(o);
  if (o->record) {
    free(o->r_fate); free(o->r_ind); free(o->r_draws); free(o->r_state);
    o->nrec = n_emit;
    o->r_fate = (int32_t*)calloc((size_t)n_emit + 1, 4);
    o->r_ind = (int32_t*)calloc((size_t)n_emit + 1, 4);
    o->r_draws = (int32_t*)calloc((size_t)n_emit + 1, 4);
    o->r_state = (double*)calloc((size_t)n_emit * 9 + 1, 8);
  }
  int64_t nseg = 0, nscat = 0, nesc = 0, nabs = 0, nstop = 0;
  for (int64_t k = 0; k < n_emit; ++k) {
    packet p;
    memset(&p, 0, sizeof p);
    p.pid = (uint64_t)(o->tp.first_packet_id + k);
    p.n = 0;
    emit_core_packet(o, &p, Ep, t_now, dt);
    p.n = K;
    da.n_touched = 0;
    da.n_rtouched = 0;
    int fate = propagate_weighted(o, &p, t_now, dt, abs_scale, n_bands, &da, &nseg, &nscat);
    if (fate == F_ESCAPED) {
      double t_obs = p.t - (p.x[0] * p.D[0] + p.x[1] * p.D[1] + p.x[2] * p.D[2]) / PC_C;
      int64_t s = spectrum_count(o, t_obs, p.nu, p.e, p.D);
      if (s >= 0) {
        for (int64_t q = 0; q < da.n_touched; ++q) {
          int64_t key = da.touched[q];
          o->jac[s * (int64_t)nzb + key] -= p.e * da.acc[key];
        }
        for (int64_t q = 0; q < da.n_rtouched; ++q) {
          int64_t z = da.rtouched[q];
          o->jac_rho[s * (int64_t)o->nzones + z] -= p.e * da.rho[z];
        }
      }
      p.t = t_obs;
      nesc++;
    } else if (fate == F_ABSORBED) nabs++;
    else nstop++;
    for (int64_t q = 0; q < da.n_touched; ++q) da.acc[da.touched[q]] = 0;
    for (int64_t q = 0; q < da.n_rtouched; ++q) { da.rho[da.rtouched[q]] = 0; da.rmark[da.rtouched[q]] = 0; }
    if (o->record) {
      o->r_fate[k] = fate; o->r_ind[k] = p.ind; o->r_draws[k] = (int32_t)(p.n - K);
      double* sv = o->r_state + (size_t)k * 9;
      sv[0] = p.x[0]; sv[1] = p.x[1]; sv[2] = p.x[2]; sv[3] = p.D[0]; sv[4] = p.D[1]; sv[5] = p.D[2];
      sv[6] = p.t; sv[7] = p.e; sv[8] = p.nu;
    }
  }
  free(da.acc); free(da.touched); free(da.rho); free(da.rmark); free(da.rtouched);
  finish_step(o, dt, n_emit, nesc);
  o->step++;
  if (st) {
    memset(st, 0, sizeof *st);
    st->n_packets = n_emit; st->n_escaped = nesc; st->n_absorbed = nabs; st->n_stopped = nstop;
    st->n_segments = nseg; st->n_scatters = nscat;
  }
  return SED_OK;
}

int oracle_diff_vjp(oracle_ctx* o, const double* grad_flux, double* grad_scale, sed_step_stats* st)
{
  if (!o || !grad_flux || !grad_scale) return SED_ERR_ARG;
  if (!o->jac) return fail(o, SED_ERR_STATE, "no weighted forward");
  size_t nzb = (size_t)o->nzones * (size_t)o->diff_bands;
  for (size_t q = 0; q < nzb; ++q) grad_scale[q] = 0;
  for (int64_t s = 0; s < o->nspec; ++s) {
    if (grad_flux[s] == 0) continue;
    for (size_t q = 0; q < nzb; ++q) grad_scale[q] += grad_flux[s] * o->jac[(size_t)s * nzb + q];
  }
  if (st) memset(st, 0, sizeof *st);
  return SED_OK;
}

/* d flux / d ln(rho) of each zone, the opacity per unit mass held: both
 * extinctions of the zone scale with its density; the estimator is the
 * pathwise derivative of the absorption weight plus the score of the
 * scattering path (likelihood ratio), per escaped packet */
int oracle_diff_vjp_density(oracle_ctx* o, const double* grad_flux, double* grad_rho, sed_step_stats* st)
{
  if (!o || !grad_flux || !grad_rho) return SED_ERR_ARG;
  if (!o->jac_rho) return fail(o, SED_ERR_STATE, "no weighted forward");
  for (int z = 0; z < o->nzones; ++z) grad_rho[z] = 0;
  for (int64_t s = 0; s < o->nspec; ++s) {
    if (grad_flux[s] == 0) continue;
    for (int z = 0; z < o->nzones; ++z) grad_rho[z] += grad_flux[s] * o->jac_rho[(size_t)s * o->nzones + z];
  }
  if (st) memset(st, 0, sizeof *st);
  return SED_OK;
}

int oracle_diff_jacobian(oracle_ctx* o, double* jac, sed_step_stats* st)
{
  if (!o || !jac) return SED_ERR_ARG;
  if (!o->jac) return fail(o, SED_ERR_STATE, "no weighted forward");
  memcpy(jac, o->jac, (size_t)o->jac_n * sizeof(double));
  if (st) memset(st, 0, sizeof *st);
  return SED_OK;
}

/* ---------------------------------------------------------------- temperature
 * transport::solve_eq_temperature (src/transport/solve_equilibrium.cpp:66-96)
 * for LTE: per zone temp_brent_method (:227-320) on rad_eq_function_LTE with
 * solve_flag 0 (:113-170): the emission sum_i 4 pi kappa_abs B_nu(T) dnu with
 * the tables of the last set_opacity, minus the zone's normalised e_abs.
 * set_Tgas_to_Trad: T = (e_rad / a)^(1/4) (:72-74). */
static double blackbody_nu(double T, double nu)  /* transport_opacity.cpp:322-326 */
{
  double zeta = PC_H * nu / PC_K / T;
  return 2.0 * nu * nu * nu * PC_H / PC_C / PC_C / (exp(zeta) - 1);
}

static double rad_eq_lte(const oracle_ctx* o, int c, double T)
{
  int nn = o->nu.n;
  double E_emitted = 0.;
  double E_absorbed = o->e_abs[c];
  if (nn == 1) {
    E_emitted = 4.0 * PC_PI * o->abs[c] * PC_SB / PC_PI * pow(T, 4);
  } else {
    for (int i = 0; i < nn; i++) {
      double dnu = lg_delta(&o->nu, i);
      double nu = lg_center(&o->nu, i);
      double B_nu = blackbody_nu(T, nu);
      double kappa_abs = o->abs[(size_t)c * nn + i];
      E_emitted += 4.0 * PC_PI * kappa_abs * B_nu * dnu;
    }
  }
  return (E_emitted - E_absorbed);
}

#define ORACLE_SIGN(a, b) ((b) >= 0.0 ? fabs(a) : -fabs(a))
static double temp_brent(const oracle_ctx* o, int cell, int* failed)
{
  double brent_solve_tolerance = 1.0e-2;
  int ITMAX = 100;
  double EPS = 3.0e-8;
  double a = o->op.temp_min, b = o->op.temp_max, c = b, d = 0, e = 0, min1, min2;
  double fa = rad_eq_lte(o, cell, a), fb = rad_eq_lte(o, cell, b);
  double fc, p, q, r, s, tol1, xm;
  fc = fb;
  for (int iter = 1; iter <= ITMAX; iter++) {
    if ((fb > 0.0 && fc > 0.0) || (fb < 0.0 && fc < 0.0)) { c = a; fc = fa; e = d = b - a; }
    if (fabs(fc) < fabs(fb)) { a = b; b = c; c = a; fa = fb; fb = fc; fc = fa; }
    tol1 = 2.0 * EPS * fabs(b) + 0.5 * brent_solve_tolerance;
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
    if (fabs(d) > tol1) b += d;
    else b += ORACLE_SIGN(tol1, xm);
    fb = rad_eq_lte(o, cell, b);
  }
  (*failed)++;
  return 0.0;  /* "Maximum number of iterations exceeded in zbrent" */
}

int oracle_solve_temperature(oracle_ctx* o, int32_t set_Tgas_to_Trad, double* T_gas, int32_t* n_unsolved)
{
  if (!o || !o->have_grid) return SED_ERR_STATE;
  if (!o->have_opacity) return fail(o, SED_ERR_STATE, "opacity tables not set");
  int failed = 0;
  for (int i = 0; i < o->nzones; i++) {
    if (set_Tgas_to_Trad) o->T[i] = pow(o->e_rad[i] / PC_A, 0.25);
    else o->T[i] = temp_brent(o, i, &failed);
  }
  if (T_gas) memcpy(T_gas, o->T, (size_t)o->nzones * sizeof(double));
  if (n_unsolved) *n_unsolved = failed;
  return SED_OK;
}

int oracle_get_spectrum(oracle_ctx* o, double* flux, double* click)
{
  if (!o) return SED_ERR_ARG;
  if (flux) memcpy(flux, o->flux, (size_t)o->nspec * sizeof(double));
  if (click) memcpy(click, o->click, (size_t)o->nspec * sizeof(double));
  return SED_OK;
}

int oracle_get_zone_tallies(oracle_ctx* o, double* J, double* e_abs, double* e_rad, double* fx, double* fy, double* fz, double* fr)
{
  if (!o || !o->have_grid) return SED_ERR_STATE;
  size_t nz = (size_t)o->nzones, nj = o->tp.store_Jnu ? (size_t)o->nu.n : 1;
  if (J) memcpy(J, o->J, nz * nj * sizeof(double));
  if (e_abs) memcpy(e_abs, o->e_abs, nz * sizeof(double));
  if (e_rad) memcpy(e_rad, o->e_rad, nz * sizeof(double));
  if (fx) memcpy(fx, o->fx, nz * sizeof(double));
  if (fy) memcpy(fy, o->fy, nz * sizeof(double));
  if (fz) memcpy(fz, o->fz, nz * sizeof(double));
  if (fr) memcpy(fr, o->fr, nz * sizeof(double));
  return SED_OK;
}

int oracle_get_opacity(oracle_ctx* o, double* abs, double* scat, double* cdf, double* n_elec, double* eps_imc,
                       double* planck, double* ross, double* L_th)
{
  if (!o || !o->have_grid) return SED_ERR_STATE;
  size_t nz = (size_t)o->nzones, n = nz * (size_t)o->nu.n;
  if (abs) memcpy(abs, o->abs, n * sizeof(double));
  if (scat) memcpy(scat, o->scat, n * sizeof(double));
  if (cdf) memcpy(cdf, o->cdf, n * sizeof(double));
  if (n_elec) memcpy(n_elec, o->n_elec, nz * sizeof(double));
  if (eps_imc) memcpy(eps_imc, o->eps_imc, nz * sizeof(double));
  if (planck) memcpy(planck, o->planck, nz * sizeof(double));
  if (ross) memcpy(ross, o->ross, nz * sizeof(double));
  if (L_th) memcpy(L_th, o->L_th, nz * sizeof(double));
  return SED_OK;
}

int oracle_record_packets(oracle_ctx* o, int32_t enable)
{
  if (!o) return SED_ERR_ARG;
  o->record = enable;
  return SED_OK;
}

int oracle_get_packet_records(oracle_ctx* o, int64_t n, int32_t* fate, int32_t* ind, int32_t* draws, double* state9)
{
  if (!o || !o->record || n > o->nrec) return SED_ERR_STATE;
  if (fate) memcpy(fate, o->r_fate, (size_t)n * 4);
  if (ind) memcpy(ind, o->r_ind, (size_t)n * 4);
  if (draws) memcpy(draws, o->r_draws, (size_t)n * 4);
  if (state9) memcpy(state9, o->r_state, (size_t)n * 9 * 8);
  return SED_OK;
}

const char* oracle_last_error(oracle_ctx* o) { return o ? o->err : "null context"; }

void oracle_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) { oracle_philox4x32_10(ctr, key, out); }
double oracle_uniform(uint32_t seed, uint64_t pid, uint32_t step, uint32_t n) { return oracle_packet_uniform(seed, pid, step, n); }

void oracle_ctx_destroy(oracle_ctx* o)
{
  if (!o) return;
  free_grid(o);
  free(o->nu.x); free(o->st.x); free(o->sn.x); free(o->sm.x); free(o->sp.x);
  free(o->flux); free(o->click); free(o->core_cdf);
  free(o->r_fate); free(o->r_ind); free(o->r_draws); free(o->r_state);
  if (o->have_atoms) {
    free(o->ion_off); free(o->lev_off); free(o->lev_ion); free(o->lev_g); free(o->lev_ic); free(o->photo_off);
    free(o->line_off); free(o->line_l); free(o->line_u); free(o->line_bin); free(o->ion_chi); free(o->lev_E);
    free(o->lev_Eion); free(o->photo_E); free(o->photo_s); free(o->line_nu); free(o->line_f);
    free(o->fuzz_off); free(o->fuzz_ion); free(o->fuzz_bin); free(o->fuzz_nu); free(o->fuzz_gf); free(o->fuzz_El);
  }
  free(o->zero_eps);
  free(o->jac);
  free(o->gflux); free(o->gclick); free(o->L_emit); free(o->L_dep); free(o->radio_cdf); free(o->gamma_frac);
  free(o->compton); free(o->photoion); free(o->gn.x);
  free(o->c_state); free(o->c_ind); free(o->c_type); free(o->r_type);
  free(o->jac_rho);
  free(o);
}
