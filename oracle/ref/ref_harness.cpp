// oracle/ref/ref_harness.cpp -- TEST INFRASTRUCTURE (oracle harness only).
//
// Drives the reference's own `transport` class (src/transport/transport.h)
// built from its unchanged sources.  Three modes:
//
//   replay   one transport step that follows transport::step
//            (src/transport/transport.cpp:26-140) call for call, except that
//            before each packet the Philox stand-in for the GSL generator is
//            pointed at that packet's (seed, packet id, step) stream.  The
//            reference therefore consumes exactly the uniform deviates the
//            CUDA packet kernel consumes, and per-packet outcomes (fate, zone,
//            number of deviates drawn, final phase-space state) can be
//            compared one for one.
//   free     transport::step itself, OpenMP threads, free-running streams;
//            prints the wall time of each step (the timed CPU baseline).
//   opacity  transport::init + set_opacity only; dumps the opacity tables.
//   gpu      (sedona_ref_gpu only, built with SED_GPU_BINDING) transport::init,
//            then the steps run by the compiled C++ binding of the B200
//            library (pubsed_b200/binding/transport_gpu.cpp): the binding
//            fills the C ABI's structs from the live transport, steps on the
//            device and copies the results back into the transport, whose
//            tables and tallies are then dumped as in the other modes.
//
// Inputs: a Lua parameter file (read by the reference's ParameterReader),
// the model file it names, and optionally a "store" file whose datasets and
// attributes are served through the HDF5 stand-in (synthetic atomic data,
// fuzz line lists, 3-D Cartesian models).
//
// Outputs: raw little-endian arrays <out>.<name>.f64 / .i32 / .i64 plus
// <out>.meta.json describing them.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <limits>
#include <list>
#include <sstream>
#include <string>
#include <vector>
#include <omp.h>

#include "hdf5.h"
#include "hdf5_hl.h"
#include "shims_control.h"

#define private public
#define protected public
#include "transport.h"
#include "radioactive.h"
#include "hydro_homologous.h"
#include "grid_1D_sphere.h"
#include "grid_3D_cart.h"
#include "ParameterReader.h"
#include "physical_constants.h"
#undef private
#undef protected
#ifdef SED_GPU_BINDING
#include "transport_gpu.h"
#endif

namespace pc = physical_constants;

namespace {

struct Out {
  std::string prefix;
  std::string sfx;  // appended to array and scalar names (one set per replayed step)
  std::ostringstream meta;
  bool first = true;
  void arr(const std::string& name0, const void* p, size_t bytes, const char* ext, size_t count)
  {
    const std::string name = name0 + sfx;
    std::string fn = prefix + "." + name + "." + ext;
    FILE* f = std::fopen(fn.c_str(), "wb");
    if (!f) { std::perror(fn.c_str()); std::exit(2); }
    if (bytes) std::fwrite(p, 1, bytes, f);
    std::fclose(f);
    meta << (first ? "" : ",") << "\n  \"" << name << "\": {\"file\": \"" << fn << "\", \"type\": \"" << ext
         << "\", \"count\": " << count << "}";
    first = false;
  }
  void f64(const std::string& n, const std::vector<double>& v) { arr(n, v.data(), v.size() * 8, "f64", v.size()); }
  void i32(const std::string& n, const std::vector<int32_t>& v) { arr(n, v.data(), v.size() * 4, "i32", v.size()); }
  void i64(const std::string& n, const std::vector<int64_t>& v) { arr(n, v.data(), v.size() * 8, "i64", v.size()); }
  std::ostringstream scalars;
  bool sfirst = true;
  void scalar(const std::string& n, double v)
  {
    char buf[64];
    std::snprintf(buf, sizeof buf, "%.17g", v);
    scalars << (sfirst ? "" : ", ") << "\"" << n << sfx << "\": " << buf;
    sfirst = false;
  }
  void finish()
  {
    std::string fn = prefix + ".meta.json";
    std::ofstream f(fn);
    f << "{\"arrays\": {" << meta.str() << "\n},\n \"scalars\": {" << scalars.str() << "}}\n";
  }
};

// Store file: sequence of records
//   u8 kind (0 = f64 dataset, 1 = i32 dataset, 2 = i32 attribute)
//   u32 n + bytes: file name;  u32 n + bytes: object path
//   kind 2: u32 n + bytes attribute name; i32 value
//   kind 0/1: u32 rank; u64 dims[rank]; u64 count; payload
void load_store(const char* path)
{
  FILE* f = std::fopen(path, "rb");
  if (!f) { std::perror(path); std::exit(2); }
  auto rd = [&](void* p, size_t n) { if (std::fread(p, 1, n, f) != n) { std::fprintf(stderr, "truncated store\n"); std::exit(2); } };
  auto rstr = [&]() { uint32_t n; rd(&n, 4); std::string s(n, '\0'); if (n) rd(&s[0], n); return s; };
  for (;;) {
    uint8_t kind;
    if (std::fread(&kind, 1, 1, f) != 1) break;
    std::string file = rstr(), obj = rstr();
    if (kind == 2) {
      std::string attr = rstr();
      int32_t v; rd(&v, 4);
      oracle_h5_put_attr_int(file.c_str(), obj.c_str(), attr.c_str(), v);
      continue;
    }
    uint32_t rank; rd(&rank, 4);
    std::vector<hsize_t> dims(rank);
    for (uint32_t k = 0; k < rank; ++k) { uint64_t d; rd(&d, 8); dims[k] = d; }
    uint64_t n; rd(&n, 8);
    if (kind == 0) {
      std::vector<double> v(n); if (n) rd(v.data(), n * 8);
      oracle_h5_put_double(file.c_str(), obj.c_str(), v.data(), n, (int)rank, dims.data());
    } else {
      std::vector<int32_t> v(n); if (n) rd(v.data(), n * 4);
      oracle_h5_put_int(file.c_str(), obj.c_str(), v.data(), n, (int)rank, dims.data());
    }
  }
  std::fclose(f);
}

double now() { return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); }

// number of deviates emit_inner_source takes per packet (src/transport/emission.cpp:399-473)
uint32_t core_draws_per_packet(transport& t)
{
  uint32_t k = (t.r_core_ == 0) ? 2 : 4;  // direction (and position on the core)
  if (!(t.core_frequency_ > 0)) k += 2;    // frequency bin + position in bin
  return k + 1;                            // emission time
}

void dump_tables(transport& t, Out& o)
{
  grid_general* g = t.grid;
  int nz = g->n_zones, nn = t.nu_grid_.size();
  std::vector<double> ab((size_t)nz * nn), sc((size_t)nz * nn, 0.0), em((size_t)nz * nn), j((size_t)nz * (t.store_Jnu_ ? nn : 1));
  for (int i = 0; i < nz; ++i) {
    for (int k = 0; k < nn; ++k) {
      ab[(size_t)i * nn + k] = t.abs_opacity_[i][k];
      if (!t.omit_scattering_) sc[(size_t)i * nn + k] = t.scat_opacity_[i][k];
      em[(size_t)i * nn + k] = t.emissivity_[i].get(k);
    }
    for (size_t k = 0; k < t.J_nu_[i].size(); ++k) j[(size_t)i * t.J_nu_[i].size() + k] = t.J_nu_[i][k];
  }
  std::vector<double> ne(nz), pm(nz), rm(nz), lth(nz), epsimc(nz), eabs(nz), erad(nz), fx(nz), fy(nz), fz(nz), fr(nz), tg(nz);
  for (int i = 0; i < nz; ++i) {
    ne[i] = g->z[i].n_elec; pm[i] = t.planck_mean_opacity_[i]; rm[i] = t.rosseland_mean_opacity_[i];
    lth[i] = g->z[i].L_thermal; epsimc[i] = g->z[i].eps_imc; eabs[i] = g->z[i].e_abs; erad[i] = g->z[i].e_rad;
    fx[i] = g->z[i].fx_rad; fy[i] = g->z[i].fy_rad; fz[i] = g->z[i].fz_rad; fr[i] = g->z[i].fr_rad; tg[i] = g->z[i].T_gas;
  }
  std::vector<double> nu(nn), nul(nn);
  for (int k = 0; k < nn; ++k) { nu[k] = t.nu_grid_[k]; nul[k] = t.nu_grid_.left(k); }
  o.f64("abs", ab); o.f64("scat", sc); o.f64("emis_cdf", em); o.f64("J_nu", j);
  o.f64("n_elec", ne); o.f64("planck_mean", pm); o.f64("rosseland_mean", rm); o.f64("L_thermal", lth);
  o.f64("eps_imc", epsimc); o.f64("e_abs", eabs); o.f64("e_rad", erad);
  o.f64("fx_rad", fx); o.f64("fy_rad", fy); o.f64("fz_rad", fz); o.f64("fr_rad", fr); o.f64("T_gas", tg);
  o.f64("nu_right", nu); o.f64("nu_left", nul);
  o.f64("spec_flux", t.optical_spectrum.flux);
  o.f64("spec_click", t.optical_spectrum.click);
  o.scalar("n_zones", nz); o.scalar("n_nu", nn); o.scalar("t_now", t.t_now_);
  o.scalar("spec_n_t", t.optical_spectrum.time_grid.size());
  o.scalar("spec_n_nu", t.optical_spectrum.wave_grid.size());
  o.scalar("spec_n_mu", t.optical_spectrum.mu_grid.size());
  o.scalar("spec_n_phi", t.optical_spectrum.phi_grid.size());
}

// Per-packet deviate counts of an emission that starts with the radioactive
// packets (transport::emit_radioactive, src/transport/emission.cpp:165-243):
// zone, time, gamma-ray or positron, three for the position, two for the
// direction, and two more for an optical photon's frequency; each core
// packet then takes K.  The gamma-ray fraction of the sampled zone comes
// from the reference's own radioactive::decay and zone_emission_cdf_.
struct RadioWalk {
  transport* t;
  int64_t n_radio;
  uint32_t K;
  std::vector<double> gfrac;
  std::vector<uint32_t> counts;
};

uint32_t radio_walk_count(void* user, uint64_t k, const double* u, uint32_t n)
{
  RadioWalk* w = static_cast<RadioWalk*>(user);
  uint32_t total = 0;
  if ((int64_t)k >= w->n_radio) total = w->K;
  else if (n >= 3) total = (u[2] < w->gfrac[w->t->zone_emission_cdf_.sample(u[0])]) ? 8u : 10u;
  if (total != 0 && n == total && (int64_t)k < w->n_radio) w->counts.push_back(total);
  return total;
}

// transport::step (src/transport/transport.cpp:26-140) with per-packet
// stream selection; returns the number of escaped packets
int replay_step(transport& t, double dt, uint32_t seed, uint32_t step, Out& o, int threads)
{
  if (t.steady_state) dt = 1;
  t.set_opacity(dt);
  t.reduce_opacities();
  t.reduce_Lthermal();
  if (t.use_ddmc_) t.compute_diffusion_probabilities(dt);
  t.wipe_radiation();

  // the packets the last step left (the census) keep the front of the
  // vector; emission appends after them
  const size_t n_before = t.particles.size();
  const uint32_t K = core_draws_per_packet(t);
  const int64_t n_radio_req = t.params_->getScalar<int>("particles_n_emit_radioactive");
  RadioWalk walk;
  walk.t = &t;
  walk.n_radio = 0;
  walk.K = K;
  if (n_radio_req > 0) {
    // emit_radioactive's first deviate (the remainder test, emission.cpp:
    // 187-189) comes from a stream no packet uses
    radioactive radio;
    const int force = t.params_->getScalar<int>("force_rprocess_heating");
    for (int i = 0; i < t.grid->n_zones; ++i) {
      double gf = 0;
      radio.decay(t.grid->elems_Z, t.grid->elems_A, t.grid->z[i].X_gas, t.t_now_, &gf, force);
      walk.gfrac.push_back(gf);
    }
    walk.n_radio = n_radio_req;
    oracle_rng_walk(seed, n_before, step, 1, radio_walk_count, &walk);
  } else {
    oracle_rng_emission(seed, n_before, step, K);
  }
  t.emit_particles(dt);
  const size_t n = t.particles.size();
  uint64_t radio_draws = 0;
  if (n_radio_req > 0) {
    if ((int64_t)walk.counts.size() != n_radio_req) {
      std::fprintf(stderr, "replay: %zu radioactive packets emitted, %lld requested\n", walk.counts.size(),
                   (long long)n_radio_req);
      std::exit(3);
    }
    radio_draws = 1;
    for (uint32_t c : walk.counts) radio_draws += c;
  }
  const size_t n_core = n - n_before - walk.counts.size();
  const size_t n_q = n_before + walk.counts.size();  // census + radioactive: the queued packets
  if (oracle_rng_emission_draws() != radio_draws + (uint64_t)K * n_core) {
    std::fprintf(stderr, "replay: emission drew %llu deviates for %zu packets (expected %u each); only core emission is replayable\n",
                 (unsigned long long)oracle_rng_emission_draws(), n, K);
    std::exit(3);
  }

  std::vector<int32_t> fate(n), ind(n), draws(n), ptype(n), spec_bin(n, -1);
  std::vector<double> st((size_t)n * 9);
  const double T0 = now();
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads)
  for (long i = 0; i < (long)n; ++i) {
    particle& p = t.particles[i];
    // census packets draw this step's stream from its start; radioactive
    // packets keep drawing from where their emission stopped; both record
    // all their deviates, core packets the ones after emission.  Records
    // list the core packets first, then the queued (census, radioactive) ones.
    const bool queued = i < (long)n_q;
    const uint32_t n0 = i < (long)n_before ? 0u : (queued ? walk.counts[i - n_before] : K);
    oracle_rng_packet(seed, (uint64_t)i, step, n0);
    p.fate = t.propagate(p, dt);
    const long r = queued ? (long)n_core + i : i - (long)n_q;
    draws[r] = (int32_t)(oracle_rng_packet_draws() - (queued ? 0 : K));
    if (p.fate == escaped) {
      double t_obs = p.t - p.x_dot_d() / pc::c;
      if (p.type == photon) t.optical_spectrum.count(t_obs, p.nu, p.e, p.D);
      if (p.type == gammaray) t.gamma_spectrum.count(t_obs, p.nu, p.e, p.D);
      p.t = t_obs;
    }
    fate[r] = (int32_t)p.fate; ind[r] = p.ind; ptype[r] = (int32_t)p.type;
    double* s = &st[(size_t)r * 9];
    s[0] = p.x[0]; s[1] = p.x[1]; s[2] = p.x[2]; s[3] = p.D[0]; s[4] = p.D[1]; s[5] = p.D[2];
    s[6] = p.t; s[7] = p.e; s[8] = p.nu;
  }
  const double T1 = now();
  int n_escaped = t.clean_up_particle_vector();
  if (t.steady_state && t.core_fix_luminosity_) {
    double per_esc = (1.0 * n_escaped) / (1.0 * n);
    double fac = 1.0 / per_esc;
    t.optical_spectrum.rescale(fac);
    for (int i = 0; i < t.grid->n_zones; ++i) {
      t.grid->z[i].e_rad *= fac;
      if (t.store_Jnu_)
        for (size_t j = 0; j < (size_t)t.nu_grid_.size(); ++j) t.J_nu_[i][j] *= fac;
    }
  }
  t.reduce_radiation(dt);
  // the temperature solve transport::step runs next (transport.cpp:126-132);
  // dump_tables then records the solved T_gas
  if (t.radiative_eq == 1 && t.fix_Tgas_during_transport_ == 0 && t.solve_Tgas_with_updated_opacities_ == 0)
    t.solve_eq_temperature();
  // advance time step (transport.cpp:136) and record the packets carried on
  if (!t.steady_state) t.t_now_ += dt;
  if (!t.steady_state) {
    const size_t nc = t.particles.size();
    std::vector<int32_t> cind(nc), ctype(nc);
    std::vector<double> cst(nc * 9);
    for (size_t k = 0; k < nc; ++k) {
      const particle& p = t.particles[k];
      cind[k] = p.ind; ctype[k] = (int32_t)p.type;
      double* s = &cst[k * 9];
      s[0] = p.x[0]; s[1] = p.x[1]; s[2] = p.x[2]; s[3] = p.D[0]; s[4] = p.D[1]; s[5] = p.D[2];
      s[6] = p.t; s[7] = p.e; s[8] = p.nu;
    }
    o.i32("census_ind", cind); o.i32("census_type", ctype); o.f64("census_state", cst);
    o.scalar("n_census_before", (double)n_before);
  }
  o.i32("pkt_fate", fate); o.i32("pkt_ind", ind); o.i32("pkt_draws", draws); o.f64("pkt_state", st);
  if (!t.steady_state) o.i32("pkt_type", ptype);
  o.scalar("n_packets", (double)n); o.scalar("n_escaped", n_escaped); o.scalar("propagate_seconds", T1 - T0);
  o.scalar("draws_per_emitted_packet", K);
  if (n_radio_req > 0) {
    std::vector<double> le(t.grid->n_zones), ld(t.grid->n_zones);
    for (int i = 0; i < t.grid->n_zones; ++i) { le[i] = t.grid->z[i].L_radio_emit; ld[i] = t.grid->z[i].L_radio_dep; }
    o.f64("L_radio_emit", le); o.f64("L_radio_dep", ld);
    o.f64("gamma_flux", t.gamma_spectrum.flux); o.f64("gamma_click", t.gamma_spectrum.click);
    o.scalar("n_radioactive", (double)walk.counts.size());
  }
  return n_escaped;
}

void usage()
{
  std::fprintf(stderr,
               "usage: sedona_ref <replay|free|opacity|gpu> <param.lua> <out_prefix> [--store FILE] [--seed S]\n"
               "                  [--step N] [--steps N] [--threads T] [--dt DT] [--precision P]\n");
  std::exit(1);
}
}  // namespace

int main(int argc, char** argv)
{
  if (argc < 4) usage();
  std::string mode = argv[1], pfile = argv[2];
  Out o;
  o.prefix = argv[3];
  uint32_t seed = 0, step = 0;
  int steps = 1, threads = omp_get_max_threads(), precision = 0;
  double dt = 1.0;
  for (int a = 4; a < argc; ++a) {
    std::string k = argv[a];
    if (a + 1 >= argc) usage();
    std::string v = argv[++a];
    if (k == "--store") load_store(v.c_str());
    else if (k == "--seed") seed = (uint32_t)std::stoul(v);
    else if (k == "--step") step = (uint32_t)std::stoul(v);
    else if (k == "--steps") steps = std::stoi(v);
    else if (k == "--threads") threads = std::stoi(v);
    else if (k == "--dt") dt = std::stod(v);
    else if (k == "--precision") precision = std::stoi(v);
    else usage();
  }
  omp_set_num_threads(threads);

  ParameterReader params(pfile, 0);
  std::string grid_type = params.getScalar<std::string>("grid_type");
  grid_general* grid = nullptr;
  if (grid_type == "grid_1D_sphere") grid = new grid_1D_sphere;
  else if (grid_type == "grid_3D_cart") grid = new grid_3D_cart;
  else { std::fprintf(stderr, "unsupported grid_type %s\n", grid_type.c_str()); return 3; }
  grid->init(&params);

  transport t;
  // initialize_particles (called by transport::init) draws 8 deviates per
  // packet: packet k from stream k at step number 0xFFFFFFFF
  const int n_init = params.getScalar<int>("particles_n_initialize");
  if (n_init > 0) oracle_rng_emission(seed, 0, 0xFFFFFFFFu, 8);
  const double Ti0 = now();
  t.init(&params, grid);
  const double Ti1 = now();
  if (n_init > 0 && oracle_rng_emission_draws() != 8ull * (uint64_t)t.particles.size()) {
    std::fprintf(stderr, "replay: initialisation drew %llu deviates for %zu packets\n",
                 (unsigned long long)oracle_rng_emission_draws(), t.particles.size());
    return 3;
  }
  oracle_rng_free_running();
  o.scalar("init_seconds", Ti1 - Ti0);
  o.scalar("threads", threads);

  if (mode == "opacity") {
    double dtt = t.steady_state ? 1.0 : dt;
    const double T0 = now();
    t.set_opacity(dtt);
    const double T1 = now();
    t.reduce_opacities();
    o.scalar("set_opacity_seconds", T1 - T0);
    dump_tables(t, o);
  } else if (mode == "replay") {
    // time-dependent runs: the driver's homologous hydro step moves the grid
    // to t + dt before each transport step (SedonaClass.cpp:346-358)
    hydro_homologous hydro;
    const bool use_hydro = !t.steady_state && params.getScalar<std::string>("hydro_module") == "homologous";
    if (use_hydro) hydro.init(&params, grid);
    if (n_init > 0) {
      std::vector<int32_t> cind, ctype;
      std::vector<double> cst;
      for (const particle& p : t.particles) {
        cind.push_back(p.ind); ctype.push_back((int32_t)p.type);
        const double v[9] = {p.x[0], p.x[1], p.x[2], p.D[0], p.D[1], p.D[2], p.t, p.e, p.nu};
        cst.insert(cst.end(), v, v + 9);
      }
      o.i32("init_ind", cind); o.i32("init_type", ctype); o.f64("init_state", cst);
    }
    for (int s = 0; s < steps; ++s) {
      o.sfx = steps > 1 ? "_s" + std::to_string(s) : "";
      if (use_hydro) hydro.step(dt);
      replay_step(t, dt, seed, step + (uint32_t)s, o, threads);
      if (steps > 1) dump_tables(t, o);
    }
    o.sfx = "";
    dump_tables(t, o);
    // the reference's own text outputs of this step: spectrum_array::print
    // (<prefix>_spectrum.dat) and, for 1D spheres, grid_1D_sphere::
    // write_plotfile (plt_00001.dat in the working directory); their HDF5
    // halves go to the stand-in, which writes nothing
    t.optical_spectrum.set_name(o.prefix + "_spectrum");
    t.optical_spectrum.print(0);
    if (params.getScalar<int>("particles_n_emit_radioactive") > 0) {
      t.gamma_spectrum.set_name(o.prefix + "_gamma");
      t.gamma_spectrum.print(0);
    }
    if (grid_type == "grid_1D_sphere") grid->write_plotfile(1, t.t_now_, 0);
  } else if (mode == "free") {
    oracle_rng_free_running();
    std::vector<double> times, opac_times;
    for (int s = 0; s < steps; ++s) {
      const double T0 = now();
      t.step(dt);
      const double T1 = now();
      times.push_back(T1 - T0);
    }
    // separately time the opacity build alone (set_opacity is the first phase of step)
    const double T2 = now();
    t.set_opacity(t.steady_state ? 1.0 : dt);
    const double T3 = now();
    opac_times.push_back(T3 - T2);
    o.f64("step_seconds", times);
    o.f64("set_opacity_seconds", opac_times);
    dump_tables(t, o);
  } else if (mode == "gpu") {
#ifdef SED_GPU_BINDING
    hydro_homologous hydro;
    const bool use_hydro = !t.steady_state && params.getScalar<std::string>("hydro_module") == "homologous";
    if (use_hydro) hydro.init(&params, grid);
    sed_binding::GpuTransport* b = sed_binding::attach(t, &params, precision, 0);
    if (!b) { std::fprintf(stderr, "gpu: %s\n", sed_binding::last_error(nullptr)); return 5; }
    std::vector<double> esc;
    for (int s = 0; s < steps; ++s) {
      if (use_hydro) hydro.step(dt);
      sed_step_stats st{};
      const int rc = sed_binding::step(t, b, dt, &st);
      if (rc) { std::fprintf(stderr, "gpu: step %d: %s\n", s, sed_binding::last_error(b)); return 6; }
      esc.push_back((double)st.n_escaped);
    }
    o.f64("n_escaped_steps", esc);
    dump_tables(t, o);
    sed_binding::detach(b);
#else
    (void)precision;
    std::fprintf(stderr, "gpu mode needs the sedona_ref_gpu build\n");
    return 4;
#endif
  } else {
    usage();
  }
  o.finish();
  return 0;
}
