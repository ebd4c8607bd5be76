// oracle/ref/shims.cpp -- TEST INFRASTRUCTURE (oracle harness only).
//
// Link-time stand-ins that let the reference's own transport, grid and
// opacity sources build and run on a machine without MPI, GSL or HDF5:
//  * MPI: one rank; collectives copy their send buffer.
//  * GSL RNG: Philox4x32-10 (oracle/philox.h).  In replay mode the harness
//    selects the (seed, packet, step) stream before each packet so the
//    reference consumes exactly the deviates the GPU kernel consumes.
//  * HDF5: an in-memory store of datasets/attributes filled by the harness.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <chrono>
#include <map>
#include <string>
#include <vector>

#include "mpi.h"
#include "gsl/gsl_rng.h"
#include "gsl/gsl_vector.h"
#include "hdf5.h"
#include "hdf5_hl.h"
#include "shims_control.h"
#include "../philox.h"

// ------------------------------------------------------------------ MPI
extern "C" {
int MPI_Init(int*, char***) { return 0; }
int MPI_Finalize(void) { return 0; }
int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return 0; }
int MPI_Barrier(MPI_Comm) { return 0; }
static size_t mpi_size(MPI_Datatype t)
{
  switch (t) {
    case MPI_INT: return sizeof(int);
    case MPI_DOUBLE: return sizeof(double);
    case MPI_FLOAT: return sizeof(float);
    case MPI_CHAR: return 1;
    default: return sizeof(long);
  }
}
int MPI_Allreduce(const void* s, void* d, int n, MPI_Datatype t, MPI_Op, MPI_Comm)
{
  if (s != MPI_IN_PLACE && s != d) std::memmove(d, s, (size_t)n * mpi_size(t));
  return 0;
}
int MPI_Reduce(const void* s, void* d, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm)
{
  if (s != MPI_IN_PLACE && s != d && d) std::memmove(d, s, (size_t)n * mpi_size(t));
  return 0;
}
int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return 0; }
int MPI_Scatter(const void* s, int sc, MPI_Datatype st, void* d, int, MPI_Datatype, int, MPI_Comm)
{
  if (s != d && d && s) std::memmove(d, s, (size_t)sc * mpi_size(st));
  return 0;
}
int MPI_Gather(const void* s, int sc, MPI_Datatype st, void* d, int, MPI_Datatype, int, MPI_Comm)
{
  if (s != d && d && s) std::memmove(d, s, (size_t)sc * mpi_size(st));
  return 0;
}
double MPI_Wtime(void)
{
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}
}

// ------------------------------------------------------------------ RNG
namespace {
enum RngMode { FREE = 0, PACKET = 1, EMIT = 2, WALK = 3 };
struct RngThreadState {
  int mode = FREE;
  uint32_t seed = 0;
  uint64_t pid = 0;
  uint32_t step = 0;
  uint32_t n = 0;          // next draw index of the current packet
  uint64_t emit_base = 0;  // first packet id of an emission batch
  uint32_t emit_k = 1;     // draws per emitted packet
  uint64_t emit_g = 0;     // draws taken in the current emission batch
  // WALK: per-packet draw counts decided by the harness as the draws come
  uint32_t walk_prefix = 0;  // draws served before the first packet
  uint64_t walk_pkt = 0;     // current packet, relative to emit_base
  double walk_u[32];         // the current packet's draws so far
  oracle_rng_count_fn walk_fn = nullptr;
  void* walk_user = nullptr;
};
thread_local RngThreadState g_rng;
const gsl_rng_type g_type = {"philox4x32_10"};
}

extern "C" {
const gsl_rng_type* gsl_rng_default = &g_type;
unsigned long gsl_rng_default_seed = 0;
const gsl_rng_type* gsl_rng_env_setup(void) { return &g_type; }
gsl_rng* gsl_rng_alloc(const gsl_rng_type* T)
{
  gsl_rng* r = (gsl_rng*)std::calloc(1, sizeof(gsl_rng));
  r->type = T;
  r->state = &r->seed;
  return r;
}
void gsl_rng_free(gsl_rng* r) { std::free(r); }
void gsl_rng_set(const gsl_rng* rc, unsigned long seed)
{
  gsl_rng* r = const_cast<gsl_rng*>(rc);
  r->seed = seed;
  r->n = 0;
}
static double free_uniform(gsl_rng* r)
{
  uint64_t n = r->n++;
  uint32_t ctr[4] = {(uint32_t)(n >> 1), (uint32_t)(n >> 33), 0x0F5EEu, 0x0F5EEu};
  uint32_t key[2] = {(uint32_t)r->seed, (uint32_t)((uint64_t)r->seed >> 32)};
  uint32_t w[4];
  oracle_philox4x32_10(ctr, key, w);
  return (n & 1u) ? oracle_u01_from_words(w[2], w[3]) : oracle_u01_from_words(w[0], w[1]);
}
unsigned long gsl_rng_get(const gsl_rng* rc)
{
  gsl_rng* r = const_cast<gsl_rng*>(rc);
  return (unsigned long)(free_uniform(r) * 4294967296.0);
}
double gsl_rng_uniform(const gsl_rng* rc)
{
  RngThreadState& s = g_rng;
  if (s.mode == PACKET) return oracle_packet_uniform(s.seed, s.pid, s.step, s.n++);
  if (s.mode == EMIT) {
    uint64_t g = s.emit_g++;
    return oracle_packet_uniform(s.seed, s.emit_base + g / s.emit_k, s.step, (uint32_t)(g % s.emit_k));
  }
  if (s.mode == WALK) {
    s.emit_g++;
    if (s.walk_prefix > 0) {  // a stream no packet uses
      --s.walk_prefix;
      return oracle_packet_uniform(s.seed, ~0ull, s.step, s.walk_prefix);
    }
    const double u = oracle_packet_uniform(s.seed, s.emit_base + s.walk_pkt, s.step, s.n);
    if (s.n < 32) s.walk_u[s.n] = u;
    ++s.n;
    const uint32_t total = s.walk_fn(s.walk_user, s.walk_pkt, s.walk_u, s.n);
    if (total != 0 && s.n >= total) { ++s.walk_pkt; s.n = 0; }
    return u;
  }
  return free_uniform(const_cast<gsl_rng*>(rc));
}
size_t gsl_rng_size(const gsl_rng*) { return sizeof(unsigned long); }
void* gsl_rng_state(const gsl_rng* r) { return r->state; }

// non-LTE linear algebra is never reached by the harness
static void nlte_unreachable(const char* f)
{
  std::fprintf(stderr, "oracle shim: %s called (non-LTE path is not supported by the harness)\n", f);
  std::abort();
}
gsl_vector* gsl_vector_calloc(size_t) { nlte_unreachable("gsl_vector_calloc"); return nullptr; }
void gsl_vector_set_zero(gsl_vector*) { nlte_unreachable("gsl_vector_set_zero"); }
void gsl_vector_set(gsl_vector*, size_t, double) { nlte_unreachable("gsl_vector_set"); }
double gsl_vector_get(const gsl_vector*, size_t) { nlte_unreachable("gsl_vector_get"); return 0; }
gsl_matrix* gsl_matrix_calloc(size_t, size_t) { nlte_unreachable("gsl_matrix_calloc"); return nullptr; }
void gsl_matrix_set_zero(gsl_matrix*) { nlte_unreachable("gsl_matrix_set_zero"); }
void gsl_matrix_set(gsl_matrix*, size_t, size_t, double) { nlte_unreachable("gsl_matrix_set"); }
double gsl_matrix_get(const gsl_matrix*, size_t, size_t) { nlte_unreachable("gsl_matrix_get"); return 0; }
gsl_permutation* gsl_permutation_alloc(size_t) { nlte_unreachable("gsl_permutation_alloc"); return nullptr; }
void gsl_permutation_init(gsl_permutation*) { nlte_unreachable("gsl_permutation_init"); }
int gsl_linalg_LU_decomp(gsl_matrix*, gsl_permutation*, int*) { nlte_unreachable("gsl_linalg_LU_decomp"); return 0; }
int gsl_linalg_LU_solve(const gsl_matrix*, const gsl_permutation*, const gsl_vector*, gsl_vector*) { nlte_unreachable("gsl_linalg_LU_solve"); return 0; }
}

void oracle_rng_free_running() { g_rng.mode = FREE; }
void oracle_rng_packet(uint32_t seed, uint64_t pid, uint32_t step, uint32_t n0)
{
  g_rng.mode = PACKET;
  g_rng.seed = seed;
  g_rng.pid = pid;
  g_rng.step = step;
  g_rng.n = n0;
}
uint32_t oracle_rng_packet_draws() { return g_rng.n; }
void oracle_rng_emission(uint32_t seed, uint64_t pid_base, uint32_t step, uint32_t draws_per_packet)
{
  g_rng.mode = EMIT;
  g_rng.seed = seed;
  g_rng.step = step;
  g_rng.emit_base = pid_base;
  g_rng.emit_k = draws_per_packet ? draws_per_packet : 1;
  g_rng.emit_g = 0;
}
uint64_t oracle_rng_emission_draws() { return g_rng.emit_g; }
void oracle_rng_walk(uint32_t seed, uint64_t pid_base, uint32_t step, uint32_t n_prefix, oracle_rng_count_fn fn,
                     void* user)
{
  g_rng.mode = WALK;
  g_rng.seed = seed;
  g_rng.step = step;
  g_rng.emit_base = pid_base;
  g_rng.emit_g = 0;
  g_rng.n = 0;
  g_rng.walk_prefix = n_prefix;
  g_rng.walk_pkt = 0;
  g_rng.walk_fn = fn;
  g_rng.walk_user = user;
}

// ------------------------------------------------------------------ HDF5
namespace {
struct Dset {
  bool is_int = false;
  std::vector<double> d;
  std::vector<int> i;
  std::vector<hsize_t> dims;
};
struct H5File {
  std::map<std::string, Dset> dsets;
  std::map<std::string, int> attrs;  // key "obj|attr"
};
std::map<std::string, H5File> g_files;
std::map<hid_t, std::string> g_open;
hid_t g_next = 1000;

std::string norm(const char* p)
{
  std::string s(p ? p : "");
  while (!s.empty() && s[0] == '/') s.erase(0, 1);
  while (!s.empty() && s.back() == '/') s.pop_back();
  std::string out;
  for (size_t k = 0; k < s.size(); ++k) {  // collapse "//"
    if (s[k] == '/' && !out.empty() && out.back() == '/') continue;
    out.push_back(s[k]);
  }
  return out;
}
H5File* file_of(hid_t h)
{
  auto it = g_open.find(h);
  if (it == g_open.end()) return nullptr;
  auto f = g_files.find(it->second);
  return f == g_files.end() ? nullptr : &f->second;
}
const Dset* find(hid_t h, const char* name)
{
  H5File* f = file_of(h);
  if (!f) return nullptr;
  auto it = f->dsets.find(norm(name));
  return it == f->dsets.end() ? nullptr : &it->second;
}
}

extern "C" {
void oracle_h5_clear(void) { g_files.clear(); g_open.clear(); }
void oracle_h5_put_double(const char* file, const char* path, const double* v, size_t n, int rank, const hsize_t* dims)
{
  Dset d;
  d.d.assign(v, v + n);
  if (rank > 0) d.dims.assign(dims, dims + rank); else d.dims.push_back(n);
  g_files[file].dsets[norm(path)] = d;
}
void oracle_h5_put_int(const char* file, const char* path, const int* v, size_t n, int rank, const hsize_t* dims)
{
  Dset d;
  d.is_int = true;
  d.i.assign(v, v + n);
  if (rank > 0) d.dims.assign(dims, dims + rank); else d.dims.push_back(n);
  g_files[file].dsets[norm(path)] = d;
}
void oracle_h5_put_attr_int(const char* file, const char* obj, const char* attr, int v)
{
  g_files[file].attrs[norm(obj) + "|" + attr] = v;
}

hid_t H5Fopen(const char* name, unsigned, hid_t)
{
  if (g_files.find(name) == g_files.end()) return -1;
  hid_t h = g_next++;
  g_open[h] = name;
  return h;
}
hid_t H5Fcreate(const char*, unsigned, hid_t, hid_t) { return g_next++; }
herr_t H5Fclose(hid_t h) { g_open.erase(h); return 0; }
hid_t H5Gopen1(hid_t, const char*) { return g_next++; }
hid_t H5Gopen2(hid_t, const char*, hid_t) { return g_next++; }
hid_t H5Gcreate1(hid_t, const char*, size_t) { return g_next++; }
herr_t H5Gclose(hid_t) { return 0; }
herr_t H5Gget_objinfo(hid_t h, const char* name, int, H5G_stat_t*)
{
  H5File* f = file_of(h);
  if (!f) return -1;
  std::string g = norm(name);
  for (auto& kv : f->dsets)
    if (kv.first.compare(0, g.size() + 1, g + "/") == 0) return 0;
  for (auto& kv : f->attrs)
    if (kv.first.compare(0, g.size() + 1, g + "|") == 0) return 0;
  return -1;
}
hid_t H5Dopen1(hid_t, const char*) { return g_next++; }
hid_t H5Dcreate1(hid_t, const char*, hid_t, hid_t, hid_t) { return g_next++; }
herr_t H5Dclose(hid_t) { return 0; }
herr_t H5Dwrite(hid_t, hid_t, hid_t, hid_t, hid_t, const void*) { return 0; }
herr_t H5Dread(hid_t, hid_t, hid_t, hid_t, hid_t, void*) { return -1; }
hid_t H5Dget_space(hid_t) { return g_next++; }
hid_t H5Screate_simple(int, const hsize_t*, const hsize_t*) { return g_next++; }
herr_t H5Sclose(hid_t) { return 0; }
herr_t H5Sselect_hyperslab(hid_t, H5S_seloper_t, const hsize_t*, const hsize_t*, const hsize_t*, const hsize_t*) { return 0; }
int H5Sget_simple_extent_dims(hid_t, hsize_t*, hsize_t*) { return -1; }
hid_t H5Tcreate(int, size_t) { return g_next++; }
hid_t H5Tcopy(hid_t) { return g_next++; }
herr_t H5Tset_size(hid_t, size_t) { return 0; }
herr_t H5Eset_auto1(void*, void*) { return 0; }

herr_t H5LTread_dataset_double(hid_t h, const char* name, double* buf)
{
  const Dset* d = find(h, name);
  if (!d) return -1;
  if (d->is_int) for (size_t k = 0; k < d->i.size(); ++k) buf[k] = d->i[k];
  else std::memcpy(buf, d->d.data(), d->d.size() * sizeof(double));
  return 0;
}
herr_t H5LTread_dataset_float(hid_t h, const char* name, float* buf)
{
  const Dset* d = find(h, name);
  if (!d) return -1;
  for (size_t k = 0; k < d->d.size(); ++k) buf[k] = (float)d->d[k];
  return 0;
}
herr_t H5LTread_dataset_int(hid_t h, const char* name, int* buf)
{
  const Dset* d = find(h, name);
  if (!d) return -1;
  if (d->is_int) std::memcpy(buf, d->i.data(), d->i.size() * sizeof(int));
  else for (size_t k = 0; k < d->d.size(); ++k) buf[k] = (int)d->d[k];
  return 0;
}
herr_t H5LTmake_dataset(hid_t, const char*, int, const hsize_t*, hid_t, const void*) { return 0; }
herr_t H5LTfind_dataset(hid_t h, const char* name) { return find(h, name) ? 1 : 0; }
herr_t H5LTget_attribute_int(hid_t h, const char* obj, const char* attr, int* out)
{
  H5File* f = file_of(h);
  if (!f) return -1;
  auto it = f->attrs.find(norm(obj) + "|" + attr);
  if (it == f->attrs.end()) return -1;
  *out = it->second;
  return 0;
}
herr_t H5LTget_dataset_info(hid_t h, const char* name, hsize_t* dims, H5T_class_t*, size_t*)
{
  const Dset* d = find(h, name);
  if (!d) return -1;
  for (size_t k = 0; k < d->dims.size(); ++k) dims[k] = d->dims[k];
  return 0;
}
}
