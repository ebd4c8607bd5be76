// mixed_kernel.cuh -- the mixed-precision packet kernel for homologous 1D
// spheres (FP32 {abs, scat} tables and emissivity CDF, FP64 packet state).
// Included by transport_kernel.cu inside its anonymous namespace, after the
// shared helpers (emit_core, spectrum_count, cdf_row_sample, the batch zone
// tables).
//
// It runs the steps of propagate_monte_carlo (src/transport/transport.cpp:
// 260-484), do_scatter and isotropic_scatter (src/transport/scatter.cpp:
// 12-70, 303-351) and is held, like the mixed form of propagate_kernel, to
// the reference's spectra within Monte Carlo noise, not to its bits.  What
// differs is how much a segment costs:
//
//  * The optical depth to the next interaction is drawn once per flight
//    (after emission and after each interaction) and the depth a segment
//    crosses is subtracted when the segment ends at a zone wall, a
//    frequency-bin step or the end of the step.  The reference draws a new
//    depth every segment; for an exponential depth both give the same
//    distribution of interaction points (the remaining depth of an
//    exponential is again exponential), and segments that end at a wall or
//    a bin step then cost no deviate and no logarithm.
//  * One Philox4x32-10 block per interaction: word 0 is the next flight's
//    optical depth, word 1 the absorption test, word 2 the emissivity-CDF
//    deviate, word 3 the comoving direction cosine.  The deviates the
//    interaction needs beyond those are recycled (Devroye, Non-Uniform
//    Random Variate Generation, 1986, on reusing a uniform after a
//    comparison): given the outcome of "u <= eps", u / eps (or
//    (u - eps) / (1 - eps)) is again uniform on [0, 1) and independent of the
//    outcome, so it gives the effective-scattering test and then the
//    azimuth; given the CDF bin k that u >= cdf[k-1] selected,
//    (u - cdf[k-1]) / (cdf[k] - cdf[k-1]) is uniform and gives the position
//    within the bin.  A recycled deviate keeps 2^32 p distinct values when
//    its branch has probability p.
//  * FP64 square roots, reciprocal square roots and reciprocals from the
//    hardware's FP64 approximations refined by one Newton-Raphson step with
//    its second-order term (Markstein, IA-64 and Elementary Functions,
//    2000): the approximation's ~2^-20 relative error cubed is below FP64
//    rounding.  They are not correctly rounded, which the mixed form does
//    not need; position, time, frequency and the Lorentz transforms stay
//    FP64.
//  * -ln(u) in FP32 from the hardware logarithm, the interaction and
//    bin-step distances as FP32 quotients (they set where a segment ends,
//    not the state it carries).
//  * The zone's walls are loaded once per zone visit, |x|^2 and x.D once
//    per move.
//  * The frequency bin comes from the FP32 index estimate where it lies
//    clear of a wall (loc_within_mixed), and after a redistribution from the
//    interaction itself, with its opacity loaded there.
//  * 64 registers, 32 warps per SM: the zone-visit tally sums and the state
//    a packet reads only at its start or end sit in each thread's slots of
//    shared memory, and a visit's sums go to one of 32 global tally copies
//    by fire-and-forget reductions.
namespace mixed {

constexpr float W32 = 2.3283064365386963e-10f;  // 2^-32

// -ln(u), u = (w + 1/2) 2^-32 in (0, 1), from the hardware logarithm: a few
// ulp relative where u < 1/2, an absolute error below 2^-21 in the optical
// depth above (a short flight's depth off by what rounding the FP32 opacity
// of a unit optical depth already moves it).  One code path for all lanes:
// a branch to a series near u = 1 cost 2.6% of the Type Ia step.
__device__ __forceinline__ float neg_log_u(uint32_t w)
{
  return -__logf(((float)w + 0.5f) * W32);
}

// the zone's walls, as get_next_zone (grid_1D_sphere.cpp:510-590) derives
// them: outer wall and inner wall after the core substitution, held for the
// zone visit.  The neighbours are formed where next_zone needs them: from
// the zone index and the inner wall for one model, from the signs of the
// batch's wall table for a batch (outer wall negative past the model's last
// zone, inner wall negative where there is no inner neighbour, -0.0 for the
// r = 0 centre of a model's zone 0), which spares the batch a neighbour-table
// load per segment.
struct Walls {
  double r_o, r_i;
};

template <int BATCH>
__device__ __forceinline__ Walls zone_walls(const StepArgs& A, const GridDev& G, int i)
{
  Walls w;
  if constexpr (BATCH) {  // one 16-byte load; the neighbours ride in the signs
    const double2 rw = __ldg(A.zone_wall + i);
    w.r_o = rw.x;
    w.r_i = rw.y;
  } else {
    w.r_o = __ldg(G.r_out.right + i);
    w.r_i = (i != 0) ? __ldg(G.r_out.right + i - 1) : G.r_out.min;
    if (A.core_radius >= w.r_i) w.r_i = A.core_radius;
  }
  return w;
}

// distance to zone iz's boundary along D and the zone entered there, with
// the reference's tiny_offset push across the wall
template <int BATCH>
__device__ __forceinline__ int next_zone(const StepArgs& A, const GridDev& G, const Walls& w, int iz, double rsq,
                                         double xd, double* l)
{
  int in_nbr, out_nbr;
  bool no_inner;
  if constexpr (BATCH) {  // a model's zones are consecutive; the signs mark its edges and the core
    const bool in_edge = __double_as_longlong(w.r_i) < 0;  // the sign bit, -0.0 included
    in_nbr = in_edge ? -1 : iz - 1;
    out_nbr = (w.r_o < 0) ? -2 : iz + 1;
    no_inner = in_edge && (w.r_i == 0);
  } else {  // the inner wall is the core's when the substitution moved it there
    in_nbr = (iz == 0 || w.r_i == A.core_radius) ? -1 : iz - 1;
    out_nbr = (iz + 1 == G.nzones) ? -2 : iz + 1;
    no_inner = (iz == 0) && (w.r_i == 0);
  }
  const double l_out = sqrt_nr(fma(xd, xd, fma(w.r_o, w.r_o, -rsq))) - xd;
  // the inner wall's distance for every lane (a warp nearly always holds
  // inward and outward photons), kept where the photon moves inward and
  // meets it
  const double rad = fma(xd, xd, fma(w.r_i, w.r_i, -rsq));
  const double l_in_c = -xd - sqrt_nr(fmax(rad, 0.0));
  const double l_in = (!no_inner && xd < 0 && rad >= 0) ? l_in_c : -1.0;
  constexpr double tiny_offset = 1 + 1e-6;
  constexpr double inv_tiny_offset = 1 / tiny_offset;
  if ((l_out < l_in) || (l_in < 0)) {
    *l = (out_nbr == -2) ? l_out * inv_tiny_offset : l_out * tiny_offset;
    return out_nbr;
  }
  *l = (in_nbr == -1) ? l_in * inv_tiny_offset : l_in * tiny_offset;
  return in_nbr;
}

// isotropic_scatter (scatter.cpp:303-351) on a homologous flow, with the
// comoving direction from mu and the azimuth deviate vphi, and (redist) the
// comoving frequency from the zone's emissivity CDF with deviate word w_cdf
// Returns the comoving frequency bin of a redistributed photon (-1 for a
// coherent scatter) and its width times c t in *dnu_num.
template <typename CT>
__device__ __forceinline__ int scatter(const StepArgs& A, Pkt& p, double rsq, double xd, double mu, float vphi,
                                       uint32_t w_cdf, bool redist, float* dnu_num)
{
  int kbin = -1;
  const double gamma = rsqrt_nr(fma(-rsq, A.inv_ct2, 1.0));
  const double dshift_in = gamma * fma(-xd, A.inv_ct, 1.0);
  p.e = p.e * dshift_in;
  p.nu = p.nu * dshift_in;
  float sf, cf;
  __sincosf(fmaf((float)(2.0 * PI), vphi, -(float)PI), &sf, &cf);
  const double smu = sqrt_nr(fma(-mu, mu, 1.0));
  const double Dn0 = smu * (double)cf, Dn1 = smu * (double)sf, Dn2 = mu;
  if (redist) {  // transport::sample_photon_frequency (emission.cpp:27-46)
    const int nn = A.nu.n;
    if (nn == 1) p.nu = loc_sample(A.nu, 0, 0.5);
    else {
      const double u = (double)w_cdf * (1.0 / 4294967296.0);
      int k = cdf_row_sample<CT>(A, p.ind, u);
      if (k > nn - 1) k = nn - 1;
      const CT* row = reinterpret_cast<const CT*>(A.cdf) + (size_t)p.ind * nn;
      const double lo = (k == 0) ? 0.0 : (double)__ldg(row + k - 1);
      const double hi = (double)__ldg(row + k);
      float f = __fdividef((float)(u - lo), (float)(hi - lo));
      f = fminf(fmaxf(f, 0.0f), 0.99999994f);
      // locate_array::sample (locate_array.cpp:237-242) with the bin's walls
      // kept for the next segment
      const double wl = (k == 0) ? A.nu.min : __ldg(A.nu.right + k - 1);
      const double wr = __ldg(A.nu.right + k);
      p.nu = wl + (wr - wl) * (double)f;
      kbin = k;
      *dnu_num = (float)((wr - wl) * A.ct);
    }
  }
  // comoving -> lab with the velocity reversed, beta = x / (c t)
  const double b0 = p.x[0] * A.inv_ct, b1 = p.x[1] * A.inv_ct, b2 = p.x[2] * A.inv_ct;
  const double bdp = -fma(b0, Dn0, fma(b1, Dn1, b2 * Dn2));
  const double vd_out = gamma * (1 - bdp);
  const double gf = gamma * fma(-gamma * bdp, rcp_nr(gamma + 1), 1.0);
  const double inv_vd = rcp_nr(vd_out);
  const double D0 = inv_vd * fma(gf, b0, Dn0);
  const double D1 = inv_vd * fma(gf, b1, Dn1);
  const double D2 = inv_vd * fma(gf, b2, Dn2);
  const double inv_norm = rsqrt_nr(fma(D0, D0, fma(D1, D1, D2 * D2)));
  p.D[0] = D0 * inv_norm;
  p.D[1] = D1 * inv_norm;
  p.D[2] = D2 * inv_norm;
  p.e = p.e * vd_out;
  p.nu = p.nu * vd_out;
  return kbin;
}

// adds one zone visit's tallies: to the block's shared copy [5][nz] when
// A.smem_zones, else to global copy rep_off / (5 nz) of the n_rep copies
// (rep_off < 0: the arrays themselves).  The targets are formed here, from
// the shared array and the kernel's arguments, rather than held as five
// pointers across the packet loop.
__device__ __forceinline__ void add_visit(const StepArgs& A, double* s_tal, int nz, int64_t rep_off, int z,
                                          double e, double fx, double fy, double fz, double fr)
{
  if (A.smem_zones) {
    atomicAdd(s_tal + z, e);
    if (A.tally_forces) {
      atomicAdd(s_tal + nz + z, fx);
      atomicAdd(s_tal + 2 * nz + z, fy);
      atomicAdd(s_tal + 3 * nz + z, fz);
      atomicAdd(s_tal + 4 * nz + z, fr);
    }
  } else if (rep_off >= 0) {
    double* b = A.zone_rep + rep_off + z;
    atomicAdd(b, e);
    if (A.tally_forces) {
      atomicAdd(b + nz, fx);
      atomicAdd(b + 2 * nz, fy);
      atomicAdd(b + 3 * nz, fz);
      atomicAdd(b + 4 * nz, fr);
    }
  } else {
    atomicAdd(A.e_abs + z, e);
    if (A.tally_forces) {
      atomicAdd(A.fx + z, fx);
      atomicAdd(A.fy + z, fy);
      atomicAdd(A.fz + z, fz);
      atomicAdd(A.fr + z, fr);
    }
  }
}

// 8 bytes from global memory to a shared-memory slot without a register
// holding them in between (cp.async, cached in L1); cp_async_wait completes
// the thread's copies before the slot is read
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem)
{
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// the state emit_mixed_kernel stored for core packet q
__device__ __forceinline__ void load_emitted(const StepArgs& A, Pkt& p, int64_t q)
{
  const int64_t n = A.em_n;
  const double* s = A.em_state + q;
  p.x[0] = __ldg(s); p.x[1] = __ldg(s + n); p.x[2] = __ldg(s + 2 * n);
  p.D[0] = __ldg(s + 3 * n); p.D[1] = __ldg(s + 4 * n); p.D[2] = __ldg(s + 5 * n);
  p.t = __ldg(s + 6 * n); p.e = __ldg(s + 7 * n); p.nu = __ldg(s + 8 * n);
  p.ind = __ldg(A.em_ind + q);
}

}  // namespace mixed

// Emission of the core packets ahead of the packet kernel
// (emit_inner_source, src/transport/emission.cpp:370-485): one thread per
// packet, all lanes of a warp on the same code, the packet's state, zone and
// first optical depth (the emission's spare deviate) stored for the packet
// kernel.  Emission is the longest stretch of the packet kernel's loop
// (double-precision sincos, searches of the core CDF and of the zone walls);
// inside the persistent loop one lane emitting holds its whole warp.
template <int BATCH>
__global__ void __launch_bounds__(256) emit_mixed_kernel(const StepArgs A, const GridDev G)
{
  using namespace mixed;
  const int64_t n = A.em_n;
  uint32_t step = A.step;
  if constexpr (BATCH) step = *A.step_dev;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
    Pkt p;
    PacketRng rng;
    float tau;
    if constexpr (BATCH) {
      const int m = find_model(A.models, A.n_models, q);
      const BatchModel& M = A.models[m];
      rng.init(M.seed, (uint64_t)(M.first_pid + (q - M.pkt_off)), step, 0);
      BatchZoneOf zf;
      zf.slice = G.r_out;
      zf.slice.n = M.n_zones;
      zf.slice.min = M.r_min;
      zf.slice.right = G.r_out.right + M.zone_off;
      zf.zone_off = M.zone_off;
      DrawWords d{rng};
      emit_core<0>(A, G, p, d, M.core_radius, M.Ep, M.core_cdf, zf);
      tau = neg_log_u(d.word());
      A.em_model[q] = m;
    } else {
      rng.init(A.seed, (uint64_t)A.first_pid + q, step, 0);
      DrawWords d{rng};
      emit_core<0>(A, G, p, d, A.core_radius, A.Ep, A.core_cdf, GridZoneOf<0>{G});
      tau = neg_log_u(d.word());
    }
    double* s = A.em_state + q;
    s[0] = p.x[0]; s[n] = p.x[1]; s[2 * n] = p.x[2];
    s[3 * n] = p.D[0]; s[4 * n] = p.D[1]; s[5 * n] = p.D[2];
    s[6 * n] = p.t; s[7 * n] = p.e; s[8 * n] = p.nu;
    A.em_ind[q] = p.ind;
    A.em_tau[q] = tau;
  }
}

// BATCH = 0: one model (core packets, then the queue of census and
// radioactive photons); BATCH = 1: the batched 1D models of sed_batch_*.
// Core packets come from emit_mixed_kernel's buffers.
template <int BATCH, int THREADS, int MINB>
__global__ void __launch_bounds__(THREADS, MINB) propagate_mixed_kernel(const StepArgs A, const GridDev G)
{
  using namespace mixed;
  using CT = float;
  extern __shared__ double s_tal[];  // [5][nz] when A.smem_zones
  // the block's event counters, added to once per packet (escaped, absorbed,
  // stopped, segments, interactions, segment-limit stops)
  __shared__ unsigned long long s_cnt[6];
  if (threadIdx.x < 6) s_cnt[threadIdx.x] = 0;
  const int nz = G.nzones;
  const int nn = A.nu.n;
  const int nj = A.store_Jnu ? nn : 1;
  if (A.smem_zones)
    for (int i = threadIdx.x; i < 5 * nz; i += blockDim.x) s_tal[i] = 0.0;
  __syncthreads();
  const int64_t rep_off = (!A.smem_zones && A.n_rep > 0) ? (int64_t)(blockIdx.x % A.n_rep) * 5 * nz : -1;
  const float2* __restrict__ opac = reinterpret_cast<const float2*>(A.opac);
  const int32_t limit = A.max_segments > 0 ? A.max_segments : 10000000;
  const uint32_t K_core = ((A.core_radius == 0 ? 2u : 4u) + (A.core_freq > 0 ? 0u : 2u) + 1u + 3u) / 4u;
  uint32_t step = A.step;
  if constexpr (BATCH) step = *A.step_dev;
  Pkt p;
  PacketRng rng;
  int fate = ABSORBED;  // no packet yet
  bool have = false;
  int32_t seg = 0;
  const int tid = threadIdx.x;
  // What the loop reads only when a packet starts or ends, or one segment
  // after forming it, sits in the thread's own slots of shared memory
  // rather than in registers: the packet's queue index, the Philox counter
  // where its records count draws from and where its interactions start
  // (one block per interaction), the {abs, scat} and bin width of a
  // redistributed photon's new bin, and for a batch the model and the
  // claimed queue range.
  __shared__ unsigned long long s_pid[THREADS];
  __shared__ uint32_t s_k0[THREADS], s_n0[THREADS];
  __shared__ float2 s_nab[BATCH ? THREADS : 1];
  __shared__ float s_ndnu[BATCH ? THREADS : 1];
  __shared__ int s_m[BATCH ? THREADS : 1];
  __shared__ long long s_qn[BATCH ? THREADS : 1], s_qe[BATCH ? THREADS : 1];
  if constexpr (BATCH) { s_qn[tid] = 0; s_qe[tid] = 0; }
  // zone-visit tallies (e_abs, fx, fy, fz, fr), summed in the thread's own
  // columns of shared memory (held in registers they cost the ten that take
  // the kernel from 28 to 24 warps per SM: Type Ia packet kernel 631 ms
  // against 661 ms).  One model's kernel keeps two slots: the zone being
  // visited and the zone the packet came from.  A photon that steps back
  // over the wall it just crossed carries on with that zone's sums; only a
  // move to a third zone sends the older slot's sums to the tally copies
  // (Type Ia packet kernel 562 -> 551 ms).  The batched kernel keeps one
  // slot: with two its 64-register shapes spill and its step ran 1-4 %
  // slower.  acc holds the current zone and its slot as (zone << 1) | slot
  // (-1 before the packet's first segment), s_oz the zone whose sums sit in
  // the other slot (-1: none); a slot that holds no zone holds zeros.  With
  // one slot acc is the zone itself and the slot is zeroed when a visit
  // starts.
  constexpr int SLOTS = BATCH ? 1 : 2;
  int acc = -1;
  __shared__ double s_acc[SLOTS][5][THREADS];
  __shared__ int s_oz[SLOTS == 2 ? THREADS : 1];
  auto flush_slot = [&](int z, int k) {  // send slot k's sums for zone z and zero the slot
    double* a = &s_acc[k][0][tid];
    add_visit(A, s_tal, nz, rep_off, z, a[0], a[THREADS], a[2 * THREADS], a[3 * THREADS], a[4 * THREADS]);
    a[0] = 0.0; a[THREADS] = 0.0; a[2 * THREADS] = 0.0; a[3 * THREADS] = 0.0; a[4 * THREADS] = 0.0;
  };
  for (int k = 0; k < SLOTS; ++k)
    for (int q = 0; q < 5; ++q) s_acc[k][q][tid] = 0.0;
  if constexpr (SLOTS == 2) s_oz[tid] = -1;
  Walls wl{};
  double rsq = 0, xd = 0;
  float tau_rem = 0;  // optical depth left to the next interaction
  bool live = true;   // the lane still takes packets from the queue
  // after a redistribution: the photon's comoving bin (its lab frequency
  // transforms back into that bin at the next segment's start, which is the
  // interaction point), its {abs, scat}, loaded ahead, and its width times
  // c t; -1 when the next segment has to locate its bin.  One model's kernel
  // holds the last two in registers (its segment loop ran 4% slower with
  // them in shared memory at the same occupancy); the batched kernel keeps
  // them in s_nab, s_ndnu, which it needs to fit 72 registers.
  int nxt_bin = -1;
  float2 nxt_ab = make_float2(0.f, 0.f);
  float nxt_dnu = 0.f;
  for (;;) {
    // The lanes of the warp meet here every iteration.  Without it, lanes
    // whose packet ended, or that took a shorter branch, drift apart and the
    // warp runs their iterations group after group with few lanes each;
    // lanes that have run out of packets stay in the loop, idle, until the
    // whole warp has.
    __syncwarp();
    if (!__any_sync(0xffffffffu, live)) break;
    if (!live) continue;
    if (fate != MOVING) {
      if (have) {
        if constexpr (SLOTS == 2) {
          if (acc >= 0) {
            const int oz = s_oz[tid];
            flush_slot(acc >> 1, acc & 1);
            if (oz >= 0) flush_slot(oz, (acc & 1) ^ 1);
            s_oz[tid] = -1;
            acc = -1;
          }
        } else if (acc >= 0) {
          add_visit(A, s_tal, nz, rep_off, acc, s_acc[0][0][tid], s_acc[0][1][tid], s_acc[0][2][tid],
                    s_acc[0][3][tid], s_acc[0][4][tid]);
        }
        atomicAdd(s_cnt + 3, (unsigned long long)seg);
        atomicAdd(s_cnt + 4, (unsigned long long)(rng.n - s_n0[tid]));
        if (fate == ESCAPED) {
          const double t_obs = p.t - (p.x[0] * p.D[0] + p.x[1] * p.D[1] + p.x[2] * p.D[2]) / C_LIGHT;
          if constexpr (BATCH) {
            const int m = s_m[tid];
            const int64_t so = A.models[m].spec_off;
            spectrum_count(A, A.flux + so, A.click + so, t_obs, p.nu, p.e, p.D);
            atomicAdd(A.model_escaped + m, 1ULL);
          } else {
            spectrum_count(A, A.flux, A.click, t_obs, p.nu, p.e, p.D);
          }
          p.t = t_obs;
          atomicAdd(s_cnt + 0, 1ULL);
        } else if (fate == ABSORBED) {
          atomicAdd(s_cnt + 1, 1ULL);
        } else {
          atomicAdd(s_cnt + 2, 1ULL);
        }
        if (A.rec_fate) {
          const unsigned long long pid = s_pid[tid];
          A.rec_fate[pid] = fate;
          A.rec_ind[pid] = p.ind;
          A.rec_draws[pid] = (int32_t)(rng.n - s_k0[tid]);
          if (A.rec_type) A.rec_type[pid] = TYPE_PHOTON;
          double* s = A.rec_state + pid * 9;
          s[0] = p.x[0]; s[1] = p.x[1]; s[2] = p.x[2];
          s[3] = p.D[0]; s[4] = p.D[1]; s[5] = p.D[2];
          s[6] = p.t; s[7] = p.e; s[8] = p.nu;
        }
        have = false;
      }
      if constexpr (BATCH) {
        long long q_next = s_qn[tid], q_end = s_qe[tid];
        if (q_next >= q_end) {
          q_next = (long long)atomicAdd(A.counters + C_QUEUE, (unsigned long long)A.queue_chunk);
          q_end = q_next + A.queue_chunk;
          if (q_end > A.n_packets) q_end = A.n_packets;
          s_qe[tid] = q_end;
        }
        if (q_next >= A.n_packets) { live = false; continue; }
        const unsigned long long pid = (unsigned long long)q_next;
        s_qn[tid] = q_next + 1;
        s_pid[tid] = pid;
        const int m = __ldg(A.em_model + pid);
        s_m[tid] = m;
        const BatchModel& M = A.models[m];
        const uint32_t K = (M.emit_draws + 3u) / 4u;
        // the stream continues after the emission's blocks
        rng.init(M.seed, (uint64_t)(M.first_pid + ((int64_t)pid - M.pkt_off)), step, K);
        s_k0[tid] = K;
        load_emitted(A, p, (int64_t)pid);
        tau_rem = __ldg(A.em_tau + pid);
      } else {
        const unsigned long long pid = atomicAdd(A.counters + C_QUEUE, 1ULL);
        if (pid >= (unsigned long long)A.n_packets) { live = false; continue; }
        s_pid[tid] = pid;
        if (A.q_n != nullptr && (int64_t)pid >= A.n_core) {
          // a queued photon: census (stream position 0) or an optical
          // photon the gamma-ray kernel handed over at its stream position
          const int64_t k = (int64_t)pid - A.n_core;
          const uint32_t qn = A.q_n[k];
          if (qn == RADIO_NO_PHOTON) continue;
          const double* q = A.q_state + (size_t)k * 9;
          p.x[0] = q[0]; p.x[1] = q[1]; p.x[2] = q[2];
          p.D[0] = q[3]; p.D[1] = q[4]; p.D[2] = q[5];
          p.t = q[6]; p.e = q[7]; p.nu = q[8];
          p.ind = A.q_ind[k];
          rng.init(A.seed, (uint64_t)(A.radio_first_pid + k), step, qn);
          s_k0[tid] = 0;
          tau_rem = neg_log_u(rng.block().x);
        } else {
          rng.init(A.seed, (uint64_t)A.first_pid + pid, step, K_core);  // after the emission's blocks
          s_k0[tid] = K_core;
          load_emitted(A, p, (int64_t)pid);
          tau_rem = __ldg(A.em_tau + pid);
        }
      }
      fate = MOVING;
      if (p.ind == -1) fate = ABSORBED;
      else if (p.ind == -2) fate = ESCAPED;
      seg = 0;
      nxt_bin = -1;
      if constexpr (SLOTS == 1) {
        acc = -1;
        s_acc[0][0][tid] = 0.0; s_acc[0][1][tid] = 0.0; s_acc[0][2][tid] = 0.0; s_acc[0][3][tid] = 0.0;
        s_acc[0][4][tid] = 0.0;
      }
      have = true;
      s_n0[tid] = rng.n;
      if (fate != MOVING) continue;
      rsq = fma(p.x[0], p.x[0], fma(p.x[1], p.x[1], p.x[2] * p.x[2]));
      xd = fma(p.D[0], p.x[0], fma(p.D[1], p.x[1], p.D[2] * p.x[2]));
    }
    // ------------------------------------------------------------- segment
    if (seg >= limit) { fate = STOPPED; atomicAdd(s_cnt + 5, 1ULL); continue; }
    ++seg;
    const int iz = p.ind;
    if (iz != (SLOTS == 2 ? (acc >> 1) : acc)) {  // a zone change (or the packet's first segment)
      if constexpr (SLOTS == 2) {
        const int k = (acc < 0) ? 0 : ((acc & 1) ^ 1);  // the other slot takes zone iz
        const int oz = s_oz[tid];
        if (oz >= 0 && oz != iz) flush_slot(oz, k);  // a third zone: the older visit's sums go out
        s_oz[tid] = acc >> 1;                        // the zone just left keeps its slot
        acc = (iz << 1) | k;
      } else {
        if (acc >= 0)
          add_visit(A, s_tal, nz, rep_off, acc, s_acc[0][0][tid], s_acc[0][1][tid], s_acc[0][2][tid],
                    s_acc[0][3][tid], s_acc[0][4][tid]);
        acc = iz;
        s_acc[0][0][tid] = 0.0; s_acc[0][1][tid] = 0.0; s_acc[0][2][tid] = 0.0; s_acc[0][3][tid] = 0.0;
        s_acc[0][4][tid] = 0.0;
      }
      wl = zone_walls<BATCH>(A, G, iz);
    }
    double d_bn;
    int new_ind = next_zone<BATCH>(A, G, wl, iz, rsq, xd, &d_bn);
    // comoving frequency and the opacity of its bin (transport_opacity.cpp:268-299)
    const double gamma = rsqrt_nr(fma(-rsq, A.inv_ct2, 1.0));
    const double dshift = gamma * fma(-xd, A.inv_ct, 1.0);
    int i_nu;
    float2 ab;
    float dnu_num;
    if (nxt_bin >= 0) {  // the redistributed photon's bin, located and loaded at the interaction
      i_nu = nxt_bin;
      if constexpr (BATCH) {
        cp_async_wait();
        ab = s_nab[tid];
        dnu_num = s_ndnu[tid];
      } else {
        ab = nxt_ab;
        dnu_num = nxt_dnu;
      }
      nxt_bin = -1;
    } else {
      i_nu = loc_within_mixed(A.nu, p.nu * dshift);
      ab = __ldg(opac + (size_t)iz * nn + i_nu);
      dnu_num = (float)(loc_delta(A.nu, i_nu) * A.ct);
    }
    const float a_f = ab.x;
    const float s_f = A.omit_scat ? 0.0f : ab.y;
    const float op_f = a_f + s_f;
    // distance over which the comoving frequency drifts by the bin's width,
    // with the hardware's ~2^-20 reciprocal (it sets where the segment ends)
    double r_nu;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r_nu) : "d"(p.nu));
    const double d_nu = fabs((double)dnu_num * r_nu);
    if (d_nu < d_bn) { d_bn = d_nu; new_ind = iz; }
    const float tot_f = op_f * (float)dshift;  // lab-frame extinction
    const double d_sc = (tot_f > 0.0f) ? (double)__fdividef(tau_rem, tot_f) : (double)INFINITY;
    const double d_tm = A.steady ? (double)INFINITY : (A.tstop - p.t) * C_LIGHT;
    int event;
    double this_d;
    if ((d_sc < d_bn) && (d_sc < d_tm)) { event = 0; this_d = d_sc; }
    else if (d_bn < d_tm) { event = 1; this_d = d_bn; }
    else { event = 2; this_d = d_tm; }
    // tallies (transport.cpp:361-392)
    const double this_E = p.e * this_d;
    const double eps_imc = __ldg(A.eps_imc + iz);
    const double ed = this_E * dshift;
    double* sa = &s_acc[SLOTS == 2 ? (acc & 1) : 0][0][tid];
    sa[0] = fma(ed * dshift * (double)a_f, eps_imc, sa[0]);
    atomicAdd(A.J + (size_t)iz * nj + (A.store_Jnu ? i_nu : 0), this_E);
    if (A.tally_forces) {
      const double wd = ed * (double)op_f * dshift;
      sa[THREADS] = fma(wd, p.D[0], sa[THREADS]);
      sa[2 * THREADS] = fma(wd, p.D[1], sa[2 * THREADS]);
      sa[3 * THREADS] = fma(wd, p.D[2], sa[3 * THREADS]);
      sa[4 * THREADS] = fma(wd * xd, rsqrt_nr(rsq), sa[4 * THREADS]);
    }
    // move
    p.x[0] = fma(this_d, p.D[0], p.x[0]);
    p.x[1] = fma(this_d, p.D[1], p.x[1]);
    p.x[2] = fma(this_d, p.D[2], p.x[2]);
    constexpr double INV_C = 1.0 / C_LIGHT;
    p.t = fma(this_d, INV_C, p.t);
    rsq = fma(p.x[0], p.x[0], fma(p.x[1], p.x[1], p.x[2] * p.x[2]));
    xd = fma(p.D[0], p.x[0], fma(p.D[1], p.x[1], p.D[2] * p.x[2]));
    if (event != 0) tau_rem = fmaxf(0.0f, fmaf(-tot_f, (float)this_d, tau_rem));  // depth crossed
    if (event == 1) {
      if (new_ind == -1) {
        if (A.bound_in_reflect) { p.D[0] = -p.D[0]; p.D[1] = -p.D[1]; p.D[2] = -p.D[2]; xd = -xd; }
        else { p.ind = new_ind; fate = ABSORBED; }
      } else if (new_ind == -2) {
        if (A.bound_out_reflect) { p.D[0] = -p.D[0]; p.D[1] = -p.D[1]; p.D[2] = -p.D[2]; xd = -xd; }
        else { p.ind = new_ind; fate = ESCAPED; }
      } else {
        p.ind = new_ind;
      }
    } else if (event == 0) {
      // do_scatter (scatter.cpp:12-70): u <= eps is the absorption branch;
      // the deviate left over from each test is recycled into the next
      const uint4 blk = rng.block();
      tau_rem = neg_log_u(blk.x);  // the next flight's depth
      const float u1 = (float)blk.y * W32;
      const float num = u1 * op_f;
      bool redist = false;
      float v;
      if (num <= a_f && a_f > 0.0f) {
        v = __fdividef(num, a_f);
        redist = true;
        if (!A.radiative_eq) {
          const float ei = (float)eps_imc;
          if (v > ei) v = __fdividef(v - ei, 1.0f - ei);  // effective scattering
          else { fate = ABSORBED; redist = false; }
        }
      } else {
        v = __fdividef(num - a_f, s_f);
      }
      if (fate == MOVING) {
        const double mu = 1.0 - 2.0 * ((double)blk.w * (1.0 / 4294967296.0));
        float dnu_new = 0.f;
        nxt_bin = scatter<CT>(A, p, rsq, xd, mu, fminf(fmaxf(v, 0.0f), 1.0f), blk.z, redist, &dnu_new);
        if (nxt_bin >= 0) {  // the new bin's {abs, scat}, loaded ahead of its use
          if constexpr (BATCH) {
            cp_async8(s_nab + tid, opac + (size_t)iz * nn + nxt_bin);
            s_ndnu[tid] = dnu_new;
          } else {
            nxt_ab = __ldg(opac + (size_t)iz * nn + nxt_bin);
            nxt_dnu = dnu_new;
          }
        }
        xd = fma(p.D[0], p.x[0], fma(p.D[1], p.x[1], p.D[2] * p.x[2]));
      }
    } else {
      fate = STOPPED;
    }
  }
  cp_async_wait();
  __syncthreads();
  if (threadIdx.x < 6) {
    constexpr int slot[6] = {C_ESCAPED, C_ABSORBED, C_STOPPED, C_SEGMENTS, C_SCATTERS, C_LIMIT};
    const unsigned long long v = s_cnt[threadIdx.x];
    if (v) atomicAdd(A.counters + slot[threadIdx.x], v);
  }
  if (A.smem_zones) {
    double* g[5] = {A.e_abs, A.fx, A.fy, A.fz, A.fr};
    for (int i = threadIdx.x; i < 5 * nz; i += blockDim.x) {
      const double v = s_tal[i];
      if (v != 0.0 || isnan(v)) atomicAdd(g[i / nz] + (i % nz), v);
    }
  }
}
