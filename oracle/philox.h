/* oracle/philox.h -- TEST INFRASTRUCTURE (oracle only).
 *
 * Counter-based Philox4x32-10 generator restated from the published
 * algorithm (Salmon, Moraes, Dror, Shaw, "Parallel Random Numbers: As Easy
 * as 1, 2, 3", SC'11): ten rounds of two 32x32->64 multiplies with the
 * multipliers 0xD2511F53 / 0xCD9E8D57 and a Weyl key schedule with
 * increments 0x9E3779B9 / 0xBB67AE85.  This copy is independent of the CUDA
 * product header; both are pinned to the published known-answer vectors by
 * the CPU tests.
 *
 * Draw convention shared by the oracle, the reference harness and the GPU
 * packet kernel (it replaces thread_RNG::uniform, src/transport/thread_RNG.cpp:91-99):
 *   key     = { seed, 0 }
 *   counter = { n >> 1, packet_id (low 32), packet_id (high 32), step }
 *   draw n of a packet uses output words (0,1) when n is even, (2,3) when odd,
 *   u = ((w_a >> 5) * 2^26 + (w_b >> 6)) * 2^-53, a double in [0, 1).
 */
#ifndef ORACLE_PHILOX_H
#define ORACLE_PHILOX_H

#include <stdint.h>

static inline void oracle_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4])
{
  uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
  uint32_t k0 = key_in[0], k1 = key_in[1];
  for (int r = 0; r < 10; ++r) {
    if (r > 0) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
    uint64_t p0 = (uint64_t)0xD2511F53u * (uint64_t)c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * (uint64_t)c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

static inline double oracle_u01_from_words(uint32_t a, uint32_t b)
{
  return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6)) * (1.0 / 9007199254740992.0);
}

/* draw n of packet `pid` in transport step `step` */
static inline double oracle_packet_uniform(uint32_t seed, uint64_t pid, uint32_t step, uint32_t n)
{
  uint32_t ctr[4] = { n >> 1, (uint32_t)pid, (uint32_t)(pid >> 32), step };
  uint32_t key[2] = { seed, 0u };
  uint32_t w[4];
  oracle_philox4x32_10(ctr, key, w);
  return (n & 1u) ? oracle_u01_from_words(w[2], w[3]) : oracle_u01_from_words(w[0], w[1]);
}

#endif
