/*
 * oracle/irbc_rng.h -- TEST INFRASTRUCTURE (oracle side). Not part of the
 * shipped library; only tests, smoke() and bench.py's CPU-baseline leg use it.
 *
 * The draw stream that replaces the reference's Mersenne Twister.
 *
 * The reference draws all of its random numbers from per-thread MT19937
 * objects seeded with time(0) (maincode.cpp:58-66): uniforms through
 * CRandomMersenne::Random() (Src/mersenne.cpp:108-112, 32-bit resolution,
 * u = bits * 2^-32) and normals through StochasticLib1::Normal
 * (Src/stoc1.cpp:746-765).  With one OpenMP thread the ORDER in which the
 * step functions consume draws is fixed; that order is what parity needs.
 *
 * This file defines the replacement stream: Philox4x32-10 (Salmon, Moraes,
 * Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11), keyed
 * by the run seed.  Draw number k of a (stream, epoch) pair is
 *     block = philox(ctr = {k/4 lo, k/4 hi, epoch, stream}, key = seed)
 *     uniform_k = block[k % 4] * 2^-32                     (in [0,1))
 *     normal_k  = sqrt(-2 ln u1) cos(2 pi u2),
 *                 u1 = (block'[0] + 1) 2^-32, u2 = block'[1] 2^-32,
 *                 block' = philox(ctr = {k lo, k hi, epoch, stream})
 * The reference consumes draw k as its k-th call in that phase; the CUDA
 * library computes k for each cell / vertex with a scan, so both sides see
 * the same numbers without any tape being stored.
 */
#ifndef IRBC_ORACLE_RNG_H
#define IRBC_ORACLE_RNG_H

#include <stdint.h>
#include <math.h>

/* stream ids (counter word 3) */
enum {
  ORC_STREAM_INIT = 1,       /* solvent, vertex, parasite init + knob placement */
  ORC_STREAM_COLLIDE_U = 2,  /* grid shift (3) then rand1, rand2 per cell      */
  ORC_STREAM_COLLIDE_N = 3,  /* ghost-particle normals, 3 per filled cell     */
  ORC_STREAM_BOND = 4        /* bond_dynamics uniforms                          */
};

static inline void orc_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2],
                                     uint32_t out[4]) {
  uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
  uint32_t k0 = key_in[0], k1 = key_in[1];
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)0xD2511F53u * (uint64_t)c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * (uint64_t)c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

static inline void orc_block(uint64_t seed, uint32_t stream, uint64_t epoch, uint64_t blk,
                             uint32_t out[4]) {
  uint32_t ctr[4] = {(uint32_t)blk, (uint32_t)(blk >> 32), (uint32_t)epoch,
                     stream | ((uint32_t)(epoch >> 32) << 8)};
  uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  orc_philox4x32_10(ctr, key, out);
}

static inline double orc_uniform(uint64_t seed, uint32_t stream, uint64_t epoch, uint64_t k) {
  uint32_t o[4];
  orc_block(seed, stream, epoch, k >> 2, o);
  return (double)o[k & 3u] * (1.0 / 4294967296.0);
}

static inline double orc_normal(uint64_t seed, uint32_t stream, uint64_t epoch, uint64_t k) {
  uint32_t o[4];
  orc_block(seed, stream, epoch, k, o);
  double u1 = ((double)o[0] + 1.0) * (1.0 / 4294967296.0);
  double u2 = (double)o[1] * (1.0 / 4294967296.0);
  return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

#endif
