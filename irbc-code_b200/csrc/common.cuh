// common.cuh -- device parameters, the Philox draw stream and the small
// geometric helpers shared by the solvent and membrane kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace irbc {

// Everything a kernel needs to know about one simulation, passed by value.
struct DevParams {
  double a, Lx, Ly, Lz, dtcd, navg, Theta, walls, mass, cosalpha, sinalpha;
  double kappasa, kappad, kappav, kappab, pmass, dtmd, ks, dthr, FD, Fg, el0, PRmass, paraR;
  double Pi, elap, onrate, offrate, wallspeed;
  double Sarea0, Volume0, theta0, cth0, sth0;  // cos/sin(theta0*Pi/180) from the host libm
  int nx, ny, nz;        // collision grid: Lx/a, Ly/a, Lz/a + 1 (maincode.cpp:113-115)
  int64_t ncell;
  int nv, ne, nt;
  int nligx, nligy, nlig;  // ligand grid 0.5 apart (maincode.cpp:77-93)
  int randno;
  uint64_t seed;
  // the draw epoch (step index) of a launch is *ebase + its offset argument:
  // the host writes the base once per step call, so that a captured
  // sequence of steps replays with the right epochs
  const uint64_t* ebase;
  // run-time health word of the simulation (HEALTH_* bits), or null
  int* health;
  // Sarea and Volume as a fixed warp tree instead of the reference's
  // left-to-right sum (the FP32-bulk solvent, which claims no bit parity)
  int tree_sums;
};

// Health bits, raised by the kernels that write the state and read back by
// the host (irbc_sync, irbc_health): a solvent particle whose position or
// velocity is not finite, or whose height left [-a, Lz + a]; a membrane
// vertex whose force or velocity is not finite.  The checks ride on values
// the kernels hold in registers anyway and write only when something is
// wrong.
enum : int { HEALTH_SOLVENT = 1, HEALTH_MEMBRANE = 2 };
__device__ __forceinline__ void raise_health(const DevParams& p, bool bad, int bit) {
  if (bad && p.health) atomicOr(p.health, bit);
}
template <typename R>
__device__ __forceinline__ bool solvent_bad(const DevParams& p, R X, R Y, R Z, R VX, R VY, R VZ) {
  const R s = X + Y + VX + VY + VZ;
  return !isfinite(s) || !(Z >= R(-p.a) && Z <= R(p.Lz + p.a));
}

__device__ __forceinline__ uint64_t epoch_of(const DevParams& p, uint64_t off) { return *p.ebase + off; }

// draw streams (counter word 3); the same numbering as the oracle's
enum : uint32_t { STREAM_INIT = 1, STREAM_COLLIDE_U = 2, STREAM_COLLIDE_N = 3, STREAM_BOND = 4 };

// Philox4x32-10 (Salmon et al., SC'11): 10 rounds of the published
// multiply/xor round with the Weyl key schedule.
__host__ __device__ inline void philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                              uint32_t k0, uint32_t k1, uint32_t out[4]) {
#ifdef __CUDA_ARCH__
#pragma unroll
#endif
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
    uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
    c1 = (uint32_t)p1;
    c3 = (uint32_t)p0;
    c0 = n0;
    c2 = n2;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

__host__ __device__ inline void draw_block(uint64_t seed, uint32_t stream, uint64_t epoch, uint64_t blk,
                                           uint32_t out[4]) {
  philox4x32_10((uint32_t)blk, (uint32_t)(blk >> 32), (uint32_t)epoch,
                stream | ((uint32_t)(epoch >> 32) << 8), (uint32_t)seed, (uint32_t)(seed >> 32), out);
}

// k-th uniform of (stream, epoch): 32 random bits times 2^-32, the
// resolution of the reference's Random() (Src/mersenne.cpp:108-112)
__host__ __device__ inline double draw_uniform(uint64_t seed, uint32_t stream, uint64_t epoch, uint64_t k) {
  uint32_t o[4];
  draw_block(seed, stream, epoch, k >> 2, o);
  return (double)o[k & 3u] * (1.0 / 4294967296.0);
}

// k-th standard normal: Box-Muller on block k
__device__ inline double draw_normal(uint64_t seed, uint32_t stream, uint64_t epoch, uint64_t k) {
  uint32_t o[4];
  draw_block(seed, stream, epoch, k, o);
  double u1 = ((double)o[0] + 1.0) * (1.0 / 4294967296.0);
  double u2 = (double)o[1] * (1.0 / 4294967296.0);
  return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

// the collision grid's random shift (Src/solfuncs.cpp:116-118): uniforms 0, 1, 2 of the
// COLLIDE_U stream, times a
__device__ __forceinline__ void grid_shift(const DevParams& p, uint64_t epoch, double r[3]) {
  uint32_t o[4];
  draw_block(p.seed, STREAM_COLLIDE_U, epoch, 0, o);
  r[0] = p.a * ((double)o[0] * (1.0 / 4294967296.0));
  r[1] = p.a * ((double)o[1] * (1.0 / 4294967296.0));
  r[2] = p.a * ((double)o[2] * (1.0 / 4294967296.0));
}

// counting-sort slots: particle i0 + u * stride (u < K) of cell c[u] (-1:
// none) gets a slot in its cell's counter.  The particles are nearly sorted
// by cell in memory (the physical re-sort), so lanes with equal cells mostly
// form runs of consecutive lanes: a run's first lane adds the run's length
// with one atomic and the run's lanes take consecutive slots from its
// result.  Equal cells in separate runs take separate atomics; the slots
// stay distinct and their order within a cell is free (the collision ranks
// a cell's particles by reference index).  Runs are found with a ballot and
// a shuffle, not with match_any (whose address-unit throughput bound the
// count kernel).  The in-range lanes of a warp are a prefix of it (the
// index grows with the lane).  The K claims of a thread are issued before
// any result is used.
constexpr int kCountPer = 4;
template <int K>
__device__ __forceinline__ void claim_slots(int* cnt, const int c[K], int64_t i0, int stride, int64_t n,
                                            int slot[K]) {
  const int lane = threadIdx.x & 31;
  const unsigned upto = (lane == 31) ? 0xffffffffu : ((2u << lane) - 1u);  // lanes <= this one
  int head[K], base[K];
#pragma unroll
  for (int u = 0; u < K; ++u) {
    const bool in = i0 + (int64_t)u * stride < n;
    const int prev = __shfl_up_sync(0xffffffffu, c[u], 1);
    const bool starts = in && (lane == 0 || prev != c[u]);
    const unsigned heads = __ballot_sync(0xffffffffu, starts);
    const int nin = __popc(__ballot_sync(0xffffffffu, in));
    const unsigned mine = heads & upto;
    head[u] = mine ? 31 - __clz(mine) : lane;
    base[u] = 0;
    if (starts) {
      const unsigned after = heads & ~upto;
      const int end = after ? __ffs(after) - 1 : nin;
      base[u] = atomicAdd(&cnt[c[u]], end - lane);
    }
  }
#pragma unroll
  for (int u = 0; u < K; ++u) {
    const int b = __shfl_sync(0xffffffffu, base[u], head[u]);
    if (i0 + (int64_t)u * stride < n) slot[u] = b + (lane - head[u]);
  }
}

// periodic wrap by repeated subtraction (bbound, Src/solfuncs.cpp:603-622).
// The reference's loop never ends for an infinite coordinate and runs for
// ages for a huge one (reachable only through a degenerate contact time);
// here a coordinate beyond 64 periods is first reduced with fmod (exact,
// |result| < lx) and a non-finite one passes through unchanged, so every
// call ends after at most 64 subtractions.  Below 64 periods the result is
// the reference's.
template <typename R>
__device__ __forceinline__ R bbound(R x, R lx) {
  if (!(fabs(x) < R(64) * lx)) {
    if (!isfinite(x)) return x;
    x = fmod(x, lx);
  }
  if (x > lx) { while (x > lx) x -= lx; }
  if (x < R(0)) { while (x < R(0)) x += lx; }
  return x;
}

// cindex[fx][fy][fz] (maincode.cpp:112-136); entries never assigned are 0
__device__ __forceinline__ int cell_of(const DevParams& p, int fx, int fy, int fz) {
  if (fx >= 0 && fx < p.nx && fy >= 0 && fy < p.ny && fz >= 0 && fz < p.nz)
    return (fx * p.ny + fy) * p.nz + fz;
  return 0;
}

// cross product cp (Src/memfuncs.cpp:47-52)
template <typename R>
__device__ __forceinline__ void cp(const R A[3], const R B[3], R C[3]) {
  C[0] = (A[1] * B[2]) - (B[1] * A[2]);
  C[1] = (A[2] * B[0]) - (B[2] * A[0]);
  C[2] = (A[0] * B[1]) - (B[0] * A[1]);
}

// SolveP3 (Src/poly34.cpp:26-55): trigonometric (three real roots) or
// Cardano (one) form, then the root selection of Solve
// (Src/solfuncs.cpp:369-396): the smallest root in [0, dtmd], else the next.
__device__ __forceinline__ double solve_p3_tt(double aa, double b, double c, double dtmd) {
  // SolveP3 (Src/poly34.cpp:26-55) + root selection of Solve (Src/solfuncs.cpp:369-396)
  const double TwoPi = 6.28318530717958648, eps = 1e-14;
  double x[3];
  int nroot;
  double a2 = aa * aa;
  double q = (a2 - 3 * b) / 9;
  double r = (aa * (2 * a2 - 9 * b) + 27 * c) / 54;
  double r2 = r * r;
  double q3 = q * q * q;
  if (r2 < q3) {
    double t = r / sqrt(q3);
    if (t < -1) t = -1;
    if (t > 1) t = 1;
    t = acos(t);
    aa /= 3; q = -2 * sqrt(q);
    x[0] = q * cos(t / 3) - aa;
    x[1] = q * cos((t + TwoPi) / 3) - aa;
    x[2] = q * cos((t - TwoPi) / 3) - aa;
    nroot = 3;
  } else {
    double A = -pow(fabs(r) + sqrt(r2 - q3), 1. / 3);
    if (r < 0) A = -A;
    double B = (A == 0) ? 0 : q / A;
    aa /= 3;
    x[0] = (A + B) - aa;
    x[1] = -0.5 * (A + B) - aa;
    x[2] = 0.5 * sqrt(3.) * (A - B);
    if (fabs(x[2]) < eps) { x[2] = x[1]; nroot = 2; } else nroot = 1;
  }
  double tt;
  if (nroot == 3 || nroot == 2) {
    // sort three values ascending (std::sort on 3 doubles without NaN)
    double u0 = x[0], u1 = x[1], u2 = x[2], t;
    if (u1 < u0) { t = u0; u0 = u1; u1 = t; }
    if (u2 < u1) { t = u1; u1 = u2; u2 = t; }
    if (u1 < u0) { t = u0; u0 = u1; u1 = t; }
    tt = u0;
    if ((tt < 0) || (tt > dtmd)) {
      tt = u1;
      if ((tt < 0) || (tt > dtmd)) tt = u2;
    }
  } else {
    tt = x[0];
  }
  return tt;
}

}  // namespace irbc
