// kernels.cu -- sm_100a kernels of the FP64 timestep.
//
// Every expression keeps the operand order of the reference function it
// restates (compiled with --fmad=false), so the FP64 results agree with the
// reference to the last bit wherever only + - * / sqrt are involved, and to
// the last-ulp differences of the libm transcendentals (cos, sin, acos, pow,
// exp, log) elsewhere.
#include <cstdio>
#include "sim.h"
#include "multi.h"
#include "cells_tile.cuh"

namespace irbc {

static inline unsigned nblk(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

// ================================================================ set-up ====
// solvent positions and velocities, maincode.cpp:96-107: draw 6j+k of the
// INIT stream is component k of particle j
__global__ void k_init_solvent(DevParams p, Solvent s) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= s.n) return;
  const double vmax = sqrt(3.0 * p.Theta / p.mass);
  const uint64_t b = 6 * (uint64_t)i;
  s.x[i] = (p.Lx * draw_uniform(p.seed, STREAM_INIT, 0, b + 0));
  s.y[i] = (p.Ly * draw_uniform(p.seed, STREAM_INIT, 0, b + 1));
  s.z[i] = (p.Lz * draw_uniform(p.seed, STREAM_INIT, 0, b + 2));
  SolVel r;
  r.vx = -vmax + 2.0 * vmax * draw_uniform(p.seed, STREAM_INIT, 0, b + 3);
  r.vy = -vmax + 2.0 * vmax * draw_uniform(p.seed, STREAM_INIT, 0, b + 4);
  r.vz = -vmax + 2.0 * vmax * draw_uniform(p.seed, STREAM_INIT, 0, b + 5);
  r.id = (int)i;
  r.pad = 0;
  s.v[i] = r;
  s.indio[i] = 1;
  s.pid[i] = 0;
}

__global__ void k_set_u64(uint64_t* d, uint64_t v) { *d = v; }
void launch_set_u64(uint64_t* d, uint64_t v, cudaStream_t st) { k_set_u64<<<1, 1, 0, st>>>(d, v); }

void launch_init_solvent(const DevParams& p, Solvent& s, cudaStream_t st) {
  if (s.n) k_init_solvent<<<nblk(s.n, 256), 256, 0, st>>>(p, s);
}

__global__ void k_pack_vel(Solvent s, const double* vx, const double* vy, const double* vz, const int* id) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= s.n) return;
  SolVel r = s.v[i];
  if (vx) { r.vx = vx[i]; r.vy = vy[i]; r.vz = vz[i]; }
  if (id) r.id = id[i];
  r.pad = 0;
  s.v[i] = r;
}
__global__ void k_unpack_vel(Solvent s, double* vx, double* vy, double* vz, int* id) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= s.n) return;
  const SolVel r = s.v[i];
  if (vx) { vx[i] = r.vx; vy[i] = r.vy; vz[i] = r.vz; }
  if (id) id[i] = r.id;
}
__global__ void k_iota(int* d, int64_t n) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) d[i] = (int)i;
}
void launch_iota(int* d, int64_t n, cudaStream_t st) {
  if (n > 0) k_iota<<<nblk(n, 256), 256, 0, st>>>(d, n);
}
void launch_pack_vel(Solvent& s, const double* vx, const double* vy, const double* vz, const int* id,
                     cudaStream_t st) {
  if (s.n) k_pack_vel<<<nblk(s.n, 256), 256, 0, st>>>(s, vx, vy, vz, id);
}
void launch_unpack_vel(const Solvent& s, double* vx, double* vy, double* vz, int* id, cudaStream_t st) {
  if (s.n) k_unpack_vel<<<nblk(s.n, 256), 256, 0, st>>>(s, vx, vy, vz, id);
}

// the solvent in reference order (get_state): particle i goes to position
// id of the second buffer set; velocities = 0 moves positions, cell and
// flag, velocities = 1 moves the velocities into x2, y2, z2.  Ids out of
// range are counted in *bad and skipped.
__global__ void k_unpermute(Solvent s, int velocities, int* bad) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= s.n) return;
  const SolVel r = s.v[i];
  const int id = r.id;
  if (id < 0 || id >= s.n) {
    atomicAdd(bad, 1);
    return;
  }
  if (velocities) {
    s.x2[id] = r.vx; s.y2[id] = r.vy; s.z2[id] = r.vz;
  } else {
    s.x2[id] = s.x[i]; s.y2[id] = s.y[i]; s.z2[id] = s.z[i];
    s.pid2[id] = s.pid[i]; s.indio2[id] = s.indio[i];
  }
}
void launch_unpermute(const Solvent& s, int velocities, int* bad, cudaStream_t st) {
  if (s.n) k_unpermute<<<nblk(s.n, 256), 256, 0, st>>>(s, velocities, bad);
}

// inside/outside ray test, sortsolvent_initial1 (Src/solfuncs.cpp:31-94).
// Triangle data staged in shared memory tiles: normal X (Normaldt), the
// three corners and the centroid x (tries[].cmx).
constexpr int kTriTile = 128;
__global__ void k_classify(DevParams p, Solvent s, Membrane m, const double* tri) {
  __shared__ double sh[kTriTile * 13];
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double px = 0, py = 0, pz = 0;
  if (i < s.n) { px = s.x[i]; py = s.y[i]; pz = s.z[i]; }
  const double Rd0 = 1.0, Rd1 = 0.0, Rd2 = 0.0;
  double Q1[3] = {px + Rd0 * 0.3, py + Rd1 * 0.3, pz + Rd2 * 0.3};
  double Q2[3] = {px + Rd0 * 0.7, py + Rd1 * 0.7, pz + Rd2 * 0.7};
  int count = 0;
  for (int t0 = 0; t0 < p.nt; t0 += kTriTile) {
    int nt = min(kTriTile, p.nt - t0);
    __syncthreads();
    for (int q = threadIdx.x; q < nt * 13; q += blockDim.x) sh[q] = tri[(int64_t)t0 * 13 + q];
    __syncthreads();
    for (int j = 0; j < nt; ++j) {
      const double* T = sh + j * 13;
      const double X[3] = {T[0], T[1], T[2]};
      const double v1[3] = {T[3], T[4], T[5]}, v2[3] = {T[6], T[7], T[8]}, v3[3] = {T[9], T[10], T[11]};
      double dotP1Q1 = (v1[0] - Q1[0]) * X[0] + (v1[1] - Q1[1]) * X[1] + (v1[2] - Q1[2]) * X[2];
      double dotQ2Q1 = (Q2[0] - Q1[0]) * X[0] + (Q2[1] - Q1[1]) * X[1] + (Q2[2] - Q1[2]) * X[2];
      double P0[3];
      for (int k = 0; k < 3; ++k) P0[k] = Q1[k] + ((dotP1Q1 / dotQ2Q1) * (Q2[k] - Q1[k]));
      double P2P1[3] = {v2[0] - v1[0], v2[1] - v1[1], v2[2] - v1[2]};
      double P3P2[3] = {v3[0] - v2[0], v3[1] - v2[1], v3[2] - v2[2]};
      double P1P3[3] = {v1[0] - v3[0], v1[1] - v3[1], v1[2] - v3[2]};
      double P0P1[3] = {P0[0] - v1[0], P0[1] - v1[1], P0[2] - v1[2]};
      double P0P2[3] = {P0[0] - v2[0], P0[1] - v2[1], P0[2] - v2[2]};
      double P0P3[3] = {P0[0] - v3[0], P0[1] - v3[1], P0[2] - v3[2]};
      double f1[3], f2[3], f3[3];
      cp(P2P1, P0P1, f1); cp(P3P2, P0P2, f2); cp(P1P3, P0P3, f3);
      double ch1 = f1[0] * X[0] + f1[1] * X[1] + f1[2] * X[2];
      double ch2 = f2[0] * X[0] + f2[1] * X[1] + f2[2] * X[2];
      double ch3 = f3[0] * X[0] + f3[1] * X[1] + f3[2] * X[2];
      if ((ch1 >= 0) && (ch2 >= 0) && (ch3 >= 0) && (T[12] >= px)) count += 1;
    }
  }
  if (i < s.n) s.indio[i] = ((count % 2) == 0) ? 1 : 0;
}

__global__ void k_classify_tri(DevParams p, Membrane m, double* tri) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= p.nt) return;
  int p1 = m.t1[j], p2 = m.t2[j], p3 = m.t3[j];
  const double Lx = p.Lx, Ly = p.Ly;
  double A[3], B[3], X[3];
  A[0] = (m.x[p2] + m.ix[p2] * Lx) - (m.x[p1] + m.ix[p1] * Lx);
  A[1] = (m.y[p2] + m.iy[p2] * Ly) - (m.y[p1] + m.iy[p1] * Ly);
  A[2] = m.z[p2] - m.z[p1];
  B[0] = (m.x[p3] + m.ix[p3] * Lx) - (m.x[p1] + m.ix[p1] * Lx);
  B[1] = (m.y[p3] + m.iy[p3] * Ly) - (m.y[p1] + m.iy[p1] * Ly);
  B[2] = m.z[p3] - m.z[p1];
  cp(A, B, X);
  double* T = tri + (int64_t)j * 13;
  T[0] = X[0]; T[1] = X[1]; T[2] = X[2];
  T[3] = m.x[p1]; T[4] = m.y[p1]; T[5] = m.z[p1];
  T[6] = m.x[p2]; T[7] = m.y[p2]; T[8] = m.z[p2];
  T[9] = m.x[p3]; T[10] = m.y[p3]; T[11] = m.z[p3];
  // tricm (Src/memfuncs.cpp:25,28)
  double cmx = ((m.x[p1] + m.ix[p1] * Lx) + (m.x[p2] + m.ix[p2] * Lx) + (m.x[p3] + m.ix[p3] * Lx)) / 3.0;
  T[12] = fmod(cmx, Lx);
}

void launch_classify(const DevParams& p, Solvent& s, const Membrane& m, cudaStream_t st) {
  double* tri = nullptr;
  cudaMallocAsync(&tri, sizeof(double) * 13 * (size_t)p.nt, st);
  k_classify_tri<<<nblk(p.nt, 128), 128, 0, st>>>(p, m, tri);
  if (s.n) k_classify<<<nblk(s.n, 256), 256, 0, st>>>(p, s, m, tri);
  cudaFreeAsync(tri, st);
}

// ================================================================ scan ======
// Exclusive scan of up to three int arrays at once (null input = zeros):
// per-block sums, one block scanning the block sums, then the per-block
// rescan with offsets.  totals[k] receives the sum of array k.
constexpr int kScanT = 256, kScanItems = 4, kScanTile = kScanT * kScanItems;

int64_t scan_part_blocks(int64_t n) { return (n + kScanTile - 1) / kScanTile; }

__device__ __forceinline__ int ld0(const int* a, int64_t i) { return a ? a[i] : 0; }

__device__ __forceinline__ void scan_part_block(const int* a, const int* b, const int* c, int64_t n, int* part,
                                                int64_t bid) {
  int64_t base = bid * kScanTile + threadIdx.x * kScanItems;
  int s[3] = {0, 0, 0};
  for (int q = 0; q < kScanItems; ++q) {
    int64_t i = base + q;
    if (i < n) { s[0] += ld0(a, i); s[1] += ld0(b, i); s[2] += ld0(c, i); }
  }
  for (int k = 0; k < 3; ++k) {
    int x = s[k];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    s[k] = x;
  }
  __shared__ int ws[3][kScanT / 32];
  if ((threadIdx.x & 31) == 0)
    for (int k = 0; k < 3; ++k) ws[k][threadIdx.x >> 5] = s[k];
  __syncthreads();
  if (threadIdx.x < 3) {
    int t = 0;
    for (int q = 0; q < kScanT / 32; ++q) t += ws[threadIdx.x][q];
    part[bid * 3 + threadIdx.x] = t;
  }
}
__global__ void k_scan_part(const int* a, const int* b, const int* c, int64_t n, int* part) {
  scan_part_block(a, b, c, n, part, blockIdx.x);
}

// one block: exclusive scan of the block sums in place, totals out
__device__ __forceinline__ void scan_top_block(int* part, int64_t nb, int* totals) {
  __shared__ int carry[3];
  if (threadIdx.x < 3) carry[threadIdx.x] = 0;
  __syncthreads();
  for (int64_t b0 = 0; b0 < nb; b0 += blockDim.x) {
    int64_t b = b0 + threadIdx.x;
    for (int k = 0; k < 3; ++k) {
      int x = b < nb ? part[b * 3 + k] : 0;
      int orig = x;
      const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
      for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
      }
      __shared__ int ws[32];
      if (lane == 31) ws[w] = x;
      __syncthreads();
      if (w == 0) {
        int y = lane < (int)(blockDim.x >> 5) ? ws[lane] : 0;
        int yo = y;
        for (int o = 1; o < 32; o <<= 1) {
          int z = __shfl_up_sync(0xffffffffu, y, o);
          if (lane >= o) y += z;
        }
        if (lane < (int)(blockDim.x >> 5)) ws[lane] = y - yo;
      }
      __syncthreads();
      int excl = x - orig + ws[w] + carry[k];
      if (b < nb) part[b * 3 + k] = excl;
      __syncthreads();
      if (threadIdx.x == blockDim.x - 1) carry[k] = excl + orig;
      __syncthreads();
    }
  }
  if (threadIdx.x < 3 && totals) totals[threadIdx.x] = carry[threadIdx.x];
}
__global__ void k_scan_top(int* part, int64_t nb, int* totals) { scan_top_block(part, nb, totals); }

__device__ __forceinline__ void scan_final_block(const int* a, const int* b, const int* c, int* oa, int* ob, int* oc,
                                                 int64_t n, const int* part, int64_t bid) {
  int64_t base = bid * kScanTile + threadIdx.x * kScanItems;
  int loc[3][kScanItems];
  int s[3] = {0, 0, 0};
  for (int q = 0; q < kScanItems; ++q) {
    int64_t i = base + q;
    int va = i < n ? ld0(a, i) : 0, vb = i < n ? ld0(b, i) : 0, vc = i < n ? ld0(c, i) : 0;
    loc[0][q] = s[0]; loc[1][q] = s[1]; loc[2][q] = s[2];
    s[0] += va; s[1] += vb; s[2] += vc;
  }
  // exclusive scan of per-thread sums across the block
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __shared__ int ws[3][kScanT / 32];
  int ex[3];
  for (int k = 0; k < 3; ++k) {
    int x = s[k];
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) ws[k][w] = x;
    ex[k] = x - s[k];
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    int acc = 0;
    for (int q = 0; q < kScanT / 32; ++q) { int t = ws[threadIdx.x][q]; ws[threadIdx.x][q] = acc; acc += t; }
  }
  __syncthreads();
  for (int k = 0; k < 3; ++k) ex[k] += ws[k][w] + part[bid * 3 + k];
  for (int q = 0; q < kScanItems; ++q) {
    int64_t i = base + q;
    if (i < n) {
      if (oa) oa[i] = ex[0] + loc[0][q];
      if (ob) ob[i] = ex[1] + loc[1][q];
      if (oc) oc[i] = ex[2] + loc[2][q];
    }
  }
}
__global__ void k_scan_final(const int* a, const int* b, const int* c, int* oa, int* ob, int* oc,
                             int64_t n, const int* part) {
  scan_final_block(a, b, c, oa, ob, oc, n, part, blockIdx.x);
}

void launch_scan3(const int* a, const int* b, const int* c, int* oa, int* ob, int* oc, int* totals,
                  int64_t n, int* part, cudaStream_t st) {
  int64_t nb = scan_part_blocks(n);
  if (nb == 0) return;
  k_scan_part<<<(unsigned)nb, kScanT, 0, st>>>(a, b, c, n, part);
  k_scan_top<<<1, 1024, 0, st>>>(part, nb, totals);
  k_scan_final<<<(unsigned)nb, kScanT, 0, st>>>(a, b, c, oa, ob, oc, n, part);
}

// ============================================================== collide =====
// CollisionStep (Src/solfuncs.cpp:109-323) as: vertex binning + shift,
// counting sort of the solvent (count -> scan -> scatter), then one warp per
// tile of 32 cells for the cell statistics in reference order and the
// rotation (CollisionDyn, :700-736; cells_tile.cuh).

__device__ __forceinline__ int shifted_cell(const DevParams& p, double x, double y, double z, const double r[3]) {
  int fx = (int)floor(bbound(x - r[0], p.Lx));
  int fy = (int)floor(bbound(y - r[1], p.Ly));
  int fz = (int)floor(z - r[2] + 1.0);
  return cell_of(p, fx, fy, fz);
}

// vertices and parasite into the shifted grid (:149-162); vertex keys sorted
// by (cell, vertex) with a bitonic sort in shared memory
__device__ __forceinline__ void vbin_block(const DevParams& p, const Membrane& m, int* ncm, uint64_t eoff) {
  const uint64_t epoch = epoch_of(p, eoff);
  extern __shared__ uint64_t sk[];
  double r[3];
  grid_shift(p, epoch, r);
  int n2 = 1;
  while (n2 < p.nv) n2 <<= 1;
  for (int i = threadIdx.x; i < n2; i += blockDim.x) {
    if (i < p.nv) {
      int c = shifted_cell(p, m.x[i], m.y[i], m.z[i], r);
      m.pid[i] = c;
      atomicAdd(&ncm[c], 1);
      sk[i] = ((uint64_t)(uint32_t)c << 32) | (uint32_t)i;
    } else {
      sk[i] = ~0ull;
    }
  }
  if (threadIdx.x == 0) {
    MemScalars* sc = m.sc;
    sc->paraid = shifted_cell(p, sc->para[0], sc->para[1], sc->para[2], r);
  }
  __syncthreads();
  for (int k = 2; k <= n2; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < n2; i += blockDim.x) {
        int l = i ^ j;
        if (l > i) {
          uint64_t a = sk[i], b = sk[l];
          bool up = ((i & k) == 0);
          if ((a > b) == up) { sk[i] = b; sk[l] = a; }
        }
      }
      __syncthreads();
    }
  }
  for (int i = threadIdx.x; i < p.nv; i += blockDim.x) m.vkey[i] = sk[i];
}
__global__ void k_vbin(DevParams p, Membrane m, int* ncm, uint64_t eoff) { vbin_block(p, m, ncm, eoff); }

// cell of each particle in the shifted grid; warp-aggregated slot counters
__global__ void __launch_bounds__(256) k_count(DevParams p, Solvent s, int* cnt, uint64_t eoff) {
  const uint64_t epoch = epoch_of(p, eoff);
  // the grid shift, drawn once per block
  __shared__ double sr[3];
  if (threadIdx.x == 0) grid_shift(p, epoch, sr);
  __syncthreads();
  const double r[3] = {sr[0], sr[1], sr[2]};
  // kCountPer particles per thread, a block's particles contiguous: every
  // thread's loads first, then the slot claims, so that the memory
  // latencies overlap
  const int64_t i0 = (int64_t)blockIdx.x * blockDim.x * kCountPer + threadIdx.x;
  int c[kCountPer];
#pragma unroll
  for (int u = 0; u < kCountPer; ++u) {
    const int64_t i = i0 + (int64_t)u * blockDim.x;
    c[u] = i < s.n ? shifted_cell(p, s.x[i], s.y[i], s.z[i], r) : -1;
  }
  int slot[kCountPer];
  claim_slots<kCountPer>(cnt, c, i0, blockDim.x, s.n, slot);
#pragma unroll
  for (int u = 0; u < kCountPer; ++u) {
    const int64_t i = i0 + (int64_t)u * blockDim.x;
    if (i < s.n) {
      s.pid[i] = c[u];  // the cell of this collision (particle.pid)
      s.slot[i] = slot[u];
    }
  }
}

// ghost flags for the scan: wall cells (zmax >= Lz or zmin <= 0) with fewer
// than navg solvent particles (:185-204), and membrane cells with fewer
// than navg particles of any kind (:236-244)
__device__ __forceinline__ void ghost_flags_item(const DevParams& p, const int* cnt, const int* ncm,
                                                 const MemScalars* sc, int* wflag, int* mflag, int64_t c) {
  if (c >= p.ncell) return;
  int k = (int)(c % p.nz);
  double zmin = -1.0 + (double)k * p.a, zmax = -1.0 + (double)k * p.a + p.a;
  int nn = cnt[c];
  int wall = ((zmax >= p.Lz) || (zmin <= 0)) && (nn < p.navg);
  int nt = nn + ncm[c] + (c == sc->paraid ? 1 : 0);
  int mem = (ncm[c] > 0) && (nt < p.navg);
  wflag[c] = wall;
  mflag[c] = mem;
}
__global__ void k_ghost_flags(DevParams p, const int* cnt, const int* ncm, const MemScalars* sc,
                              int* wflag, int* mflag) {
  ghost_flags_item(p, cnt, ncm, sc, wflag, mflag, (int64_t)blockIdx.x * blockDim.x + threadIdx.x);
}

// counting sort of particle indices: perm[start[cell] + slot] = i
__global__ void k_perm(const int* __restrict__ key, const int* __restrict__ slot, const int* __restrict__ start,
                       int64_t n, int* __restrict__ perm) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  perm[(int64_t)start[key[i]] + slot[i]] = (int)i;
}

// physical re-sort by collision cell (every few collisions, to keep the
// particles of a cell close in memory): gathered into the second buffer set,
// then copied back, so the arrays never change address (a captured step
// sequence stays valid)
__global__ void k_gather(Solvent s) {
  int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= s.n) return;
  const int i = s.perm[j];
  s.x2[j] = s.x[i]; s.y2[j] = s.y[i]; s.z2[j] = s.z[i];
  s.v2[j] = s.v[i];
  s.indio2[j] = s.indio[i]; s.pid2[j] = s.pid[i];
}
__global__ void k_copy_back(Solvent s) {
  int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= s.n) return;
  s.x[j] = s.x2[j]; s.y[j] = s.y2[j]; s.z[j] = s.z2[j];
  s.v[j] = s.v2[j];
  s.indio[j] = s.indio2[j]; s.pid[j] = s.pid2[j];
}


void launch_vbin(const DevParams& p, Membrane& m, Cells& c, uint64_t epoch, cudaStream_t st) {
  int n2 = 1;
  while (n2 < p.nv) n2 <<= 1;
  cudaMemsetAsync(c.ncm, 0, sizeof(int) * c.n, st);
  k_vbin<<<1, 1024, sizeof(uint64_t) * n2, st>>>(p, m, c.ncm, epoch);
}

void launch_ghost_flags(const DevParams& p, Cells& c, const Membrane& m, cudaStream_t st) {
  k_ghost_flags<<<nblk(c.n, 256), 256, 0, st>>>(p, c.cnt, c.ncm, m.sc, c.wrank, c.mrank);
}

void launch_collide_count(const DevParams& p, Solvent& s, Cells& c, uint64_t epoch, cudaStream_t st) {
  cudaMemsetAsync(c.cnt, 0, sizeof(int) * c.n, st);
  if (s.n) k_count<<<nblk(s.n, 256 * kCountPer), 256, 0, st>>>(p, s, c.cnt, epoch);
}

void launch_collide_finish(const DevParams& p, Solvent& s, Cells& c, Membrane& m, uint64_t epoch,
                           cudaStream_t st, bool resort) {
  // wrank/mrank hold the flags first, then their exclusive scans
  k_ghost_flags<<<nblk(c.n, 256), 256, 0, st>>>(p, c.cnt, c.ncm, m.sc, c.wrank, c.mrank);
  launch_scan3(c.cnt, c.wrank, c.mrank, c.start, c.wrank, c.mrank, c.totals, c.n, c.scan_part, st);
  // start[C] = Ns
  cudaMemcpyAsync(c.start + c.n, c.totals + 0, sizeof(int), cudaMemcpyDeviceToDevice, st);
  if (s.n) k_perm<<<nblk(s.n, 256), 256, 0, st>>>(s.pid, s.slot, c.start, s.n, s.perm);
  k_cells_tile<false><<<cells_tile_blocks(c.n), 32 * kTileWarps, 0, st>>>(p, s, SolventF{}, c, m, epoch);
  if (resort) launch_resort(s, st);
}

void launch_resort(Solvent& s, cudaStream_t st) {
  if (s.n) {
    k_gather<<<nblk(s.n, 256), 256, 0, st>>>(s);
    k_copy_back<<<nblk(s.n, 256), 256, 0, st>>>(s);
  }
}

// ============================================================== stream =====
// Streaming with bounce-back: reflectionFed(i, 0) (Src/solfuncs.cpp:400-598)
// then the wall treatment and wrap of maincode.cpp:515-560.  The cubic
// contact-time solver solve_p3_tt is in common.cuh.
struct VertexView {
  const double *x, *y, *z, *vx, *vy, *vz;
};

__device__ double reflection(const DevParams& p, const int* lstart, const int* lidx, const Membrane& m,
                             double& X_, double& Y_, double& Z_, double& VX, double& VY, double& VZ, int indio) {
  const double rstep = 0.0, dtmd = p.dtmd, a = p.a, Lx = p.Lx, Ly = p.Ly;
  double fulldt = rstep;
  int fx = (int)floor(bbound(X_, Lx));
  int fy = (int)floor(bbound(Y_, Ly));
  int fz = (int)floor(Z_ + 1.0);
  int pid = cell_of(p, fx, fy, fz);
  const int l0 = lstart[pid], l1 = lstart[pid + 1];
  for (int j = l0; j < l1; ++j) {
    int flg = 0;
    int jj = lidx[j];
    int p1 = m.t1[jj], p2 = m.t2[jj], p3 = m.t3[jj];
    const int xx = 0, yy = 0, p1modx = 0, p2modx = 0, p3modx = 0, p1mody = 0, p2mody = 0, p3mody = 0;
    double solvx = X_ + xx * Lx;
    double solvy = Y_ + yy * Ly;
    double solvz = Z_;
    double v1x = (m.x[p1] + p1modx * Lx) + m.vx[p1] * rstep;
    double v1y = (m.y[p1] + p1mody * Ly) + m.vy[p1] * rstep;
    double v1z = m.z[p1] + m.vz[p1] * rstep;
    double v2x = (m.x[p2] + p2modx * Lx) + m.vx[p2] * rstep;
    double v2y = (m.y[p2] + p2mody * Ly) + m.vy[p2] * rstep;
    double v2z = m.z[p2] + m.vz[p2] * rstep;
    double v3x = (m.x[p3] + p3modx * Lx) + m.vx[p3] * rstep;
    double v3y = (m.y[p3] + p3mody * Ly) + m.vy[p3] * rstep;
    double v3z = m.z[p3] + m.vz[p3] * rstep;
    double rstencilx = Lx - (3.0 * a), lstencilx = 3.0 * a;
    double rstencily = Ly - (3.0 * a), lstencily = 3.0 * a;
    if (solvx < lstencilx) {
      v1x -= (v1x > rstencilx) ? Lx : 0;
      v2x -= (v2x > rstencilx) ? Lx : 0;
      v3x -= (v3x > rstencilx) ? Lx : 0;
    } else if (solvx > rstencilx) {
      v1x += (v1x < lstencilx) ? Lx : 0;
      v2x += (v2x < lstencilx) ? Lx : 0;
      v3x += (v3x < lstencilx) ? Lx : 0;
    }
    if (solvy < lstencily) {
      v1y -= (v1y > rstencily) ? Ly : 0;
      v2y -= (v2y > rstencily) ? Ly : 0;
      v3y -= (v3y > rstencily) ? Ly : 0;
    } else if (solvy > rstencily) {
      v1y += (v1y < lstencily) ? Ly : 0;
      v2y += (v2y < lstencily) ? Ly : 0;
      v3y += (v3y < lstencily) ? Ly : 0;
    }
    const double mvx1 = m.vx[p1], mvy1 = m.vy[p1], mvz1 = m.vz[p1];
    const double mvx2 = m.vx[p2], mvy2 = m.vy[p2], mvz2 = m.vz[p2];
    const double mvx3 = m.vx[p3], mvy3 = m.vy[p3], mvz3 = m.vz[p3];
    double w1x = v1x + mvx1 * (dtmd - rstep), w1y = v1y + mvy1 * (dtmd - rstep), w1z = v1z + mvz1 * (dtmd - rstep);
    double w2x = v2x + mvx2 * (dtmd - rstep), w2y = v2y + mvy2 * (dtmd - rstep), w2z = v2z + mvz2 * (dtmd - rstep);
    double w3x = v3x + mvx3 * (dtmd - rstep), w3y = v3y + mvy3 * (dtmd - rstep), w3z = v3z + mvz3 * (dtmd - rstep);
    double X[3], Xdt[3], t0[3], t1v[3];
    t0[0] = v2x - v1x; t0[1] = v2y - v1y; t0[2] = v2z - v1z;
    t1v[0] = v3x - v1x; t1v[1] = v3y - v1y; t1v[2] = v3z - v1z;
    cp(t0, t1v, X);
    t0[0] = w2x - w1x; t0[1] = w2y - w1y; t0[2] = w2z - w1z;
    t1v[0] = w3x - w1x; t1v[1] = w3y - w1y; t1v[2] = w3z - w1z;
    cp(t0, t1v, Xdt);
    double PSt[3], PSdt[3];
    PSt[0] = solvx - v1x; PSt[1] = solvy - v1y; PSt[2] = solvz - v1z;
    PSdt[0] = (solvx + VX * (dtmd - rstep)) - w1x;
    PSdt[1] = (solvy + VY * (dtmd - rstep)) - w1y;
    PSdt[2] = (solvz + VZ * (dtmd - rstep)) - w1z;
    double bt = X[0] * PSt[0] + X[1] * PSt[1] + X[2] * PSt[2];
    double bdt = Xdt[0] * PSdt[0] + Xdt[1] * PSdt[1] + Xdt[2] * PSdt[2];
    if ((indio == 1) && (bt < 0)) flg = 1;
    if ((indio == 0) && (bt > 0)) flg = 1;
    if ((bt * bdt <= 0) && (flg == 0)) {
      double a10[3], a20[3], d1[3], d2[3], a2v[3], b1[3], b2[3], b3[3], d11[3], d22[3];
      a10[0] = v2x - v1x; a10[1] = v2y - v1y; a10[2] = v2z - v1z;
      a20[0] = v3x - v1x; a20[1] = v3y - v1y; a20[2] = v3z - v1z;
      d1[0] = mvx2 - mvx1; d1[1] = mvy2 - mvy1; d1[2] = mvz2 - mvz1;
      d2[0] = mvx3 - mvx1; d2[1] = mvy3 - mvy1; d2[2] = mvz3 - mvz1;
      const double* a1v = PSt;
      a2v[0] = VX - mvx1; a2v[1] = VY - mvy1; a2v[2] = VZ - mvz1;
      cp(a10, a20, b1);
      cp(a10, d2, d11);
      cp(d1, a20, d22);
      cp(d1, d2, b3);
      for (int k = 0; k < 3; ++k) b2[k] = d11[k] + d22[k];
      double a2b3 = a2v[0] * b3[0] + a2v[1] * b3[1] + a2v[2] * b3[2];
      double a1b3 = a1v[0] * b3[0] + a1v[1] * b3[1] + a1v[2] * b3[2];
      double a2b2 = a2v[0] * b2[0] + a2v[1] * b2[1] + a2v[2] * b2[2];
      double a1b2 = a1v[0] * b2[0] + a1v[1] * b2[1] + a1v[2] * b2[2];
      double a2b1 = a2v[0] * b1[0] + a2v[1] * b1[1] + a2v[2] * b1[2];
      double a1b1 = a1v[0] * b1[0] + a1v[1] * b1[1] + a1v[2] * b1[2];
      double tt = solve_p3_tt((a1b3 + a2b2) / a2b3, (a1b2 + a2b1) / a2b3, a1b1 / a2b3, dtmd);
      double pd[3], vd[3], PS2[3];
      PS2[0] = (solvx + VX * tt) - (v1x + mvx1 * tt);
      PS2[1] = (solvy + VY * tt) - (v1y + mvy1 * tt);
      PS2[2] = (solvz + VZ * tt) - (v1z + mvz1 * tt);
      pd[0] = (solvx + VX * tt);
      pd[1] = (solvy + VY * tt);
      pd[2] = (solvz + VZ * tt);
      a10[0] = (v2x + mvx2 * tt) - (v1x + mvx1 * tt);
      a10[1] = (v2y + mvy2 * tt) - (v1y + mvy1 * tt);
      a10[2] = (v2z + mvz2 * tt) - (v1z + mvz1 * tt);
      a20[0] = (v3x + mvx3 * tt) - (v1x + mvx1 * tt);
      a20[1] = (v3y + mvy3 * tt) - (v1y + mvy1 * tt);
      a20[2] = (v3z + mvz3 * tt) - (v1z + mvz1 * tt);
      double pa1 = PS2[0] * a10[0] + PS2[1] * a10[1] + PS2[2] * a10[2];
      double pa2 = PS2[0] * a20[0] + PS2[1] * a20[1] + PS2[2] * a20[2];
      double a1a2 = a10[0] * a20[0] + a10[1] * a20[1] + a10[2] * a20[2];
      double a12 = a10[0] * a10[0] + a10[1] * a10[1] + a10[2] * a10[2];
      double a22 = a20[0] * a20[0] + a20[1] * a20[1] + a20[2] * a20[2];
      double den = (a12 * a22) - (a1a2 * a1a2);
      double eta = ((pa1 * a22) - (pa2 * a1a2)) / den;
      double zeta = ((pa2 * a12) - (pa1 * a1a2)) / den;
      if ((eta >= 0) && (zeta >= 0) && (eta + zeta <= 1) && (tt < (dtmd - rstep))) {
        fulldt += tt;
        vd[0] = (1.0 - eta - zeta) * mvx1 + eta * mvx2 + zeta * mvx3;
        vd[1] = (1.0 - eta - zeta) * mvy1 + eta * mvy2 + zeta * mvy3;
        vd[2] = (1.0 - eta - zeta) * mvz1 + eta * mvz2 + zeta * mvz3;
        VX = 2.0 * vd[0] - VX;
        VY = 2.0 * vd[1] - VY;
        VZ = 2.0 * vd[2] - VZ;
        X_ = pd[0]; Y_ = pd[1]; Z_ = pd[2];
      }
    }
  }
  return fulldt;
}

__global__ void k_stream(DevParams p, Solvent s, const int* lstart, const int* lidx, Membrane m) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= s.n) return;
  const SolVel r = s.v[i];
  double X = s.x[i], Y = s.y[i], Z = s.z[i], VX = r.vx, VY = r.vy, VZ = r.vz;
  const double VX0 = VX, VY0 = VY, VZ0 = VZ;
  const double dtmd = p.dtmd;
  double fullts = reflection(p, lstart, lidx, m, X, Y, Z, VX, VY, VZ, s.indio[i]);
  X += VX * (dtmd - fullts);
  Y += VY * (dtmd - fullts);
  Z += VZ * (dtmd - fullts);
  const double ul = p.Lz, ll = 0;
  if (Z > ul || Z < ll) {
    double A[3], B[3];
    const double wall = Z > ul ? ul : ll;
    A[0] = X - VX * (dtmd - fullts); A[1] = Y - VY * (dtmd - fullts); A[2] = Z - VZ * (dtmd - fullts);
    double sp = (wall - A[2]) / (Z - A[2]);
    B[0] = A[0] + sp * (X - A[0]); B[1] = A[1] + sp * (Y - A[1]); B[2] = A[2] + sp * (Z - A[2]);
    double dist = sqrt(((B[0] - A[0]) * (B[0] - A[0])) + ((B[1] - A[1]) * (B[1] - A[1])) + ((B[2] - A[2]) * (B[2] - A[2])));
    double dtt = dist / sqrt((VX * VX) + (VY * VY) + (VZ * VZ));
    if (Z > ul) {  // moving top wall: v = (wallspeed, 0, 0)
      VX = p.wallspeed; VY = 0; VZ = 0;
    } else {       // bounce-back bottom wall
      VX *= -1.0; VY *= -1.0; VZ *= -1.0;
    }
    X = B[0] + VX * ((dtmd - fullts) - dtt);
    Y = B[1] + VY * ((dtmd - fullts) - dtt);
    Z = B[2] + VZ * ((dtmd - fullts) - dtt);
  }
  X = bbound(X, p.Lx);
  Y = bbound(Y, p.Ly);
  s.x[i] = X; s.y[i] = Y; s.z[i] = Z;
  if (VX != VX0 || VY != VY0 || VZ != VZ0 || VX0 != VX0) { s.v[i].vx = VX; s.v[i].vy = VY; s.v[i].vz = VZ; }
}

void launch_stream(const DevParams& p, Solvent& s, const Cells& c, const Membrane& m, cudaStream_t st) {
  if (s.n) k_stream<<<nblk(s.n, 256), 256, 0, st>>>(p, s, c.lstart, c.lidx, m);
}

// ============================================================== llist ======
// llistupdate (Src/solfuncs.cpp:326-365): triangles whose centroid lies
// within 2a of the cell centre, with the list never shrinking (entries past
// the new count keep their old values).
__global__ void k_tri_centroid(DevParams p, Membrane m) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= p.nt) return;
  int p1 = m.t1[j], p2 = m.t2[j], p3 = m.t3[j];
  const double Lx = p.Lx, Ly = p.Ly;
  m.tcx[j] = fmod((((m.x[p1] + m.ix[p1] * Lx) + (m.x[p2] + m.ix[p2] * Lx) + (m.x[p3] + m.ix[p3] * Lx)) / 3.0), Lx);
  m.tcy[j] = fmod((((m.y[p1] + m.iy[p1] * Ly) + (m.y[p2] + m.iy[p2] * Ly) + (m.y[p3] + m.iy[p3] * Ly)) / 3.0), Ly);
  m.tcz[j] = (m.z[p1] + m.z[p2] + m.z[p3]) / 3.0;
}

// One block of kLTile consecutive cells per pass; each tile of kLTile
// centroids is first culled against the block's box of cell centres (a
// conservative box test with the same minimum-image convention), and the
// survivors, compacted in index order, get the exact test of :340-350.
constexpr int kLTile = 256;
template <bool FILL>
__global__ void __launch_bounds__(kLTile) k_llist(DevParams p, Cells cl, Membrane m) {
  __shared__ double tc[3][kLTile];
  __shared__ int tj[kLTile];
  __shared__ double red[6][kLTile / 32];
  __shared__ int wcnt[kLTile / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool act = c < p.ncell;
  double cellx = 0, celly = 0, cellz = 0;
  if (act) {
    int k = (int)(c % p.nz), j = (int)((c / p.nz) % p.ny), i = (int)(c / ((int64_t)p.nz * p.ny));
    double xmin = (double)i * p.a, xmax = (double)i * p.a + p.a;
    double ymin = (double)j * p.a, ymax = (double)j * p.a + p.a;
    double zmin = -1.0 + (double)k * p.a, zmax = -1.0 + (double)k * p.a + p.a;
    cellx = (xmin + xmax) * 0.5; celly = (ymin + ymax) * 0.5; cellz = (zmin + zmax) * 0.5;
  }
  // the block's box of cell centres: min of (x, y, z, -x, -y, -z)
  double bb[6] = {act ? cellx : 1e300, act ? celly : 1e300, act ? cellz : 1e300,
                  act ? -cellx : 1e300, act ? -celly : 1e300, act ? -cellz : 1e300};
  for (int o = 16; o > 0; o >>= 1)
    for (int e = 0; e < 6; ++e) bb[e] = fmin(bb[e], __shfl_xor_sync(0xffffffffu, bb[e], o));
  if (lane == 0)
    for (int e = 0; e < 6; ++e) red[e][w] = bb[e];
  __syncthreads();
  for (int e = 0; e < 6; ++e) {
    double v = red[e][0];
    for (int u = 1; u < kLTile / 32; ++u) v = fmin(v, red[e][u]);
    bb[e] = v;
  }
  const double xm = 0.5 * (bb[0] - bb[3]), hx = 0.5 * (-bb[3] - bb[0]);
  const double ym = 0.5 * (bb[1] - bb[4]), hy = 0.5 * (-bb[4] - bb[1]);
  const double zm = 0.5 * (bb[2] - bb[5]), hz = 0.5 * (-bb[5] - bb[2]);
  const double reach = 2.0 * p.a + 1e-6;
  int count = 0;
  int old_n = act ? cl.lstart[c + 1] - cl.lstart[c] : 0;
  int64_t out0 = (FILL && act) ? cl.lstart2[c] : 0;
  const double lim = 4.0 * p.a * p.a;
  for (int t0 = 0; t0 < p.nt; t0 += kLTile) {
    const int nt = min(kLTile, p.nt - t0);
    bool keep = false;
    double tx = 0, ty = 0, tz = 0;
    if ((int)threadIdx.x < nt) {
      tx = m.tcx[t0 + threadIdx.x]; ty = m.tcy[t0 + threadIdx.x]; tz = m.tcz[t0 + threadIdx.x];
      double dx = tx - xm, dy = ty - ym;
      dx -= p.Lx * round(dx / p.Lx);
      dy -= p.Ly * round(dy / p.Ly);
      keep = (fabs(dx) - hx < reach) && (fabs(dy) - hy < reach) && (fabs(tz - zm) - hz < reach);
    }
    const unsigned bal = __ballot_sync(0xffffffffu, keep);
    __syncthreads();  // the previous tile's survivors are consumed
    if (lane == 0) wcnt[w] = __popc(bal);
    __syncthreads();
    int off = 0, K = 0;
    for (int u = 0; u < kLTile / 32; ++u) { const int cu = wcnt[u]; off += (u < w) ? cu : 0; K += cu; }
    if (keep) {
      const int pos = off + __popc(bal & ((1u << lane) - 1));
      tc[0][pos] = tx; tc[1][pos] = ty; tc[2][pos] = tz;
      tj[pos] = t0 + threadIdx.x;
    }
    __syncthreads();
    if (act) {
      for (int q = 0; q < K; ++q) {
        double xxx1 = tc[0][q] - cellx;
        double yyy1 = tc[1][q] - celly;
        xxx1 -= p.Lx * round(xxx1 / p.Lx);
        yyy1 -= p.Ly * round(yyy1 / p.Ly);
        double zzz = fabs(tc[2][q] - cellz);
        double A1aa = xxx1 * xxx1 + yyy1 * yyy1 + zzz * zzz;
        if (A1aa < lim) {
          if (FILL) cl.lidx2[out0 + count] = tj[q];
          count += 1;
        }
      }
    }
  }
  if (!act) return;
  if (!FILL) {
    cl.lcnt[c] = count > old_n ? count : old_n;
  } else {
    const int64_t in0 = cl.lstart[c];
    for (int q = count; q < old_n; ++q) cl.lidx2[out0 + q] = cl.lidx[in0 + q];
  }
}

int64_t launch_llist_count(const DevParams& p, Cells& c, const Membrane& m, cudaStream_t st) {
  k_tri_centroid<<<nblk(p.nt, 128), 128, 0, st>>>(p, m);
  k_llist<false><<<nblk(c.n, kLTile), kLTile, 0, st>>>(p, c, m);
  launch_scan3(c.lcnt, nullptr, nullptr, c.lstart2, nullptr, nullptr, c.totals + 8, c.n, c.scan_part, st);
  int tot = 0;
  cudaMemcpyAsync(&tot, c.totals + 8, sizeof(int), cudaMemcpyDeviceToHost, st);
  cudaStreamSynchronize(st);
  cudaMemcpyAsync(c.lstart2 + c.n, c.totals + 8, sizeof(int), cudaMemcpyDeviceToDevice, st);
  return tot;
}

// the new lists are built in the second buffers (the old ones give the
// stale tails) and copied back, so the list arrays keep their addresses
void launch_llist_fill(const DevParams& p, Cells& c, const Membrane& m, int64_t total, cudaStream_t st) {
  k_llist<true><<<nblk(c.n, kLTile), kLTile, 0, st>>>(p, c, m);
  cudaMemcpyAsync(c.lstart, c.lstart2, sizeof(int) * (c.n + 1), cudaMemcpyDeviceToDevice, st);
  if (total > 0) cudaMemcpyAsync(c.lidx, c.lidx2, sizeof(int) * total, cudaMemcpyDeviceToDevice, st);
}

// cells with a non-empty list: their rank (lrank), the cell of each rank
// (acell), their number and the longest list (host copies nact, lmax)
__global__ void k_lflags(DevParams p, Cells cl) {
  int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= p.ncell) return;
  const int len = cl.lstart[c + 1] - cl.lstart[c];
  cl.lrank[c] = len > 0 ? 1 : 0;
  if (len > 0) atomicMax(cl.totals + 7, len);
}
__global__ void k_acell(DevParams p, Cells cl) {
  int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= p.ncell) return;
  if (cl.lstart[c + 1] > cl.lstart[c]) cl.acell[cl.lrank[c]] = (int)c;
}
int launch_llist_ranks(const DevParams& p, Cells& c, cudaStream_t st) {
  cudaMemsetAsync(c.totals + 7, 0, sizeof(int), st);
  k_lflags<<<nblk(c.n, 256), 256, 0, st>>>(p, c);
  launch_scan3(c.lrank, nullptr, nullptr, c.lrank, nullptr, nullptr, c.totals + 4, c.n, c.scan_part, st);
  k_acell<<<nblk(c.n, 256), 256, 0, st>>>(p, c);
  int h[4] = {0, 0, 0, 0};
  cudaMemcpyAsync(h, c.totals + 4, sizeof(h), cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) return -1;
  c.nact = h[0];
  c.lmax = h[3];
  return 5;
}

// ============================================================ membrane =====
#define UXm(v) (m.x[v] + m.ix[v] * p.Lx)
#define UYm(v) (m.y[v] + m.iy[v] * p.Ly)

// vertex half-kick and force reset (maincode.cpp:487-496)
__global__ void k_half_kick(DevParams p, Membrane m) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.nv) return;
  m.vx[i] += (m.fx[i] * p.dtmd / (2.0 * p.pmass));
  m.vy[i] += (m.fy[i] * p.dtmd / (2.0 * p.pmass));
  m.vz[i] += (m.fz[i] * p.dtmd / (2.0 * p.pmass));
  m.fx[i] = 0.0; m.fy[i] = 0.0; m.fz[i] = 0.0;
}
void launch_half_kick(const DevParams& p, Membrane& m, cudaStream_t st) {
  k_half_kick<<<nblk(p.nv, 128), 128, 0, st>>>(p, m);
}

// vertex drift with image counters (maincode.cpp:566-574, bboundmx/my
// Src/solfuncs.cpp:625-659) and parasite drift (:576-598)
__global__ void k_drift(DevParams p, Membrane m) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < p.nv) {
    double x = m.x[i], y = m.y[i], z = m.z[i];
    x += (m.vx[i] * p.dtmd);
    y += (m.vy[i] * p.dtmd);
    z += (m.vz[i] * p.dtmd);
    if (x > p.Lx) { x -= p.Lx; m.ix[i] += 1; }
    if (x < 0) { x += p.Lx; m.ix[i] -= 1; }
    if (y > p.Ly) { y -= p.Ly; m.iy[i] += 1; }
    if (y < 0) { y += p.Ly; m.iy[i] -= 1; }
    m.x[i] = x; m.y[i] = y; m.z[i] = z;
  }
  if (i == 0) {
    MemScalars* sc = m.sc;
    for (int k = 0; k < 3; ++k)
      sc->para[k] += (sc->paraV[k] * p.dtmd) + (sc->paraft[k] * p.dtmd * p.dtmd / (2.0 * p.PRmass));
    if (sc->para[0] > p.Lx) { sc->para[0] -= p.Lx; sc->paradx += 1; }
    else if (sc->para[0] < 0) { sc->para[0] += p.Lx; sc->paradx -= 1; }
    if (sc->para[1] > p.Ly) { sc->para[1] -= p.Ly; sc->parady += 1; }
    else if (sc->para[1] < 0) { sc->para[1] += p.Ly; sc->parady -= 1; }
  }
}
void launch_drift(const DevParams& p, Membrane& m, cudaStream_t st) {
  k_drift<<<nblk(p.nv, 128), 128, 0, st>>>(p, m);
}

// Areatri / Voltri (Src/memfuncs.cpp:124-157)
__device__ __forceinline__ double areatri(const DevParams& p, const Membrane& m, int p1, int p2, int p3) {
  double A[3], B[3], eta[3];
  A[0] = UXm(p2) - UXm(p1); A[1] = UYm(p2) - UYm(p1); A[2] = m.z[p2] - m.z[p1];
  B[0] = UXm(p3) - UXm(p1); B[1] = UYm(p3) - UYm(p1); B[2] = m.z[p3] - m.z[p1];
  cp(A, B, eta);
  return 0.5 * sqrt(eta[0] * eta[0] + eta[1] * eta[1] + eta[2] * eta[2]);
}
__device__ __forceinline__ double voltri(const DevParams& p, const Membrane& m, int p1, int p2, int p3) {
  double A[3], B[3], C[3], D[3], Cn[3], E1[3], E2[3];
  A[0] = UXm(p1); A[1] = UYm(p1); A[2] = m.z[p1];
  B[0] = UXm(p2); B[1] = UYm(p2); B[2] = m.z[p2];
  C[0] = UXm(p3); C[1] = UYm(p3); C[2] = m.z[p3];
  Cn[0] = (A[0] + B[0] + C[0]) / 3.0;
  Cn[1] = (A[1] + B[1] + C[1]) / 3.0;
  Cn[2] = (A[2] + B[2] + C[2]) / 3.0;
  E1[0] = UXm(p2) - UXm(p1); E1[1] = UYm(p2) - UYm(p1); E1[2] = m.z[p2] - m.z[p1];
  E2[0] = UXm(p3) - UXm(p1); E2[1] = UYm(p3) - UYm(p1); E2[2] = m.z[p3] - m.z[p1];
  cp(E1, E2, D);
  return (1.0 / 6.0) * ((D[0] * Cn[0]) + (D[1] * Cn[1]) + (D[2] * Cn[2]));
}

__global__ void k_tri_av(DevParams p, Membrane m) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.nt) return;
  m.area[i] = areatri(p, m, m.t1[i], m.t2[i], m.t3[i]);
  m.vol[i] = voltri(p, m, m.t1[i], m.t2[i], m.t3[i]);
}
// TotalVA sums in triangle order (one thread per sum, as the reference's
// one-thread reduction does)
__global__ void k_seqsum(DevParams p, Membrane m) {
  if (threadIdx.x == 0) {
    double t = 0;
    for (int i = 0; i < p.nt; ++i) t += m.area[i];
    m.sc->Sarea = t;
  } else if (threadIdx.x == 32) {
    double t = 0;
    for (int i = 0; i < p.nt; ++i) t += m.vol[i];
    m.sc->Volume = t;
  }
}
void launch_total_va(const DevParams& p, Membrane& m, cudaStream_t st) {
  k_tri_av<<<nblk(p.nt, 128), 128, 0, st>>>(p, m);
  k_seqsum<<<1, 64, 0, st>>>(p, m);
}

// force_calculate_dt (Src/memfuncs.cpp:214-441) as a gather: every vertex
// walks its contributions in the reference's accumulation order (edges,
// then triangles, then bending dihedrals, each ascending) and recomputes
// each term with the reference's expression, so the per-vertex sums are
// formed in the same order as the one-thread reference.
enum { INC_EDGE = 0, INC_TRI = 1, INC_DIH = 2 };

__device__ void edge_terms(const DevParams& p, const Membrane& m, int i, int role, double ff[3]) {
  int l1 = m.e1[i], l2 = m.e2[i];
  double l0 = m.l0[i];
  double A[3];
  A[0] = UXm(l1) - UXm(l2); A[1] = UYm(l1) - UYm(l2); A[2] = m.z[l1] - m.z[l2];
  double aa = sqrt(A[0] * A[0] + A[1] * A[1] + A[2] * A[2]);
  A[0] /= aa; A[1] /= aa; A[2] /= aa;
  double xx = aa / (2.5 * l0);
  double xxx = 1.0 / (4.0 * (1.0 - xx) * (1.0 - xx));
  const double kp = m.kappap[i];
  if (role == 0) {
    for (int k = 0; k < 3; ++k) ff[k] += (-1.0 / (p.elap)) * (xxx - 0.25 + xx) * A[k];
    for (int k = 0; k < 3; ++k) ff[k] += kp * A[k] / (aa * aa);
  } else {
    for (int k = 0; k < 3; ++k) ff[k] += (1.0 / (p.elap)) * (xxx - 0.25 + xx) * A[k];
    for (int k = 0; k < 3; ++k) ff[k] += -kp * A[k] / (aa * aa);
  }
}

__device__ void tri_terms(const DevParams& p, const Membrane& m, double Sarea, double Volume, int i, int corner,
                          double ff[3]) {
  int l1 = m.t1[i], l2 = m.t2[i], l3 = m.t3[i];
  double beta = -p.kappasa * (Sarea - p.Sarea0) / p.Sarea0;
  double betav = -p.kappav * (Volume - p.Volume0) / (p.Volume0);
  double area = areatri(p, m, l1, l2, l3);
  double alpha = beta / (4.0 * area);
  double alphad = -p.kappad * (area - m.tarea[i]) / (4.0 * m.tarea[i] * area);
  double A21[3], A13[3], A32[3], eta[3], C[3], B[3];
  A21[0] = UXm(l2) - UXm(l1); A21[1] = UYm(l2) - UYm(l1); A21[2] = m.z[l2] - m.z[l1];
  A13[0] = UXm(l1) - UXm(l3); A13[1] = UYm(l1) - UYm(l3); A13[2] = m.z[l1] - m.z[l3];
  A32[0] = UXm(l3) - UXm(l2); A32[1] = UYm(l3) - UYm(l2); A32[2] = m.z[l3] - m.z[l2];
  cp(A13, A21, eta);
  const double* side = corner == 0 ? A32 : (corner == 1 ? A13 : A21);
  cp(eta, side, C);
  for (int k = 0; k < 3; ++k) ff[k] += alpha * C[k];
  for (int k = 0; k < 3; ++k) ff[k] += alphad * C[k];
  B[0] = (UXm(l1) + UXm(l2) + UXm(l3)) / 3.0;
  B[1] = (UYm(l1) + UYm(l2) + UYm(l3)) / 3.0;
  B[2] = (m.z[l1] + m.z[l2] + m.z[l3]) / 3.0;
  cp(B, side, C);
  for (int k = 0; k < 3; ++k) ff[k] += betav * ((eta[k] / 3.0) + C[k]) / 6.0;
}

// role: 0 = l1, 1 = l4, 2 = l2, 3 = l3 (the order the reference updates them)
__device__ void dih_term(const DevParams& p, const Membrane& m, int i, int role, double ff[3]) {
  int l2, l3;
  if (m.iedge[i] == -1) { l3 = m.e1[i]; l2 = m.e2[i]; } else { l2 = m.e1[i]; l3 = m.e2[i]; }
  int l1 = m.es1[i], l4 = m.es2[i];
  double a21[3], a31[3], a24[3], a34[3], a32[3], t1[3], t2[3], eta[3], zeta[3], C[3], D[3], E[3], F[3];
  a21[0] = UXm(l2) - UXm(l1); a21[1] = UYm(l2) - UYm(l1); a21[2] = m.z[l2] - m.z[l1];
  a31[0] = UXm(l3) - UXm(l1); a31[1] = UYm(l3) - UYm(l1); a31[2] = m.z[l3] - m.z[l1];
  a24[0] = UXm(l2) - UXm(l4); a24[1] = UYm(l2) - UYm(l4); a24[2] = m.z[l2] - m.z[l4];
  a34[0] = UXm(l3) - UXm(l4); a34[1] = UYm(l3) - UYm(l4); a34[2] = m.z[l3] - m.z[l4];
  a32[0] = UXm(l3) - UXm(l2); a32[1] = UYm(l3) - UYm(l2); a32[2] = m.z[l3] - m.z[l2];
  t1[0] = (UXm(l1) + UXm(l2) + UXm(l3)) / 3.0;
  t1[1] = (UYm(l1) + UYm(l2) + UYm(l3)) / 3.0;
  t1[2] = (m.z[l1] + m.z[l2] + m.z[l3]) / 3.0;
  t2[0] = (UXm(l4) + UXm(l2) + UXm(l3)) / 3.0;
  t2[1] = (UYm(l4) + UYm(l2) + UYm(l3)) / 3.0;
  t2[2] = (m.z[l4] + m.z[l2] + m.z[l3]) / 3.0;
  cp(a21, a31, eta);
  cp(a34, a24, zeta);
  double etam = sqrt(eta[0] * eta[0] + eta[1] * eta[1] + eta[2] * eta[2]);
  double zetam = sqrt(zeta[0] * zeta[0] + zeta[1] * zeta[1] + zeta[2] * zeta[2]);
  double costh = (eta[0] * zeta[0] + eta[1] * zeta[1] + eta[2] * zeta[2]) / (etam * zetam);
  if (costh > 1.0) costh = 1.0;
  if (costh < -1.0) costh = -1.0;
  if (costh == 1.0) costh -= 0.0005;
  if (costh == -1.0) costh += 0.0005;
  double sinth = sqrt(1.0 - costh * costh);
  double tt0 = t1[0] - t2[0];
  double tt1 = t1[1] - t2[1];
  double factor = (((eta[0] - zeta[0]) * tt0) + ((eta[1] - zeta[1]) * tt1) + ((eta[2] - zeta[2]) * (t1[2] - t2[2])));
  double fact = (factor >= 0.0) ? 1.0 : -1.0;
  sinth = fact * sinth;
  double betab = p.kappab * (sinth * p.cth0 - costh * p.sth0) / sinth;
  double b11 = -(betab * costh) / (etam * etam);
  double b22 = -(betab * costh) / (zetam * zetam);
  double b12 = betab / (etam * zetam);
  if (role <= 1) {
    cp(eta, a32, C);
    cp(zeta, a32, D);
    if (role == 0) for (int k = 0; k < 3; ++k) ff[k] += b11 * C[k] + b12 * D[k];
    else for (int k = 0; k < 3; ++k) ff[k] += -b12 * C[k] - b22 * D[k];
  } else if (role == 2) {
    cp(eta, a31, C); cp(zeta, a31, D); cp(eta, a34, E); cp(zeta, a34, F);
    for (int k = 0; k < 3; ++k) ff[k] += -b11 * C[k] + b12 * (E[k] - D[k]) + b22 * F[k];
  } else {
    cp(eta, a21, C); cp(zeta, a21, D); cp(eta, a24, E); cp(zeta, a24, F);
    for (int k = 0; k < 3; ++k) ff[k] += b11 * C[k] + b12 * (-E[k] + D[k]) - b22 * F[k];
  }
}

// parasite-vertex WCA term of pfdt (Src/memfuncs.cpp:459-475)
__device__ __forceinline__ bool wca(const DevParams& p, const Membrane& m, const MemScalars* sc, int i, double X[3]) {
  double cutoff = p.paraR, epsilon = 0.1, sigma = 0.890898718 * cutoff;
  double A[3];
  A[0] = (sc->para[0] + sc->paradx * p.Lx) - (m.x[i] + m.ix[i] * p.Lx);
  A[1] = (sc->para[1] + sc->parady * p.Ly) - (m.y[i] + m.iy[i] * p.Ly);
  A[2] = sc->para[2] - m.z[i];
  double aa = A[0] * A[0] + A[1] * A[1] + A[2] * A[2];
  if (aa <= cutoff * cutoff) {
    double ex = (sigma * sigma * sigma * sigma * sigma * sigma) / (aa * aa * aa);
    X[0] = (24.0 * epsilon / aa) * ((2.0 * ex * ex) - ex) * A[0];
    X[1] = (24.0 * epsilon / aa) * ((2.0 * ex * ex) - ex) * A[1];
    X[2] = (24.0 * epsilon / aa) * ((2.0 * ex * ex) - ex) * A[2];
    return true;
  }
  return false;
}

// per vertex: pfdt's -X, force_calculate_dt's ff, gravity, bond spring and
// wall repulsion, in the order of maincode.cpp:603-665
__global__ void k_vertex_forces(DevParams p, Membrane m, const double* xlig, const double* ylig,
                                int do_pfdt, int do_forces, int do_ext) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.nv) return;
  const MemScalars* sc = m.sc;
  double f[3] = {m.fx[i], m.fy[i], m.fz[i]};
  if (do_pfdt) {
    double X[3];
    if (wca(p, m, sc, i, X)) { f[0] -= X[0]; f[1] -= X[1]; f[2] -= X[2]; }
  }
  if (do_forces) {
    double ff[3] = {0.0, 0.0, 0.0};
    const double Sarea = sc->Sarea, Volume = sc->Volume;
    for (int q = m.inc_start[i]; q < m.inc_start[i + 1]; ++q) {
      int e = m.inc[q];
      int kind = (e >> 30) & 3, role = (e >> 27) & 7, item = e & ((1 << 27) - 1);
      if (kind == INC_EDGE) edge_terms(p, m, item, role, ff);
      else if (kind == INC_TRI) tri_terms(p, m, Sarea, Volume, item, role, ff);
      else dih_term(p, m, item, role, ff);
    }
    f[0] += ff[0]; f[1] += ff[1]; f[2] += ff[2];
  }
  if (do_ext) {
    f[2] += -p.Fg / (double)p.nv;                       // :606-610
    if (m.bondi[i] == 1) {                              // :612-640
      int jj = m.bondl[i];
      double A[3];
      A[0] = m.x[i] - xlig[jj];
      A[1] = m.y[i] - ylig[jj];
      A[2] = m.z[i];
      A[0] -= p.Lx * round(A[0] / p.Lx);
      A[1] -= p.Ly * round(A[1] / p.Ly);
      double aa = sqrt(A[0] * A[0] + A[1] * A[1] + A[2] * A[2]);
      A[0] /= aa; A[1] /= aa; A[2] /= aa;
      if (aa > p.el0) {
        f[0] += -p.ks * (aa - p.el0) * A[0];
        f[1] += -p.ks * (aa - p.el0) * A[1];
        f[2] += -p.ks * (aa - p.el0) * A[2];
      }
    }
    double cc = m.z[i];                                 // :643-653
    if (cc < 0.5) f[2] += 300.0 * exp(-50.0 * cc);
    cc = p.Lz - m.z[i];                                 // :655-665
    if (cc < 0.5) f[2] -= 300.0 * exp(-50.0 * cc);
  }
  m.fx[i] = f[0]; m.fy[i] = f[1]; m.fz[i] = f[2];
}

// pfdt's parasite sum in vertex order (Src/memfuncs.cpp:469-482)
__global__ void k_para_sum(DevParams p, Membrane m) {
  if (threadIdx.x != 0) return;
  MemScalars* sc = m.sc;
  double fx = 0, fy = 0, fz = 0, X[3];
  for (int i = 0; i < p.nv; ++i)
    if (wca(p, m, sc, i, X)) { fx += X[0]; fy += X[1]; fz += X[2]; }
  sc->parafdt[0] += fx; sc->parafdt[1] += fy; sc->parafdt[2] += fz;
}

void launch_pfdt_forces(const DevParams& p, Membrane& m, int do_pfdt, int do_forces, int do_ext,
                        cudaStream_t st) {
  k_vertex_forces<<<nblk(p.nv, 64), 64, 0, st>>>(p, m, m.xlig, m.ylig, do_pfdt, do_forces, do_ext);
  if (do_pfdt) k_para_sum<<<1, 32, 0, st>>>(p, m);
}

// ================================================================ bonds =====
// liglist membership (maincode.cpp:138-154): cell centre within 1.5 of the
// ligand after the reference's fabs-then-round test
__device__ __forceinline__ bool in_liglist(const DevParams& p, int cell, double xl, double yl) {
  int k = cell % p.nz, j = (cell / p.nz) % p.ny, i = cell / (p.nz * p.ny);
  double zmax = -1.0 + (double)k * p.a + p.a;
  if (!(zmax <= 2.0)) return false;
  double xmin = (double)i * p.a, xmax = (double)i * p.a + p.a;
  double ymin = (double)j * p.a, ymax = (double)j * p.a + p.a;
  double A0 = fabs(((xmin + xmax) * 0.5) - xl);
  double A1 = fabs(((ymin + ymax) * 0.5) - yl);
  A0 -= p.Lx * round(A0 / p.Lx);
  A1 -= p.Ly * round(A1 / p.Ly);
  return (A0 < 1.5) && (A1 < 1.5);
}

// bond preparation (maincode.cpp:668-723): poff of bonded vertices, pon and
// the candidate ligands (sorted by squared distance, then index) of free
// knobs near the wall.  Candidates are enumerated on the 0.5-spaced ligand
// grid around the vertex instead of walking the whole cell list: only
// ligands within dthr can pass the reference's distance test.
__global__ void k_bond_prep(DevParams p, Membrane m, const double* xlig, const double* ylig) {
  int ii = blockIdx.x * blockDim.x + threadIdx.x;
  if (ii >= p.nv) return;
  double A[3], B[3];
  if (m.bondi[ii] == 1) {
    int p1modx = m.ix[ii], p1mody = m.iy[ii], jj = m.bondl[ii];
    A[0] = (m.x[ii] + p1modx * p.Lx) - (xlig[jj] + p1modx * p.Lx);
    A[1] = (m.y[ii] + p1mody * p.Ly) - (ylig[jj] + p1mody * p.Ly);
    A[2] = m.z[ii] - 0.0;
    double xx = sqrt(A[0] * A[0] + A[1] * A[1] + A[2] * A[2]);
    if (xx > p.el0) {
      B[0] = -p.ks * (xx - p.el0) * A[0] / xx;
      B[1] = -p.ks * (xx - p.el0) * A[1] / xx;
      B[2] = -p.ks * (xx - p.el0) * A[2] / xx;
    } else {
      B[0] = B[1] = B[2] = 0.0;
    }
    double bb = sqrt(B[0] * B[0] + B[1] * B[1] + B[2] * B[2]);
    double koff = p.offrate * exp(bb / p.FD);
    m.poff[ii] = 1.0 - exp(-koff * p.dtmd);
  } else if ((m.z[ii] < p.dthr) && (m.bondi[ii] == 0) && (m.knob[ii] == 1)) {
    const int pid = m.pid[ii];
    m.pon[ii] = 1.0 - exp(-p.onrate * p.dtmd);
    int n = 0;
    double* pd = m.pair_d + (int64_t)ii * kMaxPairs;
    int* pj = m.pair_j + (int64_t)ii * kMaxPairs;
    const int p1modx = m.ix[ii], p1mody = m.iy[ii];
    const double vx = m.x[ii], vy = m.y[ii];
    int gx0 = (int)floor((vx - p.dthr) / 0.5) - 1, gx1 = (int)floor((vx + p.dthr) / 0.5) + 1;
    int gy0 = (int)floor((vy - p.dthr) / 0.5) - 1, gy1 = (int)floor((vy + p.dthr) / 0.5) + 1;
    gx0 = max(gx0, 0); gy0 = max(gy0, 0);
    gx1 = min(gx1, p.nligx - 1); gy1 = min(gy1, p.nligy - 1);
    for (int gx = gx0; gx <= gx1; ++gx) {
      for (int gy = gy0; gy <= gy1; ++gy) {
        int j = gx * p.nligy + gy;
        double xl = xlig[j], yl = ylig[j];
        if (!in_liglist(p, pid, xl, yl)) continue;
        A[0] = (vx + p1modx * p.Lx) - (xl + p1modx * p.Lx);
        A[1] = (vy + p1mody * p.Ly) - (yl + p1mody * p.Ly);
        A[2] = m.z[ii] - 0.0;
        double aaa = (A[0] * A[0] + A[1] * A[1] + A[2] * A[2]);
        if (aaa <= p.dthr * p.dthr && n < kMaxPairs) {
          // insertion by (distance, index), the order of std::sort on pairs
          int r = n++;
          while (r > 0 && (pd[r - 1] > aaa || (pd[r - 1] == aaa && pj[r - 1] > j))) {
            pd[r] = pd[r - 1]; pj[r] = pj[r - 1]; --r;
          }
          pd[r] = aaa; pj[r] = j;
        }
      }
    }
    m.npair[ii] = n;
  }
}

// bond_dynamics (maincode.cpp:16-54): serial over vertices; draw k of the
// BOND stream is the reference's k-th RanGen[0].Random() of the step
__global__ void k_bond_dyn(DevParams p, Membrane m, uint64_t eoff) {
  const uint64_t epoch = epoch_of(p, eoff);
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  uint64_t k = 0;
  for (int ii = 0; ii < p.nv; ++ii) {
    if (m.bondi[ii] == 1) {
      double randoff = draw_uniform(p.seed, STREAM_BOND, epoch, k++);
      int jj = m.bondl[ii];
      if (m.poff[ii] > randoff) { m.bondi[ii] = 0; m.bondl[ii] = p.randno; m.ligi[jj] = 0; }
    } else if ((m.z[ii] < p.dthr) && (m.bondi[ii] == 0) && (m.knob[ii] == 1)) {
      const int n = m.npair[ii];
      for (int q = 0; q < n; ++q) {
        int j = m.pair_j[(int64_t)ii * kMaxPairs + q];
        double pon = m.pon[ii];
        double randon = draw_uniform(p.seed, STREAM_BOND, epoch, k++);
        if ((pon > randon) && (m.ligi[j] == 0)) { m.ligi[j] = 1; m.bondi[ii] = 1; m.bondl[ii] = j; }
      }
    }
  }
}

// second half-kick (maincode.cpp:727-744)
__global__ void k_kick2(DevParams p, Membrane m) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < p.nv) {
    m.vx[i] += (m.fx[i] * p.dtmd / (2.0 * p.pmass));
    m.vy[i] += (m.fy[i] * p.dtmd / (2.0 * p.pmass));
    m.vz[i] += (m.fz[i] * p.dtmd / (2.0 * p.pmass));
  }
  if (i == 0) {
    MemScalars* sc = m.sc;
    for (int k = 0; k < 3; ++k) sc->paraV[k] += ((sc->paraft[k] + sc->parafdt[k]) * p.dtmd / (2.0 * p.PRmass));
    for (int k = 0; k < 3; ++k) { sc->paraft[k] = sc->parafdt[k]; sc->parafdt[k] = 0.0; }
  }
}
void launch_bonds(const DevParams& p, Membrane& m, uint64_t epoch, cudaStream_t st) {
  k_bond_prep<<<nblk(p.nv, 128), 128, 0, st>>>(p, m, m.xlig, m.ylig);
  k_bond_dyn<<<1, 32, 0, st>>>(p, m, epoch);
}

void launch_kick2(const DevParams& p, Membrane& m, cudaStream_t st) {
  k_kick2<<<nblk(p.nv, 128), 128, 0, st>>>(p, m);
}

// ========================================================== observables ===
// Quantities the reference does not compute (its only outputs are the files):
// out[0] = solvent temperature sum m|v - u|^2 / (3 N), u the mean velocity
// of the particle's z-layer of height a (the Couette flow's own kinetic
// energy is not heat), out[1..3] = membrane centre of mass (unwrapped),
// out[4] = Sarea, out[5] = Volume, out[6] = bonds, out[7] = mean solvent
// vx, out[8] = sum m|v|^2 / (3 N) (flow included).  prof[2k], prof[2k+1] =
// sum vx and count in the z-layer [k a, (k+1) a).
__device__ __forceinline__ int obs_layer(double z, double a, int n) {
  int b = (int)floor(z / a);
  return b < 0 ? 0 : (b >= n ? n - 1 : b);
}
__global__ void k_obs_solvent(DevParams p, Solvent s, double* out, double* lay, int nlay, double* prof, int nbins) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double e = 0, vxs = 0;
  if (i < s.n) {
    const SolVel r = s.v[i];
    double vx = r.vx, vy = r.vy, vz = r.vz;
    e = p.mass * (vx * vx + vy * vy + vz * vz);
    vxs = vx;
    const double z = s.z[i];
    double* L = lay + 4 * obs_layer(z, p.a, nlay);
    atomicAdd(L, vx);
    atomicAdd(L + 1, vy);
    atomicAdd(L + 2, vz);
    atomicAdd(L + 3, 1.0);
    if (prof) {
      const int b = obs_layer(z, p.a, nbins);
      atomicAdd(&prof[2 * b], vx);
      atomicAdd(&prof[2 * b + 1], 1.0);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    e += __shfl_down_sync(0xffffffffu, e, o);
    vxs += __shfl_down_sync(0xffffffffu, vxs, o);
  }
  if ((threadIdx.x & 31) == 0) { atomicAdd(&out[8], e); atomicAdd(&out[9], vxs); }
}
__global__ void k_obs_membrane(DevParams p, Membrane m, double* out, const double* lay, int nlay, int64_t ns) {
  if (threadIdx.x != 0) return;
  double cx = 0, cy = 0, cz = 0;
  int bonds = 0;
  for (int i = 0; i < p.nv; ++i) {
    cx += m.x[i] + m.ix[i] * p.Lx; cy += m.y[i] + m.iy[i] * p.Ly; cz += m.z[i];
    bonds += m.bondi[i] == 1;
  }
  // sum m|v - u|^2 = sum m|v|^2 - sum over layers of m |S|^2 / n (S the
  // layer's velocity sum, n its count)
  double flow = 0;
  for (int b = 0; b < nlay; ++b) {
    const double* L = lay + 4 * b;
    if (L[3] > 0) flow += p.mass * (L[0] * L[0] + L[1] * L[1] + L[2] * L[2]) / L[3];
  }
  out[0] = ns ? (out[8] - flow) / (3.0 * (double)ns) : 0.0;
  out[1] = cx / p.nv; out[2] = cy / p.nv; out[3] = cz / p.nv;
  out[4] = m.sc->Sarea; out[5] = m.sc->Volume; out[6] = bonds;
  out[7] = ns ? out[9] / (double)ns : 0.0;
  out[8] = ns ? out[8] / (3.0 * (double)ns) : 0.0;
}
void launch_observables(const DevParams& p, const Solvent& s, const Membrane& m, double* obs, int nbins,
                        cudaStream_t st) {
  int nlay = (int)(p.Lz / p.a);
  nlay = nlay < 1 ? 1 : (nlay > kObsMaxBins ? kObsMaxBins : nlay);
  double* lay = obs + kObsLayers;
  double* prof = nbins > 0 ? obs + 64 : nullptr;
  cudaMemsetAsync(obs, 0, sizeof(double) * 16, st);
  cudaMemsetAsync(lay, 0, sizeof(double) * 4 * nlay, st);
  if (prof) cudaMemsetAsync(prof, 0, sizeof(double) * 2 * nbins, st);
  if (s.n) k_obs_solvent<<<nblk(s.n, 256), 256, 0, st>>>(p, s, obs, lay, nlay, prof, nbins);
  k_obs_membrane<<<1, 32, 0, st>>>(p, m, obs, lay, nlay, s.n);
}

// ============================== one launch per phase over a cohort (multi.h) ==
// the counters of a collision cleared: cnt (solvent per cell) and ncm
// (membrane vertices per cell), 256 cells per block
__global__ void __launch_bounds__(256) km_zero(Member* __restrict__ mem, const int2* __restrict__ tab) {
  KM_MEMBER;
  const int64_t c = (int64_t)b * blockDim.x + threadIdx.x;
  if (c < M.c.n) { M.c.cnt[c] = 0; M.c.ncm[c] = 0; }
}
__global__ void __launch_bounds__(1024) km_vbin(Member* __restrict__ mem, const int2* __restrict__ tab,
                                                uint64_t eoff) {
  KM_MEMBER;
  vbin_block(M.p, M.m, M.c.ncm, eoff);
}
__global__ void __launch_bounds__(256) km_ghost(Member* __restrict__ mem, const int2* __restrict__ tab) {
  KM_MEMBER;
  ghost_flags_item(M.p, M.c.cnt, M.c.ncm, M.m.sc, M.c.wrank, M.c.mrank, (int64_t)b * blockDim.x + threadIdx.x);
}
// the scans of (cnt, wrank, mrank) into (start, wrank, mrank), as launch_scan3
__global__ void __launch_bounds__(kScanT) km_scan_part(Member* __restrict__ mem, const int2* __restrict__ tab) {
  KM_MEMBER;
  scan_part_block(M.c.cnt, M.c.wrank, M.c.mrank, M.c.n, M.c.scan_part, b);
}
// one block per member; also start[C] = the particle total
__global__ void __launch_bounds__(1024) km_scan_top(Member* __restrict__ mem, const int2* __restrict__ tab) {
  KM_MEMBER;
  scan_top_block(M.c.scan_part, (M.c.n + kScanTile - 1) / kScanTile, M.c.totals);
  __syncthreads();
  if (threadIdx.x == 0) M.c.start[M.c.n] = M.c.totals[0];
}
__global__ void __launch_bounds__(kScanT) km_scan_final(Member* __restrict__ mem, const int2* __restrict__ tab) {
  KM_MEMBER;
  scan_final_block(M.c.cnt, M.c.wrank, M.c.mrank, M.c.start, M.c.wrank, M.c.mrank, M.c.n, M.c.scan_part, b);
}

void set_collide_kernel_limits() {
  cudaFuncSetAttribute(k_vbin, cudaFuncAttributeMaxDynamicSharedMemorySize, 8192 * sizeof(uint64_t));
  cudaFuncSetAttribute(km_vbin, cudaFuncAttributeMaxDynamicSharedMemorySize, 8192 * sizeof(uint64_t));
}

int multi_collide_front(const MultiPlan& P, uint64_t eoff, cudaStream_t st) {
  km_zero<<<P.blocks[MP_ZERO], 256, 0, st>>>(P.mem, P.table(MP_ZERO));
  km_vbin<<<P.blocks[MP_VBIN], 1024, P.vbin_smem, st>>>(P.mem, P.table(MP_VBIN), eoff);
  return 2;
}

int multi_collide_scan(const MultiPlan& P, cudaStream_t st) {
  km_ghost<<<P.blocks[MP_GHOST], 256, 0, st>>>(P.mem, P.table(MP_GHOST));
  km_scan_part<<<P.blocks[MP_SCAN], kScanT, 0, st>>>(P.mem, P.table(MP_SCAN));
  km_scan_top<<<P.blocks[MP_SCAN_TOP], 1024, 0, st>>>(P.mem, P.table(MP_SCAN_TOP));
  km_scan_final<<<P.blocks[MP_SCAN], kScanT, 0, st>>>(P.mem, P.table(MP_SCAN));
  return 4;
}

}  // namespace irbc
