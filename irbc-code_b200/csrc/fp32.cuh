// fp32.cuh -- (part of fast.cu) the FP32-bulk solvent: positions and velocities stored as
// float4 (x, y, z, inside-flag bits) and (vx, vy, vz, reference-index bits),
// 32 bytes per particle.  Free flight, walls, wrap, binning and the SRD
// rotation run in float; the per-cell momentum and relative-energy sums are
// accumulated in double; particles near the membrane are promoted to double
// for reflectionFed and its cubic root solve; the membrane itself stays FP64.
#include <cstdio>
#include "fast.h"
#include "fp32.h"
#include "cells_tile.cuh"

namespace irbc {

static inline unsigned nbf(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

// ---- conversions between the FP64 arrays (set-up, state exchange) and FP32
__global__ void k_to_f32(Solvent s, SolventF f) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= s.n) return;
  f.pos[i] = make_float4((float)s.x[i], (float)s.y[i], (float)s.z[i], __int_as_float(s.indio[i]));
  const SolVel r = s.v[i];
  f.vel[i] = make_float4((float)r.vx, (float)r.vy, (float)r.vz, __int_as_float(r.id));
  f.pid[i] = s.pid[i];
}
__global__ void k_to_f64(SolventF f, Solvent s) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= s.n) return;
  float4 p = f.pos[i], v = f.vel[i];
  s.x[i] = p.x; s.y[i] = p.y; s.z[i] = p.z; s.indio[i] = __float_as_int(p.w);
  SolVel r;
  r.vx = v.x; r.vy = v.y; r.vz = v.z; r.id = __float_as_int(v.w); r.pad = 0;
  s.v[i] = r;
  s.pid[i] = f.pid[i];
}
void f32_from_f64(Solvent& s, SolventF& f, cudaStream_t st) {
  if (s.n) k_to_f32<<<nbf(s.n, 256), 256, 0, st>>>(s, f);
}
void f32_to_f64(SolventF& f, Solvent& s, cudaStream_t st) {
  if (s.n) k_to_f64<<<nbf(s.n, 256), 256, 0, st>>>(f, s);
}

// ---- collision --------------------------------------------------------------
__device__ __forceinline__ int shifted_cell_f(const DevParams& p, float4 q, const double r[3]) {
  int fx = (int)floor(bbound((double)q.x - r[0], p.Lx));
  int fy = (int)floor(bbound((double)q.y - r[1], p.Ly));
  int fz = (int)floor((double)q.z - r[2] + 1.0);
  return cell_of(p, fx, fy, fz);
}

// block `bid` of the count: kCountPer particles per thread
__device__ __forceinline__ void count_f_block(const DevParams& p, const SolventF& f, int* cnt, int* slot,
                                              uint64_t eoff, int64_t bid) {
  const uint64_t epoch = epoch_of(p, eoff);
  // the grid shift, drawn once per block
  __shared__ double sr[3];
  if (threadIdx.x == 0) grid_shift(p, epoch, sr);
  __syncthreads();
  const double r[3] = {sr[0], sr[1], sr[2]};
  const int64_t i0 = bid * blockDim.x * kCountPer + threadIdx.x;
  int c[kCountPer];
#pragma unroll
  for (int u = 0; u < kCountPer; ++u) {
    const int64_t i = i0 + (int64_t)u * blockDim.x;
    c[u] = i < f.n ? shifted_cell_f(p, f.pos[i], r) : -1;
  }
  int sl[kCountPer];
  claim_slots<kCountPer>(cnt, c, i0, blockDim.x, f.n, sl);
#pragma unroll
  for (int u = 0; u < kCountPer; ++u) {
    const int64_t i = i0 + (int64_t)u * blockDim.x;
    if (i < f.n) {
      f.pid[i] = c[u];  // the cell of this collision
      slot[i] = sl[u];
    }
  }
}
__global__ void __launch_bounds__(256) k_count_f(DevParams p, SolventF f, int* cnt, int* slot, uint64_t eoff) {
  count_f_block(p, f, cnt, slot, eoff, blockIdx.x);
}

__device__ __forceinline__ void perm_f_item(const int* __restrict__ key, const int* __restrict__ slot,
                                            const int* __restrict__ start, int64_t n, int* __restrict__ perm,
                                            int64_t i) {
  if (i >= n) return;
  perm[(int64_t)start[key[i]] + slot[i]] = (int)i;
}
__global__ void k_perm_f(const int* __restrict__ key, const int* __restrict__ slot, const int* __restrict__ start,
                         int64_t n, int* __restrict__ perm) {
  perm_f_item(key, slot, start, n, perm, (int64_t)blockIdx.x * blockDim.x + threadIdx.x);
}

// physical re-sort by collision cell every kResortEvery collisions
__device__ __forceinline__ void gather_f_item(const SolventF& f, const int* __restrict__ perm, int64_t j) {
  if (j >= f.n) return;
  const int i = perm[j];
  f.pos2[j] = f.pos[i];
  f.vel2[j] = f.vel[i];
  f.pid2[j] = f.pid[i];
}
__device__ __forceinline__ void copy_back_f_item(const SolventF& f, int64_t j) {
  if (j >= f.n) return;
  f.pos[j] = f.pos2[j];
  f.vel[j] = f.vel2[j];
  f.pid[j] = f.pid2[j];
}
__global__ void k_gather_f(SolventF f, const int* __restrict__ perm) {
  gather_f_item(f, perm, (int64_t)blockIdx.x * blockDim.x + threadIdx.x);
}
__global__ void k_copy_back_f(SolventF f) { copy_back_f_item(f, (int64_t)blockIdx.x * blockDim.x + threadIdx.x); }

void launch_collide_count_f(const DevParams& p, SolventF& f, Solvent& s, Cells& c, uint64_t epoch,
                            cudaStream_t st) {
  cudaMemsetAsync(c.cnt, 0, sizeof(int) * c.n, st);
  if (f.n) k_count_f<<<nbf(f.n, 256 * kCountPer), 256, 0, st>>>(p, f, c.cnt, s.slot, epoch);
}

// per-cell statistics (sums in double, reference particle order) and the
// float rotation: k_cells_tile<true> (cells_tile.cuh)
void launch_collide_finish_f(const DevParams& p, SolventF& f, Solvent& s, Cells& c, Membrane& m, uint64_t epoch,
                             cudaStream_t st, bool resort) {
  launch_ghost_flags(p, c, m, st);
  launch_scan3(c.cnt, c.wrank, c.mrank, c.start, c.wrank, c.mrank, c.totals, c.n, c.scan_part, st);
  cudaMemcpyAsync(c.start + c.n, c.totals + 0, sizeof(int), cudaMemcpyDeviceToDevice, st);
  if (f.n) k_perm_f<<<nbf(f.n, 256), 256, 0, st>>>(f.pid, s.slot, c.start, f.n, s.perm);
  k_cells_tile<true><<<cells_tile_blocks(c.n), 32 * kTileWarps, 0, st>>>(p, s, f, c, m, epoch);
  if (resort) launch_resort_f(f, s, st);
}

void launch_resort_f(SolventF& f, Solvent& s, cudaStream_t st) {
  if (f.n) {
    k_gather_f<<<nbf(f.n, 256), 256, 0, st>>>(f, s.perm);
    k_copy_back_f<<<nbf(f.n, 256), 256, 0, st>>>(f);
  }
}

// ---- streaming ------------------------------------------------------------------
// free flight, walls and wrap in float (maincode.cpp:516-560); particles in
// cells with triangles are handed to the near-membrane kernels (double
// precision)
// the shifted-free cell of a position (the list lookup of the streaming)
__device__ __forceinline__ int stream_cell_f(const DevParams& p, float4 q, float Lx, float Ly) {
  int fx = (int)floorf(bbound(q.x, Lx));
  int fy = (int)floorf(bbound(q.y, Ly));
  int fz = (int)floorf(q.z + 1.0f);
  return cell_of(p, fx, fy, fz);
}

// free flight, walls and wrap of particle i, loaded as (q, v), whose cell
// pid has the list [l0, l1): particles in cells with triangles are handed
// to the near-membrane kernels (double precision)
__device__ __forceinline__ void stream_f_apply(const DevParams& p, const SolventF& f, const int* __restrict__ lrank,
                                               int* bcnt, int* bucket, int* queue, int* qn, int hcap, int64_t i,
                                               float4 q, float4 v, int pid, int l0, int l1) {
  const float Lx = (float)p.Lx, Ly = (float)p.Ly, Lz = (float)p.Lz, dt = (float)p.dtmd;
  if (l1 > l0) {
    hand_off(lrank, pid, l1 - l0, hcap, (int)i, bcnt, bucket, queue, qn);
    return;
  }
  float X = q.x + v.x * dt, Y = q.y + v.y * dt, Z = q.z + v.z * dt;
  if (Z > Lz || Z < 0.0f) {
    const float wall = Z > Lz ? Lz : 0.0f;
    float ax = X - v.x * dt, ay = Y - v.y * dt, az = Z - v.z * dt;
    float sp = (wall - az) / (Z - az);
    float bx = ax + sp * (X - ax), by = ay + sp * (Y - ay), bz = az + sp * (Z - az);
    float dist = sqrtf((bx - ax) * (bx - ax) + (by - ay) * (by - ay) + (bz - az) * (bz - az));
    float dtt = dist / sqrtf(v.x * v.x + v.y * v.y + v.z * v.z);
    if (Z > Lz) { v.x = (float)p.wallspeed; v.y = 0.0f; v.z = 0.0f; }
    else { v.x = -v.x; v.y = -v.y; v.z = -v.z; }
    X = bx + v.x * (dt - dtt); Y = by + v.y * (dt - dtt); Z = bz + v.z * (dt - dtt);
    f.vel[i] = v;
  }
  X = bbound(X, Lx);
  Y = bbound(Y, Ly);
  raise_health(p, solvent_bad(p, X, Y, Z, v.x, v.y, v.z), HEALTH_SOLVENT);
  f.pos[i] = make_float4(X, Y, Z, q.w);
}

__device__ __forceinline__ void stream_f_item(const DevParams& p, const SolventF& f, const int* __restrict__ lstart,
                                              const int* __restrict__ lrank, int* bcnt, int* bucket, int* queue,
                                              int* qn, int hcap, int64_t i) {
  if (i >= f.n) return;
  const float4 q = f.pos[i], v = f.vel[i];
  const int pid = stream_cell_f(p, q, (float)p.Lx, (float)p.Ly);
  const int l0 = __ldg(lstart + pid), l1 = __ldg(lstart + pid + 1);
  stream_f_apply(p, f, lrank, bcnt, bucket, queue, qn, hcap, i, q, v, pid, l0, l1);
}

__global__ void __launch_bounds__(256) k_stream_f(DevParams p, SolventF f, const int* __restrict__ lstart,
                                                  const int* __restrict__ lrank, int* bcnt, int* bucket,
                                                  int* queue, int* qn, int hcap) {
  stream_f_item(p, f, lstart, lrank, bcnt, bucket, queue, qn, hcap, (int64_t)blockIdx.x * blockDim.x + threadIdx.x);
}

int fast_stream_f(const DevParams& p, SolventF& f, const Cells& c, FastBufs& fb, int buf, cudaStream_t st,
                  cudaEvent_t ev0, cudaEvent_t ev1, cudaEvent_t snap) {
  cudaMemsetAsync(fb.qn, 0, sizeof(int), st);
  if (f.n) {
    if (ev0) cudaEventRecord(ev0, st);
    k_stream_f<<<nbf(f.n, 256), 256, 0, st>>>(p, f, c.lstart, c.lrank, fb.bcnt, fb.bucket, fb.queue, fb.qn,
                                              fb.hcap);
    if (ev1) cudaEventRecord(ev1, st);
    if (snap) cudaStreamWaitEvent(st, snap, 0);
    Solvent none;
    none.n = f.n;
    return 1 + launch_stream_cells<true>(p, none, f, c, fb, buf, st);
  }
  return 0;
}

}  // namespace irbc
