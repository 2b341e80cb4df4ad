// multi.cuh -- (part of fast.cu) one launch per phase over a cohort of FP32
// simulations (multi.h): the fused kernels of the streaming, the membrane
// chain and the collision's particle phases.  Each block reads its member
// and its block index within that member from the phase's block table
// (KM_MEMBER) and runs the single-simulation kernel's device code.
#include "multi.h"

namespace irbc {

// ---- streaming -------------------------------------------------------------
__global__ void __launch_bounds__(256, 8) km_stream_f(Member* __restrict__ mem, const int2* __restrict__ tab,
                                                   int par) {
  KM_MEMBER;
  // copies: the descriptor is not reloaded after the stores below
  const DevParams p = M.p;
  const SolventF f = M.f;
  const int* __restrict__ lstart = M.c.lstart;
  const int* __restrict__ lrank = M.c.lrank;
  int* const bcnt = M.fb.bcnt;
  int* const bucket = M.fb.bucket;
  int* const queue = M.fb.queue;
  int* const qn = M.fb.qn + par;
  const int hcap = M.fb.hcap;
  const int64_t n = f.n;
  const float Lx = (float)p.Lx, Ly = (float)p.Ly;
  constexpr int K = kMultiStreamPer;
  for (int pass = 0; pass < kMultiStreamPasses; ++pass) {
    const int64_t i0 = ((int64_t)b * kMultiStreamPasses + pass) * blockDim.x * K + threadIdx.x;
    if (i0 >= n) break;
    // every load of the thread's particles first, then their cells' list
    // bounds, then the updates: the latencies overlap
    float4 q[K], v[K];
    int pid[K], l0[K], l1[K];
#pragma unroll
    for (int u = 0; u < K; ++u) {
      const int64_t i = i0 + (int64_t)u * blockDim.x;
      if (i < n) { q[u] = f.pos[i]; v[u] = f.vel[i]; }
    }
#pragma unroll
    for (int u = 0; u < K; ++u) {
      const int64_t i = i0 + (int64_t)u * blockDim.x;
      if (i < n) {
        pid[u] = stream_cell_f(p, q[u], Lx, Ly);
        l0[u] = __ldg(lstart + pid[u]);
        l1[u] = __ldg(lstart + pid[u] + 1);
      }
    }
#pragma unroll
    for (int u = 0; u < K; ++u) {
      const int64_t i = i0 + (int64_t)u * blockDim.x;
      if (i < n) stream_f_apply(p, f, lrank, bcnt, bucket, queue, qn, hcap, i, q[u], v[u], pid[u], l0[u], l1[u]);
    }
  }
}

// members with long lists: a block per listed cell (and the overflow
// blocks) of the single-simulation long-list kernel
__global__ void __launch_bounds__(256, 2) km_stream_cells(Member* __restrict__ mem, const int2* __restrict__ tab,
                                                       int par, int cap) {
  KM_MEMBER;
  // copies: the descriptor is not reloaded after the walk's stores; the
  // snapshot buffer of this parity chosen without indexing the descriptor
  DevParams p = M.p;
  Solvent s = M.s;
  SolventF f = M.f;
  const Snap sn = par ? M.fb.snap[1] : M.fb.snap[0];
  const TriPre* const pre = par ? M.fb.pre[1] : M.fb.pre[0];
  int* const qn = M.fb.qn;
  // the overflow counter of the next step starts at zero
  if (b == 0 && threadIdx.x == 0) qn[par ^ 1] = 0;
  const int nblk = (int)M.fb.bcap + kOverflowBlocks;
  stream_cells_block<true>(p, s, f, M.c.lstart, M.c.lidx, M.c.acell, M.fb.bcnt, M.fb.bucket, sn, pre, M.fb.queue,
                           qn + par, M.c.totals + 4, M.fb.border, b, nblk, cap);
}

// members with short lists: kMultiCellsPer (= kShortWarps) warps per block,
// each one listed cell of the single-simulation short-list kernel
__global__ void __launch_bounds__(32 * kShortWarps, kShortMinBlocks)
    km_stream_cells_short(Member* __restrict__ mem, const int2* __restrict__ tab, int par) {
  KM_MEMBER;
  DevParams p = M.p;
  Solvent s = M.s;
  SolventF f = M.f;
  const TriPre* const pre = par ? M.fb.pre[1] : M.fb.pre[0];
  int* const qn = M.fb.qn;
  // the overflow counter of the next step starts at zero
  if (b == 0 && threadIdx.x == 0) qn[par ^ 1] = 0;
  __shared__ LaneStage stage[kMultiCellsPer];
  const int w = (int)(threadIdx.x >> 5);
  const int a = b * kMultiCellsPer + w;
  if (a >= (int)M.fb.bcap) return;
  stream_cells_warp<true>(p, s, f, M.c.lidx, M.fb.arng, M.fb.bcnt, M.fb.bucket, pre, M.fb.queue, qn + par,
                          M.c.totals + 4, a, stage[w]);
}

// then their queues (the bulk kernel's overflow and the particles the
// short-list kernel handed on): kQueueBlocksMember blocks per member
__global__ void __launch_bounds__(256, 2) km_stream_queue(Member* __restrict__ mem, const int2* __restrict__ tab,
                                                       int par) {
  KM_MEMBER;
  DevParams p = M.p;
  Solvent s = M.s;
  SolventF f = M.f;
  const Snap sn = par ? M.fb.snap[1] : M.fb.snap[0];
  const TriPre* const pre = par ? M.fb.pre[1] : M.fb.pre[0];
  const int64_t gw = (int64_t)b * 8 + (threadIdx.x >> 5);
  overflow_walk<true>(p, s, f, M.c.lstart, M.c.lidx, sn, pre, M.fb.queue, M.fb.qn + par, gw,
                      (int64_t)kQueueBlocksMember * 8, threadIdx.x & 31);
}

int multi_stream(const MultiPlan& P, int par, cudaStream_t st, cudaEvent_t snap) {
  km_stream_f<<<P.blocks[MP_STREAM], 256, 0, st>>>(P.mem, P.table(MP_STREAM), par);
  if (snap) cudaStreamWaitEvent(st, snap, 0);
  // as the plain launch (launch_stream_cells): one warp per listed cell and
  // one lane per particle for the members with short lists, eight warps per
  // cell for the others, one launch per class
  const int n0 = P.cells_short, n1 = P.blocks[MP_CELLS] - P.cells_short;
  int k = 1;
  if (n0 > 0) {
    km_stream_cells_short<<<n0, 32 * kShortWarps, 0, st>>>(P.mem, P.table(MP_CELLS), par);
    ++k;
  }
  if (P.blocks[MP_QUEUE] > 0) {
    km_stream_queue<<<P.blocks[MP_QUEUE], 256, 0, st>>>(P.mem, P.table(MP_QUEUE), par);
    ++k;
  }
  if (n1 > 0) {
    km_stream_cells<<<n1, 256, stage_bytes(P.cells_cap), st>>>(P.mem, P.table(MP_CELLS) + n0, par, P.cells_cap);
    ++k;
  }
  return k;
}

// ---- membrane chain (the wide kernels' phases) --------------------------------
__global__ void __launch_bounds__(128) km_drift(Member* __restrict__ mem, const int2* __restrict__ tab) {
  KM_MEMBER;
  m_drift_item(M.p, M.m, b * blockDim.x + threadIdx.x);
}
__global__ void __launch_bounds__(128) km_av(Member* __restrict__ mem, const int2* __restrict__ tab) {
  KM_MEMBER;
  m_av_item(M.p, M.m, b * blockDim.x + threadIdx.x);
}
__global__ void __launch_bounds__(256) km_sum_edges(Member* __restrict__ mem, const int2* __restrict__ tab) {
  KM_MEMBER;
  sum_edges_block(M.p, M.m, M.fb.slot, 1, M.fb.vd, M.fb.vw, M.fb.vX, b);
}
__global__ void __launch_bounds__(128) km_force_tri(Member* __restrict__ mem, const int2* __restrict__ tab) {
  KM_MEMBER;
  const int k = b * blockDim.x + threadIdx.x;
  if (k < M.p.nt) force_item(M.p, M.m, M.fb.slot, M.p.ne + k);
}
__global__ void __launch_bounds__(32 * kGW) km_gather(Member* __restrict__ mem, const int2* __restrict__ tab) {
  KM_MEMBER;
  gather_block(M.p, M.m, M.fb.slot, M.fb.gstart, M.fb.gidx, b);
}
__global__ void __launch_bounds__(kTailT) km_tail(Member* __restrict__ mem, const int2* __restrict__ tab,
                                                  uint64_t eoff) {
  KM_MEMBER;
  __shared__ TailSmem S;
  tail_b_block(M.p, M.m, M.fb.vd, M.fb.vw, M.fb.vX, epoch_of(M.p, eoff), S);
}

int multi_membrane(const MultiPlan& P, uint64_t eoff, cudaStream_t st) {
  km_drift<<<P.blocks[MP_DRIFT], 128, 0, st>>>(P.mem, P.table(MP_DRIFT));
  km_av<<<P.blocks[MP_AV], 128, 0, st>>>(P.mem, P.table(MP_AV));
  km_sum_edges<<<P.blocks[MP_SUM_EDGES], 256, P.sum_smem, st>>>(P.mem, P.table(MP_SUM_EDGES));
  km_force_tri<<<P.blocks[MP_FORCE_TRI], 128, 0, st>>>(P.mem, P.table(MP_FORCE_TRI));
  km_gather<<<P.blocks[MP_GATHER], 32 * kGW, 0, st>>>(P.mem, P.table(MP_GATHER));
  km_tail<<<P.blocks[MP_TAIL], kTailT, 0, st>>>(P.mem, P.table(MP_TAIL), eoff);
  return 6;
}

// next half-kick, snapshot `buf` and its triangle records
__global__ void __launch_bounds__(128) km_kick(Member* __restrict__ mem, const int2* __restrict__ tab, int buf) {
  KM_MEMBER;
  kick_snap_item(M.p, M.m, M.fb.snap[buf], b * blockDim.x + threadIdx.x);
}
__global__ void __launch_bounds__(128) km_tri_prep(Member* __restrict__ mem, const int2* __restrict__ tab,
                                                   int buf) {
  KM_MEMBER;
  const int j = b * blockDim.x + threadIdx.x;
  if (j < M.p.nt) tri_prep_one(M.p, M.m, j, M.m.vx, M.m.vy, M.m.vz, M.fb.pre[buf]);
}

int multi_kick(const MultiPlan& P, int buf, cudaStream_t st) {
  km_kick<<<P.blocks[MP_KICK], 128, 0, st>>>(P.mem, P.table(MP_KICK), buf);
  km_tri_prep<<<P.blocks[MP_TRI_PREP], 128, 0, st>>>(P.mem, P.table(MP_TRI_PREP), buf);
  return 2;
}

// ---- collision: particle phases ---------------------------------------------------
__global__ void __launch_bounds__(256) km_count(Member* __restrict__ mem, const int2* __restrict__ tab,
                                                uint64_t eoff) {
  KM_MEMBER;
  count_f_block(M.p, M.f, M.c.cnt, M.s.slot, eoff, b);
}
__global__ void __launch_bounds__(256) km_perm(Member* __restrict__ mem, const int2* __restrict__ tab) {
  KM_MEMBER;
  perm_f_item(M.f.pid, M.s.slot, M.c.start, M.f.n, M.s.perm, (int64_t)b * blockDim.x + threadIdx.x);
}
__global__ void __launch_bounds__(32 * kTileWarps) km_tile(Member* __restrict__ mem, const int2* __restrict__ tab,
                                                           uint64_t eoff) {
  KM_MEMBER;
  // copies: the descriptor is not reloaded after the tile's stores
  const DevParams p = M.p;
  Solvent s = M.s;
  SolventF f = M.f;
  const Cells c = M.c;
  const Membrane m = M.m;
  cells_tile_block<true>(p, s, f, c, m, eoff, b);
}
__global__ void __launch_bounds__(256) km_move(Member* __restrict__ mem, const int2* __restrict__ tab, int back) {
  KM_MEMBER;
  const int64_t j = (int64_t)b * blockDim.x + threadIdx.x;
  if (back) copy_back_f_item(M.f, j);
  else gather_f_item(M.f, M.s.perm, j);
}

int multi_collide_count(const MultiPlan& P, uint64_t eoff, cudaStream_t st) {
  km_count<<<P.blocks[MP_COUNT], 256, 0, st>>>(P.mem, P.table(MP_COUNT), eoff);
  return 1;
}

int multi_collide_back(const MultiPlan& P, uint64_t eoff, bool resort, cudaStream_t st) {
  km_perm<<<P.blocks[MP_PERM], 256, 0, st>>>(P.mem, P.table(MP_PERM));
  km_tile<<<P.blocks[MP_TILE], 32 * kTileWarps, 0, st>>>(P.mem, P.table(MP_TILE), eoff);
  if (!resort) return 2;
  km_move<<<P.blocks[MP_MOVE], 256, 0, st>>>(P.mem, P.table(MP_MOVE), 0);
  km_move<<<P.blocks[MP_MOVE], 256, 0, st>>>(P.mem, P.table(MP_MOVE), 1);
  return 4;
}

// ---- kernel limits (host) ---------------------------------------------------------------
// Every kernel's dynamic shared-memory limit on the current device, set
// before any launch: irbc_create calls this for each new simulation, so a
// launch issued by one host thread never races another thread's first-
// launch attribute call (the request server sets new simulations up on
// threads of their own while others step).
void set_kernel_limits() {
  const int cells = stage_bytes(kStageLong);
  const int sums = 2 * kSumSmemT * (int)sizeof(double);
  const auto dyn = cudaFuncAttributeMaxDynamicSharedMemorySize;
  cudaFuncSetAttribute(k_stream_cells<true>, dyn, cells);
  cudaFuncSetAttribute(k_stream_cells<false>, dyn, cells);
  cudaFuncSetAttribute(km_stream_cells, dyn, cells);
  // eight blocks of the short-list kernels (24 KB of staging each) per SM
  const auto carve = cudaFuncAttributePreferredSharedMemoryCarveout;
  cudaFuncSetAttribute(k_stream_cells_short<true>, carve, (int)cudaSharedmemCarveoutMaxShared);
  cudaFuncSetAttribute(k_stream_cells_short<false>, carve, (int)cudaSharedmemCarveoutMaxShared);
  cudaFuncSetAttribute(km_stream_cells_short, carve, (int)cudaSharedmemCarveoutMaxShared);
  cudaFuncSetAttribute(k_m_sum, dyn, sums);
  cudaFuncSetAttribute(k_sum_edges, dyn, sums);
  cudaFuncSetAttribute(km_sum_edges, dyn, sums);
  cudaFuncSetAttribute(k_membrane_block, dyn, 96 * 1024);
  cudaFuncSetAttribute(k_membrane_cluster, dyn, 200 * 1024);
  set_collide_kernel_limits();
}

// ---- the tables' sizes (host) -------------------------------------------------------
void multi_blocks(const Member& M, int out[MP_NPHASE]) {
  const DevParams& p = M.p;
  const int64_t ns = M.f.n, nc = M.c.n;
  out[MP_STREAM] = (int)nbf(ns, 256 * kMultiStreamPer * kMultiStreamPasses);
  {
    // short lists: kMultiCellsPer listed cells per block, then the queue
    // walk; long lists: a block per listed cell and the overflow blocks
    const bool shrt = short_lists(M.fb.hcap);
    out[MP_CELLS] = (int)(shrt ? (M.fb.bcap + kMultiCellsPer - 1) / kMultiCellsPer : M.fb.bcap + kOverflowBlocks);
    out[MP_QUEUE] = shrt ? kQueueBlocksMember : 0;
  }
  out[MP_DRIFT] = (int)nb(p.nv, 128);
  out[MP_AV] = (int)nb(p.nt, 128);
  out[MP_SUM_EDGES] = 1 + (int)nb(2 * p.ne + p.nv, 256);
  out[MP_FORCE_TRI] = (int)nb(p.nt, 128);
  out[MP_GATHER] = (int)nb(p.nv, kGW);
  out[MP_TAIL] = 1;
  out[MP_KICK] = (int)nb(p.nv, 128);
  out[MP_TRI_PREP] = (int)nb(p.nt, 128);
  out[MP_ZERO] = (int)nb(nc, 256);
  out[MP_VBIN] = 1;
  out[MP_COUNT] = (int)nbf(ns, 256 * kCountPer);
  out[MP_GHOST] = (int)nb(nc, 256);
  out[MP_SCAN] = (int)scan_part_blocks(nc);
  out[MP_SCAN_TOP] = 1;
  out[MP_PERM] = (int)nbf(ns, 256);
  out[MP_TILE] = (int)cells_tile_blocks(nc);
  out[MP_MOVE] = (int)nbf(ns, 256);
}

void multi_smem(const Member& M, int out[2]) {
  const DevParams& p = M.p;
  int n2 = 1;
  while (n2 < p.nv) n2 <<= 1;
  out[0] = (int)sizeof(uint64_t) * n2;
  out[1] = p.nt <= kSumSmemT ? 2 * p.nt * (int)sizeof(double) : 0;
}

}  // namespace irbc
