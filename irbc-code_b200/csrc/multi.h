// multi.h -- one launch per phase over many FP32 simulations (a cohort).
//
// A cohort's members advance in lock step: the same step parity, the same
// collision phase.  Each phase of the step (bulk streaming, near-membrane
// streaming, every membrane kernel, every collision kernel) is ONE launch
// whose blocks are split among the members: member r owns a contiguous run
// of each phase's blocks, each block reads (member, block index within the
// member) from the phase's block table with one load, and then runs
// exactly the device code the single-simulation kernel runs, on that
// member's buffers, with its block index within the member.  A member
// therefore computes bit for bit what it computes alone.
#pragma once
#include "fp32.h"

namespace irbc {

// what the kernels of one simulation read: its parameters and the device
// addresses of its buffers (the handle's own allocations)
struct Member {
  DevParams p;
  Solvent s;
  SolventF f;
  Cells c;
  Membrane m;
  FastBufs fb;
};

enum MultiPhase : int {
  MP_STREAM, MP_CELLS, MP_QUEUE,                                  // streaming
  MP_DRIFT, MP_AV, MP_SUM_EDGES, MP_FORCE_TRI, MP_GATHER, MP_TAIL,  // membrane
  MP_KICK, MP_TRI_PREP,                                           // next half-kick and snapshot
  MP_ZERO, MP_VBIN, MP_COUNT, MP_GHOST, MP_SCAN, MP_SCAN_TOP, MP_PERM, MP_TILE, MP_MOVE,  // collision
  MP_NPHASE
};

// device tables of a cohort, built by the host from its members: for each
// phase k, entry blockIdx.x of blk + off[k] holds (member, block index
// within the member), so a block finds its member with one load
struct MultiPlan {
  Member* mem = nullptr;         // [n]
  int2* blk = nullptr;           // every phase's block table, concatenated
  int64_t off[MP_NPHASE] = {};   // where phase k's table starts
  int n = 0;
  int blocks[MP_NPHASE] = {};    // each phase's grid
  // near-membrane streaming: phase MP_CELLS's table lists the blocks of the
  // members with short lists first (cells_short of them), then the others;
  // cells_cap: the staging piece of the long-list launch.  MP_QUEUE: the
  // queue walk after the short-list kernel (short-list members only)
  int cells_short = 0;
  int cells_cap = 1;
  int vbin_smem = 0;             // vertex binning: the largest member's sort
  int sum_smem = 0;              // ordered Sarea / Volume sums: the largest member's staging
  const int2* table(int k) const { return blk + off[k]; }
};

// the fused bulk streaming kernel: particles per thread in flight at once,
// and passes per block (a block covers 256 * kMultiStreamPer *
// kMultiStreamPasses particles of its member, so that reading the member's
// descriptor is paid once per that many)
constexpr int kMultiStreamPer = 1, kMultiStreamPasses = 8;
// listed cells (one warp each) per block of the fused short-list
// near-membrane kernel
constexpr int kMultiCellsPer = kShortWarps;

// blocks of each phase for one member (host)
void multi_blocks(const Member& M, int out[MP_NPHASE]);
// dynamic shared memory of the phases for one member (host): vbin, sum
void multi_smem(const Member& M, int out[2]);

// fused launches; par = the step's parity: the snapshot buffer the
// streaming reads and the overflow counter it uses (fb.qn[par]; the
// near-membrane kernel clears fb.qn[par ^ 1] for the next step).  snap
// (optional): the event the near-membrane kernel waits for (the snapshot's
// producer).  Each returns the number of kernels it launched.
int multi_stream(const MultiPlan& P, int par, cudaStream_t st, cudaEvent_t snap);
int multi_membrane(const MultiPlan& P, uint64_t eoff, cudaStream_t st);
int multi_kick(const MultiPlan& P, int buf, cudaStream_t st);
// A collision, in this order: multi_collide_front (kernels.cu: the cell
// counters cleared, the vertices binned), multi_collide_count (fast.cu: the
// particles counted into their shifted cells), multi_collide_scan
// (kernels.cu: ghost flags and the three-array scan, start[C] included),
// multi_collide_back (fast.cu: the counting-sort scatter, the collision
// tiles and, when `resort`, the physical re-sort by cell).
int multi_collide_front(const MultiPlan& P, uint64_t eoff, cudaStream_t st);
int multi_collide_count(const MultiPlan& P, uint64_t eoff, cudaStream_t st);
int multi_collide_scan(const MultiPlan& P, cudaStream_t st);
int multi_collide_back(const MultiPlan& P, uint64_t eoff, bool resort, cudaStream_t st);

#ifdef __CUDACC__
// this block's member and its block index within that member.  M refers
// to the descriptor in global memory; a kernel that stores to global memory
// in its loop copies the parts it reads into its own variables first
// (through the reference, the compiler must reload them after each store,
// which it cannot tell apart from the descriptor).
#define KM_MEMBER                                   \
  const int2 km_e_ = __ldg(tab + blockIdx.x);       \
  const int b = km_e_.y;                            \
  Member& M = mem[km_e_.x]
#endif

}  // namespace irbc
