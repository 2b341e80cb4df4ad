// fast.h -- buffers and launchers of the production step (fast.cu).
#pragma once
#include "sim.h"

namespace irbc {

// per-triangle data of reflectionFed at rstep = 0 (Src/solfuncs.cpp:457-517)
struct TriPre {
  double X[3], Xdt[3], A1[3], A2[3];
};

// vertex positions/velocities as seen by one streaming step
struct Snap {
  double *x, *y, *z, *vx, *vy, *vz;
  const int *t1, *t2, *t3;
};

// near-membrane streaming: particles per listed cell taken by the cell's
// block, the longest list staged in its shared memory, and the blocks that
// walk the overflow queue
constexpr int kBucket = 32;
constexpr int kHeavyList = 1024;
constexpr int kOverflowBlocks = 8;
// Lists of up to kShortList entries (staging capacity hcap) take the
// short-list path: one warp per listed cell, its lanes shared among the
// cell's particles, from a staging of kLanePiece entries per warp
// (kShortWarps such warps per block), then the overflow queue's walk.
// Longer lists: the near-membrane kernel stages a listed cell's TriPre
// records in shared memory a piece at a time, eight warps per block
// (kStageLong entries per piece).  The kernel's registers allow two
// eight-warp blocks per SM, which a whole 1024-entry list per block also
// allows, so a bucketed list (at most kHeavyList entries) is one piece.
constexpr int kShortList = 128, kStageLong = kHeavyList;
constexpr int kShortWarps = 4, kLanePiece = 64;
// blocks of eight warps that walk the overflow queue after the short-list
// kernel: per simulation alone, and per member of a cohort
constexpr int kQueueBlocks = 64, kQueueBlocksMember = 32;
// the short-list kernel runs without the full test's registers: 64 per
// thread, eight blocks (32 warps) per SM
constexpr int kShortMinBlocks = 8;
inline bool short_lists(int hcap) { return hcap <= kShortList; }
// the staging piece of the long-list kernel
inline int stage_cap(int hcap) { return hcap < kStageLong ? (hcap > 0 ? hcap : 1) : kStageLong; }
inline int stage_bytes(int cap) { return cap * (int)(sizeof(TriPre) + sizeof(int)); }

struct FastBufs {
  Snap snap[2];
  TriPre* pre[2] = {nullptr, nullptr};
  int* queue = nullptr;   // overflow: particles of full buckets or over-long lists (capacity Ns)
  int* qn = nullptr;
  int* bcnt = nullptr;    // particles handed to each listed cell this step (reset by k_stream_cells)
  int* bucket = nullptr;  // kBucket particle slots per listed cell
  int64_t bcap = 0;       // listed cells the buckets have room for
  int* border = nullptr;  // the listed cell (rank) of each k_stream_cells block: longest lists first
  int2* arng = nullptr;   // (first entry, length) of each listed cell's list, by rank (bcap of them)
  bool one_block = false; // the membrane step as one block per launch (small meshes)
  bool cluster = false;   // the membrane step as one launch of a thread-block cluster (any mesh)
  int hcap = kHeavyList;  // list entries k_stream_cells stages (its shared memory); longer lists go
                          // to the overflow queue
  double* slot = nullptr; // force terms: 3 doubles per slot, 4E + 9T + 4E slots
  int* gstart = nullptr;  // per-vertex slot lists in the reference's order
  int* gidx = nullptr;
  int* vd = nullptr;      // bond draws per vertex this step
  int* vw = nullptr;      // vertex within the parasite's WCA cutoff
  double* vX = nullptr;   // its WCA force (3 per vertex)
};

// these return the number of kernels they launched
int fast_kick_prep(const DevParams& p, Membrane& m, FastBufs& f, int buf, cudaStream_t st);
void fast_snap_prep(const DevParams& p, Membrane& m, FastBufs& f, int buf, cudaStream_t st);
// list length of each listed cell (rank a < nact) into len[a], and its
// (first entry, length) into rng[a]
void launch_rank_lengths(const Cells& c, int* len, int2* rng, cudaStream_t st);
// the staging capacity for lists of at most lmax entries: lmax rounded up
// to 64, at least 64, at most kHeavyList
inline int heavy_cap(int lmax) {
  int c = ((lmax + 63) / 64) * 64;
  return c < 64 ? 64 : (c > kHeavyList ? kHeavyList : c);
}
// ev0/ev1 (optional) are recorded around the bulk kernel k_stream_fast.  The
// bulk kernel reads no membrane data; the near-membrane kernels read the
// snapshot `buf` and first wait for `snap` (optional: its producer).
// Returns the number of kernels it launched.
int fast_stream(const DevParams& p, Solvent& s, const Cells& c, FastBufs& f, int buf, cudaStream_t st,
                cudaEvent_t ev0 = nullptr, cudaEvent_t ev1 = nullptr, cudaEvent_t snap = nullptr);
// these return the number of kernels they launched
int fast_drift_va(const DevParams& p, Membrane& m, cudaStream_t st, bool with_sum);
bool is_membrane_kernel(const void* fn);
// next_kick: also the next step's half-kick and snapshot into next_buf,
// after waiting for `readers` (optional: the last streaming that read it)
int fast_forces_tail(const DevParams& p, Membrane& m, FastBufs& f, uint64_t epoch, int next_kick, int next_buf,
                     cudaStream_t st, bool sum_pending, cudaEvent_t readers = nullptr);
// the whole membrane step of irbc_step (drift .. bond_dynamics, then the
// next half-kick and snapshot as fast_forces_tail): in one launch of a
// thread-block cluster when f.cluster, in one block per launch when
// f.one_block, else fast_drift_va + fast_forces_tail
int fast_membrane_step(const DevParams& p, Membrane& m, FastBufs& f, uint64_t epoch, int next_kick, int next_buf,
                       cudaStream_t st, cudaEvent_t readers = nullptr);
// whether a mesh suits the one-block membrane step
bool one_block_fits(const DevParams& p);
// every kernel's dynamic shared-memory limit on the current device (before
// any launch; irbc_create calls it)
void set_kernel_limits();

}  // namespace irbc
