// fp32.h -- the FP32-bulk solvent state and its launchers (fp32.cuh).
#pragma once
#include "fast.h"

namespace irbc {

// 32 bytes per particle: (x, y, z, inside flag as int bits) and
// (vx, vy, vz, reference index as int bits); two buffer sets for the
// counting sort; pid = collision cell of the last collision
struct SolventF {
  int64_t n = 0;
  float4 *pos = nullptr, *vel = nullptr, *pos2 = nullptr, *vel2 = nullptr;
  int *pid = nullptr, *pid2 = nullptr;
};

void f32_from_f64(Solvent& s, SolventF& f, cudaStream_t st);
void f32_to_f64(SolventF& f, Solvent& s, cudaStream_t st);
void launch_collide_count_f(const DevParams& p, SolventF& f, Solvent& s, Cells& c, uint64_t epoch,
                            cudaStream_t st);
void launch_collide_finish_f(const DevParams& p, SolventF& f, Solvent& s, Cells& c, Membrane& m, uint64_t epoch,
                             cudaStream_t st, bool resort);
void launch_resort_f(SolventF& f, Solvent& s, cudaStream_t st);
// ev0/ev1 (optional) are recorded around the bulk kernel k_stream_f; the
// near-membrane kernels wait for `snap` (optional: the snapshot's
// producer).  Returns the number of kernels it launched.
int fast_stream_f(const DevParams& p, SolventF& f, const Cells& c, FastBufs& fb, int buf, cudaStream_t st,
                  cudaEvent_t ev0 = nullptr, cudaEvent_t ev1 = nullptr, cudaEvent_t snap = nullptr);

}  // namespace irbc
