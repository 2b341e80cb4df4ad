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

struct FastBufs {
  Snap snap[2];
  TriPre* pre[2] = {nullptr, nullptr};
  int* queue = nullptr;   // particles with long cell lists (capacity Ns)
  int* qn = nullptr;
  double* slot = nullptr; // force terms: 3 doubles per slot, 4E + 9T + 4E slots
  int* gstart = nullptr;  // per-vertex slot lists in the reference's order
  int* gidx = nullptr;
  int* vd = nullptr;      // bond draws per vertex this step
  int* vw = nullptr;      // vertex within the parasite's WCA cutoff
  double* vX = nullptr;   // its WCA force (3 per vertex)
};

void fast_kick_prep(const DevParams& p, Membrane& m, FastBufs& f, int buf, cudaStream_t st);
void fast_snap_prep(const DevParams& p, Membrane& m, FastBufs& f, int buf, cudaStream_t st);
void fast_stream(const DevParams& p, Solvent& s, const Cells& c, FastBufs& f, int buf, cudaStream_t st);
// these return the number of kernels they launched
int fast_drift_va(const DevParams& p, Membrane& m, cudaStream_t st, bool with_sum);
int fast_forces_tail(const DevParams& p, Membrane& m, FastBufs& f, uint64_t epoch, int next_kick, int next_buf,
                     cudaStream_t st, bool sum_pending);

}  // namespace irbc
