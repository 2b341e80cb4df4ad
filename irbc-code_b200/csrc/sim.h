// sim.h -- device-resident state of one simulation and the launchers of the
// kernels that advance it.  Layout in HBM (FP64 build):
//   solvent    SoA double x,y,z; one 32-byte record (vx, vy, vz, reference
//              index) per particle; int indio, pid; re-sorted physically by
//              collision cell every kResortEvery collisions (second buffer set)
//   cells      int cnt, start (exclusive scan), ncm (membrane vertices),
//              ghost ranks
//   llist      CSR lstart[C+1], lidx[cap], double-buffered
//   membrane   SoA vertex arrays, topology, per-vertex incidence lists
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "common.cuh"

namespace irbc {

// velocity and reference index of a solvent particle in one 32-byte record:
// the collision, which visits particles in cell order, reads and writes one
// sector per particle
struct __align__(16) SolVel {
  double vx, vy, vz;
  int id, pad;
};

struct Solvent {
  int64_t n = 0;
  double *x = nullptr, *y = nullptr, *z = nullptr;
  SolVel* v = nullptr;
  int *indio = nullptr, *pid = nullptr;
  double *x2 = nullptr, *y2 = nullptr, *z2 = nullptr;
  SolVel* v2 = nullptr;
  int *indio2 = nullptr, *pid2 = nullptr;
  int *key = nullptr, *slot = nullptr;
  int *perm = nullptr;          // particle indices grouped by collision cell
  int64_t ncoll = 0;            // collisions so far (host count)
  int64_t resorted = 0;         // ncoll at the last physical re-sort
};

// every kResortEvery-th collision also re-sorts the particle arrays
// physically by cell; in between the cells read their particles through perm
constexpr int kResortEvery = 16;

struct Cells {
  int64_t n = 0;
  int *cnt = nullptr, *start = nullptr, *ncm = nullptr, *wrank = nullptr, *mrank = nullptr;
  int *totals = nullptr;        // [0] particles, [1] wall ghost cells, [2] membrane ghost cells,
                                // [4] cells with a list, [7] longest list, [8] llist entries,
                                // [11] bad particle ids seen by get_state
  int *lstart = nullptr, *lidx = nullptr, *lstart2 = nullptr, *lidx2 = nullptr, *lcnt = nullptr;
  int64_t lcap = 0, lcap2 = 0;
  int *lrank = nullptr;         // rank among the cells with a non-empty list
  int *acell = nullptr;         // the cell of each such rank
  int nact = 0, lmax = 0;       // (host) their number and the longest list
  int *scan_part = nullptr;     // scan scratch: 3 ints per block
  int64_t scan_blocks = 0;
};

// device scalars of the membrane / parasite (one small struct)
struct MemScalars {
  double Sarea, Volume;
  double para[3], paraV[3], paraft[3], parafdt[3];
  int paradx, parady, paraid, pad;
};

struct Membrane {
  int nv = 0, ne = 0, nt = 0;
  double *x = nullptr, *y = nullptr, *z = nullptr, *vx = nullptr, *vy = nullptr, *vz = nullptr;
  double *fx = nullptr, *fy = nullptr, *fz = nullptr, *poff = nullptr, *pon = nullptr;
  int *pid = nullptr, *ix = nullptr, *iy = nullptr, *bondi = nullptr, *bondl = nullptr, *knob = nullptr;
  int *e1 = nullptr, *e2 = nullptr, *es1 = nullptr, *es2 = nullptr, *iedge = nullptr;
  int *t1 = nullptr, *t2 = nullptr, *t3 = nullptr;
  double *l0 = nullptr, *kappap = nullptr, *tarea = nullptr;
  double *area = nullptr, *vol = nullptr;     // per triangle, TotalVA terms
  double *tcx = nullptr, *tcy = nullptr, *tcz = nullptr;  // centroids for llistupdate
  int *inc_start = nullptr, *inc = nullptr;   // per-vertex contributions in reference order
  uint64_t *vkey = nullptr;                   // (cell << 32 | vertex), sorted each collision
  int *npair = nullptr;                       // bond candidates per vertex
  double *pair_d = nullptr;
  int *pair_j = nullptr;
  int *ligi = nullptr;
  double *xlig = nullptr, *ylig = nullptr;   // ligand grid (maincode.cpp:77-93)
  MemScalars* sc = nullptr;
};

// observables scratch (doubles): [0, 16) results and sums; from 64 the
// velocity profile of irbc_velocity_profile (2 per bin); from kObsLayers the
// per-layer sums of vx, vy, vz and the count behind the temperature
constexpr int kObsMaxBins = 2048;
constexpr int kObsLayers = 64 + 2 * kObsMaxBins;
constexpr int kObsDoubles = kObsLayers + 4 * kObsMaxBins;

constexpr int kMaxPairs = 64;        // bond candidates per vertex (<= 25 with dthr = 0.5)

// ---- launchers (kernels.cu) ---------------------------------------------------
void launch_init_solvent(const DevParams& p, Solvent& s, cudaStream_t st);
// *d = v in stream order (no host staging, no host wait)
void launch_set_u64(uint64_t* d, uint64_t v, cudaStream_t st);
// velocity records from / to plain arrays (state exchange); a null vx keeps
// the velocities, a null id keeps the indices
// d[i] = i for i < n
void launch_iota(int* d, int64_t n, cudaStream_t st);
void launch_pack_vel(Solvent& s, const double* vx, const double* vy, const double* vz, const int* id,
                     cudaStream_t st);
void launch_unpack_vel(const Solvent& s, double* vx, double* vy, double* vz, int* id, cudaStream_t st);
void launch_unpermute(const Solvent& s, int velocities, int* bad, cudaStream_t st);
void launch_classify(const DevParams& p, Solvent& s, const Membrane& m, cudaStream_t st);
// a collision = launch_vbin (membrane only) + launch_collide_count (solvent
// only) in any order or on two streams, then launch_collide_finish
// the shared-memory limits of the collision kernels on the current device
void set_collide_kernel_limits();
void launch_vbin(const DevParams& p, Membrane& m, Cells& c, uint64_t epoch, cudaStream_t st);
void launch_collide_count(const DevParams& p, Solvent& s, Cells& c, uint64_t epoch, cudaStream_t st);
// resort: also re-sort the arrays physically by this collision's cells
void launch_collide_finish(const DevParams& p, Solvent& s, Cells& c, Membrane& m, uint64_t epoch,
                           cudaStream_t st, bool resort);
// physical re-sort by the cells of the latest collision (any time after it)
void launch_resort(Solvent& s, cudaStream_t st);
void launch_ghost_flags(const DevParams& p, Cells& c, const Membrane& m, cudaStream_t st);
void launch_stream(const DevParams& p, Solvent& s, const Cells& c, const Membrane& m, cudaStream_t st);
// returns the total list length the update needs (host sync inside)
int64_t launch_llist_count(const DevParams& p, Cells& c, const Membrane& m, cudaStream_t st);
// total: the entry count launch_llist_count returned (both list buffers hold it)
void launch_llist_fill(const DevParams& p, Cells& c, const Membrane& m, int64_t total, cudaStream_t st);
// lrank / acell / nact / lmax of the current lists (host sync inside);
// returns the kernels launched, -1 on a CUDA error
int launch_llist_ranks(const DevParams& p, Cells& c, cudaStream_t st);
void launch_half_kick(const DevParams& p, Membrane& m, cudaStream_t st);
void launch_drift(const DevParams& p, Membrane& m, cudaStream_t st);
void launch_total_va(const DevParams& p, Membrane& m, cudaStream_t st);
void launch_pfdt_forces(const DevParams& p, Membrane& m, int do_pfdt, int do_forces, int do_ext,
                        cudaStream_t st);
void launch_bonds(const DevParams& p, Membrane& m, uint64_t epoch, cudaStream_t st);
void launch_kick2(const DevParams& p, Membrane& m, cudaStream_t st);
void launch_scan3(const int* a, const int* b, const int* c, int* oa, int* ob, int* oc, int* totals,
                  int64_t n, int* part, cudaStream_t st);
// obs: the kObsDoubles scratch; nbins > 0 also fills the velocity profile
// (obs + 64, nbins <= kObsMaxBins)
void launch_observables(const DevParams& p, const Solvent& s, const Membrane& m, double* obs, int nbins,
                        cudaStream_t st);

int64_t scan_part_blocks(int64_t n);

}  // namespace irbc
