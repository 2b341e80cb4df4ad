// binning.cu -- standalone random-shift cell binning (counting sort) for
// callers that hold particle positions in device memory.
//
// Follows the binning of CollisionStep (Src/solfuncs.cpp:139-147): cell of a
// particle in the grid shifted by (rx, ry, rz) is cindex[floor(bbound(x-rx))]
// [floor(bbound(y-ry))][floor(z-rz+1)], then Cells[c].sol lists the
// particles of each cell in ascending index.  Here that list is the counting
// sort: start[C+1] (exclusive scan of the counts) and order[n] (particle
// indices grouped by cell, ascending within each cell).
#include <cstdint>
#include "irbc.h"
#include "sim.h"

namespace irbc {

__global__ void k_bin_cell(DevParams p, const double* x, const double* y, const double* z, int64_t n,
                           double rx, double ry, double rz, int* cell, int* slot, int* cnt) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned act = __ballot_sync(0xffffffffu, i < n);
  if (i >= n) return;
  const double r[3] = {rx, ry, rz};
  int fx = (int)floor(bbound(x[i] - r[0], p.Lx));
  int fy = (int)floor(bbound(y[i] - r[1], p.Ly));
  int fz = (int)floor(z[i] - r[2] + 1.0);
  int c = cell_of(p, fx, fy, fz);
  unsigned peers = __match_any_sync(act, c);
  int leader = __ffs(peers) - 1;
  int lane = threadIdx.x & 31;
  int rank = __popc(peers & ((1u << lane) - 1));
  int base = 0;
  if (lane == leader) base = atomicAdd(&cnt[c], __popc(peers));
  base = __shfl_sync(peers, base, leader);
  cell[i] = c;
  slot[i] = base + rank;
}

__global__ void k_bin_scatter(const int* cell, const int* slot, const int* start, int64_t n, int* order) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  order[(int64_t)start[cell[i]] + slot[i]] = (int)i;
}

// ascending particle index within each cell (insertion sort per segment)
__global__ void k_bin_segsort(const int* start, int64_t ncell, int* order) {
  int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  const int s0 = start[c], s1 = start[c + 1];
  for (int q = s0 + 1; q < s1; ++q) {
    int v = order[q];
    int r = q;
    while (r > s0 && order[r - 1] > v) { order[r] = order[r - 1]; --r; }
    order[r] = v;
  }
}

// The full sort on caller-provided scratch: cnt[C], slot[n], part[3*blocks+3], totals[4].
void bin_particles(const DevParams& p, const double* x, const double* y, const double* z, int64_t n,
                   double rx, double ry, double rz, int* cell, int* start, int* order, int* cnt, int* slot,
                   int* part, int* totals, cudaStream_t st) {
  cudaMemsetAsync(cnt, 0, sizeof(int) * p.ncell, st);
  if (n) k_bin_cell<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(p, x, y, z, n, rx, ry, rz, cell, slot, cnt);
  launch_scan3(cnt, nullptr, nullptr, start, nullptr, nullptr, totals, p.ncell, part, st);
  cudaMemcpyAsync(start + p.ncell, totals, sizeof(int), cudaMemcpyDeviceToDevice, st);
  if (n) k_bin_scatter<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(cell, slot, start, n, order);
  k_bin_segsort<<<(unsigned)((p.ncell + 255) / 256), 256, 0, st>>>(start, p.ncell, order);
}

}  // namespace irbc
