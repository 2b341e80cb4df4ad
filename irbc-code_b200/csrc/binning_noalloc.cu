// binning_noalloc.cu -- the random-shift binning of irbc_bin_particles
// without any memory allocation, for callers that cannot allocate device
// memory while they run: code inside an allocator callback or a memory
// pool's reservation path, host threads that must not take the driver's
// allocation lock, and embedders whose device memory is budgeted up front.
//
// Its scratch (per-cell counters, scan partial sums and totals) lives in one
// file-scope __device__ array of fixed size, present on every GPU that loads
// the library until the process exits.  The caller passes the particle
// positions and the three output arrays, all in device memory.
#include <cstdint>
#include <mutex>

#include "irbc.h"
#include "sim.h"

namespace irbc {

// limits of the static scratch
constexpr int64_t kNoAllocMaxCells = 1 << 20;                      // 1,048,576 cells (4 MiB of counters)
constexpr int64_t kNoAllocScanBlocks = (kNoAllocMaxCells + 1024) / 1024 + 1;  // scan tiles of 1024
constexpr int64_t kNoAllocInts = kNoAllocMaxCells + 3 * kNoAllocScanBlocks + 3 + 8;

// [0, C) counters | 3 ints per scan tile | totals
static __device__ __align__(256) int g_bin_scratch[kNoAllocInts];

__global__ void k_na_count(DevParams p, const double* x, const double* y, const double* z, int64_t n,
                           double rx, double ry, double rz, int* cell, int* cnt) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned act = __ballot_sync(0xffffffffu, i < n);
  if (i >= n) return;
  int fx = (int)floor(bbound(x[i] - rx, p.Lx));
  int fy = (int)floor(bbound(y[i] - ry, p.Ly));
  int fz = (int)floor(z[i] - rz + 1.0);
  int c = cell_of(p, fx, fy, fz);
  unsigned peers = __match_any_sync(act, c);
  int leader = __ffs(peers) - 1;
  if ((int)(threadIdx.x & 31) == leader) atomicAdd(&cnt[c], __popc(peers));
  cell[i] = c;
}

// second pass: the counters (cleared again) hand out positions in each cell
__global__ void k_na_fill(const int* cell, const int* start, int64_t n, int* cnt, int* order) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int c = cell[i];
  order[(int64_t)start[c] + atomicAdd(&cnt[c], 1)] = (int)i;
}

__global__ void k_na_segsort(const int* start, int64_t ncell, int* order) {
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

namespace {
// Device address of g_bin_scratch per device ordinal.  The host symbol is a
// stand-in and must not be handed to a kernel, so the address is looked up
// once per device with cudaGetSymbolAddress while that device is current,
// and kept for the life of the process.  A cudaDeviceReset unloads the
// module and can move the array, leaving the kept address stale: this entry
// point must not be used on a device after it has been reset.
std::mutex g_scratch_mu;
int* g_scratch_dev[256] = {nullptr};

int scratch_for_current_device(int** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256) return IRBC_ERR_CUDA;
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_dev[dev]) {
    void* ptr = nullptr;
    if (cudaGetSymbolAddress(&ptr, g_bin_scratch) != cudaSuccess || !ptr) return IRBC_ERR_CUDA;
    g_scratch_dev[dev] = static_cast<int*>(ptr);
  }
  *out = g_scratch_dev[dev];
  return 0;
}
}  // namespace

}  // namespace irbc

using namespace irbc;

extern "C" int irbc_bin_particles_noalloc(const irbc_params* p, const double* x, const double* y,
                                          const double* z, int64_t n, double rx, double ry, double rz,
                                          int32_t* cell, int32_t* start, int32_t* order) {
  if (!p || n < 0 || (n > 0 && (!x || !y || !z || !cell || !order)) || !start) return IRBC_ERR_ARG;
  if (p->a != 1.0 || p->Lx <= 0 || p->Ly <= 0 || p->Lz <= 0 || n >= (1LL << 31)) return IRBC_ERR_ARG;
  if (!(rx >= 0 && rx < 1 && ry >= 0 && ry < 1 && rz >= 0 && rz < 1)) return IRBC_ERR_ARG;
  DevParams d{};  // the grid fields the binning reads
  d.a = p->a; d.Lx = p->Lx; d.Ly = p->Ly; d.Lz = p->Lz;
  d.nx = (int)(p->Lx / p->a);
  d.ny = (int)(p->Ly / p->a);
  d.nz = (int)(p->Lz / p->a) + 1;
  d.ncell = (int64_t)d.nx * d.ny * d.nz;
  if (d.ncell > kNoAllocMaxCells) return IRBC_ERR_CAPACITY;  // box beyond the static scratch
  int* base = nullptr;
  int rc = scratch_for_current_device(&base);
  if (rc) return rc;
  int* cnt = base;
  int* part = base + kNoAllocMaxCells;
  int* totals = part + 3 * kNoAllocScanBlocks + 3;
  const cudaStream_t st = 0;
  // the array keeps the previous call's contents: clear the counters
  if (cudaMemsetAsync(cnt, 0, sizeof(int) * d.ncell, st) != cudaSuccess) return IRBC_ERR_CUDA;
  if (n) k_na_count<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(d, x, y, z, n, rx, ry, rz, cell, cnt);
  launch_scan3(cnt, nullptr, nullptr, start, nullptr, nullptr, totals, d.ncell, part, st);
  if (cudaMemcpyAsync(start + d.ncell, totals, sizeof(int), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
    return IRBC_ERR_CUDA;
  if (cudaMemsetAsync(cnt, 0, sizeof(int) * d.ncell, st) != cudaSuccess) return IRBC_ERR_CUDA;
  if (n) k_na_fill<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(cell, start, n, cnt, order);
  k_na_segsort<<<(unsigned)((d.ncell + 255) / 256), 256, 0, st>>>(start, d.ncell, order);
  if (cudaGetLastError() != cudaSuccess) return IRBC_ERR_CUDA;
  return cudaStreamSynchronize(st) == cudaSuccess ? 0 : IRBC_ERR_CUDA;
}
