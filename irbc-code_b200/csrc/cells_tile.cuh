// cells_tile.cuh -- the per-cell part of CollisionStep (Src/solfuncs.cpp:164-318)
// and the rotation of CollisionDyn / CollisionDynmem / CollisionDynpara
// (:700-810), as one kernel over tiles of 32 consecutive collision cells.
//
// One block of two warps per tile.  The tile's particles are contiguous in
// perm (the counting sort's output), so the block gathers their velocity
// records into shared memory with independent loads (no dependent chain
// per cell) and ranks each particle within its cell by reference index
// (the order of Cells[].sol).  Lane l of the first warp then forms cell l's
// vcm and ThE with the sums in the reference's order while lane l of the
// second draws its axis, and the block rotates the tile's particles and
// writes their records back.  Sharing a tile between two warps halves the
// shared memory and the gather registers per warp.  A tile with more
// particles than the shared buffer holds falls back to one lane per cell
// reading global memory.
//
// Included by kernels.cu (FP64 solvent) and fp32.cuh (FP32-bulk solvent).
#pragma once
#include "fp32.h"

namespace irbc {

__device__ __forceinline__ void rotate_v(double v[3], const double* P, double cosalpha, double sinalpha) {
  // CollisionDyn (:711-733) with the cell's vcm (P[0..2]), axis (P[3..5]), ThE (P[6])
  double unit[3] = {P[3], P[4], P[5]}, dvv[3], dvp[3], dvn[3], dvpn[3];
  double scalev = P[6];
  for (int k = 0; k < 3; ++k) dvv[k] = v[k] - P[k];
  double xxx = dvv[0] * unit[0] + dvv[1] * unit[1] + dvv[2] * unit[2];
  for (int k = 0; k < 3; ++k) dvp[k] = xxx * unit[k];
  for (int k = 0; k < 3; ++k) dvn[k] = dvv[k] - dvp[k];
  cp(dvn, unit, dvpn);
  for (int k = 0; k < 3; ++k) v[k] = P[k] + scalev * (cosalpha * dvn[k] + sinalpha * dvpn[k] + dvp[k]);
}

// the FP32-bulk rotation: float arithmetic on the float-rounded parameters
__device__ __forceinline__ float4 rotate_f(float4 v, const double* P, float cosalpha, float sinalpha) {
  const float ax = (float)P[0], ay = (float)P[1], az = (float)P[2];
  const float ux = (float)P[3], uy = (float)P[4], uz = (float)P[5], s = (float)P[6];
  float dx = v.x - ax, dy = v.y - ay, dz = v.z - az;
  float xx = dx * ux + dy * uy + dz * uz;
  float px = xx * ux, py = xx * uy, pz = xx * uz;
  float nx = dx - px, ny = dy - py, nz = dz - pz;
  float cx = (ny * uz) - (uy * nz), cy = (nz * ux) - (uz * nx), cz = (nx * uy) - (ux * ny);
  v.x = ax + s * (cosalpha * nx + sinalpha * cx + px);
  v.y = ay + s * (cosalpha * ny + sinalpha * cy + py);
  v.z = az + s * (cosalpha * nz + sinalpha * cz + pz);
  return v;
}

// vcm, axis and ThE of cell c (7 doubles into P) given its n solvent
// particles in reference order (vel_at(q, v) yields the q-th); rotates the
// cell's vertices and the parasite.  Sums in the order of :164-258: solvent,
// wall ghost, vertices in vertex order, parasite, membrane ghost.
// the per-cell values cell_par reads besides the velocities; loaded before
// the tile's gather so that their latency overlaps it
struct CellLook {
  int nmem, wrank, mrank, para, nwall;
};
__device__ __forceinline__ CellLook look_cell(const Cells& cl, const Membrane& m, int64_t c) {
  CellLook k;
  k.nmem = cl.ncm[c];
  k.wrank = cl.wrank[c];
  k.mrank = cl.mrank[c];
  k.para = (c == m.sc->paraid) ? 1 : 0;
  k.nwall = cl.totals[1];
  return k;
}

// the cell's membrane members: its vertices (entries [v0, v0 + nmem) of the
// sorted (cell, vertex) keys) and whether it holds the parasite
struct CellMembers {
  int nmem, v0;
  bool para;
};

// vcm (P[0..2]) and ThE (P[6]) of cell c given its n solvent particles in
// reference order (vel_at(q, v) yields the q-th).  Sums in the order of
// :164-258: solvent, wall ghost, vertices in vertex order, parasite,
// membrane ghost.
template <class VelAt>
__device__ __forceinline__ CellMembers cell_sums(const DevParams& p, const Cells& cl, const Membrane& m,
                                                 uint64_t epoch, int64_t c, int n, const CellLook& look,
                                                 VelAt vel_at, double P[7]) {
  const MemScalars* sc = m.sc;
  double vcm[3] = {0.0, 0.0, 0.0}, ncc = 0.0;
  int nc = 0;
  for (int q = 0; q < n; ++q) {
    double v[3];
    vel_at(q, v);
    vcm[0] += p.mass * v[0];
    vcm[1] += p.mass * v[1];
    vcm[2] += p.mass * v[2];
    ncc += (1 * p.mass);
    nc += 1;
  }
  const int k = c < 0x7fffffff ? (int)((unsigned)c % (unsigned)p.nz) : (int)(c % p.nz);
  const double zmin = -1.0 + (double)k * p.a, zmax = -1.0 + (double)k * p.a + p.a;
  {
    // wall ghost particle (:185-204): mean (navg - n) * wallspeed in x at the top
    int nn = nc;
    if ((zmax >= p.Lz || zmin <= 0) && nn < p.navg) {
      const uint64_t g = 3 * (uint64_t)look.wrank;
      const double sd = sqrt((p.navg - nn) * p.Theta / p.mass);
      const double mx = zmax >= p.Lz ? (p.navg - nn) * p.wallspeed : 0.0;
      vcm[0] += p.mass * (draw_normal(p.seed, STREAM_COLLIDE_N, epoch, g + 0) * sd + mx);
      vcm[1] += p.mass * (draw_normal(p.seed, STREAM_COLLIDE_N, epoch, g + 1) * sd + 0);
      vcm[2] += p.mass * (draw_normal(p.seed, STREAM_COLLIDE_N, epoch, g + 2) * sd + 0);
      ncc = p.navg * p.mass;
    }
  }
  // vertices of this cell: their range in the sorted (cell, vertex) keys
  const int nmem = look.nmem;
  int v0 = 0;
  if (nmem > 0) {
    int lo = 0, hi = p.nv;
    const uint64_t key0 = (uint64_t)(uint32_t)c << 32;
    while (lo < hi) { int mid = (lo + hi) >> 1; if (m.vkey[mid] < key0) lo = mid + 1; else hi = mid; }
    v0 = lo;
    for (int q = 0; q < nmem; ++q) {
      int i = (int)(m.vkey[v0 + q] & 0xffffffffu);
      vcm[0] += p.pmass * m.vx[i];
      vcm[1] += p.pmass * m.vy[i];
      vcm[2] += p.pmass * m.vz[i];
      ncc += (1 * p.pmass);
      nc += 1;
    }
  }
  const bool has_para = look.para != 0;
  if (has_para) {
    vcm[0] += p.PRmass * sc->paraV[0];
    vcm[1] += p.PRmass * sc->paraV[1];
    vcm[2] += p.PRmass * sc->paraV[2];
    ncc += (1 * p.PRmass);
    nc += 1;
  }
  {
    // membrane ghost (:236-244)
    int nn = nc;
    if ((nn < p.navg) && (nmem > 0)) {
      const uint64_t g = 3 * ((uint64_t)look.nwall + (uint64_t)look.mrank);
      const double sd = sqrt((p.navg - nn) * p.Theta / p.mass);
      vcm[0] += p.mass * (draw_normal(p.seed, STREAM_COLLIDE_N, epoch, g + 0) * sd + 0);
      vcm[1] += p.mass * (draw_normal(p.seed, STREAM_COLLIDE_N, epoch, g + 1) * sd + 0);
      vcm[2] += p.mass * (draw_normal(p.seed, STREAM_COLLIDE_N, epoch, g + 2) * sd + 0);
      ncc += (p.navg - nn) * p.mass;
    }
  }
  {
    int nn = (int)ncc;
    if (nn != 0) { vcm[0] /= (double)nn; vcm[1] /= (double)nn; vcm[2] /= (double)nn; }
  }
  double dvv = 0.0;
  for (int q = 0; q < n; ++q) {
    double v[3];
    vel_at(q, v);
    double A0 = v[0] - vcm[0], A1 = v[1] - vcm[1], A2 = v[2] - vcm[2];
    double aa = (A0 * A0 + A1 * A1 + A2 * A2);
    dvv += (p.mass * aa);
  }
  for (int q = 0; q < nmem; ++q) {
    int i = (int)(m.vkey[v0 + q] & 0xffffffffu);
    double A0 = m.vx[i] - vcm[0], A1 = m.vy[i] - vcm[1], A2 = m.vz[i] - vcm[2];
    double aa = (A0 * A0 + A1 * A1 + A2 * A2);
    dvv += (p.pmass * aa);
  }
  if (has_para) {
    double A0 = sc->paraV[0] - vcm[0], A1 = sc->paraV[1] - vcm[1], A2 = sc->paraV[2] - vcm[2];
    double aa = (A0 * A0 + A1 * A1 + A2 * A2);
    dvv += (p.PRmass * aa);
  }
  double ThE = 1.0;
  if ((nc > 0) && (dvv != 0)) ThE = sqrt(3.0 * ((double)nc - 1.0) * p.Theta / (dvv));
  P[0] = vcm[0]; P[1] = vcm[1]; P[2] = vcm[2];
  P[6] = ThE;
  return CellMembers{nmem, v0, has_para};
}

// the collision axis of cell c (P[3..5], :262-271): uniforms 3+2c and 4+2c
// of the COLLIDE_U stream (one Philox block when both fall into it)
__device__ __forceinline__ void cell_axis(const DevParams& p, uint64_t epoch, int64_t c, double P[7]) {
  double rand1, rand2;
  {
    const uint64_t k1 = 3 + 2 * (uint64_t)c, k2 = k1 + 1;
    uint32_t o1[4], o2[4];
    draw_block(p.seed, STREAM_COLLIDE_U, epoch, k1 >> 2, o1);
    if ((k2 >> 2) == (k1 >> 2)) { for (int e = 0; e < 4; ++e) o2[e] = o1[e]; }
    else draw_block(p.seed, STREAM_COLLIDE_U, epoch, k2 >> 2, o2);
    rand1 = 2.0 * p.Pi * ((double)o1[k1 & 3u] * (1.0 / 4294967296.0));
    rand2 = -1.0 + (2.0 * ((double)o2[k2 & 3u] * (1.0 / 4294967296.0)));
  }
  P[3] = sqrt(1.0 - (rand2 * rand2)) * cos(rand1);
  P[4] = sqrt(1.0 - (rand2 * rand2)) * sin(rand1);
  P[5] = rand2;
}

// CollisionDynmem (:739-776) and CollisionDynpara (:779-810), in double:
// the cell's vertices and the parasite rotated with the cell's parameters
__device__ __forceinline__ void cell_rotate_members(const DevParams& p, const Membrane& m, const CellMembers& cm,
                                                    const double P[7]) {
  const int nmem = cm.nmem, v0 = cm.v0;
  const bool has_para = cm.para;
  for (int q = 0; q < nmem; ++q) {
    int i = (int)(m.vkey[v0 + q] & 0xffffffffu);
    double v[3] = {m.vx[i], m.vy[i], m.vz[i]};
    rotate_v(v, P, p.cosalpha, p.sinalpha);
    m.vx[i] = v[0]; m.vy[i] = v[1]; m.vz[i] = v[2];
  }
  if (has_para) {
    MemScalars* scw = m.sc;
    double v[3] = {scw->paraV[0], scw->paraV[1], scw->paraV[2]};
    rotate_v(v, P, p.cosalpha, p.sinalpha);
    scw->paraV[0] = v[0]; scw->paraV[1] = v[1]; scw->paraV[2] = v[2];
  }
}

// all seven parameters of cell c, then its vertices and parasite rotated
template <class VelAt>
__device__ __forceinline__ void cell_par(const DevParams& p, const Cells& cl, const Membrane& m, uint64_t epoch,
                                         int64_t c, int n, const CellLook& look, VelAt vel_at, double P[7]) {
  const CellMembers cm = cell_sums(p, cl, m, epoch, c, n, look, vel_at, P);
  cell_axis(p, epoch, c, P);
  cell_rotate_members(p, m, cm, P);
}

constexpr int kTileCells = 32;   // cells per tile (one per lane of the first warp)
constexpr int kTileCap = 400;    // particles a tile holds in shared memory (mean 32 * navg)
constexpr int kTileWarps = 2;    // warps per block; the block's two warps share one tile
constexpr int kTileThreads = 32 * kTileWarps;
constexpr int kTilePer = (kTileCap + kTileThreads - 1) / kTileThreads;  // gathers in flight per thread
constexpr int kMaxSeg = 48;      // fallback: cells up to this size sort in registers

// one block's tile, in perm order; ord lists each cell's particles in
// reference order
struct CellTile {
  double vx[kTileCap], vy[kTileCap], vz[kTileCap];
  double P[kTileCells][7];
  int id[kTileCap];
  int st[kTileCells + 1];
  unsigned short ord[kTileCap];
  unsigned char cell[kTileCap];
};

template <bool F32>
__device__ __forceinline__ int load_id(const Solvent& s, const SolventF& f, int q) {
  if constexpr (F32) return __float_as_int(f.vel[q].w);
  else return s.v[q].id;
}

template <bool F32>
__device__ __forceinline__ void load_particle(const Solvent& s, const SolventF& f, int q, int& id, double v[3]) {
  if constexpr (F32) {
    float4 a = f.vel[q];
    id = __float_as_int(a.w);
    v[0] = (double)a.x; v[1] = (double)a.y; v[2] = (double)a.z;
  } else {
    const SolVel r = s.v[q];
    id = r.id;
    v[0] = r.vx; v[1] = r.vy; v[2] = r.vz;
  }
}

template <bool F32>
__device__ __forceinline__ void store_rotated(const DevParams& p, Solvent& s, SolventF& f, int q, int id,
                                              const double v[3], const double* P) {
  if constexpr (F32) {
    float4 a = make_float4((float)v[0], (float)v[1], (float)v[2], __int_as_float(id));
    f.vel[q] = rotate_f(a, P, (float)p.cosalpha, (float)p.sinalpha);
  } else {
    double w[3] = {v[0], v[1], v[2]};
    rotate_v(w, P, p.cosalpha, p.sinalpha);
    SolVel r;
    r.vx = w[0]; r.vy = w[1]; r.vz = w[2]; r.id = id; r.pad = 0;
    s.v[q] = r;
  }
}

// fallback for an over-full tile: cell c with its n particles at PP[0..n).
// Up to kMaxSeg particles are sorted in registers; up to kMaxSelect they are
// visited in reference order by successive selection (O(n) per particle,
// the two passes of cell_par each walk the order once); beyond that, a
// cell only a corrupted state can produce, the sums run in perm order so
// the kernel still ends in bounded time.
constexpr int kMaxSelect = 4096;
template <bool F32>
__device__ void cell_from_global(const DevParams& p, Solvent& s, SolventF& f, const Cells& cl, const Membrane& m,
                                 uint64_t epoch, int64_t c, const int* PP, int n) {
  int ord[kMaxSeg], oid[kMaxSeg];
  const bool small = n <= kMaxSeg;
  if (small) {
    for (int q = 0; q < n; ++q) {
      int pq = PP[q], idq = load_id<F32>(s, f, pq);
      int r = q;
      while (r > 0 && oid[r - 1] > idq) { ord[r] = ord[r - 1]; oid[r] = oid[r - 1]; --r; }
      ord[r] = pq;
      oid[r] = idq;
    }
  }
  // cursor of the selection walk: the q-th particle follows the (q-1)-th
  int cur_q = -1, cur_id = -1, cur_at = 0;
  auto nth = [&](int q) -> int {
    if (small) return ord[q];
    if (n > kMaxSelect) return PP[q];
    if (q != cur_q + 1) { cur_q = -1; cur_id = -1; }
    int best = 0x7fffffff, at = PP[0];
    for (int u = 0; u < n; ++u) {
      const int idu = load_id<F32>(s, f, PP[u]);
      if (idu > cur_id && idu < best) { best = idu; at = PP[u]; }
    }
    cur_q = q; cur_id = best; cur_at = at;
    return cur_at;
  };
  double P[7];
  cell_par(p, cl, m, epoch, c, n, look_cell(cl, m, c),
           [&](int q, double v[3]) { int id; load_particle<F32>(s, f, nth(q), id, v); }, P);
  for (int q = 0; q < n; ++q) {
    int id;
    double v[3];
    load_particle<F32>(s, f, PP[q], id, v);
    store_rotated<F32>(p, s, f, PP[q], id, v, P);
  }
}

// block `bid` of the collision tiles: one tile of kTileCells consecutive
// cells, shared by the block's two warps.  Both warps gather the tile's
// particles and rank them; then warp 0 forms each cell's ordered sums
// (vcm, ThE: lane l for cell l) while warp 1 draws each cell's rotation
// axis, the two halves of the cell's parameters; warp 0 then rotates the
// cells' membrane vertices and the parasite, and both warps rotate and
// write back the particles.  Every value is computed by the same
// operations in the same order as in cell_par.
template <bool F32>
__device__ __forceinline__ void cells_tile_block(const DevParams& p, Solvent& s, SolventF& f, const Cells& cl,
                                                 const Membrane& m, uint64_t eoff, int64_t bid) {
  const uint64_t epoch = epoch_of(p, eoff);
  __shared__ CellTile t;
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int64_t c0 = bid * kTileCells;
  if (c0 >= p.ncell) return;  // whole block
  const int ncl = (int)min((int64_t)kTileCells, p.ncell - c0);
  const int* __restrict__ perm = s.perm;
  const int S0 = cl.start[c0];
  const int stl = cl.start[c0 + min(lane, ncl)] - S0;
  const int total = cl.start[c0 + ncl] - S0;  // the same for the whole block
  if (total > kTileCap) {
    if (w == 0 && lane < ncl) {
      const int n = cl.start[c0 + lane + 1] - S0 - stl;
      cell_from_global<F32>(p, s, f, cl, m, epoch, c0 + lane, perm + S0 + stl, n);
    }
    return;
  }
  if (w == 0) {
    t.st[lane] = stl;
    if (lane == 0) t.st[kTileCells] = total;
  }
  // warp 0's cell values, in flight during the gather
  CellLook look{};
  if (w == 0 && lane < ncl) look = look_cell(cl, m, c0 + lane);
  // gather: one record per particle; every perm entry of the thread's
  // slots is loaded first, then every record, so the tile waits for two
  // memory latencies.  Each thread keeps its slots' particle and reference
  // indices for the write-back.
  int qv[kTilePer], idv[kTilePer];
  {
    double vv[kTilePer][3];
#pragma unroll
    for (int u = 0; u < kTilePer; ++u) {
      const int j = u * kTileThreads + tid;
      qv[u] = j < total ? perm[S0 + j] : -1;
    }
#pragma unroll
    for (int u = 0; u < kTilePer; ++u)
      if (qv[u] >= 0) load_particle<F32>(s, f, qv[u], idv[u], vv[u]);
#pragma unroll
    for (int u = 0; u < kTilePer; ++u) {
      const int j = u * kTileThreads + tid;
      if (qv[u] >= 0) {
        t.id[j] = idv[u];
        t.vx[j] = vv[u][0]; t.vy[j] = vv[u][1]; t.vz[j] = vv[u][2];
      }
    }
  }
  __syncthreads();
  if (w == 0) {
    const int e = t.st[lane + 1];
    for (int j = stl; j < e; ++j) t.cell[j] = (unsigned char)lane;
  }
  __syncthreads();
  // rank of each particle within its cell by reference index (indices are
  // unique): ord[b + rank] = its tile slot, the order of Cells[].sol
  for (int j = tid; j < total; j += kTileThreads) {
    const int l = t.cell[j], b = t.st[l], e = t.st[l + 1], me = t.id[j];
    int r = 0;
#pragma unroll 4
    for (int u = b; u < e; ++u) r += (t.id[u] < me) ? 1 : 0;
    t.ord[b + r] = (unsigned short)j;
  }
  __syncthreads();
  CellMembers cm{0, 0, false};
  if (lane < ncl) {
    double P[7];
    if (w == 0) {
      const int b = stl, n = t.st[lane + 1] - stl;
      cm = cell_sums(p, cl, m, epoch, c0 + lane, n, look,
                     [&](int q, double v[3]) {
                       const int j = t.ord[b + q];
                       v[0] = t.vx[j]; v[1] = t.vy[j]; v[2] = t.vz[j];
                     },
                     P);
      t.P[lane][0] = P[0]; t.P[lane][1] = P[1]; t.P[lane][2] = P[2]; t.P[lane][6] = P[6];
    } else {
      cell_axis(p, epoch, c0 + lane, P);
      t.P[lane][3] = P[3]; t.P[lane][4] = P[4]; t.P[lane][5] = P[5];
    }
  }
  __syncthreads();
  if (w == 0 && (cm.nmem > 0 || cm.para)) {
    double P[7];
    for (int e = 0; e < 7; ++e) P[e] = t.P[lane][e];
    cell_rotate_members(p, m, cm, P);
  }
  // rotation and write-back of this thread's slots
#pragma unroll
  for (int u = 0; u < kTilePer; ++u) {
    const int j = u * kTileThreads + tid;
    if (qv[u] >= 0) {
      const double v[3] = {t.vx[j], t.vy[j], t.vz[j]};
      store_rotated<F32>(p, s, f, qv[u], idv[u], v, t.P[t.cell[j]]);
    }
  }
}
template <bool F32>
__global__ void __launch_bounds__(32 * kTileWarps) k_cells_tile(DevParams p, Solvent s, SolventF f, Cells cl,
                                                               Membrane m, uint64_t eoff) {
  cells_tile_block<F32>(p, s, f, cl, m, eoff, blockIdx.x);
}

inline unsigned cells_tile_blocks(int64_t ncell) {
  return (unsigned)((ncell + kTileCells - 1) / kTileCells);  // one tile per block
}

}  // namespace irbc
