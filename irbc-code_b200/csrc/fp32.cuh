// fp32.cuh -- (part of fast.cu) the FP32-bulk solvent: positions and velocities stored as
// float4 (x, y, z, inside-flag bits) and (vx, vy, vz, reference-index bits),
// 32 bytes per particle.  Free flight, walls, wrap, binning and the SRD
// rotation run in float; the per-cell momentum and relative-energy sums are
// accumulated in double; particles near the membrane are promoted to double
// for reflectionFed and its cubic root solve; the membrane itself stays FP64.
#include <cstdio>
#include "fast.h"
#include "fp32.h"

namespace irbc {

static inline unsigned nbf(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

// ---- conversions between the FP64 arrays (set-up, state exchange) and FP32
__global__ void k_to_f32(Solvent s, SolventF f) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= s.n) return;
  f.pos[i] = make_float4((float)s.x[i], (float)s.y[i], (float)s.z[i], __int_as_float(s.indio[i]));
  f.vel[i] = make_float4((float)s.vx[i], (float)s.vy[i], (float)s.vz[i], __int_as_float(s.id[i]));
  f.pid[i] = s.pid[i];
}
__global__ void k_to_f64(SolventF f, Solvent s) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= s.n) return;
  float4 p = f.pos[i], v = f.vel[i];
  s.x[i] = p.x; s.y[i] = p.y; s.z[i] = p.z; s.indio[i] = __float_as_int(p.w);
  s.vx[i] = v.x; s.vy[i] = v.y; s.vz[i] = v.z; s.id[i] = __float_as_int(v.w);
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

__global__ void k_count_f(DevParams p, SolventF f, int* cnt, int* key, int* slot, uint64_t epoch) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t o[4];
  draw_block(p.seed, STREAM_COLLIDE_U, epoch, 0, o);
  const double r[3] = {p.a * ((double)o[0] * (1.0 / 4294967296.0)), p.a * ((double)o[1] * (1.0 / 4294967296.0)),
                       p.a * ((double)o[2] * (1.0 / 4294967296.0))};
  unsigned act = __ballot_sync(0xffffffffu, i < f.n);
  if (i >= f.n) return;
  int c = shifted_cell_f(p, f.pos[i], r);
  unsigned peers = __match_any_sync(act, c);
  int leader = __ffs(peers) - 1;
  int lane = threadIdx.x & 31;
  int rank = __popc(peers & ((1u << lane) - 1));
  int base = 0;
  if (lane == leader) base = atomicAdd(&cnt[c], __popc(peers));
  base = __shfl_sync(peers, base, leader);
  key[i] = c;
  slot[i] = base + rank;
}

__global__ void k_perm_f(const int* __restrict__ key, const int* __restrict__ slot, const int* __restrict__ start,
                         int64_t n, int* __restrict__ perm) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  perm[(int64_t)start[key[i]] + slot[i]] = (int)i;
}

// physical re-sort by collision cell every kResortEvery collisions
__global__ void k_gather_f(SolventF f, const int* __restrict__ perm) {
  int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= f.n) return;
  const int i = perm[j];
  f.pos2[j] = f.pos[i];
  f.vel2[j] = f.vel[i];
  f.pid2[j] = f.pid[i];
}

// per-cell statistics, one thread per cell, sums in double in reference
// particle order (CollisionStep, Src/solfuncs.cpp:164-318)
constexpr int kMaxSegF = 48;
__global__ void k_cells_f(DevParams p, SolventF f, const int* __restrict__ perm, Cells cl, Membrane m,
                          uint64_t epoch) {
  int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= p.ncell) return;
  const int64_t s0 = cl.start[c];
  const int n = cl.start[c + 1] - (int)s0;
  const int* __restrict__ PP = perm + s0;
  int ord[kMaxSegF], oid[kMaxSegF];
  const bool small = n <= kMaxSegF;
  if (small) {
    for (int q = 0; q < n; ++q) {
      int pq = PP[q];
      int idq = __float_as_int(f.vel[pq].w);
      int r = q;
      while (r > 0 && oid[r - 1] > idq) { ord[r] = ord[r - 1]; oid[r] = oid[r - 1]; --r; }
      ord[r] = pq;
      oid[r] = idq;
    }
  }
  auto nth = [&](int q) -> int64_t {
    if (small) return ord[q];
    int last = -1;
    int64_t at = PP[0];
    for (int t = 0; t <= q; ++t) {
      int best = 0x7fffffff;
      for (int u = 0; u < n; ++u) {
        int v = __float_as_int(f.vel[PP[u]].w);
        if (v > last && v < best) { best = v; at = PP[u]; }
      }
      last = best;
    }
    return at;
  };
  const MemScalars* sc = m.sc;
  double vcm[3] = {0.0, 0.0, 0.0}, ncc = 0.0;
  int nc = 0;
  for (int q = 0; q < n; ++q) {
    float4 v = f.vel[nth(q)];
    vcm[0] += p.mass * (double)v.x;
    vcm[1] += p.mass * (double)v.y;
    vcm[2] += p.mass * (double)v.z;
    ncc += (1 * p.mass);
    nc += 1;
  }
  const int k = (int)(c % p.nz);
  const double zmin = -1.0 + (double)k * p.a, zmax = -1.0 + (double)k * p.a + p.a;
  {
    int nn = nc;
    uint64_t g = 3 * (uint64_t)cl.wrank[c];
    if ((zmax >= p.Lz || zmin <= 0) && nn < p.navg) {
      const double sd = sqrt((p.navg - nn) * p.Theta / p.mass);
      const double mx = zmax >= p.Lz ? (p.navg - nn) * p.wallspeed : 0.0;
      vcm[0] += p.mass * (draw_normal(p.seed, STREAM_COLLIDE_N, epoch, g + 0) * sd + mx);
      vcm[1] += p.mass * (draw_normal(p.seed, STREAM_COLLIDE_N, epoch, g + 1) * sd + 0);
      vcm[2] += p.mass * (draw_normal(p.seed, STREAM_COLLIDE_N, epoch, g + 2) * sd + 0);
      ncc = p.navg * p.mass;
    }
  }
  const int nmem = cl.ncm[c];
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
  const bool has_para = (c == sc->paraid);
  if (has_para) {
    for (int q = 0; q < 3; ++q) vcm[q] += p.PRmass * sc->paraV[q];
    ncc += (1 * p.PRmass);
    nc += 1;
  }
  {
    int nn = nc;
    if ((nn < p.navg) && (nmem > 0)) {
      uint64_t g = 3 * ((uint64_t)cl.totals[1] + (uint64_t)cl.mrank[c]);
      const double sd = sqrt((p.navg - nn) * p.Theta / p.mass);
      for (int q = 0; q < 3; ++q) vcm[q] += p.mass * (draw_normal(p.seed, STREAM_COLLIDE_N, epoch, g + q) * sd + 0);
      ncc += (p.navg - nn) * p.mass;
    }
  }
  {
    int nn = (int)ncc;
    if (nn != 0) { vcm[0] /= (double)nn; vcm[1] /= (double)nn; vcm[2] /= (double)nn; }
  }
  const double rand1 = 2.0 * p.Pi * draw_uniform(p.seed, STREAM_COLLIDE_U, epoch, 3 + 2 * (uint64_t)c);
  const double rand2 = -1.0 + (2.0 * draw_uniform(p.seed, STREAM_COLLIDE_U, epoch, 4 + 2 * (uint64_t)c));
  double dvv = 0.0;
  for (int q = 0; q < n; ++q) {
    float4 v = f.vel[nth(q)];
    double A0 = (double)v.x - vcm[0], A1 = (double)v.y - vcm[1], A2 = (double)v.z - vcm[2];
    dvv += (p.mass * (A0 * A0 + A1 * A1 + A2 * A2));
  }
  for (int q = 0; q < nmem; ++q) {
    int i = (int)(m.vkey[v0 + q] & 0xffffffffu);
    double A0 = m.vx[i] - vcm[0], A1 = m.vy[i] - vcm[1], A2 = m.vz[i] - vcm[2];
    dvv += (p.pmass * (A0 * A0 + A1 * A1 + A2 * A2));
  }
  if (has_para) {
    double A0 = sc->paraV[0] - vcm[0], A1 = sc->paraV[1] - vcm[1], A2 = sc->paraV[2] - vcm[2];
    dvv += (p.PRmass * (A0 * A0 + A1 * A1 + A2 * A2));
  }
  double ThE = 1.0;
  if ((nc > 0) && (dvv != 0)) ThE = sqrt(3.0 * ((double)nc - 1.0) * p.Theta / (dvv));
  double P[7];
  P[0] = vcm[0]; P[1] = vcm[1]; P[2] = vcm[2];
  P[3] = sqrt(1.0 - (rand2 * rand2)) * cos(rand1);
  P[4] = sqrt(1.0 - (rand2 * rand2)) * sin(rand1);
  P[5] = rand2;
  P[6] = ThE;
  float* out = cl.parf + c * 8;
  for (int q = 0; q < 7; ++q) out[q] = (float)P[q];
  // vertices and parasite: rotated in double (CollisionDynmem / Dynpara)
  for (int q = 0; q < nmem; ++q) {
    int i = (int)(m.vkey[v0 + q] & 0xffffffffu);
    double v[3] = {m.vx[i], m.vy[i], m.vz[i]};
    double unit[3] = {P[3], P[4], P[5]}, dv[3], dvp[3], dvn[3], dvpn[3];
    for (int e = 0; e < 3; ++e) dv[e] = v[e] - P[e];
    double xxx = dv[0] * unit[0] + dv[1] * unit[1] + dv[2] * unit[2];
    for (int e = 0; e < 3; ++e) { dvp[e] = xxx * unit[e]; dvn[e] = dv[e] - dvp[e]; }
    cp(dvn, unit, dvpn);
    for (int e = 0; e < 3; ++e) v[e] = P[e] + ThE * (p.cosalpha * dvn[e] + p.sinalpha * dvpn[e] + dvp[e]);
    m.vx[i] = v[0]; m.vy[i] = v[1]; m.vz[i] = v[2];
  }
  if (has_para) {
    MemScalars* scw = m.sc;
    double v[3] = {scw->paraV[0], scw->paraV[1], scw->paraV[2]};
    double unit[3] = {P[3], P[4], P[5]}, dv[3], dvp[3], dvn[3], dvpn[3];
    for (int e = 0; e < 3; ++e) dv[e] = v[e] - P[e];
    double xxx = dv[0] * unit[0] + dv[1] * unit[1] + dv[2] * unit[2];
    for (int e = 0; e < 3; ++e) { dvp[e] = xxx * unit[e]; dvn[e] = dv[e] - dvp[e]; }
    cp(dvn, unit, dvpn);
    for (int e = 0; e < 3; ++e) scw->paraV[e] = P[e] + ThE * (p.cosalpha * dvn[e] + p.sinalpha * dvpn[e] + dvp[e]);
  }
}

// rotation of the solvent in float (CollisionDyn, Src/solfuncs.cpp:700-736)
__global__ void __launch_bounds__(256) k_rotate_f(SolventF f, const float* __restrict__ parf, float cosalpha,
                                                  float sinalpha) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= f.n) return;
  const float4* P4 = reinterpret_cast<const float4*>(parf + (int64_t)f.pid[i] * 8);
  float4 a = __ldg(P4), b = __ldg(P4 + 1);   // vcm xyz, ux | uy uz ThE -
  float4 v = f.vel[i];
  float ux = a.w, uy = b.x, uz = b.y, s = b.z;
  float dx = v.x - a.x, dy = v.y - a.y, dz = v.z - a.z;
  float xx = dx * ux + dy * uy + dz * uz;
  float px = xx * ux, py = xx * uy, pz = xx * uz;
  float nx = dx - px, ny = dy - py, nz = dz - pz;
  float cx = (ny * uz) - (uy * nz), cy = (nz * ux) - (uz * nx), cz = (nx * uy) - (ux * ny);
  v.x = a.x + s * (cosalpha * nx + sinalpha * cx + px);
  v.y = a.y + s * (cosalpha * ny + sinalpha * cy + py);
  v.z = a.z + s * (cosalpha * nz + sinalpha * cz + pz);
  f.vel[i] = v;
}

void launch_collide_f(const DevParams& p, SolventF& f, Solvent& s, Cells& c, Membrane& m, uint64_t epoch,
                      cudaStream_t st) {
  cudaMemsetAsync(c.cnt, 0, sizeof(int) * c.n, st);
  cudaMemsetAsync(c.ncm, 0, sizeof(int) * c.n, st);
  launch_vbin(p, m, c, epoch, st);
  if (f.n) k_count_f<<<nbf(f.n, 256), 256, 0, st>>>(p, f, c.cnt, s.key, s.slot, epoch);
  launch_ghost_flags(p, c, m, st);
  launch_scan3(c.cnt, c.wrank, c.mrank, c.start, c.wrank, c.mrank, c.totals, c.n, c.scan_part, st);
  cudaMemcpyAsync(c.start + c.n, c.totals + 0, sizeof(int), cudaMemcpyDeviceToDevice, st);
  if (f.n) k_perm_f<<<nbf(f.n, 256), 256, 0, st>>>(s.key, s.slot, c.start, f.n, s.perm);
  std::swap(f.pid, s.key);  // pid = cell of this collision, in place
  k_cells_f<<<nbf(c.n, 128), 128, 0, st>>>(p, f, s.perm, c, m, epoch);
  if (f.n) k_rotate_f<<<nbf(f.n, 256), 256, 0, st>>>(f, c.parf, (float)p.cosalpha, (float)p.sinalpha);
  if (f.n && (++s.ncoll % kResortEvery) == 0) {
    k_gather_f<<<nbf(f.n, 256), 256, 0, st>>>(f, s.perm);
    std::swap(f.pos, f.pos2); std::swap(f.vel, f.vel2); std::swap(f.pid, f.pid2);
  }
}

// ---- streaming ------------------------------------------------------------------
// free flight, walls and wrap in float (maincode.cpp:516-560); particles in
// cells with triangles are queued for the double-precision kernel
__global__ void __launch_bounds__(256) k_stream_f(DevParams p, SolventF f, const int* __restrict__ lstart,
                                                  int* queue, int* qn) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= f.n) return;
  const float Lx = (float)p.Lx, Ly = (float)p.Ly, Lz = (float)p.Lz, dt = (float)p.dtmd;
  float4 q = f.pos[i], v = f.vel[i];
  int fx = (int)floorf(bbound(q.x, Lx));
  int fy = (int)floorf(bbound(q.y, Ly));
  int fz = (int)floorf(q.z + 1.0f);
  int pid = cell_of(p, fx, fy, fz);
  if (__ldg(lstart + pid + 1) > __ldg(lstart + pid)) {
    unsigned mk = __activemask();
    int leader = __ffs(mk) - 1, lane = threadIdx.x & 31;
    int base = 0;
    if (lane == leader) base = atomicAdd(qn, __popc(mk));
    base = __shfl_sync(mk, base, leader);
    queue[base + __popc(mk & ((1u << lane) - 1))] = (int)i;
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
  f.pos[i] = make_float4(X, Y, Z, q.w);
}

// near the membrane: promote to double and run the FP64 warp kernel logic
__global__ void __launch_bounds__(256) k_stream_heavy_f(DevParams p, SolventF f, const int* __restrict__ lstart,
                                                        const int* __restrict__ lidx, Snap sn,
                                                        const TriPre* __restrict__ pre, const int* queue,
                                                        const int* qn) {
  const int lane = threadIdx.x & 31;
  const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int nq = *qn;
  for (int64_t q = w; q < nq; q += nw) {
    const int64_t i = queue[q];
    float4 q4 = f.pos[i], v4 = f.vel[i];
    double X = q4.x, Y = q4.y, Z = q4.z, VX = v4.x, VY = v4.y, VZ = v4.z;
    const int indio = __float_as_int(q4.w);
    int fx = (int)floor(bbound(X, p.Lx));
    int fy = (int)floor(bbound(Y, p.Ly));
    int fz = (int)floor(Z + 1.0);
    int pid = cell_of(p, fx, fy, fz);
    const int l0 = lstart[pid], l1 = lstart[pid + 1];
    double fulldt = 0.0;
    stream_heavy_walk(p, sn, pre, lidx, l0, l1, lane, indio, X, Y, Z, VX, VY, VZ, fulldt);
    if (lane == 0) {
      finish_stream(p, fulldt, X, Y, Z, VX, VY, VZ);
      f.pos[i] = make_float4((float)X, (float)Y, (float)Z, q4.w);
      f.vel[i] = make_float4((float)VX, (float)VY, (float)VZ, v4.w);
    }
  }
}

void fast_stream_f(const DevParams& p, SolventF& f, const Cells& c, FastBufs& fb, int buf, cudaStream_t st) {
  cudaMemsetAsync(fb.qn, 0, sizeof(int), st);
  if (f.n) {
    k_stream_f<<<nbf(f.n, 256), 256, 0, st>>>(p, f, c.lstart, fb.queue, fb.qn);
    k_stream_heavy_f<<<148 * 4, 256, 0, st>>>(p, f, c.lstart, c.lidx, fb.snap[buf], fb.pre[buf], fb.queue, fb.qn);
  }
}

}  // namespace irbc
