// fast.cu -- the production step: streaming that hands particles in cells
// with triangles to the near-membrane kernel, and the membrane update as
// wide per-vertex / per-item kernels plus one-CTA ordered reductions (Sarea /
// Volume, the parasite sum, bond_dynamics) that run on a side stream beside
// the solvent kernels.
//
// Results equal the one-kernel-per-phase path (kernels.cu) bit for bit.
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cooperative_groups.h>
#include "fast.h"
#include "fp32.h"

namespace irbc {

static inline unsigned nb(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

#define UXm(v) (m.x[v] + m.ix[v] * p.Lx)
#define UYm(v) (m.y[v] + m.iy[v] * p.Ly)

// ======================================================== triangle prep ===
// For the streaming step: each triangle's corners at t (A1,B1,C1, no image
// shift) and at t+dtmd, and the normals X = (B1-A1)x(C1-A1), Xdt likewise,
// as reflectionFed computes them (Src/solfuncs.cpp:457-509).  Also a copy of
// the vertex positions and velocities the streaming kernels read, so the
// membrane may move on while they run.
__device__ void tri_prep_one(const DevParams& p, const Membrane& m, int j, const double* vx, const double* vy,
                             const double* vz, TriPre* out) {
  int p1 = m.t1[j], p2 = m.t2[j], p3 = m.t3[j];
  const double rstep = 0.0, dtmd = p.dtmd, Lx = p.Lx, Ly = p.Ly;
  const int z0 = 0;
  double v1x = (m.x[p1] + z0 * Lx) + vx[p1] * rstep, v1y = (m.y[p1] + z0 * Ly) + vy[p1] * rstep,
         v1z = m.z[p1] + vz[p1] * rstep;
  double v2x = (m.x[p2] + z0 * Lx) + vx[p2] * rstep, v2y = (m.y[p2] + z0 * Ly) + vy[p2] * rstep,
         v2z = m.z[p2] + vz[p2] * rstep;
  double v3x = (m.x[p3] + z0 * Lx) + vx[p3] * rstep, v3y = (m.y[p3] + z0 * Ly) + vy[p3] * rstep,
         v3z = m.z[p3] + vz[p3] * rstep;
  double w1x = v1x + vx[p1] * (dtmd - rstep), w1y = v1y + vy[p1] * (dtmd - rstep), w1z = v1z + vz[p1] * (dtmd - rstep);
  double w2x = v2x + vx[p2] * (dtmd - rstep), w2y = v2y + vy[p2] * (dtmd - rstep), w2z = v2z + vz[p2] * (dtmd - rstep);
  double w3x = v3x + vx[p3] * (dtmd - rstep), w3y = v3y + vy[p3] * (dtmd - rstep), w3z = v3z + vz[p3] * (dtmd - rstep);
  double t0[3], t1v[3], X[3], Xdt[3];
  t0[0] = v2x - v1x; t0[1] = v2y - v1y; t0[2] = v2z - v1z;
  t1v[0] = v3x - v1x; t1v[1] = v3y - v1y; t1v[2] = v3z - v1z;
  cp(t0, t1v, X);
  t0[0] = w2x - w1x; t0[1] = w2y - w1y; t0[2] = w2z - w1z;
  t1v[0] = w3x - w1x; t1v[1] = w3y - w1y; t1v[2] = w3z - w1z;
  cp(t0, t1v, Xdt);
  TriPre q;
  q.X[0] = X[0]; q.X[1] = X[1]; q.X[2] = X[2];
  q.Xdt[0] = Xdt[0]; q.Xdt[1] = Xdt[1]; q.Xdt[2] = Xdt[2];
  q.A1[0] = v1x; q.A1[1] = v1y; q.A1[2] = v1z;
  q.A2[0] = w1x; q.A2[1] = w1y; q.A2[2] = w1z;
  out[j] = q;
}

// ================================================================ stream =====
// reflectionFed's per-triangle test and hit, reading the vertex snapshot.
// Returns true if the triangle was hit (state updated).  `q` holds the
// triangle's precomputed normals, used when the particle is outside the
// periodic stencil bands (3a from each side wall), where reflectionFed
// applies no shift.
__device__ __forceinline__ bool tri_visit(const DevParams& p, const Snap& sn, const TriPre& q, int jj,
                                          double& X_, double& Y_, double& Z_, double& VX, double& VY, double& VZ,
                                          int indio, double& fulldt, bool use_pre) {
  const double rstep = 0.0, dtmd = p.dtmd, a = p.a, Lx = p.Lx, Ly = p.Ly;
  int flg = 0;
  const double solvx = X_ + 0 * Lx, solvy = Y_ + 0 * Ly, solvz = Z_;
  double bt, bdt;
  double v1x, v1y, v1z, v2x, v2y, v2z, v3x, v3y, v3z;
  int p1, p2, p3;
  if (use_pre) {
    double PSt0 = solvx - q.A1[0], PSt1 = solvy - q.A1[1], PSt2 = solvz - q.A1[2];
    double PD0 = (solvx + VX * (dtmd - rstep)) - q.A2[0];
    double PD1 = (solvy + VY * (dtmd - rstep)) - q.A2[1];
    double PD2 = (solvz + VZ * (dtmd - rstep)) - q.A2[2];
    bt = q.X[0] * PSt0 + q.X[1] * PSt1 + q.X[2] * PSt2;
    bdt = q.Xdt[0] * PD0 + q.Xdt[1] * PD1 + q.Xdt[2] * PD2;
    if ((indio == 1) && (bt < 0)) flg = 1;
    if ((indio == 0) && (bt > 0)) flg = 1;
    if (!((bt * bdt <= 0) && (flg == 0))) return false;
    // the corners are read only for a crossing candidate
    p1 = sn.t1[jj]; p2 = sn.t2[jj]; p3 = sn.t3[jj];
    v1x = q.A1[0]; v1y = q.A1[1]; v1z = q.A1[2];
    v2x = (sn.x[p2] + 0 * Lx) + sn.vx[p2] * rstep; v2y = (sn.y[p2] + 0 * Ly) + sn.vy[p2] * rstep;
    v2z = sn.z[p2] + sn.vz[p2] * rstep;
    v3x = (sn.x[p3] + 0 * Lx) + sn.vx[p3] * rstep; v3y = (sn.y[p3] + 0 * Ly) + sn.vy[p3] * rstep;
    v3z = sn.z[p3] + sn.vz[p3] * rstep;
  } else {
    p1 = sn.t1[jj]; p2 = sn.t2[jj]; p3 = sn.t3[jj];
    v1x = (sn.x[p1] + 0 * Lx) + sn.vx[p1] * rstep; v1y = (sn.y[p1] + 0 * Ly) + sn.vy[p1] * rstep;
    v1z = sn.z[p1] + sn.vz[p1] * rstep;
    v2x = (sn.x[p2] + 0 * Lx) + sn.vx[p2] * rstep; v2y = (sn.y[p2] + 0 * Ly) + sn.vy[p2] * rstep;
    v2z = sn.z[p2] + sn.vz[p2] * rstep;
    v3x = (sn.x[p3] + 0 * Lx) + sn.vx[p3] * rstep; v3y = (sn.y[p3] + 0 * Ly) + sn.vy[p3] * rstep;
    v3z = sn.z[p3] + sn.vz[p3] * rstep;
    double rstencilx = Lx - (3.0 * a), lstencilx = 3.0 * a, rstencily = Ly - (3.0 * a), lstencily = 3.0 * a;
    if (solvx < lstencilx) {
      v1x -= (v1x > rstencilx) ? Lx : 0; v2x -= (v2x > rstencilx) ? Lx : 0; v3x -= (v3x > rstencilx) ? Lx : 0;
    } else if (solvx > rstencilx) {
      v1x += (v1x < lstencilx) ? Lx : 0; v2x += (v2x < lstencilx) ? Lx : 0; v3x += (v3x < lstencilx) ? Lx : 0;
    }
    if (solvy < lstencily) {
      v1y -= (v1y > rstencily) ? Ly : 0; v2y -= (v2y > rstencily) ? Ly : 0; v3y -= (v3y > rstencily) ? Ly : 0;
    } else if (solvy > rstencily) {
      v1y += (v1y < lstencily) ? Ly : 0; v2y += (v2y < lstencily) ? Ly : 0; v3y += (v3y < lstencily) ? Ly : 0;
    }
    double w1x = v1x + sn.vx[p1] * (dtmd - rstep), w1y = v1y + sn.vy[p1] * (dtmd - rstep), w1z = v1z + sn.vz[p1] * (dtmd - rstep);
    double w2x = v2x + sn.vx[p2] * (dtmd - rstep), w2y = v2y + sn.vy[p2] * (dtmd - rstep), w2z = v2z + sn.vz[p2] * (dtmd - rstep);
    double w3x = v3x + sn.vx[p3] * (dtmd - rstep), w3y = v3y + sn.vy[p3] * (dtmd - rstep), w3z = v3z + sn.vz[p3] * (dtmd - rstep);
    double X[3], Xdt[3], t0[3], t1v[3];
    t0[0] = v2x - v1x; t0[1] = v2y - v1y; t0[2] = v2z - v1z;
    t1v[0] = v3x - v1x; t1v[1] = v3y - v1y; t1v[2] = v3z - v1z;
    cp(t0, t1v, X);
    t0[0] = w2x - w1x; t0[1] = w2y - w1y; t0[2] = w2z - w1z;
    t1v[0] = w3x - w1x; t1v[1] = w3y - w1y; t1v[2] = w3z - w1z;
    cp(t0, t1v, Xdt);
    double PSt0 = solvx - v1x, PSt1 = solvy - v1y, PSt2 = solvz - v1z;
    double PD0 = (solvx + VX * (dtmd - rstep)) - w1x;
    double PD1 = (solvy + VY * (dtmd - rstep)) - w1y;
    double PD2 = (solvz + VZ * (dtmd - rstep)) - w1z;
    bt = X[0] * PSt0 + X[1] * PSt1 + X[2] * PSt2;
    bdt = Xdt[0] * PD0 + Xdt[1] * PD1 + Xdt[2] * PD2;
    if ((indio == 1) && (bt < 0)) flg = 1;
    if ((indio == 0) && (bt > 0)) flg = 1;
    if (!((bt * bdt <= 0) && (flg == 0))) return false;
  }
  // crossing candidate: contact time from the cubic, barycentric test (:526-594)
  const double mvx1 = sn.vx[p1], mvy1 = sn.vy[p1], mvz1 = sn.vz[p1];
  const double mvx2 = sn.vx[p2], mvy2 = sn.vy[p2], mvz2 = sn.vz[p2];
  const double mvx3 = sn.vx[p3], mvy3 = sn.vy[p3], mvz3 = sn.vz[p3];
  double a10[3], a20[3], d1[3], d2[3], a1v[3], a2v[3], b1[3], b2[3], b3[3], d11[3], d22[3];
  a10[0] = v2x - v1x; a10[1] = v2y - v1y; a10[2] = v2z - v1z;
  a20[0] = v3x - v1x; a20[1] = v3y - v1y; a20[2] = v3z - v1z;
  d1[0] = mvx2 - mvx1; d1[1] = mvy2 - mvy1; d1[2] = mvz2 - mvz1;
  d2[0] = mvx3 - mvx1; d2[1] = mvy3 - mvy1; d2[2] = mvz3 - mvz1;
  a1v[0] = solvx - v1x; a1v[1] = solvy - v1y; a1v[2] = solvz - v1z;
  a2v[0] = VX - mvx1; a2v[1] = VY - mvy1; a2v[2] = VZ - mvz1;
  cp(a10, a20, b1);
  cp(a10, d2, d11);
  cp(d1, a20, d22);
  cp(d1, d2, b3);
  for (int k = 0; k < 3; ++k) b2[k] = d11[k] + d22[k];
  double a2b3 = a2v[0] * b3[0] + a2v[1] * b3[1] + a2v[2] * b3[2];
  double a1b3 = a1v[0] * b3[0] + a1v[1] * b3[1] + a1v[2] * b3[2];
  double a2b2 = a2v[0] * b2[0] + a2v[1] * b2[1] + a2v[2] * b2[2];
  double a1b2 = a1v[0] * b2[0] + a1v[1] * b2[1] + a1v[2] * b2[2];
  double a2b1 = a2v[0] * b1[0] + a2v[1] * b1[1] + a2v[2] * b1[2];
  double a1b1 = a1v[0] * b1[0] + a1v[1] * b1[1] + a1v[2] * b1[2];
  double tt = solve_p3_tt((a1b3 + a2b2) / a2b3, (a1b2 + a2b1) / a2b3, a1b1 / a2b3, dtmd);
  double PS2[3], pd[3];
  PS2[0] = (solvx + VX * tt) - (v1x + mvx1 * tt);
  PS2[1] = (solvy + VY * tt) - (v1y + mvy1 * tt);
  PS2[2] = (solvz + VZ * tt) - (v1z + mvz1 * tt);
  pd[0] = (solvx + VX * tt); pd[1] = (solvy + VY * tt); pd[2] = (solvz + VZ * tt);
  a10[0] = (v2x + mvx2 * tt) - (v1x + mvx1 * tt);
  a10[1] = (v2y + mvy2 * tt) - (v1y + mvy1 * tt);
  a10[2] = (v2z + mvz2 * tt) - (v1z + mvz1 * tt);
  a20[0] = (v3x + mvx3 * tt) - (v1x + mvx1 * tt);
  a20[1] = (v3y + mvy3 * tt) - (v1y + mvy1 * tt);
  a20[2] = (v3z + mvz3 * tt) - (v1z + mvz1 * tt);
  double pa1 = PS2[0] * a10[0] + PS2[1] * a10[1] + PS2[2] * a10[2];
  double pa2 = PS2[0] * a20[0] + PS2[1] * a20[1] + PS2[2] * a20[2];
  double a1a2 = a10[0] * a20[0] + a10[1] * a20[1] + a10[2] * a20[2];
  double a12 = a10[0] * a10[0] + a10[1] * a10[1] + a10[2] * a10[2];
  double a22 = a20[0] * a20[0] + a20[1] * a20[1] + a20[2] * a20[2];
  double den = (a12 * a22) - (a1a2 * a1a2);
  double eta = ((pa1 * a22) - (pa2 * a1a2)) / den;
  double zeta = ((pa2 * a12) - (pa1 * a1a2)) / den;
  if ((eta >= 0) && (zeta >= 0) && (eta + zeta <= 1) && (tt < (dtmd - rstep))) {
    fulldt += tt;
    double vd0 = (1.0 - eta - zeta) * mvx1 + eta * mvx2 + zeta * mvx3;
    double vd1 = (1.0 - eta - zeta) * mvy1 + eta * mvy2 + zeta * mvy3;
    double vd2 = (1.0 - eta - zeta) * mvz1 + eta * mvz2 + zeta * mvz3;
    VX = 2.0 * vd0 - VX; VY = 2.0 * vd1 - VY; VZ = 2.0 * vd2 - VZ;
    X_ = pd[0]; Y_ = pd[1]; Z_ = pd[2];
    return true;
  }
  return false;
}

// free flight, walls and wrap after the membrane (maincode.cpp:516-560)
__device__ __forceinline__ void finish_stream(const DevParams& p, double fullts, double& X, double& Y, double& Z,
                                              double& VX, double& VY, double& VZ) {
  const double dtmd = p.dtmd;
  X += VX * (dtmd - fullts);
  Y += VY * (dtmd - fullts);
  Z += VZ * (dtmd - fullts);
  const double ul = p.Lz, ll = 0;
  if (Z > ul || Z < ll) {
    double A[3], B[3];
    const double wall = Z > ul ? ul : ll;
    A[0] = X - VX * (dtmd - fullts); A[1] = Y - VY * (dtmd - fullts); A[2] = Z - VZ * (dtmd - fullts);
    double sp = (wall - A[2]) / (Z - A[2]);
    B[0] = A[0] + sp * (X - A[0]); B[1] = A[1] + sp * (Y - A[1]); B[2] = A[2] + sp * (Z - A[2]);
    double dist = sqrt(((B[0] - A[0]) * (B[0] - A[0])) + ((B[1] - A[1]) * (B[1] - A[1])) + ((B[2] - A[2]) * (B[2] - A[2])));
    double dtt = dist / sqrt((VX * VX) + (VY * VY) + (VZ * VZ));
    if (Z > ul) { VX = p.wallspeed; VY = 0; VZ = 0; }
    else { VX *= -1.0; VY *= -1.0; VZ *= -1.0; }
    X = B[0] + VX * ((dtmd - fullts) - dtt);
    Y = B[1] + VY * ((dtmd - fullts) - dtt);
    Z = B[2] + VZ * ((dtmd - fullts) - dtt);
  }
  X = bbound(X, p.Lx);
  Y = bbound(Y, p.Ly);
}

__device__ __forceinline__ bool in_stencil(const DevParams& p, double x, double y) {
  return (x < 3.0 * p.a) || (x > p.Lx - (3.0 * p.a)) || (y < 3.0 * p.a) || (y > p.Ly - (3.0 * p.a));
}

// hand-off of a particle whose cell has triangles: into the bucket of its
// cell (rank lrank among the listed cells) when the list fits the staging
// capacity hcap of the near-membrane kernels and the bucket has room, else
// onto the overflow queue
__device__ __forceinline__ void hand_off(const int* __restrict__ lrank, int pid, int len, int hcap, int i,
                                         int* bcnt, int* bucket, int* queue, int* qn) {
  if (len <= hcap) {
    const int a = lrank[pid];
    const int slot = atomicAdd(bcnt + a, 1);
    if (slot < kBucket) { bucket[(int64_t)a * kBucket + slot] = i; return; }
  }
  const int q = atomicAdd(qn, 1);
  queue[q] = i;
}

// one thread per particle: free flight, walls and wrap for particles whose
// cell has no triangles; the others are handed to the near-membrane kernels
// and left untouched here
__global__ void __launch_bounds__(256) k_stream_fast(DevParams p, Solvent s, const int* __restrict__ lstart,
                                                     const int* __restrict__ lrank, int* bcnt, int* bucket,
                                                     int* queue, int* qn, int hcap) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= s.n) return;
  double X = s.x[i], Y = s.y[i], Z = s.z[i];
  const SolVel r = s.v[i];
  double VX = r.vx, VY = r.vy, VZ = r.vz;
  const double VX0 = VX, VY0 = VY, VZ0 = VZ;
  int fx = (int)floor(bbound(X, p.Lx));
  int fy = (int)floor(bbound(Y, p.Ly));
  int fz = (int)floor(Z + 1.0);
  int pid = cell_of(p, fx, fy, fz);
  const int l0 = __ldg(lstart + pid), l1 = __ldg(lstart + pid + 1);
  if (l1 > l0) {
    hand_off(lrank, pid, l1 - l0, hcap, (int)i, bcnt, bucket, queue, qn);
    return;
  }
  finish_stream(p, 0.0, X, Y, Z, VX, VY, VZ);
  raise_health(p, solvent_bad(p, X, Y, Z, VX, VY, VZ), HEALTH_SOLVENT);
  s.x[i] = X; s.y[i] = Y; s.z[i] = Z;
  if (VX != VX0 || VY != VY0 || VZ != VZ0 || VX0 != VX0) { s.v[i].vx = VX; s.v[i].vy = VY; s.v[i].vz = VZ; }
}

// reflectionFed's crossing test on the precomputed normals (the use_pre
// case of tri_visit, :461-517): whether the full test can hit
__device__ __forceinline__ bool tri_crossing(const DevParams& p, const TriPre& q, double X, double Y, double Z,
                                             double VX, double VY, double VZ, int indio) {
  const double rstep = 0.0, dtmd = p.dtmd;
  double PSt0 = X - q.A1[0], PSt1 = Y - q.A1[1], PSt2 = Z - q.A1[2];
  double PD0 = (X + VX * (dtmd - rstep)) - q.A2[0];
  double PD1 = (Y + VY * (dtmd - rstep)) - q.A2[1];
  double PD2 = (Z + VZ * (dtmd - rstep)) - q.A2[2];
  const double bt = q.X[0] * PSt0 + q.X[1] * PSt1 + q.X[2] * PSt2;
  const double bdt = q.Xdt[0] * PD0 + q.Xdt[1] * PD1 + q.Xdt[2] * PD2;
  int flg = 0;
  if ((indio == 1) && (bt < 0)) flg = 1;
  if ((indio == 0) && (bt > 0)) flg = 1;
  return (bt * bdt <= 0) && (flg == 0);
}

// The triangle walk of reflectionFed for one particle, by a whole warp:
// lanes run the crossing test on 32 list entries at a time, and every
// crossing candidate gets the full test (contact time, barycentric test) on
// its own lane, all from the same particle state.  The reference's loop
// changes the state only at a hit, so up to and including the first hit of
// the 32 these are exactly its tests: the lowest hit is applied and the walk
// resumes after it with the updated state -- the same sequence of states as
// the sequential loop.  Inside the periodic stencil bands every entry gets
// the full test (its shifted corners are not precomputed).  tri(e) gives the
// TriPre of list entry e, jj(e) its triangle.
// The walk covers entries [cur, end) and leaves cur at or past end, so a
// list can be walked in consecutive pieces with the same result.
template <class TriAt, class IdAt>
__device__ __forceinline__ void heavy_walk(const DevParams& p, const Snap& sn, TriAt tri, IdAt jj, int end, int lane,
                                           int indio, double& X, double& Y, double& Z, double& VX, double& VY,
                                           double& VZ, double& fulldt, int& cur) {
  const int len = end;
  while (cur < len) {
    const bool pre = !in_stencil(p, X, Y);
    const int e = cur + lane;
    bool cand = false;
    if (e < len) cand = pre ? tri_crossing(p, tri(e), X, Y, Z, VX, VY, VZ, indio) : true;
    double x = X, y = Y, z = Z, vx = VX, vy = VY, vz = VZ, fd = 0.0;
    const bool hit = cand && tri_visit(p, sn, tri(e), jj(e), x, y, z, vx, vy, vz, indio, fd, pre);
    const unsigned hb = __ballot_sync(0xffffffffu, hit);
    if (hb == 0u) {
      cur += 32;
      continue;
    }
    const int src = __ffs(hb) - 1;
    X = __shfl_sync(0xffffffffu, x, src);
    Y = __shfl_sync(0xffffffffu, y, src);
    Z = __shfl_sync(0xffffffffu, z, src);
    VX = __shfl_sync(0xffffffffu, vx, src);
    VY = __shfl_sync(0xffffffffu, vy, src);
    VZ = __shfl_sync(0xffffffffu, vz, src);
    fulldt += __shfl_sync(0xffffffffu, fd, src);
    cur += src + 1;
  }
}

// particle state in double for the walk, and its write-back
template <bool F32>
struct HeavyIO {
  __device__ static void load(const Solvent& s, const SolventF& f, int64_t i, double st[6], int& indio) {
    if constexpr (F32) {
      const float4 q4 = f.pos[i], v4 = f.vel[i];
      st[0] = q4.x; st[1] = q4.y; st[2] = q4.z; st[3] = v4.x; st[4] = v4.y; st[5] = v4.z;
      indio = __float_as_int(q4.w);
    } else {
      const SolVel r = s.v[i];
      st[0] = s.x[i]; st[1] = s.y[i]; st[2] = s.z[i]; st[3] = r.vx; st[4] = r.vy; st[5] = r.vz;
      indio = s.indio[i];
    }
  }
  __device__ static void store(Solvent& s, SolventF& f, int64_t i, const double st[6], const double st0[6]) {
    if constexpr (F32) {
      f.pos[i] = make_float4((float)st[0], (float)st[1], (float)st[2], f.pos[i].w);
      f.vel[i] = make_float4((float)st[3], (float)st[4], (float)st[5], f.vel[i].w);
    } else {
      s.x[i] = st[0]; s.y[i] = st[1]; s.z[i] = st[2];
      if (st[3] != st0[3] || st[4] != st0[4] || st[5] != st0[5] || st0[3] != st0[3]) {
        s.v[i].vx = st[3]; s.v[i].vy = st[4]; s.v[i].vz = st[5];
      }
    }
  }
};

template <bool F32, class TriAt, class IdAt>
__device__ __forceinline__ void heavy_particle_from(const DevParams& p, Solvent& s, SolventF& f, const Snap& sn,
                                                    int64_t i, int lane, int len, TriAt tri, IdAt ids,
                                                    const double st_in[6], int indio) {
  double st[6], st0[6];
  for (int k = 0; k < 6; ++k) st0[k] = st[k] = st_in[k];
  double fulldt = 0.0;
  int cur = 0;
  heavy_walk(p, sn, tri, ids, len, lane, indio, st[0], st[1], st[2], st[3], st[4], st[5], fulldt, cur);
  if (lane == 0) {
    finish_stream(p, fulldt, st[0], st[1], st[2], st[3], st[4], st[5]);
    raise_health(p, solvent_bad(p, st[0], st[1], st[2], st[3], st[4], st[5]), HEALTH_SOLVENT);
    HeavyIO<F32>::store(s, f, i, st, st0);
  }
}
template <bool F32, class TriAt, class IdAt>
__device__ __forceinline__ void heavy_particle(const DevParams& p, Solvent& s, SolventF& f, const Snap& sn,
                                               int64_t i, int lane, int len, TriAt tri, IdAt ids) {
  double st[6];
  int indio;
  HeavyIO<F32>::load(s, f, i, st, indio);
  heavy_particle_from<F32>(p, s, f, sn, i, lane, len, tri, ids, st, indio);
}

// The overflow queue (particles of full buckets, lists longer than the
// staging): warp gw of tw walks queued particles gw, gw + tw, ..., a warp per
// particle, reading its cell's list from global memory.
template <bool F32>
__device__ __forceinline__ void overflow_walk(const DevParams& p, Solvent& s, SolventF& f,
                                              const int* __restrict__ lstart, const int* __restrict__ lidx,
                                              const Snap& sn, const TriPre* __restrict__ pre, const int* queue,
                                              const int* qn, int64_t gw, int64_t tw, int lane) {
  const int nq = *qn;
  for (int64_t q = gw; q < nq; q += tw) {
    const int64_t i = queue[q];
    double X, Y, Z;
    if constexpr (F32) { const float4 q4 = f.pos[i]; X = q4.x; Y = q4.y; Z = q4.z; }
    else { X = s.x[i]; Y = s.y[i]; Z = s.z[i]; }
    int fx = (int)floor(bbound(X, p.Lx));
    int fy = (int)floor(bbound(Y, p.Ly));
    int fz = (int)floor(Z + 1.0);
    const int pid = cell_of(p, fx, fy, fz);
    const int* L = lidx + lstart[pid];
    heavy_particle<F32>(p, s, f, sn, i, lane, lstart[pid + 1] - lstart[pid],
                        [&](int e) -> const TriPre& { return pre[L[e]]; }, [&](int e) { return L[e]; });
  }
}

// one TriPre record through the read-only path as six 16-byte loads (the
// records are 96 bytes from a 256-byte aligned base)
__device__ __forceinline__ TriPre ldg_tri(const TriPre* __restrict__ q) {
  const double2* r = reinterpret_cast<const double2*>(q);
  const double2 a = __ldg(r), b = __ldg(r + 1), c = __ldg(r + 2), d = __ldg(r + 3), e = __ldg(r + 4),
                g = __ldg(r + 5);
  TriPre t;
  t.X[0] = a.x; t.X[1] = a.y; t.X[2] = b.x;
  t.Xdt[0] = b.y; t.Xdt[1] = c.x; t.Xdt[2] = c.y;
  t.A1[0] = d.x; t.A1[1] = d.y; t.A1[2] = e.x;
  t.A2[0] = e.y; t.A2[1] = g.x; t.A2[2] = g.y;
  return t;
}

// Short lists (hcap <= kShortList; small meshes: a few dozen entries and
// about ten particles per listed cell), in two launches.
//
// (1) stream_cells_warp: one warp per listed cell.  The warp stages the list
// in its shared memory kLanePiece entries at a time, every lane loading
// different entries, the records as twelve arrays (lanes that read
// consecutive entries hit distinct banks).  The n particles of the cell's
// bucket get G = 32 / n lanes each; lane g of a particle runs the crossing
// test on the precomputed normals for entries g, g + G, ...  reflectionFed's
// loop (Src/solfuncs.cpp:400-598) changes a particle's state only at a hit,
// and a hit needs the crossing test to pass first, so a particle with no
// candidate in its whole list leaves the loop unchanged: its owner lane
// (g = 0) finishes it here (walls, wrap, write-back).  A particle with a
// candidate, or one inside the periodic stencil bands (where every entry
// gets the full test), is appended to the overflow queue instead: few
// particles (about 0.6% of those in listed cells, plus the bands), and the
// full test that only they need keeps its registers out of this kernel,
// which would otherwise hold it to a quarter of the warps an SM can run.
//
// (2) the queue launch (overflow_walk): a warp per queued particle walks
// its cell's list with the reference's loop from the start -- the bulk
// kernel's overflow (full buckets) and the particles appended by (1).
struct LaneStage {
  double tp[12][kLanePiece];
};

__device__ __forceinline__ TriPre staged_tri(const LaneStage& S, int e) {
  TriPre q;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    q.X[k] = S.tp[k][e];
    q.Xdt[k] = S.tp[3 + k][e];
    q.A1[k] = S.tp[6 + k][e];
    q.A2[k] = S.tp[9 + k][e];
  }
  return q;
}

// listed cell a (a < bcap; ranks from nact on have nothing to do)
template <bool F32>
__device__ __forceinline__ void stream_cells_warp(const DevParams& p, Solvent& s, SolventF& f,
                                                  const int* __restrict__ lidx, const int2* __restrict__ arng,
                                                  int* bcnt, const int* __restrict__ bucket,
                                                  const TriPre* __restrict__ pre, int* queue, int* qn,
                                                  const int* __restrict__ nactp, int a, LaneStage& S) {
  const int lane = threadIdx.x & 31;
  // The loads that depend only on a go out together with the count of
  // listed cells: every rank below the bucket capacity has a bucket, a
  // count and a range slot (stale beyond nact, and unused there), so the
  // chain of dependent loads before the tests is count, state, list, records
  const int2 rg = __ldg(arng + a);
  const int slot = bucket[(int64_t)a * kBucket + lane];
  int nraw = 0;
  if (lane == 0) nraw = bcnt[a];
  const int nact = *nactp;
  if (a >= nact) return;
  // lane 0 resets the count for the next step (an empty bucket stays 0)
  if (lane == 0 && nraw) bcnt[a] = 0;
  const int n = min(__shfl_sync(0xffffffffu, nraw, 0), kBucket);
  if (n == 0) return;
  const int l0 = rg.x, len = rg.y;
  const int G = 32 / n;                     // lanes per particle
  const int k = lane / G, g = lane - k * G;  // this lane's particle and its place among the particle's lanes
  const bool act = k < n, own = act && g == 0;
  const int64_t i = __shfl_sync(0xffffffffu, slot, k);  // the particle in bucket slot k
  double st[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0}, st0[6];
  int indio = 0;
  if (act) HeavyIO<F32>::load(s, f, i, st, indio);
  for (int u = 0; u < 6; ++u) st0[u] = st[u];
  const bool band = act && in_stencil(p, st[0], st[1]);
  bool cand = false;
  for (int c0 = 0; c0 < len; c0 += kLanePiece) {
    const int m = min(len - c0, kLanePiece);
    if (c0 > 0) __syncwarp();  // every lane is done with the previous piece
    int jj[kLanePiece / 32];
#pragma unroll
    for (int u = 0; u < kLanePiece / 32; ++u) {
      const int e = lane + 32 * u;
      jj[u] = e < m ? __ldg(lidx + l0 + c0 + e) : 0;
    }
#pragma unroll
    for (int u = 0; u < kLanePiece / 32; ++u) {
      const int e = lane + 32 * u;
      if (e < m) {
        const TriPre t = ldg_tri(pre + jj[u]);
#pragma unroll
        for (int r = 0; r < 3; ++r) {
          S.tp[r][e] = t.X[r];
          S.tp[3 + r][e] = t.Xdt[r];
          S.tp[6 + r][e] = t.A1[r];
          S.tp[9 + r][e] = t.A2[r];
        }
      }
    }
    __syncwarp();
    if (act && !band && !cand) {
      for (int e = g; e < m; e += G) {
        if (tri_crossing(p, staged_tri(S, e), st[0], st[1], st[2], st[3], st[4], st[5], indio)) {
          cand = true;
          break;
        }
      }
    }
  }
  // the particle's lanes are bits k*G .. k*G+G-1
  const unsigned to_queue = __ballot_sync(0xffffffffu, act && (band || cand));
  const unsigned mine = G == 32 ? 0xffffffffu : (((1u << G) - 1u) << (k * G));
  if (own) {
    if (to_queue & mine) {
      queue[atomicAdd(qn, 1)] = (int)i;
    } else {
      finish_stream(p, 0.0, st[0], st[1], st[2], st[3], st[4], st[5]);
      raise_health(p, solvent_bad(p, st[0], st[1], st[2], st[3], st[4], st[5]), HEALTH_SOLVENT);
      HeavyIO<F32>::store(s, f, i, st, st0);
    }
  }
}

// Particles in cells with long lists (reflectionFed, Src/solfuncs.cpp:400-598,
// then the walls and wrap).  Block a < nact takes the bucket of listed cell
// a: its list's TriPre records and triangle indices are staged in shared
// memory once, then each warp walks one particle of the bucket at a time
// from there (the walk's per-entry test reads no global memory).  The
// bucket count is reset for the next step.  Blocks from nact on walk the
// overflow queue (full buckets, lists longer than kHeavyList), a warp per
// particle, from global memory.  nact is read on the device and the grid
// is sized by the bucket capacity, so a captured launch stays valid across
// list updates.
// block `bid` of `nblk`
template <bool F32>
__device__ __forceinline__ void stream_cells_block(const DevParams& p, Solvent& s, SolventF& f,
                                                   const int* __restrict__ lstart, const int* __restrict__ lidx,
                                                   const int* __restrict__ acell, int* bcnt,
                                                   const int* __restrict__ bucket, const Snap& sn,
                                                   const TriPre* __restrict__ pre, const int* queue, const int* qn,
                                                   const int* __restrict__ nactp, const int* __restrict__ border,
                                                   int bid, int nblk, int cap) {
  extern __shared__ double sh[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int nact = *nactp;
  if (bid >= nact) {
    overflow_walk<F32>(p, s, f, lstart, lidx, sn, pre, queue, qn, (int64_t)(bid - nact) * nw + w,
                       (int64_t)(nblk - nact) * nw, lane);
    return;
  }
  // Every thread reads the cell's bucket count and list bounds itself, so
  // that the particle loads below go out beside the list's staging instead
  // of after it.  The count is reset once everyone has read it (after the
  // first barrier); an empty bucket stays 0 and needs no reset.
  const int a = border[bid];
  const int n = min(bcnt[a], kBucket);
  if (n == 0) return;
  const int c = acell[a];
  // this warp's particles are q = w, w + nw, ... (n <= kBucket = 32): lane
  // j loads the j-th one's state and keeps its walk state (position,
  // velocity, time spent, list cursor) between the pieces of the list
  const int mine = n > w ? (n - w + nw - 1) / nw : 0;
  int64_t pi = -1;
  double pst[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0}, p0[6], pfd = 0.0;
  int pind = 0, pcur = 0;
  if (lane < mine) {
    pi = bucket[(int64_t)a * kBucket + w + lane * nw];
    HeavyIO<F32>::load(s, f, pi, pst, pind);
  }
  for (int k = 0; k < 6; ++k) p0[k] = pst[k];
  const int l0 = lstart[c], len = lstart[c + 1] - l0;  // len <= hcap (hand_off)
  // the list in pieces of `cap` entries (the shared staging): every
  // particle walks a piece before the next is staged, so each walk still
  // visits the entries in list order
  TriPre* st = reinterpret_cast<TriPre*>(sh);
  int* sj = reinterpret_cast<int*>(st + cap);
  for (int c0 = 0; c0 == 0 || c0 < len; c0 += cap) {
    const int c1 = min(len, c0 + cap);
    if (c0 > 0) __syncthreads();  // the previous piece's walks are done
    for (int e = threadIdx.x; e < c1 - c0; e += blockDim.x) {
      const int jj = lidx[l0 + c0 + e];
      sj[e] = jj;
      st[e] = pre[jj];
    }
    __syncthreads();
    if (c0 == 0 && threadIdx.x == 0) bcnt[a] = 0;
    for (int k = 0; k < mine; ++k) {
      int cur = __shfl_sync(0xffffffffu, pcur, k);
      if (cur >= c1) continue;  // warp-uniform
      double X = __shfl_sync(0xffffffffu, pst[0], k), Y = __shfl_sync(0xffffffffu, pst[1], k);
      double Z = __shfl_sync(0xffffffffu, pst[2], k), VX = __shfl_sync(0xffffffffu, pst[3], k);
      double VY = __shfl_sync(0xffffffffu, pst[4], k), VZ = __shfl_sync(0xffffffffu, pst[5], k);
      double fd = __shfl_sync(0xffffffffu, pfd, k);
      const int indio = __shfl_sync(0xffffffffu, pind, k);
      heavy_walk(p, sn, [&](int e) -> const TriPre& { return st[e - c0]; }, [&](int e) { return sj[e - c0]; }, c1,
                 lane, indio, X, Y, Z, VX, VY, VZ, fd, cur);
      if (lane == k) {
        pst[0] = X; pst[1] = Y; pst[2] = Z; pst[3] = VX; pst[4] = VY; pst[5] = VZ;
        pfd = fd;
        pcur = cur;
      }
    }
  }
  // each lane ends its own particle: walls, wrap, health, write-back
  if (lane < mine) {
    finish_stream(p, pfd, pst[0], pst[1], pst[2], pst[3], pst[4], pst[5]);
    raise_health(p, solvent_bad(p, pst[0], pst[1], pst[2], pst[3], pst[4], pst[5]), HEALTH_SOLVENT);
    HeavyIO<F32>::store(s, f, pi, pst, p0);
  }
}
template <bool F32>
__global__ void __launch_bounds__(256) k_stream_cells(DevParams p, Solvent s, SolventF f,
                                                      const int* __restrict__ lstart, const int* __restrict__ lidx,
                                                      const int* __restrict__ acell, int* bcnt,
                                                      const int* __restrict__ bucket, Snap sn,
                                                      const TriPre* __restrict__ pre, const int* queue,
                                                      const int* qn, const int* __restrict__ nactp,
                                                      const int* __restrict__ border, int cap) {
  stream_cells_block<F32>(p, s, f, lstart, lidx, acell, bcnt, bucket, sn, pre, queue, qn, nactp, border,
                          (int)blockIdx.x, (int)gridDim.x, cap);
}

// the short-list form: kShortWarps warps per block, one listed cell each
// (ranks below the bucket capacity bcap)
template <bool F32>
__global__ void __launch_bounds__(32 * kShortWarps, kShortMinBlocks)
    k_stream_cells_short(DevParams p, Solvent s, SolventF f, const int* __restrict__ lidx,
                         const int2* __restrict__ arng, int* bcnt, const int* __restrict__ bucket,
                         const TriPre* __restrict__ pre, int* queue, int* qn, const int* __restrict__ nactp,
                         int bcap) {
  __shared__ LaneStage stage[kShortWarps];
  const int w = (int)(threadIdx.x >> 5);
  const int a = (int)blockIdx.x * kShortWarps + w;
  if (a >= bcap) return;
  stream_cells_warp<F32>(p, s, f, lidx, arng, bcnt, bucket, pre, queue, qn, nactp, a, stage[w]);
}

// the queue after the short-list form: a warp per queued particle
template <bool F32>
__global__ void __launch_bounds__(256, 2) k_stream_queue(DevParams p, Solvent s, SolventF f,
                                                      const int* __restrict__ lstart, const int* __restrict__ lidx,
                                                      Snap sn, const TriPre* __restrict__ pre, const int* queue,
                                                      const int* qn) {
  const int64_t tw = (int64_t)gridDim.x * (blockDim.x >> 5);
  const int64_t gw = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  overflow_walk<F32>(p, s, f, lstart, lidx, sn, pre, queue, qn, gw, tw, threadIdx.x & 31);
}

// ========================================================= membrane step ====
// force terms of every edge (WLC + POW), triangle (local/global area and
// volume) and bending dihedral, stored per term in slots so the per-vertex
// gather can add them in the reference's order (Src/memfuncs.cpp:233-427)
// item t of [edges | triangles | dihedrals]: its force terms into the slots
__device__ void force_item(const DevParams& p, const Membrane& m, double* __restrict__ slot, int t) {
  const MemScalars* sc = m.sc;
  if (t < p.ne) {
    int i = t;
    int l1 = m.e1[i], l2 = m.e2[i];
    double l0 = m.l0[i];
    double A[3];
    A[0] = UXm(l1) - UXm(l2); A[1] = UYm(l1) - UYm(l2); A[2] = m.z[l1] - m.z[l2];
    double aa = sqrt(A[0] * A[0] + A[1] * A[1] + A[2] * A[2]);
    A[0] /= aa; A[1] /= aa; A[2] /= aa;
    double xx = aa / (2.5 * l0);
    double xxx = 1.0 / (4.0 * (1.0 - xx) * (1.0 - xx));
    const double kp = m.kappap[i];
    double* S = slot + (int64_t)12 * i;
    for (int k = 0; k < 3; ++k) {
      S[0 + k] = (-1.0 / (p.elap)) * (xxx - 0.25 + xx) * A[k];
      S[3 + k] = kp * A[k] / (aa * aa);
      S[6 + k] = (1.0 / (p.elap)) * (xxx - 0.25 + xx) * A[k];
      S[9 + k] = -kp * A[k] / (aa * aa);
    }
    return;
  }
  t -= p.ne;
  if (t < p.nt) {
    int i = t;
    int l1 = m.t1[i], l2 = m.t2[i], l3 = m.t3[i];
    const double Sarea = sc->Sarea, Volume = sc->Volume;
    double beta = -p.kappasa * (Sarea - p.Sarea0) / p.Sarea0;
    double betav = -p.kappav * (Volume - p.Volume0) / (p.Volume0);
    double A0[3], B0[3], e0[3];
    A0[0] = UXm(l2) - UXm(l1); A0[1] = UYm(l2) - UYm(l1); A0[2] = m.z[l2] - m.z[l1];
    B0[0] = UXm(l3) - UXm(l1); B0[1] = UYm(l3) - UYm(l1); B0[2] = m.z[l3] - m.z[l1];
    cp(A0, B0, e0);
    double area = 0.5 * sqrt(e0[0] * e0[0] + e0[1] * e0[1] + e0[2] * e0[2]);
    double alpha = beta / (4.0 * area);
    double alphad = -p.kappad * (area - m.tarea[i]) / (4.0 * m.tarea[i] * area);
    double A21[3], A13[3], A32[3], eta[3], C[3], B[3];
    A21[0] = UXm(l2) - UXm(l1); A21[1] = UYm(l2) - UYm(l1); A21[2] = m.z[l2] - m.z[l1];
    A13[0] = UXm(l1) - UXm(l3); A13[1] = UYm(l1) - UYm(l3); A13[2] = m.z[l1] - m.z[l3];
    A32[0] = UXm(l3) - UXm(l2); A32[1] = UYm(l3) - UYm(l2); A32[2] = m.z[l3] - m.z[l2];
    cp(A13, A21, eta);
    B[0] = (UXm(l1) + UXm(l2) + UXm(l3)) / 3.0;
    B[1] = (UYm(l1) + UYm(l2) + UYm(l3)) / 3.0;
    B[2] = (m.z[l1] + m.z[l2] + m.z[l3]) / 3.0;
    double* S = slot + (int64_t)12 * p.ne + (int64_t)27 * i;
    const double* sides[3] = {A32, A13, A21};
    for (int c = 0; c < 3; ++c) {
      cp(eta, sides[c], C);
      for (int k = 0; k < 3; ++k) { S[6 * c + k] = alpha * C[k]; S[6 * c + 3 + k] = alphad * C[k]; }
      cp(B, sides[c], C);
      for (int k = 0; k < 3; ++k) S[18 + 3 * c + k] = betav * ((eta[k] / 3.0) + C[k]) / 6.0;
    }
    return;
  }
  t -= p.nt;
  if (t < p.ne) {
    int i = t;
    int l2, l3;
    if (m.iedge[i] == -1) { l3 = m.e1[i]; l2 = m.e2[i]; } else { l2 = m.e1[i]; l3 = m.e2[i]; }
    int l1 = m.es1[i], l4 = m.es2[i];
    double a21[3], a31[3], a24[3], a34[3], a32[3], t1[3], t2[3], eta[3], zeta[3], C[3], D[3], E[3], F[3];
    a21[0] = UXm(l2) - UXm(l1); a21[1] = UYm(l2) - UYm(l1); a21[2] = m.z[l2] - m.z[l1];
    a31[0] = UXm(l3) - UXm(l1); a31[1] = UYm(l3) - UYm(l1); a31[2] = m.z[l3] - m.z[l1];
    a24[0] = UXm(l2) - UXm(l4); a24[1] = UYm(l2) - UYm(l4); a24[2] = m.z[l2] - m.z[l4];
    a34[0] = UXm(l3) - UXm(l4); a34[1] = UYm(l3) - UYm(l4); a34[2] = m.z[l3] - m.z[l4];
    a32[0] = UXm(l3) - UXm(l2); a32[1] = UYm(l3) - UYm(l2); a32[2] = m.z[l3] - m.z[l2];
    t1[0] = (UXm(l1) + UXm(l2) + UXm(l3)) / 3.0;
    t1[1] = (UYm(l1) + UYm(l2) + UYm(l3)) / 3.0;
    t1[2] = (m.z[l1] + m.z[l2] + m.z[l3]) / 3.0;
    t2[0] = (UXm(l4) + UXm(l2) + UXm(l3)) / 3.0;
    t2[1] = (UYm(l4) + UYm(l2) + UYm(l3)) / 3.0;
    t2[2] = (m.z[l4] + m.z[l2] + m.z[l3]) / 3.0;
    cp(a21, a31, eta);
    cp(a34, a24, zeta);
    double etam = sqrt(eta[0] * eta[0] + eta[1] * eta[1] + eta[2] * eta[2]);
    double zetam = sqrt(zeta[0] * zeta[0] + zeta[1] * zeta[1] + zeta[2] * zeta[2]);
    double costh = (eta[0] * zeta[0] + eta[1] * zeta[1] + eta[2] * zeta[2]) / (etam * zetam);
    if (costh > 1.0) costh = 1.0;
    if (costh < -1.0) costh = -1.0;
    if (costh == 1.0) costh -= 0.0005;
    if (costh == -1.0) costh += 0.0005;
    double sinth = sqrt(1.0 - costh * costh);
    double tt0 = t1[0] - t2[0];
    double tt1 = t1[1] - t2[1];
    double factor = (((eta[0] - zeta[0]) * tt0) + ((eta[1] - zeta[1]) * tt1) + ((eta[2] - zeta[2]) * (t1[2] - t2[2])));
    double fact = (factor >= 0.0) ? 1.0 : -1.0;
    sinth = fact * sinth;
    double betab = p.kappab * (sinth * p.cth0 - costh * p.sth0) / sinth;
    double b11 = -(betab * costh) / (etam * etam);
    double b22 = -(betab * costh) / (zetam * zetam);
    double b12 = betab / (etam * zetam);
    double* S = slot + (int64_t)12 * p.ne + (int64_t)27 * p.nt + (int64_t)12 * i;
    cp(eta, a32, C);
    cp(zeta, a32, D);
    for (int k = 0; k < 3; ++k) { S[k] = b11 * C[k] + b12 * D[k]; S[3 + k] = -b12 * C[k] - b22 * D[k]; }
    cp(eta, a31, C); cp(zeta, a31, D); cp(eta, a34, E); cp(zeta, a34, F);
    for (int k = 0; k < 3; ++k) S[6 + k] = -b11 * C[k] + b12 * (E[k] - D[k]) + b22 * F[k];
    cp(eta, a21, C); cp(zeta, a21, D); cp(eta, a24, E); cp(zeta, a24, F);
    for (int k = 0; k < 3; ++k) S[9 + k] = b11 * C[k] + b12 * (-E[k] + D[k]) - b22 * F[k];
  }
}

__device__ __forceinline__ bool wca_f(const DevParams& p, const Membrane& m, const MemScalars* sc, int i, double X[3]) {
  double cutoff = p.paraR, epsilon = 0.1, sigma = 0.890898718 * cutoff;
  double A[3];
  A[0] = (sc->para[0] + sc->paradx * p.Lx) - (m.x[i] + m.ix[i] * p.Lx);
  A[1] = (sc->para[1] + sc->parady * p.Ly) - (m.y[i] + m.iy[i] * p.Ly);
  A[2] = sc->para[2] - m.z[i];
  double aa = A[0] * A[0] + A[1] * A[1] + A[2] * A[2];
  if (aa <= cutoff * cutoff) {
    double ex = (sigma * sigma * sigma * sigma * sigma * sigma) / (aa * aa * aa);
    X[0] = (24.0 * epsilon / aa) * ((2.0 * ex * ex) - ex) * A[0];
    X[1] = (24.0 * epsilon / aa) * ((2.0 * ex * ex) - ex) * A[1];
    X[2] = (24.0 * epsilon / aa) * ((2.0 * ex * ex) - ex) * A[2];
    return true;
  }
  return false;
}

// ligand (xl, yl) on the ligand list of a cell (maincode.cpp:138-154)
__device__ __forceinline__ bool in_liglist_f(const DevParams& p, int cell, double xl, double yl) {
  int k = cell % p.nz, j = (cell / p.nz) % p.ny, i = cell / (p.nz * p.ny);
  double zmax = -1.0 + (double)k * p.a + p.a;
  if (!(zmax <= 2.0)) return false;
  double xmin = (double)i * p.a, xmax = (double)i * p.a + p.a;
  double ymin = (double)j * p.a, ymax = (double)j * p.a + p.a;
  double A0 = fabs(((xmin + xmax) * 0.5) - xl);
  double A1 = fabs(((ymin + ymax) * 0.5) - yl);
  A0 -= p.Lx * round(A0 / p.Lx);
  A1 -= p.Ly * round(A1 / p.Ly);
  return (A0 < 1.5) && (A1 < 1.5);
}

constexpr int kTailT = 1024, kTailDraws = 4096, kWcaList = 512;

// ================================================= membrane step, wide form ===
// The membrane step spread over many SMs: per-vertex and per-triangle work in wide kernels, the ordered
// reductions (Sarea, Volume, the parasite sum, bond_dynamics) in one CTA
// reading shared memory.

// drift + image counters (maincode.cpp:566-574) and parasite drift (:576-598)
__device__ __forceinline__ void m_drift_item(const DevParams& p, Membrane& m, int i) {
  if (i < p.nv) {
    double x = m.x[i], y = m.y[i], z = m.z[i];
    x += (m.vx[i] * p.dtmd);
    y += (m.vy[i] * p.dtmd);
    z += (m.vz[i] * p.dtmd);
    if (x > p.Lx) { x -= p.Lx; m.ix[i] += 1; }
    if (x < 0) { x += p.Lx; m.ix[i] -= 1; }
    if (y > p.Ly) { y -= p.Ly; m.iy[i] += 1; }
    if (y < 0) { y += p.Ly; m.iy[i] -= 1; }
    m.x[i] = x; m.y[i] = y; m.z[i] = z;
  }
  if (i == 0) {
    MemScalars* sc = m.sc;
    for (int k = 0; k < 3; ++k)
      sc->para[k] += (sc->paraV[k] * p.dtmd) + (sc->paraft[k] * p.dtmd * p.dtmd / (2.0 * p.PRmass));
    if (sc->para[0] > p.Lx) { sc->para[0] -= p.Lx; sc->paradx += 1; }
    else if (sc->para[0] < 0) { sc->para[0] += p.Lx; sc->paradx -= 1; }
    if (sc->para[1] > p.Ly) { sc->para[1] -= p.Ly; sc->parady += 1; }
    else if (sc->para[1] < 0) { sc->para[1] += p.Ly; sc->parady -= 1; }
  }
}
__global__ void k_m_drift(DevParams p, Membrane m) { m_drift_item(p, m, blockIdx.x * blockDim.x + threadIdx.x); }

// Areatri / Voltri terms per triangle (Src/memfuncs.cpp:124-157)
__device__ __forceinline__ void m_av_item(const DevParams& p, Membrane& m, int i) {
  if (i >= p.nt) return;
  int l1 = m.t1[i], l2 = m.t2[i], l3 = m.t3[i];
  double A[3], B[3], eta[3], Cn[3];
  A[0] = UXm(l2) - UXm(l1); A[1] = UYm(l2) - UYm(l1); A[2] = m.z[l2] - m.z[l1];
  B[0] = UXm(l3) - UXm(l1); B[1] = UYm(l3) - UYm(l1); B[2] = m.z[l3] - m.z[l1];
  cp(A, B, eta);
  m.area[i] = 0.5 * sqrt(eta[0] * eta[0] + eta[1] * eta[1] + eta[2] * eta[2]);
  Cn[0] = (UXm(l1) + UXm(l2) + UXm(l3)) / 3.0;
  Cn[1] = (UYm(l1) + UYm(l2) + UYm(l3)) / 3.0;
  Cn[2] = (m.z[l1] + m.z[l2] + m.z[l3]) / 3.0;
  m.vol[i] = (1.0 / 6.0) * ((eta[0] * Cn[0]) + (eta[1] * Cn[1]) + (eta[2] * Cn[2]));
}
__global__ void k_m_av(DevParams p, Membrane m) { m_av_item(p, m, blockIdx.x * blockDim.x + threadIdx.x); }

// TotalVA's sums, left to right in triangle order, from shared memory
constexpr int kSumSmemT = 12288;

// a[0] + a[1] + ... + a[n-1] added left to right (the reference's one-thread
// order); the terms come in 16 at a time with 128-bit shared-memory loads so
// that only the chain of additions is serial
__device__ __forceinline__ double ordered_sum(const double* a, int n) {
  double t = 0.0;
  int i = 0;
  if ((reinterpret_cast<uintptr_t>(a) & 15) == 0) {
    const double2* a2 = reinterpret_cast<const double2*>(a);
    const int n16 = n & ~15;
    // the next 16 terms are loaded while the current 16 are added (32
    // registers of terms: the kernels calling this run <= 256 threads)
    double2 cur[8], nxt[8];
    if (n16 > 0) {
#pragma unroll
      for (int k = 0; k < 8; ++k) cur[k] = a2[k];
    }
    for (; i < n16; i += 16) {
      const bool more = i + 16 < n16;
      if (more) {
#pragma unroll
        for (int k = 0; k < 8; ++k) nxt[k] = a2[((i + 16) >> 1) + k];
      }
#pragma unroll
      for (int k = 0; k < 8; ++k) { t += cur[k].x; t += cur[k].y; }
      if (more) {
#pragma unroll
        for (int k = 0; k < 8; ++k) cur[k] = nxt[k];
      }
    }
  }
  for (; i < n; ++i) t += a[i];
  return t;
}

// Sum of a[0..n) by one warp in a fixed order: lane l adds its contiguous
// run left to right, then the 32 partial sums meet in a butterfly; lane 0's
// value is the result (the same for every launch and launch layout)
__device__ __forceinline__ double warp_tree_sum(const double* a, int n, int lane) {
  const int c = (n + 31) / 32;
  const int b = min(lane * c, n), e = min(b + c, n);
  double t = 0.0;
  for (int i = b; i < e; ++i) t += a[i];
  for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  return __shfl_sync(0xffffffffu, t, 0);
}

// Sarea and Volume (TotalVA, Src/memfuncs.cpp:161-190) from the triangle
// terms a[] and v[], by warp 0 (Sarea) and warp 1 (Volume) of the block:
// the threads t < 64 call it.  Left to right in one thread, the
// reference's order; or, with p.tree_sums, as a fixed warp tree.
__device__ __forceinline__ void area_volume_sums(const DevParams& p, const Membrane& m, const double* a,
                                                 const double* v, int t) {
  const int lane = t & 31;
  const double* src = t < 32 ? a : v;
  double* out = t < 32 ? &m.sc->Sarea : &m.sc->Volume;
  if (p.tree_sums) {
    const double r = warp_tree_sum(src, p.nt, lane);
    if (lane == 0) *out = r;
  } else if (lane == 0) {
    *out = ordered_sum(src, p.nt);
  }
}

__global__ void __launch_bounds__(256) k_m_sum(DevParams p, Membrane m) {
  extern __shared__ double sh[];
  const bool staged = p.nt <= kSumSmemT;
  if (staged) {
    for (int i = threadIdx.x; i < p.nt; i += blockDim.x) { sh[i] = m.area[i]; sh[p.nt + i] = m.vol[i]; }
    __syncthreads();
  }
  const double* a = staged ? sh : m.area;
  const double* v = staged ? sh + p.nt : m.vol;
  if (threadIdx.x < 64) area_volume_sums(p, m, a, v, threadIdx.x);
}

// per vertex: bond preparation (maincode.cpp:668-723), the number of bond
// draws and the WCA flag for k_tail_b.  It reads positions (after the
// drift) and bond states only, so it runs beside the force terms; the
// second half-kick (:727-733) is applied by the force gather.
__device__ __forceinline__ void bond_prep_item(const DevParams& p, Membrane& m, int* __restrict__ vd,
                                            int* __restrict__ vw, double* __restrict__ vX, int ii) {
  if (ii >= p.nv) return;
  double A[3], B[3];
  int nd = 0;
  if (m.bondi[ii] == 1) {
    int p1modx = m.ix[ii], p1mody = m.iy[ii], jj = m.bondl[ii];
    A[0] = (m.x[ii] + p1modx * p.Lx) - (m.xlig[jj] + p1modx * p.Lx);
    A[1] = (m.y[ii] + p1mody * p.Ly) - (m.ylig[jj] + p1mody * p.Ly);
    A[2] = m.z[ii] - 0.0;
    double xx = sqrt(A[0] * A[0] + A[1] * A[1] + A[2] * A[2]);
    if (xx > p.el0) {
      B[0] = -p.ks * (xx - p.el0) * A[0] / xx;
      B[1] = -p.ks * (xx - p.el0) * A[1] / xx;
      B[2] = -p.ks * (xx - p.el0) * A[2] / xx;
    } else {
      B[0] = B[1] = B[2] = 0.0;
    }
    double bb = sqrt(B[0] * B[0] + B[1] * B[1] + B[2] * B[2]);
    double koff = p.offrate * exp(bb / p.FD);
    m.poff[ii] = 1.0 - exp(-koff * p.dtmd);
    nd = 1;
  } else if ((m.z[ii] < p.dthr) && (m.bondi[ii] == 0) && (m.knob[ii] == 1)) {
    const int pid = m.pid[ii];
    m.pon[ii] = 1.0 - exp(-p.onrate * p.dtmd);
    int n = 0;
    double* pd = m.pair_d + (int64_t)ii * kMaxPairs;
    int* pj = m.pair_j + (int64_t)ii * kMaxPairs;
    const int p1modx = m.ix[ii], p1mody = m.iy[ii];
    const double vx = m.x[ii], vy = m.y[ii];
    int gx0 = max((int)floor((vx - p.dthr) / 0.5) - 1, 0), gx1 = min((int)floor((vx + p.dthr) / 0.5) + 1, p.nligx - 1);
    int gy0 = max((int)floor((vy - p.dthr) / 0.5) - 1, 0), gy1 = min((int)floor((vy + p.dthr) / 0.5) + 1, p.nligy - 1);
    for (int gx = gx0; gx <= gx1; ++gx) {
      for (int gy = gy0; gy <= gy1; ++gy) {
        int j = gx * p.nligy + gy;
        double xl = m.xlig[j], yl = m.ylig[j];
        if (!in_liglist_f(p, pid, xl, yl)) continue;
        A[0] = (vx + p1modx * p.Lx) - (xl + p1modx * p.Lx);
        A[1] = (vy + p1mody * p.Ly) - (yl + p1mody * p.Ly);
        A[2] = m.z[ii] - 0.0;
        double aaa = (A[0] * A[0] + A[1] * A[1] + A[2] * A[2]);
        if (aaa <= p.dthr * p.dthr && n < kMaxPairs) {
          int r = n++;
          while (r > 0 && (pd[r - 1] > aaa || (pd[r - 1] == aaa && pj[r - 1] > j))) { pd[r] = pd[r - 1]; pj[r] = pj[r - 1]; --r; }
          pd[r] = aaa; pj[r] = j;
        }
      }
    }
    m.npair[ii] = n;
    nd = n;
  }
  double X[3];
  const bool in_wca = wca_f(p, m, m.sc, ii, X);
  vw[ii] = in_wca ? 1 : 0;
  if (in_wca) { vX[3 * ii] = X[0]; vX[3 * ii + 1] = X[1]; vX[3 * ii + 2] = X[2]; }
  vd[ii] = nd;
}
// Block 0: TotalVA's two ordered sums (as k_m_sum).  Blocks 1..: the edge
// and bending terms and the bond preparation, which do not depend on
// Sarea / Volume, so they overlap the sums.  The triangle terms follow in
// k_force_tri.
__device__ __forceinline__ void sum_edges_block(const DevParams& p, Membrane& m, double* __restrict__ slot,
                                                int do_sum, int* __restrict__ vd, int* __restrict__ vw,
                                                double* __restrict__ vX, int bid) {
  if (bid == 0) {
    if (!do_sum) return;
    extern __shared__ double sh[];
    const bool staged = p.nt <= kSumSmemT;
    if (staged) {
      for (int i = threadIdx.x; i < p.nt; i += blockDim.x) { sh[i] = m.area[i]; sh[p.nt + i] = m.vol[i]; }
      __syncthreads();
    }
    const double* a = staged ? sh : m.area;
    const double* v = staged ? sh + p.nt : m.vol;
    if (threadIdx.x < 64) area_volume_sums(p, m, a, v, threadIdx.x);
    return;
  }
  const int k = (bid - 1) * blockDim.x + threadIdx.x;  // 0 .. 2E + V
  if (k < p.ne) force_item(p, m, slot, k);
  else if (k < 2 * p.ne) force_item(p, m, slot, p.nt + k);  // dihedral k - E
  else bond_prep_item(p, m, vd, vw, vX, k - 2 * p.ne);
}
__global__ void __launch_bounds__(256) k_sum_edges(DevParams p, Membrane m, double* __restrict__ slot, int do_sum,
                                                    int* __restrict__ vd, int* __restrict__ vw,
                                                    double* __restrict__ vX) {
  sum_edges_block(p, m, slot, do_sum, vd, vw, vX, (int)blockIdx.x);
}
__global__ void k_force_tri(DevParams p, Membrane m, double* __restrict__ slot) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < p.nt) force_item(p, m, slot, p.ne + k);
}

// warp per vertex: lanes stage the vertex's force slots in shared memory,
// lanes 0-2 add them up component-wise in the reference's order, lane 0
// applies pfdt's -X first and the external forces after (maincode.cpp:603-665)
constexpr int kGW = 4, kGSlots = 64;
// vertex i by one warp; shw: kGSlots * 3 + 3 doubles of this warp's shared memory
__device__ __forceinline__ void gather_vertex(const DevParams& p, Membrane& m, const double* __restrict__ slot,
                                              const int* __restrict__ gstart, const int* __restrict__ gidx, int i,
                                              int lane, double* shw) {
  double* ffsw = shw + kGSlots * 3;
  const int q0 = gstart[i], q1 = gstart[i + 1];
  double acc = 0.0;
  for (int c0 = q0; c0 < q1; c0 += kGSlots) {
    const int nc = min(kGSlots, q1 - c0);
    for (int e = lane; e < nc * 3; e += 32) {
      const int q = e / 3, k = e - 3 * q;
      shw[e] = slot[3 * (int64_t)gidx[c0 + q] + k];
    }
    __syncwarp();
    if (lane < 3)
      for (int q = 0; q < nc; ++q) acc += shw[3 * q + lane];
    __syncwarp();
  }
  if (lane < 3) ffsw[lane] = acc;
  __syncwarp();
  if (lane != 0) return;
  const MemScalars* sc = m.sc;
  double f[3] = {m.fx[i], m.fy[i], m.fz[i]};
  double X[3];
  if (wca_f(p, m, sc, i, X)) { f[0] -= X[0]; f[1] -= X[1]; f[2] -= X[2]; }
  f[0] += ffsw[0]; f[1] += ffsw[1]; f[2] += ffsw[2];
  f[2] += -p.Fg / (double)p.nv;
  if (m.bondi[i] == 1) {
    int jj = m.bondl[i];
    double A[3];
    A[0] = m.x[i] - m.xlig[jj];
    A[1] = m.y[i] - m.ylig[jj];
    A[2] = m.z[i];
    A[0] -= p.Lx * round(A[0] / p.Lx);
    A[1] -= p.Ly * round(A[1] / p.Ly);
    double aa = sqrt(A[0] * A[0] + A[1] * A[1] + A[2] * A[2]);
    A[0] /= aa; A[1] /= aa; A[2] /= aa;
    if (aa > p.el0) {
      f[0] += -p.ks * (aa - p.el0) * A[0];
      f[1] += -p.ks * (aa - p.el0) * A[1];
      f[2] += -p.ks * (aa - p.el0) * A[2];
    }
  }
  double cc = m.z[i];
  if (cc < 0.5) f[2] += 300.0 * exp(-50.0 * cc);
  cc = p.Lz - m.z[i];
  if (cc < 0.5) f[2] -= 300.0 * exp(-50.0 * cc);
  m.fx[i] = f[0]; m.fy[i] = f[1]; m.fz[i] = f[2];
  // second half-kick (maincode.cpp:727-733)
  const double vx = m.vx[i] + (f[0] * p.dtmd / (2.0 * p.pmass));
  const double vy = m.vy[i] + (f[1] * p.dtmd / (2.0 * p.pmass));
  const double vz = m.vz[i] + (f[2] * p.dtmd / (2.0 * p.pmass));
  m.vx[i] = vx; m.vy[i] = vy; m.vz[i] = vz;
  const double chk = f[0] + f[1] + f[2] + vx + vy + vz;
  raise_health(p, !isfinite(chk), HEALTH_MEMBRANE);
}
__device__ __forceinline__ void gather_block(const DevParams& p, Membrane& m, const double* __restrict__ slot,
                                             const int* __restrict__ gstart, const int* __restrict__ gidx, int bid) {
  __shared__ double sh[kGW][kGSlots * 3 + 3];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int i = bid * kGW + w;
  if (i >= p.nv) return;
  gather_vertex(p, m, slot, gstart, gidx, i, lane, sh[w]);
}
__global__ void __launch_bounds__(32 * kGW) k_force_gather_w(DevParams p, Membrane m, const double* __restrict__ slot,
                                                           const int* __restrict__ gstart,
                                                           const int* __restrict__ gidx) {
  gather_block(p, m, slot, gstart, gidx, (int)blockIdx.x);

}


// One CTA: exclusive scans of the per-vertex draw counts and WCA flags (each
// thread owns a contiguous run of vertices, so order is kept), the bond
// draws marked as events in parallel and applied in draw order by one warp
// (bond_dynamics, maincode.cpp:16-54), and pfdt's parasite sum in vertex
// order with the parasite kick (Src/memfuncs.cpp:469-482, maincode.cpp:736-744).
struct TailSmem {
  double s_wx[kWcaList * 3];
  int s_d[kTailT], s_w[kTailT];
  int s_wlist[kWcaList];
  int s_evv[kTailDraws];
  short s_evr[kTailDraws];
  int s_tot[2];
};

// the whole block (at most kTailT threads); S in shared memory
__device__ void tail_b_block(const DevParams& p, Membrane& m, const int* __restrict__ vd, const int* __restrict__ vw,
                             const double* __restrict__ vX, uint64_t epoch, TailSmem& S) {
  int* s_d = S.s_d;
  int* s_w = S.s_w;
  int* s_wlist = S.s_wlist;
  double* s_wx = S.s_wx;
  int* s_evv = S.s_evv;
  short* s_evr = S.s_evr;
  int* s_tot = S.s_tot;
  const int T = blockDim.x, tid = threadIdx.x;
  MemScalars* sc = m.sc;
  const int chunk = (p.nv + T - 1) / T;
  const int v0 = min(tid * chunk, p.nv), v1 = min(v0 + chunk, p.nv);
  int nd = 0, nw = 0;
  for (int ii = v0; ii < v1; ++ii) { nd += vd[ii]; nw += vw[ii]; }
  s_d[tid] = nd; s_w[tid] = nw;
  __syncthreads();
  if (tid < 64) {
    int* arr = tid < 32 ? s_d : s_w;
    const int lane = tid & 31;
    int carry = 0;
    for (int base = 0; base < T; base += 32) {
      int x = arr[base + lane], v = x;
      for (int o = 1; o < 32; o <<= 1) { int y = __shfl_up_sync(0xffffffffu, v, o); if (lane >= o) v += y; }
      arr[base + lane] = carry + v - x;
      carry += __shfl_sync(0xffffffffu, v, 31);
    }
    if (lane == 0) s_tot[tid >> 5] = carry;
  }
  __syncthreads();
  const bool fits = s_tot[0] <= kTailDraws && s_tot[1] <= kWcaList;
  if (fits) {
    int od = s_d[tid], ow = s_w[tid];
    for (int ii = v0; ii < v1; ++ii) {
      const int n = vd[ii];
      if (n > 0) {
        if (m.bondi[ii] == 1) {
          double u = draw_uniform(p.seed, STREAM_BOND, epoch, (uint64_t)od);
          s_evv[od] = (m.poff[ii] > u) ? ii : -1;
          s_evr[od] = -1;
        } else {
          const double pon = m.pon[ii];
          for (int r = 0; r < n; ++r) {
            double u = draw_uniform(p.seed, STREAM_BOND, epoch, (uint64_t)(od + r));
            s_evv[od + r] = (pon > u) ? ii : -1;
            s_evr[od + r] = r;
          }
        }
        od += n;
      }
      if (vw[ii]) {
        s_wx[3 * ow] = vX[3 * ii]; s_wx[3 * ow + 1] = vX[3 * ii + 1]; s_wx[3 * ow + 2] = vX[3 * ii + 2];
        s_wlist[ow++] = ii;
      }
    }
  }
  __syncthreads();
  if (tid == 32) {
    double fx = 0, fy = 0, fz = 0;
    if (fits) {
      for (int q = 0; q < s_tot[1]; ++q) { fx += s_wx[3 * q]; fy += s_wx[3 * q + 1]; fz += s_wx[3 * q + 2]; }
    } else {
      for (int ii = 0; ii < p.nv; ++ii) {
        double X[3];
        if (wca_f(p, m, sc, ii, X)) { fx += X[0]; fy += X[1]; fz += X[2]; }
      }
    }
    sc->parafdt[0] += fx; sc->parafdt[1] += fy; sc->parafdt[2] += fz;
    for (int c = 0; c < 3; ++c) sc->paraV[c] += ((sc->paraft[c] + sc->parafdt[c]) * p.dtmd / (2.0 * p.PRmass));
    for (int c = 0; c < 3; ++c) { sc->paraft[c] = sc->parafdt[c]; sc->parafdt[c] = 0.0; }
  }
  if (fits && tid < 32) {
    const int ndt = s_tot[0];
    for (int k0 = 0; k0 < ndt; k0 += 32) {
      const int k = k0 + tid;
      unsigned ev = __ballot_sync(0xffffffffu, k < ndt && s_evv[k] >= 0);
      if (tid == 0) {
        while (ev) {
          const int b = __ffs(ev) - 1;
          ev &= ev - 1;
          const int ii = s_evv[k0 + b], r = s_evr[k0 + b];
          if (r < 0) {
            int jj = m.bondl[ii];
            m.bondi[ii] = 0; m.bondl[ii] = p.randno; m.ligi[jj] = 0;
          } else {
            int j = m.pair_j[(int64_t)ii * kMaxPairs + r];
            if (m.ligi[j] == 0) { m.ligi[j] = 1; m.bondi[ii] = 1; m.bondl[ii] = j; }
          }
        }
      }
    }
  } else if (!fits && tid == 0) {
    uint64_t k = 0;
    for (int ii = 0; ii < p.nv; ++ii) {
      if (m.bondi[ii] == 1) {
        double randoff = draw_uniform(p.seed, STREAM_BOND, epoch, k++);
        int jj = m.bondl[ii];
        if (m.poff[ii] > randoff) { m.bondi[ii] = 0; m.bondl[ii] = p.randno; m.ligi[jj] = 0; }
      } else if (vd[ii] > 0) {
        const int n = m.npair[ii];
        for (int r = 0; r < n; ++r) {
          int j = m.pair_j[(int64_t)ii * kMaxPairs + r];
          double pon = m.pon[ii];
          double randon = draw_uniform(p.seed, STREAM_BOND, epoch, k++);
          if ((pon > randon) && (m.ligi[j] == 0)) { m.ligi[j] = 1; m.bondi[ii] = 1; m.bondl[ii] = j; }
        }
      }
    }
  }
}
__global__ void __launch_bounds__(kTailT) k_tail_b(DevParams p, Membrane m, const int* __restrict__ vd,
                                                   const int* __restrict__ vw, const double* __restrict__ vX,
                                                   uint64_t eoff) {
  __shared__ TailSmem S;
  tail_b_block(p, m, vd, vw, vX, epoch_of(p, eoff), S);
}

// half-kick + snapshot + triangle prep as separate launches (after a
// collision, or at the first step)
__device__ __forceinline__ void kick_snap_item(const DevParams& p, Membrane& m, const Snap& sn, int i) {
  if (i >= p.nv) return;
  double vx = m.vx[i] + (m.fx[i] * p.dtmd / (2.0 * p.pmass));
  double vy = m.vy[i] + (m.fy[i] * p.dtmd / (2.0 * p.pmass));
  double vz = m.vz[i] + (m.fz[i] * p.dtmd / (2.0 * p.pmass));
  m.vx[i] = vx; m.vy[i] = vy; m.vz[i] = vz;
  m.fx[i] = 0.0; m.fy[i] = 0.0; m.fz[i] = 0.0;
  sn.x[i] = m.x[i]; sn.y[i] = m.y[i]; sn.z[i] = m.z[i];
  sn.vx[i] = vx; sn.vy[i] = vy; sn.vz[i] = vz;
}
__global__ void k_kick_snap(DevParams p, Membrane m, Snap sn) {
  kick_snap_item(p, m, sn, blockIdx.x * blockDim.x + threadIdx.x);
}
__global__ void k_tri_prep(DevParams p, Membrane m, TriPre* pre) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < p.nt) tri_prep_one(p, m, j, m.vx, m.vy, m.vz, pre);
}

__global__ void k_snap(DevParams p, Membrane m, Snap sn) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.nv) return;
  sn.x[i] = m.x[i]; sn.y[i] = m.y[i]; sn.z[i] = m.z[i];
  sn.vx[i] = m.vx[i]; sn.vy[i] = m.vy[i]; sn.vz[i] = m.vz[i];
}

// ================================================================ launch ======
// the membrane chain's kernels (the side stream's work): a captured graph
// gives them the side stream's high priority
constexpr int kBlockT = 512;      // threads of the one-block membrane kernels
constexpr int kBlockMaxV = 1024;  // meshes up to this many vertices use them
__global__ void __launch_bounds__(kBlockT) k_membrane_block(DevParams p, Membrane m, FastBufs f, uint64_t eoff);
__global__ void __launch_bounds__(kBlockT) k_kick_prep_block(DevParams p, Membrane m, Snap sn, TriPre* pre);
constexpr int kClusterCTAs = 8, kClusterT = 512;  // the cluster membrane kernel's blocks and threads
__global__ void __launch_bounds__(kClusterT)
    k_membrane_cluster(DevParams p, Membrane m, FastBufs f, uint64_t eoff, int next_kick, int next_buf);

bool is_membrane_kernel(const void* fn) {
  const void* k[] = {(const void*)k_m_drift, (const void*)k_m_av, (const void*)k_m_sum,
                     (const void*)k_sum_edges, (const void*)k_force_tri, (const void*)k_force_gather_w,
                     (const void*)k_tail_b, (const void*)k_kick_snap, (const void*)k_membrane_block,
                     (const void*)k_membrane_cluster,
                     (const void*)k_kick_prep_block,
                     (const void*)k_tri_prep, (const void*)k_snap};
  for (const void* q : k)
    if (q == fn) return true;
  return false;
}

__global__ void k_rank_lengths(Cells c, int nact, int* len, int2* rng) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= nact) return;
  const int cell = c.acell[a];
  const int l0 = c.lstart[cell];
  len[a] = c.lstart[cell + 1] - l0;
  rng[a] = make_int2(l0, c.lstart[cell + 1] - l0);
}
void launch_rank_lengths(const Cells& c, int* len, int2* rng, cudaStream_t st) {
  if (c.nact > 0) k_rank_lengths<<<nb(c.nact, 256), 256, 0, st>>>(c, c.nact, len, rng);
}

void fast_snap_prep(const DevParams& p, Membrane& m, FastBufs& f, int buf, cudaStream_t st) {
  k_snap<<<nb(p.nv, 128), 128, 0, st>>>(p, m, f.snap[buf]);
  k_tri_prep<<<nb(p.nt, 128), 128, 0, st>>>(p, m, f.pre[buf]);
}

// half-kick, snapshot and triangle prep of a small mesh in one block
__global__ void __launch_bounds__(kBlockT) k_kick_prep_block(DevParams p, Membrane m, Snap sn, TriPre* pre) {
  for (int i = threadIdx.x; i < p.nv; i += blockDim.x) kick_snap_item(p, m, sn, i);
  __syncthreads();
  for (int j = threadIdx.x; j < p.nt; j += blockDim.x) tri_prep_one(p, m, j, m.vx, m.vy, m.vz, pre);
}

int fast_kick_prep(const DevParams& p, Membrane& m, FastBufs& f, int buf, cudaStream_t st) {
  if (f.one_block) {
    k_kick_prep_block<<<1, kBlockT, 0, st>>>(p, m, f.snap[buf], f.pre[buf]);
    return 1;
  }
  k_kick_snap<<<nb(p.nv, 128), 128, 0, st>>>(p, m, f.snap[buf]);
  k_tri_prep<<<nb(p.nt, 128), 128, 0, st>>>(p, m, f.pre[buf]);
  return 2;
}

// returns the number of kernels it launched
template <bool F32>
static int launch_stream_cells(const DevParams& p, Solvent& s, SolventF& sf, const Cells& c, FastBufs& f, int buf,
                               cudaStream_t st) {
  // short lists (small simulations: many listed cells of a few dozen
  // entries, ~10 particles each): one warp per cell and one lane per
  // particle, no staging; long lists: eight warps share a cell's staging,
  // which holds a piece of the list at a time (stage_cap), so its size does
  // not grow with the longest list.
  if (short_lists(f.hcap)) {
    if (f.bcap > 0)
      k_stream_cells_short<F32><<<nb(f.bcap, kShortWarps), 32 * kShortWarps, 0, st>>>(
          p, s, sf, c.lidx, f.arng, f.bcnt, f.bucket, f.pre[buf], f.queue, f.qn, c.totals + 4, (int)f.bcap);
    k_stream_queue<F32><<<kQueueBlocks, 256, 0, st>>>(p, s, sf, c.lstart, c.lidx, f.snap[buf], f.pre[buf], f.queue,
                                                      f.qn);
    return f.bcap > 0 ? 2 : 1;
  }
  const int cap = stage_cap(f.hcap);
  k_stream_cells<F32><<<(unsigned)f.bcap + kOverflowBlocks, 256, stage_bytes(cap), st>>>(
      p, s, sf, c.lstart, c.lidx, c.acell, f.bcnt, f.bucket, f.snap[buf], f.pre[buf], f.queue, f.qn,
      c.totals + 4, f.border, cap);
  return 1;
}

int fast_stream(const DevParams& p, Solvent& s, const Cells& c, FastBufs& f, int buf, cudaStream_t st,
                cudaEvent_t ev0, cudaEvent_t ev1, cudaEvent_t snap) {
  cudaMemsetAsync(f.qn, 0, sizeof(int), st);
  if (s.n) {
    if (ev0) cudaEventRecord(ev0, st);
    k_stream_fast<<<nb(s.n, 256), 256, 0, st>>>(p, s, c.lstart, c.lrank, f.bcnt, f.bucket, f.queue, f.qn,
                                                 f.hcap);
    if (ev1) cudaEventRecord(ev1, st);
    if (snap) cudaStreamWaitEvent(st, snap, 0);
    SolventF none;
    return 1 + launch_stream_cells<false>(p, s, none, c, f, buf, st);
  }
  return 0;
}

// drift and the per-triangle TotalVA terms; with_sum also forms Sarea and
// Volume (otherwise fast_forces_tail does, beside the edge terms)
int fast_drift_va(const DevParams& p, Membrane& m, cudaStream_t st, bool with_sum) {
  k_m_drift<<<nb(p.nv, 128), 128, 0, st>>>(p, m);
  k_m_av<<<nb(p.nt, 128), 128, 0, st>>>(p, m);
  if (!with_sum) return 2;
  const size_t sm = p.nt <= kSumSmemT ? 2 * (size_t)p.nt * sizeof(double) : 0;
  k_m_sum<<<1, 256, sm, st>>>(p, m);
  return 3;
}

// ================================================= membrane step, one block ===
// The membrane step of a small mesh in one block: the phases of the wide
// kernels separated by __syncthreads instead of kernel boundaries.  A
// simulation then launches two kernels for its membrane per step instead
// of eight, which is what limits many small simulations sharing a GPU.
// Each phase calls the same per-item functions in the same order as the
// wide kernels, so results are bit for bit the same.
__global__ void __launch_bounds__(kBlockT) k_membrane_block(DevParams p, Membrane m, FastBufs f, uint64_t eoff) {
  extern __shared__ double shb[];
  const int T = blockDim.x, t = threadIdx.x;
  for (int i = t; i < p.nv; i += T) m_drift_item(p, m, i);
  __syncthreads();
  for (int i = t; i < p.nt; i += T) {
    m_av_item(p, m, i);
    shb[i] = m.area[i];
    shb[p.nt + i] = m.vol[i];
  }
  __syncthreads();
  // warps 0 and 1: Sarea and Volume (area_volume_sums); the others: edge and
  // bending terms and the bond preparation
  if (t < 64) area_volume_sums(p, m, shb, shb + p.nt, t);
  else {
    const int n = 2 * p.ne + p.nv;
    for (int k = t - 64; k < n; k += T - 64) {
      if (k < p.ne) force_item(p, m, f.slot, k);
      else if (k < 2 * p.ne) force_item(p, m, f.slot, p.nt + k);
      else bond_prep_item(p, m, f.vd, f.vw, f.vX, k - 2 * p.ne);
    }
  }
  __syncthreads();
  for (int k = t; k < p.nt; k += T) force_item(p, m, f.slot, p.ne + k);
  __syncthreads();
  {
    const int lane = t & 31;
    double* shw = shb + (t >> 5) * (kGSlots * 3 + 3);
    for (int i = t >> 5; i < p.nv; i += T >> 5) gather_vertex(p, m, f.slot, f.gstart, f.gidx, i, lane, shw);
  }
  __syncthreads();
  tail_b_block(p, m, f.vd, f.vw, f.vX, epoch_of(p, eoff), *reinterpret_cast<TailSmem*>(shb));
}

// ================================================ membrane step, one cluster ===
// The whole membrane step of a mesh of any size in ONE launch: a cluster of
// kClusterCTAs blocks of kClusterT threads, co-scheduled on one GPC, whose
// phases are separated by cluster barriers (barrier.cluster arrive.release /
// wait.acquire: every global write of one phase is visible to all blocks of
// the cluster in the next) instead of kernel boundaries.  Each phase calls
// the same per-item functions in the same order as the wide kernels, so
// results are bit for bit the same; the chain of eight dependent launches
// becomes one.  next_kick: the next step's half-kick, snapshot next_buf and
// its triangle records follow in the same launch.
__global__ void __launch_bounds__(kClusterT)
    k_membrane_cluster(DevParams p, Membrane m, FastBufs f, uint64_t eoff, int next_kick, int next_buf) {
  extern __shared__ double shc[];
  cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
  const int T = blockDim.x, t = threadIdx.x;
  const int cta = (int)cl.block_rank();
  const int g = cta * T + t, G = kClusterCTAs * T;
  for (int i = g; i < p.nv; i += G) m_drift_item(p, m, i);
  cl.sync();
  for (int i = g; i < p.nt; i += G) m_av_item(p, m, i);
  cl.sync();
  // block 0's warps 0 and 1: Sarea and Volume (area_volume_sums), staged in its
  // shared memory when they fit; every other thread of the cluster: the
  // edge and bending terms and the bond preparation
  const bool staged = p.nt <= kSumSmemT;
  if (cta == 0 && staged) {
    for (int i = t; i < p.nt; i += T) { shc[i] = m.area[i]; shc[p.nt + i] = m.vol[i]; }
    __syncthreads();
  }
  if (cta == 0 && t < 64) {
    area_volume_sums(p, m, staged ? shc : m.area, staged ? shc + p.nt : m.vol, t);
  } else {
    const int n = 2 * p.ne + p.nv;
    for (int k = g - 64; k < n; k += G - 64) {
      if (k < p.ne) force_item(p, m, f.slot, k);
      else if (k < 2 * p.ne) force_item(p, m, f.slot, p.nt + k);  // dihedral k - E
      else bond_prep_item(p, m, f.vd, f.vw, f.vX, k - 2 * p.ne);
    }
  }
  cl.sync();
  for (int k = g; k < p.nt; k += G) force_item(p, m, f.slot, p.ne + k);
  cl.sync();
  {
    const int lane = t & 31;
    double* shw = shc + (t >> 5) * (kGSlots * 3 + 3);
    for (int i = g >> 5; i < p.nv; i += G >> 5) gather_vertex(p, m, f.slot, f.gstart, f.gidx, i, lane, shw);
  }
  cl.sync();
  if (cta == 0) tail_b_block(p, m, f.vd, f.vw, f.vX, epoch_of(p, eoff), *reinterpret_cast<TailSmem*>(shc));
  if (!next_kick) return;
  cl.sync();
  for (int i = g; i < p.nv; i += G) kick_snap_item(p, m, f.snap[next_buf], i);
  cl.sync();
  for (int j = g; j < p.nt; j += G) tri_prep_one(p, m, j, m.vx, m.vy, m.vz, f.pre[next_buf]);
}

static size_t cluster_smem(const DevParams& p) {
  size_t b = std::max((size_t)(kClusterT / 32) * (kGSlots * 3 + 3) * sizeof(double), sizeof(TailSmem));
  return p.nt <= kSumSmemT ? std::max(b, 2 * (size_t)p.nt * sizeof(double)) : b;
}

static size_t block_smem(const DevParams& p) {
  size_t b = std::max((size_t)(kBlockT / 32) * (kGSlots * 3 + 3) * sizeof(double), sizeof(TailSmem));
  return std::max(b, 2 * (size_t)p.nt * sizeof(double));
}

bool one_block_fits(const DevParams& p) { return p.nv <= kBlockMaxV && 2 * (size_t)p.nt * sizeof(double) <= 96 * 1024; }

int fast_membrane_step(const DevParams& p, Membrane& m, FastBufs& f, uint64_t epoch, int next_kick, int next_buf,
                       cudaStream_t st, cudaEvent_t readers) {
  if (f.cluster) {
    // the snapshot the kick writes was read by the previous streaming
    if (next_kick && readers) cudaStreamWaitEvent(st, readers, 0);
    // one cluster of kClusterCTAs blocks
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(kClusterCTAs);
    cfg.blockDim = dim3(kClusterT);
    cfg.dynamicSmemBytes = cluster_smem(p);
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = kClusterCTAs;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k_membrane_cluster, p, m, f, epoch, next_kick, next_buf);
    return 1;
  }
  if (!f.one_block)
    return fast_drift_va(p, m, st, false) + fast_forces_tail(p, m, f, epoch, next_kick, next_buf, st, true, readers);
  const size_t smem = block_smem(p);
  k_membrane_block<<<1, kBlockT, smem, st>>>(p, m, f, epoch);
  int n = 1;
  if (next_kick) {
    if (readers) cudaStreamWaitEvent(st, readers, 0);
    n += fast_kick_prep(p, m, f, next_buf, st);
  }
  return n;
}

int fast_forces_tail(const DevParams& p, Membrane& m, FastBufs& f, uint64_t epoch, int next_kick, int next_buf,
                     cudaStream_t st, bool sum_pending, cudaEvent_t readers) {
  const size_t sm = (sum_pending && p.nt <= kSumSmemT) ? 2 * (size_t)p.nt * sizeof(double) : 0;
  k_sum_edges<<<1 + nb(2 * p.ne + p.nv, 256), 256, sm, st>>>(p, m, f.slot, sum_pending ? 1 : 0, f.vd, f.vw, f.vX);
  k_force_tri<<<nb(p.nt, 128), 128, 0, st>>>(p, m, f.slot);
  k_force_gather_w<<<nb(p.nv, kGW), 32 * kGW, 0, st>>>(p, m, f.slot, f.gstart, f.gidx);
  k_tail_b<<<1, kTailT, 0, st>>>(p, m, f.vd, f.vw, f.vX, epoch);
  int n = 4;
  if (next_kick) {
    if (readers) cudaStreamWaitEvent(st, readers, 0);
    n += fast_kick_prep(p, m, f, next_buf, st);
  }
  return n;
}


}  // namespace irbc

// FP32-bulk solvent kernels share the device helpers above
#include "fp32.cuh"

// one launch per phase over a cohort of FP32 simulations
#include "multi.cuh"
