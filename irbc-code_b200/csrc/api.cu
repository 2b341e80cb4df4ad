// api.cu -- the C ABI of include/irbc.h: one handle per simulation, the
// host-side set-up that main() performs before its loop (maincode.cpp:
// 94-446), state exchange in the reference's layout, the step sequence of
// the loop body (maincode.cpp:461-764) and the output writers.
#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <mutex>
#include <string>
#include <vector>

#include "cohort.h"
#include "fast.h"
#include "fp32.h"
#include "multi.h"
#include "irbc.h"
#include "sim.h"

using namespace irbc;

namespace irbc {
std::atomic<int64_t> g_launches{0};
}

struct irbc_handle {
  uint64_t uid = 0;        // unique for the life of the process (a freed handle's address can return)
  void* rec = nullptr;     // device staging of irbc_record_async
  irbc_params P{};
  DevParams dp{};
  Solvent s;
  Cells c;
  Membrane m;
  cudaStream_t st = nullptr;   // solvent kernels; every public call orders on it
  cudaStream_t st2 = nullptr;  // membrane kernels, run beside the solvent ones (== st with one stream)
  cudaStream_t st2_own = nullptr;  // the side stream this handle created
  int mem_mode = 1;                // membrane step: 1 wide kernels, 2 one block, 3 one cluster
  FastBufs fb;
  bool fp32 = false;           // solvent held in sf (float4) between exchanges
  SolventF sf;
  int snap_buf = 0;            // which snapshot the next streaming step reads
  bool snap_ready = false;     // snapshot/triangle prep of the next step done
  cudaEvent_t ev_snap = nullptr, ev_mem = nullptr, ev_coll = nullptr, ev_str[2] = {nullptr, nullptr};
  cudaEvent_t ev_vbin = nullptr;
  uint64_t* ebase = nullptr;   // device: the draw epoch base of the current call (DevParams::ebase)
  int64_t ebase_val = 0;       // its value as last written
  // captured step sequences (irbc_step): one per starting configuration
  struct StepGraph {
    cudaGraphExec_t exec = nullptr;
    int colsteps0 = 0, parity = 0;
    double wallspeed = 0;
    int64_t launches = 0, collisions = 0;
  };
  std::vector<StepGraph> graphs;
  bool graphs_on = false;  // measured slower than stream launches on the large box: opt in
  bool capturing = false;
  std::string err;
  bool have_mesh = false;
  int64_t step = 0;
  int colsteps = -1, upd = 0, filecc = 0, filec = 0, bbi = 0;
  int csteps = 10, uplist = 83;
  double report[9] = {0};
  std::vector<double> xlig, ylig;
  double* obs = nullptr;  // device scratch for observables
  // run-time health word (DevParams::health) and its page-locked host
  // mirror, copied after every irbc_step call (ev_health marks the copy)
  int* health = nullptr;
  int* health_host = nullptr;
  cudaEvent_t ev_health = nullptr;
  int64_t launches0 = 0;
  // CUDA-event profiling window
  bool prof = false;
  cudaEvent_t ev_begin = nullptr, ev_end = nullptr;
  std::vector<cudaEvent_t> ev_pool;
  size_t ev_used = 0;
  struct Mark { int cat; size_t start, end; };  // a timed span: pool indices of its two events
  std::vector<Mark> ev_marks;
  int64_t prof_launch0 = 0;
};

namespace {

int fail(irbc_handle* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  return code;
}

#define CK(call)                                                                         \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return fail(h, IRBC_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

template <typename T>
cudaError_t dalloc(T** p, int64_t n) {
  *p = nullptr;
  if (n <= 0) n = 1;
  return cudaMalloc((void**)p, sizeof(T) * (size_t)n);
}

template <typename T>
void dfree(T*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}

void fill_devparams_from(const irbc_params& P, DevParams& d) {
  d.a = P.a; d.Lx = P.Lx; d.Ly = P.Ly; d.Lz = P.Lz; d.dtcd = P.dtcd; d.navg = P.navg;
  d.Theta = P.Theta; d.walls = P.walls; d.mass = P.mass; d.cosalpha = P.cosalpha; d.sinalpha = P.sinalpha;
  d.kappasa = P.kappasa; d.kappad = P.kappad; d.kappav = P.kappav; d.kappab = P.kappab; d.pmass = P.pmass;
  d.dtmd = P.dtmd; d.ks = P.ks; d.dthr = P.dthr; d.FD = P.FD; d.Fg = P.Fg; d.el0 = P.el0;
  d.PRmass = P.PRmass; d.paraR = P.paraR; d.Pi = P.Pi; d.elap = P.elap; d.onrate = P.onrate;
  d.offrate = P.offrate; d.randno = P.randno; d.seed = P.seed;
  d.nx = (int)(P.Lx / P.a);
  d.ny = (int)(P.Ly / P.a);
  d.nz = (int)(P.Lz / P.a) + 1;
  d.ncell = (int64_t)d.nx * d.ny * d.nz;
  d.tree_sums = P.precision == IRBC_FP32 ? 1 : 0;
}

void fill_devparams(irbc_handle* h) { fill_devparams_from(h->P, h->dp); }

// ligand grid (maincode.cpp:77-93)
void build_ligands(irbc_handle* h) {
  h->xlig.clear(); h->ylig.clear();
  double xmin = 0.0, ymin = 0.0;
  int ny = 0;
  while (xmin < h->P.Lx) {
    int k = 0;
    while (ymin < h->P.Ly) { h->xlig.push_back(xmin); h->ylig.push_back(ymin); ymin += 0.5; ++k; }
    ny = k;
    xmin += 0.5; ymin = 0;
  }
  h->dp.nligy = ny;
  h->dp.nlig = (int)h->xlig.size();
  h->dp.nligx = ny ? h->dp.nlig / ny : 0;
}

void free_membrane(Membrane& m) {
  for (double** p : {&m.x, &m.y, &m.z, &m.vx, &m.vy, &m.vz, &m.fx, &m.fy, &m.fz, &m.poff, &m.pon, &m.l0,
                     &m.kappap, &m.tarea, &m.area, &m.vol, &m.tcx, &m.tcy, &m.tcz, &m.pair_d})
    dfree(*p);
  for (int** p : {&m.pid, &m.ix, &m.iy, &m.bondi, &m.bondl, &m.knob, &m.e1, &m.e2, &m.es1, &m.es2, &m.iedge,
                  &m.t1, &m.t2, &m.t3, &m.inc_start, &m.inc, &m.npair, &m.pair_j})
    dfree(*p);
  dfree(m.vkey);
}

// Host copy of the membrane used during set-up.
struct HostMesh {
  int nv = 0, ne = 0, nt = 0;
  std::vector<double> x, y, z, vx, vy, vz;
  std::vector<int> ix, iy;
  std::vector<int> e1, e2, es1, es2, iedge, t1, t2, t3;
  std::vector<double> l0, kappap, tarea, cmx, cmy, cmz;
  double Sarea0 = 0, Volume0 = 0, theta0 = 0, center[3] = {0, 0, 0};
};

inline void hcp(const double A[], const double B[], double C[]) {
  C[0] = (A[1] * B[2]) - (B[1] * A[2]);
  C[1] = (A[2] * B[0]) - (B[2] * A[0]);
  C[2] = (A[0] * B[1]) - (B[0] * A[1]);
}

double h_areatri(const HostMesh& M, double Lx, double Ly, int p1, int p2, int p3) {
  auto UX = [&](int v) { return M.x[v] + M.ix[v] * Lx; };
  auto UY = [&](int v) { return M.y[v] + M.iy[v] * Ly; };
  double A[3] = {UX(p2) - UX(p1), UY(p2) - UY(p1), M.z[p2] - M.z[p1]};
  double B[3] = {UX(p3) - UX(p1), UY(p3) - UY(p1), M.z[p3] - M.z[p1]};
  double eta[3];
  hcp(A, B, eta);
  return 0.5 * sqrt(eta[0] * eta[0] + eta[1] * eta[1] + eta[2] * eta[2]);
}

double h_voltri(const HostMesh& M, double Lx, double Ly, int p1, int p2, int p3) {
  auto UX = [&](int v) { return M.x[v] + M.ix[v] * Lx; };
  auto UY = [&](int v) { return M.y[v] + M.iy[v] * Ly; };
  double A[3] = {UX(p1), UY(p1), M.z[p1]}, B[3] = {UX(p2), UY(p2), M.z[p2]}, C[3] = {UX(p3), UY(p3), M.z[p3]};
  double Cn[3];
  for (int k = 0; k < 3; ++k) Cn[k] = (A[k] + B[k] + C[k]) / 3.0;
  double E1[3] = {UX(p2) - UX(p1), UY(p2) - UY(p1), M.z[p2] - M.z[p1]};
  double E2[3] = {UX(p3) - UX(p1), UY(p3) - UY(p1), M.z[p3] - M.z[p1]};
  double D[3];
  hcp(E1, E2, D);
  return (1.0 / 6.0) * ((D[0] * Cn[0]) + (D[1] * Cn[1]) + (D[2] * Cn[2]));
}

// edgest (maincode.cpp:276-342): the third vertex of the first and of the
// last triangle (in file order) holding both ends of each edge.  A map from
// the vertex pair to its triangles replaces the E x T scan.
void build_edgest(HostMesh& M) {
  M.es1.assign(M.ne, 0); M.es2.assign(M.ne, 0);
  std::vector<std::vector<int>> vt(M.nv);
  for (int j = 0; j < M.nt; ++j) { vt[M.t1[j]].push_back(j); vt[M.t2[j]].push_back(j); vt[M.t3[j]].push_back(j); }
  for (int i = 0; i < M.ne; ++i) {
    int l1 = M.e1[i], l2 = M.e2[i];
    std::vector<int> both;
    for (int j : vt[l1]) {
      if (M.t1[j] == l2 || M.t2[j] == l2 || M.t3[j] == l2) both.push_back(j);
    }
    std::sort(both.begin(), both.end());
    both.erase(std::unique(both.begin(), both.end()), both.end());
    auto third = [&](int j, int& out) {
      if (M.t1[j] != l1 && M.t1[j] != l2) out = M.t1[j];
      if (M.t2[j] != l1 && M.t2[j] != l2) out = M.t2[j];
      if (M.t3[j] != l1 && M.t3[j] != l2) out = M.t3[j];
    };
    if (!both.empty()) { third(both.front(), M.es1[i]); third(both.back(), M.es2[i]); }
  }
}

// makeiedge (Src/memfuncs.cpp:533-588) after centerofmass (:55-74)
void build_iedge(HostMesh& M, double Lx, double Ly, double Lz) {
  double rr[3] = {0, 0, 0};
  for (int i = 0; i < M.nv; ++i) { rr[0] += M.x[i] + M.ix[i] * Lx; rr[1] += M.y[i] + M.iy[i] * Ly; rr[2] += M.z[i]; }
  M.center[0] = fmod(rr[0] / (double)M.nv, Lx);
  M.center[1] = fmod(rr[1] / (double)M.nv, Ly);
  M.center[2] = fmod(rr[2] / (double)M.nv, Lz);
  M.iedge.assign(M.ne, 1);
  for (int i = 0; i < M.ne; ++i) {
    int l2 = M.e1[i], l3 = M.e2[i], l1 = M.es1[i], l4 = M.es2[i];
    double a21[3] = {M.x[l2] - M.x[l1], M.y[l2] - M.y[l1], M.z[l2] - M.z[l1]};
    double a31[3] = {M.x[l3] - M.x[l1], M.y[l3] - M.y[l1], M.z[l3] - M.z[l1]};
    double a24[3] = {M.x[l2] - M.x[l4], M.y[l2] - M.y[l4], M.z[l2] - M.z[l4]};
    double a34[3] = {M.x[l3] - M.x[l4], M.y[l3] - M.y[l4], M.z[l3] - M.z[l4]};
    double t1[3], t2[3], eta[3], zeta[3];
    t1[0] = (M.x[l1] + M.x[l2] + M.x[l3]) / 3.0; t1[1] = (M.y[l1] + M.y[l2] + M.y[l3]) / 3.0;
    t1[2] = (M.z[l1] + M.z[l2] + M.z[l3]) / 3.0;
    t2[0] = (M.x[l4] + M.x[l2] + M.x[l3]) / 3.0; t2[1] = (M.y[l4] + M.y[l2] + M.y[l3]) / 3.0;
    t2[2] = (M.z[l4] + M.z[l2] + M.z[l3]) / 3.0;
    hcp(a21, a31, eta);
    hcp(a34, a24, zeta);
    double che1 = eta[0] * (t1[0] - M.center[0]) + eta[1] * (t1[1] - M.center[1]) + eta[2] * (t1[2] - M.center[2]);
    double che2 = zeta[0] * (t2[0] - M.center[0]) + zeta[1] * (t2[1] - M.center[1]) + zeta[2] * (t2[2] - M.center[2]);
    if ((che1 >= 0) && (che2 >= 0)) M.iedge[i] = 1;
    else if ((che1 < 0) && (che2 < 0)) M.iedge[i] = -1;
    else M.iedge[i] = 1;
  }
}

// per-vertex contribution lists in the order force_calculate_dt adds them
void build_incidence(const HostMesh& M, std::vector<int>& start, std::vector<int>& inc) {
  std::vector<std::vector<int>> L(M.nv);
  auto enc = [](int kind, int role, int item) { return (kind << 30) | (role << 27) | item; };
  for (int i = 0; i < M.ne; ++i) {
    L[M.e1[i]].push_back(enc(0, 0, i));
    L[M.e2[i]].push_back(enc(0, 1, i));
  }
  for (int i = 0; i < M.nt; ++i) {
    L[M.t1[i]].push_back(enc(1, 0, i));
    L[M.t2[i]].push_back(enc(1, 1, i));
    L[M.t3[i]].push_back(enc(1, 2, i));
  }
  for (int i = 0; i < M.ne; ++i) {
    int l2, l3;
    if (M.iedge[i] == -1) { l3 = M.e1[i]; l2 = M.e2[i]; } else { l2 = M.e1[i]; l3 = M.e2[i]; }
    int l1 = M.es1[i], l4 = M.es2[i];
    L[l1].push_back(enc(2, 0, i));
    L[l4].push_back(enc(2, 1, i));
    L[l2].push_back(enc(2, 2, i));
    L[l3].push_back(enc(2, 3, i));
  }
  start.assign(M.nv + 1, 0);
  inc.clear();
  for (int v = 0; v < M.nv; ++v) {
    start[v] = (int)inc.size();
    inc.insert(inc.end(), L[v].begin(), L[v].end());
  }
  start[M.nv] = (int)inc.size();
}

template <typename T>
int up(irbc_handle* h, T* d, const std::vector<T>& v) {
  if (v.empty()) return 0;
  CK(cudaMemcpyAsync(d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, h->st));
  return 0;
}
template <typename T>
int up(irbc_handle* h, T* d, const T* v, int64_t n) {
  if (n <= 0) return 0;
  CK(cudaMemcpyAsync(d, v, sizeof(T) * (size_t)n, cudaMemcpyHostToDevice, h->st));
  return 0;
}
template <typename T>
int down(irbc_handle* h, T* v, const T* d, int64_t n) {
  if (n <= 0 || !v) return 0;
  CK(cudaMemcpyAsync(v, d, sizeof(T) * (size_t)n, cudaMemcpyDeviceToHost, h->st));
  return 0;
}

void free_fast(FastBufs& f) {
  for (int b = 0; b < 2; ++b) {
    for (double** q : {&f.snap[b].x, &f.snap[b].y, &f.snap[b].z, &f.snap[b].vx, &f.snap[b].vy, &f.snap[b].vz})
      dfree(*q);
    dfree(f.pre[b]);
  }
  dfree(f.slot); dfree(f.gstart); dfree(f.gidx); dfree(f.vd); dfree(f.vw); dfree(f.vX);
}

// per-vertex force slots in the order force_calculate_dt adds the terms:
// slots 4i..4i+3 of edge i (l1 WLC, l1 POW, l2 WLC, l2 POW), 9 per triangle
// after 4E (alpha, alphad per corner, then the three volume terms), 4 per
// dihedral after 4E+9T (l1, l4, l2, l3)
void build_gather(const HostMesh& M, const std::vector<int>& start, const std::vector<int>& inc,
                  std::vector<int>& gstart, std::vector<int>& gidx) {
  const int base_t = 4 * M.ne, base_d = 4 * M.ne + 9 * M.nt;
  gstart.assign(M.nv + 1, 0);
  gidx.clear();
  for (int v = 0; v < M.nv; ++v) {
    gstart[v] = (int)gidx.size();
    for (int q = start[v]; q < start[v + 1]; ++q) {
      int e = inc[q];
      int kind = (e >> 30) & 3, role = (e >> 27) & 7, item = e & ((1 << 27) - 1);
      if (kind == 0) {
        gidx.push_back(4 * item + 2 * role);
        gidx.push_back(4 * item + 2 * role + 1);
      } else if (kind == 1) {
        gidx.push_back(base_t + 9 * item + 2 * role);
        gidx.push_back(base_t + 9 * item + 2 * role + 1);
        gidx.push_back(base_t + 9 * item + 6 + role);
      } else {
        gidx.push_back(base_d + 4 * item + role);
      }
    }
  }
  gstart[M.nv] = (int)gidx.size();
}

void invalidate_graphs(irbc_handle* h);

// allocates the membrane and uploads the topology
int upload_mesh(irbc_handle* h, const HostMesh& M) {
  Membrane& m = h->m;
  if (M.nv > 8192) return fail(h, IRBC_ERR_ARG, "at most 8192 membrane vertices");
  invalidate_graphs(h);
  free_membrane(m);
  free_fast(h->fb);
  h->snap_ready = false;
  m.nv = M.nv; m.ne = M.ne; m.nt = M.nt;
  for (double** p : {&m.x, &m.y, &m.z, &m.vx, &m.vy, &m.vz, &m.fx, &m.fy, &m.fz, &m.poff, &m.pon})
    CK(dalloc(p, M.nv));
  for (int** p : {&m.pid, &m.ix, &m.iy, &m.bondi, &m.bondl, &m.knob, &m.npair}) CK(dalloc(p, M.nv));
  CK(dalloc(&m.vkey, M.nv));
  CK(dalloc(&m.pair_d, (int64_t)M.nv * kMaxPairs));
  CK(dalloc(&m.pair_j, (int64_t)M.nv * kMaxPairs));
  for (int** p : {&m.e1, &m.e2, &m.es1, &m.es2, &m.iedge}) CK(dalloc(p, M.ne));
  for (double** p : {&m.l0, &m.kappap}) CK(dalloc(p, M.ne));
  for (int** p : {&m.t1, &m.t2, &m.t3}) CK(dalloc(p, M.nt));
  for (double** p : {&m.tarea, &m.area, &m.vol, &m.tcx, &m.tcy, &m.tcz}) CK(dalloc(p, M.nt));
  std::vector<int> start, inc;
  build_incidence(M, start, inc);
  CK(dalloc(&m.inc_start, M.nv + 1));
  CK(dalloc(&m.inc, (int64_t)inc.size()));
  if (up(h, m.inc_start, start) || up(h, m.inc, inc)) return IRBC_ERR_CUDA;
  {
    FastBufs& f = h->fb;
    for (int b = 0; b < 2; ++b) {
      for (double** q : {&f.snap[b].x, &f.snap[b].y, &f.snap[b].z, &f.snap[b].vx, &f.snap[b].vy, &f.snap[b].vz})
        CK(dalloc(q, M.nv));
      CK(dalloc(&f.pre[b], M.nt));
      f.snap[b].t1 = m.t1; f.snap[b].t2 = m.t2; f.snap[b].t3 = m.t3;
    }
    std::vector<int> gstart, gidx;
    build_gather(M, start, inc, gstart, gidx);
    CK(dalloc(&f.slot, 3 * (int64_t)(8 * M.ne + 9 * M.nt)));
    CK(dalloc(&f.gstart, M.nv + 1));
    CK(dalloc(&f.gidx, (int64_t)gidx.size()));
    CK(dalloc(&f.vd, M.nv));
    CK(dalloc(&f.vw, M.nv));
    CK(dalloc(&f.vX, 3 * (int64_t)M.nv));
    if (up(h, f.gstart, gstart) || up(h, f.gidx, gidx)) return IRBC_ERR_CUDA;
  }
  if (up(h, m.e1, M.e1) || up(h, m.e2, M.e2) || up(h, m.es1, M.es1) || up(h, m.es2, M.es2) ||
      up(h, m.iedge, M.iedge) || up(h, m.l0, M.l0) || up(h, m.kappap, M.kappap) || up(h, m.t1, M.t1) ||
      up(h, m.t2, M.t2) || up(h, m.t3, M.t3) || up(h, m.tarea, M.tarea))
    return IRBC_ERR_CUDA;
  CK(cudaMemsetAsync(m.npair, 0, sizeof(int) * M.nv, h->st));
  h->dp.nv = M.nv; h->dp.ne = M.ne; h->dp.nt = M.nt;
  h->dp.Sarea0 = M.Sarea0; h->dp.Volume0 = M.Volume0; h->dp.theta0 = M.theta0;
  // cos/sin(theta0*Pi/180) evaluated on the host exactly as the reference
  // does inside its bending loop (Src/memfuncs.cpp:401)
  h->dp.cth0 = cos(M.theta0 * h->P.Pi / 180.0);
  h->dp.sth0 = sin(M.theta0 * h->P.Pi / 180.0);
  h->have_mesh = true;
  h->fb.one_block = h->mem_mode == 2 && one_block_fits(h->dp);
  h->fb.cluster = h->mem_mode == 3;
  return 0;
}

int64_t launches_in(const irbc_handle* h) { return g_launches.load() - h->launches0; }

// the status for a health word: 0, or IRBC_ERR_HEALTH with the message
int health_status(irbc_handle* h, int flags) {
  if (!flags) return 0;
  std::string m = "health check:";
  if (flags & HEALTH_SOLVENT) m += " a solvent particle became non-finite or left the box;";
  if (flags & HEALTH_MEMBRANE) m += " a membrane vertex became non-finite;";
  return fail(h, IRBC_ERR_HEALTH, m);
}

// a fresh state: clears the health word and its host mirror
cudaError_t clear_health(irbc_handle* h) {
  *h->health_host = 0;
  return cudaMemsetAsync(h->health, 0, sizeof(int), h->st);
}

// epoch base for the launches that follow on the main stream (the side
// stream joins after it through the usual events)
cudaError_t set_epoch_base(irbc_handle* h, uint64_t base) {
  h->ebase_val = (int64_t)base;
  launch_set_u64(h->ebase, base, h->st);
  return cudaGetLastError();
}

void invalidate_graphs(irbc_handle* h) {
  for (auto& g : h->graphs)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  h->graphs.clear();
}

// the solvent kernels of the handle's precision
// physical re-sort of the solvent by the latest collision's cells
int resort_any(irbc_handle* h, cudaStream_t st) {
  if (h->fp32) launch_resort_f(h->sf, h->s, st);
  else launch_resort(h->s, st);
  h->s.resorted = h->s.ncoll;
  return h->s.n ? 2 : 0;
}

// returns the number of kernels launched: vbin, count, ghost flags, three
// scan kernels, perm, cells, and the physical re-sort when due (never while
// a step sequence is being captured; irbc_step re-sorts between captured
// sequences).  With a side stream the vertex binning runs there (after
// whatever the side stream already holds: the membrane of the previous
// step) while the solvent's cell counts start at once on the main stream.
int collide_any(irbc_handle* h, uint64_t epoch, cudaStream_t st, cudaStream_t side = nullptr) {
  h->s.ncoll += 1;
  const bool resort = !h->capturing && h->s.ncoll - h->s.resorted >= kResortEvery;
  if (resort) h->s.resorted = h->s.ncoll;
  launch_vbin(h->dp, h->m, h->c, epoch, side ? side : st);
  if (h->fp32) launch_collide_count_f(h->dp, h->sf, h->s, h->c, epoch, st);
  else launch_collide_count(h->dp, h->s, h->c, epoch, st);
  if (side) {
    cudaEventRecord(h->ev_vbin, side);
    cudaStreamWaitEvent(st, h->ev_vbin, 0);
  }
  if (h->fp32) launch_collide_finish_f(h->dp, h->sf, h->s, h->c, h->m, epoch, st, resort);
  else launch_collide_finish(h->dp, h->s, h->c, h->m, epoch, st, resort);
  return 8 + (resort && h->s.n ? 2 : 0);
}

// profiling: a pair of events around a launch group of a category
enum { PROF_STREAM = 0, PROF_COLLIDE = 1, PROF_MEMBRANE = 2, PROF_STREAM_BULK = 3 };
cudaEvent_t next_event(irbc_handle* h) {
  if (h->ev_used == h->ev_pool.size()) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    h->ev_pool.push_back(e);
  }
  return h->ev_pool[h->ev_used++];
}
struct ProfScope {
  irbc_handle* h;
  size_t mark;
  cudaStream_t st;
  bool on;
  ProfScope(irbc_handle* hh, int cat, cudaStream_t s = nullptr)
      : h(hh), mark(0), st(s ? s : hh->st), on(hh->prof && !hh->capturing) {
    if (!on) return;
    const size_t idx = h->ev_used;
    cudaEventRecord(next_event(h), st);
    mark = h->ev_marks.size();
    h->ev_marks.push_back({cat, idx, idx});
  }
  ~ProfScope() {
    if (!on) return;
    h->ev_marks[mark].end = h->ev_used;
    cudaEventRecord(next_event(h), st);
  }
};

// the streaming kernels; in a profiling window the bulk kernel alone is
// bracketed by a pair of events of its own
// returns the number of kernels it launched
int stream_any(irbc_handle* h, int buf, cudaStream_t st, cudaEvent_t snap = nullptr) {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (h->prof && !h->capturing) {
    h->ev_marks.push_back({PROF_STREAM_BULK, h->ev_used, h->ev_used + 1});
    e0 = next_event(h);
    e1 = next_event(h);
  }
  // the staging capacity follows the longest list; captured steps keep the
  // largest, so that a replay stays valid after the lists grow
  h->fb.hcap = (h->graphs_on || h->capturing) ? kHeavyList : heavy_cap(h->c.lmax);
  if (h->fp32) return fast_stream_f(h->dp, h->sf, h->c, h->fb, buf, st, e0, e1, snap);
  return fast_stream(h->dp, h->s, h->c, h->fb, buf, st, e0, e1, snap);
}

}  // namespace

// ============================================================== C ABI ======
extern "C" void irbc_params_default(irbc_params* p) {
  std::memset(p, 0, sizeof(*p));
  p->a = 1.0; p->Lx = 60.0; p->Ly = 40.0; p->Lz = 40.0; p->Ns = 960000;
  p->dtcd = 0.02; p->navg = 10.0; p->Theta = 1.0; p->walls = 3.0; p->mass = 1.0;
  p->cosalpha = -0.70710678118; p->sinalpha = 0.70710678118;
  p->Nt = 600; p->kappasa = 60000.0; p->kappad = 1200.0; p->kappav = 6000.0; p->kappab = 100.0;
  p->pmass = 10.0 * 1.0; p->dtmd = 0.002; p->ks = 6000.0; p->dthr = 0.50; p->FD = 1200.0;
  p->Fg = 40.0; p->el0 = 0.1; p->PRmass = 10.0; p->paraR = 1.7; p->Pi = 3.141592653;
  p->elap = 0.0005; p->shear = 1200.0; p->onrate = 0.005; p->offrate = 0.015;
  p->warm_steps = 250000; p->warm_speed = 0.1; p->out_every = 5000; p->randno = 12345678;
  p->seed = 12345; p->precision = IRBC_FP64; p->device = 0;
}

extern "C" int64_t irbc_footprint_bytes(const irbc_params* p, int32_t nv, int32_t ne, int32_t nt) {
  int64_t nx = (int64_t)(p->Lx / p->a), ny = (int64_t)(p->Ly / p->a), nz = (int64_t)(p->Lz / p->a) + 1;
  int64_t C = nx * ny * nz;
  int64_t ns = p->Ns;
  int64_t b = ns * (2 * (3 * 8 + 32 + 2 * 4) + 4 * 4);  // two buffer sets + key/slot/perm/stream queue
  if (p->precision == IRBC_FP32) b += ns * (2 * 32 + 2 * 4);  // float4 sets + cell ids
  b += C * (7 * 4) + (C + 1) * 4 * 3;                // cell counts/ranks + cell and llist starts
  b += (int64_t)nv * (12 * 8 + 8 * 4 + kMaxPairs * 12) + (int64_t)ne * 40 + (int64_t)nt * 80;
  b += 2 * (int64_t)(4 * p->Lx * 4 * p->Ly) * 16;    // ligands
  b += 2 * C * 4 * 8;                                 // llist entries (typical)
  return b;
}

// why the calling thread's last irbc_create failed (irbc_last_error(NULL))
static thread_local std::string g_create_err;
static int create_failed(int code, const char* what) {
  const cudaError_t e = cudaGetLastError();
  g_create_err = std::string("irbc_create: ") + what + (e != cudaSuccess ? std::string(": ") + cudaGetErrorString(e) : "");
  return code;
}

extern "C" int irbc_create(const irbc_params* p, irbc_handle** out) {
  g_create_err.clear();
  irbc_handle* h = nullptr;
  if (!p || !out) return IRBC_ERR_ARG;
  *out = nullptr;
  if (p->Lx <= 0 || p->Ly <= 0 || p->Lz <= 0 || p->a != 1.0 || p->Ns < 0 || p->dtmd <= 0)
    return IRBC_ERR_ARG;
  if (p->precision != IRBC_FP64 && p->precision != IRBC_FP32) return IRBC_ERR_ARG;
  int64_t nx = (int64_t)(p->Lx / p->a), ny = (int64_t)(p->Ly / p->a), nz = (int64_t)(p->Lz / p->a) + 1;
  if (nx * ny * nz >= (1LL << 31) || p->Ns >= (1LL << 31)) return IRBC_ERR_ARG;
  h = new irbc_handle();
  {
    static std::atomic<uint64_t> next_uid{1};
    h->uid = next_uid.fetch_add(1);
  }
  h->P = *p;
  cudaError_t e = cudaSetDevice(p->device);
  if (e != cudaSuccess) { delete h; return create_failed(IRBC_ERR_CUDA, "cudaSetDevice"); }
  if (cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking) != cudaSuccess) {
    delete h;
    return create_failed(IRBC_ERR_CUDA, "stream");
  }
  {
    // the membrane chain is latency bound: give its stream the higher priority
    int lo = 0, hi = 0;
    cudaDeviceGetStreamPriorityRange(&lo, &hi);
    if (cudaStreamCreateWithPriority(&h->st2, cudaStreamNonBlocking, hi) != cudaSuccess) {
      cudaStreamDestroy(h->st);
      delete h;
      return IRBC_ERR_CUDA;
    }
    h->st2_own = h->st2;
    for (cudaEvent_t* e : {&h->ev_snap, &h->ev_mem, &h->ev_coll, &h->ev_str[0], &h->ev_str[1], &h->ev_vbin,
                           &h->ev_health})
      cudaEventCreateWithFlags(e, cudaEventDisableTiming);
  }
  {
    // the kernels' shared-memory limits, before this simulation's first
    // launch (and never racing another thread's launches)
    static std::mutex limits_mu;
    std::lock_guard<std::mutex> lk(limits_mu);
    set_kernel_limits();
    cudaGetLastError();
  }
  fill_devparams(h);
  build_ligands(h);
  h->csteps = (int)(p->dtcd / p->dtmd);
  h->uplist = (int)(0.5 / (p->walls * p->dtmd));
  Solvent& s = h->s;
  Cells& c = h->c;
  s.n = p->Ns;
  c.n = h->dp.ncell;
  int rc = 0;
  auto A = [&](cudaError_t err) { if (err != cudaSuccess && rc == 0) rc = IRBC_ERR_CUDA; };
  for (double** q : {&s.x, &s.y, &s.z, &s.x2, &s.y2, &s.z2}) A(dalloc(q, s.n));
  A(dalloc(&s.v, s.n));
  A(dalloc(&s.v2, s.n));
  for (int** q : {&s.indio, &s.pid, &s.indio2, &s.pid2, &s.key, &s.slot, &s.perm}) A(dalloc(q, s.n));
  for (int** q : {&c.cnt, &c.ncm, &c.wrank, &c.mrank, &c.lcnt, &c.lrank, &c.acell}) A(dalloc(q, c.n));
  A(dalloc(&c.start, c.n + 1));
  A(dalloc(&c.lstart, c.n + 1));
  A(dalloc(&c.lstart2, c.n + 1));
  A(dalloc(&c.totals, 12));
  c.scan_blocks = scan_part_blocks(c.n + 1);
  A(dalloc(&c.scan_part, c.scan_blocks * 3 + 3));
  c.lcap = c.lcap2 = std::max<int64_t>(1024, c.n / 16);
  A(dalloc(&c.lidx, c.lcap));
  A(dalloc(&c.lidx2, c.lcap2));
  A(dalloc(&h->m.ligi, h->dp.nlig));
  A(dalloc(&h->m.xlig, h->dp.nlig));
  A(dalloc(&h->m.ylig, h->dp.nlig));
  A(dalloc(&h->m.sc, 1));
  A(dalloc(&h->ebase, 1));
  h->dp.ebase = h->ebase;
  A(dalloc(&h->obs, kObsDoubles));
  A(dalloc(&h->health, 1));
  h->dp.health = h->health;
  A(cudaHostAlloc((void**)&h->health_host, sizeof(int), cudaHostAllocDefault));
  A(dalloc(&h->fb.queue, s.n));
  A(dalloc(&h->fb.qn, 4));
  if (p->precision == IRBC_FP32) {
    h->fp32 = true;
    h->sf.n = s.n;
    for (float4** q : {&h->sf.pos, &h->sf.vel, &h->sf.pos2, &h->sf.vel2}) A(dalloc(q, s.n));
    A(dalloc(&h->sf.pid, s.n));
    A(dalloc(&h->sf.pid2, s.n));
  }
  if (rc) { irbc_destroy(h); return create_failed(rc, "device allocation"); }
  cudaMemsetAsync(c.lstart, 0, sizeof(int) * (c.n + 1), h->st);
  cudaMemsetAsync(h->m.ligi, 0, sizeof(int) * h->dp.nlig, h->st);
  cudaMemsetAsync(h->m.sc, 0, sizeof(MemScalars), h->st);
  cudaMemsetAsync(h->ebase, 0, sizeof(uint64_t), h->st);
  cudaMemsetAsync(h->health, 0, sizeof(int), h->st);
  *h->health_host = 0;
  cudaMemsetAsync(s.pid, 0, sizeof(int) * std::max<int64_t>(1, s.n), h->st);
  cudaMemcpyAsync(h->m.xlig, h->xlig.data(), sizeof(double) * h->dp.nlig, cudaMemcpyHostToDevice, h->st);
  cudaMemcpyAsync(h->m.ylig, h->ylig.data(), sizeof(double) * h->dp.nlig, cudaMemcpyHostToDevice, h->st);
  if (cudaStreamSynchronize(h->st) != cudaSuccess) { irbc_destroy(h); return create_failed(IRBC_ERR_CUDA, "set-up copies"); }
  // the vertex bitonic sort stages up to 8192 keys in dynamic shared memory
  h->launches0 = g_launches.load();
  *out = h;
  return 0;
}

extern "C" void irbc_destroy(irbc_handle* h) {
  if (!h) return;
  cudaSetDevice(h->P.device);
  if (h->st) cudaStreamSynchronize(h->st);
  if (h->st2_own) cudaStreamSynchronize(h->st2_own);
  invalidate_graphs(h);
  free_fast(h->fb);
  dfree(h->fb.queue); dfree(h->fb.qn); dfree(h->fb.bcnt); dfree(h->fb.bucket); dfree(h->fb.border);
  dfree(h->fb.arng);
  if (h->rec) cudaFree(h->rec);
  for (float4** q : {&h->sf.pos, &h->sf.vel, &h->sf.pos2, &h->sf.vel2}) dfree(*q);
  dfree(h->sf.pid); dfree(h->sf.pid2);
  for (cudaEvent_t e : {h->ev_snap, h->ev_mem, h->ev_coll, h->ev_str[0], h->ev_str[1], h->ev_vbin, h->ev_health})
    if (e) cudaEventDestroy(e);
  dfree(h->health);
  if (h->health_host) cudaFreeHost(h->health_host);
  if (h->st2_own) cudaStreamDestroy(h->st2_own);
  Solvent& s = h->s;
  Cells& c = h->c;
  for (double** q : {&s.x, &s.y, &s.z, &s.x2, &s.y2, &s.z2}) dfree(*q);
  dfree(s.v);
  dfree(s.v2);
  for (int** q : {&s.indio, &s.pid, &s.indio2, &s.pid2, &s.key, &s.slot, &s.perm}) dfree(*q);
  for (int** q : {&c.cnt, &c.ncm, &c.wrank, &c.mrank, &c.lcnt, &c.lrank, &c.acell, &c.start, &c.lstart,
                  &c.lstart2, &c.totals,
                  &c.scan_part, &c.lidx, &c.lidx2})
    dfree(*q);
  free_membrane(h->m);
  dfree(h->m.ligi); dfree(h->m.xlig); dfree(h->m.ylig); dfree(h->ebase); dfree(h->m.sc); dfree(h->obs);
  for (cudaEvent_t e : h->ev_pool) cudaEventDestroy(e);
  if (h->ev_begin) cudaEventDestroy(h->ev_begin);
  if (h->ev_end) cudaEventDestroy(h->ev_end);
  if (h->st) cudaStreamDestroy(h->st);
  delete h;
}

extern "C" const char* irbc_last_error(const irbc_handle* h) { return h ? h->err.c_str() : g_create_err.c_str(); }
extern "C" int64_t irbc_ncell(const irbc_handle* h) { return h ? h->dp.ncell : -1; }
extern "C" int32_t irbc_nlig(const irbc_handle* h) { return h ? h->dp.nlig : -1; }
extern "C" int64_t irbc_launch_count(const irbc_handle* h) { return h ? launches_in(h) : -1; }
// the health word after everything queued so far; IRBC_ERR_HEALTH when set
static int check_health(irbc_handle* h) {
  CK(cudaMemcpyAsync(h->health_host, h->health, sizeof(int), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  return health_status(h, *h->health_host);
}

extern "C" int irbc_sync(irbc_handle* h) {
  if (!h) return IRBC_ERR_ARG;
  cudaSetDevice(h->P.device);
  CK(cudaStreamSynchronize(h->st));
  return check_health(h);
}

extern "C" int irbc_health(irbc_handle* h, int32_t* flags) {
  if (!h) return IRBC_ERR_ARG;
  cudaSetDevice(h->P.device);
  const int rc = check_health(h);
  if (flags) *flags = *h->health_host;
  return rc == IRBC_ERR_HEALTH ? 0 : rc;
}

// ---- llist -----------------------------------------------------------------
// ranks of the cells with a list, and room for them in the near-membrane
// streaming buckets
static int refresh_listed(irbc_handle* h) {
  Cells& c = h->c;
  const int k = launch_llist_ranks(h->dp, c, h->st);
  if (k < 0) return fail(h, IRBC_ERR_CUDA, cudaGetErrorString(cudaGetLastError()));
  g_launches += k;
  FastBufs& f = h->fb;
  if (c.nact > f.bcap) {
    invalidate_graphs(h);  // the buckets move
    dfree(f.bcnt);
    dfree(f.bucket);
    dfree(f.border);
    dfree(f.arng);
    f.bcap = c.nact + c.nact / 2 + 64;
    CK(dalloc(&f.bcnt, f.bcap));
    CK(dalloc(&f.bucket, f.bcap * kBucket));
    CK(dalloc(&f.border, f.bcap));
    CK(dalloc(&f.arng, f.bcap));
    CK(cudaMemsetAsync(f.bcnt, 0, sizeof(int) * f.bcap, h->st));
  }
  // the near-membrane streaming takes the listed cells longest list first,
  // so that the heaviest blocks do not start last (order of work only)
  if (c.nact > 0) {
    std::vector<int> len(c.nact), order(c.nact);
    launch_rank_lengths(c, f.border, f.arng, h->st);
    g_launches += 1;
    CK(cudaMemcpyAsync(len.data(), f.border, sizeof(int) * c.nact, cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    for (int a = 0; a < c.nact; ++a) order[a] = a;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return len[x] > len[y]; });
    CK(cudaMemcpyAsync(f.border, order.data(), sizeof(int) * c.nact, cudaMemcpyHostToDevice, h->st));
    CK(cudaStreamSynchronize(h->st));
  }
  return 0;
}

static int do_llist(irbc_handle* h) {
  Cells& c = h->c;
  int64_t need = launch_llist_count(h->dp, c, h->m, h->st);
  g_launches += 3 + 3;
  if (need > c.lcap2) {
    dfree(c.lidx2);
    c.lcap2 = need + need / 4 + 1024;
    CK(dalloc(&c.lidx2, c.lcap2));
  }
  if (need > c.lcap) {
    // the live list moves: grow it keeping its entries (the stale tails)
    invalidate_graphs(h);
    int* grown = nullptr;
    const int64_t cap = need + need / 4 + 1024;
    CK(dalloc(&grown, cap));
    CK(cudaMemcpyAsync(grown, c.lidx, sizeof(int) * c.lcap, cudaMemcpyDeviceToDevice, h->st));
    CK(cudaStreamSynchronize(h->st));
    dfree(c.lidx);
    c.lidx = grown;
    c.lcap = cap;
  }
  launch_llist_fill(h->dp, c, h->m, need, h->st);
  g_launches += 1;
  CK(cudaGetLastError());
  return refresh_listed(h);
}

extern "C" int irbc_llist_update(irbc_handle* h) {
  if (!h) return IRBC_ERR_ARG;
  if (!h->have_mesh) return fail(h, IRBC_ERR_STATE, "no mesh");
  return do_llist(h);
}

// ---- set-up ------------------------------------------------------------------
extern "C" int irbc_init(irbc_handle* h, const double* V, int32_t nv, const int32_t* E, int32_t ne,
                         const int32_t* T, int32_t nt, int32_t nknobs) {
  if (!h || !V || !E || !T || nv <= 0 || ne <= 0 || nt <= 0) return IRBC_ERR_ARG;
  if (nknobs < 0 || nknobs > nv) return fail(h, IRBC_ERR_ARG, "knob count must be in [0, nv]");
  for (int i = 0; i < 2 * ne; ++i) if (E[i] < 0 || E[i] >= nv) return fail(h, IRBC_ERR_ARG, "edge index out of range");
  for (int i = 0; i < 3 * nt; ++i) if (T[i] < 0 || T[i] >= nv) return fail(h, IRBC_ERR_ARG, "triangle index out of range");
  cudaSetDevice(h->P.device);
  const irbc_params& p = h->P;
  const uint64_t seed = p.seed;
  uint64_t k = 6 * (uint64_t)p.Ns;  // INIT draws after the solvent's
  auto U = [&]() { return draw_uniform(seed, STREAM_INIT, 0, k++); };
  // solvent (maincode.cpp:96-107) on the device
  launch_init_solvent(h->dp, h->s, h->st);
  g_launches += 1;
  HostMesh M;
  M.nv = nv; M.ne = ne; M.nt = nt;
  M.x.resize(nv); M.y.resize(nv); M.z.resize(nv); M.vx.resize(nv); M.vy.resize(nv); M.vz.resize(nv);
  M.ix.assign(nv, 0); M.iy.assign(nv, 0);
  // vertices (maincode.cpp:171-206)
  double vmax = sqrt(3.0 * p.Theta / (p.pmass));
  std::vector<double> zcrds;
  for (int i = 0; i < nv; ++i) {
    zcrds.push_back(V[3 * i + 2]);
    M.x[i] = V[3 * i]; M.y[i] = V[3 * i + 1]; M.z[i] = V[3 * i + 2];
    M.vx[i] = -vmax + 2.0 * vmax * U();
    M.vy[i] = -vmax + 2.0 * vmax * U();
    M.vz[i] = -vmax + 2.0 * vmax * U();
  }
  std::sort(zcrds.begin(), zcrds.end());
  double Center[3];
  Center[2] = -zcrds.front() + 0.3;
  Center[0] = p.Lx / 2.0 + 10.0;
  Center[1] = p.Ly / 2.0;
  for (int i = 0; i < nv; ++i) { M.x[i] += Center[0]; M.y[i] += Center[1]; M.z[i] += Center[2]; }
  double numer = 1.73205080757 * ((double)nv - 2.0) - 5.0 * p.Pi;
  double denom = 1.73205080757 * ((double)nv - 2.0) - 3.0 * p.Pi;
  M.theta0 = 180.0 * acos(numer / denom) / p.Pi;
  // parasite (maincode.cpp:212-225)
  MemScalars sc{};
  sc.para[0] = Center[0] - 2.0; sc.para[1] = Center[1]; sc.para[2] = Center[2];
  vmax = sqrt(3.0 * p.Theta / (p.PRmass));
  for (int q = 0; q < 3; ++q) sc.paraV[q] = -vmax + 2.0 * vmax * U();
  // edges (maincode.cpp:239-257)
  M.e1.resize(ne); M.e2.resize(ne); M.l0.resize(ne); M.kappap.resize(ne);
  double meanedge = 0, meanedge2 = 0;
  for (int i = 0; i < ne; ++i) {
    int a1 = E[2 * i], a2 = E[2 * i + 1];
    M.e1[i] = a1; M.e2[i] = a2;
    double distx = (M.x[a1] - M.x[a2]) * (M.x[a1] - M.x[a2]);
    double disty = (M.y[a1] - M.y[a2]) * (M.y[a1] - M.y[a2]);
    double distz = (M.z[a1] - M.z[a2]) * (M.z[a1] - M.z[a2]);
    M.l0[i] = sqrt(distx + disty + distz);
    meanedge += M.l0[i];
    meanedge2 += M.l0[i] * M.l0[i];
  }
  h->report[0] = meanedge / (double)ne;
  h->report[1] = sqrt((meanedge2 / (double)ne) - ((meanedge / (double)ne) * (meanedge / (double)ne)));
  M.t1.resize(nt); M.t2.resize(nt); M.t3.resize(nt);
  for (int i = 0; i < nt; ++i) { M.t1[i] = T[3 * i]; M.t2[i] = T[3 * i + 1]; M.t3[i] = T[3 * i + 2]; }
  build_edgest(M);
  // TotalVA0 (Src/memfuncs.cpp:192-211)
  {
    double totA = 0, totV = 0;
    for (int i = 0; i < nt; ++i) {
      totA += h_areatri(M, p.Lx, p.Ly, M.t1[i], M.t2[i], M.t3[i]);
      totV += h_voltri(M, p.Lx, p.Ly, M.t1[i], M.t2[i], M.t3[i]);
    }
    M.Sarea0 = totA; M.Volume0 = totV;
  }
  // kappap (maincode.cpp:347-361)
  for (int i = 0; i < ne; ++i) {
    double ll0 = M.l0[i], lmax = 2.5 * ll0, x0 = ll0 / lmax, onemx0 = 1.0 - x0;
    double shear1 = 1.0 / (4.0 * onemx0 * onemx0);
    double shear2 = x0 / (2.0 * onemx0 * onemx0 * onemx0);
    double shear4 = (1.732 / (4.0 * p.elap * lmax * x0));
    double sh = shear4 * shear2 - shear4 * shear1 + shear4 * 0.25;
    M.kappap[i] = (p.shear - sh) * 4.0 * ll0 * ll0 * ll0 / (3.0 * 1.732);
  }
  double areaC = 2.0 * p.shear + p.kappasa + p.kappad;
  h->report[2] = M.Sarea0; h->report[3] = M.Volume0; h->report[4] = p.shear;
  h->report[5] = (4.0 * areaC * p.shear) / (areaC + p.shear);
  h->report[6] = (areaC - p.shear) / (areaC + p.shear);
  h->report[8] = M.theta0;
  M.tarea.resize(nt);
  for (int i = 0; i < nt; ++i) M.tarea[i] = h_areatri(M, p.Lx, p.Ly, M.t1[i], M.t2[i], M.t3[i]);
  build_iedge(M, p.Lx, p.Ly, p.Lz);
  int rc = upload_mesh(h, M);
  if (rc) return rc;
  Membrane& m = h->m;
  std::vector<int> zeros(nv, 0), randno(nv, p.randno);
  std::vector<double> dz(nv, 0.0);
  if (up(h, m.x, M.x) || up(h, m.y, M.y) || up(h, m.z, M.z) || up(h, m.vx, M.vx) || up(h, m.vy, M.vy) ||
      up(h, m.vz, M.vz) || up(h, m.ix, zeros) || up(h, m.iy, zeros) || up(h, m.pid, zeros) ||
      up(h, m.bondi, zeros) || up(h, m.bondl, randno) || up(h, m.knob, zeros) || up(h, m.fx, dz) ||
      up(h, m.fy, dz) || up(h, m.fz, dz) || up(h, m.poff, dz) || up(h, m.pon, dz))
    return IRBC_ERR_CUDA;
  CK(cudaMemcpyAsync(m.sc, &sc, sizeof(sc), cudaMemcpyHostToDevice, h->st));
  CK(cudaMemsetAsync(m.ligi, 0, sizeof(int) * h->dp.nlig, h->st));
  // TotalVA, pfdt, force_calculate_dt (maincode.cpp:385-387)
  launch_total_va(h->dp, m, h->st);
  launch_pfdt_forces(h->dp, m, 1, 1, 0, h->st);
  g_launches += 4;
  // inside/outside and the reference's sort permutation (Src/solfuncs.cpp:17-106)
  launch_classify(h->dp, h->s, m, h->st);
  g_launches += 2;
  if (p.Ns > 0) {
    std::vector<int> indio(p.Ns);
    if (down(h, indio.data(), h->s.indio, p.Ns)) return IRBC_ERR_CUDA;
    CK(cudaStreamSynchronize(h->st));
    struct K { int indio; int idx; bool operator<(const K& r) const { return indio < r.indio; } };
    std::vector<K> keys(p.Ns);
    for (int64_t i = 0; i < p.Ns; ++i) keys[i] = {indio[i], (int)i};
    std::sort(keys.begin(), keys.end());
    std::vector<int> id(p.Ns);
    for (int64_t r = 0; r < p.Ns; ++r) id[keys[r].idx] = (int)r;
    // reference indices into the velocity records (key is free between collisions)
    if (up(h, h->s.key, id)) return IRBC_ERR_CUDA;
    launch_pack_vel(h->s, nullptr, nullptr, nullptr, h->s.key, h->st);
    g_launches += 1;
  }
  // llistupdate (maincode.cpp:391) on empty lists
  CK(cudaMemsetAsync(h->c.lstart, 0, sizeof(int) * (h->c.n + 1), h->st));
  rc = do_llist(h);
  if (rc) return rc;
  // knobs (maincode.cpp:394-433): sequential draws on the host
  std::vector<int> knob(nv, 0);
  {
    std::vector<double> parea;
    for (int i = 0; i < nt; ++i) parea.push_back(M.tarea[i] / M.Sarea0);
    int knob_count = 0;
    while (knob_count < nknobs) {
      double rad = U();
      double aaa = 0;
      for (int j = 0; j < nt; ++j) {
        aaa += parea[j];
        if (aaa > rad) {
          // IRandom(1,3) (Src/mersenne.cpp:115-125)
          int radi = int((double)(uint32_t)(3 - 1 + 1) * U() + 1);
          if (radi > 3) radi = 3;
          if ((radi == 1) && (knob[M.t1[j]] == 0)) { knob[M.t1[j]] = 1; knob_count += 1; break; }
          else if ((radi == 2) && (knob[M.t2[j]] == 0)) { knob[M.t2[j]] = 1; knob_count += 1; break; }
          else if ((radi == 3) && (knob[M.t3[j]] == 0)) { knob[M.t3[j]] = 1; knob_count += 1; break; }
        }
      }
    }
    h->report[7] = knob_count;
  }
  if (up(h, m.knob, knob)) return IRBC_ERR_CUDA;
  h->step = 0; h->colsteps = -1; h->upd = 0; h->filecc = 0; h->filec = 0; h->bbi = 0;
  if (h->fp32) f32_from_f64(h->s, h->sf, h->st);
  CK(cudaStreamSynchronize(h->st));
  CK(cudaGetLastError());
  return 0;
}

extern "C" int irbc_init_report(const irbc_handle* h, double out[9]) {
  if (!h || !out) return IRBC_ERR_ARG;
  for (int k = 0; k < 9; ++k) out[k] = h->report[k];
  return 0;
}

// ---- mesh / state exchange ---------------------------------------------------
extern "C" int irbc_set_mesh(irbc_handle* h, const irbc_mesh* mm) {
  if (!h || !mm || mm->nv <= 0) return IRBC_ERR_ARG;
  cudaSetDevice(h->P.device);
  HostMesh M;
  M.nv = mm->nv; M.ne = mm->ne; M.nt = mm->nt;
  M.e1.assign(mm->e1, mm->e1 + mm->ne); M.e2.assign(mm->e2, mm->e2 + mm->ne);
  M.es1.assign(mm->es1, mm->es1 + mm->ne); M.es2.assign(mm->es2, mm->es2 + mm->ne);
  M.iedge.assign(mm->iedge, mm->iedge + mm->ne);
  M.l0.assign(mm->l0, mm->l0 + mm->ne); M.kappap.assign(mm->kappap, mm->kappap + mm->ne);
  M.t1.assign(mm->t1, mm->t1 + mm->nt); M.t2.assign(mm->t2, mm->t2 + mm->nt); M.t3.assign(mm->t3, mm->t3 + mm->nt);
  M.tarea.assign(mm->tarea, mm->tarea + mm->nt);
  M.Sarea0 = mm->Sarea0; M.Volume0 = mm->Volume0; M.theta0 = mm->theta0;
  for (int k = 0; k < 3; ++k) M.center[k] = mm->center[k];
  return upload_mesh(h, M);
}

extern "C" int irbc_get_mesh(irbc_handle* h, irbc_mesh* mm) {
  if (!h || !mm) return IRBC_ERR_ARG;
  if (!h->have_mesh) return fail(h, IRBC_ERR_STATE, "no mesh");
  const Membrane& m = h->m;
  mm->nv = m.nv; mm->ne = m.ne; mm->nt = m.nt;
  if (mm->e1) {
    if (down(h, mm->e1, m.e1, m.ne) || down(h, mm->e2, m.e2, m.ne) || down(h, mm->l0, m.l0, m.ne) ||
        down(h, mm->kappap, m.kappap, m.ne) || down(h, mm->es1, m.es1, m.ne) || down(h, mm->es2, m.es2, m.ne) ||
        down(h, mm->iedge, m.iedge, m.ne))
      return IRBC_ERR_CUDA;
  }
  if (mm->t1) {
    if (down(h, mm->t1, m.t1, m.nt) || down(h, mm->t2, m.t2, m.nt) || down(h, mm->t3, m.t3, m.nt) ||
        down(h, mm->tarea, m.tarea, m.nt))
      return IRBC_ERR_CUDA;
  }
  mm->Sarea0 = h->dp.Sarea0; mm->Volume0 = h->dp.Volume0; mm->theta0 = h->dp.theta0;
  CK(cudaStreamSynchronize(h->st));
  return 0;
}

extern "C" int irbc_set_state(irbc_handle* h, const irbc_view* v) {
  if (!h || !v) return IRBC_ERR_ARG;
  if (!h->have_mesh) return fail(h, IRBC_ERR_STATE, "set the mesh first");
  if (v->ns != h->s.n) return fail(h, IRBC_ERR_ARG, "solvent count differs from Ns");
  if (v->nv != h->m.nv) return fail(h, IRBC_ERR_ARG, "vertex count differs from the mesh");
  if (v->ncell != h->dp.ncell || v->nlig != h->dp.nlig) return fail(h, IRBC_ERR_ARG, "grid size differs");
  cudaSetDevice(h->P.device);
  Solvent& s = h->s;
  Membrane& m = h->m;
  const int64_t n = s.n;
  if (v->sx) {
    // velocities go through the free second position set into the velocity
    // records, with the reference index (the array position) made on the
    // device
    if (up(h, s.x, v->sx, n) || up(h, s.y, v->sy, n) || up(h, s.z, v->sz, n) || up(h, s.x2, v->svx, n) ||
        up(h, s.y2, v->svy, n) || up(h, s.z2, v->svz, n) || up(h, s.pid, v->spid, n) ||
        up(h, s.indio, v->sindio, n))
      return IRBC_ERR_CUDA;
    launch_iota(s.key, n, h->st);
    launch_pack_vel(s, s.x2, s.y2, s.z2, s.key, h->st);
    g_launches += 2;
    if (h->fp32) f32_from_f64(h->s, h->sf, h->st);
    CK(cudaStreamSynchronize(h->st));
  }
  const int nv = m.nv;
  if (v->x) {
    if (up(h, m.x, v->x, nv) || up(h, m.y, v->y, nv) || up(h, m.z, v->z, nv) || up(h, m.vx, v->vx, nv) ||
        up(h, m.vy, v->vy, nv) || up(h, m.vz, v->vz, nv) || up(h, m.fx, v->fx, nv) || up(h, m.fy, v->fy, nv) ||
        up(h, m.fz, v->fz, nv) || up(h, m.poff, v->poff, nv) || up(h, m.pon, v->pon, nv) ||
        up(h, m.pid, v->pid, nv) || up(h, m.ix, v->ix, nv) || up(h, m.iy, v->iy, nv) ||
        up(h, m.bondi, v->bondi, nv) || up(h, m.bondl, v->bondl, nv) || up(h, m.knob, v->knob, nv))
      return IRBC_ERR_CUDA;
  }
  MemScalars sc{};
  for (int k = 0; k < 3; ++k) {
    sc.para[k] = v->para[k]; sc.paraV[k] = v->paraV[k]; sc.paraft[k] = v->paraft[k]; sc.parafdt[k] = v->parafdt[k];
  }
  sc.paradx = v->paradx; sc.parady = v->parady; sc.paraid = v->paraid;
  sc.Sarea = v->Sarea; sc.Volume = v->Volume;
  CK(cudaMemcpyAsync(m.sc, &sc, sizeof(sc), cudaMemcpyHostToDevice, h->st));
  if (v->ligi && up(h, m.ligi, v->ligi, h->dp.nlig)) return IRBC_ERR_CUDA;
  if (v->llen) {
    Cells& c = h->c;
    int64_t tot = 0;
    for (int64_t i = 0; i < c.n; ++i) tot += v->llen[i];
    if (tot >= (1LL << 31)) return fail(h, IRBC_ERR_ARG, "list entries exceed the int range");
    if (tot > c.lcap) {
      CK(cudaStreamSynchronize(h->st));
      invalidate_graphs(h);
      dfree(c.lidx);
      c.lcap = tot + 1024;
      CK(dalloc(&c.lidx, c.lcap));
    }
    // list starts: the lengths scanned on the device
    if (up(h, c.lcnt, v->llen, c.n) || up(h, c.lidx, v->lidx, tot)) return IRBC_ERR_CUDA;
    launch_scan3(c.lcnt, nullptr, nullptr, c.lstart, nullptr, nullptr, c.totals + 8, c.n, c.scan_part, h->st);
    CK(cudaMemcpyAsync(c.lstart + c.n, c.totals + 8, sizeof(int), cudaMemcpyDeviceToDevice, h->st));
    g_launches += 3;
    int rc = refresh_listed(h);
    if (rc) return rc;
  }
  h->dp.wallspeed = v->wallspeed;
  h->step = v->step; h->colsteps = v->colsteps; h->upd = v->upd; h->filecc = v->filecc; h->filec = v->filec;
  CK(clear_health(h));
  CK(cudaStreamSynchronize(h->st));
  return 0;
}

extern "C" int64_t irbc_llist_total(irbc_handle* h) {
  if (!h) return IRBC_ERR_ARG;
  cudaSetDevice(h->P.device);
  int t = 0;
  // on the handle's stream: after the list update that wrote the total
  if (cudaMemcpyAsync(&t, h->c.lstart + h->c.n, sizeof(int), cudaMemcpyDeviceToHost, h->st) != cudaSuccess ||
      cudaStreamSynchronize(h->st) != cudaSuccess)
    return IRBC_ERR_CUDA;
  return t;
}

extern "C" int irbc_get_state(irbc_handle* h, irbc_view* v) {
  if (!h || !v) return IRBC_ERR_ARG;
  cudaSetDevice(h->P.device);
  Solvent& s = h->s;
  Membrane& m = h->m;
  v->ns = s.n; v->nv = m.nv; v->ncell = h->dp.ncell; v->nlig = h->dp.nlig;
  if (h->fp32 && v->sx) f32_to_f64(h->sf, h->s, h->st);
  CK(cudaStreamSynchronize(h->st));
  const int64_t n = s.n;
  if (v->sx && n) {
    // un-permuted on the device into the second buffer set, then copied
    // straight into the caller's arrays
    int* bad = h->c.totals + 11;
    CK(cudaMemsetAsync(bad, 0, sizeof(int), h->st));
    launch_unpermute(s, 0, bad, h->st);
    g_launches += 1;
    if (down(h, v->sx, s.x2, n) || down(h, v->sy, s.y2, n) || down(h, v->sz, s.z2, n) ||
        down(h, v->spid, s.pid2, n) || down(h, v->sindio, s.indio2, n))
      return IRBC_ERR_CUDA;
    launch_unpermute(s, 1, bad, h->st);
    g_launches += 1;
    if (down(h, v->svx, s.x2, n) || down(h, v->svy, s.y2, n) || down(h, v->svz, s.z2, n)) return IRBC_ERR_CUDA;
    int nbad = 0;
    CK(cudaMemcpyAsync(&nbad, bad, sizeof(int), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    if (nbad) return fail(h, IRBC_ERR_STATE, "corrupt particle ids");
  }
  const int nv = m.nv;
  if (v->x && nv) {
    if (down(h, v->x, m.x, nv) || down(h, v->y, m.y, nv) || down(h, v->z, m.z, nv) || down(h, v->vx, m.vx, nv) ||
        down(h, v->vy, m.vy, nv) || down(h, v->vz, m.vz, nv) || down(h, v->fx, m.fx, nv) ||
        down(h, v->fy, m.fy, nv) || down(h, v->fz, m.fz, nv) || down(h, v->poff, m.poff, nv) ||
        down(h, v->pon, m.pon, nv) || down(h, v->pid, m.pid, nv) || down(h, v->ix, m.ix, nv) ||
        down(h, v->iy, m.iy, nv) || down(h, v->bondi, m.bondi, nv) || down(h, v->bondl, m.bondl, nv) ||
        down(h, v->knob, m.knob, nv))
      return IRBC_ERR_CUDA;
  }
  MemScalars sc{};
  CK(cudaMemcpyAsync(&sc, m.sc, sizeof(sc), cudaMemcpyDeviceToHost, h->st));
  if (v->ligi && down(h, v->ligi, m.ligi, h->dp.nlig)) return IRBC_ERR_CUDA;
  CK(cudaStreamSynchronize(h->st));
  for (int k = 0; k < 3; ++k) {
    v->para[k] = sc.para[k]; v->paraV[k] = sc.paraV[k]; v->paraft[k] = sc.paraft[k]; v->parafdt[k] = sc.parafdt[k];
  }
  v->paradx = sc.paradx; v->parady = sc.parady; v->paraid = sc.paraid;
  v->Sarea = sc.Sarea; v->Volume = sc.Volume; v->wallspeed = h->dp.wallspeed;
  if (v->llen) {
    Cells& c = h->c;
    std::vector<int> start(c.n + 1);
    if (down(h, start.data(), c.lstart, c.n + 1)) return IRBC_ERR_CUDA;
    CK(cudaStreamSynchronize(h->st));
    for (int64_t i = 0; i < c.n; ++i) v->llen[i] = start[i + 1] - start[i];
    if (v->lidx) {
      if (start[c.n] > v->lcap) return fail(h, IRBC_ERR_CAPACITY, "lidx capacity too small");
      if (down(h, v->lidx, c.lidx, start[c.n])) return IRBC_ERR_CUDA;
    }
  }
  v->step = h->step; v->colsteps = h->colsteps; v->upd = h->upd; v->filecc = h->filecc; v->filec = h->filec;
  CK(cudaStreamSynchronize(h->st));
  return 0;
}

// ---- phases --------------------------------------------------------------------
extern "C" int irbc_collide(irbc_handle* h, int64_t epoch) {
  if (!h) return IRBC_ERR_ARG;
  if (!h->have_mesh) return fail(h, IRBC_ERR_STATE, "no mesh");
  CK(set_epoch_base(h, (uint64_t)epoch));
  g_launches += collide_any(h, 0, h->st);
  CK(cudaGetLastError());
  return 0;
}
extern "C" int irbc_stream(irbc_handle* h) {
  if (!h || !h->have_mesh) return IRBC_ERR_ARG;
  fast_snap_prep(h->dp, h->m, h->fb, 0, h->st);
  g_launches += 2 + stream_any(h, 0, h->st);
  h->snap_ready = false;
  CK(cudaGetLastError());
  return 0;
}
extern "C" int irbc_total_va(irbc_handle* h) {
  if (!h || !h->have_mesh) return IRBC_ERR_ARG;
  launch_total_va(h->dp, h->m, h->st);
  g_launches += 2;
  CK(cudaGetLastError());
  return 0;
}
extern "C" int irbc_pfdt(irbc_handle* h) {
  if (!h || !h->have_mesh) return IRBC_ERR_ARG;
  launch_pfdt_forces(h->dp, h->m, 1, 0, 0, h->st);
  g_launches += 2;
  CK(cudaGetLastError());
  return 0;
}
extern "C" int irbc_forces(irbc_handle* h) {
  if (!h || !h->have_mesh) return IRBC_ERR_ARG;
  launch_pfdt_forces(h->dp, h->m, 0, 1, 0, h->st);
  g_launches += 1;
  CK(cudaGetLastError());
  return 0;
}
extern "C" int irbc_bond_dynamics(irbc_handle* h, int64_t epoch) {
  if (!h || !h->have_mesh) return IRBC_ERR_ARG;
  CK(set_epoch_base(h, (uint64_t)epoch));
  launch_bonds(h->dp, h->m, 0, h->st);
  g_launches += 2;
  CK(cudaGetLastError());
  return 0;
}

// maincode.cpp:462-602
extern "C" int irbc_step_part1(irbc_handle* h) {
  if (!h) return IRBC_ERR_ARG;
  if (!h->have_mesh) return fail(h, IRBC_ERR_STATE, "no mesh");
  const irbc_params& p = h->P;
  const int64_t s = h->step;
  h->dp.wallspeed = (s < p.warm_steps) ? p.warm_speed : p.walls;
  h->colsteps += 1; h->bbi += 1; h->upd += 1;
  if (s > 0) h->filecc += 1;
  CK(set_epoch_base(h, (uint64_t)s));
  if (h->colsteps == h->csteps) {
    ProfScope ps(h, PROF_COLLIDE);
    g_launches += collide_any(h, 0, h->st);
    h->colsteps = 0;
  }
  const int buf = (int)(s & 1);
  {
    ProfScope ps(h, PROF_MEMBRANE);
    g_launches += fast_kick_prep(h->dp, h->m, h->fb, buf, h->st);
  }
  if (h->upd == h->uplist) {
    int rc = do_llist(h);
    if (rc) return rc;
    h->upd = 0;
  }
  {
    ProfScope ps(h, PROF_STREAM);
    g_launches += stream_any(h, buf, h->st);
  }
  {
    ProfScope ps(h, PROF_MEMBRANE);
    g_launches += fast_drift_va(h->dp, h->m, h->st, true);
  }
  h->snap_ready = false;
  CK(cudaGetLastError());
  return 0;
}

// maincode.cpp:603-762
extern "C" int irbc_step_part2(irbc_handle* h) {
  if (!h) return IRBC_ERR_ARG;
  if (!h->have_mesh) return fail(h, IRBC_ERR_STATE, "no mesh");
  const int64_t s = h->step;
  CK(set_epoch_base(h, (uint64_t)s));
  {
    ProfScope ps(h, PROF_MEMBRANE);
    g_launches += fast_forces_tail(h->dp, h->m, h->fb, 0, 0, (int)((s + 1) & 1), h->st, false);
  }
  if (h->filecc == h->P.out_every) { h->filec += 1; h->filecc = 0; }
  h->step = s + 1;
  CK(cudaGetLastError());
  return 0;
}

// One timestep of the pipelined schedule: step s streams the solvent
// (h->st) while the membrane drifts, computes forces and bonds for s and
// prepares the snapshot of s+1 (h->st2).  Collisions, llist updates and the
// snapshot buffers (two, by step parity) are ordered by events.  eoff is the
// step's draw-epoch offset from the current base; last: the step ends a
// call or a captured sequence (the next step's half-kick is not fused into
// this one).  dry: advance the host counters only (the launches are in a
// captured sequence being replayed).
static int step_one(irbc_handle* h, int64_t eoff, bool last, bool dry) {
  const irbc_params& p = h->P;
  cudaStream_t ms = h->st, ss = h->st2;
  const int64_t s = h->step;
  h->dp.wallspeed = (s < p.warm_steps) ? p.warm_speed : p.walls;
  h->colsteps += 1; h->bbi += 1; h->upd += 1;
  if (s > 0) h->filecc += 1;
  const int buf = (int)(s & 1);
  if (h->colsteps == h->csteps) {
    if (dry) {
      h->s.ncoll += 1;
    } else {
      {
        ProfScope ps(h, PROF_COLLIDE, ms);
        g_launches += collide_any(h, (uint64_t)eoff, ms, ss);
      }
      CK(cudaEventRecord(h->ev_coll, ms));
      CK(cudaStreamWaitEvent(ss, h->ev_coll, 0));
    }
    h->colsteps = 0;
    h->snap_ready = false;
  }
  if (!h->snap_ready && !dry) {
    CK(cudaStreamWaitEvent(ss, h->ev_str[buf], 0));
    ProfScope ps(h, PROF_MEMBRANE, ss);
    g_launches += fast_kick_prep(h->dp, h->m, h->fb, buf, ss);
  }
  if (h->upd == h->uplist) {
    // never inside a captured sequence.  Positions of step s are final once
    // the side stream reaches here; its drift of step s waits for the update
    CK(cudaEventRecord(h->ev_snap, ss));
    CK(cudaStreamWaitEvent(ms, h->ev_snap, 0));
    int rc = do_llist(h);
    if (rc) return rc;
    h->upd = 0;
    CK(cudaEventRecord(h->ev_coll, ms));
    CK(cudaStreamWaitEvent(ss, h->ev_coll, 0));
  }
  // the next step's snapshot goes to the other buffer, read by the
  // previous step's streaming
  const bool next_collides = (h->colsteps + 1 == h->csteps);
  const int next_kick = (!last && !next_collides) ? 1 : 0;
  if (!dry) {
    // The streams meet only where they share data.  The bulk streaming
    // kernel reads no membrane data and starts at once; the near-membrane
    // kernel waits for the snapshot `buf` (ev_snap: the side stream so far).
    // The membrane step runs on, and only its writing of the next snapshot
    // (buf ^ 1) waits for the streaming that last read that buffer.
    CK(cudaEventRecord(h->ev_snap, ss));
    {
      ProfScope ps(h, PROF_STREAM, ms);
      g_launches += stream_any(h, buf, ms, h->ev_snap);
    }
    CK(cudaEventRecord(h->ev_str[buf], ms));
    {
      ProfScope ps(h, PROF_MEMBRANE, ss);
      g_launches += fast_membrane_step(h->dp, h->m, h->fb, (uint64_t)eoff, next_kick, buf ^ 1, ss,
                                       h->ev_str[buf ^ 1]);
    }
    CK(cudaEventRecord(h->ev_mem, ss));
  }
  h->snap_ready = next_kick != 0;
  if (h->filecc == p.out_every) { h->filec += 1; h->filecc = 0; }
  h->step = s + 1;
  return 0;
}

constexpr int kGraphSteps = 24;  // two collision cycles per captured sequence

// records every stream-ordering event on the main stream: after a capture
// (whose records belong to the graph) and after each graph launch, so that
// later waits refer to work outside any graph and follow the launch
static cudaError_t rearm_events(irbc_handle* h) {
  for (cudaEvent_t e : {h->ev_str[0], h->ev_str[1], h->ev_snap, h->ev_mem, h->ev_coll, h->ev_vbin}) {
    cudaError_t r = cudaEventRecord(e, h->st);
    if (r != cudaSuccess) return r;
  }
  return cudaSuccess;
}

// a captured sequence can stand for the next kGraphSteps steps when no list
// update falls inside them, the wall speed is the same throughout, and the
// previous step did not fuse this step's half-kick
static bool graph_fits(const irbc_handle* h, int64_t remaining) {
  if (!h->graphs_on || remaining < kGraphSteps || h->snap_ready) return false;
  if (h->upd + kGraphSteps >= h->uplist) return false;
  const int64_t s = h->step, w = h->P.warm_steps;
  return (s + kGraphSteps <= w) || (s >= w);
}

// the kGraphSteps steps from the current configuration, captured once; the
// host counters are left where they were
static irbc_handle::StepGraph* graph_for(irbc_handle* h) {
  const double ws = (h->step < h->P.warm_steps) ? h->P.warm_speed : h->P.walls;
  const int parity = (int)(h->step & 1);
  for (auto& g : h->graphs)
    if (g.colsteps0 == h->colsteps && g.parity == parity && g.wallspeed == ws) return &g;
  cudaStream_t ms = h->st, ss = h->st2;
  // counters to restore after the capture
  const int64_t step = h->step, ncoll = h->s.ncoll, resorted = h->s.resorted;
  const int colsteps = h->colsteps, bbi = h->bbi, upd = h->upd, filecc = h->filecc, filec = h->filec;
  const bool snap = h->snap_ready;
  const double wsp = h->dp.wallspeed;
  const int64_t l0 = g_launches.load();
  h->capturing = true;
  cudaGraph_t graph = nullptr;
  bool ok = cudaStreamBeginCapture(ms, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
  int rc = 0;
  if (ok) {
    // every event the steps wait on is first recorded inside the capture,
    // so no wait reaches outside it; then the side stream forks off
    for (cudaEvent_t e : {h->ev_str[0], h->ev_str[1], h->ev_snap, h->ev_mem, h->ev_coll})
      ok = ok && cudaEventRecord(e, ms) == cudaSuccess;
    ok = ok && cudaStreamWaitEvent(ss, h->ev_coll, 0) == cudaSuccess;
    for (int k = 0; ok && k < kGraphSteps; ++k) {
      rc = step_one(h, k, k == kGraphSteps - 1, false);
      ok = rc == 0;
    }
    if (ok) ok = cudaStreamWaitEvent(ms, h->ev_mem, 0) == cudaSuccess;
    cudaError_t e = cudaStreamEndCapture(ms, &graph);
    ok = ok && e == cudaSuccess && graph != nullptr;
  }
  h->capturing = false;
  cudaGetLastError();
  rearm_events(h);
  const int64_t launches = g_launches.load() - l0;
  const int64_t collisions = h->s.ncoll - ncoll;
  g_launches -= launches;
  h->step = step; h->s.ncoll = ncoll; h->s.resorted = resorted;
  h->colsteps = colsteps; h->bbi = bbi; h->upd = upd; h->filecc = filecc; h->filec = filec;
  h->snap_ready = snap; h->dp.wallspeed = wsp;
  if (ok) {
    // the side stream's priority does not travel into the graph by itself:
    // give the membrane chain's kernel nodes the high priority explicitly
    int lo = 0, hi = 0;
    cudaDeviceGetStreamPriorityRange(&lo, &hi);
    size_t nn = 0;
    cudaGraphGetNodes(graph, nullptr, &nn);
    std::vector<cudaGraphNode_t> nodes(nn);
    if (nn) cudaGraphGetNodes(graph, nodes.data(), &nn);
    for (cudaGraphNode_t nd : nodes) {
      cudaGraphNodeType t;
      if (cudaGraphNodeGetType(nd, &t) != cudaSuccess || t != cudaGraphNodeTypeKernel) continue;
      cudaKernelNodeParams kp{};
      if (cudaGraphKernelNodeGetParams(nd, &kp) != cudaSuccess || !is_membrane_kernel(kp.func)) continue;
      cudaKernelNodeAttrValue v{};
      v.priority = hi;
      cudaGraphKernelNodeSetAttribute(nd, cudaKernelNodeAttributePriority, &v);
    }
    cudaGetLastError();
  }
  cudaGraphExec_t exec = nullptr;
  // the kernel nodes' priorities apply only when the graph is instantiated
  // to use them
  if (ok) ok = cudaGraphInstantiateWithFlags(&exec, graph, cudaGraphInstantiateFlagUseNodePriority) == cudaSuccess;
  if (graph) cudaGraphDestroy(graph);
  cudaGetLastError();  // a refused capture leaves no sticky error
  if (!ok) {
    h->graphs_on = false;  // stay on plain launches from here on
    return nullptr;
  }
  irbc_handle::StepGraph g;
  g.exec = exec; g.colsteps0 = colsteps; g.parity = parity; g.wallspeed = ws;
  g.launches = launches; g.collisions = collisions;
  h->graphs.push_back(g);
  return &h->graphs.back();
}

// n timesteps.  Whole sequences of kGraphSteps steps are launched as one
// captured CUDA graph when they fit (graph_fits); the other steps, the list
// updates among them, are launched one by one.  Either way the launches,
// their order and their results are the same.
extern "C" int irbc_step(irbc_handle* h, int64_t n) {
  if (!h || n < 0) return IRBC_ERR_ARG;
  if (!h->have_mesh) return fail(h, IRBC_ERR_STATE, "no mesh");
  cudaSetDevice(h->P.device);
  // the health word as of the end of an earlier call, without waiting: a
  // simulation found unhealthy is not stepped further
  if (cudaEventQuery(h->ev_health) == cudaSuccess && *h->health_host) return health_status(h, *h->health_host);
  cudaStream_t ms = h->st, ss = h->st2;
  // epochs: base h->step; the side stream starts after everything already
  // queued on the main one
  CK(set_epoch_base(h, (uint64_t)h->step));
  CK(cudaEventRecord(h->ev_coll, ms));
  CK(cudaStreamWaitEvent(ss, h->ev_coll, 0));
  int64_t k = 0;
  while (k < n) {
    if (graph_fits(h, n - k)) {
      irbc_handle::StepGraph* g = graph_for(h);
      if (g) {
        // the side stream's earlier work ends before the base moves
        CK(cudaStreamWaitEvent(ms, h->ev_mem, 0));
        CK(set_epoch_base(h, (uint64_t)h->step));
        CK(cudaGraphLaunch(g->exec, ms));
        g_launches += g->launches;
        for (int j = 0; j < kGraphSteps; ++j) step_one(h, j, j == kGraphSteps - 1, true);
        if (h->s.ncoll - h->s.resorted >= kResortEvery) g_launches += resort_any(h, ms);
        CK(rearm_events(h));
        CK(cudaStreamWaitEvent(ss, h->ev_coll, 0));
        k += kGraphSteps;
        continue;
      }
    }
    // a plain step; the step before a collision never fuses the next
    // half-kick, so captured sequences start at collision steps
    int rc = step_one(h, h->step - h->ebase_val, k == n - 1, false);
    if (rc) return rc;
    k += 1;
  }
  CK(cudaStreamWaitEvent(ms, h->ev_mem, 0));
  CK(cudaMemcpyAsync(h->health_host, h->health, sizeof(int), cudaMemcpyDeviceToHost, ms));
  CK(cudaEventRecord(h->ev_health, ms));
  CK(cudaGetLastError());
  return 0;
}

extern "C" int irbc_set_streams(irbc_handle* h, int32_t n) {
  if (!h || (n != 1 && n != 2)) return IRBC_ERR_ARG;
  cudaSetDevice(h->P.device);
  CK(cudaStreamSynchronize(h->st));
  CK(cudaStreamSynchronize(h->st2_own));
  cudaStream_t want = n == 1 ? h->st : h->st2_own;
  if (want != h->st2) {
    invalidate_graphs(h);  // captured with the other stream layout
    h->st2 = want;
  }
  return 0;
}

extern "C" int irbc_set_membrane_kernels(irbc_handle* h, int32_t mode) {
  if (!h || mode < 1 || mode > 3) return IRBC_ERR_ARG;
  cudaSetDevice(h->P.device);
  CK(cudaStreamSynchronize(h->st));
  CK(cudaStreamSynchronize(h->st2_own));
  h->mem_mode = mode;
  if (h->have_mesh) {
    const bool ob = mode == 2, cl = mode == 3;
    if (ob && !one_block_fits(h->dp)) return fail(h, IRBC_ERR_CAPACITY, "mesh too large for the one-block membrane step");
    if (ob != h->fb.one_block || cl != h->fb.cluster) invalidate_graphs(h);
    h->fb.one_block = ob;
    h->fb.cluster = cl;
  }
  return 0;
}

extern "C" int irbc_set_graphs(irbc_handle* h, int32_t on) {
  if (!h) return IRBC_ERR_ARG;
  h->graphs_on = on != 0;
  if (!h->graphs_on) invalidate_graphs(h);
  return 0;
}

// ---- cohorts: one launch per phase over many simulations (cohort.h) -----------
namespace irbc {

struct Cohort {
  int device = 0;
  cudaStream_t ms = nullptr, ss = nullptr;  // solvent phases / membrane phases, as a handle's two streams
  cudaEvent_t ev_snap = nullptr, ev_mem = nullptr, ev_coll = nullptr, ev_str[2] = {nullptr, nullptr};
  cudaEvent_t ev_join = nullptr;
  MultiPlan plan;                       // device tables of `members`
  std::vector<irbc_handle*> members;    // the plan's members, in order
  std::vector<uint64_t> uids;           // their handles' unique ids
  std::vector<Member> host;             // their descriptors as uploaded
  size_t cap = 0;                       // members the device tables have room for
  size_t tab_cap = 0;                   // block-table entries they have room for
  int64_t ncoll = 0;                    // collisions of this cohort: a physical re-sort every kResortEvery
  bool ok = false;
};

Cohort* cohort_create(int device) {
  Cohort* c = new Cohort();
  c->device = device;
  if (cudaSetDevice(device) != cudaSuccess) return c;
  int lo = 0, hi = 0;
  cudaDeviceGetStreamPriorityRange(&lo, &hi);
  bool ok = cudaStreamCreateWithFlags(&c->ms, cudaStreamNonBlocking) == cudaSuccess &&
            cudaStreamCreateWithPriority(&c->ss, cudaStreamNonBlocking, hi) == cudaSuccess;
  for (cudaEvent_t* e : {&c->ev_snap, &c->ev_mem, &c->ev_coll, &c->ev_str[0], &c->ev_str[1], &c->ev_join})
    ok = ok && cudaEventCreateWithFlags(e, cudaEventDisableTiming) == cudaSuccess;
  c->ok = ok;
  return c;
}

void cohort_destroy(Cohort* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->ms) cudaStreamSynchronize(c->ms);
  if (c->ss) cudaStreamSynchronize(c->ss);
  for (cudaEvent_t e : {c->ev_snap, c->ev_mem, c->ev_coll, c->ev_str[0], c->ev_str[1], c->ev_join})
    if (e) cudaEventDestroy(e);
  if (c->ms) cudaStreamDestroy(c->ms);
  if (c->ss) cudaStreamDestroy(c->ss);
  if (c->plan.mem) cudaFree(c->plan.mem);
  if (c->plan.blk) cudaFree(c->plan.blk);
  delete c;
}

int64_t cohort_key(const irbc_handle* h) {
  if (!h || !h->fp32 || !h->have_mesh || h->capturing) return -1;
  int64_t k = h->P.device;
  k = k * 4096 + h->csteps;
  k = k * 4096 + (h->colsteps + 1);
  k = k * 2 + (h->step & 1);
  k = k * 2 + (h->snap_ready ? 1 : 0);
  return k;
}

static Member member_of(irbc_handle* h) {
  // every byte defined (padding too), so that descriptors compare bytewise
  Member M;
  std::memset(&M, 0, sizeof(M));
  M.p = h->dp;
  M.s = h->s;
  M.f = h->sf;
  M.c = h->c;
  M.m = h->m;
  M.fb = h->fb;
  // the staging capacity follows the longest list (as stream_any does for
  // plain launches)
  M.fb.hcap = heavy_cap(h->c.lmax);
  // host-only counters that no kernel reads
  M.s.ncoll = M.s.resorted = 0;
  return M;
}

// (Re)builds and uploads the device tables of the current members; both
// streams are idle when it returns, so no kernel reads the old tables
static int cohort_upload(Cohort* c) {
  if (cudaStreamSynchronize(c->ms) != cudaSuccess || cudaStreamSynchronize(c->ss) != cudaSuccess)
    return IRBC_ERR_CUDA;
  const size_t n = c->members.size();
  MultiPlan& P = c->plan;
  P.n = (int)n;
  c->host.resize(n);
  c->uids.resize(n);
  std::vector<std::array<int, MP_NPHASE>> nbk(n);
  int64_t tot[MP_NPHASE] = {};
  P.vbin_smem = P.sum_smem = 0;
  P.cells_short = 0;
  P.cells_cap = 1;
  std::vector<int> cls(n);  // the near-membrane class of each member: 0 short lists, 1 long lists
  for (size_t r = 0; r < n; ++r) {
    c->host[r] = member_of(c->members[r]);
    c->uids[r] = c->members[r]->uid;
    int sm[2];
    multi_blocks(c->host[r], nbk[r].data());
    multi_smem(c->host[r], sm);
    for (int k = 0; k < MP_NPHASE; ++k) tot[k] += nbk[r][k];
    const int hcap = c->host[r].fb.hcap;
    cls[r] = short_lists(hcap) ? 0 : 1;
    if (cls[r] == 0) P.cells_short += nbk[r][MP_CELLS];
    else P.cells_cap = std::max(P.cells_cap, stage_cap(hcap));
    P.vbin_smem = std::max(P.vbin_smem, sm[0]);
    P.sum_smem = std::max(P.sum_smem, sm[1]);
  }
  // the block tables: phase by phase, member by member
  int64_t all = 0;
  for (int k = 0; k < MP_NPHASE; ++k) {
    if (tot[k] >= (1LL << 31)) return IRBC_ERR_CAPACITY;
    P.off[k] = all;
    P.blocks[k] = (int)tot[k];
    all += tot[k];
  }
  std::vector<int2> tab((size_t)all);
  for (int k = 0; k < MP_NPHASE; ++k) {
    int64_t q = P.off[k];
    // the near-membrane blocks class by class (one launch per class)
    for (int pass = 0; pass < (k == MP_CELLS ? 2 : 1); ++pass)
      for (size_t r = 0; r < n; ++r) {
        if (k == MP_CELLS && cls[r] != pass) continue;
        for (int b = 0; b < nbk[r][k]; ++b) tab[(size_t)q++] = make_int2((int)r, b);
      }
  }
  if (n > c->cap || (size_t)all > c->tab_cap) {
    if (P.mem) cudaFree(P.mem);
    if (P.blk) cudaFree(P.blk);
    P.mem = nullptr;
    P.blk = nullptr;
    c->cap = n + n / 2 + 8;
    c->tab_cap = (size_t)all + (size_t)all / 2 + 1024;
    if (cudaMalloc((void**)&P.mem, c->cap * sizeof(Member)) != cudaSuccess ||
        cudaMalloc((void**)&P.blk, c->tab_cap * sizeof(int2)) != cudaSuccess)
      return IRBC_ERR_CUDA;
  }
  // From pageable memory a copy returns once its data is staged, before it
  // lands; a plain cudaMemcpy would land through the legacy stream, which
  // the cohort's non-blocking streams do not follow.  So: queued on the
  // cohort's own stream, and waited for, before any kernel reads the tables.
  if (cudaMemcpyAsync(P.mem, c->host.data(), n * sizeof(Member), cudaMemcpyHostToDevice, c->ms) != cudaSuccess ||
      cudaMemcpyAsync(P.blk, tab.data(), tab.size() * sizeof(int2), cudaMemcpyHostToDevice, c->ms) != cudaSuccess ||
      cudaStreamSynchronize(c->ms) != cudaSuccess)
    return IRBC_ERR_CUDA;
  return 0;
}

// whether the uploaded descriptor of member r still describes its handle:
// the same handle (its unique id: a destroyed handle's address, and its
// buffers' addresses, can come back for a new simulation of another size)
// and every byte of the descriptor the same
static bool member_current(const Cohort* c, size_t r) {
  if (c->uids[r] != c->members[r]->uid) return false;
  const Member now = member_of(c->members[r]);
  return std::memcmp(&now, &c->host[r], sizeof(Member)) == 0;
}

int cohort_step(Cohort* c, const std::vector<irbc_handle*>& all, int64_t n, std::vector<int>& status) {
  status.assign(all.size(), 0);
  if (!c || !c->ok || n < 0) return IRBC_ERR_ARG;
  if (all.empty() || n == 0) return 0;
  cudaSetDevice(c->device);
  // members already found unhealthy are not stepped (as irbc_step)
  std::vector<irbc_handle*> hs;
  for (size_t i = 0; i < all.size(); ++i) {
    irbc_handle* h = all[i];
    if (cudaEventQuery(h->ev_health) == cudaSuccess && *h->health_host) status[i] = health_status(h, *h->health_host);
    else hs.push_back(h);
  }
  if (hs.empty()) return 0;
  const int64_t key = cohort_key(hs[0]);
  for (irbc_handle* h : hs)
    if (key < 0 || cohort_key(h) != key || h->P.device != c->device) return IRBC_ERR_ARG;
  cudaStream_t ms = c->ms, ss = c->ss;
  int64_t launched = 0;
  // the cohort's work follows each member's earlier work; the epochs of
  // this call are each member's step count plus the step's offset
  for (irbc_handle* h : hs) {
    if (cudaEventRecord(c->ev_join, h->st) != cudaSuccess || cudaStreamWaitEvent(ms, c->ev_join, 0) != cudaSuccess)
      return IRBC_ERR_CUDA;
    h->ebase_val = h->step;
    launch_set_u64(h->ebase, (uint64_t)h->step, ms);
    if (cudaMemsetAsync(h->fb.qn, 0, 2 * sizeof(int), ms) != cudaSuccess) return IRBC_ERR_CUDA;
    launched += 1;
  }
  if (cudaEventRecord(c->ev_coll, ms) != cudaSuccess || cudaStreamWaitEvent(ss, c->ev_coll, 0) != cudaSuccess)
    return IRBC_ERR_CUDA;
  // the device tables: rebuilt when the members changed or a member's
  // buffers, capacities or wall speed moved
  bool stale = hs.size() != c->members.size() || c->uids.size() != hs.size();
  for (size_t r = 0; !stale && r < hs.size(); ++r) stale = hs[r] != c->members[r] || c->uids[r] != hs[r]->uid;
  for (size_t r = 0; !stale && r < hs.size(); ++r) stale = !member_current(c, r);
  if (stale) {
    c->members = hs;
    int rc = cohort_upload(c);
    if (rc) return rc;
  }
  irbc_handle* h0 = hs[0];
  const int csteps = h0->csteps;
  for (int64_t k = 0; k < n; ++k) {
    const int buf = (int)(h0->step & 1);
    bool moved = false;
    for (irbc_handle* h : hs) {
      const irbc_params& p = h->P;
      const double ws = (h->step < p.warm_steps) ? p.warm_speed : p.walls;
      if (ws != h->dp.wallspeed) { h->dp.wallspeed = ws; moved = true; }
      h->colsteps += 1; h->bbi += 1; h->upd += 1;
      if (h->step > 0) h->filecc += 1;
    }
    if (moved) {
      int rc = cohort_upload(c);
      if (rc) return rc;
    }
    const bool collide = h0->colsteps == csteps;
    if (collide) {
      c->ncoll += 1;
      const bool resort = c->ncoll % kResortEvery == 0;
      for (irbc_handle* h : hs) {
        h->s.ncoll += 1;
        if (resort) h->s.resorted = h->s.ncoll;
        h->colsteps = 0;
        h->snap_ready = false;
      }
      // the vertex binning reads the positions, and the tiles rotate the
      // vertex velocities, of the previous step's membrane step (side
      // stream): the collision waits for it (step_one bins on the side
      // stream for the same reason)
      if (cudaStreamWaitEvent(ms, c->ev_mem, 0) != cudaSuccess) return IRBC_ERR_CUDA;
      launched += multi_collide_front(c->plan, (uint64_t)k, ms);
      launched += multi_collide_count(c->plan, (uint64_t)k, ms);
      launched += multi_collide_scan(c->plan, ms);
      launched += multi_collide_back(c->plan, (uint64_t)k, resort, ms);
      if (cudaEventRecord(c->ev_coll, ms) != cudaSuccess || cudaStreamWaitEvent(ss, c->ev_coll, 0) != cudaSuccess)
        return IRBC_ERR_CUDA;
    }
    if (!h0->snap_ready) {
      if (cudaStreamWaitEvent(ss, c->ev_str[buf], 0) != cudaSuccess) return IRBC_ERR_CUDA;
      launched += multi_kick(c->plan, buf, ss);
    }
    // list updates (rare, per member, with host waits): positions of this
    // step are final once the side stream reaches here
    bool listed = false;
    for (irbc_handle* h : hs) {
      if (h->upd != h->uplist) continue;
      if (!listed) {
        if (cudaEventRecord(c->ev_snap, ss) != cudaSuccess || cudaStreamWaitEvent(ms, c->ev_snap, 0) != cudaSuccess)
          return IRBC_ERR_CUDA;
        listed = true;
      }
      if (cudaEventRecord(c->ev_join, ms) != cudaSuccess || cudaStreamWaitEvent(h->st, c->ev_join, 0) != cudaSuccess)
        return IRBC_ERR_CUDA;
      int rc = do_llist(h);
      if (rc) return rc;
      h->upd = 0;
      if (cudaEventRecord(c->ev_join, h->st) != cudaSuccess || cudaStreamWaitEvent(ms, c->ev_join, 0) != cudaSuccess)
        return IRBC_ERR_CUDA;
    }
    if (listed) {
      int rc = cohort_upload(c);  // lists, buckets and staging may have moved or grown
      if (rc) return rc;
    }
    const bool next_collides = h0->colsteps + 1 == csteps;
    const bool next_kick = k != n - 1 && !next_collides;
    // as step_one: the bulk streaming starts at once, the near-membrane
    // kernel waits for the snapshot, the membrane step runs beside them and
    // writes the next snapshot only after the streaming that read it
    if (cudaEventRecord(c->ev_snap, ss) != cudaSuccess) return IRBC_ERR_CUDA;
    launched += multi_stream(c->plan, buf, ms, c->ev_snap);
    if (cudaEventRecord(c->ev_str[buf], ms) != cudaSuccess) return IRBC_ERR_CUDA;
    launched += multi_membrane(c->plan, (uint64_t)k, ss);
    if (next_kick) {
      if (cudaStreamWaitEvent(ss, c->ev_str[buf ^ 1], 0) != cudaSuccess) return IRBC_ERR_CUDA;
      launched += multi_kick(c->plan, buf ^ 1, ss);
    }
    if (cudaEventRecord(c->ev_mem, ss) != cudaSuccess) return IRBC_ERR_CUDA;
    for (irbc_handle* h : hs) {
      h->snap_ready = next_kick;
      if (h->filecc == h->P.out_every) { h->filec += 1; h->filecc = 0; }
      h->step += 1;
    }
  }
  // each member's own stream follows the cohort's work; its health word
  // is copied for the next irbc_step (as at the end of irbc_step)
  if (cudaStreamWaitEvent(ms, c->ev_mem, 0) != cudaSuccess || cudaEventRecord(c->ev_join, ms) != cudaSuccess)
    return IRBC_ERR_CUDA;
  for (irbc_handle* h : hs) {
    if (cudaStreamWaitEvent(h->st, c->ev_join, 0) != cudaSuccess ||
        cudaMemcpyAsync(h->health_host, h->health, sizeof(int), cudaMemcpyDeviceToHost, h->st) != cudaSuccess ||
        cudaEventRecord(h->ev_health, h->st) != cudaSuccess)
      return IRBC_ERR_CUDA;
  }
  g_launches += launched;
  return cudaGetLastError() == cudaSuccess ? 0 : IRBC_ERR_CUDA;
}

}  // namespace irbc

// ---- output ----------------------------------------------------------------------
namespace {
struct VertexCopy {
  std::vector<double> x, y, z;
  std::vector<int> ix, iy, bondi;
};
int pull_vertices(irbc_handle* h, VertexCopy& V) {
  const Membrane& m = h->m;
  V.x.resize(m.nv); V.y.resize(m.nv); V.z.resize(m.nv); V.ix.resize(m.nv); V.iy.resize(m.nv); V.bondi.resize(m.nv);
  if (down(h, V.x.data(), m.x, m.nv) || down(h, V.y.data(), m.y, m.nv) || down(h, V.z.data(), m.z, m.nv) ||
      down(h, V.ix.data(), m.ix, m.nv) || down(h, V.iy.data(), m.iy, m.nv) || down(h, V.bondi.data(), m.bondi, m.nv))
    return IRBC_ERR_CUDA;
  CK(cudaStreamSynchronize(h->st));
  return 0;
}
}  // namespace

// RBCdata record (maincode.cpp:749-753)
namespace {
__global__ void k_pack_record(Membrane m, int nv, double* d, int32_t* q) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  d[i] = m.x[i]; d[nv + i] = m.y[i]; d[2 * nv + i] = m.z[i];
  q[i] = m.ix[i]; q[nv + i] = m.iy[i]; q[2 * nv + i] = m.bondi[i];
}
}  // namespace

extern "C" int64_t irbc_record_bytes(const irbc_handle* h) {
  return h ? (int64_t)h->m.nv * (3 * (int64_t)sizeof(double) + 3 * (int64_t)sizeof(int32_t)) : -1;
}

extern "C" int irbc_record_async(irbc_handle* h, void* host, int64_t bytes) {
  if (!h || !host) return IRBC_ERR_ARG;
  if (!h->have_mesh) return fail(h, IRBC_ERR_STATE, "no mesh");
  const int64_t need = irbc_record_bytes(h);
  if (bytes < need) return fail(h, IRBC_ERR_CAPACITY, "record buffer too small");
  cudaSetDevice(h->P.device);
  if (!h->rec) CK(cudaMalloc(&h->rec, (size_t)need));
  const int nv = h->m.nv;
  double* d = static_cast<double*>(h->rec);
  int32_t* q = reinterpret_cast<int32_t*>(d + 3 * (size_t)nv);
  k_pack_record<<<(nv + 255) / 256, 256, 0, h->st>>>(h->m, nv, d, q);
  g_launches += 1;
  CK(cudaMemcpyAsync(host, h->rec, (size_t)need, cudaMemcpyDeviceToHost, h->st));
  return 0;
}

extern "C" int irbc_write_rbcdata(irbc_handle* h, const char* path, int32_t append) {
  if (!h || !path || !h->have_mesh) return IRBC_ERR_ARG;
  VertexCopy V;
  int rc = pull_vertices(h, V);
  if (rc) return rc;
  FILE* f = fopen(path, append ? "a" : "w");
  if (!f) return fail(h, IRBC_ERR_IO, std::string("cannot open ") + path);
  fprintf(f, "#%d\n", h->filec);
  for (int i = 0; i < h->m.nv; ++i)
    fprintf(f, "%lf\t%lf\t%lf\t%d\t%d\t%d\n", V.x[i], V.y[i], V.z[i], V.ix[i], V.iy[i], V.bondi[i]);
  fclose(f);
  return 0;
}

// STL surface (filewrite, Src/memfuncs.cpp:590-626): iostream default format
extern "C" int irbc_write_stl(irbc_handle* h, const char* path) {
  if (!h || !path || !h->have_mesh) return IRBC_ERR_ARG;
  VertexCopy V;
  int rc = pull_vertices(h, V);
  if (rc) return rc;
  const Membrane& m = h->m;
  std::vector<int> t1(m.nt), t2(m.nt), t3(m.nt);
  if (down(h, t1.data(), m.t1, m.nt) || down(h, t2.data(), m.t2, m.nt) || down(h, t3.data(), m.t3, m.nt))
    return IRBC_ERR_CUDA;
  CK(cudaStreamSynchronize(h->st));
  std::ofstream f(path);
  if (!f) return fail(h, IRBC_ERR_IO, std::string("cannot open ") + path);
  const double Lx = h->P.Lx, Ly = h->P.Ly;
  auto UX = [&](int q) { return V.x[q] + V.ix[q] * Lx; };
  auto UY = [&](int q) { return V.y[q] + V.iy[q] * Ly; };
  f << "solid ascii" << std::endl;
  for (int kk = 0; kk < m.nt; ++kk) {
    int l1 = t1[kk], l2 = t2[kk], l3 = t3[kk];
    double A[3] = {UX(l2) - UX(l1), UY(l2) - UY(l1), V.z[l2] - V.z[l1]};
    double B[3] = {UX(l3) - UX(l1), UY(l3) - UY(l1), V.z[l3] - V.z[l1]};
    double N[3];
    hcp(A, B, N);
    f << "facet normal" << "\t" << N[0] << "\t" << N[1] << "\t" << N[2] << std::endl;
    f << "outer loop" << std::endl;
    f << "vertex" << "\t" << UX(l1) << "\t" << UY(l1) << "\t" << V.z[l1] << std::endl;
    f << "vertex" << "\t" << UX(l2) << "\t" << UY(l2) << "\t" << V.z[l2] << std::endl;
    f << "vertex" << "\t" << UX(l3) << "\t" << UY(l3) << "\t" << V.z[l3] << std::endl;
    f << "endloop" << std::endl;
    f << "endfacet" << std::endl;
  }
  f << "endsolid" << std::endl;
  return 0;
}

extern "C" int irbc_observables(irbc_handle* h, double* out, int32_t nout) {
  if (!h || !out || nout <= 0) return IRBC_ERR_ARG;
  if (h->fp32) f32_to_f64(h->sf, h->s, h->st);
  launch_observables(h->dp, h->s, h->m, h->obs, 0, h->st);
  g_launches += 2;
  double buf[16] = {0};
  CK(cudaMemcpyAsync(buf, h->obs, sizeof(double) * 16, cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  for (int k = 0; k < nout && k < 16; ++k) out[k] = buf[k];
  return 0;
}

extern "C" int irbc_velocity_profile(irbc_handle* h, double* out, int32_t nbins) {
  if (!h || !out || nbins <= 0 || nbins > kObsMaxBins) return IRBC_ERR_ARG;
  if (h->fp32) f32_to_f64(h->sf, h->s, h->st);
  launch_observables(h->dp, h->s, h->m, h->obs, nbins, h->st);
  g_launches += 2;
  std::vector<double> buf(2 * nbins);
  CK(cudaMemcpyAsync(buf.data(), h->obs + 64, sizeof(double) * 2 * nbins, cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  for (int k = 0; k < nbins; ++k) out[k] = buf[2 * k + 1] > 0 ? buf[2 * k] / buf[2 * k + 1] : 0.0;
  return 0;
}

// ---- standalone binning ------------------------------------------------------------
namespace irbc {
void bin_particles(const DevParams& p, const double* x, const double* y, const double* z, int64_t n,
                   double rx, double ry, double rz, int* cell, int* start, int* order, int* cnt, int* slot,
                   int* part, int* totals, cudaStream_t st);
}

extern "C" int irbc_bin_particles(const irbc_params* p, const double* x, const double* y, const double* z,
                                  int64_t n, double rx, double ry, double rz, int32_t* cell, int32_t* start,
                                  int32_t* order) {
  if (!p || n < 0 || (n > 0 && (!x || !y || !z || !cell || !order)) || !start) return IRBC_ERR_ARG;
  if (p->a != 1.0 || p->Lx <= 0 || p->Ly <= 0 || p->Lz <= 0 || n >= (1LL << 31)) return IRBC_ERR_ARG;
  if (!(rx >= 0 && rx < 1 && ry >= 0 && ry < 1 && rz >= 0 && rz < 1)) return IRBC_ERR_ARG;
  DevParams d{};
  fill_devparams_from(*p, d);
  int *cnt = nullptr, *slot = nullptr, *part = nullptr, *totals = nullptr;
  int64_t nb = scan_part_blocks(d.ncell);
  cudaError_t e = dalloc(&cnt, d.ncell);
  if (e == cudaSuccess) e = dalloc(&slot, n);
  if (e == cudaSuccess) e = dalloc(&part, 3 * nb + 3);
  if (e == cudaSuccess) e = dalloc(&totals, 4);
  if (e == cudaSuccess) {
    bin_particles(d, x, y, z, n, rx, ry, rz, cell, start, order, cnt, slot, part, totals, 0);
    g_launches += 6;
    e = cudaStreamSynchronize(0);
  }
  dfree(cnt); dfree(slot); dfree(part); dfree(totals);
  return e == cudaSuccess ? 0 : IRBC_ERR_CUDA;
}

// ---- profiling window and host buffers ------------------------------------------------
// device time of a stretch of calls with two events on the handle's
// stream and nothing in between (no per-phase events)
extern "C" int irbc_timer_begin(irbc_handle* h) {
  if (!h) return IRBC_ERR_ARG;
  cudaSetDevice(h->P.device);
  if (!h->ev_begin) { CK(cudaEventCreate(&h->ev_begin)); CK(cudaEventCreate(&h->ev_end)); }
  CK(cudaEventRecord(h->ev_begin, h->st));
  return 0;
}
extern "C" int irbc_timer_end(irbc_handle* h, double* ms) {
  if (!h || !ms || !h->ev_begin) return IRBC_ERR_ARG;
  cudaSetDevice(h->P.device);
  CK(cudaEventRecord(h->ev_end, h->st));
  CK(cudaEventSynchronize(h->ev_end));
  float t = 0.f;
  CK(cudaEventElapsedTime(&t, h->ev_begin, h->ev_end));
  *ms = t;
  return 0;
}

extern "C" int irbc_profile_begin(irbc_handle* h) {
  if (!h) return IRBC_ERR_ARG;
  cudaSetDevice(h->P.device);
  if (!h->ev_begin) { CK(cudaEventCreate(&h->ev_begin)); CK(cudaEventCreate(&h->ev_end)); }
  h->ev_used = 0;
  h->ev_marks.clear();
  h->prof = true;
  h->prof_launch0 = g_launches.load();
  CK(cudaEventRecord(h->ev_begin, h->st));
  return 0;
}

extern "C" int irbc_profile_end(irbc_handle* h, double* out, int32_t nout) {
  if (!h || !out) return IRBC_ERR_ARG;
  if (!h->prof) return fail(h, IRBC_ERR_STATE, "no profiling window open");
  CK(cudaEventRecord(h->ev_end, h->st));
  CK(cudaEventSynchronize(h->ev_end));
  h->prof = false;
  double r[10] = {0};
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, h->ev_begin, h->ev_end));
  r[0] = ms;
  for (auto& mk : h->ev_marks) {
    float t = 0;
    CK(cudaEventElapsedTime(&t, h->ev_pool[mk.start], h->ev_pool[mk.end]));
    const int slot = mk.cat == PROF_STREAM_BULK ? 8 : 1 + 2 * mk.cat;
    r[slot] += t;
    r[slot + 1] += 1;
  }
  r[7] = (double)(g_launches.load() - h->prof_launch0);
  for (int k = 0; k < nout && k < 10; ++k) out[k] = r[k];
  return 0;
}

extern "C" void* irbc_host_alloc(size_t bytes) {
  void* p = nullptr;
  if (cudaMallocHost(&p, bytes) != cudaSuccess) return nullptr;
  return p;
}
extern "C" void irbc_host_free(void* p) {
  if (p) cudaFreeHost(p);
}
