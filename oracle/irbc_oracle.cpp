/*
 * oracle/irbc_oracle.cpp -- TEST INFRASTRUCTURE: CPU oracle (see
 * oracle/irbc_oracle.h).  Single-threaded restatement of the reference
 * timestep; each function names the reference lines it follows.  Never
 * linked into the shipped library.
 */
#include "irbc_oracle.h"
#include "irbc_rng.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <utility>
#include <vector>

using std::vector;

struct orc_ctx {
  orc_params p;
  uint64_t seed;
  uint64_t init_draws;  // INIT-stream cursor
  int nx, ny, nz;
  int64_t ncell;
  int csteps, uplist;
  // mesh
  int nv, ne, nt;
  vector<int> e1, e2, es1, es2, iedge, t1, t2, t3;
  vector<double> l0, kappap, cmx, cmy, cmz, tarea;
  double Sarea0, Volume0, theta0, center[3];
  // solvent
  int64_t ns;
  vector<double> sx, sy, sz, svx, svy, svz;
  vector<int> spid, sindio;
  // vertices
  vector<double> x, y, z, vx, vy, vz, fx, fy, fz, poff, pon;
  vector<int> pid, ix, iy, bondi, bondl, knob;
  // parasite
  double para[3], paraV[3], paraft[3], parafdt[3];
  int paradx, parady, paraid;
  // ligands
  int nlig;
  vector<double> xlig, ylig;
  vector<int> ligi;
  // cells
  vector<vector<int>> llist;
  double Sarea, Volume, wallspeed;
  int64_t step;
  int colsteps, upd, filecc, filec, bbi;
  // diagnostics
  double meanedge, stdedge, young, poisson, areaC;
  int knobcount;
  uint64_t last_normals, last_bond_draws;
  // per-vertex candidate ligand lists (vert::Pairs, define.h:138)
  vector<vector<std::pair<double, int>>> pairs;
};

extern "C" void orc_params_default(orc_params* p) {
  std::memset(p, 0, sizeof(*p));
  p->a = 1.0; p->Lx = 60.0; p->Ly = 40.0; p->Lz = 40.0; p->Ns = 960000;
  p->dtcd = 0.02; p->navg = 10.0; p->Theta = 1.0; p->walls = 3.0; p->mass = 1.0;
  p->cosalpha = -0.70710678118; p->sinalpha = 0.70710678118;
  p->Nt = 600; p->kappasa = 60000.0; p->kappad = 1200.0; p->kappav = 6000.0;
  p->kappab = 100.0; p->pmass = 10.0 * 1.0; p->dtmd = 0.002; p->ks = 6000.0;
  p->dthr = 0.50; p->FD = 1200.0; p->Fg = 40.0; p->el0 = 0.1;
  p->PRmass = 10.0; p->paraR = 1.7; p->Pi = 3.141592653;
  p->elap = 0.0005; p->shear = 1200.0; p->onrate = 0.005; p->offrate = 0.015;
  p->warm_steps = 250000; p->warm_speed = 0.1; p->out_every = 5000; p->randno = 12345678;
}

static void derive(orc_ctx* c) {
  const orc_params& p = c->p;
  c->nx = (int)(p.Lx / p.a);              // maincode.cpp:113-115
  c->ny = (int)(p.Ly / p.a);
  c->nz = (int)(p.Lz / p.a) + 1;
  c->ncell = (int64_t)c->nx * c->ny * c->nz;
  c->csteps = (int)(p.dtcd / p.dtmd);     // maincode.cpp:455
  c->uplist = (int)(0.5 / (p.walls * p.dtmd));  // maincode.cpp:460
  c->llist.assign(c->ncell, vector<int>());
  // ligand grid, maincode.cpp:77-93
  c->xlig.clear(); c->ylig.clear();
  double xmin = 0.0, ymin = 0.0;
  while (xmin < p.Lx) {
    while (ymin < p.Ly) { c->xlig.push_back(xmin); c->ylig.push_back(ymin); ymin += 0.5; }
    xmin += 0.5; ymin = 0;
  }
  c->nlig = (int)c->xlig.size();
  c->ligi.assign(c->nlig, 0);
}

extern "C" orc_ctx* orc_create(const orc_params* p, uint64_t seed) {
  orc_ctx* c = new orc_ctx();
  c->p = *p; c->seed = seed; c->init_draws = 0;
  derive(c);
  c->nv = c->ne = c->nt = 0; c->ns = 0;
  c->Sarea0 = c->Volume0 = c->theta0 = 0; c->center[0] = c->center[1] = c->center[2] = 0;
  for (int k = 0; k < 3; ++k) c->para[k] = c->paraV[k] = c->paraft[k] = c->parafdt[k] = 0;
  c->paradx = c->parady = c->paraid = 0;
  c->Sarea = c->Volume = 0; c->wallspeed = 0;
  c->step = 0; c->colsteps = -1; c->upd = 0; c->filecc = 0; c->filec = 0; c->bbi = 0;
  c->last_normals = c->last_bond_draws = 0; c->knobcount = 0;
  return c;
}
extern "C" void orc_destroy(orc_ctx* c) { delete c; }
extern "C" int64_t orc_ncell(const orc_ctx* c) { return c->ncell; }
extern "C" uint64_t orc_last_normals(const orc_ctx* c) { return c->last_normals; }
extern "C" uint64_t orc_last_bond_draws(const orc_ctx* c) { return c->last_bond_draws; }

// ---------------------------------------------------------------- helpers
static inline double U_init(orc_ctx* c) {
  return orc_uniform(c->seed, ORC_STREAM_INIT, 0, c->init_draws++);
}
// IRandom (Src/mersenne.cpp:115-125) over the replacement uniform
static inline int IRand(orc_ctx* c, int mn, int mx) {
  if (mx <= mn) return (mx == mn) ? mn : (int)0x80000000;
  int r = int((double)(uint32_t)(mx - mn + 1) * U_init(c) + mn);
  if (r > mx) r = mx;
  return r;
}
// cp (Src/memfuncs.cpp:47-52)
static inline void cp(const double A[], const double B[], double C[]) {
  C[0] = (A[1] * B[2]) - (B[1] * A[2]);
  C[1] = (A[2] * B[0]) - (B[2] * A[0]);
  C[2] = (A[0] * B[1]) - (B[0] * A[1]);
}
// bbound (Src/solfuncs.cpp:603-622)
static inline double bbound(double x, double lx) {
  if (x > lx) { while (x > lx) x -= lx; }
  if (x < 0) { while (x < 0) x += lx; }
  return x;
}
// cindex[fx][fy][fz] (maincode.cpp:112-136): unset entries are 0
static inline int cell_of(const orc_ctx* c, int fx, int fy, int fz) {
  if (fx >= 0 && fx < c->nx && fy >= 0 && fy < c->ny && fz >= 0 && fz < c->nz)
    return (int)(((int64_t)fx * c->ny + fy) * c->nz + fz);
  return 0;
}
static inline void cell_bounds(const orc_ctx* c, int64_t id, double b[6]) {
  const double a = c->p.a;
  int k = (int)(id % c->nz);
  int j = (int)((id / c->nz) % c->ny);
  int i = (int)(id / ((int64_t)c->nz * c->ny));
  b[0] = (double)i * a; b[1] = (double)i * a + a;       // xmin, xmax
  b[2] = (double)j * a; b[3] = (double)j * a + a;       // ymin, ymax
  b[4] = -1.0 + (double)k * a; b[5] = -1.0 + (double)k * a + a;  // zmin, zmax
}
// unwrapped coordinate of vertex v (vts[v].x + vts[v].ix*Lx)
#define UX(v) (c->x[v] + c->ix[v] * c->p.Lx)
#define UY(v) (c->y[v] + c->iy[v] * c->p.Ly)

// Areatri (Src/memfuncs.cpp:144-157)
static double areatri(const orc_ctx* c, int p1, int p2, int p3) {
  double A[3], B[3], eta[3];
  A[0] = UX(p2) - UX(p1); A[1] = UY(p2) - UY(p1); A[2] = c->z[p2] - c->z[p1];
  B[0] = UX(p3) - UX(p1); B[1] = UY(p3) - UY(p1); B[2] = c->z[p3] - c->z[p1];
  cp(A, B, eta);
  return 0.5 * sqrt(eta[0] * eta[0] + eta[1] * eta[1] + eta[2] * eta[2]);
}
// Normaldt (Src/memfuncs.cpp:110-122)
static void normaldt(const orc_ctx* c, int p1, int p2, int p3, double X[]) {
  double A[3], B[3];
  A[0] = UX(p2) - UX(p1); A[1] = UY(p2) - UY(p1); A[2] = c->z[p2] - c->z[p1];
  B[0] = UX(p3) - UX(p1); B[1] = UY(p3) - UY(p1); B[2] = c->z[p3] - c->z[p1];
  cp(A, B, X);
}
// Voltri (Src/memfuncs.cpp:124-142)
static double voltri(const orc_ctx* c, int p1, int p2, int p3) {
  double A[3], B[3], C[3], D[3], Cn[3];
  A[0] = UX(p1); A[1] = UY(p1); A[2] = c->z[p1];
  B[0] = UX(p2); B[1] = UY(p2); B[2] = c->z[p2];
  C[0] = UX(p3); C[1] = UY(p3); C[2] = c->z[p3];
  Cn[0] = (A[0] + B[0] + C[0]) / 3.0;
  Cn[1] = (A[1] + B[1] + C[1]) / 3.0;
  Cn[2] = (A[2] + B[2] + C[2]) / 3.0;
  normaldt(c, p1, p2, p3, D);
  return (1.0 / 6.0) * ((D[0] * Cn[0]) + (D[1] * Cn[1]) + (D[2] * Cn[2]));
}

// ------------------------------------------------------------------ set-up
// tricm (Src/memfuncs.cpp:18-31)
static void tricm(orc_ctx* c) {
  for (int i = 0; i < c->nt; ++i) {
    int p1 = c->t1[i], p2 = c->t2[i], p3 = c->t3[i];
    c->cmx[i] = (UX(p1) + UX(p2) + UX(p3)) / 3.0;
    c->cmy[i] = (UY(p1) + UY(p2) + UY(p3)) / 3.0;
    c->cmz[i] = (c->z[p1] + c->z[p2] + c->z[p3]) / 3.0;
    c->cmx[i] = fmod(c->cmx[i], c->p.Lx);
    c->cmy[i] = fmod(c->cmy[i], c->p.Ly);
  }
}
// sortsolvent_initial1 classification (Src/solfuncs.cpp:17-94); returns indio
static void classify_solvent(orc_ctx* c) {
  double Rd[3] = {1.0, 0.0, 0.0};
  for (int64_t i = 0; i < c->ns; ++i) {
    int count = 0;
    double Q1[3], Q2[3], X[3], P0[3];
    Q1[0] = c->sx[i] + Rd[0] * 0.3; Q1[1] = c->sy[i] + Rd[1] * 0.3; Q1[2] = c->sz[i] + Rd[2] * 0.3;
    Q2[0] = c->sx[i] + Rd[0] * 0.7; Q2[1] = c->sy[i] + Rd[1] * 0.7; Q2[2] = c->sz[i] + Rd[2] * 0.7;
    for (int j = 0; j < c->nt; ++j) {
      int p1 = c->t1[j], p2 = c->t2[j], p3 = c->t3[j];
      normaldt(c, p1, p2, p3, X);
      double dotP1Q1 = (c->x[p1] - Q1[0]) * X[0] + (c->y[p1] - Q1[1]) * X[1] + (c->z[p1] - Q1[2]) * X[2];
      double dotQ2Q1 = (Q2[0] - Q1[0]) * X[0] + (Q2[1] - Q1[1]) * X[1] + (Q2[2] - Q1[2]) * X[2];
      for (int k = 0; k < 3; ++k) P0[k] = Q1[k] + ((dotP1Q1 / dotQ2Q1) * (Q2[k] - Q1[k]));
      double P2P1[3] = {c->x[p2] - c->x[p1], c->y[p2] - c->y[p1], c->z[p2] - c->z[p1]};
      double P3P2[3] = {c->x[p3] - c->x[p2], c->y[p3] - c->y[p2], c->z[p3] - c->z[p2]};
      double P1P3[3] = {c->x[p1] - c->x[p3], c->y[p1] - c->y[p3], c->z[p1] - c->z[p3]};
      double P0P1[3] = {P0[0] - c->x[p1], P0[1] - c->y[p1], P0[2] - c->z[p1]};
      double P0P2[3] = {P0[0] - c->x[p2], P0[1] - c->y[p2], P0[2] - c->z[p2]};
      double P0P3[3] = {P0[0] - c->x[p3], P0[1] - c->y[p3], P0[2] - c->z[p3]};
      double f1[3], f2[3], f3[3];
      cp(P2P1, P0P1, f1); cp(P3P2, P0P2, f2); cp(P1P3, P0P3, f3);
      double ch1 = f1[0] * X[0] + f1[1] * X[1] + f1[2] * X[2];
      double ch2 = f2[0] * X[0] + f2[1] * X[1] + f2[2] * X[2];
      double ch3 = f3[0] * X[0] + f3[1] * X[1] + f3[2] * X[2];
      if ((ch1 >= 0) && (ch2 >= 0) && (ch3 >= 0) && (c->cmx[j] >= c->sx[i])) count += 1;
    }
    c->sindio[i] = ((count % 2) == 0) ? 1 : 0;
  }
}

// centerofmass (Src/memfuncs.cpp:55-74)
static void centerofmass(orc_ctx* c) {
  double rr[3] = {0, 0, 0};
  for (int i = 0; i < c->nv; ++i) { rr[0] += UX(i); rr[1] += UY(i); rr[2] += c->z[i]; }
  c->center[0] = rr[0] / (double)c->nv;
  c->center[1] = rr[1] / (double)c->nv;
  c->center[2] = rr[2] / (double)c->nv;
  c->center[0] = fmod(c->center[0], c->p.Lx);
  c->center[1] = fmod(c->center[1], c->p.Ly);
  c->center[2] = fmod(c->center[2], c->p.Lz);
}

// makeiedge (Src/memfuncs.cpp:533-588)
static void makeiedge(orc_ctx* c) {
  for (int i = 0; i < c->ne; ++i) {
    int l2 = c->e1[i], l3 = c->e2[i], l1 = c->es1[i], l4 = c->es2[i];
    double a21[3] = {c->x[l2] - c->x[l1], c->y[l2] - c->y[l1], c->z[l2] - c->z[l1]};
    double a31[3] = {c->x[l3] - c->x[l1], c->y[l3] - c->y[l1], c->z[l3] - c->z[l1]};
    double a24[3] = {c->x[l2] - c->x[l4], c->y[l2] - c->y[l4], c->z[l2] - c->z[l4]};
    double a34[3] = {c->x[l3] - c->x[l4], c->y[l3] - c->y[l4], c->z[l3] - c->z[l4]};
    double t1[3], t2[3], tt1[3], tt2[3], eta[3], zeta[3];
    t1[0] = (c->x[l1] + c->x[l2] + c->x[l3]) / 3.0;
    t1[1] = (c->y[l1] + c->y[l2] + c->y[l3]) / 3.0;
    t1[2] = (c->z[l1] + c->z[l2] + c->z[l3]) / 3.0;
    t2[0] = (c->x[l4] + c->x[l2] + c->x[l3]) / 3.0;
    t2[1] = (c->y[l4] + c->y[l2] + c->y[l3]) / 3.0;
    t2[2] = (c->z[l4] + c->z[l2] + c->z[l3]) / 3.0;
    for (int k = 0; k < 3; ++k) { tt1[k] = t1[k] - c->center[k]; tt2[k] = t2[k] - c->center[k]; }
    cp(a21, a31, eta);
    cp(a34, a24, zeta);
    double che1 = eta[0] * tt1[0] + eta[1] * tt1[1] + eta[2] * tt1[2];
    double che2 = zeta[0] * tt2[0] + zeta[1] * tt2[1] + zeta[2] * tt2[2];
    if ((che1 >= 0) && (che2 >= 0)) c->iedge[i] = 1;
    else if ((che1 < 0) && (che2 < 0)) c->iedge[i] = -1;
    else c->iedge[i] = 1;  // the reference prints an error and keeps 1
  }
}

static void alloc_vertices(orc_ctx* c, int nv) {
  c->nv = nv;
  for (auto* v : {&c->x, &c->y, &c->z, &c->vx, &c->vy, &c->vz, &c->fx, &c->fy, &c->fz, &c->poff, &c->pon})
    v->assign(nv, 0.0);
  for (auto* v : {&c->pid, &c->ix, &c->iy, &c->bondi, &c->bondl, &c->knob}) v->assign(nv, 0);
  c->pairs.assign(nv, {});
}
static void alloc_solvent(orc_ctx* c, int64_t ns) {
  c->ns = ns;
  for (auto* v : {&c->sx, &c->sy, &c->sz, &c->svx, &c->svy, &c->svz}) v->assign(ns, 0.0);
  c->spid.assign(ns, 0); c->sindio.assign(ns, 0);
}

// main() set-up, maincode.cpp:94-446 (solvent init :96-107, mesh :157-391,
// knobs :394-433).  Files are replaced by arrays.
extern "C" int orc_init(orc_ctx* c, const double* V, int32_t nv, const int32_t* E, int32_t ne,
                        const int32_t* T, int32_t nt, int32_t nknobs, int32_t do_sort) {
  const orc_params& p = c->p;
  c->init_draws = 0;
  // solvent, maincode.cpp:96-107
  alloc_solvent(c, p.Ns);
  double vmax = sqrt(3.0 * p.Theta / p.mass);
  for (int64_t j = 0; j < p.Ns; ++j) {
    c->sx[j] = (p.Lx * U_init(c));
    c->sy[j] = (p.Ly * U_init(c));
    c->sz[j] = (p.Lz * U_init(c));
    c->svx[j] = -vmax + 2.0 * vmax * U_init(c);
    c->svy[j] = -vmax + 2.0 * vmax * U_init(c);
    c->svz[j] = -vmax + 2.0 * vmax * U_init(c);
  }
  // vertices, maincode.cpp:157-206
  alloc_vertices(c, nv);
  vmax = sqrt(3.0 * p.Theta / (p.pmass));
  vector<double> zcrds;
  for (int i = 0; i < nv; ++i) {
    zcrds.push_back(V[3 * i + 2]);
    c->x[i] = V[3 * i]; c->y[i] = V[3 * i + 1]; c->z[i] = V[3 * i + 2];
    c->vx[i] = -vmax + 2.0 * vmax * U_init(c);
    c->vy[i] = -vmax + 2.0 * vmax * U_init(c);
    c->vz[i] = -vmax + 2.0 * vmax * U_init(c);
    c->bondl[i] = p.randno;
  }
  std::sort(zcrds.begin(), zcrds.end());
  double Center[3];
  Center[2] = -zcrds.front() + 0.3;
  Center[0] = p.Lx / 2.0 + 10.0;
  Center[1] = p.Ly / 2.0;
  for (int i = 0; i < nv; ++i) { c->x[i] += Center[0]; c->y[i] += Center[1]; c->z[i] += Center[2]; }
  double numer = 1.73205080757 * ((double)p.Nt - 2.0) - 5.0 * p.Pi;
  double denom = 1.73205080757 * ((double)p.Nt - 2.0) - 3.0 * p.Pi;
  c->theta0 = 180.0 * acos(numer / denom) / p.Pi;
  // parasite, maincode.cpp:212-225
  c->para[0] = Center[0] - 2.0; c->para[1] = Center[1]; c->para[2] = Center[2];
  vmax = sqrt(3.0 * p.Theta / (p.PRmass));
  for (int k = 0; k < 3; ++k) c->paraV[k] = -vmax + 2.0 * vmax * U_init(c);
  c->paradx = c->parady = 0;
  for (int k = 0; k < 3; ++k) { c->paraft[k] = 0.0; c->parafdt[k] = 0.0; }
  // edges, maincode.cpp:239-257
  c->ne = ne; c->e1.assign(ne, 0); c->e2.assign(ne, 0); c->l0.assign(ne, 0); c->kappap.assign(ne, 0);
  double meanedge = 0, meanedge2 = 0;
  for (int i = 0; i < ne; ++i) {
    c->e1[i] = E[2 * i]; c->e2[i] = E[2 * i + 1];
    int a1 = c->e1[i], a2 = c->e2[i];
    double distx = (c->x[a1] - c->x[a2]) * (c->x[a1] - c->x[a2]);
    double disty = (c->y[a1] - c->y[a2]) * (c->y[a1] - c->y[a2]);
    double distz = (c->z[a1] - c->z[a2]) * (c->z[a1] - c->z[a2]);
    c->l0[i] = sqrt(distx + disty + distz);
    meanedge += c->l0[i];
    meanedge2 += c->l0[i] * c->l0[i];
  }
  c->meanedge = meanedge / (double)ne;
  c->stdedge = sqrt((meanedge2 / (double)ne) - ((meanedge / (double)ne) * (meanedge / (double)ne)));
  // triangles, maincode.cpp:264-271
  c->nt = nt; c->t1.assign(nt, 0); c->t2.assign(nt, 0); c->t3.assign(nt, 0);
  c->cmx.assign(nt, 0); c->cmy.assign(nt, 0); c->cmz.assign(nt, 0); c->tarea.assign(nt, 0);
  for (int i = 0; i < nt; ++i) { c->t1[i] = T[3 * i]; c->t2[i] = T[3 * i + 1]; c->t3[i] = T[3 * i + 2]; }
  // edgest, maincode.cpp:276-342
  c->es1.assign(ne, 0); c->es2.assign(ne, 0); c->iedge.assign(ne, 0);
  for (int i = 0; i < ne; ++i) {
    int l1 = c->e1[i], l2 = c->e2[i];
    for (int j = 0; j < nt; ++j) {
      int f1 = (l1 == c->t1[j]) + (l1 == c->t2[j]) + (l1 == c->t3[j]);
      int f2 = (l2 == c->t1[j]) + (l2 == c->t2[j]) + (l2 == c->t3[j]);
      if (f1 > 0 && f2 > 0) {
        if (c->t1[j] != l1 && c->t1[j] != l2) c->es1[i] = c->t1[j];
        if (c->t2[j] != l1 && c->t2[j] != l2) c->es1[i] = c->t2[j];
        if (c->t3[j] != l1 && c->t3[j] != l2) c->es1[i] = c->t3[j];
        break;
      }
    }
    for (int j = nt - 1; j >= 0; j--) {
      int f1 = (l1 == c->t1[j]) + (l1 == c->t2[j]) + (l1 == c->t3[j]);
      int f2 = (l2 == c->t1[j]) + (l2 == c->t2[j]) + (l2 == c->t3[j]);
      if (f1 > 0 && f2 > 0) {
        if (c->t1[j] != l1 && c->t1[j] != l2) c->es2[i] = c->t1[j];
        if (c->t2[j] != l1 && c->t2[j] != l2) c->es2[i] = c->t2[j];
        if (c->t3[j] != l1 && c->t3[j] != l2) c->es2[i] = c->t3[j];
        break;
      }
    }
  }
  // TotalVA0, Src/memfuncs.cpp:192-211
  {
    double totV = 0, totA = 0;
    for (int i = 0; i < nt; ++i) {
      totA += areatri(c, c->t1[i], c->t2[i], c->t3[i]);
      totV += voltri(c, c->t1[i], c->t2[i], c->t3[i]);
    }
    c->Sarea0 = totA; c->Volume0 = totV;
  }
  // kappap, maincode.cpp:347-361
  const double elap = p.elap, shear = p.shear;
  for (int i = 0; i < ne; ++i) {
    double ll0 = c->l0[i];
    double lmax = 2.5 * ll0;
    double x0 = ll0 / lmax;
    double onemx0 = 1.0 - x0;
    double shear1 = 1.0 / (4.0 * onemx0 * onemx0);
    double shear2 = x0 / (2.0 * onemx0 * onemx0 * onemx0);
    double shear4 = (1.732 / (4.0 * elap * lmax * x0));
    double sh = shear4 * shear2 - shear4 * shear1 + shear4 * 0.25;
    c->kappap[i] = (shear - sh) * 4.0 * ll0 * ll0 * ll0 / (3.0 * 1.732);
  }
  c->areaC = 2.0 * shear + p.kappasa + p.kappad;
  c->young = (4.0 * c->areaC * shear) / (c->areaC + shear);
  c->poisson = (c->areaC - shear) / (c->areaC + shear);
  for (int i = 0; i < nt; ++i) c->tarea[i] = areatri(c, c->t1[i], c->t2[i], c->t3[i]);
  // maincode.cpp:383-391
  centerofmass(c);
  makeiedge(c);
  orc_total_va(c);
  orc_pfdt(c);
  orc_forces(c);
  tricm(c);
  classify_solvent(c);
  if (do_sort) {
    // sort(solvent) by indio (Src/solfuncs.cpp:96): reproduce the same
    // std::sort permutation with a key-only comparator.
    struct K { int indio; int64_t idx; bool operator<(const K& r) const { return indio < r.indio; } };
    vector<K> keys(c->ns);
    for (int64_t i = 0; i < c->ns; ++i) keys[i] = {c->sindio[i], i};
    std::sort(keys.begin(), keys.end());
    auto perm = [&](vector<double>& v) { vector<double> o(c->ns); for (int64_t i = 0; i < c->ns; ++i) o[i] = v[keys[i].idx]; v.swap(o); };
    perm(c->sx); perm(c->sy); perm(c->sz); perm(c->svx); perm(c->svy); perm(c->svz);
    vector<int> o(c->ns);
    for (int64_t i = 0; i < c->ns; ++i) o[i] = c->sindio[keys[i].idx];
    c->sindio.swap(o);
  }
  orc_llist_update(c);
  // knobs, maincode.cpp:394-433
  vector<double> parea;
  for (int i = 0; i < nt; ++i) parea.push_back(c->tarea[i] / c->Sarea0);
  int knob_count = 0;
  while (knob_count < nknobs) {
    double rad = U_init(c);
    double aaa = 0;
    for (int j = 0; j < (int)parea.size(); ++j) {
      aaa += parea[j];
      if (aaa > rad) {
        int radi = IRand(c, 1, 3);
        if ((radi == 1) && (c->knob[c->t1[j]] == 0)) { c->knob[c->t1[j]] = 1; knob_count += 1; break; }
        else if ((radi == 2) && (c->knob[c->t2[j]] == 0)) { c->knob[c->t2[j]] = 1; knob_count += 1; break; }
        else if ((radi == 3) && (c->knob[c->t3[j]] == 0)) { c->knob[c->t3[j]] = 1; knob_count += 1; break; }
      }
    }
  }
  c->knobcount = 0;
  for (int i = 0; i < nv; ++i) c->knobcount += c->knob[i];
  c->step = 0; c->colsteps = -1; c->upd = 0; c->filecc = 0; c->filec = 0; c->bbi = 0;
  return 0;
}

extern "C" void orc_init_report(const orc_ctx* c, double out[9]) {
  out[0] = c->meanedge; out[1] = c->stdedge; out[2] = c->Sarea0; out[3] = c->Volume0;
  out[4] = c->p.shear; out[5] = c->young; out[6] = c->poisson; out[7] = c->knobcount;
  out[8] = c->theta0;
}

// --------------------------------------------------------------- import/export
extern "C" int orc_set_mesh(orc_ctx* c, const orc_mesh* m) {
  c->nv = m->nv; c->ne = m->ne; c->nt = m->nt;
  c->e1.assign(m->e1, m->e1 + m->ne); c->e2.assign(m->e2, m->e2 + m->ne);
  c->l0.assign(m->l0, m->l0 + m->ne); c->kappap.assign(m->kappap, m->kappap + m->ne);
  c->es1.assign(m->es1, m->es1 + m->ne); c->es2.assign(m->es2, m->es2 + m->ne);
  c->iedge.assign(m->iedge, m->iedge + m->ne);
  c->t1.assign(m->t1, m->t1 + m->nt); c->t2.assign(m->t2, m->t2 + m->nt); c->t3.assign(m->t3, m->t3 + m->nt);
  c->cmx.assign(m->cmx, m->cmx + m->nt); c->cmy.assign(m->cmy, m->cmy + m->nt); c->cmz.assign(m->cmz, m->cmz + m->nt);
  c->tarea.assign(m->tarea, m->tarea + m->nt);
  c->Sarea0 = m->Sarea0; c->Volume0 = m->Volume0; c->theta0 = m->theta0;
  for (int k = 0; k < 3; ++k) c->center[k] = m->center[k];
  if ((int)c->x.size() != c->nv) alloc_vertices(c, c->nv);
  return 0;
}
extern "C" int orc_get_mesh(const orc_ctx* c, orc_mesh* m) {
  m->nv = c->nv; m->ne = c->ne; m->nt = c->nt;
  if (m->e1) { std::copy(c->e1.begin(), c->e1.end(), m->e1); std::copy(c->e2.begin(), c->e2.end(), m->e2);
    std::copy(c->l0.begin(), c->l0.end(), m->l0); std::copy(c->kappap.begin(), c->kappap.end(), m->kappap);
    std::copy(c->es1.begin(), c->es1.end(), m->es1); std::copy(c->es2.begin(), c->es2.end(), m->es2);
    std::copy(c->iedge.begin(), c->iedge.end(), m->iedge); }
  if (m->t1) { std::copy(c->t1.begin(), c->t1.end(), m->t1); std::copy(c->t2.begin(), c->t2.end(), m->t2);
    std::copy(c->t3.begin(), c->t3.end(), m->t3); std::copy(c->cmx.begin(), c->cmx.end(), m->cmx);
    std::copy(c->cmy.begin(), c->cmy.end(), m->cmy); std::copy(c->cmz.begin(), c->cmz.end(), m->cmz);
    std::copy(c->tarea.begin(), c->tarea.end(), m->tarea); }
  m->Sarea0 = c->Sarea0; m->Volume0 = c->Volume0; m->theta0 = c->theta0;
  for (int k = 0; k < 3; ++k) m->center[k] = c->center[k];
  return 0;
}

extern "C" int orc_set_state(orc_ctx* c, const orc_view* v) {
  if (v->ncell != c->ncell || v->nlig != c->nlig) return -1;
  alloc_solvent(c, v->ns);
  std::copy(v->sx, v->sx + v->ns, c->sx.begin()); std::copy(v->sy, v->sy + v->ns, c->sy.begin());
  std::copy(v->sz, v->sz + v->ns, c->sz.begin()); std::copy(v->svx, v->svx + v->ns, c->svx.begin());
  std::copy(v->svy, v->svy + v->ns, c->svy.begin()); std::copy(v->svz, v->svz + v->ns, c->svz.begin());
  std::copy(v->spid, v->spid + v->ns, c->spid.begin()); std::copy(v->sindio, v->sindio + v->ns, c->sindio.begin());
  int nv = v->nv;
  if ((int)c->x.size() != nv) alloc_vertices(c, nv);
  c->nv = nv;
  std::copy(v->x, v->x + nv, c->x.begin()); std::copy(v->y, v->y + nv, c->y.begin()); std::copy(v->z, v->z + nv, c->z.begin());
  std::copy(v->vx, v->vx + nv, c->vx.begin()); std::copy(v->vy, v->vy + nv, c->vy.begin()); std::copy(v->vz, v->vz + nv, c->vz.begin());
  std::copy(v->fx, v->fx + nv, c->fx.begin()); std::copy(v->fy, v->fy + nv, c->fy.begin()); std::copy(v->fz, v->fz + nv, c->fz.begin());
  std::copy(v->poff, v->poff + nv, c->poff.begin()); std::copy(v->pon, v->pon + nv, c->pon.begin());
  std::copy(v->pid, v->pid + nv, c->pid.begin()); std::copy(v->ix, v->ix + nv, c->ix.begin()); std::copy(v->iy, v->iy + nv, c->iy.begin());
  std::copy(v->bondi, v->bondi + nv, c->bondi.begin()); std::copy(v->bondl, v->bondl + nv, c->bondl.begin());
  std::copy(v->knob, v->knob + nv, c->knob.begin());
  for (int k = 0; k < 3; ++k) { c->para[k] = v->para[k]; c->paraV[k] = v->paraV[k]; c->paraft[k] = v->paraft[k]; c->parafdt[k] = v->parafdt[k]; }
  c->paradx = v->paradx; c->parady = v->parady; c->paraid = v->paraid;
  std::copy(v->ligi, v->ligi + c->nlig, c->ligi.begin());
  int64_t off = 0;
  for (int64_t i = 0; i < c->ncell; ++i) {
    c->llist[i].assign(v->lidx + off, v->lidx + off + v->llen[i]);
    off += v->llen[i];
  }
  c->Sarea = v->Sarea; c->Volume = v->Volume; c->wallspeed = v->wallspeed;
  c->step = v->step; c->colsteps = v->colsteps; c->upd = v->upd; c->filecc = v->filecc; c->filec = v->filec;
  return 0;
}
extern "C" int64_t orc_llist_total(const orc_ctx* c) {
  int64_t t = 0;
  for (auto& l : c->llist) t += (int64_t)l.size();
  return t;
}
extern "C" int orc_get_state(const orc_ctx* c, orc_view* v) {
  v->ns = c->ns; v->nv = c->nv; v->ncell = c->ncell; v->nlig = c->nlig;
  if (v->sx) {
    std::copy(c->sx.begin(), c->sx.end(), v->sx); std::copy(c->sy.begin(), c->sy.end(), v->sy);
    std::copy(c->sz.begin(), c->sz.end(), v->sz); std::copy(c->svx.begin(), c->svx.end(), v->svx);
    std::copy(c->svy.begin(), c->svy.end(), v->svy); std::copy(c->svz.begin(), c->svz.end(), v->svz);
    std::copy(c->spid.begin(), c->spid.end(), v->spid); std::copy(c->sindio.begin(), c->sindio.end(), v->sindio);
  }
  if (v->x) {
    std::copy(c->x.begin(), c->x.end(), v->x); std::copy(c->y.begin(), c->y.end(), v->y); std::copy(c->z.begin(), c->z.end(), v->z);
    std::copy(c->vx.begin(), c->vx.end(), v->vx); std::copy(c->vy.begin(), c->vy.end(), v->vy); std::copy(c->vz.begin(), c->vz.end(), v->vz);
    std::copy(c->fx.begin(), c->fx.end(), v->fx); std::copy(c->fy.begin(), c->fy.end(), v->fy); std::copy(c->fz.begin(), c->fz.end(), v->fz);
    std::copy(c->poff.begin(), c->poff.end(), v->poff); std::copy(c->pon.begin(), c->pon.end(), v->pon);
    std::copy(c->pid.begin(), c->pid.end(), v->pid); std::copy(c->ix.begin(), c->ix.end(), v->ix); std::copy(c->iy.begin(), c->iy.end(), v->iy);
    std::copy(c->bondi.begin(), c->bondi.end(), v->bondi); std::copy(c->bondl.begin(), c->bondl.end(), v->bondl);
    std::copy(c->knob.begin(), c->knob.end(), v->knob);
  }
  for (int k = 0; k < 3; ++k) { v->para[k] = c->para[k]; v->paraV[k] = c->paraV[k]; v->paraft[k] = c->paraft[k]; v->parafdt[k] = c->parafdt[k]; }
  v->paradx = c->paradx; v->parady = c->parady; v->paraid = c->paraid;
  if (v->ligi) std::copy(c->ligi.begin(), c->ligi.end(), v->ligi);
  if (v->llen) {
    int64_t off = 0;
    for (int64_t i = 0; i < c->ncell; ++i) {
      v->llen[i] = (int32_t)c->llist[i].size();
      if (v->lidx) {
        if (off + (int64_t)c->llist[i].size() > v->lcap) return -2;
        std::copy(c->llist[i].begin(), c->llist[i].end(), v->lidx + off);
      }
      off += (int64_t)c->llist[i].size();
    }
  }
  v->Sarea = c->Sarea; v->Volume = c->Volume; v->wallspeed = c->wallspeed;
  v->step = c->step; v->colsteps = c->colsteps; v->upd = c->upd; v->filecc = c->filecc; v->filec = c->filec;
  return 0;
}

// ------------------------------------------------------------------ collide
// CollisionStep (Src/solfuncs.cpp:109-323) with CollisionDyn/Dynmem/Dynpara
// (:700-810).  The grid shift and per-cell axes are the COLLIDE_U draws
// 0..2 and 3+2c, 4+2c; ghost normals are the COLLIDE_N draws in the order
// wall cells (ascending), then membrane cells (ascending), x, y, z each.
static inline void rotate(double v[3], const double vcm[3], double rand1, double rand2, double ThE,
                          double cosalpha, double sinalpha) {
  double thet = rand1, zz = rand2;
  double unit[3], dvv[3], dvp[3], dvn[3], dvpn[3];
  unit[0] = sqrt(1.0 - (zz * zz)) * cos(thet);
  unit[1] = sqrt(1.0 - (zz * zz)) * sin(thet);
  unit[2] = zz;
  double scalev = ThE;
  for (int k = 0; k < 3; ++k) dvv[k] = v[k] - vcm[k];
  double xxx = dvv[0] * unit[0] + dvv[1] * unit[1] + dvv[2] * unit[2];
  for (int k = 0; k < 3; ++k) dvp[k] = xxx * unit[k];
  for (int k = 0; k < 3; ++k) dvn[k] = dvv[k] - dvp[k];
  cp(dvn, unit, dvpn);
  for (int k = 0; k < 3; ++k) v[k] = vcm[k] + scalev * (cosalpha * dvn[k] + sinalpha * dvpn[k] + dvp[k]);
}

extern "C" void orc_collide(orc_ctx* c, int64_t epoch) {
  const orc_params& p = c->p;
  const int64_t C = c->ncell;
  uint64_t ucur = 0, ncur = 0;
  auto U = [&]() { return orc_uniform(c->seed, ORC_STREAM_COLLIDE_U, (uint64_t)epoch, ucur++); };
  auto N = [&](double m, double s) { return orc_normal(c->seed, ORC_STREAM_COLLIDE_N, (uint64_t)epoch, ncur++) * s + m; };
  double rpos[3];
  rpos[0] = p.a * U(); rpos[1] = p.a * U(); rpos[2] = p.a * U();
  vector<double> vcm(3 * C, 0.0), ncc(C, 0.0), dvv(C, 0.0), ThE(C, 0.0), r1(C), r2(C);
  vector<int> nc(C, 0), nmem(C, 0);
  // binning, :139-162
  vector<int64_t> start(C + 1, 0);
  for (int64_t i = 0; i < c->ns; ++i) {
    int fx = (int)floor(bbound(c->sx[i] - rpos[0], p.Lx));
    int fy = (int)floor(bbound(c->sy[i] - rpos[1], p.Ly));
    int fz = (int)floor(c->sz[i] - rpos[2] + 1.0);
    c->spid[i] = cell_of(c, fx, fy, fz);
  }
  for (int i = 0; i < c->nv; ++i) {
    int fx = (int)floor(bbound(c->x[i] - rpos[0], p.Lx));
    int fy = (int)floor(bbound(c->y[i] - rpos[1], p.Ly));
    int fz = (int)floor(c->z[i] - rpos[2] + 1.0);
    c->pid[i] = cell_of(c, fx, fy, fz);
    nmem[c->pid[i]] += 1;
  }
  {
    int fx = (int)floor(bbound(c->para[0] - rpos[0], p.Lx));
    int fy = (int)floor(bbound(c->para[1] - rpos[1], p.Ly));
    int fz = (int)floor(c->para[2] - rpos[2] + 1.0);
    c->paraid = cell_of(c, fx, fy, fz);
  }
  // per-cell solvent lists in particle order (counting sort, stable)
  for (int64_t i = 0; i < c->ns; ++i) start[c->spid[i] + 1] += 1;
  for (int64_t k = 0; k < C; ++k) start[k + 1] += start[k];
  vector<int64_t> sol(c->ns), fill(start.begin(), start.end() - 1);
  for (int64_t i = 0; i < c->ns; ++i) sol[fill[c->spid[i]]++] = i;
  // momentum of solvent, :164-176
  for (int64_t ii = 0; ii < C; ++ii) {
    for (int64_t q = start[ii]; q < start[ii + 1]; ++q) {
      int64_t pi = sol[q];
      vcm[3 * ii + 0] += p.mass * c->svx[pi];
      vcm[3 * ii + 1] += p.mass * c->svy[pi];
      vcm[3 * ii + 2] += p.mass * c->svz[pi];
      ncc[ii] += (1 * p.mass);
      nc[ii] += 1;
    }
  }
  // wall ghosts, :178-206
  for (int64_t i = 0; i < C; ++i) {
    double b[6]; cell_bounds(c, i, b);
    int nn = nc[i];
    if (b[5] >= p.Lz) {
      if (nn < p.navg) {
        vcm[3 * i + 0] += p.mass * N((p.navg - nn) * c->wallspeed, sqrt((p.navg - nn) * p.Theta / p.mass));
        vcm[3 * i + 1] += p.mass * N(0, sqrt((p.navg - nn) * p.Theta / p.mass));
        vcm[3 * i + 2] += p.mass * N(0, sqrt((p.navg - nn) * p.Theta / p.mass));
        ncc[i] = p.navg * p.mass;
      }
    } else if (b[4] <= 0) {
      if (nn < p.navg) {
        vcm[3 * i + 0] += p.mass * N(0, sqrt((p.navg - nn) * p.Theta / p.mass));
        vcm[3 * i + 1] += p.mass * N(0, sqrt((p.navg - nn) * p.Theta / p.mass));
        vcm[3 * i + 2] += p.mass * N(0, sqrt((p.navg - nn) * p.Theta / p.mass));
        ncc[i] = p.navg * p.mass;
      }
    }
  }
  // vertices, :208-220 (Cells[ii].mem is in vertex order)
  for (int i = 0; i < c->nv; ++i) {
    int ii = c->pid[i];
    vcm[3 * ii + 0] += p.pmass * c->vx[i];
    vcm[3 * ii + 1] += p.pmass * c->vy[i];
    vcm[3 * ii + 2] += p.pmass * c->vz[i];
    ncc[ii] += (1 * p.pmass);
    nc[ii] += 1;
  }
  // parasite, :223-228
  {
    int pi = c->paraid;
    vcm[3 * pi + 0] += p.PRmass * c->paraV[0];
    vcm[3 * pi + 1] += p.PRmass * c->paraV[1];
    vcm[3 * pi + 2] += p.PRmass * c->paraV[2];
    ncc[pi] += (1 * p.PRmass);
    nc[pi] += 1;
  }
  // membrane-cell ghosts, :230-245
  for (int64_t ii = 0; ii < C; ++ii) {
    int nn = nc[ii];
    if ((nn < p.navg) && (nmem[ii] > 0)) {
      vcm[3 * ii + 0] += p.mass * N(0, sqrt((p.navg - nn) * p.Theta / p.mass));
      vcm[3 * ii + 1] += p.mass * N(0, sqrt((p.navg - nn) * p.Theta / p.mass));
      vcm[3 * ii + 2] += p.mass * N(0, sqrt((p.navg - nn) * p.Theta / p.mass));
      ncc[ii] += (p.navg - nn) * p.mass;
    }
  }
  c->last_normals = ncur;
  // vcm /= (int)ncc, :248-261
  for (int64_t ii = 0; ii < C; ++ii) {
    int nn = (int)ncc[ii];
    if (nn != 0) {
      vcm[3 * ii + 0] /= (double)nn;
      vcm[3 * ii + 1] /= (double)nn;
      vcm[3 * ii + 2] /= (double)nn;
    }
  }
  // axes, :262-271
  for (int64_t i = 0; i < C; ++i) {
    r1[i] = 2.0 * p.Pi * U();
    r2[i] = -1.0 + (2.0 * U());
  }
  // relative kinetic energy, :273-307
  for (int64_t ii = 0; ii < C; ++ii) {
    for (int64_t q = start[ii]; q < start[ii + 1]; ++q) {
      int64_t pi = sol[q];
      double A0 = c->svx[pi] - vcm[3 * ii + 0];
      double A1 = c->svy[pi] - vcm[3 * ii + 1];
      double A2 = c->svz[pi] - vcm[3 * ii + 2];
      double aa = (A0 * A0 + A1 * A1 + A2 * A2);
      dvv[ii] += (p.mass * aa);
    }
  }
  for (int i = 0; i < c->nv; ++i) {
    int ii = c->pid[i];
    double A0 = c->vx[i] - vcm[3 * ii + 0];
    double A1 = c->vy[i] - vcm[3 * ii + 1];
    double A2 = c->vz[i] - vcm[3 * ii + 2];
    double aa = (A0 * A0 + A1 * A1 + A2 * A2);
    dvv[ii] += (p.pmass * aa);
  }
  {
    int pi = c->paraid;
    double A0 = c->paraV[0] - vcm[3 * pi + 0];
    double A1 = c->paraV[1] - vcm[3 * pi + 1];
    double A2 = c->paraV[2] - vcm[3 * pi + 2];
    double aa = (A0 * A0 + A1 * A1 + A2 * A2);
    dvv[pi] += (p.PRmass * aa);
  }
  // thermostat, :310-318
  for (int64_t i = 0; i < C; ++i) {
    ThE[i] = 1.0;
    if ((nc[i] > 0) && (dvv[i] != 0)) ThE[i] = sqrt(3.0 * ((double)nc[i] - 1.0) * p.Theta / (dvv[i]));
  }
  // rotations, :700-810
  for (int64_t i = 0; i < c->ns; ++i) {
    int pi = c->spid[i];
    double v[3] = {c->svx[i], c->svy[i], c->svz[i]};
    rotate(v, &vcm[3 * pi], r1[pi], r2[pi], ThE[pi], p.cosalpha, p.sinalpha);
    c->svx[i] = v[0]; c->svy[i] = v[1]; c->svz[i] = v[2];
  }
  for (int i = 0; i < c->nv; ++i) {
    int pi = c->pid[i];
    double v[3] = {c->vx[i], c->vy[i], c->vz[i]};
    rotate(v, &vcm[3 * pi], r1[pi], r2[pi], ThE[pi], p.cosalpha, p.sinalpha);
    c->vx[i] = v[0]; c->vy[i] = v[1]; c->vz[i] = v[2];
  }
  {
    int pi = c->paraid;
    rotate(c->paraV, &vcm[3 * pi], r1[pi], r2[pi], ThE[pi], p.cosalpha, p.sinalpha);
  }
}

// --------------------------------------------------------------- llist
// llistupdate (Src/solfuncs.cpp:326-365), including the stale tail: the
// list keeps max(old, new) entries and only the first `new` are rewritten.
extern "C" void orc_llist_update(orc_ctx* c) {
  const orc_params& p = c->p;
  for (int64_t i = 0; i < c->ncell; ++i) {
    double b[6]; cell_bounds(c, i, b);
    int count = 0;
    int nt = (int)c->llist[i].size();
    vector<int>& L = c->llist[i];
    for (int j = 0; j < c->nt; ++j) {
      int p1 = c->t1[j], p2 = c->t2[j], p3 = c->t3[j];
      double cellx = (b[0] + b[1]) * 0.5;
      double celly = (b[2] + b[3]) * 0.5;
      double cellz = (b[4] + b[5]) * 0.5;
      double xxx1 = fmod((((c->x[p1] + c->ix[p1] * p.Lx) + (c->x[p2] + c->ix[p2] * p.Lx) + (c->x[p3] + c->ix[p3] * p.Lx)) / 3.0), p.Lx) - cellx;
      double yyy1 = fmod((((c->y[p1] + c->iy[p1] * p.Ly) + (c->y[p2] + c->iy[p2] * p.Ly) + (c->y[p3] + c->iy[p3] * p.Ly)) / 3.0), p.Ly) - celly;
      xxx1 -= p.Lx * round(xxx1 / p.Lx);
      yyy1 -= p.Ly * round(yyy1 / p.Ly);
      double zzz = fabs(((c->z[p1] + c->z[p2] + c->z[p3]) / 3.0) - cellz);
      double A1aa = xxx1 * xxx1 + yyy1 * yyy1 + zzz * zzz;
      if (A1aa < 4.0 * p.a * p.a) {
        count += 1;
        if (count > nt) L.push_back(j);
        else L[count - 1] = j;
      }
    }
  }
}

// ------------------------------------------------------------- bounce-back
// SolveP3 (Src/poly34.cpp:26-55): trigonometric / Cardano cubic roots.
extern "C" int orc_solve_p3(double* x, double aa, double b, double c) {
  const double TwoPi = 6.28318530717958648;
  const double eps = 1e-14;
  double a2 = aa * aa;
  double q = (a2 - 3 * b) / 9;
  double r = (aa * (2 * a2 - 9 * b) + 27 * c) / 54;
  double r2 = r * r;
  double q3 = q * q * q;
  double A, B;
  if (r2 < q3) {
    double t = r / sqrt(q3);
    if (t < -1) t = -1;
    if (t > 1) t = 1;
    t = acos(t);
    aa /= 3; q = -2 * sqrt(q);
    x[0] = q * cos(t / 3) - aa;
    x[1] = q * cos((t + TwoPi) / 3) - aa;
    x[2] = q * cos((t - TwoPi) / 3) - aa;
    return 3;
  } else {
    A = -pow(fabs(r) + sqrt(r2 - q3), 1. / 3);
    if (r < 0) A = -A;
    B = (A == 0) ? 0 : q / A;
    aa /= 3;
    x[0] = (A + B) - aa;
    x[1] = -0.5 * (A + B) - aa;
    x[2] = 0.5 * sqrt(3.) * (A - B);
    if (fabs(x[2]) < eps) { x[2] = x[1]; return 2; }
    return 1;
  }
}
// Solve (Src/solfuncs.cpp:369-396) with dtmd as the window.
static double solve_tt(double aa, double bb, double cc, double dtmd) {
  double dt[3];
  int n = orc_solve_p3(dt, aa, bb, cc);
  double tt;
  if ((n == 3) || (n == 2)) {
    std::sort(dt, dt + 3);
    tt = dt[0];
    if ((tt < 0) || (tt > dtmd)) {
      tt = dt[1];
      if ((tt < 0) || (tt > dtmd)) tt = dt[2];
    }
  } else {
    tt = dt[0];
  }
  return tt;
}
extern "C" double orc_solve_cubic(double aa, double bb, double cc) { return solve_tt(aa, bb, cc, 0.002); }

// reflectionFed(i, 0.0) (Src/solfuncs.cpp:400-598).  The image offsets of
// the reference (:435-451) are all zero, so solv* is the particle position.
extern "C" double orc_reflection(orc_ctx* c, int64_t i) {
  const orc_params& p = c->p;
  const double rstep = 0.0, dtmd = p.dtmd, a = p.a, Lx = p.Lx, Ly = p.Ly;
  double fulldt = rstep;
  int fx = (int)floor(bbound(c->sx[i], Lx));
  int fy = (int)floor(bbound(c->sy[i], Ly));
  int fz = (int)floor(c->sz[i] + 1.0);
  int pid = cell_of(c, fx, fy, fz);
  const vector<int>& L = c->llist[pid];
  for (size_t j = 0; j < L.size(); ++j) {
    int flg = 0;
    int jj = L[j];
    int p1 = c->t1[jj], p2 = c->t2[jj], p3 = c->t3[jj];
    const int p1modx = 0, p2modx = 0, p3modx = 0, p1mody = 0, p2mody = 0, p3mody = 0;
    const int xx = 0, yy = 0;
    double solvx = c->sx[i] + xx * Lx;
    double solvy = c->sy[i] + yy * Ly;
    double solvz = c->sz[i];
    double A1[3], B1[3], C1[3], A2[3], B2[3], C2[3];
    double v1x = (c->x[p1] + p1modx * Lx) + c->vx[p1] * rstep;
    double v1y = (c->y[p1] + p1mody * Ly) + c->vy[p1] * rstep;
    double v1z = c->z[p1] + c->vz[p1] * rstep;
    double v2x = (c->x[p2] + p2modx * Lx) + c->vx[p2] * rstep;
    double v2y = (c->y[p2] + p2mody * Ly) + c->vy[p2] * rstep;
    double v2z = c->z[p2] + c->vz[p2] * rstep;
    double v3x = (c->x[p3] + p3modx * Lx) + c->vx[p3] * rstep;
    double v3y = (c->y[p3] + p3mody * Ly) + c->vy[p3] * rstep;
    double v3z = c->z[p3] + c->vz[p3] * rstep;
    double rstencilx = Lx - (3.0 * a), lstencilx = 3.0 * a;
    double rstencily = Ly - (3.0 * a), lstencily = 3.0 * a;
    if (solvx < lstencilx) {
      v1x -= (v1x > rstencilx) ? Lx : 0;
      v2x -= (v2x > rstencilx) ? Lx : 0;
      v3x -= (v3x > rstencilx) ? Lx : 0;
    } else if (solvx > rstencilx) {
      v1x += (v1x < lstencilx) ? Lx : 0;
      v2x += (v2x < lstencilx) ? Lx : 0;
      v3x += (v3x < lstencilx) ? Lx : 0;
    }
    if (solvy < lstencily) {
      v1y -= (v1y > rstencily) ? Ly : 0;
      v2y -= (v2y > rstencily) ? Ly : 0;
      v3y -= (v3y > rstencily) ? Ly : 0;
    } else if (solvy > rstencily) {
      v1y += (v1y < lstencily) ? Ly : 0;
      v2y += (v2y < lstencily) ? Ly : 0;
      v3y += (v3y < lstencily) ? Ly : 0;
    }
    A1[0] = v1x; A1[1] = v1y; A1[2] = v1z;
    B1[0] = v2x; B1[1] = v2y; B1[2] = v2z;
    C1[0] = v3x; C1[1] = v3y; C1[2] = v3z;
    double w1x = v1x + c->vx[p1] * (dtmd - rstep), w1y = v1y + c->vy[p1] * (dtmd - rstep), w1z = v1z + c->vz[p1] * (dtmd - rstep);
    double w2x = v2x + c->vx[p2] * (dtmd - rstep), w2y = v2y + c->vy[p2] * (dtmd - rstep), w2z = v2z + c->vz[p2] * (dtmd - rstep);
    double w3x = v3x + c->vx[p3] * (dtmd - rstep), w3y = v3y + c->vy[p3] * (dtmd - rstep), w3z = v3z + c->vz[p3] * (dtmd - rstep);
    A2[0] = w1x; A2[1] = w1y; A2[2] = w1z;
    B2[0] = w2x; B2[1] = w2y; B2[2] = w2z;
    C2[0] = w3x; C2[1] = w3y; C2[2] = w3z;
    // Normal (Src/memfuncs.cpp:96-108)
    double X[3], Xdt[3], t0[3], t1v[3];
    for (int k = 0; k < 3; ++k) { t0[k] = B1[k] - A1[k]; t1v[k] = C1[k] - A1[k]; }
    cp(t0, t1v, X);
    for (int k = 0; k < 3; ++k) { t0[k] = B2[k] - A2[k]; t1v[k] = C2[k] - A2[k]; }
    cp(t0, t1v, Xdt);
    double PSt[3], PSdt[3];
    PSt[0] = solvx - v1x; PSt[1] = solvy - v1y; PSt[2] = solvz - v1z;
    PSdt[0] = (solvx + c->svx[i] * (dtmd - rstep)) - w1x;
    PSdt[1] = (solvy + c->svy[i] * (dtmd - rstep)) - w1y;
    PSdt[2] = (solvz + c->svz[i] * (dtmd - rstep)) - w1z;
    double bt = X[0] * PSt[0] + X[1] * PSt[1] + X[2] * PSt[2];
    double bdt = Xdt[0] * PSdt[0] + Xdt[1] * PSdt[1] + Xdt[2] * PSdt[2];
    if ((c->sindio[i] == 1) && (bt < 0)) flg = 1;
    if ((c->sindio[i] == 0) && (bt > 0)) flg = 1;
    if ((bt * bdt <= 0) && (flg == 0)) {
      double a10[3], a20[3], d1[3], d2[3], a1[3], a2[3], b1[3], b2[3], b3[3], d11[3], d22[3];
      a10[0] = v2x - v1x; a10[1] = v2y - v1y; a10[2] = v2z - v1z;
      a20[0] = v3x - v1x; a20[1] = v3y - v1y; a20[2] = v3z - v1z;
      d1[0] = c->vx[p2] - c->vx[p1]; d1[1] = c->vy[p2] - c->vy[p1]; d1[2] = c->vz[p2] - c->vz[p1];
      d2[0] = c->vx[p3] - c->vx[p1]; d2[1] = c->vy[p3] - c->vy[p1]; d2[2] = c->vz[p3] - c->vz[p1];
      a1[0] = PSt[0]; a1[1] = PSt[1]; a1[2] = PSt[2];
      a2[0] = c->svx[i] - c->vx[p1]; a2[1] = c->svy[i] - c->vy[p1]; a2[2] = c->svz[i] - c->vz[p1];
      cp(a10, a20, b1);
      cp(a10, d2, d11);
      cp(d1, a20, d22);
      cp(d1, d2, b3);
      for (int k = 0; k < 3; ++k) b2[k] = d11[k] + d22[k];
      double a2b3 = a2[0] * b3[0] + a2[1] * b3[1] + a2[2] * b3[2];
      double a1b3 = a1[0] * b3[0] + a1[1] * b3[1] + a1[2] * b3[2];
      double a2b2 = a2[0] * b2[0] + a2[1] * b2[1] + a2[2] * b2[2];
      double a1b2 = a1[0] * b2[0] + a1[1] * b2[1] + a1[2] * b2[2];
      double a2b1 = a2[0] * b1[0] + a2[1] * b1[1] + a2[2] * b1[2];
      double a1b1 = a1[0] * b1[0] + a1[1] * b1[1] + a1[2] * b1[2];
      double tt = solve_tt((a1b3 + a2b2) / a2b3, (a1b2 + a2b1) / a2b3, a1b1 / a2b3, dtmd);
      double pd[3], vd[3];
      PSdt[0] = (solvx + c->svx[i] * tt) - (v1x + c->vx[p1] * tt);
      PSdt[1] = (solvy + c->svy[i] * tt) - (v1y + c->vy[p1] * tt);
      PSdt[2] = (solvz + c->svz[i] * tt) - (v1z + c->vz[p1] * tt);
      pd[0] = (solvx + c->svx[i] * tt);
      pd[1] = (solvy + c->svy[i] * tt);
      pd[2] = (solvz + c->svz[i] * tt);
      a10[0] = (v2x + c->vx[p2] * tt) - (v1x + c->vx[p1] * tt);
      a10[1] = (v2y + c->vy[p2] * tt) - (v1y + c->vy[p1] * tt);
      a10[2] = (v2z + c->vz[p2] * tt) - (v1z + c->vz[p1] * tt);
      a20[0] = (v3x + c->vx[p3] * tt) - (v1x + c->vx[p1] * tt);
      a20[1] = (v3y + c->vy[p3] * tt) - (v1y + c->vy[p1] * tt);
      a20[2] = (v3z + c->vz[p3] * tt) - (v1z + c->vz[p1] * tt);
      double pa1 = PSdt[0] * a10[0] + PSdt[1] * a10[1] + PSdt[2] * a10[2];
      double pa2 = PSdt[0] * a20[0] + PSdt[1] * a20[1] + PSdt[2] * a20[2];
      double a1a2 = a10[0] * a20[0] + a10[1] * a20[1] + a10[2] * a20[2];
      double a12 = a10[0] * a10[0] + a10[1] * a10[1] + a10[2] * a10[2];
      double a22 = a20[0] * a20[0] + a20[1] * a20[1] + a20[2] * a20[2];
      double den = (a12 * a22) - (a1a2 * a1a2);
      double eta = ((pa1 * a22) - (pa2 * a1a2)) / den;
      double zeta = ((pa2 * a12) - (pa1 * a1a2)) / den;
      if ((eta >= 0) && (zeta >= 0) && (eta + zeta <= 1) && (tt < (dtmd - rstep))) {
        fulldt += tt;
        vd[0] = (1.0 - eta - zeta) * c->vx[p1] + eta * c->vx[p2] + zeta * c->vx[p3];
        vd[1] = (1.0 - eta - zeta) * c->vy[p1] + eta * c->vy[p2] + zeta * c->vy[p3];
        vd[2] = (1.0 - eta - zeta) * c->vz[p1] + eta * c->vz[p2] + zeta * c->vz[p3];
        c->svx[i] = 2.0 * vd[0] - c->svx[i];
        c->svy[i] = 2.0 * vd[1] - c->svy[i];
        c->svz[i] = 2.0 * vd[2] - c->svz[i];
        c->sx[i] = pd[0]; c->sy[i] = pd[1]; c->sz[i] = pd[2];
      }
    }
  }
  return fulldt;
}

// streaming with walls, maincode.cpp:510-562
extern "C" void orc_stream(orc_ctx* c) {
  const orc_params& p = c->p;
  const double dtmd = p.dtmd;
  for (int64_t i = 0; i < c->ns; ++i) {
    double fullts = orc_reflection(c, i);
    double& X = c->sx[i]; double& Y = c->sy[i]; double& Z = c->sz[i];
    double& VX = c->svx[i]; double& VY = c->svy[i]; double& VZ = c->svz[i];
    X += VX * (dtmd - fullts);
    Y += VY * (dtmd - fullts);
    Z += VZ * (dtmd - fullts);
    double ul = p.Lz, ll = 0;
    double A[3], B[3];
    if (Z > ul) {
      A[0] = X - VX * (dtmd - fullts); A[1] = Y - VY * (dtmd - fullts); A[2] = Z - VZ * (dtmd - fullts);
      double s = (ul - A[2]) / (Z - A[2]);
      B[0] = A[0] + s * (X - A[0]); B[1] = A[1] + s * (Y - A[1]); B[2] = A[2] + s * (Z - A[2]);
      double dist = sqrt(((B[0] - A[0]) * (B[0] - A[0])) + ((B[1] - A[1]) * (B[1] - A[1])) + ((B[2] - A[2]) * (B[2] - A[2])));
      double dtt = dist / sqrt((VX * VX) + (VY * VY) + (VZ * VZ));
      VX = c->wallspeed; VY = 0; VZ = 0;
      X = B[0] + VX * ((dtmd - fullts) - dtt);
      Y = B[1] + VY * ((dtmd - fullts) - dtt);
      Z = B[2] + VZ * ((dtmd - fullts) - dtt);
    } else if (Z < ll) {
      A[0] = X - VX * (dtmd - fullts); A[1] = Y - VY * (dtmd - fullts); A[2] = Z - VZ * (dtmd - fullts);
      double s = (ll - A[2]) / (Z - A[2]);
      B[0] = A[0] + s * (X - A[0]); B[1] = A[1] + s * (Y - A[1]); B[2] = A[2] + s * (Z - A[2]);
      double dist = sqrt(((B[0] - A[0]) * (B[0] - A[0])) + ((B[1] - A[1]) * (B[1] - A[1])) + ((B[2] - A[2]) * (B[2] - A[2])));
      double dtt = dist / sqrt((VX * VX) + (VY * VY) + (VZ * VZ));
      VX *= -1.0; VY *= -1.0; VZ *= -1.0;
      X = B[0] + VX * ((dtmd - fullts) - dtt);
      Y = B[1] + VY * ((dtmd - fullts) - dtt);
      Z = B[2] + VZ * ((dtmd - fullts) - dtt);
    }
    X = bbound(X, p.Lx);
    Y = bbound(Y, p.Ly);
  }
}

// ---------------------------------------------------------------- membrane
// TotalVA (Src/memfuncs.cpp:161-190)
extern "C" void orc_total_va(orc_ctx* c) {
  double totA = 0, totV = 0;
  for (int i = 0; i < c->nt; ++i) totA += areatri(c, c->t1[i], c->t2[i], c->t3[i]);
  c->Sarea = totA;
  for (int i = 0; i < c->nt; ++i) totV += voltri(c, c->t1[i], c->t2[i], c->t3[i]);
  c->Volume = totV;
}

// pfdt (Src/memfuncs.cpp:443-484): parasite-vertex WCA
extern "C" void orc_pfdt(orc_ctx* c) {
  const orc_params& p = c->p;
  double cutoff = p.paraR, epsilon = 0.1, sigma = 0.890898718 * cutoff;
  double fx = 0, fy = 0, fz = 0, A[3], X[3];
  for (int i = 0; i < c->nv; ++i) {
    A[0] = (c->para[0] + c->paradx * p.Lx) - (c->x[i] + c->ix[i] * p.Lx);
    A[1] = (c->para[1] + c->parady * p.Ly) - (c->y[i] + c->iy[i] * p.Ly);
    A[2] = c->para[2] - c->z[i];
    double aa = A[0] * A[0] + A[1] * A[1] + A[2] * A[2];
    if (aa <= cutoff * cutoff) {
      double ex = (sigma * sigma * sigma * sigma * sigma * sigma) / (aa * aa * aa);
      X[0] = (24.0 * epsilon / aa) * ((2.0 * ex * ex) - ex) * A[0];
      X[1] = (24.0 * epsilon / aa) * ((2.0 * ex * ex) - ex) * A[1];
      X[2] = (24.0 * epsilon / aa) * ((2.0 * ex * ex) - ex) * A[2];
      fx += X[0]; fy += X[1]; fz += X[2];
      c->fx[i] -= X[0]; c->fy[i] -= X[1]; c->fz[i] -= X[2];
    }
  }
  c->parafdt[0] += fx; c->parafdt[1] += fy; c->parafdt[2] += fz;
}

// force_calculate_dt (Src/memfuncs.cpp:214-441), one thread: ff accumulates
// edges, then triangles, then dihedrals, and is added to fmapdt at the end.
extern "C" void orc_forces(orc_ctx* c) {
  const orc_params& p = c->p;
  const int nv = c->nv;
  vector<double> ffx(nv, 0.0), ffy(nv, 0.0), ffz(nv, 0.0);
  double A[3], A21[3], A13[3], A32[3], B[3], eta[3], C[3];
  double a21[3], a31[3], a24[3], a34[3], zeta[3], t1[3], t2[3], a32[3], D[3], fact;
  double b11, b12, b22, E[3], F[3];
  int l2 = 0, l3 = 0;
  const double elap = p.elap;
  for (int i = 0; i < c->ne; ++i) {
    int l1 = c->e1[i], m2 = c->e2[i];
    double l0 = c->l0[i];
    A[0] = UX(l1) - UX(m2); A[1] = UY(l1) - UY(m2); A[2] = c->z[l1] - c->z[m2];
    double aa = sqrt(A[0] * A[0] + A[1] * A[1] + A[2] * A[2]);
    A[0] /= aa; A[1] /= aa; A[2] /= aa;
    double xx = aa / (2.5 * l0);
    double xxx = 1.0 / (4.0 * (1.0 - xx) * (1.0 - xx));
    ffx[l1] += (-1.0 / (elap)) * (xxx - 0.25 + xx) * A[0];
    ffy[l1] += (-1.0 / (elap)) * (xxx - 0.25 + xx) * A[1];
    ffz[l1] += (-1.0 / (elap)) * (xxx - 0.25 + xx) * A[2];
    ffx[m2] += (1.0 / (elap)) * (xxx - 0.25 + xx) * A[0];
    ffy[m2] += (1.0 / (elap)) * (xxx - 0.25 + xx) * A[1];
    ffz[m2] += (1.0 / (elap)) * (xxx - 0.25 + xx) * A[2];
    ffx[l1] += c->kappap[i] * A[0] / (aa * aa);
    ffy[l1] += c->kappap[i] * A[1] / (aa * aa);
    ffz[l1] += c->kappap[i] * A[2] / (aa * aa);
    ffx[m2] += -c->kappap[i] * A[0] / (aa * aa);
    ffy[m2] += -c->kappap[i] * A[1] / (aa * aa);
    ffz[m2] += -c->kappap[i] * A[2] / (aa * aa);
  }
  for (int i = 0; i < c->nt; ++i) {
    int l1 = c->t1[i], m2 = c->t2[i], m3 = c->t3[i];
    double beta = -p.kappasa * (c->Sarea - c->Sarea0) / c->Sarea0;
    double betav = -p.kappav * (c->Volume - c->Volume0) / (c->Volume0);
    double area = areatri(c, l1, m2, m3);
    double alpha = beta / (4.0 * area);
    double alphad = -p.kappad * (area - c->tarea[i]) / (4.0 * c->tarea[i] * area);
    A21[0] = UX(m2) - UX(l1); A21[1] = UY(m2) - UY(l1); A21[2] = c->z[m2] - c->z[l1];
    A13[0] = UX(l1) - UX(m3); A13[1] = UY(l1) - UY(m3); A13[2] = c->z[l1] - c->z[m3];
    A32[0] = UX(m3) - UX(m2); A32[1] = UY(m3) - UY(m2); A32[2] = c->z[m3] - c->z[m2];
    cp(A13, A21, eta);
    cp(eta, A32, C);
    ffx[l1] += alpha * C[0]; ffy[l1] += alpha * C[1]; ffz[l1] += alpha * C[2];
    ffx[l1] += alphad * C[0]; ffy[l1] += alphad * C[1]; ffz[l1] += alphad * C[2];
    cp(eta, A13, C);
    ffx[m2] += alpha * C[0]; ffy[m2] += alpha * C[1]; ffz[m2] += alpha * C[2];
    ffx[m2] += alphad * C[0]; ffy[m2] += alphad * C[1]; ffz[m2] += alphad * C[2];
    cp(eta, A21, C);
    ffx[m3] += alpha * C[0]; ffy[m3] += alpha * C[1]; ffz[m3] += alpha * C[2];
    ffx[m3] += alphad * C[0]; ffy[m3] += alphad * C[1]; ffz[m3] += alphad * C[2];
    B[0] = (UX(l1) + UX(m2) + UX(m3)) / 3.0;
    B[1] = (UY(l1) + UY(m2) + UY(m3)) / 3.0;
    B[2] = (c->z[l1] + c->z[m2] + c->z[m3]) / 3.0;
    cp(B, A32, C);
    ffx[l1] += betav * ((eta[0] / 3.0) + C[0]) / 6.0;
    ffy[l1] += betav * ((eta[1] / 3.0) + C[1]) / 6.0;
    ffz[l1] += betav * ((eta[2] / 3.0) + C[2]) / 6.0;
    cp(B, A13, C);
    ffx[m2] += betav * ((eta[0] / 3.0) + C[0]) / 6.0;
    ffy[m2] += betav * ((eta[1] / 3.0) + C[1]) / 6.0;
    ffz[m2] += betav * ((eta[2] / 3.0) + C[2]) / 6.0;
    cp(B, A21, C);
    ffx[m3] += betav * ((eta[0] / 3.0) + C[0]) / 6.0;
    ffy[m3] += betav * ((eta[1] / 3.0) + C[1]) / 6.0;
    ffz[m3] += betav * ((eta[2] / 3.0) + C[2]) / 6.0;
  }
  const double cth0 = cos(c->theta0 * p.Pi / 180.0), sth0 = sin(c->theta0 * p.Pi / 180.0);
  for (int i = 0; i < c->ne; ++i) {
    if (c->iedge[i] == 1) { l2 = c->e1[i]; l3 = c->e2[i]; }
    if (c->iedge[i] == -1) { l3 = c->e1[i]; l2 = c->e2[i]; }
    int l1 = c->es1[i], l4 = c->es2[i];
    a21[0] = UX(l2) - UX(l1); a21[1] = UY(l2) - UY(l1); a21[2] = c->z[l2] - c->z[l1];
    a31[0] = UX(l3) - UX(l1); a31[1] = UY(l3) - UY(l1); a31[2] = c->z[l3] - c->z[l1];
    a24[0] = UX(l2) - UX(l4); a24[1] = UY(l2) - UY(l4); a24[2] = c->z[l2] - c->z[l4];
    a34[0] = UX(l3) - UX(l4); a34[1] = UY(l3) - UY(l4); a34[2] = c->z[l3] - c->z[l4];
    a32[0] = UX(l3) - UX(l2); a32[1] = UY(l3) - UY(l2); a32[2] = c->z[l3] - c->z[l2];
    t1[0] = (UX(l1) + UX(l2) + UX(l3)) / 3.0;
    t1[1] = (UY(l1) + UY(l2) + UY(l3)) / 3.0;
    t1[2] = (c->z[l1] + c->z[l2] + c->z[l3]) / 3.0;
    t2[0] = (UX(l4) + UX(l2) + UX(l3)) / 3.0;
    t2[1] = (UY(l4) + UY(l2) + UY(l3)) / 3.0;
    t2[2] = (c->z[l4] + c->z[l2] + c->z[l3]) / 3.0;
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
    fact = (factor >= 0.0) ? 1.0 : -1.0;
    sinth = fact * sinth;
    double betab = p.kappab * (sinth * cth0 - costh * sth0) / sinth;
    b11 = -(betab * costh) / (etam * etam);
    b22 = -(betab * costh) / (zetam * zetam);
    b12 = betab / (etam * zetam);
    cp(eta, a32, C);
    cp(zeta, a32, D);
    ffx[l1] += b11 * C[0] + b12 * D[0];
    ffy[l1] += b11 * C[1] + b12 * D[1];
    ffz[l1] += b11 * C[2] + b12 * D[2];
    ffx[l4] += -b12 * C[0] - b22 * D[0];
    ffy[l4] += -b12 * C[1] - b22 * D[1];
    ffz[l4] += -b12 * C[2] - b22 * D[2];
    cp(eta, a31, C);
    cp(zeta, a31, D);
    cp(eta, a34, E);
    cp(zeta, a34, F);
    ffx[l2] += -b11 * C[0] + b12 * (E[0] - D[0]) + b22 * F[0];
    ffy[l2] += -b11 * C[1] + b12 * (E[1] - D[1]) + b22 * F[1];
    ffz[l2] += -b11 * C[2] + b12 * (E[2] - D[2]) + b22 * F[2];
    cp(eta, a21, C);
    cp(zeta, a21, D);
    cp(eta, a24, E);
    cp(zeta, a24, F);
    ffx[l3] += b11 * C[0] + b12 * (-E[0] + D[0]) - b22 * F[0];
    ffy[l3] += b11 * C[1] + b12 * (-E[1] + D[1]) - b22 * F[1];
    ffz[l3] += b11 * C[2] + b12 * (-E[2] + D[2]) - b22 * F[2];
  }
  for (int i = 0; i < nv; ++i) { c->fx[i] += ffx[i]; c->fy[i] += ffy[i]; c->fz[i] += ffz[i]; }
}

// liglist membership of ligand j in cell `cell` (maincode.cpp:138-154)
static inline bool in_liglist(const orc_ctx* c, int cell, int j) {
  double b[6]; cell_bounds(c, cell, b);
  if (!(b[5] <= 2.0)) return false;
  double A0 = fabs(((b[0] + b[1]) * 0.5) - c->xlig[j]);
  double A1 = fabs(((b[2] + b[3]) * 0.5) - c->ylig[j]);
  A0 -= c->p.Lx * round(A0 / c->p.Lx);
  A1 -= c->p.Ly * round(A1 / c->p.Ly);
  return (A0 < 1.5) && (A1 < 1.5);
}

// bond preparation, maincode.cpp:668-723
static void bond_prep(orc_ctx* c) {
  const orc_params& p = c->p;
  for (int ii = 0; ii < c->nv; ++ii) {
    double A[3], B[3];
    if (c->bondi[ii] == 1) {
      int p1modx = c->ix[ii], p1mody = c->iy[ii], jj = c->bondl[ii];
      A[0] = (c->x[ii] + p1modx * p.Lx) - (c->xlig[jj] + p1modx * p.Lx);
      A[1] = (c->y[ii] + p1mody * p.Ly) - (c->ylig[jj] + p1mody * p.Ly);
      A[2] = c->z[ii] - 0.0;
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
      c->poff[ii] = 1.0 - exp(-koff * p.dtmd);
    } else if ((c->z[ii] < p.dthr) && (c->bondi[ii] == 0) && (c->knob[ii] == 1)) {
      auto& P = c->pairs[ii];
      P.clear();
      int pid = c->pid[ii];
      double kon = p.onrate;
      c->pon[ii] = 1.0 - exp(-kon * p.dtmd);
      for (int j = 0; j < c->nlig; ++j) {
        if (!in_liglist(c, pid, j)) continue;
        int p1modx = c->ix[ii], p1mody = c->iy[ii];
        A[0] = (c->x[ii] + p1modx * p.Lx) - (c->xlig[j] + p1modx * p.Lx);
        A[1] = (c->y[ii] + p1mody * p.Ly) - (c->ylig[j] + p1mody * p.Ly);
        A[2] = c->z[ii] - 0.0;
        double aaa = (A[0] * A[0] + A[1] * A[1] + A[2] * A[2]);
        if (aaa <= p.dthr * p.dthr) P.push_back(std::make_pair(aaa, j));
      }
      std::sort(P.begin(), P.end());
    }
  }
}

// bond_dynamics (maincode.cpp:16-54), draws from the BOND stream in order
extern "C" void orc_bond_dynamics(orc_ctx* c, int64_t epoch) {
  const orc_params& p = c->p;
  uint64_t k = 0;
  for (int ii = 0; ii < c->nv; ++ii) {
    if (c->bondi[ii] == 1) {
      double randoff = orc_uniform(c->seed, ORC_STREAM_BOND, (uint64_t)epoch, k++);
      int jj = c->bondl[ii];
      if (c->poff[ii] > randoff) {
        c->bondi[ii] = 0;
        c->bondl[ii] = p.randno;
        c->ligi[jj] = 0;
      }
    } else if ((c->z[ii] < p.dthr) && (c->bondi[ii] == 0) && (c->knob[ii] == 1)) {
      for (size_t jkl = 0; jkl < c->pairs[ii].size(); ++jkl) {
        int j = c->pairs[ii][jkl].second;
        double pon = c->pon[ii];
        double randon = orc_uniform(c->seed, ORC_STREAM_BOND, (uint64_t)epoch, k++);
        if ((pon > randon) && (c->ligi[j] == 0)) {
          c->ligi[j] = 1;
          c->bondi[ii] = 1;
          c->bondl[ii] = j;
        }
      }
    }
  }
  c->last_bond_draws = k;
}

// ---------------------------------------------------------------- the step
// maincode.cpp:462-602
extern "C" void orc_step_part1(orc_ctx* c) {
  const orc_params& p = c->p;
  const int64_t s = c->step;
  c->wallspeed = (s < p.warm_steps) ? p.warm_speed : p.walls;
  c->colsteps += 1; c->bbi += 1; c->upd += 1;
  if (s > 0) c->filecc += 1;
  if (c->colsteps == c->csteps) { orc_collide(c, s); c->colsteps = 0; }
  for (int i = 0; i < c->nv; ++i) {  // :487-496
    c->vx[i] += (c->fx[i] * p.dtmd / (2.0 * p.pmass));
    c->vy[i] += (c->fy[i] * p.dtmd / (2.0 * p.pmass));
    c->vz[i] += (c->fz[i] * p.dtmd / (2.0 * p.pmass));
    c->fx[i] = 0.0; c->fy[i] = 0.0; c->fz[i] = 0.0;
  }
  if (c->upd == c->uplist) { orc_llist_update(c); c->upd = 0; }
  orc_stream(c);
  for (int i = 0; i < c->nv; ++i) {  // :566-574 with bboundmx/my (Src/solfuncs.cpp:625-659)
    c->x[i] += (c->vx[i] * p.dtmd);
    c->y[i] += (c->vy[i] * p.dtmd);
    c->z[i] += (c->vz[i] * p.dtmd);
    if (c->x[i] > p.Lx) { c->x[i] -= p.Lx; c->ix[i] += 1; }
    if (c->x[i] < 0) { c->x[i] += p.Lx; c->ix[i] -= 1; }
    if (c->y[i] > p.Ly) { c->y[i] -= p.Ly; c->iy[i] += 1; }
    if (c->y[i] < 0) { c->y[i] += p.Ly; c->iy[i] -= 1; }
  }
  for (int k = 0; k < 3; ++k)  // :576-578
    c->para[k] += (c->paraV[k] * p.dtmd) + (c->paraft[k] * p.dtmd * p.dtmd / (2.0 * p.PRmass));
  if (c->para[0] > p.Lx) { c->para[0] -= p.Lx; c->paradx += 1; }
  else if (c->para[0] < 0) { c->para[0] += p.Lx; c->paradx -= 1; }
  if (c->para[1] > p.Ly) { c->para[1] -= p.Ly; c->parady += 1; }
  else if (c->para[1] < 0) { c->para[1] += p.Ly; c->parady -= 1; }
  orc_total_va(c);
}

// maincode.cpp:603-762
extern "C" void orc_step_part2(orc_ctx* c) {
  const orc_params& p = c->p;
  const int64_t s = c->step;
  orc_pfdt(c);
  orc_forces(c);
  for (int i = 0; i < c->nv; ++i) c->fz[i] += -p.Fg / (double)c->nv;  // :606-610
  for (int i = 0; i < c->nv; ++i) {  // :612-640
    if (c->bondi[i] == 1) {
      int jj = c->bondl[i];
      double A[3], B1[3];
      A[0] = c->x[i] - c->xlig[jj];
      A[1] = c->y[i] - c->ylig[jj];
      A[2] = c->z[i];
      A[0] -= p.Lx * round(A[0] / p.Lx);
      A[1] -= p.Ly * round(A[1] / p.Ly);
      double aa = sqrt(A[0] * A[0] + A[1] * A[1] + A[2] * A[2]);
      A[0] /= aa; A[1] /= aa; A[2] /= aa;
      if (aa > p.el0) {
        B1[0] = -p.ks * (aa - p.el0) * A[0];
        B1[1] = -p.ks * (aa - p.el0) * A[1];
        B1[2] = -p.ks * (aa - p.el0) * A[2];
        c->fx[i] += B1[0]; c->fy[i] += B1[1]; c->fz[i] += B1[2];
      }
    }
  }
  for (int i = 0; i < c->nv; ++i) {  // :643-653
    double cc = c->z[i];
    if (cc < 0.5) c->fz[i] += 300.0 * exp(-50.0 * cc);
  }
  for (int i = 0; i < c->nv; ++i) {  // :655-665
    double cc = p.Lz - c->z[i];
    if (cc < 0.5) c->fz[i] -= 300.0 * exp(-50.0 * cc);
  }
  bond_prep(c);
  orc_bond_dynamics(c, s);
  for (int i = 0; i < c->nv; ++i) {  // :727-733
    c->vx[i] += (c->fx[i] * p.dtmd / (2.0 * p.pmass));
    c->vy[i] += (c->fy[i] * p.dtmd / (2.0 * p.pmass));
    c->vz[i] += (c->fz[i] * p.dtmd / (2.0 * p.pmass));
  }
  for (int k = 0; k < 3; ++k) c->paraV[k] += ((c->paraft[k] + c->parafdt[k]) * p.dtmd / (2.0 * p.PRmass));
  for (int k = 0; k < 3; ++k) { c->paraft[k] = c->parafdt[k]; c->parafdt[k] = 0.0; }
  if (c->filecc == p.out_every) { c->filec += 1; c->filecc = 0; }
  c->step = s + 1;
}

extern "C" void orc_step(orc_ctx* c, int64_t n) {
  for (int64_t k = 0; k < n; ++k) { orc_step_part1(c); orc_step_part2(c); }
}

// ------------------------------------------------------------------ output
// RBCdata record (maincode.cpp:749-753)
extern "C" int orc_write_rbcdata(const orc_ctx* c, const char* path, int append) {
  FILE* f = fopen(path, append ? "a" : "w");
  if (!f) return -1;
  fprintf(f, "#%d\n", c->filec);
  for (int i = 0; i < c->nv; ++i)
    fprintf(f, "%lf\t%lf\t%lf\t%d\t%d\t%d\n", c->x[i], c->y[i], c->z[i], c->ix[i], c->iy[i], c->bondi[i]);
  fclose(f);
  return 0;
}
// STL writer (Src/memfuncs.cpp:590-626)
extern "C" int orc_write_stl(const orc_ctx* c, const char* path) {
  std::ofstream f(path);
  if (!f) return -1;
  f << "solid ascii" << std::endl;
  for (int kk = 0; kk < c->nt; ++kk) {
    int l1 = c->t1[kk], l2 = c->t2[kk], l3 = c->t3[kk];
    double N[3];
    normaldt(c, l1, l2, l3, N);
    f << "facet normal" << "\t" << N[0] << "\t" << N[1] << "\t" << N[2] << std::endl;
    f << "outer loop" << std::endl;
    f << "vertex" << "\t" << UX(l1) << "\t" << UY(l1) << "\t" << c->z[l1] << std::endl;
    f << "vertex" << "\t" << UX(l2) << "\t" << UY(l2) << "\t" << c->z[l2] << std::endl;
    f << "vertex" << "\t" << UX(l3) << "\t" << UY(l3) << "\t" << c->z[l3] << std::endl;
    f << "endloop" << std::endl;
    f << "endfacet" << std::endl;
  }
  f << "endsolid" << std::endl;
  return 0;
}
