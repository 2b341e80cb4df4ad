/*
 * oracle/ref_hooks.cpp -- TEST INFRASTRUCTURE, linked only into the
 * reference build under oracle/_ref/ (see oracle/Makefile).
 *
 * The reference's main() (maincode.cpp:56-770) is compiled unchanged except
 * that, through -D on the command line, its calls to TotalVA, CollisionStep,
 * llistupdate and sortsolvent_initial1 land on the hooks below, and main is
 * renamed irbc_ref_main.  Each hook calls the reference's own function and
 * then lets the harness
 *   - select the draw stream the next phase consumes (ref_replay_rng.cpp),
 *   - hand a snapshot of the global state to the caller once per step
 *     (right after TotalVA, maincode.cpp:602), and
 *   - stop the run after a given number of steps (by a C++ exception thrown
 *     from serial code, which unwinds main normally).
 * The state accessors copy the reference's globals (define.h:182-429) into
 * the oracle's view structs so the tests can compare them field by field.
 */
#include "define.h"
// compile-time parameters of this build (define.h:35-73), captured before
// the macros are removed so they cannot collide with field names below
namespace refc {
const double Pi_ = Pi;
const double Theta_ = Theta;
const long randno_ = randno;
const double a_ = a;
const double Lx_ = Lx;
const double Ly_ = Ly;
const double Lz_ = Lz;
const long Ns_ = Ns;
const double dtcd_ = dtcd;
const double navg_ = navg;
const double walls_ = walls;
const double mass_ = mass;
const double cosalpha_ = cosalpha;
const double sinalpha_ = sinalpha;
const long Nt_ = Nt;
const double kappasa_ = kappasa;
const double kappad_ = kappad;
const double kappav_ = kappav;
const double kappab_ = kappab;
const double pmass_ = pmass;
const double dtmd_ = dtmd;
const double ks_ = ks;
const double dthr_ = dthr;
const double FD_ = FD;
const double Fg_ = Fg;
const double el0_ = el0;
const double PRmass_ = PRmass;
const double paraR_ = paraR;
}  // namespace refc
#undef Pi
#undef Theta
#undef randno
#undef a
#undef Lx
#undef Ly
#undef Lz
#undef Ns
#undef dtcd
#undef navg
#undef walls
#undef mass
#undef cosalpha
#undef sinalpha
#undef Nt
#undef kappasa
#undef kappad
#undef kappav
#undef kappab
#undef pmass
#undef dtmd
#undef ks
#undef dthr
#undef FD
#undef Fg
#undef el0
#undef PRmass
#undef paraR
#include "irbc_oracle.h"
#include "irbc_rng.h"

#include <chrono>
#include <cstring>
#include <exception>

int irbc_ref_main(int argc, char* argv[]);
void bond_dynamics();

// The draw-stream controls exist only in the replay builds (linked with
// ref_replay_rng.cpp); the timing builds keep the reference's own RNG.
extern "C" void ref_rng_seed(uint64_t seed) __attribute__((weak));
extern "C" void ref_rng_set_uniform(uint32_t stream, uint64_t epoch) __attribute__((weak));
extern "C" void ref_rng_set_normal(uint32_t stream, uint64_t epoch) __attribute__((weak));
extern "C" uint64_t ref_rng_uniform_cursor() __attribute__((weak));
extern "C" uint64_t ref_rng_normal_cursor() __attribute__((weak));
#define RNG_CALL(f, ...) do { if (f) f(__VA_ARGS__); } while (0)

typedef void (*ref_cb_t)(int64_t step);

namespace {
struct StopRun {};
int64_t g_calls = 0;        // TotalVA calls so far (0 = the init call)
int64_t g_stop_step = -1;   // throw after the snapshot of this step
ref_cb_t g_cb = nullptr;
int g_fast_init = 0;
int g_llist_calls = 0;
double g_t0 = 0;
double g_step_time[1 << 16];
int64_t g_nstep_times = 0;

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

int64_t current_step() { return g_calls - 1; }

void reset_globals() {
  RanGen.clear(); sto.clear(); vts.clear(); vtso.clear(); edges.clear(); edgest.clear();
  iedge.clear(); tries.clear(); tarea.clear(); fmapdt.clear(); solvent.clear(); Cells.clear();
  xlig.clear(); ylig.clear(); ligi.clear();
  std::memset(cindex, 0, sizeof(cindex));
  for (int k = 0; k < 3; ++k) para[k] = paraV[k] = paraft[k] = parafdt[k] = 0;
  paradx = parady = paraid = 0; Sarea = Volume = Sarea0 = Volume0 = 0; wallspeed = 0;
}
}  // namespace

// ---- hooks (called from maincode.cpp through -D renames) -------------------
void irbc_hook_TotalVA() {
  TotalVA();
  int64_t k = g_calls++;
  if (k == 0) return;  // maincode.cpp:385, during set-up
  int64_t s = k - 1;
  if (g_nstep_times < (1 << 16)) g_step_time[g_nstep_times++] = now_s();
  // everything RanGen draws after this point in step s is bond_dynamics
  RNG_CALL(ref_rng_set_uniform, ORC_STREAM_BOND, (uint64_t)s);
  if (g_cb) g_cb(s);
  if (g_stop_step >= 0 && s >= g_stop_step) throw StopRun();
}

void irbc_hook_CollisionStep() {
  // TotalVA has run once at set-up and once per finished step, so the step
  // in progress is g_calls - 1
  uint64_t s = (uint64_t)current_step();
  RNG_CALL(ref_rng_set_uniform, ORC_STREAM_COLLIDE_U, s);
  RNG_CALL(ref_rng_set_normal, ORC_STREAM_COLLIDE_N, s);
  CollisionStep();
}

void irbc_hook_llistupdate() {
  g_llist_calls++;
  llistupdate();
}

// sortsolvent_initial1 (Src/solfuncs.cpp:17-106).  With fast_init the
// classification loop runs over OpenMP threads (each particle is
// independent, so the flags are the same) before the reference's own sort.
void irbc_hook_sortsolvent_initial1() {
  if (!g_fast_init) { sortsolvent_initial1(); return; }
  const long n = (long)solvent.size();
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; ++i) {
    double Q1[3], Q2[3], X[3], P0[3];
    int count = 0;
    Q1[0] = solvent[i].xpos + 1.0 * 0.3; Q1[1] = solvent[i].ypos + 0.0 * 0.3; Q1[2] = solvent[i].zpos + 0.0 * 0.3;
    Q2[0] = solvent[i].xpos + 1.0 * 0.7; Q2[1] = solvent[i].ypos + 0.0 * 0.7; Q2[2] = solvent[i].zpos + 0.0 * 0.7;
    for (unsigned j = 0; j < tries.size(); ++j) {
      int p1 = tries[j].l1, p2 = tries[j].l2, p3 = tries[j].l3;
      Normaldt(p1, p2, p3, X);
      double dotP1Q1 = (vts[p1].x - Q1[0]) * X[0] + (vts[p1].y - Q1[1]) * X[1] + (vts[p1].z - Q1[2]) * X[2];
      double dotQ2Q1 = (Q2[0] - Q1[0]) * X[0] + (Q2[1] - Q1[1]) * X[1] + (Q2[2] - Q1[2]) * X[2];
      for (int k = 0; k < 3; ++k) P0[k] = Q1[k] + ((dotP1Q1 / dotQ2Q1) * (Q2[k] - Q1[k]));
      double P2P1[3] = {vts[p2].x - vts[p1].x, vts[p2].y - vts[p1].y, vts[p2].z - vts[p1].z};
      double P3P2[3] = {vts[p3].x - vts[p2].x, vts[p3].y - vts[p2].y, vts[p3].z - vts[p2].z};
      double P1P3[3] = {vts[p1].x - vts[p3].x, vts[p1].y - vts[p3].y, vts[p1].z - vts[p3].z};
      double P0P1[3] = {P0[0] - vts[p1].x, P0[1] - vts[p1].y, P0[2] - vts[p1].z};
      double P0P2[3] = {P0[0] - vts[p2].x, P0[1] - vts[p2].y, P0[2] - vts[p2].z};
      double P0P3[3] = {P0[0] - vts[p3].x, P0[1] - vts[p3].y, P0[2] - vts[p3].z};
      double f1[3], f2[3], f3[3];
      cp(P2P1, P0P1, f1); cp(P3P2, P0P2, f2); cp(P1P3, P0P3, f3);
      double ch1 = f1[0] * X[0] + f1[1] * X[1] + f1[2] * X[2];
      double ch2 = f2[0] * X[0] + f2[1] * X[1] + f2[2] * X[2];
      double ch3 = f3[0] * X[0] + f3[1] * X[1] + f3[2] * X[2];
      if ((ch1 >= 0) && (ch2 >= 0) && (ch3 >= 0) && (tries[j].cmx >= solvent[i].xpos)) count += 1;
    }
    solvent[i].indio = ((count % 2) == 0) ? 1 : 0;
  }
  sort(solvent.begin(), solvent.end());
}

// ---- run control --------------------------------------------------------------
extern "C" int ref_run(int argc, char** argv, int64_t stop_step, ref_cb_t cb, uint64_t seed,
                       int fast_init) {
  reset_globals();
  g_calls = 0; g_stop_step = stop_step; g_cb = cb; g_fast_init = fast_init;
  g_llist_calls = 0; g_nstep_times = 0;
  RNG_CALL(ref_rng_seed, seed);
  RNG_CALL(ref_rng_set_uniform, ORC_STREAM_INIT, 0);
  RNG_CALL(ref_rng_set_normal, ORC_STREAM_COLLIDE_N, 0);
  g_t0 = now_s();
  try {
    irbc_ref_main(argc, argv);
  } catch (const StopRun&) {
    return 0;
  }
  return 1;  // main returned on its own (4e6 steps)
}
extern "C" int64_t ref_step_times(double* out, int64_t cap) {
  int64_t n = g_nstep_times < cap ? g_nstep_times : cap;
  for (int64_t i = 0; i < n; ++i) out[i] = g_step_time[i] - g_t0;
  return n;
}
extern "C" int ref_llist_calls() { return g_llist_calls; }
extern "C" void ref_set_threads(int n) { omp_set_num_threads(n); }
extern "C" int ref_max_threads() { return omp_get_max_threads(); }
extern "C" uint64_t ref_uniform_cursor() { return ref_rng_uniform_cursor ? ref_rng_uniform_cursor() : 0; }
extern "C" uint64_t ref_normal_cursor() { return ref_rng_normal_cursor ? ref_rng_normal_cursor() : 0; }

// ---- compiled-in parameters (define.h:35-73, maincode.cpp:347-348) -----------
extern "C" void ref_get_params(orc_params* p) {
  using namespace refc;
  std::memset(p, 0, sizeof(*p));
  p->shear = 1200.0;      // maincode.cpp:348
  p->warm_steps = 250000; // maincode.cpp:463
  p->warm_speed = 0.1;    // maincode.cpp:465
  p->out_every = 5000;    // maincode.cpp:746
  p->a = a_; p->Lx = Lx_; p->Ly = Ly_; p->Lz = Lz_; p->Ns = Ns_;
  p->dtcd = dtcd_; p->navg = navg_; p->Theta = Theta_; p->walls = walls_; p->mass = mass_;
  p->cosalpha = cosalpha_; p->sinalpha = sinalpha_; p->Nt = (int32_t)Nt_;
  p->kappasa = kappasa_; p->kappad = kappad_; p->kappav = kappav_; p->kappab = kappab_;
  p->pmass = pmass_; p->dtmd = dtmd_; p->ks = ks_; p->dthr = dthr_; p->FD = FD_; p->Fg = Fg_;
  p->el0 = el0_; p->PRmass = PRmass_; p->paraR = paraR_; p->Pi = Pi_;
  p->elap = 0.0005;       // maincode.cpp:347 (set inside main)
  p->onrate = onrate; p->offrate = offrate;  // argv[1..2] once main has run
  p->randno = (int32_t)randno_;
}

// ---- state accessors -------------------------------------------------------
extern "C" void ref_get_mesh(orc_mesh* m) {
  m->nv = (int)vts.size(); m->ne = (int)edges.size(); m->nt = (int)tries.size();
  if (m->e1) for (int i = 0; i < m->ne; ++i) {
    m->e1[i] = edges[i].l1; m->e2[i] = edges[i].l2; m->l0[i] = edges[i].l0; m->kappap[i] = edges[i].kappap;
    m->es1[i] = edgest[i].l1; m->es2[i] = edgest[i].l2; m->iedge[i] = iedge[i];
  }
  if (m->t1) for (int i = 0; i < m->nt; ++i) {
    m->t1[i] = tries[i].l1; m->t2[i] = tries[i].l2; m->t3[i] = tries[i].l3;
    m->cmx[i] = tries[i].cmx; m->cmy[i] = tries[i].cmy; m->cmz[i] = tries[i].cmz; m->tarea[i] = tarea[i];
  }
  m->Sarea0 = Sarea0; m->Volume0 = Volume0; m->theta0 = theta0;
  for (int k = 0; k < 3; ++k) m->center[k] = center[k];
}

extern "C" int64_t ref_llist_total() {
  int64_t t = 0;
  for (auto& c : Cells) t += (int64_t)c.llist.size();
  return t;
}

extern "C" int ref_get_state(orc_view* v, int64_t s) {
  v->ns = (int64_t)solvent.size(); v->nv = (int)vts.size(); v->ncell = (int64_t)Cells.size();
  v->nlig = (int)ligi.size();
  if (v->sx) for (int64_t i = 0; i < v->ns; ++i) {
    const particle& q = solvent[i];
    v->sx[i] = q.xpos; v->sy[i] = q.ypos; v->sz[i] = q.zpos;
    v->svx[i] = q.vx; v->svy[i] = q.vy; v->svz[i] = q.vz; v->spid[i] = q.pid; v->sindio[i] = q.indio;
  }
  if (v->x) for (int i = 0; i < v->nv; ++i) {
    const vert& q = vts[i];
    v->x[i] = q.x; v->y[i] = q.y; v->z[i] = q.z; v->vx[i] = q.vx; v->vy[i] = q.vy; v->vz[i] = q.vz;
    v->fx[i] = fmapdt[i].fx; v->fy[i] = fmapdt[i].fy; v->fz[i] = fmapdt[i].fz;
    v->poff[i] = q.poff; v->pon[i] = q.pon; v->pid[i] = q.pid; v->ix[i] = q.ix; v->iy[i] = q.iy;
    v->bondi[i] = q.bondi; v->bondl[i] = q.bondl; v->knob[i] = q.knob;
  }
  for (int k = 0; k < 3; ++k) { v->para[k] = para[k]; v->paraV[k] = paraV[k]; v->paraft[k] = paraft[k]; v->parafdt[k] = parafdt[k]; }
  v->paradx = paradx; v->parady = parady; v->paraid = paraid;
  if (v->ligi) for (int j = 0; j < v->nlig; ++j) v->ligi[j] = ligi[j];
  if (v->llen) {
    int64_t off = 0;
    for (int64_t i = 0; i < v->ncell; ++i) {
      const auto& L = Cells[i].llist;
      v->llen[i] = (int32_t)L.size();
      if (v->lidx) {
        if (off + (int64_t)L.size() > v->lcap) return -2;
        for (size_t j = 0; j < L.size(); ++j) v->lidx[off + j] = L[j];
      }
      off += (int64_t)L.size();
    }
  }
  v->Sarea = Sarea; v->Volume = Volume; v->wallspeed = wallspeed;
  // loop counters of main at the TotalVA point of step s (maincode.cpp:450-484)
  const int csteps = (int)(refc::dtcd_ / refc::dtmd_), uplist = (int)(0.5 / (refc::walls_ * refc::dtmd_));
  v->step = s;
  v->colsteps = (int)(s % csteps);
  v->upd = (int)((s + 1) % uplist);
  v->filecc = s == 0 ? 0 : (int)(((s - 1) % 5000) + 1);
  v->filec = s == 0 ? 0 : (int)((s - 1) / 5000);
  return 0;
}

extern "C" int ref_set_state(const orc_view* v) {
  if (v->ncell != (int64_t)Cells.size() || v->nlig != (int)ligi.size() || v->nv != (int)vts.size()) return -1;
  solvent.resize(v->ns);
  for (int64_t i = 0; i < v->ns; ++i) {
    particle& q = solvent[i];
    q.xpos = v->sx[i]; q.ypos = v->sy[i]; q.zpos = v->sz[i];
    q.vx = v->svx[i]; q.vy = v->svy[i]; q.vz = v->svz[i]; q.pid = v->spid[i]; q.indio = v->sindio[i];
  }
  for (int i = 0; i < v->nv; ++i) {
    vert& q = vts[i];
    q.x = v->x[i]; q.y = v->y[i]; q.z = v->z[i]; q.vx = v->vx[i]; q.vy = v->vy[i]; q.vz = v->vz[i];
    fmapdt[i].fx = v->fx[i]; fmapdt[i].fy = v->fy[i]; fmapdt[i].fz = v->fz[i];
    q.poff = v->poff[i]; q.pon = v->pon[i]; q.pid = v->pid[i]; q.ix = v->ix[i]; q.iy = v->iy[i];
    q.bondi = v->bondi[i]; q.bondl = v->bondl[i]; q.knob = v->knob[i];
  }
  for (int k = 0; k < 3; ++k) { para[k] = v->para[k]; paraV[k] = v->paraV[k]; paraft[k] = v->paraft[k]; parafdt[k] = v->parafdt[k]; }
  paradx = v->paradx; parady = v->parady; paraid = v->paraid;
  for (int j = 0; j < v->nlig; ++j) ligi[j] = v->ligi[j];
  int64_t off = 0;
  for (int64_t i = 0; i < v->ncell; ++i) {
    Cells[i].llist.assign(v->lidx + off, v->lidx + off + v->llen[i]);
    off += v->llen[i];
  }
  Sarea = v->Sarea; Volume = v->Volume; wallspeed = v->wallspeed;
  return 0;
}

// ---- direct calls of the reference's functions (one thread) -----------------
extern "C" void ref_call_collide(uint64_t epoch) {
  RNG_CALL(ref_rng_set_uniform, ORC_STREAM_COLLIDE_U, epoch);
  RNG_CALL(ref_rng_set_normal, ORC_STREAM_COLLIDE_N, epoch);
  CollisionStep();
}
extern "C" void ref_call_llist() { llistupdate(); }
extern "C" void ref_call_totalva() { TotalVA(); }
extern "C" void ref_call_pfdt() { pfdt(); }
extern "C" void ref_call_forces() { force_calculate_dt(); }
extern "C" double ref_call_reflection(int i) { return reflectionFed(i, 0.0); }
extern "C" double ref_call_solve(double aa, double bb, double cc) { return Solve(aa, bb, cc); }
extern "C" int ref_call_solvep3(double* x, double aa, double b, double c) { return SolveP3(x, aa, b, c); }
extern "C" void ref_call_bond_dynamics(uint64_t epoch) {
  RNG_CALL(ref_rng_set_uniform, ORC_STREAM_BOND, epoch);
  bond_dynamics();
}
extern "C" void ref_call_filewrite(const char* path) {
  char buf[1024];
  std::strncpy(buf, path, sizeof(buf) - 1); buf[sizeof(buf) - 1] = 0;
  filewrite(buf);
}
