/*
 * oracle/irbc_oracle.h -- TEST INFRASTRUCTURE: the CPU oracle.
 *
 * A single-threaded CPU restatement of the reference timestep
 * (Dasanna/iRBC-code maincode.cpp:461-764 and the functions it calls in
 * Src/solfuncs.cpp, Src/memfuncs.cpp, Src/poly34.cpp).  It exists only to
 * check the CUDA library: tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg may load it; the shipped library never does.
 *
 * Every arithmetic expression keeps the reference's operand order so that,
 * built with the same compiler flags (IEEE double, no FMA contraction), the
 * oracle reproduces the compiled reference bit for bit.  That is checked by
 * tests/test_oracle_vs_ref.py against the reference compiled from its own
 * sources (oracle/Makefile, target `ref`).
 *
 * Random numbers come from the counter stream in oracle/irbc_rng.h, consumed
 * in exactly the order the reference consumes its Mersenne Twister draws
 * with one OpenMP thread.
 */
#ifndef IRBC_ORACLE_H
#define IRBC_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Runtime copy of the compile-time parameters of define.h:35-73 plus the
 * constants hard-coded in main (maincode.cpp:347-348, 460-470, 746). */
typedef struct orc_params {
  double a, Lx, Ly, Lz;          /* define.h:42-45 */
  int64_t Ns;                    /* define.h:46 */
  double dtcd, navg, Theta, walls, mass, cosalpha, sinalpha; /* define.h:47-54 */
  int32_t Nt;                    /* define.h:57 */
  double kappasa, kappad, kappav, kappab, pmass, dtmd, ks, dthr, FD, Fg, el0; /* define.h:59-69 */
  double PRmass, paraR;          /* define.h:72-73 */
  double Pi;                     /* define.h:35 (3.141592653) */
  double elap, shear;            /* maincode.cpp:347-348 */
  double onrate, offrate;        /* argv[1], argv[2] */
  int64_t warm_steps;            /* maincode.cpp:463 (250000) */
  double warm_speed;             /* maincode.cpp:465 (0.1) */
  int64_t out_every;             /* maincode.cpp:746 (5000) */
  int32_t randno;                /* define.h:37 (12345678) */
  int32_t pad_;
} orc_params;

/* Static membrane topology after set-up (maincode.cpp:227-391). */
typedef struct orc_mesh {
  int32_t nv, ne, nt, pad_;
  int32_t *e1, *e2;          /* edges[].l1/l2 (0-based)            */
  double *l0, *kappap;       /* edges[].l0, edges[].kappap         */
  int32_t *es1, *es2;        /* edgest[].l1/l2                      */
  int32_t *iedge;            /* iedge[]                             */
  int32_t *t1, *t2, *t3;     /* tries[].l1/l2/l3                    */
  double *cmx, *cmy, *cmz;   /* tries[].cm* (tricm)                 */
  double *tarea;             /* tarea[]                             */
  double Sarea0, Volume0, theta0;
  double center[3];
} orc_mesh;

/* Dynamic state.  The llist (cell -> triangle lists, Src/solfuncs.cpp:326)
 * is exported as per-cell lengths llen[ncell] plus the concatenated entries
 * lidx[] in cell order. */
typedef struct orc_view {
  int64_t ns;
  double *sx, *sy, *sz, *svx, *svy, *svz;
  int32_t *spid, *sindio;
  int32_t nv, pad0_;
  double *x, *y, *z, *vx, *vy, *vz, *fx, *fy, *fz, *poff, *pon;
  int32_t *pid, *ix, *iy, *bondi, *bondl, *knob;
  double para[3], paraV[3], paraft[3], parafdt[3];
  int32_t paradx, parady, paraid, nlig;
  int32_t *ligi;
  int64_t ncell;
  int32_t *llen;
  int64_t lcap;              /* capacity of lidx (entries)  */
  int32_t *lidx;
  double Sarea, Volume, wallspeed;
  /* loop counters of maincode.cpp:450-455 and the next step index */
  int64_t step;
  int32_t colsteps, upd, filecc, filec;
} orc_view;

typedef struct orc_ctx orc_ctx;

void orc_params_default(orc_params* p);
orc_ctx* orc_create(const orc_params* p, uint64_t seed);
void orc_destroy(orc_ctx* c);

/* --- set-up (maincode.cpp:77-446) --------------------------------------- */
/* Places the raw mesh, builds edges/edgest/iedge/kappap/tarea, draws vertex
 * and parasite velocities, computes init forces.  V is nv*3 raw coordinates,
 * E ne*2 and T nt*3 0-based indices.  Draws from the INIT stream continue
 * from where orc_init_solvent left off, as in main. */
int orc_init(orc_ctx* c, const double* V, int32_t nv, const int32_t* E, int32_t ne,
             const int32_t* T, int32_t nt, int32_t nknobs, int32_t do_sort);
/* Diagnostics printed by main (maincode.cpp:256-257, 345-346, 366-368, 446):
 * out[0..8] = mean edge, std edge, Sarea0, Volume0, shear, young, poisson,
 * knob count, theta0. */
void orc_init_report(const orc_ctx* c, double out[9]);

int orc_set_mesh(orc_ctx* c, const orc_mesh* m);
int orc_get_mesh(const orc_ctx* c, orc_mesh* m);
int orc_set_state(orc_ctx* c, const orc_view* v);
int64_t orc_llist_total(const orc_ctx* c);
int orc_get_state(const orc_ctx* c, orc_view* v);

/* --- phases ---------------------------------------------------------------- */
void orc_collide(orc_ctx* c, int64_t epoch);          /* CollisionStep */
void orc_llist_update(orc_ctx* c);                    /* llistupdate   */
void orc_stream(orc_ctx* c);                          /* maincode.cpp:510-562 */
double orc_reflection(orc_ctx* c, int64_t i);         /* reflectionFed(i, 0) */
void orc_total_va(orc_ctx* c);                        /* TotalVA       */
void orc_pfdt(orc_ctx* c);                            /* pfdt          */
void orc_forces(orc_ctx* c);                          /* force_calculate_dt */
void orc_bond_dynamics(orc_ctx* c, int64_t epoch);    /* bond_dynamics */
/* Whole step split where the reference calls TotalVA (maincode.cpp:602):
 * part 1 = :462-602 (counters .. TotalVA), part 2 = :603-762. */
void orc_step_part1(orc_ctx* c);
void orc_step_part2(orc_ctx* c);
void orc_step(orc_ctx* c, int64_t n);

/* cubic root selection Solve (Src/solfuncs.cpp:369-396) and SolveP3
 * (Src/poly34.cpp:26-55), exported for unit tests */
double orc_solve_cubic(double aa, double bb, double cc);
int orc_solve_p3(double* x, double aa, double b, double c);

/* Membrane output formats (maincode.cpp:749-753, Src/memfuncs.cpp:590-626). */
int orc_write_rbcdata(const orc_ctx* c, const char* path, int append);
int orc_write_stl(const orc_ctx* c, const char* path);

/* cell count of the collision grid and draws consumed so far */
int64_t orc_ncell(const orc_ctx* c);
uint64_t orc_last_normals(const orc_ctx* c);
uint64_t orc_last_bond_draws(const orc_ctx* c);

#ifdef __cplusplus
}
#endif
#endif
