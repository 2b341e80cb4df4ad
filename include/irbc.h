/*
 * irbc.h -- C ABI of the B200 iRBC timestep library (libirbc.so).
 *
 * Drop-in for the step of Dasanna/iRBC-code.  The reference has no library
 * interface: its step is the loop body of main() (maincode.cpp:461-764)
 * acting on the globals of define.h:182-429 through the void functions of
 * Include/solfuncs.h:19-30 and Include/memfuncs.h:49-64.  Each entry point
 * below names the reference code it replaces.  A handle owns all device
 * memory of one simulation; one host thread drives a handle at a time;
 * handles are independent.  Every call returns 0 on success or a negative
 * status; irbc_last_error() gives the message.  Sizes are plain integers,
 * arrays are caller-owned host memory, nothing here exposes CUDA or torch
 * types.
 */
#ifndef IRBC_H
#define IRBC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define IRBC_OK 0
#define IRBC_ERR_ARG -1      /* invalid argument or size                    */
#define IRBC_ERR_CUDA -2     /* CUDA runtime error (device fault, no device)  */
#define IRBC_ERR_STATE -3    /* call out of order (no mesh, no solvent)       */
#define IRBC_ERR_CAPACITY -4 /* a list outgrew its capacity                   */
#define IRBC_ERR_IO -5       /* file could not be written                     */
#define IRBC_ERR_HEALTH -6   /* the state went bad: non-finite or out of box   */

#define IRBC_FP64 0          /* all solvent arithmetic in double               */
#define IRBC_FP32 1          /* solvent state and arithmetic in float          */

/* Runtime form of the compile-time parameters of define.h:35-73, the
 * constants main() hard-codes (maincode.cpp:347-348, 463-470, 746) and the
 * argv values (maincode.cpp:73-74).  irbc_params_default() fills the
 * define.h values. */
typedef struct irbc_params {
  double a, Lx, Ly, Lz;          /* define.h:42-45                 */
  int64_t Ns;                    /* define.h:46                    */
  double dtcd, navg, Theta, walls, mass, cosalpha, sinalpha; /* define.h:47-54 */
  int32_t Nt;                    /* define.h:57 (vertex count)     */
  double kappasa, kappad, kappav, kappab, pmass, dtmd, ks, dthr, FD, Fg, el0; /* :59-69 */
  double PRmass, paraR;          /* define.h:72-73                 */
  double Pi;                     /* define.h:35 (3.141592653)      */
  double elap, shear;            /* maincode.cpp:347-348           */
  double onrate, offrate;        /* argv[1], argv[2]               */
  int64_t warm_steps;            /* maincode.cpp:463 (250000)      */
  double warm_speed;             /* maincode.cpp:465 (0.1)         */
  int64_t out_every;             /* maincode.cpp:746 (5000)        */
  int32_t randno;                /* define.h:37 (12345678)         */
  int32_t pad_;
  /* not in the reference */
  uint64_t seed;                 /* key of the Philox draw stream  */
  int32_t precision;             /* IRBC_FP64 or IRBC_FP32         */
  int32_t device;                /* CUDA device ordinal            */
} irbc_params;

/* Static membrane topology (maincode.cpp:227-391): edges, edgest (bending
 * partners), iedge, triangles with centroids (tricm) and rest areas. */
typedef struct irbc_mesh {
  int32_t nv, ne, nt, pad_;
  int32_t *e1, *e2;
  double *l0, *kappap;
  int32_t *es1, *es2, *iedge;
  int32_t *t1, *t2, *t3;
  double *cmx, *cmy, *cmz, *tarea;
  double Sarea0, Volume0, theta0;
  double center[3];
} irbc_mesh;

/* Dynamic state in the reference's layout (define.h:82-139 fields as SoA).
 * Solvent arrays are in the reference's particle order.  The cell ->
 * triangle lists (Cells[].llist) are llen[ncell] plus their concatenation
 * lidx[] (capacity lcap).  A NULL array pointer skips that group. */
typedef struct irbc_view {
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
  int64_t lcap;
  int32_t *lidx;
  double Sarea, Volume, wallspeed;
  int64_t step;
  int32_t colsteps, upd, filecc, filec;
} irbc_view;

typedef struct irbc_handle irbc_handle;

/* ---- lifecycle --------------------------------------------------------- */
void irbc_params_default(irbc_params* p);              /* define.h:35-73 */
/* Allocates the simulation on p->device.  Replaces the global definitions of
 * define.h:182-429 and the grid build of maincode.cpp:112-154. */
int irbc_create(const irbc_params* p, irbc_handle** out);
void irbc_destroy(irbc_handle* h);
/* the message of h's last error; with h = NULL, why the calling thread's last
 * irbc_create failed */
const char* irbc_last_error(const irbc_handle* h);
/* bytes of device memory a simulation with these parameters needs (for
 * admission by HBM footprint); nv/ne/nt are the mesh sizes */
int64_t irbc_footprint_bytes(const irbc_params* p, int32_t nv, int32_t ne, int32_t nt);

/* ---- set-up (maincode.cpp:94-446) -----------------------------------------
 * V: nv*3 raw vertex coordinates as read from the vertex file; E: ne*2 and
 * T: nt*3 zero-based indices.  Places the cell (maincode.cpp:196-206), builds
 * edges/edgest/iedge/kappap/tarea (:239-375), draws vertex, parasite and
 * solvent velocities and positions from the INIT stream, classifies the
 * solvent inside/outside (Src/solfuncs.cpp:17-94, on the GPU), builds the
 * cell lists (llistupdate) and places the knobs (:394-433). */
int irbc_init(irbc_handle* h, const double* V, int32_t nv, const int32_t* E, int32_t ne,
              const int32_t* T, int32_t nt, int32_t nknobs);
/* diagnostics main() prints during set-up (maincode.cpp:256-257, 345-346,
 * 366-368, 446): mean edge, std edge, Sarea0, Volume0, shear, Young,
 * Poisson, knob count, theta0 */
int irbc_init_report(const irbc_handle* h, double out[9]);

/* ---- state exchange ---------------------------------------------------- */
int irbc_set_mesh(irbc_handle* h, const irbc_mesh* m);
int irbc_get_mesh(irbc_handle* h, irbc_mesh* m);
int irbc_set_state(irbc_handle* h, const irbc_view* v);
int irbc_get_state(irbc_handle* h, irbc_view* v);
int64_t irbc_llist_total(irbc_handle* h);
int64_t irbc_ncell(const irbc_handle* h);
int32_t irbc_nlig(const irbc_handle* h);

/* ---- the step ---------------------------------------------------------------
 * irbc_step runs n reference timesteps (maincode.cpp:461-764).  The split
 * entry points run the halves either side of the TotalVA call at
 * maincode.cpp:602 (part 1 = :462-602, part 2 = :603-762). */
int irbc_step(irbc_handle* h, int64_t n);
/* Not in the reference.  on = 1: irbc_step launches whole 24-step
 * stretches between list updates as one captured CUDA graph; on = 0 (the
 * default) launches every kernel on the two streams.  The results are the
 * same either way. */
int irbc_set_graphs(irbc_handle* h, int32_t on);
/* Not in the reference.  n = 2 (the default): the membrane kernels run on a
 * second, high-priority stream beside the solvent kernels; n = 1: every
 * kernel of the handle runs on its one stream.  One stream suits many small
 * simulations sharing a GPU (fewer streams contend for the device's
 * hardware queues); the results are the same either way. */
int irbc_set_streams(irbc_handle* h, int32_t n);
/* Not in the reference.  How irbc_step launches the membrane step: mode 1
 * (the default) as wide kernels over many SMs; mode 2 as one block per
 * launch, two kernels per step instead of eight, for meshes up to 1024
 * vertices (IRBC_ERR_CAPACITY for a larger mesh; a mesh set later keeps
 * the wide kernels); mode 3 as one launch of a thread-block cluster (8
 * blocks of 512 threads on one GPC, its phases separated by cluster
 * barriers), any mesh.  The results are the same in every mode. */
int irbc_set_membrane_kernels(irbc_handle* h, int32_t mode);
int irbc_step_part1(irbc_handle* h);
int irbc_step_part2(irbc_handle* h);

/* ---- single phases ------------------------------------------------------------ */
int irbc_collide(irbc_handle* h, int64_t epoch);   /* CollisionStep, Src/solfuncs.cpp:109-323 */
int irbc_llist_update(irbc_handle* h);             /* llistupdate, Src/solfuncs.cpp:326-365 */
int irbc_stream(irbc_handle* h);                   /* maincode.cpp:510-562 + reflectionFed */
int irbc_total_va(irbc_handle* h);                 /* TotalVA, Src/memfuncs.cpp:161-190 */
int irbc_pfdt(irbc_handle* h);                     /* pfdt, Src/memfuncs.cpp:443-484 */
int irbc_forces(irbc_handle* h);                   /* force_calculate_dt, Src/memfuncs.cpp:214-441 */
int irbc_bond_dynamics(irbc_handle* h, int64_t epoch); /* bond prep + bond_dynamics, maincode.cpp:668-725,16-54 */

/* ---- standalone binning ------------------------------------------------------------
 * Random-shift cell binning of CollisionStep (Src/solfuncs.cpp:139-147) for
 * particles held in DEVICE memory: x, y, z[n] device arrays, shift (rx, ry,
 * rz) in [0, 1).  Writes, all device arrays: cell[n] (the particle's cell
 * index, cindex semantics), start[C+1] (exclusive scan of the per-cell
 * counts, C = Lx*Ly*(Lz+1)) and order[n] (particle indices grouped by cell,
 * ascending within a cell: the Cells[].sol lists).  Uses the box of p.
 * Scratch memory is taken with cudaMalloc and released before returning. */
int irbc_bin_particles(const irbc_params* p, const double* x, const double* y, const double* z,
                       int64_t n, double rx, double ry, double rz, int32_t* cell, int32_t* start,
                       int32_t* order);

/* No counterpart in the reference.  The binning of irbc_bin_particles for
 * callers that cannot allocate device memory while they run (code inside an
 * allocator callback or memory-pool hook, threads that must not take the
 * driver's allocation lock, embedders with a fixed device-memory budget).
 * Same arguments and results; allocates nothing.  Its scratch is a fixed
 * static device array (4 MiB plus 12 KiB) that every GPU loading the library
 * keeps until the process exits, so boxes are limited to 1,048,576 cells
 * (Lx*Ly*(Lz+1)); larger boxes return IRBC_ERR_CAPACITY.  The first call on
 * a device looks up the array's device address and keeps it for the life of
 * the process; make that first call before any stream capture, and do not
 * use this entry point on a device after cudaDeviceReset (which can move
 * the array).  All calls share the one array, so calls that overlap
 * on the GPU (other host threads, other streams) race; this one runs on the
 * legacy default stream and returns after it has finished. */
int irbc_bin_particles_noalloc(const irbc_params* p, const double* x, const double* y, const double* z,
                               int64_t n, double rx, double ry, double rz, int32_t* cell, int32_t* start,
                               int32_t* order);

/* ---- output (formats of maincode.cpp:749-753 and Src/memfuncs.cpp:590-626) ---- */
int irbc_write_rbcdata(irbc_handle* h, const char* path, int32_t append);
int irbc_write_stl(irbc_handle* h, const char* path);
/* Not in the reference: the fields of the RBCdata record (vertex x, y, z,
 * ix, iy, bondi; maincode.cpp:749-753) copied to a host buffer without
 * waiting.  The layout is x[nv], y[nv], z[nv] (double) then ix[nv], iy[nv],
 * bondi[nv] (int32): irbc_record_bytes(h) bytes.  The copy is queued on
 * the handle's stream after the steps queued so far and the call returns
 * at once; the buffer holds the record once irbc_sync(h) returns.  `host`
 * should be page-locked (irbc_host_alloc) for the copy to run
 * asynchronously. */
int64_t irbc_record_bytes(const irbc_handle* h);
int irbc_record_async(irbc_handle* h, void* host, int64_t bytes);
/* observables not in the reference: out[0] = solvent kT from peculiar
 * velocities (each particle's velocity minus the mean velocity of its
 * z-layer of height a, so the Couette flow's kinetic energy is not counted
 * as heat), out[1..3] = membrane centre of mass x,y,z (unwrapped), out[4] =
 * Sarea, out[5] = Volume, out[6] = bond count, out[7] = mean solvent vx,
 * out[8] = sum m|v|^2 / (3 Ns) with the flow included; nout <= 9 values */
int irbc_observables(irbc_handle* h, double* out, int32_t nout);
/* Couette profile: mean vx of the solvent per z-layer of height a, nbins = Lz/a */
int irbc_velocity_profile(irbc_handle* h, double* out, int32_t nbins);

/* ---- health, timing and host buffers (not in the reference) ----------------------
 * The kernels that write the state check it as they go: a solvent particle
 * whose position or velocity is not finite or whose height left [-a, Lz + a]
 * sets bit 1, a membrane vertex whose force or velocity is not finite sets
 * bit 2 of the simulation's health word.  (The reference has no such check:
 * a blown-up run of it prints NaN into RBCdata.dat.)  irbc_sync waits for
 * the queued work and returns IRBC_ERR_HEALTH when the word is set;
 * irbc_step returns it, without stepping, once the word copied at the end
 * of an earlier irbc_step shows a problem.  irbc_set_state clears it. */
int irbc_sync(irbc_handle* h);
/* waits like irbc_sync and writes the health word (0: healthy) to *flags;
 * returns 0 unless the wait itself fails */
int irbc_health(irbc_handle* h, int32_t* flags);
/* kernel launches issued by this handle since creation */
int64_t irbc_launch_count(const irbc_handle* h);
/* CUDA-event timing on the handle's stream between begin and end.
 * out[0] = ms begin->end, out[1] = ms in the streaming kernels, out[2] =
 * streaming steps, out[3] = ms in the collision kernels, out[4] =
 * collisions, out[5] = ms in the membrane kernels (side stream), out[6] =
 * membrane launch groups, out[7] = kernel launches in the window, out[8] =
 * ms in the bulk streaming kernel alone (k_stream_fast / k_stream_f),
 * out[9] = its launches; nout <= 10 values are written */
/* device time (ms) between irbc_timer_begin and irbc_timer_end: two CUDA
 * events on the handle's stream and no per-phase events in between (what
 * irbc_step queues is joined back to that stream before it returns) */
int irbc_timer_begin(irbc_handle* h);
int irbc_timer_end(irbc_handle* h, double* ms);
int irbc_profile_begin(irbc_handle* h);
int irbc_profile_end(irbc_handle* h, double* out, int32_t nout);
/* ---- batches and the request server (not in the reference) -------------------
 * A batch steps independent simulations (handles, on one device) together:
 * nthreads host threads issue the members' steps so that their kernels
 * overlap on the GPU.  irbc_batch_step(b, n) advances every member n steps
 * and returns when their device work has finished.  Members stay owned by
 * the caller.  For many members, set CUDA_DEVICE_MAX_CONNECTIONS=32 in the
 * environment before the process first uses CUDA. */
typedef struct irbc_batch irbc_batch;
int irbc_batch_create(int32_t nthreads, irbc_batch** out);
void irbc_batch_destroy(irbc_batch* b);
int irbc_batch_add(irbc_batch* b, irbc_handle* h);
int irbc_batch_remove(irbc_batch* b, irbc_handle* h);
int32_t irbc_batch_size(const irbc_batch* b);
int irbc_batch_step(irbc_batch* b, int64_t n);
/* ---- launch schedules and their autotuner (not in the reference) --------------
 * How a batch launches its members' steps.  No field changes what a member
 * computes; each is checked bit for bit against its default:
 *   streams   irbc_set_streams for every member (1 or 2; default 2)
 *   membrane  irbc_set_membrane_kernels for every member (1 wide kernels,
 *             2 one block; default 1)
 *   graphs    irbc_set_graphs for every member (0 or 1; default 0)
 *   chunk     steps a pool thread issues to one member before it turns to
 *             its next member (a multiple of 24 in 24..2400; default 24)
 *   fused     1 (a batch's default; the server's default is 0): FP32
 *             members in the same phase (created or admitted together,
 *             stepped together) advance as one cohort,
 *             each phase of the step ONE kernel launch over all of them,
 *             its blocks split among the members; streams, membrane and
 *             graphs then apply only to the other members (FP64, or out of
 *             phase), which the pool of host threads steps.  0: every
 *             member through the pool. */
typedef struct irbc_schedule {
  int32_t streams, membrane, graphs, chunk, fused;
} irbc_schedule;
/* Applies s to every member now and to every member added later.  On an
 * error (IRBC_ERR_CAPACITY: a member's mesh is too large for membrane = 2)
 * every member goes back to the batch's previous schedule (the defaults if
 * none was set) and the error is returned. */
int irbc_batch_set_schedule(irbc_batch* b, const irbc_schedule* s);
int irbc_batch_get_schedule(const irbc_batch* b, irbc_schedule* s);
/* Picks the fastest of n candidates.  measure(i, ctx, &seconds) runs
 * candidate i once and returns 0 with its time, IRBC_ERR_CAPACITY when the
 * candidate cannot run (it is skipped), or another error, which ends the
 * search and is returned.  Candidates run one after another: each once
 * untimed, then `repeats` (1..64) timed runs, scored by their median.
 * Candidate 0 is the incumbent: a later candidate displaces the best so far
 * only when its median is below (1 - margin) times the best's (margin in
 * [0, 1)).  medians (n entries, or null) receives each score, -1 for a
 * skipped candidate.  IRBC_ERR_CAPACITY when every candidate was skipped. */
typedef int (*irbc_tune_measure)(int32_t candidate, void* ctx, double* seconds);
int irbc_tune_select(int32_t n, irbc_tune_measure measure, void* ctx, int32_t repeats, double margin,
                     double* medians, int32_t* best);
/* Tunes the batch's schedule on its own members, one field at a time in
 * the order fused, membrane, streams, graphs, chunk (24, 96, 240): the current
 * value against the others, each candidate scored by irbc_tune_select as
 * the host time of trial_steps batch steps with their device work waited
 * for.  Ends with the winner applied (to members added later too) and
 * written to *best.  The trial steps are ordinary steps of the members, and
 * no field changes results, so they simply advance the simulations:
 * *steps_taken receives how far every member advanced.  The tuner sets the
 * members' stream, membrane and graph options itself, replacing settings
 * made on the handles before.  IRBC_ERR_STATE for a batch without members;
 * after a step error the members are left under the candidate that failed,
 * and *steps_taken counts only the completed trial stretches. */
int irbc_batch_autotune(irbc_batch* b, int64_t trial_steps, int32_t repeats, double margin, irbc_schedule* best,
                        int64_t* steps_taken);
/* The server takes whole simulations as requests: parameters, mesh, knob
 * count and step count.  A pending request is admitted, in arrival order,
 * as soon as its footprint (irbc_footprint_bytes) fits in the device-memory
 * budget (budget_bytes <= 0: 85% of the free memory at creation); two
 * set-up threads create and initialise admitted requests on the device
 * while the stepping loop advances every set-up simulation in rounds of
 * round_steps steps (a pool of nthreads host threads, or cohorts under a
 * fused schedule); a request set up during a round joins at the next one.
 * A finished simulation yields an
 * irbc_result: its times on the server clock (seconds since creation), its
 * observables (irbc_observables) and, when submitted with keep = 1, its
 * handle; otherwise the server frees it.  A kept handle's device memory
 * stays charged to the budget until the caller hands it back with
 * irbc_server_release (which destroys it); after irbc_server_destroy the
 * caller destroys kept handles with irbc_destroy.  Each simulation computes
 * exactly what it would alone, and each has its own status: one that fails
 * (a CUDA error, or IRBC_ERR_HEALTH) ends with that status while the others
 * go on. */
typedef struct irbc_server irbc_server;
typedef struct irbc_result {
  int64_t id;
  int32_t status;          /* 0, or the error of create / init / step */
  int32_t pad_;
  int64_t steps, ns;       /* steps run, solvent particles */
  double t_submit, t_start, t_end;
  double obs[8];           /* irbc_observables at the end */
  irbc_handle* handle;     /* keep = 1: the finished simulation */
} irbc_result;
int irbc_server_create(int32_t device, int64_t budget_bytes, int32_t nthreads, int64_t round_steps,
                       irbc_server** out);
/* copies the mesh; *id identifies the request's result.  IRBC_ERR_CAPACITY
 * if its footprint exceeds the whole budget */
int irbc_server_submit(irbc_server* s, const irbc_params* p, const double* V, int32_t nv, const int32_t* E,
                       int32_t ne, const int32_t* T, int32_t nt, int32_t nknobs, int64_t nsteps, int32_t keep,
                       int64_t* id);
/* up to max finished results, waiting up to wait_s seconds for the first;
 * returns how many were written */
int32_t irbc_server_poll(irbc_server* s, irbc_result* out, int32_t max, double wait_s);
/* out: pending, active, unread results, bytes in use (kept handles not yet
 * released included), budget, particle-steps done */
int irbc_server_status(irbc_server* s, int64_t out[6]);
double irbc_server_clock(irbc_server* s);
/* the launch schedule (irbc_schedule) for simulations admitted from now on
 * and for the rounds' issue chunk (default {2, 1, 0, 24, 0}: the pool);
 * membrane = 2 applies only to meshes that fit the one-block form, the
 * others keep the wide kernels.  Results do not depend on it. */
int irbc_server_set_schedule(irbc_server* s, const irbc_schedule* sched);
/* destroys a kept handle (a polled result of a keep = 1 request) and frees
 * its share of the budget; IRBC_ERR_ARG for a handle the server did not hand
 * out */
int irbc_server_release(irbc_server* s, irbc_handle* h);
/* stops the loop; simulations still pending or running are dropped, and so
 * are the handles of results never polled */
void irbc_server_destroy(irbc_server* s);

/* page-locked host memory for fast state exchange */
void* irbc_host_alloc(size_t bytes);
void irbc_host_free(void* p);

#ifdef __cplusplus
}
#endif
#endif
