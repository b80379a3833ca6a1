/* rn.h -- C-ABI of librn.so, the B200 time-step library for the rocket
 * nozzle solver.
 *
 * Each entry point replaces one method of the reference's WebGL2 solver
 * (source/solver.js, source/spray.js); the comment on each names the line it
 * stands in for. Conventions:
 *   - every call returns int: RN_OK (0), RN_NOT_READY (1) for a poll whose
 *     data is not there yet, RN_BUSY (2) when an asynchronous read is already
 *     in flight, or a negative error code; rn_last_error() gives the message
 *     of the calling thread's last failure;
 *   - host buffers belong to the caller and are copied in or out during the
 *     call; device memory belongs to the handle;
 *   - one handle is used by one host thread at a time; its work runs in order
 *     on the handle's own CUDA stream. rn_step and rn_rescale_ambient return
 *     once the work is queued; the read functions block until their data is
 *     on the host.
 * Layout: cell (i, j) of an Nx x Nr grid is element j*Nx + i; A = (rho, rho u,
 * rho v, E) and B = (rho Z, rho F, G, rho O or inflow-speed average) are
 * float4 per cell, exactly the reference's RGBA32F state textures.
 */
#ifndef RN_H
#define RN_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

#define RN_OK 0
#define RN_NOT_READY 1
#define RN_BUSY 2
#define RN_ERR_ARG (-1)
#define RN_ERR_CUDA (-2)
#define RN_ERR_STATE (-3)
#define RN_ERR_NOMEM (-4)

/* texture names for rn_read_rect / rn_request_async (the reference reads any
 * texture it owns through _readRect, solver.js:1016) */
#define RN_TEX_A 0          /* current state A, Nx x Nr */
#define RN_TEX_B 1          /* current state B, Nx x Nr */
#define RN_TEX_STEPINFO 2   /* (dt, t_old, t_new, w), 1 x 1 */
#define RN_TEX_WALLROW 3    /* near-wall row (u, v, p, c), Nx x 1, after rn_draw_wall_row */
#define RN_TEX_PARCEL_A 4   /* parcels (x, r, u, v), 256 x 256 */
#define RN_TEX_PARCEL_B 5   /* parcels (d, m, type, x_imp), 256 x 256 */
#define RN_TEX_PARCEL_C 6   /* parcels (dm, dp_x, dp_r, 0) given to the gas last step */
#define RN_TEX_INJECTOR 7   /* injector table, 256 x 3 (the spray's uTab) */

typedef struct rn_solver* rn_handle;

/* The normalised parameter block P of the reference (simsetup.js:274-310),
 * reduced to the float32 uniforms the shaders receive. bar = (inlet[0],
 * 1.6 uInlet0, max(ramp, 0)) is solver.js:935's uBar; fan is spray.js:271's
 * 25 degrees in radians. Flags are 0/1. */
typedef struct {
  float amb[4], ambCons[4], ambB[4];
  float gamR[2];
  float inlet[4];
  float bar[3];
  float res[3];
  float gas[4];
  float Rs[3];
  float chemK[4];
  float cap[2];
  float chamberNu[2];
  float Tw, cfl, dtMax, wFloor, vMax, hllBlend, ramp, pStart, RcCells;
  int order2, inj, visc, chem;
  float mhat, tScale;
  float fuel[4], ox[4];
  float eF, eO, Ge, fan;
} rn_params;

/* one rectangle of an asynchronous read (requestAsync's reqs, solver.js:1028) */
typedef struct {
  int tex, x, y, w, h;
} rn_read_req;

/* Inputs of the FP64 read-out integrals: the exit column and its jExit, the
 * throat column, the chamber probe cell, and dx (simsetup.js:239-250, 314-348). */
typedef struct {
  int iExit, jExit, iThroat, iChamber;
  double dx, pAmb;       /* pAmb = P.amb[3] (normalised ambient pressure) */
  double Rs[3], RaN;     /* gas constants for the chamber-cell temperature */
  int inj;
} rn_integral_spec;

/* FP64 read-outs, normalised units as the reference's JavaScript computes
 * them before its SI scaling: thrust F, exhaust mass flow mdot, Mach-weighted
 * flow Mw (exit Mach = Mw/mdot), pressure-area pw and area A of the exit
 * plane; throat mass flow, oxidiser and fuel-vapour flows; chamber-cell
 * pressure and temperature ratio p/(rho Rmix); step info; every sum is a
 * Neumaier-compensated double sum. */
typedef struct {
  double F, mdot, Mw, pw, A;
  double throat_mdot, throat_mO, throat_mF;
  double chamber_p, chamber_T;
  double dt, t;
} rn_integrals_out;

/* new GPUSolver(gl) + resize(Nx, Nr) (solver.js:678, 759) */
int rn_create(int Nx, int Nr, rn_handle* out);
/* GPUSolver._free (solver.js:752) and the handle itself */
int rn_destroy(rn_handle h);
/* resize(Nx, Nr) (solver.js:759-789): reallocates and clears every buffer */
int rn_resize(rn_handle h, int Nx, int Nr);
/* setMask(u8) (solver.js:791-799): nonzero = solid */
int rn_set_mask(rn_handle h, const uint8_t* mask);
/* setGeometry({mask, geoA, geoG, geoM, jWall}) (solver.js:801-814): geoA is
 * (Nx+1) x (Nr+1) float4, geoG and geoM Nx x Nr float4, jWall Nx float4 or NULL */
int rn_set_geometry(rn_handle h, const uint8_t* mask, const float* geoA, const float* geoG, const float* geoM,
                    const float* jWall);
/* setState(A, B) (solver.js:816-828): all three state slots, clears dt/t and
 * the spray ring */
int rn_set_state(rn_handle h, const float* A, const float* B);
/* readAll() (solver.js:1075) */
int rn_get_state(rn_handle h, float* A, float* B);
/* step(n, P) (solver.js:849-891), including GPUSpray.step (spray.js:256-297)
 * when P->inj is set: queued on the handle's stream. For n of two periods or
 * more (12 steps, 4 with sprays) the handle captures one period of its
 * launches into a CUDA graph and replays it (the same kernels, the same
 * bits); not while profiling, and not while the caller is itself capturing
 * the handle's stream. */
int rn_step(rn_handle h, int n, const rn_params* P);
/* rescaleAmbient(fp, fT, du, P) (solver.js:998-1010) */
int rn_rescale_ambient(rn_handle h, float fp, float fT, float du, const rn_params* P);
/* drawWallRow() (solver.js:986-996): fills RN_TEX_WALLROW */
int rn_draw_wall_row(rn_handle h);
/* _readRect(tex, x, y, w, h) (solver.js:1016-1025): blocking, w*h*4 floats */
int rn_read_rect(rn_handle h, int tex, int x, int y, int w, int hgt, float* out);
/* readStepInfo() (solver.js:1072) */
int rn_read_step_info(rn_handle h, float out[4]);
/* requestAsync(reqs, tag) (solver.js:1028-1048): copies into pinned memory
 * behind an event; RN_BUSY when a read is already in flight */
int rn_request_async(rn_handle h, const rn_read_req* reqs, int nreq, int tag);
/* pollAsync() (solver.js:1050-1065): RN_NOT_READY until the copies are done,
 * then writes the concatenated floats (requests in order) and the tag;
 * RN_ERR_STATE when nothing is in flight; RN_ERR_ARG if cap_floats is short */
int rn_poll_async(rn_handle h, int* tag, float* out, size_t cap_floats);
/* cancelAsync() (solver.js:1066-1070) */
int rn_cancel_async(rn_handle h);
/* GPUSpray.setInjector({tab}) (spray.js:236-241): 256 x 3 float4 */
int rn_spray_set_injector(rn_handle h, const float* tab);
/* The injector table built on the device from its spray elements (the fill of
 * buildInjectorTable, simsetup.js:181-237): weights normalised and spread over
 * the 256 rows by largest remainder (ties in element order), rows written in
 * element order; the same table rn_spray_set_injector would upload. Element
 * lengths in cells, speeds in U_REF, angles in radians. */
#define RN_MAX_INJECTOR_ELEMENTS 64
typedef struct {
  double type, weight, x, r, angle, speed, drop, cone, width, xi;
} rn_injector_element;
int rn_spray_build_injector(rn_handle h, const rn_injector_element* el, int n);
/* A pre-populated parcel ring (no reference counterpart: the reference only
 * spawns parcels from the injector): PA = (x, r, u, v) and PB = (d, m, type,
 * x_imp), 65,536 float4 each in the ring's layout, become the current
 * parcels; the given head is where the next 4 spawn. Dead slots have m <= 0. */
int rn_spray_set_parcels(rn_handle h, const float* PA, const float* PB, int head);
/* GPUSpray.reset() (spray.js:242-254) */
int rn_spray_reset(rn_handle h);
/* Live parcels summed over every spray step since the ring was last set
 * (rn_spray_reset, rn_spray_set_parcels, rn_set_state): the parcel-steps the
 * handle has simulated. Counted on the device by the parcel kernel; blocks
 * until the handle's queued steps are done. No reference counterpart. */
int rn_spray_parcel_steps(rn_handle h, long long* out);
/* GPUSpray.stats(P) (spray.js:312-320): out = (fuel mass, oxidiser mass,
 * live parcels, mean diameter). Returns RN_ERR_STATE (once, then clears it) if
 * a fast-precision deposit since the last call fell outside the fixed-point
 * range of the deposit sums (a parcel far heavier or faster than
 * mhat*dtMax/4 and vMax allow) and was clamped. */
int rn_spray_stats(rn_handle h, double out[4]);
/* The read-outs the reference computes in JavaScript from column read-backs
 * (exitPerformance simsetup.js:314-337, chamberPerformance 239-250,
 * cellPrimSI 338-348), evaluated on the device in FP64. */
int rn_integrals(rn_handle h, const rn_integral_spec* spec, rn_integrals_out* out);
/* waits for all queued work of the handle */
int rn_sync(rn_handle h);
/* Bounded wait: polls the handle's stream until its work is done or
 * timeout_ms elapse; RN_NOT_READY on timeout (the work keeps running). */
int rn_wait(rn_handle h, int timeout_ms);
/* number of kernels this handle has launched (for launch accounting) */
int rn_kernel_launches(rn_handle h, long long* out);
/* Arithmetic of the step kernels. The reference's shaders run in GLSL highp,
 * whose division and square root may be off by up to a few ulp and whose
 * compilers may fuse multiply-adds.
 *   RN_PRECISION_FAST (default): the hardware's approximate division and
 *     square root (within 2 ulp) and fused multiply-adds, the same latitude;
 *     spray deposits summed per cell in 64-bit fixed point (order-independent);
 *   RN_PRECISION_EXACT: IEEE-rounded division and square root, no fusion, and
 *     spray deposits summed in parcel-index order as the reference's blending
 *     does, so the state reproduces the CPU oracle of the shader passes bit
 *     for bit except where pow/exp/log/sin/cos differ in the last bit. About
 *     1.7x slower.
 * Both are deterministic: the same inputs give the same bits, run to run.
 * No reference counterpart (the reference has one shader build). */
#define RN_PRECISION_FAST 0
#define RN_PRECISION_EXACT 1
int rn_set_precision(rn_handle h, int mode);
int rn_get_precision(rn_handle h, int* mode);

/* Tile shape of the stage/physics kernels (a thread per cell):
 * RN_TILE_16x15, RN_TILE_16x16, RN_TILE_16x8, RN_TILE_32x15 or RN_TILE_14x16. A new handle
 * starts with RN_TILE_14x16 when the grid's 14 x 16 tiles number at most 3 per
 * SM (all resident at once), else with RN_TILE_16x15. rn_autotune times `steps` steps
 * with each shape on a copy of the handle's current state (the state, step
 * info and spray ring are restored afterwards), keeps the fastest and returns
 * it in *chosen. No reference counterpart (the reference draws full-screen
 * fragment passes). */
#define RN_TILE_16x16 0
#define RN_TILE_16x8 1
#define RN_TILE_16x15 2   /* 16 x 15 cells on 256 threads */
#define RN_TILE_32x15 3   /* 32 x 15 cells on 512 threads */
#define RN_TILE_14x16 4   /* 14 x 16 cells on 256 threads */
int rn_set_tile(rn_handle h, int shape);
int rn_get_tile(rn_handle h, int* shape);
int rn_autotune(rn_handle h, const rn_params* P, int steps, int* chosen);

/* Batched stepping (no reference counterpart; the reference runs one grid
 * per page). A batch steps many solver handles of uneven grid sizes with one
 * launch per kernel kind per step: every tile of every member is a block of
 * the same grid. Members must share the physics flags (visc, chem, inj) and
 * the precision; each keeps its own state, geometry, dt and parameter block.
 * rn_batch_step captures the periodic 6-step launch sequence in a CUDA graph
 * and replays it. While in a batch a handle must not be stepped on its own;
 * all other handle calls (reads, integrals) work between batch steps.
 * Removing a member leaves its handle where the batch left it. */
typedef struct rn_batch_t* rn_batch;
int rn_batch_create(rn_batch* out);
int rn_batch_destroy(rn_batch b);
/* adds h with parameter block P; *slot receives its index in the batch */
int rn_batch_add(rn_batch b, rn_handle h, const rn_params* P, int* slot);
int rn_batch_remove(rn_batch b, rn_handle h);
int rn_batch_set_params(rn_batch b, rn_handle h, const rn_params* P);
int rn_batch_size(rn_batch b, int* members, long long* cells);
int rn_batch_step(rn_batch b, int n);
/* Runs every member to its own stop, in chunks of `chunk` steps: member m
 * keeps stepping while the simulated time of its current state (step info
 * t_new, in the solver's time units) is below t_end[m] and, with max_steps >
 * 0, the run has taken fewer than max_steps steps; both are checked before
 * each chunk, so each member takes the steps of the host loop
 * `while (t < t_end) rn_step(h, chunk, P)`. The checks run on the device (one
 * small kernel and one 4(n+1)-byte read-back per chunk); a stopped member's
 * blocks return at once and leave the launch (a rebuilt block table and
 * graph) once the stopped members' blocks number at least one per SM and an
 * eighth of the launch. steps[m] (may be NULL) receives the steps member m
 * took.
 * Returns when every member has stopped. The batch form of the reference's
 * frame loop (app.js:965 calls step(n, P) until the user stops it). */
int rn_batch_run(rn_batch b, const double* t_end, int chunk, long long max_steps, long long* steps);
int rn_batch_sync(rn_batch b);
/* tile shape of the batch's launches (RN_TILE_*) */
int rn_batch_set_tile(rn_batch b, int shape);
/* times `steps` batch steps with each tile shape on copies of the members'
 * current states (states, step info and spray rings are restored), keeps the
 * fastest and returns it in *chosen */
int rn_batch_autotune(rn_batch b, int steps, int* chosen);
/* the batch's CUDA stream (a cudaStream_t) */
int rn_batch_stream(rn_batch b, void** stream);
/* number of kernels the batch has launched (graph replays included) */
int rn_batch_kernel_launches(rn_batch b, long long* out);

/* Steady-state residual (no reference counterpart: the reference has no
 * convergence measure). rn_residual_mark snapshots the current A plane and
 * step info on the device (allocating the snapshot on first use);
 * rn_residual returns in FP64, for each component c of A = (rho, rho u,
 * rho v, E), the RMS over fluid cells of (A_c - A_c at the mark) / (t - t_mark):
 * out[0..3], with out[4] = t - t_mark and out[5] = the fluid-cell count. With
 * one step between the two calls this is the L2 norm of dU/dt of that step.
 * Deterministic (fixed reduction order); blocks until out is filled. */
int rn_residual_mark(rn_handle h);
int rn_residual(rn_handle h, double out[6]);

/* Flow-separation read-out on the device (wallSeparation, simsetup.js:352-373):
 * walks the near-wall row (the FS_WALLROW values, solver.js:665-674, built on
 * the fly from the current state and jWall) upstream from iExit and returns
 * the separation column with its FP64 read-outs; only these scalars reach the
 * host. rn_set_wall_profile uploads, per column i (x = (i + 0.5) dx), the wall
 * slope (R(x + dx/2) - R(x - dx/2)) / dx, hypot(1, slope) and R(x), in metres,
 * once per geometry. found = 0 where the reference returns null. */
typedef struct {
  int iThroat, iExit;
  double dx, xt, xe, Rt;   /* metres */
  double paSi, pRef;       /* ambient pressure (Pa) and the pressure unit P_REF (Pa) */
} rn_separation_spec;
typedef struct {
  int found, last;         /* last = separation column (or -1) */
  double x, frac, eps, pRatio, Msep;
} rn_separation_out;
int rn_set_wall_profile(rn_handle h, const double* slope, const double* hyp, const double* radius);
int rn_wall_separation(rn_handle h, const rn_separation_spec* spec, rn_separation_out* out);

/* Derived display fields into a headless device buffer (FS_DERIVED,
 * render.js:60-134): per cell (t, Z, normalised T, Mach) with t the selected
 * field mapped to its display range, (0, 0, 0, -1) in walls. field is the
 * reference's uField: 0 temperature, 1 Mach, 2 schlieren, 3 log10 p, 4 log10
 * rho, 5 speed, 6 vorticity, 7 exhaust fraction, 9 log10 eddy/laminar
 * viscosity, 10 unburnt fraction, 11 fuel vapour, 12 oxidiser, 13 burning rate.
 * The spec carries the shader's uniforms. Fields 9 and 13 need P (the
 * step's parameter block) and read the split step's T2, recomputed from the
 * last step's stage-1 state (0 if no step ran since the state was set). The
 * buffer (Nx*Nr float4) belongs to the handle (rn_derived_buffer gives its
 * device address); `out` (Nx*Nr*4 floats) may be NULL. No reference
 * counterpart for the buffer: the reference draws it to the screen. */
typedef struct {
  int field;
  float range[2];           /* uRange */
  float RaN, Rs[3];         /* uRaN, uRs */
  float chemV[4];           /* uChemV */
  float Tscale[4];          /* uTscale: (T_REF, Tc K, Ta K, unused) */
  float schlGain, velScale, dx;
} rn_derived_spec;
int rn_derived(rn_handle h, const rn_derived_spec* spec, const rn_params* P, float* out);
int rn_derived_buffer(rn_handle h, void** dev);

/* Cut-cell geometry builder on the device (buildCutGeometry, cutcell.js:14-186,
 * plus buildSimSetup's geoM turbulence length and boundary-layer band,
 * simsetup.js:51-63, and the near-wall row jWall): builds the handle's mask,
 * geoA, geoG, geoM and jWall in place of rn_set_geometry, bit-identical to the
 * host builder. Lengths in cells unless stated. The wall enters as the
 * reference's Float32Array radius table Rtab (Nx*8+1 entries, cutcell.js:22)
 * and as RinAt(x) at the abscissae the builder samples, per column i
 * (RN_CUT_SAMPLES doubles): x = i, i + 0.5, i + (a + 0.5)/8 (a < 8),
 * i + (b + 0.5)/12 (b < 12), i + 1; each entry is read only where
 * x <= xeC. rinCol is the setup's Float32Array of the wall radius at the column
 * centres in metres (+inf beyond the exit). No reference counterpart for the
 * device placement (the reference builds on the CPU). */
#define RN_CUT_SAMPLES 23
typedef struct {
  int Nx, Nr;
  int cut;                  /* wallModel 'cut' (1) or 'stair' (0) */
  int base;                 /* base / boat-tail body present */
  int nSolids;              /* chamber hardware blocks (at most 64) */
  int iExit;                /* jWall is set for columns 0..iExit */
  double xeC, twC, xBaseC, bodyC;
  double dx, xt, xe, Rt;    /* metres */
  const float* Rtab;
  const double* rin;        /* Nx * RN_CUT_SAMPLES */
  const double* solids;     /* nSolids * (x0, x1, r0, r1) */
  const float* rinCol;      /* Nx */
} rn_cut_spec;
typedef struct {
  int nCut, nMerged;        /* fluid cells with kappa < 0.98; merged slivers */
} rn_cut_stats;
int rn_build_geometry(rn_handle h, const rn_cut_spec* spec, rn_cut_stats* stats);
/* the handle's geometry planes back on the host (any pointer may be NULL);
 * sizes as rn_set_geometry's, jWall Nx float4. No reference counterpart (the
 * reference keeps its geometry on the host). */
int rn_get_geometry(rn_handle h, uint8_t* mask, float* geoA, float* geoG, float* geoM, float* jWall);

/* Solve server: continuous batching of whole solves on one GPU (no
 * reference counterpart; the reference runs one interactive solve per page).
 * rn_serve_submit copies a request (grid, geometry, initial state, P, stop
 * criteria) into the arrival queue and returns its id at once. A worker thread
 * admits queued requests in arrival order while their device bytes
 * (rn_solve_bytes) fit in the budget, adds each to the batch of its physics
 * class (visc, chem, inj; classes run on separate streams and overlap), steps
 * every batch check_every steps per tick, and evaluates each solve's FP64
 * density residual (rn_residual over the tick's last step) and time after the
 * tick. A solve whose residual fell to drop x its first value, whose time
 * reached t_end or whose steps reached max_steps (tested in that order, at
 * tick granularity) gets its FP64 read-outs and final state copied out and
 * frees its memory, which admits later arrivals. A solve's result does not
 * depend on what else is in the mix. */
typedef struct rn_server_t* rn_server;
typedef struct {
  size_t hbm_budget;   /* device bytes admitted solves may hold; 0 = 80 % of the free memory at creation */
  int max_active;      /* most solves on the device at once; 0 = limited by the budget only */
  int check_every;     /* steps per tick (>= 2) */
  int precision;       /* RN_PRECISION_* of every solve */
  int tile;            /* RN_TILE_* of the class batches */
  long long max_active_cells;   /* most grid cells on the device at once; 0 = no limit. Enough cells to
                                   fill the GPU keep its throughput; fewer concurrent solves finish sooner */
} rn_server_opts;
typedef struct {
  int Nx, Nr;
  const uint8_t* mask;              /* as rn_set_geometry */
  const float* geoA;
  const float* geoG;
  const float* geoM;
  const float* jWall;               /* or NULL */
  const float* A;                   /* initial state, as rn_set_state */
  const float* B;
  const float* injTab;              /* 256 x 3 float4 when P.inj, else NULL */
  rn_params P;
  rn_integral_spec spec;            /* read-out columns for the result */
  double drop;                      /* density-residual drop that ends the solve (0: off) */
  double t_end;                     /* normalised time that ends the solve (0: off) */
  long long max_steps;              /* step count that ends the solve (0: off) */
  const float* parcelsA;            /* a pre-populated parcel ring (rn_spray_set_parcels), or NULL */
  const float* parcelsB;
  int parcelHead;
} rn_solve_request;
#define RN_SOLVE_CONVERGED 0
#define RN_SOLVE_TIME 1
#define RN_SOLVE_MAX_STEPS 2
#define RN_SOLVE_REJECTED (-1)      /* needs more than the whole budget */
#define RN_SOLVE_FAILED (-2)
typedef struct {
  int status;                       /* RN_SOLVE_* */
  int pad_;
  long long steps;
  double t, residual0, residual;    /* final normalised time; first and last density residual */
  double submit_ms, admit_ms, done_ms;   /* server clock, ms since rn_server_create */
  rn_integrals_out integrals;       /* FP64 read-outs of the final state */
} rn_solve_result;
typedef struct {
  long long queued, active, finished, bytes_used, bytes_budget, ticks, admitted;
  long long failed;     /* 1 once the CUDA context broke: every solve then failed and submit refuses */
  long long evicted;    /* solves that failed alone (setup, allocation, a non-finite residual) */
} rn_serve_status;
int rn_server_default_opts(rn_server_opts* opts);
int rn_server_create(const rn_server_opts* opts, rn_server* out);
/* stops the worker after its current tick; unfinished solves are dropped */
int rn_server_destroy(rn_server s);
int rn_serve_submit(rn_server s, const rn_solve_request* req, long long* id);
/* RN_NOT_READY until request id has finished; then fills res and, if not
 * NULL, the final state planes (Nx*Nr*4 floats each), and forgets the id */
int rn_serve_poll(rn_server s, long long id, rn_solve_result* res, float* A, float* B);
/* rn_serve_poll after waiting up to timeout_ms for the request to finish */
int rn_serve_wait(rn_server s, long long id, int timeout_ms, rn_solve_result* res, float* A, float* B);
int rn_serve_stats(rn_server s, rn_serve_status* out);
/* device bytes the server charges a solve of an Nx x Nr grid against its budget */
int rn_solve_bytes(int Nx, int Nr, long long* bytes);
/* Failure isolation: a solve whose own work fails (its setup or upload at
 * admission, an allocation, a non-finite residual) is evicted alone with
 * RN_SOLVE_FAILED, its memory freed, and every other solve carries on
 * unchanged. A class batch whose step fails while the CUDA context stays
 * usable evicts that class's solves. Only a broken context (a sticky CUDA
 * error) fails every solve and latches `failed`.
 * Host-side fault injection for tests (nothing faults on the GPU): the next
 * request submitted to s fails as a device allocation would (RN_ERR_NOMEM)
 * at its admission (RN_INJECT_ADMIT) or in its first tick (RN_INJECT_TICK). */
#define RN_INJECT_ADMIT 1
#define RN_INJECT_TICK 2
int rn_serve_inject(rn_server s, int where);

/* the handle's CUDA stream (a cudaStream_t), so a caller can order its own
 * work (timing events, cache flushes) with the handle's kernels */
int rn_get_stream(rn_handle h, void** stream);

/* Per-kernel device time: with profiling on, every kernel the handle launches
 * is bracketed by CUDA events on its stream. enable = 1: launch by launch
 * (rn_step does not replay its graph, so the times include the gaps in
 * which the GPU waits for the host's next launch); enable = 2: steps without
 * sprays run as replays of a graph of one period that holds an event pair
 * around each kernel (event-record nodes), read after every replay, so each
 * kernel is timed as it runs back to back with the others; the steps before
 * the first whole period, and spray steps, are timed launch by launch. 0
 * turns it off. rn_profile_read waits for the stream, returns milliseconds
 * and launch counts per kernel kind (indexed by RN_K_*) accumulated since the
 * last read, and clears them. */
#define RN_K_REDUCE 0
#define RN_K_STAGE1 1
#define RN_K_STAGE2 2
#define RN_K_PHYSICS 3
#define RN_K_PARCELS 4   /* parcel update + deposit sort + segment sums */
#define RN_K_APPLY 5
#define RN_K_OTHER 6     /* rescale, wall row, integrals */
#define RN_K_STAGE2_PHYSICS 7   /* stage 2 fused with the viscous/wall/reaction split step */
#define RN_NKERNELS 8
int rn_profile(rn_handle h, int enable);
int rn_profile_read(rn_handle h, double ms[RN_NKERNELS], long long launches[RN_NKERNELS]);

/* FP64 read-outs without any device allocation. No counterpart in the
 * reference (its read-outs are JavaScript over read-back columns). Same
 * results as rn_integrals, for callers that cannot allocate device memory
 * when they need a read-out: an application that reserves the whole device
 * memory budget up front and forbids later allocation, or a latency-critical
 * loop that cannot take cudaMalloc's implicit synchronisation. The caller
 * passes its own device buffers: state planes A and B (Nx*Nr float4), geoA
 * ((Nx+1)*(Nr+1) float4), mask (Nx*Nr bytes) and the step-info float4;
 * stream is a cudaStream_t or NULL. Scratch lives in a file-scope __device__
 * array (per-row terms of up to RN_STATIC_MAX_ROWS rows, 256 KiB, held by
 * every GPU that loads the library until exit); Nr above that limit is
 * rejected with RN_ERR_ARG. The first call on a device looks up the array's
 * device address; make it before any stream capture. The call cannot be made
 * while its stream is being captured (it ends with a blocking read-back):
 * it then returns RN_ERR_ARG and queues nothing. The looked-up address does
 * not survive cudaDeviceReset: do not call it after a reset in the same
 * process. Calls share the array: calls that overlap on the GPU race.
 * Blocks until `out` is filled. */
#define RN_STATIC_MAX_ROWS 4096
int rn_integrals_static(const float* A, const float* B, const float* geoA, const uint8_t* mask, int Nx, int Nr,
                        const float* stepinfo, const rn_integral_spec* spec, rn_integrals_out* out, void* stream);

/* message of the calling thread's last error ("" if none) */
const char* rn_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
