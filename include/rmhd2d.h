/*
 * rmhd2d.h -- C ABI of librmhd2d, a B200-native (sm_100a) 2D resistive-MHD
 * RK2 step that drops in for the single-GPU Thrust library of
 * keita-akutagawa/ResistiveMHD_GPU
 * (ResistiveMHD_singleGPU_thrust/lib_ResistiveMHD_2D_GPU_periodicXY and
 *  .../lib_ResistiveMHD_2D_GPU_symmetricXY).
 *
 * Plain C types only: pointers, sizes, ints and doubles.  Every function
 * returns an rmhd2d_status (0 = success).  The reference library performs no
 * error checks at all; here a failure leaves the solver unchanged where
 * possible and rmhd2d_last_error() describes it.
 *
 * State layout at the boundary is the reference's: an array of nx*ny cells,
 * cell k = j + i*ny (y fastest), each cell 8 doubles in the order of the
 * reference's ConservationParameter (conservation_parameter_struct.hpp:5-27):
 *   rho, rhoU, rhoV, rhoW, bX, bY, bZ, e
 * nx and ny include 3 ghost layers per side (the periodic period is nx-6);
 * bX of cell (i,j) lives on the x-face i+1/2 and bY on the y-face j+1/2.
 *
 * Threading: a solver is used from one host thread at a time.  Work is
 * enqueued on the solver's CUDA stream; functions that return host values
 * (rmhd2d_get_dt, rmhd2d_check_crashed, rmhd2d_get_state, ...) synchronise
 * that stream.  Several solvers may coexist in one process (the reference
 * allows one, through process-global __constant__ state).
 */
#ifndef RMHD2D_H
#define RMHD2D_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RMHD2D_ABI_VERSION 3
#define RMHD2D_GHOST 3

typedef enum {
    RMHD2D_OK = 0,
    RMHD2D_ERR_INVALID = 1,     /* bad argument or configuration */
    RMHD2D_ERR_CUDA = 2,        /* a CUDA runtime call failed */
    RMHD2D_ERR_NO_DEVICE = 3,   /* no usable sm_100 device */
    RMHD2D_ERR_STATE = 4,       /* call not valid in the solver's current state */
    RMHD2D_ERR_IO = 5,          /* file could not be written or read */
    RMHD2D_ERR_KERNEL = 6       /* a kernel reported an internal error (bounded wait expired) */
} rmhd2d_status;

typedef enum {
    RMHD2D_BC_PERIODIC = 0,     /* Boundary::periodicBoundaryX2nd/Y2nd (TP boundary.cu:4-141) */
    RMHD2D_BC_SYMMETRIC = 1,    /* Boundary::symmetricBoundaryX2nd/Y2nd (TS boundary.cu:4-206): mirror copies,
                                   normal-B ghosts integrated from div B = 0 */
    /* The multi-GPU library's walls (ResistiveMHD_multiGPU_cuda/ResistiveMHD2D_GPU/boundary.cu): */
    RMHD2D_BC_ZERO_GRADIENT = 2,/* copies of the nearest interior cell (its symmetricBoundaryY2nd, :292-337;
                                   the x = xmax side of its flare wall); x or y walls */
    RMHD2D_BC_WALL = 3,         /* conducting wall (wallBoundaryY2nd, :48-119): the first interior cell's density,
                                   pressure, normal B and bZ with zero velocity and bY; y walls only */
    RMHD2D_BC_FLARE = 4         /* flareBoundaryX2nd (:196-245): line-tied at x = xmin (the wall state keeping v),
                                   zero gradient at x = xmax; x walls only */
} rmhd2d_bc;

typedef enum {
    /* FP64, bit-identical to the reference evaluated in IEEE binary64 without
       fused multiply-add (the reference's own host build). */
    RMHD2D_FP64_EXACT = 0,
    /* FP64 with fused multiply-add and only the selected HLLD candidate
       fluxes; differs from EXACT by rounding only. */
    RMHD2D_FP64_FAST = 1,
    /* FP32 bulk: MUSCL reconstruction, HLLD and eta*J fluxes in single
       precision; pressure recovery from total energy, corner-EMF
       accumulation, flux-difference update and dt reduction in FP64; state
       stored in FP64.  No counterpart in the reference (its FP32 library
       lib_ResistiveMHD_2D_GPU_single runs everything in float). */
    RMHD2D_FP32_BULK = 2
} rmhd2d_precision;

typedef enum {
    /* The single-GPU library's CT: the stage-1 corner EMF (the arithmetic
       mean of the four numerical induction fluxes) updates the face B of
       both stages (TP resistiveMHD_2D.cu:133-195, ct.cu:22-59). */
    RMHD2D_CT_STAGE1 = 0,
    /* CT-Contact: B advances by flux differences in both stages, and one CT
       from the step input's faces ends the step, with the mean of the two
       stages' contact EMFs -- the arithmetic mean plus corrections upwinded
       by the signs of the mass fluxes against per-cell reference EMFs
       u bY - v bX - eta jZ (the multi-GPU library's
       ResistiveMHD2D_GPU/ct.cu:26-257 with the ordering of its oneStepRK2,
       resistiveMHD2D.cu:147-221), on this library's fluxes and dt.  Runs in
       FP64 without contraction whatever cfg.precision; no batches, adjoint
       or rmhd2d_profile_step. */
    RMHD2D_CT_CONTACT = 1
} rmhd2d_ct_scheme;

typedef struct {
    int nx, ny;                 /* cells per direction incl. 3 ghost layers per side; both >= 12 */
    double dx, dy;              /* cell sizes (reference const.hpp:7,12) */
    double gamma_mhd;           /* ratio of specific heats (const.hpp:18) */
    double cfl;                 /* CFL number (const.hpp:17) */
    double eps;                 /* EPS regulariser of the reference (const.hpp:4) */
    double eta;                 /* scalar eta: the resistive term when no eta table is set,
                                   and always the diffusive dt limit dx^2/eta (resistiveMHD_2D.cu:288) */
    int bc;                     /* rmhd2d_bc of the x walls (and of the y walls when bc_y = -1);
                                   PERIODIC, SYMMETRIC, ZERO_GRADIENT or FLARE */
    int bc_y;                   /* rmhd2d_bc of the y walls (PERIODIC, SYMMETRIC, ZERO_GRADIENT or WALL),
                                   or -1 for the same as bc; periodic x with
                                   symmetric y is the reference's oneStepRK2PeriodicXSymmetricY
                                   (lib_ResistiveMHD_2D_GPU_single/resistiveMHD_2D.cu:198-259) */
    int precision;              /* rmhd2d_precision */
    int device;                 /* CUDA device ordinal */
    void *stream;               /* cudaStream_t to enqueue on, or NULL for a solver-owned stream */
    int ct_scheme;              /* rmhd2d_ct_scheme */
} rmhd2d_config;

typedef struct rmhd2d_solver rmhd2d_solver;

/* Fills cfg with defaults (gamma 5/3, cfl 0.4, eps 1e-20, periodic x and y, FP64 exact). */
void rmhd2d_config_default(rmhd2d_config *cfg);

/* Replaces the constructor ResistiveMHD2D::ResistiveMHD2D()
   (TP resistiveMHD_2D.cu:11-22) together with the link-time globals of
   const.hpp:4-25 and initializeDeviceConstants() (const.cu:4-24). */
int rmhd2d_create(const rmhd2d_config *cfg, rmhd2d_solver **out);
int rmhd2d_destroy(rmhd2d_solver *s);

/* Replaces the body of the user's ResistiveMHD2D::initializeU()
   (e.g. examples2D/plasmoid/main_plasmoid.cu:132-156): uploads a full state
   (ghosts included) from host memory in the layout above.  With
   apply_boundary != 0 the boundary of the configured kind is applied
   afterwards, as the reference drivers do at the end of initializeU. */
int rmhd2d_set_state(rmhd2d_solver *s, const double *host_state, int apply_boundary);

/* Same as rmhd2d_set_state from device memory (any CUDA-visible pointer).
   The copy is enqueued on the solver's stream, which does not wait for the
   legacy default stream or any other: the data must be complete when the
   call is made (synchronise the stream that produced it first). */
int rmhd2d_set_state_device(rmhd2d_solver *s, const double *device_state, int apply_boundary);

/* Replaces ResistiveMHD2D::getU() (TP resistiveMHD_2D.cu:431-434): copies
   the full state into host memory (nx*ny*8 doubles). */
int rmhd2d_get_state(rmhd2d_solver *s, double *host_state);

/* Sets a cell-centred resistivity table (nx*ny doubles, k = j + i*ny) used
   by the resistive flux instead of the uniform eta; NULL returns to uniform
   eta.  Replaces the driver's getEta() (main_plasmoid.cu:159-172) sampled at
   cell centres, as the driver's addResistiveTermToFluxF/G kernels sample it. */
int rmhd2d_set_eta_table(rmhd2d_solver *s, const double *host_eta);

/* Replaces Boundary::periodicBoundaryX2nd + Y2nd (TP boundary.cu:4-141) or
   symmetricBoundaryX2nd + Y2nd (TS boundary.cu:4-206) applied to U. */
int rmhd2d_apply_boundary(rmhd2d_solver *s);

/* Replaces ResistiveMHD2D::calculateDt() (TP resistiveMHD_2D.cu:277-291):
   returns the dt the next step will use, CFL * min(min_cells 1/(|u|/dx + ...),
   dx^2/eta, dy^2/eta). */
int rmhd2d_calculate_dt(rmhd2d_solver *s, double *dt);

/* Replaces ResistiveMHD2D::oneStepRK2() (TP resistiveMHD_2D.cu:133-195,
   TS resistiveMHD_2D.cu:133-195): one Heun RK2 step with constrained
   transport.  Enqueued asynchronously, as one launch of a CUDA graph of the
   step captured on first use; while the caller is capturing the solver's
   stream, the step's kernels are enqueued into that capture instead.
   Graphs are captured again after rmhd2d_set_tile_shape and
   rmhd2d_set_eta_table. */
int rmhd2d_step_rk2(rmhd2d_solver *s);

/* nsteps calls of rmhd2d_step_rk2, replayed from a captured CUDA graph of
   two steps. */
int rmhd2d_run(rmhd2d_solver *s, int nsteps);

/* Measurement hooks (the reference has no timers).
   rmhd2d_run_timed: rmhd2d_run(nsteps) bracketed by CUDA events on the
   solver's stream; waits and returns the elapsed device time in *ms.
   rmhd2d_profile_step: one step with CUDA events around each of its four
   launches (stage 1, boundary, stage 2, boundary + CFL reduction); waits and
   returns their device durations in ms[0..3]. */
int rmhd2d_run_timed(rmhd2d_solver *s, int nsteps, float *ms);
int rmhd2d_profile_step(rmhd2d_solver *s, float *ms4);

/* dt of the most recent step: the reference's global `dt` after
   oneStepRK2 (const.hpp:20). */
int rmhd2d_get_dt(rmhd2d_solver *s, double *dt);

/* Sum of the dt of all steps taken: the drivers' `totalTime += dt`
   (main_plasmoid.cu:325). */
int rmhd2d_get_total_time(rmhd2d_solver *s, double *t);

/* Replaces ResistiveMHD2D::checkCalculationIsCrashed()
   (TP resistiveMHD_2D.cu:294-309): *crashed = 1 if any cell of the current
   state has a NaN energy. */
int rmhd2d_check_crashed(rmhd2d_solver *s, int *crashed);

/* Replaces ResistiveMHD2D::save(dir, name, step) (TP resistiveMHD_2D.cu:198-244):
   writes dir/name_step.bin, nx*ny cells of 8 little-endian doubles in the
   field order above, i-major, byte-identical to the reference. */
int rmhd2d_save(rmhd2d_solver *s, const char *directory, const char *name_without_step, int step);

/* Reads a file written by rmhd2d_save (or the reference's save()) back into
   the solver state.  No counterpart in the reference (it cannot resume). */
int rmhd2d_load(rmhd2d_solver *s, const char *path);

/* Writes a host state in the save() format; no GPU needed.  Used by the
   save/load round trip and by host tools. */
int rmhd2d_write_snapshot(const char *path, const double *host_state, int nx, int ny);

/* Tile shape of the fused stage kernels (stage 1 / stage 2 cells per CTA):
   0: 8x32 / 9x32 and 1: 16x16 / 18x16 with 320 threads, 2 CTAs per SM;
   2: 16x32 / 18x32 with 640 threads, 1 CTA per SM (fewer redundant ring
   fluxes per cell); 3: 8x64 / 8x64 with 512 threads, 1 CTA per SM (128
   registers per thread); 4: 8x32 / 8x32 and 5: 6x32 / 7x32 with 256
   threads, 3 CTAs per SM.
   Each stage has its own shape: rmhd2d_set_tile_shape
   sets both, rmhd2d_set_stage_shapes each, rmhd2d_get_tile_shape returns
   stage 1's.  rmhd2d_autotune times trial_steps steps with each shape (CUDA
   events around each stage's launch; the state is restored afterwards),
   keeps the fastest shape of each stage, and returns stage 1's;
   rmhd2d_get_tuning returns the median ms of each stage with each shape (up
   to max entries; *n = the number of shapes tried, 0 before any autotune).
   Results do not depend on the shapes.  No counterpart in the reference
   (its launches are fixed 16x16 thread blocks). */
int rmhd2d_set_tile_shape(rmhd2d_solver *s, int shape);
int rmhd2d_set_stage_shapes(rmhd2d_solver *s, int shape1, int shape2);
int rmhd2d_get_tile_shape(const rmhd2d_solver *s, int *shape);
int rmhd2d_get_stage_shapes(const rmhd2d_solver *s, int *shape1, int *shape2);
int rmhd2d_autotune(rmhd2d_solver *s, int trial_steps, int *best_shape);
int rmhd2d_get_tuning(const rmhd2d_solver *s, int max, int *n, int *shapes, float *ms_stage1, float *ms_stage2);

/* Batches of independent runs (grid size, eta, boundary kinds per run; one
   precision and device per batch), stepped together: every RK2 stage of all
   runs is one persistent launch over a table of all runs' tiles, captured in
   a CUDA graph.  No counterpart in the reference (one run per process).
   Each run is an rmhd2d_solver owned by the batch: use rmhd2d_batch_member
   with the per-solver functions for its state, eta table, dt, total time,
   crash flag and snapshots; stepping and destroying go through the batch. */
typedef struct rmhd2d_batch rmhd2d_batch;
int rmhd2d_batch_create(const rmhd2d_config *cfgs, int nruns, rmhd2d_batch **out);
int rmhd2d_batch_destroy(rmhd2d_batch *b);
int rmhd2d_batch_size(const rmhd2d_batch *b, int *nruns);
int rmhd2d_batch_member(rmhd2d_batch *b, int run, rmhd2d_solver **member);
int rmhd2d_batch_run(rmhd2d_batch *b, int nsteps);
int rmhd2d_batch_run_timed(rmhd2d_batch *b, int nsteps, float *ms);
/* Launch configuration: tile shape (0..5, as above) and persistent CTAs per
   SM (1 up to the shape's CTAs per SM: 2 for shapes 0 and 1, 1 for 2 and 3,
   3 for 4 and 5); rmhd2d_batch_autotune times every valid pair
   (state restored afterwards) and keeps the fastest; rmhd2d_batch_get_tuning
   returns each pair tried with its ms per step (up to max entries, *n =
   the number tried). */
int rmhd2d_batch_set_launch(rmhd2d_batch *b, int shape, int ctas_per_sm);
int rmhd2d_batch_get_launch(const rmhd2d_batch *b, int *shape, int *ctas_per_sm);
int rmhd2d_batch_autotune(rmhd2d_batch *b, int trial_steps, int *best_shape, int *best_ctas_per_sm);
int rmhd2d_batch_get_tuning(const rmhd2d_batch *b, int max, int *n, int *shapes, int *ctas_per_sm,
                            float *ms_per_step);
const char *rmhd2d_batch_last_error(const rmhd2d_batch *b);

/* Discrete adjoint of the step (no counterpart in the reference).
   The adjoint differentiates the map from the initial state and the eta
   field to the state after nsteps steps, with the dt of every step held at
   its recorded value.  Branch points (minmod's choice, the HLLD region, the
   clamped wave speeds) take the derivative of the branch the forward run
   took.  Each wall kind must be periodic or symmetric (any pairing of the
   two); the step must use the stage-1-EMF CT.

   rmhd2d_run_fixed_dt: nsteps steps with the given dts (host array)
   instead of the CFL dt; the state, dt and total time advance as in
   rmhd2d_run.  Used to evaluate the frozen-dt map, e.g. for finite
   differences against the adjoint.

   rmhd2d_adjoint_forward: nsteps steps from the current state (as
   rmhd2d_run), recording each step's dt and keeping the state every
   checkpoint_interval steps (0: ceil(sqrt(nsteps))).  Memory: about
   (nsteps / interval + 2 * interval + 6) states of nx*ny*8 doubles.  A
   negative checkpoint_interval keeps the whole trajectory instead, U^n and
   the stage-1 state of every step (about 2 * nsteps + 7 states), and
   rmhd2d_adjoint_backward then recomputes no step; the gradient is the same
   bit for bit.

   rmhd2d_adjoint_dts: the nsteps dts recorded by the last forward run.

   rmhd2d_adjoint_backward: given seed = dJ/dU_N (nx*ny*8 doubles, the
   state layout above; host memory), writes dJ/dU_0 into grad_state, the
   gradient with respect to the state passed to rmhd2d_set_state with
   apply_boundary = 1 (ghost entries 0, except, with symmetric x walls, bY
   of the lower wall face (j = 2) in columns 3, 4, nx-6, nx-5 and nx-4,
   which the x walls' normal-B integration reads before the y pass replaces
   it), and, when grad_eta is not NULL,
   dJ/d eta into grad_eta (nx*ny, k = j + i*ny; the cell-centred eta field,
   the table when one is set, else the uniform eta spread over the cells).
   Each segment between checkpoints is recomputed once (not at all for a
   kept trajectory); the solver's state is restored to U_N afterwards, so
   backward may be called again with another seed.

   rmhd2d_adjoint_release: frees the recorded trajectory and workspace. */
int rmhd2d_run_fixed_dt(rmhd2d_solver *s, int nsteps, const double *host_dts);
int rmhd2d_adjoint_forward(rmhd2d_solver *s, int nsteps, int checkpoint_interval);
int rmhd2d_adjoint_dts(rmhd2d_solver *s, double *host_dts);
int rmhd2d_adjoint_backward(rmhd2d_solver *s, const double *host_seed, double *host_grad_state,
                            double *host_grad_eta);
int rmhd2d_adjoint_release(rmhd2d_solver *s);

/* CFL dt of a state held in the caller's own device memory, computed
   without allocating device memory.  No counterpart in the reference: it is
   the dt of ResistiveMHD2D::calculateDt() (TP resistiveMHD_2D.cu:277-291),
   the same value rmhd2d_calculate_dt returns for a solver holding that
   state, for callers that cannot allocate while they run: host codes whose
   own pool or arena owns the device memory and hands out pointers only, and
   checks made inside a time loop, where the cudaFree that a temporary
   buffer needs would synchronise the whole device.

   device_state: nx*ny cells in the layout above (ghosts included, every
   cell is scanned), on device cfg->device.  Reads cfg->nx, ny, dx, dy,
   gamma_mhd, cfl, eps, eta, device and stream (NULL: the default stream);
   bc, bc_y and precision are ignored.  The work is enqueued on that stream,
   which is synchronised before *dt is written.  The current device is
   restored before returning.  Errors are reported by
   rmhd2d_last_error(NULL).

   Scratch is a fixed device array inside the library: grids with more than
   RMHD2D_NOALLOC_MAX_CELLS cells (nx*ny) are rejected with
   RMHD2D_ERR_INVALID.  Every call looks up that array's address on the
   device (cudaGetSymbolAddress, which allocates nothing); the first call on
   a device also loads the library's module there, so make it once at
   initialisation, before any stream capture.  The function may not be
   called while cfg->stream is being captured (it synchronises that
   stream): it then returns RMHD2D_ERR_STATE and enqueues nothing.  All
   calls on one device share the array: calls that overlap in time (from
   several host threads) race and may return a wrong dt. */
#define RMHD2D_NOALLOC_MAX_CELLS 16777216
int rmhd2d_calculate_dt_noalloc(const rmhd2d_config *cfg, const double *device_state, double *dt);

/* ---- single domain decomposed into x slabs ----------------------------------
   Replaces the multi-GPU library's decomposition
   (ResistiveMHD_multiGPU_cuda/ResistiveMHD2D_GPU/mpi.cu:104-276: sendrecv_U
   of 3 ghost layers through host-staged MPI_Sendrecv; resistiveMHD2D.cu:550,574:
   MPI_Allreduce of dt and of the crash flag) for the single-GPU library's
   step.  A slab is a solver whose array holds a contiguous range of the
   domain's interior columns i plus 3 columns on each side: the x wall's ghost
   columns where the side is the domain's edge, else a halo of the
   neighbouring slab's first (last) 3 columns.  Periodic x over several
   slabs makes both sides of every slab halos (the first slab's low halo is
   the last slab's high edge).  The library runs the stages and fills wall
   ghosts; the host (the Python SlabDomain, resistivemhd_gpu_b200/slab.py, over
   torch.distributed) moves halo columns between slabs and combines three
   control words across slabs with a max.  The slabs' steps are then
   bit-identical to one solver on the whole domain.

   One step of every slab, in this order:
     rmhd2d_slab_stage(s, 1);  exchange(state 1); rmhd2d_slab_fill(s, 1); exchange(state 1);
     rmhd2d_slab_stage(s, 2);  exchange(state 0); rmhd2d_slab_fill(s, 2); exchange(state 0);
     rmhd2d_slab_get_words(s, w);  max-combine w over slabs;  rmhd2d_slab_set_words(s, w);
   where exchange(k) packs the own edge columns of state k on each halo side
   (rmhd2d_slab_pack) and unpacks the neighbour's into the halo
   (rmhd2d_slab_unpack).  The first exchange of a pair brings the halo's
   interior rows, which the ghost fill of a mirror y wall reads; the second
   brings the ghost rows the neighbour filled.  After rmhd2d_set_state(s, x,
   0) of each slab's part of the initial state: exchange(0);
   rmhd2d_slab_fill(s, 0); exchange(0); rmhd2d_slab_refresh_rate(s); then the
   word combination as above.  Work is enqueued on the solver's stream.
   A slab with halo columns refuses rmhd2d_step_rk2, run, run_fixed_dt,
   profile_step, autotune, calculate_dt, apply_boundary, set_state with
   apply_boundary, and the adjoint: their whole-array work needs the
   exchange. */
#define RMHD2D_SLAB_LO 1      /* the low x side borders another slab (its 3 ghost columns are a halo) */
#define RMHD2D_SLAB_HI 2      /* the high x side borders another slab */
#define RMHD2D_SLAB_ORIGIN 4  /* this slab holds the domain's first interior column (the first slab) */

/* cfg describes the slab's own array: nx = its interior columns + 6, the
   domain's ny, dx, dy and physics; cfg->bc is the x wall on the sides that
   are not halos.  sides: RMHD2D_SLAB_* flags; a slab whose low side is a wall
   must be the first (RMHD2D_SLAB_ORIGIN).  Stage-1-EMF CT only. */
int rmhd2d_create_slab(const rmhd2d_config *cfg, int sides, rmhd2d_solver **out);
/* Doubles of one packed halo: 8 fields x 3 columns x the array's row pitch. */
int rmhd2d_slab_halo_doubles(const rmhd2d_solver *s, long long *n);
/* state: 0 = the current state, 1 = the stage-1 state; side: 0 = low x,
   1 = high x.  pack copies the 3 own columns next to that side into
   dev_buf; unpack copies dev_buf (a neighbour's pack) into that side's halo
   columns (refused on a wall side).  dev_buf: device memory of
   rmhd2d_slab_halo_doubles doubles. */
int rmhd2d_slab_pack(rmhd2d_solver *s, int state, int side, double *dev_buf);
int rmhd2d_slab_unpack(rmhd2d_solver *s, int state, int side, const double *dev_buf);
/* Stage 1 (current -> stage-1 state) or stage 2 (-> current) on the own
   columns, with the dt of the combined words. */
int rmhd2d_slab_stage(rmhd2d_solver *s, int stage);
/* Ghost fill of the wall sides and of the y walls of the own columns:
   which = 0 the current state after set_state / load, 1 the stage-1 state,
   2 the current state after stage 2, with the CFL and NaN reductions of the
   own cells and wall ghosts into the next step's words; 2 ends the step. */
int rmhd2d_slab_fill(rmhd2d_solver *s, int which);
/* The CFL and NaN reductions of the current state (after set_state and its
   fill), into the words of the next step. */
int rmhd2d_slab_refresh_rate(rmhd2d_solver *s);
/* The next step's words w[0..2] = (bits of the maximum CFL rate, cell 0's dt
   candidate is NaN, crash flag), to or from 3 int64 of device memory; the
   host combines them with a max over all slabs in between.  Called after the
   exchange that ends a step (or the initial fill): on the first slab of a
   periodic-x decomposition it also completes the domain's ghost column 0,
   which that slab holds in its low halo. */
int rmhd2d_slab_get_words(rmhd2d_solver *s, long long *dev_words);
int rmhd2d_slab_set_words(rmhd2d_solver *s, const long long *dev_words);

/* Text of the last error of this solver (or of the last failed create when
   s is NULL); never NULL. */
const char *rmhd2d_last_error(const rmhd2d_solver *s);

/* Name of a status code. */
const char *rmhd2d_status_string(int status);

/* ABI version (RMHD2D_ABI_VERSION of the library). */
int rmhd2d_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif
