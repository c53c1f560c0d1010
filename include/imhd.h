/*
 * imhd.h -- C ABI of the B200 isothermal-MHD time-step library (libimhd.so).
 *
 * The reference (tsultan16/Isothermal_MHD, 3D_MPI) is a Fortran 90 program
 * whose hot path is a handful of module procedures acting on module-global
 * arrays.  This header is the drop-in boundary for that path: a Fortran
 * driver binds these entry points through ISO_C_BINDING (the binding module
 * declares these prototypes as BIND(C) interfaces), a C/C++ or Python
 * (ctypes) host binds them directly.
 *
 * Conventions
 *  - Every call returns an int status: IMHD_OK (0) or a positive IMHD_E_* code;
 *    imhd_last_error() returns a message for the calling thread.  Nothing
 *    throws across this boundary.  (The reference PRINTs and STOPs instead:
 *    vanleer_mod.f90:131-133, 3328-3331; turb_driver_mod.f90:32-35, 420-425.)
 *  - Host arrays are borrowed for the duration of the call only.  They use the
 *    reference's own layout: Fortran column-major, interior cells 1..n per
 *    axis with `ng` ghost layers on each side, field index slowest.  That is
 *    q_3d(1-ng:nx+ng,1-ng:ny+ng,1-ng:nz+ng,7), bface_3d(...,3) and
 *    qpass_3d(1-ngp:nx+ngp,...,npass) of 3D_MPI/src/grid_data_mod.f90:38-43
 *    (ng = nb = 6 and ngp = nb-2 = 4 there); ng = 0 means unpadded arrays.
 *  - State lives on the device between calls (one box per handle, one CUDA
 *    stream per handle).  A handle is not thread safe; use one per host
 *    thread.
 *  - Boundaries are periodic (boundary_type = 2, constants_mod.f90:36); the
 *    ghost zones of the reference become an index wrap inside the kernels.
 */
#ifndef IMHD_H
#define IMHD_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define IMHD_OK 0
#define IMHD_E_ARG 1        /* bad argument or configuration */
#define IMHD_E_CUDA 2       /* CUDA runtime error (no device, launch failure) */
#define IMHD_E_NOMEM 3      /* device allocation failed */
#define IMHD_E_PHYSICS 4    /* non-finite state, zero max speed or bad forcing normalisation */
#define IMHD_E_STATE 5      /* call out of order (e.g. drive without a force field) */

/* Riemann solvers (riemann_solver_type, constants_mod.f90:57) */
#define IMHD_ROE 1
#define IMHD_HLLD 2
#define IMHD_HLLE 3

/* interface reconstruction: piecewise_parabolic (vanleer_mod.f90:83) of the
 * characteristic variables (the reference's default, :1488-1818) or, with
 * primitive_reconstruction (:84), of the primitive variables (:1144-1485) */
#define IMHD_PLM 0
#define IMHD_PPM 1
#define IMHD_PLM_PRIM 2
#define IMHD_PPM_PRIM 3

/* status-word bits reported by imhd_status */
#define IMHD_S_FLOOR 1u     /* a density fell below 1e-20 and was floored (vanleer_mod.f90:3243-3262) */
#define IMHD_S_NAN 2u       /* a non-finite updated state or max speed was seen */
#define IMHD_S_ZERO_SPEED 4u/* max speed < 1e-20 (vanleer_mod.f90:3328) */
#define IMHD_S_FORCE 8u     /* forcing quadratic term <= 1e-20 (turb_driver_mod.f90:420) */
#define IMHD_S_WAIT 16u     /* a bounded wait for an asynchronous copy in a kernel gave up; the step is not valid */
#define IMHD_S_PROTECT 32u  /* flux protection found more bad cells than its list holds (2^20 per update); the step is not valid */

typedef struct imhd_config {
    int nx, ny, nz;        /* interior cells per axis (constants_mod.f90:9-11) */
    int precision;         /* 64: FP64 everywhere; 32: FP32 bulk, FP64 reductions */
    int riemann;           /* IMHD_ROE / IMHD_HLLD / IMHD_HLLE */
    int recon;             /* IMHD_PLM, IMHD_PPM, IMHD_PLM_PRIM or IMHD_PPM_PRIM */
    int npass;             /* passive scalars, 0..8 (constants_mod.f90:63) */
    double sound_speed;    /* isothermal sound speed (constants_mod.f90:35) */
    double cour;           /* COUR_def (constants_mod.f90:16) */
    double edot;           /* kinetic-energy injection rate (constants_mod.f90:44) */
    double dt_turb;        /* forcing interval (constants_mod.f90:42) */
    int ng;                /* ghost layers of host q / bface / delv arrays */
    int ng_pass;           /* ghost layers of host qpass arrays */
    int device;            /* CUDA device ordinal */
    int protect;           /* 1: flux_protection (vanleer_mod.f90:81, off in the reference) for an IMHD_ROE box: HLLE
                            * fluxes of the same interface states are kept beside the Roe fluxes (their wave speeds
                            * enter smax, :2962), and after each update the cells whose density fell below 1e-20 and
                            * their six neighbours are updated again with the HLLE fluxes on the bad cells' faces and
                            * the HLLE corner EMFs (:2086-2202); needs 21 more fields of device memory */
} imhd_config;

typedef struct imhd_box imhd_box;

/* Fill *cfg with the reference's defaults (64^3, FP64, HLLD, PLM, npass 1,
 * cs 1, COUR 0.35, Edot 1e-3, dt_turb 0.05, ng 6, ng_pass 4, device 0). */
void imhd_default_config(imhd_config* cfg);

/* Allocate a box on cfg->device.  Replaces create_grid_arrays
 * (grid_data_mod.f90:33-67), init_solver_vanleer / allocate_local_variables
 * (vanleer_mod.f90:127-244) and init_passive_solver (passive_mod.f90:44-111). */
int imhd_create(const imhd_config* cfg, imhd_box** box);

/* Copy the host state into the box: q_3d, bface_3d (ng ghosts) and qpass_3d
 * (ng_pass ghosts; may be NULL when npass = 0).  Only interior cells are read.
 * Replaces the state hand-over after init_state / read_restart
 * (driver.f90:283-333). */
int imhd_upload(imhd_box* box, const double* q, const double* bface, const double* qpass);

/* Copy the box state to host arrays in the same layout.  Ghost layers, when
 * ng > 0, are filled with periodic images, i.e. the arrays read as the
 * reference's do after boundary_conditions() (boundary_conditions_mod.f90:137-231).
 * Any pointer may be NULL to skip that array. */
int imhd_download(imhd_box* box, double* q, double* bface, double* qpass);

/* Set the turbulence forcing field delv(1-ng:nx+ng,...,3), the layout of the
 * add_random_force dummy argument (turb_driver_mod.f90:398).  Replaces the
 * hand-over of delv_re produced by generate_rand_force (:197-391). */
int imhd_set_force(imhd_box* box, const double* delv);
/* The force field of the box, in the layout of imhd_set_force. */
int imhd_get_force(imhd_box* box, double* delv);
/* This box's forcing sums of its current state over its own planes
 * (imhd_set_geometry): sums[0] = 1/2 sum rho |delv|^2, sums[1] = sum delv.m,
 * sums[2..4] = sum rho delv -- get_rho_turb's quad_term1, quad_term2 and
 * mom{x,y,z}_avg before their all-reduce (turb_driver_mod.f90:158-189).
 * Needs imhd_set_force. */
int imhd_force_sums(imhd_box* box, double* sums);
/* All ranks' sums for the box's next drive step, which then normalises the
 * kick with them instead of its own (the end_allreduce results of
 * add_random_force, turb_driver_mod.f90:402-415).  Used once. */
int imhd_set_force_sums(imhd_box* box, const double* sums);

/* One time step of the reference driver loop for one rank: copy_velocity,
 * vanleer_solve_3d(dt, drive_next) (vanleer_mod.f90:279-426, incl.
 * get_rho_turb / add_random_force when drive_next != 0), copy_velocity,
 * passive_solve_3d (passive_mod.f90:118-201), the periodic ghost fill and
 * compute_new_time_step (driver.f90:55-131, 432-448).  On return *dt_next holds
 * the new local dt = COUR*dx/cmax with COUR halved after a drive step
 * (driver.f90:109); the caller applies MIN(t_end - t, dt) (driver.f90:475).
 * A step that leaves a non-finite state or max speed returns IMHD_E_PHYSICS
 * (IMHD_S_NAN stays set in imhd_status); the reference has no such check and
 * would carry the NaN into its next dt. */
int imhd_step(imhd_box* box, double dt, int drive_next, double* dt_next);

/* cmax of the current state alone: get_max_speed_vanleer with smax = 0
 * (vanleer_mod.f90:3266-3334), used for a first dt without the 1e-15 warm-up. */
int imhd_max_speed(imhd_box* box, double* cmax);

/* out[0..5] = KE, v_rms^2 sum, momx, momy, momz (compute_KE, driver.f90:518-553)
 * and the div B sum (compute_divB, driver.f90:492-515), all FP64. */
int imhd_diagnostics(imhd_box* box, double out[6]);

/* Sticky status word (IMHD_S_* bits) and the count of floored densities;
 * reset != 0 clears both. */
int imhd_status(imhd_box* box, unsigned* flags, long long* floor_hits, int reset);

/* smax of the last step (largest interface wave speed, vanleer_mod.f90:2341,
 * 2962, 3086) and delv_max of the last forcing kick (turb_driver_mod.f90:451). */
int imhd_wave_speeds(imhd_box* box, double* smax, double* delv_max);

/* Free the box.  Replaces destroy_grid_arrays / destroy_solver_vanleer /
 * destroy_passive_solver (driver.f90:213-226). */
void imhd_destroy(imhd_box* box);

/* Message of the last failing call on this thread. */
const char* imhd_last_error(void);

/* Number of kernel launches issued by this box since creation. */
long long imhd_launch_count(imhd_box* box);

/* Run the box's device work on the caller's CUDA stream (a cudaStream_t passed
 * as void*, e.g. the stream of a host framework); NULL restores the box's own
 * stream.  No reference counterpart (the reference has no device). */
int imhd_set_stream(imhd_box* box, void* stream);

/* Per-stage CUDA-event timing of imhd_step: enable != 0 switches it on.
 * No reference counterpart; it plays the role of the reference's MPI_Wtime
 * brackets around the solve (driver.f90:52, 82-83). */
int imhd_profile(imhd_box* box, int enable);

/* Accumulated device milliseconds and timed-step counts per stage, in the
 * launch order of a step: 0 forcing sums, 1 predictor fluxes, 2 predictor
 * EMF, 3 predictor update, 4-6 corrector fluxes x/y/z, 7 corrector EMF,
 * 8 final update, 9 forcing kick, 10 passive predictor, 11 passive corrector,
 * 12 dt finalisation.  n must be IMHD_NSTAGES; reset != 0 clears them. */
#define IMHD_NSTAGES 13
int imhd_stage_times(imhd_box* box, double* ms, long long* count, int n, int reset);

/* Fill a box from a sum of Fourier modes on the cell centres,
 * v_d(x) = sum_m 2 Re(A_{m,d} exp(2 pi i k_m . x)), x = ((i+1/2)/nx, ...):
 * kvec[3m..3m+2] are integer wave numbers, amp[6m + 2d] / amp[6m + 2d + 1]
 * the real / imaginary part of A_{m,d}.  target 0 adds rho * scale * v to the
 * momentum (an initial velocity field), target 1 sets the force field to
 * scale * v.  The device counterpart of generate_rand_force's inverse DFT
 * (turb_driver_mod.f90:310-384) for generators whose amplitudes live on the
 * host, e.g. the Ornstein-Uhlenbeck forcing of isothermal_mhd_b200.forcing. */
int imhd_fourier_field(imhd_box* box, int target, const int* kvec, const double* amp, int nmodes, double scale);

/* The reference's turbulence force generator on the device
 * (turb_driver_mod.f90:23-79, 104-126, 197-391).  imhd_init_turb seeds the
 * taus88 generator (the reference's defaults are 1234, 5678, 9123,
 * constants_mod.f90:23) and sets k_max (2 in the reference; must be
 * < min(nx, ny, nz) / 2).  imhd_generate_force draws the next random
 * spectrum (serially, on the host, in the reference's order), projects it
 * solenoidal, and evaluates the separable inverse DFT on the device into the
 * box's force field, as imhd_set_force would set it; the generator state
 * advances, and imhd_turb_seeds reads it (for restart files). */
int imhd_init_turb(imhd_box* box, int s1, int s2, int s3, int k_max);
int imhd_generate_force(imhd_box* box);
int imhd_turb_seeds(imhd_box* box, int* s1, int* s2, int* s3);

/* Uniform state: density rho, zero momentum, cell-centre and face field
 * b0[3], passive scalars 0, as homogenous_stationary sets it up
 * (init_domain_mod.f90:406-479); with imhd_fourier_field it builds a
 * turbulence initial condition on the device without a host upload. */
int imhd_init_uniform(imhd_box* box, double rho, const double* b0);

/* ---- one box split over ranks: z slabs with halo planes ------------------
 * A rank's slab is a box of nz_local + 2*H planes whose planes [H, H+nz_local)
 * are its own and whose H planes on each side are copies of the neighbours'
 * (the reference's halo exchange, mpi_domain_mod.f90:618-649, 674-3091).  A
 * step runs over the whole slab with the periodic wrap in z, which corrupts
 * only the outer planes: with H >= 6 (the reference's nb, enough for PLM and
 * PPM) the own planes come out exact, and one exchange per step refreshes
 * the halo.  imhd_set_geometry gives the global dx (1 / max global edge) and
 * the own plane range [zlo, zhi): only those planes enter the step's speed
 * maxima, floor counts, status, CFL and diagnostics, so the maxima over ranks
 * equal the single-box ones.  imhd_pack_planes / imhd_unpack_planes copy
 * planes [z0, z0 + nplanes) of every state field to / from a contiguous
 * device buffer (field-major, (10 + npass) * nplanes * nx * ny elements of
 * the box's precision) for the exchange; both return when the copy is done.
 * Forcing across ranks needs global sums and is not offered on slabs. */
int imhd_set_geometry(imhd_box* box, double dx, int zlo, int zhi);
int imhd_pack_planes(imhd_box* box, int z0, int nplanes, void* dst);
int imhd_unpack_planes(imhd_box* box, int z0, int nplanes, const void* src);

/* ---- output and restart files (io_mod.f90) --------------------------------
 * Written from the box's current state on the device (the cell records are
 * packed there) and read back into it.  double_prec selects REAL*8 output,
 * otherwise SNGL (round to nearest REAL*4) as the reference's double_prec
 * switch does.
 *
 * imhd_write_xyzcube: the xyzcube_rank=XYZ_dump=N.dat stream file
 *   (io_mod.f90:249-277): per interior cell, i fastest, q(1..7) and, when
 *   npass > 0, the first passive scalar.
 * imhd_write_state_dump: the per-rank block of the parallel dump
 *   (io_mod.f90:378-432): per cell q(1..7) and every passive scalar.
 * imhd_write_cuts: the cut files of io_mod.f90:62-240 into directory dir,
 *   named as the reference names them for rank (0,0,0); flags selects them;
 *   riemann (IMHD_ROE/HLLD/HLLE) names the xcut file.
 * imhd_write_restart / imhd_read_restart: restart_mhd_rank=XYZ.dat
 *   (io_mod.f90:440-517), Fortran sequential unformatted records with
 *   gfortran's record markers: t_sim, q_3d and bface_3d with ghost width nb
 *   (6 in the reference), qpass_3d with ghost width nb - 2 when npass > 0,
 *   dump_count and the forcing generator's seeds s1, s2, s3.  Reading checks
 *   every record length against the box's shape. */
#define IMHD_CUT_X 1
#define IMHD_CUT_Y 2
#define IMHD_CUT_Z 4
#define IMHD_CUT_XYDIAG 8
#define IMHD_CUT_YZDIAG 16
#define IMHD_CUT_XYPLANE 32
int imhd_write_xyzcube(imhd_box* box, const char* path, int double_prec);
int imhd_write_state_dump(imhd_box* box, const char* path, int double_prec);
int imhd_write_cuts(imhd_box* box, const char* dir, int dump, int flags, int riemann, int double_prec);
int imhd_write_restart(imhd_box* box, const char* path, double t_sim, int nb, int dump_count, int s1, int s2, int s3);
int imhd_read_restart(imhd_box* box, const char* path, int nb, double* t_sim, int* dump_count, int* s1, int* s2,
                      int* s3);

/* ---- batches: many independent periodic boxes advanced together --------
 * All boxes of a batch share precision and device; sizes, Riemann solvers,
 * passive counts and physics parameters may differ.  Every kernel launch of a
 * step covers all boxes.  Each box keeps its own clock on the device and runs
 * the reference driver loop (driver.f90:35-186) by itself: first dt, drive
 * schedule, dt halving, COUR halving after a drive, MIN(t_end - t, dt).  One
 * step of the whole batch is captured once into a CUDA graph and replayed.
 * No reference counterpart (the reference advances one box per process). */
typedef struct imhd_batch imhd_batch;
int imhd_batch_create(const imhd_config* cfgs, int nbox, imhd_batch** batch);
int imhd_batch_upload(imhd_batch* batch, int box, const double* q, const double* bface, const double* qpass);
int imhd_batch_set_force(imhd_batch* batch, int box, const double* delv);
int imhd_batch_download(imhd_batch* batch, int box, double* q, double* bface, double* qpass);
/* Start the clock of one box: time t0, end time t_end, number of steps, first
 * dt (the reference uses 1e-15, driver.f90:249; dt0 <= 0 takes COUR*dx/cmax of
 * the uploaded state), forcing on (needs edot > 0) or off. */
int imhd_batch_schedule(imhd_batch* batch, int box, double t0, double t_end, long long steps, double dt0,
                        int forcing);
/* Replay the batch step `replays` times; boxes that have made their steps or
 * reached t_end stay as they are. */
int imhd_batch_run(imhd_batch* batch, int replays);
/* Clock of one box: time, steps made, next dt, still running. */
int imhd_batch_clock(imhd_batch* batch, int box, double* t, long long* steps, double* dt, int* active);
int imhd_batch_init_uniform(imhd_batch* batch, int box, double rho, const double* b0);
int imhd_batch_fourier_field(imhd_batch* batch, int box, int target, const int* kvec, const double* amp, int nmodes,
                             double scale);
int imhd_batch_set_stream(imhd_batch* batch, void* stream);
/* Online tuning of the batch's decomposition: the first replays of a run try
 * y/z sweep segments (16, 8, 32 faces per thread) and x tile widths (the
 * widest that each row length divides, or 32), one real step each, timed
 * with CUDA events, by coordinate descent; the fastest is kept for the rest
 * of the batch's life.  Every setting computes the same bits, so tuning
 * changes timing only: FP64 tunes both; FP32 tunes the tile width only,
 * because the first slope of a segment is computed by a separate copy of the
 * code whose FMA contraction may differ from the loop's, so the segment
 * length could move the last bit.  enable: 1 on (the default), 0 off,
 * < 0 leaves it; the current setting is returned (tile_policy 0 widest,
 * 1 always 32; z_column is the fixed z-column length of the cell kernels). */
int imhd_batch_tuning(imhd_batch* batch, int enable, int* done, int* tile_policy, int* sweep_segment,
                      int* z_column);
long long imhd_batch_launch_count(imhd_batch* batch);
void imhd_batch_destroy(imhd_batch* batch);

/* ---- serving: a request loop with continuous batching -------------------
 * imhd_server_start launches a worker thread that owns one device.  Requests
 * (a box solve: configuration, step count, initial condition, forcing) are
 * queued by imhd_server_submit from any host thread; a builder thread admits
 * them in arrival order while their device bytes fit hbm_budget_bytes (and,
 * if max_resident_cells > 0, while the resident cells stay under it) and
 * builds each box on the device while the worker steps, and the worker
 * advances all resident boxes together with the batched step (per-box clocks
 * as in imhd_batch_*).  Every steps_per_round
 * replays it retires finished boxes (result copied to host memory, device
 * memory freed) and admits waiting ones, so requests that arrive while others
 * run join the running batch.  A box's result does not depend on what else
 * is resident.  No reference counterpart (the reference runs one box per job).
 *
 * The initial condition of a request is a uniform state (rho, b0) plus the
 * velocity of nmodes Fourier modes (imhd_fourier_field's convention, target
 * velocity, amp_velocity scaled by scale_velocity); forcing != 0 drives the
 * box on the reference schedule with the force field of amp_force scaled by
 * scale_force (needs box.edot > 0).  dt0 <= 0 starts from COUR*dx/cmax of the
 * initial state; t_end <= 0 means no end time (steps alone stop the box).
 * box.precision and box.device are taken from the server. */
typedef struct {
    int device;
    int precision;                /* 32 or 64 for every box of the server */
    double hbm_budget_bytes;      /* device bytes of resident boxes */
    long long max_resident_cells; /* 0: no limit besides the budget */
    int steps_per_round;          /* graph replays between retire / admit passes */
} imhd_server_config;

typedef struct {
    imhd_config box;
    long long steps;
    double t_end, dt0;
    double rho;
    double b0[3];
    int nmodes;
    const int* kvec;              /* 3 * nmodes */
    const double* amp_velocity;   /* 6 * nmodes or NULL */
    double scale_velocity;
    const double* amp_force;      /* 6 * nmodes, used when forcing != 0 */
    double scale_force;
    int forcing;
} imhd_request;

#define IMHD_REQ_QUEUED 0
#define IMHD_REQ_RUNNING 1
#define IMHD_REQ_DONE 2
#define IMHD_REQ_FAILED 3
#define IMHD_REQ_CANCELLED 4
#define IMHD_SERVER_NSTATS 16

typedef struct imhd_server imhd_server;
void imhd_server_default_config(imhd_server_config* cfg);
int imhd_server_start(const imhd_server_config* cfg, imhd_server** server);
/* Queue a request; *id names it in imhd_server_poll.  The arrays are copied. */
int imhd_server_submit(imhd_server* server, const imhd_request* req, long long* id);
/* State of a request (IMHD_REQ_*) and info[5] = {t, steps made, latency from
 * submit to result on the host in s (-1 before), queue wait in s, status
 * bits}.  When the request is done and any of q / bface / qpass is non-NULL,
 * the result is copied there (layout of imhd_download with the request's
 * ghost widths) and released: the id is unknown afterwards.  A failed
 * request returns IMHD_E_PHYSICS with the reason in imhd_last_error. */
int imhd_server_poll(imhd_server* server, long long id, int* state, double* q, double* bface, double* qpass,
                     double* info);
/* {queued, resident, admitted, completed, failed, graph replays, kernel
 * launches, table rebuilds, resident bytes, peak resident bytes, peak
 * resident boxes, then seconds the builder spent building admitted boxes,
 * seconds the worker spent rebuilding the table and graph, stepping, reading
 * clocks and retiring, and seconds the harvester spent downloading results};
 * n >= IMHD_SERVER_NSTATS.  Admitted boxes are built by a builder thread on a
 * stream of its own, and finished boxes downloaded by a harvester thread on
 * another, while the step loop goes on; a box's memory counts against the
 * budget from its admission until its download ends. */
int imhd_server_stats(imhd_server* server, double* out, int n);
/* Stop the worker: drain != 0 finishes every queued and running request
 * first, drain == 0 cancels them.  Results stay pollable until destroy. */
int imhd_server_stop(imhd_server* server, int drain);
void imhd_server_destroy(imhd_server* server);

/* One undriven time step with PLM reconstruction, like imhd_step, for callers
 * that cannot allocate device memory: hosts that own every device buffer
 * (pool allocators, OpenACC or CUDA Fortran arrays whose runtime keeps the
 * device heap to itself) and real-time loops that forbid allocation after
 * start-up.  No reference counterpart: the reference allocates its work
 * arrays itself (vanleer_mod.f90:169-244).
 * The caller passes device buffers: state_in (read) and state_out (written),
 * distinct, each 10 + npass fields of nx*ny*nz elements of the precision's
 * type in the library's layout (rho, mx, my, mz, Bx_cc, By_cc, Bz_cc,
 * Bx_face, By_face, Bz_face, passive scalars; x fastest).  dt is read from
 * the host, *dt_next (host) receives COUR*dx/cmax, stream may be NULL; the
 * call returns when the step is done.  Reconstruction is always PLM and
 * there is no forcing kick (use imhd_create / imhd_step for PPM or driving).
 * The step's work arrays live in one 48 MiB file-scope device array held by
 * every GPU that loads the library until exit; boxes needing more
 * ((21 + npass) * nx*ny*nz * element size + 56 KiB: 64^3 in FP64 with at most
 * two passive scalars, about 80^3 in FP32 with two) are rejected with
 * IMHD_E_ARG.  All calls on a device share that array and leave their
 * contents in it: calls that overlap on the GPU race.  The first call on a
 * device looks up the array's device address and keeps it for the life of
 * the process, so the library must not be used across a cudaDeviceReset.
 * A non-finite result returns IMHD_E_PHYSICS; floored densities are not
 * reported by this entry point. */
int imhd_step_static(int precision, int nx, int ny, int nz, int riemann, int npass, double sound_speed,
                     double cour, const void* state_in, void* state_out, double dt, double* dt_next,
                     void* stream);

#ifdef __cplusplus
}
#endif

#endif /* IMHD_H */
