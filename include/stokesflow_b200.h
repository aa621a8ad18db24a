/*
 * stokesflow_b200.h -- C ABI of libstokesflow_b200.so, the B200 (sm_100a)
 * implementation of the per-timestep hot path of StokesFlow.jl:
 * marker->grid deposit, pseudo-transient Stokes solve, RK4 marker advection
 * and marker->cell rebinning, on a single domain (one GPU, no MPI).
 *
 * Conventions
 *  - Grid arrays are the reference's Julia arrays: dense, column-major
 *    (x index fastest) Float64 device buffers; an (nx, ny) array A holds
 *    A[ix, iy] (1-based) at A[(ix-1) + (iy-1)*nx].  Marker arrays are 1-D.
 *  - All array arguments are DEVICE pointers (cudaMalloc'd, managed, or
 *    Julia CuArray storage) unless the name ends in _host.
 *  - `stream` is a cudaStream_t passed as void* (NULL = legacy default).
 *    Calls are asynchronous on that stream unless a host-side scalar result is
 *    returned (sf_solve_stokes, sf_get_warnings, sf_stokes_residual_scale),
 *    which synchronises the stream.
 *  - Every function returns an sf_status (0 = SF_OK).  Warnings that the
 *    reference prints and continues past are counted on the device instead and
 *    read with sf_get_warnings.
 *  - A context owns all scratch device memory for one device; it is not
 *    thread-safe: use one context per host thread / stream.
 *  - The reference's MPI communicator / ImplicitGlobalGrid arguments (`comm`,
 *    `grid`) have no counterpart: the domain is a single rank, so every
 *    overlap sum, halo update and Allreduce is the identity.
 */
#ifndef STOKESFLOW_B200_H
#define STOKESFLOW_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    SF_OK = 0,
    SF_ERR_INVALID_ARG = 1,   /* bad size / NULL pointer / misaligned layout; reference: AssertionError */
    SF_ERR_CUDA = 2,          /* a CUDA runtime call failed (message in sf_last_error)                 */
    SF_ERR_OOM = 3,           /* scratch allocation failed                                              */
    SF_ERR_NO_DEVICE = 4,     /* no CUDA device / device index out of range                             */
    SF_ERR_NONFINITE = 5,     /* the PT iteration produced NaN/Inf (err is not finite)                  */
    SF_ERR_TOO_LARGE = 6,     /* a size exceeds what the entry point supports                           */
    SF_ERR_BUSY = 7           /* an engine's arena or instance table is full now; retry once instances
                                 have finished (admission control, sf_engine_submit)                    */
} sf_status;

typedef struct sf_ctx sf_ctx;

/* ---------------------------------------------------------------------- */
/* library / context                                                       */
/* ---------------------------------------------------------------------- */
int sf_version(void);                          /* (major<<16)|(minor<<8)|patch */
const char* sf_status_string(int status);
const char* sf_last_error(void);               /* thread-local text of the last failure */

int sf_ctx_create(int device, sf_ctx** out);
int sf_ctx_destroy(sf_ctx* ctx);
/* Bytes of device scratch currently held by the context. */
int sf_ctx_scratch_bytes(sf_ctx* ctx, int64_t* bytes);
/* Number of kernels launched through the context since its creation. */
int sf_ctx_launch_count(sf_ctx* ctx, int64_t* launches);

/* Device-side counters of the reference's printed warnings.  reset != 0
 * zeroes them after reading.  Synchronises the context's device. */
typedef struct {
    int64_t bad_markers;      /* MarkerToGrid.jl:66-67,120-121 "erroneous marker position"     */
    int64_t empty_nodes;      /* MarkerToGrid.jl:166-169 "no markers close enough" (value kept) */
    int64_t interp_failsafe;  /* MoveMarkers.jl:80-99,128-147 index-range failsafes             */
    int64_t markers_outside;  /* sf_rebin_markers: markers outside every cell                   */
} sf_warnings;
int sf_get_warnings(sf_ctx* ctx, sf_warnings* out, int reset);

/* Self-test of the bounded waits that every persistent kernel uses (a wall-clock budget on an mbarrier, then an
 * error flag instead of a hang).  One block waits on a shared-memory barrier for at most budget_ns
 * (1 .. 2e9): with arrive != 0 the barrier is completed first and *timed_out is 0; with arrive == 0 nothing
 * completes it, every thread gives up after the budget and *timed_out is 1.  Either way the kernel returns
 * and the context stays usable.  Synchronises the context's work stream. */
int sf_selftest_bounded_wait(sf_ctx* ctx, int arrive, int64_t budget_ns, int32_t* timed_out);

/* ---------------------------------------------------------------------- */
/* marker->grid deposit                                                     */
/* ---------------------------------------------------------------------- */
/* Replaces bilinearMarkerToGrid!(x_grid_min, y_grid_min, val_grid, x_m, y_m,
 * val_m, dx, dy, val_wt_sum, wt_sum, grid)  (scripts/MarkerToGrid.jl:18-38).
 * val_grid is (nx, ny).  Each node gets sum(w*val)/sum(w) over the markers of
 * its four adjacent cells, with the bilinear weights of MarkerToGrid.jl:110-155;
 * the sums are taken in ascending marker index, the order of the reference's
 * serial CPU loop, so the result is bit-identical to it and deterministic
 * (no floating-point atomics).  Nodes with zero weight keep their previous
 * value (safeDivision, :164-172) and are counted in empty_nodes; markers whose
 * cell is outside 0..nx x 0..ny are skipped and counted in bad_markers.
 * val_wt_sum / wt_sum are optional (NULL): when given they are the
 * reference's work arrays of n_sum elements with leading dimension ld_sum
 * (ld_sum >= nx), zeroed and then filled with the sums as in :24-28. */
int sf_bilinear_marker_to_grid(sf_ctx* ctx, double x_grid_min, double y_grid_min,
                               double* val_grid, int64_t nx, int64_t ny,
                               const double* x_m, const double* y_m, const double* val_m,
                               int64_t nm, double dx, double dy,
                               double* val_wt_sum, double* wt_sum, int64_t ld_sum, int64_t n_sum,
                               void* stream);

/* The deposits of one StokesFlow2D timestep in one call (the three calls of
 * StokesFlow2D_multixpu.jl:164-166: rho_vy, mu_b, mu_p): up to SF_MAX_GRIDS
 * grids over the same markers, each with its own origin, extents, output and
 * marker values.  The result is that of sf_bilinear_marker_to_grid called once
 * per grid in the given order, bit for bit: each grid as described there, the
 * warning counters summed over the grids, and val_wt_sum / wt_sum (optional,
 * large enough for every grid) holding the last grid's sums.  The markers'
 * positions are read once for all grids' cell assignments.  All arguments are
 * checked before any work starts. */
#define SF_MAX_GRIDS 4
typedef struct {
    double x_grid_min, y_grid_min;
    double* val_grid;        /* (nx, ny), column-major                              */
    int64_t nx, ny;
    const double* val_m;     /* the marker values deposited onto this grid          */
} sf_deposit_grid;
int sf_bilinear_marker_to_grids(sf_ctx* ctx, const sf_deposit_grid* grids, int n_grids,
                                const double* x_m, const double* y_m, int64_t nm, double dx, double dy,
                                double* val_wt_sum, double* wt_sum, int64_t ld_sum, int64_t n_sum,
                                void* stream);

/* Allocation-free deposit.  No counterpart in the reference: it is
 * sf_bilinear_marker_to_grid (same result, bit for bit) for callers that cannot
 * let a library allocate device memory -- a host runtime that owns the GPU
 * memory through its own pool, a latency-critical stream loop that cudaMalloc /
 * cudaFree would stall with their device-wide synchronisation, a process held
 * to a fixed memory budget.  It takes no context and allocates nothing: its
 * scratch is a fixed array inside the library (about 11 MB, held on every GPU
 * that loads the library until the process exits), so it accepts at most
 * SF_NOALLOC_MAX_MARKERS markers and grids with (nx+1)*(ny+1) <=
 * SF_NOALLOC_MAX_CELLS, and returns SF_ERR_TOO_LARGE beyond that.  It runs on
 * the calling thread's current device.  The first call on a device looks up
 * the array's device address (cudaGetSymbolAddress) and the device's SM count
 * and caches both for the life of the process; make that first call before
 * any stream capture.  A cudaDeviceReset (or any teardown of the device's
 * primary context) invalidates that cache: after one, do not call this entry
 * point again in the same process.  All calls share the one array, so
 * calls whose work overlaps on the GPU (different streams, or different host
 * threads on the same device) race and must be serialised by the caller.
 * Warning counts are not reported.  val_wt_sum / wt_sum are not produced. */
#define SF_NOALLOC_MAX_MARKERS 1048576
#define SF_NOALLOC_MAX_CELLS 262144
int sf_bilinear_marker_to_grid_noalloc(double x_grid_min, double y_grid_min, double* val_grid, int64_t nx,
                                       int64_t ny, const double* x_m, const double* y_m, const double* val_m,
                                       int64_t nm, double dx, double dy, void* stream);

/* ---------------------------------------------------------------------- */
/* pseudo-transient Stokes solve                                             */
/* ---------------------------------------------------------------------- */
typedef struct {
    double dt;               /* compute_dt of the final velocities (StokesSolver_multixpu.jl:95)      */
    double T_eff;            /* GB/s, reference definition 6*Nx*Ny*8 B / t_it (:78-81)                */
    double runtime;          /* seconds of iterations >= 11 (:38,44-46,78), CUDA-event timed          */
    int64_t iters;           /* niter                                                                 */
    double err;              /* last residual norm max(mean|Rx|, mean|Ry|, mean|divV|) (2*eps if none)*/
    int64_t n_checks;        /* residual checks performed (every ncheck iterations)                   */
    int32_t converged;       /* err <= eps                                                             */
    int32_t reserved;
    double loop_ms;          /* device time of the whole iteration loop                                */
    double bytes_per_iter;   /* essential HBM bytes of one fused PT iteration: 8*[2*(|Vx_s|+|Vy_s|+|P|+  */
                             /* |dVx|+|dVy|) + |rho_vy|+|mu_b|+|mu_p|], about 104*Nx*Ny                */
    double T_eff_essential;  /* bytes_per_iter * iters / loop time, GB/s                               */
    int64_t fused_launches;  /* launches of the fused PT iteration kernel                              */
    double fused_ms;         /* device time of the fused launches alone (0 unless timing requested)    */
} sf_solve_info;

/* Replaces solveStokes!(P, Vx_pad, Vy_pad, rho_vy, mu_b, mu_p, txx, tyy, txy,
 * divV, dtPt, Rx, Ry, dVxdt, dVydt, dtVx, dtVy, Vx_s, Vy_s, g_y, dx, dy, Nx, Ny,
 * dt, maxdisp, comm; use_free_surface_stabilization, eps, print_info, iterMax)
 * (scripts/StokesSolver_multixpu.jl:14-96).  Sizes as in the reference:
 *   P (Nx-1,Ny-1) Vx_pad (Nx+2,Ny+1) Vy_pad (Nx+1,Ny+2) rho_vy (Nx+1,Ny) mu_b (Nx,Ny)
 *   mu_p,txx,tyy,divV,dtPt (Nx-1,Ny-1) txy (Nx,Ny) Rx,dVxdt,dtVx (Nx-2,Ny-1)
 *   Ry,dVydt,dtVy (Nx-1,Ny-2) Vx_s (Nx,Ny+1) Vy_s (Nx+1,Ny).
 * State (P, Vx_s, Vy_s, dVxdt, dVydt) is read as the warm start and written
 * back; Vx_pad / Vy_pad receive the padded, mirrored velocities.  The work
 * arrays txx, tyy, txy, divV, dtPt, Rx, Ry, dtVx, dtVy may be NULL; when given
 * they end with the values the reference leaves in them.  Synchronises the
 * stream (the stopping test needs the residual on the host).  `info` may be
 * NULL.  Returns SF_ERR_NONFINITE if the residual becomes NaN/Inf. */
int sf_solve_stokes(sf_ctx* ctx, double* P, double* Vx_pad, double* Vy_pad,
                    const double* rho_vy, const double* mu_b, const double* mu_p,
                    double* txx, double* tyy, double* txy, double* divV, double* dtPt,
                    double* Rx, double* Ry, double* dVxdt, double* dVydt, double* dtVx,
                    double* dtVy, double* Vx_s, double* Vy_s, double g_y, double dx, double dy,
                    int64_t Nx, int64_t Ny, double dt, double maxdisp,
                    int use_free_surface_stabilization, double eps, int print_info,
                    int64_t iter_max, void* stream, sf_solve_info* info);

/* Scale for a relative stopping test: mean(|g_y * rho_vy|) over the interior
 * region of Ry (rho_vy[2:Nx, 2:Ny-1]), i.e. the residual norm of V = P = 0.
 * A relative tolerance rtol is the absolute eps = rtol * scale.  (No reference
 * counterpart: the reference only has the absolute eps.) */
int sf_stokes_residual_scale(sf_ctx* ctx, const double* rho_vy, int64_t Nx, int64_t Ny,
                             double g_y, void* stream, double* scale);

/* ---------------------------------------------------------------------- */
/* domain decomposition: one solve over a dims_x x dims_y grid of ranks     */
/* ---------------------------------------------------------------------- */
/* One rank of a decomposed solve: its context (whose device and work
 * stream run the rank) and its local arrays, each as in sf_solve_stokes for
 * the local grid of Nx x Ny points, which overlaps its neighbours by 2
 * points as ImplicitGlobalGrid's (init_global_grid, overlaps 2). */
typedef struct {
    sf_ctx* ctx;
    double* P;                 /* (Nx-1, Ny-1)  in/out */
    double* Vx_pad;            /* (Nx+2, Ny+1)  out    */
    double* Vy_pad;            /* (Nx+1, Ny+2)  out    */
    const double* rho_vy;      /* (Nx+1, Ny)           */
    const double* mu_b;        /* (Nx,   Ny)           */
    const double* mu_p;        /* (Nx-1, Ny-1)         */
    double* dVxdt;             /* (Nx-2, Ny-1)  in/out */
    double* dVydt;             /* (Nx-1, Ny-2)  in/out */
    double* Vx_s;              /* (Nx,   Ny+1)  in/out */
    double* Vy_s;              /* (Nx+1, Ny)    in/out */
    int32_t coord_x, coord_y;  /* the rank's position; global point = coord * (N - 2) + local point */
} sf_domain;

/* Replaces solveStokes! run on dims_x * dims_y MPI ranks
 * (StokesSolver_multixpu.jl:14-96 with update_halo! at :57 and :93, the
 * Allreduce of compute_err :103-109 and compute_dt :118-121), driven from
 * one host thread over the ranks' devices (one GPU per rank, or several
 * ranks on one GPU).  The global grid is nx_g = dims_x (Nx-2) + 2 by
 * ny_g = dims_y (Ny-2) + 2 points, and the constants (damping, max_nxy,
 * ncheck, ndtupdate) use it.  Each iteration every rank runs the fused
 * kernel on its local grid (free-slip BCs on its local edges, as the
 * reference's BC kernels do), then the first / last planes of Vx_s and Vy_s
 * are copied from the neighbours (x then y, so corners follow).  The
 * iterates are bit-identical to a single-domain solve of the global grid.
 * err is the reference's multi-rank value: the mean over ranks of each rank's
 * local mean |Rx|, |Ry|, |divV| (overlap points counted by each rank).
 * info (may be NULL) receives the global results.  Synchronous. */
int sf_solve_stokes_decomposed(sf_domain* domains, int32_t dims_x, int32_t dims_y, int64_t Nx, int64_t Ny,
                               double g_y, double dx, double dy, double dt, double maxdisp,
                               int use_free_surface_stabilization, double eps, int64_t iter_max,
                               sf_solve_info* info);

/* One rank's array for sf_sum_overlapping_values: nx x ny entries, column-major, on the context's device. */
typedef struct {
    sf_ctx* ctx;
    double* a;
    int32_t coord_x, coord_y;
} sf_rank_array;

/* Replaces sumOverlappingValues!(A, grid) (MarkerToGrid.jl:183-269): the
 * entries each rank shares with a neighbour (ox = 2 + nx - Nx planes in x,
 * oy = 2 + ny - Ny in y) become the sum of both ranks' values, x first and
 * then y (so corners collect all four), each as own + received.  Used by the
 * decomposed deposit on val_wt_sum and wt_sum.  Synchronous. */
int sf_sum_overlapping_values(sf_rank_array* ranks, int32_t dims_x, int32_t dims_y, int64_t Nx, int64_t Ny,
                              int64_t nx, int64_t ny);

/* safeDivision over a grid (MarkerToGrid.jl:164-172, launched on 1:nx x
 * 1:ny at :35): val_grid[i,j] = val_wt_sum[i,j] / wt_sum[i,j] where the
 * weight is not 0; elsewhere val_grid keeps its value and the node is counted
 * as empty (sf_warnings.empty_nodes).  The sums have leading dimension ld_sum
 * (the reference's interpolation arrays are (Nx+1, Ny) for every grid). */
int sf_safe_division(sf_ctx* ctx, double* val_grid, int64_t nx, int64_t ny, const double* val_wt_sum,
                     const double* wt_sum, int64_t ld_sum, void* stream);

/* One rank of a marker exchange: its markers before (x, y, rho, mu; n of
 * them), its output arrays (capacity entries each) and, on return, n_out. */
typedef struct {
    sf_ctx* ctx;
    const double* x;
    const double* y;
    const double* rho;
    const double* mu;
    int64_t n;
    double* x_out;
    double* y_out;
    double* rho_out;
    double* mu_out;
    int64_t capacity;
    int64_t n_out;             /* result: markers after the exchange */
    int32_t coord_x, coord_y;
} sf_marker_rank;

/* Replaces exchangeMarkers (MarkerExchange.jl:8-163) for all ranks of a
 * dims_x x dims_y grid, driven from one thread.  A marker within half a cell
 * (dx/2, dy/2) of an edge shared with a neighbour goes to that neighbour
 * (posToNeighbourIdx, :204-222, eight neighbours), its position shifted by
 * (lx - dx, ly - dy) per step; the output is the rank's kept markers in their
 * order, then the received ones by neighbour index 1..8 (:60-90, :150-157),
 * each in the sender's order.  The inputs are not modified.  If some rank's
 * capacity is too small, nothing is written, every n_out holds the size
 * needed and the call returns SF_ERR_TOO_LARGE.  Synchronous. */
int sf_exchange_markers(sf_marker_rank* ranks, int32_t dims_x, int32_t dims_y, double lx, double ly, double dx,
                        double dy);

/* ---------------------------------------------------------------------- */
/* mixed-precision and batched solves (no reference counterpart: the       */
/* reference has only the FP64 solveStokes!)                                */
/* ---------------------------------------------------------------------- */
/* One Stokes problem of a batch: the caller arrays of sf_solve_stokes
 * (state in/out, work arrays not needed) plus its scalars; the results are
 * written back into the struct. */
typedef struct {
    double* P;                 /* (Nx-1, Ny-1)  in/out */
    double* Vx_pad;            /* (Nx+2, Ny+1)  out    */
    double* Vy_pad;            /* (Nx+1, Ny+2)  out    */
    const double* rho_vy;      /* (Nx+1, Ny)           */
    const double* mu_b;        /* (Nx,   Ny)           */
    const double* mu_p;        /* (Nx-1, Ny-1)         */
    double* Vx_s;              /* (Nx,   Ny+1)  in/out */
    double* Vy_s;              /* (Nx+1, Ny)    in/out */
    int64_t Nx, Ny;
    double g_y, dx, dy;
    double dt;                 /* stabilisation dt the solve starts with (the previous timestep's) */
    double maxdisp;
    double eps;                /* absolute stopping tolerance, as solveStokes!'s eps          */
    double rel_tol;            /* if > 0: eps = rel_tol * mean|g_y rho_vy| (relative residual) */
    int32_t use_free_surface_stabilization;
    int32_t retried;           /* result: 1 if the solve restarted with dtau_local_max (retry_local_max) */
    /* results */
    double dt_out;             /* compute_dt of the final velocities */
    double err;                /* final FP64 residual norm           */
    double eps_used;
    int64_t inner_iters;       /* FP32 PT sweeps                     */
    int64_t outer_iters;       /* FP64 residual evaluations          */
    int32_t converged;
    int32_t status;            /* sf_status of this instance         */
    double batch_ms;           /* sf_solve_stokes_batch_mixed: device time of the whole batch;
                                  sf_engine: host time from submit to the step that finished it */
    double* dVxdt;             /* (Nx-2, Ny-1) in/out, or NULL: the damped rates the solve starts from and
                                  ends with, as solveStokes! keeps dVxdtau between calls (a timestep
                                  loop passes the previous solve's); NULL starts them at zero and
                                  returns nothing                                              */
    double* dVydt;             /* (Nx-1, Ny-2) in/out, or NULL: likewise dVydtau               */
} sf_batch_instance;

typedef struct {
    int64_t max_sweeps;        /* FP32 sweeps per instance at most (4,000,000)                         */
    int32_t fold_every;        /* FP32 sweeps between folds into the FP64 state at most, even (400)    */
    int32_t use_graphs;        /* replay the sweeps between folds from a captured CUDA graph (1)       */
    int32_t dtau_local_max;    /* 1: pseudo-time step of a velocity node from the largest viscosity of
                                  its stencil (both pressure cells, both shear nodes), which converges
                                  faster on soft inclusions; 0: the reference's average
                                  (StokesSolver_multixpu.jl:129-130).  The converged solution is the
                                  same either way.  Neither form converges on inclusions much stiffer
                                  than their matrix (100x diverges in FP64 too) (0)                   */
    int32_t retry_local_max;   /* 1: an instance whose residual turns non-finite restarts from its
                                  inputs with dtau_local_max = 1 (its sweeps keep counting against
                                  max_sweeps); it converges on mixed soft/stiff layouts where the
                                  reference's step diverges.  Instances that converge are unaffected (1) */
    int32_t tile_rows;         /* rows of the 32-column sweep tiles: 8, 16 or 32, or 0 to let the
                                  autotuner choose the rows and the schedule.  Each round's sweep set has
                                  a workload class (half-octave of the mean, octave of the total grid
                                  points).  The first round of a class the context has not seen begins
                                  with short timed pieces of every shape, schedule and launch mode (two
                                  each); the
                                  fastest per point is then used and recorded in the context, so later
                                  rounds and solves of that class take it at once.  Every shape and
                                  schedule computes the same bits, so the choice changes the speed
                                  only (0)                                                            */
    int32_t tile_schedule;     /* with tile_rows set: 1 strided (CTA b of G takes tiles b, b+G, ...),
                                  2 chunked (CTA b takes one contiguous run of tiles); 0 = 1.  With
                                  tile_rows 0 it must be 0 (0)                                        */
    int32_t overlap_launches;  /* with tile_rows set: 1 launches each sweep under programmatic dependent
                                  launch, so that it starts (and fences its first tensor maps) while the
                                  previous sweep drains; 0 serialises the launches.  With tile_rows 0
                                  the tuner chooses, and it must be 0 (0)                             */
    int32_t reserved;          /* 0 */
} sf_mixed_options;

/* sf_engine_stats.tune_state */
enum {
    SF_TUNE_FIXED = 0,         /* the shape was given by tile_rows                        */
    SF_TUNE_MEASURING = 1,     /* the tuner is still timing shapes                        */
    SF_TUNE_MEASURED = 2,      /* the tuner chose the fastest shape it timed              */
    SF_TUNE_CACHED = 3         /* the context held a measured shape for this workload     */
};

/* Solves n independent Stokes problems (each as in solveStokes!, with its own
 * grid size) to err <= eps by FP64 defect correction around FP32
 * pseudo-transient sweeps.  At most every fold_every sweeps the FP32
 * correction is added to the FP64 V and P and the FP64 residual of the sum is
 * evaluated: the constant term of the next sweeps.  The sweeps are the
 * reference's PT iteration (damping, pseudo-time steps, free-slip BCs) on the
 * correction; its damped rates carry over across folds, so in exact arithmetic
 * the sequence is the FP64 iteration itself.  The solve keeps the reference
 * loop's schedule (StokesSolver_multixpu.jl:43-77): the stabilisation dt is the
 * one passed in until iteration ndtupdate = 10 min(Nx, Ny) and is recomputed
 * (compute_dt) at every multiple of it; the residual check (compute_Residuals!
 * with dt_check, compute_err) runs at every multiple of ncheck = min(5 min(Nx,
 * Ny), 2000) on the same quantities as the reference's, and the solve stops at
 * the first check with err <= eps or after max_sweeps iterations -- so it stops
 * at the same iteration as sf_solve_stokes on the same inputs, apart from a
 * check whose err lies within FP32 rounding of eps.  One sweep of every
 * instance still iterating is a single kernel launch over a shared tile list.
 * opt may be NULL (defaults above).  Synchronises the stream.  The results are
 * FP32-accurate corrections of an FP64 solution, not bit-identical to
 * sf_solve_stokes. */
int sf_solve_stokes_batch_mixed(sf_ctx* ctx, sf_batch_instance* inst, int n, const sf_mixed_options* opt,
                                void* stream);

/* One problem through the batch path; info (may be NULL) receives the
 * per-instance results.  dVxdt (Nx-2, Ny-1) and dVydt (Nx-1, Ny-2) are the
 * damped rates, in/out as in solveStokes!; either may be NULL (start at zero,
 * nothing returned). */
int sf_solve_stokes_mixed(sf_ctx* ctx, double* P, double* Vx_pad, double* Vy_pad, const double* rho_vy,
                          const double* mu_b, const double* mu_p, double* Vx_s, double* Vy_s, double* dVxdt,
                          double* dVydt, double g_y,
                          double dx, double dy, int64_t Nx, int64_t Ny, double dt, double maxdisp,
                          int use_free_surface_stabilization, double eps, double rel_tol,
                          const sf_mixed_options* opt, void* stream, sf_batch_instance* info);

/* ---------------------------------------------------------------------- */
/* resident solve engine: continuous batching for a serving loop           */
/* ---------------------------------------------------------------------- */
/* The engine behind sf_solve_stokes_batch_mixed, kept alive between calls so
 * that instances can join and leave while others iterate.  It owns a device
 * arena of arena_bytes (the HBM budget of its solves) and a table of at most
 * max_instances instances.  Each sf_engine_step is one round: every admitted
 * instance folds its correction and gets its FP64 residual (and, where its
 * schedule has one, its dt update and residual check); the finished ones are
 * written back to their caller arrays and leave (arena space and table slot
 * free at once); the rest run up to fold_every FP32 sweeps, each up to its
 * next event (one launch per sweep over all of them, graph-replayed).  An instance's
 * arithmetic and stopping decisions depend on itself alone, so its results
 * are bit-identical whatever else is in the engine and whenever it joined. */
typedef struct sf_engine sf_engine;

typedef struct {
    int64_t arena_bytes;       /* budget                                        */
    int64_t arena_used;        /* bytes held by admitted instances              */
    int64_t arena_peak;
    int64_t submitted, finished, rounds;
    int64_t sweeps;            /* FP32 sweep launches (one covers all instances) */
    int32_t active;            /* admitted, not finished                         */
    int32_t pending_results;   /* finished, not yet reported by sf_engine_step   */
    int32_t tile_rows;         /* rows of the sweep tiles in use                 */
    int32_t tile_schedule;     /* 1 strided, 2 chunked                           */
    int32_t overlap_launches;  /* 1: sweeps launched overlapped                  */
    int32_t tune_state;        /* SF_TUNE_* for the current workload class       */
    int32_t tune_classes;      /* workload classes with a recorded choice in the context */
    int32_t reserved;
    int64_t tune_rounds;       /* rounds whose sweeps began with timed trial pieces */
    int64_t tune_hits;         /* workload-class changes answered from the context's record */
    double tune_ns[12];        /* the last completed measurement: ns per point-sweep of each candidate,
                                  (rows, schedule, launch) in the order 8 strided serialised, 8 strided
                                  overlapped, 8 chunked serialised, ..., 32 chunked overlapped (0: none) */
} sf_engine_stats;

/* Arena bytes one instance of Nx x Ny grid points holds while admitted. */
int sf_engine_instance_bytes(int64_t Nx, int64_t Ny, int64_t* bytes);

/* opt may be NULL (the defaults of sf_mixed_options).  The arena is
 * allocated here, once.  The engine uses ctx (its device, its record of the
 * tuner's choices) for its whole life: destroy the engine first. */
int sf_engine_create(sf_ctx* ctx, int64_t arena_bytes, int32_t max_instances, const sf_mixed_options* opt,
                     sf_engine** out);
/* Waits for the engine's work, then frees it.  Instances still admitted are
 * dropped (their caller arrays keep what they held). */
int sf_engine_destroy(sf_engine* e);

/* Admits one instance: its inputs are read after the work already queued on
 * `stream` (a stream dependency, no host wait).  *inst must stay valid until
 * sf_engine_step reports its ticket; the results are then in its arrays and
 * fields.  SF_ERR_BUSY: no room in the arena or the table right now (nothing
 * admitted); SF_ERR_TOO_LARGE: the instance can never fit this arena. */
int sf_engine_submit(sf_engine* e, sf_batch_instance* inst, void* stream, int64_t* ticket);

/* One round (see above).  Up to `cap` tickets of finished instances go to
 * finished[] (*n_finished of them; more stay pending for the next call);
 * `stream` is made to wait for their write-back, so work queued on it after
 * this call sees their results.  Returns once the round's sweeps are queued
 * (they run while the host goes on).  *n_active: instances still admitted
 * (either output pointer may be NULL).  After an error status other than
 * SF_ERR_BUSY, destroy the engine. */
int sf_engine_step(sf_engine* e, void* stream, int64_t* finished, int32_t cap, int32_t* n_finished,
                   int32_t* n_active);

int sf_engine_get_stats(sf_engine* e, sf_engine_stats* stats);

/* The stats of the engine that sf_solve_stokes_batch_mixed and
 * sf_solve_stokes_mixed keep in the context, after their last call
 * (SF_ERR_INVALID_ARG before the first). */
int sf_ctx_batch_stats(sf_ctx* ctx, sf_engine_stats* stats);

/* ---------------------------------------------------------------------- */
/* RK4 marker advection and rebinning                                        */
/* ---------------------------------------------------------------------- */
/* Replaces moveMarkersRK4!(x_m, y_m, Vx, Vy, x_vx_min, y_vx_min, x_vy_min,
 * y_vy_min, dt, lx, ly, dx, dy)  (scripts/MoveMarkers.jl:15-69): classical RK4
 * with the continuity-based velocity interpolation of interpolateV
 * (:76-174) on the padded Vx (vx_nx, vx_ny) and Vy (vy_nx, vy_ny), positions
 * clamped to [0,lx] x [0,ly].  Same operation order as the reference: the
 * result is bit-identical to it.  Failsafe index clamps are counted. */
int sf_move_markers_rk4(sf_ctx* ctx, double* x_m, double* y_m, int64_t nm,
                        const double* Vx, int64_t vx_nx, int64_t vx_ny,
                        const double* Vy, int64_t vy_nx, int64_t vy_ny,
                        double x_vx_min, double y_vx_min, double x_vy_min, double y_vy_min,
                        double dt, double lx, double ly, double dx, double dy, void* stream);

/* Marker->cell rebinning: a stable counting sort of the markers by the cell
 * topleftIndexRelDist (scripts/common.jl:22-33) gives them on a grid of nx x ny
 * nodes, cells keyed (ix, iy) in 0..nx x 0..ny -> key ix + iy*(nx+1).
 * counts[(nx+1)*(ny+1)] receives the markers per cell, offsets[(nx+1)*(ny+1)+1]
 * the exclusive prefix sum, perm[nm] the marker indices (0-based) in cell
 * order, ascending within a cell.  Markers outside every cell are left out of
 * perm (perm is then shorter: offsets[last] markers) and counted in
 * markers_outside.  counts / offsets / perm may each be NULL.  The reference
 * never reorders a rank's markers (exchangeMarkers, MarkerExchange.jl:8-163,
 * is the identity on one rank), so neither does this: x_m / y_m are not moved. */
int sf_rebin_markers(sf_ctx* ctx, const double* x_m, const double* y_m, int64_t nm,
                     double x_grid_min, double y_grid_min, double dx, double dy,
                     int64_t nx, int64_t ny, int32_t* counts, int32_t* offsets, int32_t* perm,
                     void* stream);

/* ---------------------------------------------------------------------- */
/* marker initialisation (scripts/common.jl:40-110, single rank)             */
/* ---------------------------------------------------------------------- */
/* Number of markers initializeMarkersCPU places on one rank. */
int sf_marker_count(int64_t marker_density, int64_t nx, int64_t ny, int64_t* nmx, int64_t* nmy);

/* initializeMarkersCPU (common.jl:40-90) on one rank: LinRange sub-grid
 * (x outer, y inner) plus jitter x += (u - 0.5)*jitter*dxm, u from the
 * counter-based generator sf_uniform(seed, 2m) / (seed, 2m+1).  jitter = 1 is
 * the reference's +-0.5 sub-spacing; jitter = 0 is RAND_MARKER_POS = false.
 * _host works on host memory, the other on device memory. */
int sf_init_markers_host(int64_t marker_density, double lx, double ly, double dx, double dy,
                         int64_t nx, int64_t ny, double jitter, uint64_t seed,
                         double* x_m_host, double* y_m_host);
int sf_init_markers(sf_ctx* ctx, int64_t marker_density, double lx, double ly, double dx, double dy,
                    int64_t nx, int64_t ny, double jitter, uint64_t seed,
                    double* x_m, double* y_m, void* stream);
double sf_uniform(uint64_t seed, uint64_t counter);

/* initializeMarkersCPU for the rank at (coord_x, coord_y) of a dims_x x
 * dims_y grid (common.jl:40-90 with its boundary flags): sides shared with a
 * neighbour leave the markers the neighbour places, so the ranks' markers tile
 * the global domain.  Counts, then positions in local coordinates; the
 * jitter as in sf_init_markers (its counter restarts on every rank).  With
 * jitter and an odd density the reference then exchanges the markers
 * (common.jl:94-96): call sf_exchange_markers. */
int sf_marker_count_rank(int64_t marker_density, int64_t nx, int64_t ny, int32_t coord_x, int32_t coord_y,
                         int32_t dims_x, int32_t dims_y, int64_t* nmx, int64_t* nmy);
int sf_init_markers_rank(sf_ctx* ctx, int64_t marker_density, double lx, double ly, double dx, double dy,
                         int64_t nx, int64_t ny, int32_t coord_x, int32_t coord_y, int32_t dims_x, int32_t dims_y,
                         double jitter, uint64_t seed, double* x_m, double* y_m, void* stream);

/* setInitialMarkerProperties! (common.jl:104-110) for the layered
 * air / plume / matrix model of StokesFlow2D_multixpu.jl:382-404:
 * y < air_height -> air, else (x-px)^2+(y-py)^2 < r^2 -> plume, else matrix. */
typedef struct {
    double air_height;
    double plume_x, plume_y, plume_r;
    double rho_air, rho_matrix, rho_plume;
    double mu_air, mu_matrix, mu_plume;
} sf_plume_model;
int sf_set_marker_properties_host(const sf_plume_model* model, const double* x_m_host,
                                  const double* y_m_host, int64_t nm, double x0, double y0,
                                  double* rho_m_host, double* mu_m_host);
int sf_set_marker_properties(sf_ctx* ctx, const sf_plume_model* model, const double* x_m,
                             const double* y_m, int64_t nm, double x0, double y0,
                             double* rho_m, double* mu_m, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* STOKESFLOW_B200_H */
