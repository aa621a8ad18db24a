/*
 * sf_oracle.h -- CPU oracle for the StokesFlow.jl per-timestep hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA path is
 * compared against, and the timed CPU baseline of the benchmark.  It is never
 * linked into, loaded by, or called from the product library
 * (libstokesflow_b200.so) or its Python package.
 *
 * It restates, in plain C, the algorithm of the Julia reference
 * (dastrm/StokesFlow.jl), keeping every floating-point expression in the same
 * order as the Julia source so that, compiled without FMA contraction
 * (-ffp-contract=off), it rounds exactly as the reference does:
 *   scripts/common.jl:22-33            topleftIndexRelDist
 *   scripts/common.jl:40-110           initializeMarkersCPU / setInitialMarkerProperties!
 *   scripts/MarkerToGrid.jl:18-172     bilinearMarkerToGrid!, singleCoreInterpolationCPU!, safeDivision
 *   scripts/StokesSolver_multixpu.jl   solveStokes! and its kernels
 *   scripts/MoveMarkers.jl:15-187      moveMarkersRK4!, interpolateV, bilinearInterp
 *
 * Array convention: Julia arrays are column-major Float64; an (nx, ny) array
 * A is a flat double buffer with A[ix, iy] (1-based) at A[(ix-1) + (iy-1)*nx].
 * Integer indices inside the functions are 1-based like the reference.
 */
#ifndef SF_ORACLE_H
#define SF_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* common.jl:22-33 */
void orc_topleft_index_rel_dist(double x_grid_min, double y_grid_min, double x, double y,
                                double dx, double dy, int64_t* ix, int64_t* iy,
                                double* dxij, double* dyij);

/* Counter-based uniform [0,1) generator used for every seeded input
 * (SplitMix64 finaliser of seed*2^32 + stream + counter); shared with the
 * product so both sides see the same inputs. */
double orc_uniform(uint64_t seed, uint64_t counter);

/* common.jl:40-83 on a single rank (coords = 0, dims = 1): number of markers
 * in x / y for a given marker_density. */
void orc_marker_counts(int64_t marker_density, int64_t nx, int64_t ny, int64_t* nmx, int64_t* nmy);

/* common.jl:40-90 on a single rank: regular marker layout (LinRange, x outer,
 * y inner) plus optional jitter x += (u-0.5)*jitter*dxm (reference: jitter=1,
 * i.e. +-0.5 sub-spacing, drawn from Julia's RNG; here from orc_uniform). */
void orc_init_markers(int64_t marker_density, double lx, double ly, double dx, double dy,
                      int64_t nx, int64_t ny, double jitter, uint64_t seed,
                      double* x_m, double* y_m);

/* common.jl:40-90 for the rank at (cx, cy) of a dimx x dimy grid: the
 * boundary flags (:45-48) move the limits inward by half a cell plus half a
 * marker spacing on every side that faces a neighbour (:50-60) and drop
 * floor(md/2) / ceil(md/2) marker columns there (:62-66).  lx, ly, nx, ny are
 * the rank's local sizes.  The exchange that the reference runs after jitter
 * with an odd density (:95-97) is not part of this function. */
void orc_marker_counts_rank(int64_t marker_density, int64_t nx, int64_t ny, int cx, int cy, int dimx, int dimy,
                            int64_t* nmx, int64_t* nmy);
void orc_init_markers_rank(int64_t marker_density, double lx, double ly, double dx, double dy, int64_t nx,
                           int64_t ny, int cx, int cy, int dimx, int dimy, double jitter, uint64_t seed,
                           double* x_m, double* y_m);

/* Material model used by the tests and the benchmark: a layered 'sticky air'
 * + circular plume + matrix model (StokesFlow2D_multixpu.jl:382-404 and the
 * test_StokesFlow2D.jl:208-230 variant).  kind 0 = density, 1 = viscosity. */
typedef struct {
    double air_height;
    double plume_x, plume_y, plume_r;
    double rho_air, rho_matrix, rho_plume;
    double mu_air, mu_matrix, mu_plume;
} orc_plume_model;
void orc_set_marker_properties(const orc_plume_model* m, const double* x_m, const double* y_m,
                               int64_t nm, double x0, double y0, double* rho_m, double* mu_m);

/* MarkerToGrid.jl:18-38 + :110-155 + :164-172 (single rank: the overlap sums
 * are the identity).  val_grid is (nx, ny).  val_wt_sum / wt_sum are the
 * caller's work arrays of n_sum elements with leading dimension ld_sum
 * (reference: size max(size(rho_vy), size(mu_b), size(mu_p))); they are
 * zeroed and receive the weight sums.  Counts of skipped (erroneous) markers
 * and of empty nodes (kept at their previous value) are returned. */
void orc_bilinear_marker_to_grid(double x_grid_min, double y_grid_min, double* val_grid,
                                 int64_t nx, int64_t ny, const double* x_m, const double* y_m,
                                 const double* val_m, int64_t nm, double dx, double dy,
                                 double* val_wt_sum, double* wt_sum, int64_t ld_sum, int64_t n_sum,
                                 int64_t* n_bad_markers, int64_t* n_empty_nodes);

/* StokesSolver_multixpu.jl:14-96.  Array sizes as in the reference driver
 * (StokesFlow2D_multixpu.jl:89-109):
 *   P (Nx-1,Ny-1)  Vx_pad (Nx+2,Ny+1)  Vy_pad (Nx+1,Ny+2)  rho_vy (Nx+1,Ny)
 *   mu_b (Nx,Ny)   mu_p (Nx-1,Ny-1)    txx,tyy,divV,dtPt (Nx-1,Ny-1)  txy (Nx,Ny)
 *   Rx,dVxdt,dtVx (Nx-2,Ny-1)  Ry,dVydt,dtVy (Nx-1,Ny-2)  Vx_s (Nx,Ny+1)  Vy_s (Nx+1,Ny)
 * The loop stops when err <= eps (checked every ncheck iterations) or after
 * iter_max iterations.  Returns the new dt (compute_dt of the final V).
 * nthreads > 1 runs the stencil loops with OpenMP (the reference's
 * ParallelStencil Threads backend); results do not depend on it except for the
 * summation order inside err. */
typedef struct {
    double dt_out;      /* compute_dt(Vx_s, Vy_s) after the solve            */
    double err;         /* last err computed (2*eps if no check happened)    */
    int64_t iters;      /* niter                                             */
    int64_t n_checks;   /* number of residual checks                         */
    double runtime_s;   /* wall time of iterations >= 11 (reference :38-46)   */
} orc_solve_result;

void orc_solve_stokes(double* P, double* Vx_pad, double* Vy_pad, const double* rho_vy,
                      const double* mu_b, const double* mu_p, double* txx, double* tyy,
                      double* txy, double* divV, double* dtPt, double* Rx, double* Ry,
                      double* dVxdt, double* dVydt, double* dtVx, double* dtVy, double* Vx_s,
                      double* Vy_s, double g_y, double dx, double dy, int64_t Nx, int64_t Ny,
                      double dt, double maxdisp, int use_stab, double eps, int64_t iter_max,
                      int nthreads, orc_solve_result* res);

/* StokesSolver_multixpu.jl:118-121 */
double orc_compute_dt(const double* Vx, int64_t nvx, const double* Vy, int64_t nvy,
                      double maxdisp, double dx, double dy);

/* MoveMarkers.jl:76-174 (returns vx, vy; n_fail counts failsafe clamps) */
void orc_interpolate_v(double x, double y, const double* Vx, int64_t vx_nx, int64_t vx_ny,
                       const double* Vy, int64_t vy_nx, int64_t vy_ny, double x_vx_min,
                       double y_vx_min, double x_vy_min, double y_vy_min, double dx, double dy,
                       double* vx, double* vy, int64_t* n_fail);

/* MoveMarkers.jl:15-69 */
void orc_move_markers_rk4(double* x_m, double* y_m, int64_t nm, const double* Vx, int64_t vx_nx,
                          int64_t vx_ny, const double* Vy, int64_t vy_nx, int64_t vy_ny,
                          double x_vx_min, double y_vx_min, double x_vy_min, double y_vy_min,
                          double dt, double lx, double ly, double dx, double dy, int nthreads,
                          int64_t* n_fail);

/* Marker-to-cell rebinning: cell of each marker in the basic-node grid
 * (topleftIndexRelDist with origin (0,0), cells (nx-1) x (ny-1)), and the
 * number of markers per cell.  Returns the number of markers outside every
 * cell.  Cell key = (ix-1) + (iy-1)*(nx-1). */
int64_t orc_cell_counts(const double* x_m, const double* y_m, int64_t nm, double x_grid_min,
                        double y_grid_min, double dx, double dy, int64_t nx, int64_t ny,
                        int32_t* counts);

#ifdef __cplusplus
}
#endif
#endif
