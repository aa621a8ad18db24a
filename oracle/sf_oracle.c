/*
 * sf_oracle.c -- CPU oracle for the StokesFlow.jl per-timestep hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path and the timed CPU
 * baseline.  The product library never links or calls this file.
 *
 * Every function restates the Julia reference (dastrm/StokesFlow.jl) with the
 * same floating-point expression trees.  Julia evaluates a*b+c as a separate
 * multiply and add, chains of + and * left to right, and x^2 as x*x; this file
 * is compiled with -ffp-contract=off so gcc keeps exactly those roundings.
 * Indices are 1-based like the reference; arrays are column-major.
 */
#include "sf_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* column-major 1-based element access, leading dimension ld */
#define A2(a, ld, i, j) ((a)[((i) - 1) + ((j) - 1) * (int64_t)(ld)])

static double wall_s(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

/* ------------------------------------------------------------------------ */
/* scripts/common.jl:22-33  topleftIndexRelDist                              */
/* ------------------------------------------------------------------------ */
void orc_topleft_index_rel_dist(double x_grid_min, double y_grid_min, double x, double y,
                                double dx, double dy, int64_t* ix, int64_t* iy,
                                double* dxij, double* dyij) {
    /* ix = floor(Int, (x - x_grid_min) / dx) + 1 */
    int64_t i = (int64_t)floor((x - x_grid_min) / dx) + 1;
    int64_t j = (int64_t)floor((y - y_grid_min) / dy) + 1;
    /* x_ix = x_grid_min + (ix - 1) * dx */
    double x_ix = x_grid_min + (double)(i - 1) * dx;
    double y_iy = y_grid_min + (double)(j - 1) * dy;
    *ix = i;
    *iy = j;
    *dxij = (x - x_ix) / dx;
    *dyij = (y - y_iy) / dy;
}

/* ------------------------------------------------------------------------ */
/* seeded inputs                                                              */
/* ------------------------------------------------------------------------ */
static uint64_t splitmix64_mix(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

double orc_uniform(uint64_t seed, uint64_t counter) {
    uint64_t z = splitmix64_mix(splitmix64_mix(seed) ^ (counter * 0xD1B54A32D192ED03ull));
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

/* ------------------------------------------------------------------------ */
/* scripts/common.jl:40-90  initializeMarkersCPU (single rank)               */
/* ------------------------------------------------------------------------ */
void orc_marker_counts(int64_t marker_density, int64_t nx, int64_t ny, int64_t* nmx, int64_t* nmy) {
    /* single rank: xloBNDRY = xhiBNDRY = yloBNDRY = yhiBNDRY = true (common.jl:54-57),
       so Nmx = marker_density * (Nx - 1) (common.jl:73-74) */
    *nmx = marker_density * (nx - 1);
    *nmy = marker_density * (ny - 1);
}

/* Julia LinRange(a, b, n)[k] = lerpi(k-1, n-1, a, b) = (1 - t)*a + t*b, t = (k-1)/(n-1): two products and a
 * sum, each rounded.  That is the form the reference's golden values fit: the fma form of lerpi,
 * fma(t, b, fma(-t, a, a)), differs in the last bit and puts a marker of the 5-timestep golden case
 * (test/test_StokesFlow2D.jl) on the other side of the plume boundary */
static double linrange_at(double a, double b, int64_t n, int64_t k) {
    if (n == 1) return a;
    double t = (double)(k - 1) / (double)(n - 1);
    return (1.0 - t) * a + t * b;
}

/* common.jl:43-67 for the rank at (cx, cy) of a dimx x dimy grid: limits and counts */
static void rank_layout(int64_t md, double lx, double ly, double dx, double dy, int64_t nx, int64_t ny, int cx,
                        int cy, int dimx, int dimy, double* xlimlo, double* xlimhi, double* ylimlo, double* ylimhi,
                        int64_t* nmx, int64_t* nmy) {
    double dxm = dx / (double)md, dym = dy / (double)md;
    int xlo = cx == 0, xhi = cx == dimx - 1, ylo = cy == 0, yhi = cy == dimy - 1;
    double x_less_hi = md % 2 == 0 ? dxm / 2 : dxm, y_less_hi = md % 2 == 0 ? dym / 2 : dym;
    double x_less_lo = md % 2 == 0 ? dxm / 2 : 0.0, y_less_lo = md % 2 == 0 ? dym / 2 : 0.0;
    *xlimlo = xlo ? dxm / 2 : dx / 2 + x_less_lo;
    *xlimhi = xhi ? lx - dxm / 2 : lx - dx / 2 - x_less_hi;
    *ylimlo = ylo ? dym / 2 : dy / 2 + y_less_lo;
    *ylimhi = yhi ? ly - dym / 2 : ly - dy / 2 - y_less_hi;
    int64_t lo_less = md / 2, hi_less = (md + 1) / 2;   /* floor(md/2), ceil(md/2) */
    *nmx = md * (nx - 1) - (xlo ? 0 : lo_less) - (xhi ? 0 : hi_less);
    *nmy = md * (ny - 1) - (ylo ? 0 : lo_less) - (yhi ? 0 : hi_less);
}

void orc_marker_counts_rank(int64_t marker_density, int64_t nx, int64_t ny, int cx, int cy, int dimx, int dimy,
                            int64_t* nmx, int64_t* nmy) {
    double a, b, c, d;
    rank_layout(marker_density, 1.0, 1.0, 1.0, 1.0, nx, ny, cx, cy, dimx, dimy, &a, &b, &c, &d, nmx, nmy);
}

void orc_init_markers_rank(int64_t marker_density, double lx, double ly, double dx, double dy, int64_t nx,
                           int64_t ny, int cx, int cy, int dimx, int dimy, double jitter, uint64_t seed,
                           double* x_m, double* y_m) {
    double dxm = dx / (double)marker_density;
    double dym = dy / (double)marker_density;
    double xlimlo, xlimhi, ylimlo, ylimhi;
    int64_t nmx, nmy;
    rank_layout(marker_density, lx, ly, dx, dy, nx, ny, cx, cy, dimx, dimy, &xlimlo, &xlimhi, &ylimlo, &ylimhi,
                &nmx, &nmy);
    int64_t m = 0;
    for (int64_t ix = 1; ix <= nmx; ++ix) {       /* x outer, y inner (common.jl:85-91) */
        double xc = linrange_at(xlimlo, xlimhi, nmx, ix);
        for (int64_t iy = 1; iy <= nmy; ++iy) {
            x_m[m] = xc;
            y_m[m] = linrange_at(ylimlo, ylimhi, nmy, iy);
            ++m;
        }
    }
    if (jitter != 0.0) {
        /* common.jl:94-96: x_m .+= (rand(Nm) .- 0.5) .* dxm; here scaled by jitter */
        int64_t nm = nmx * nmy;
        for (int64_t k = 0; k < nm; ++k) {
            double ux = orc_uniform(seed, (uint64_t)(2 * k));
            double uy = orc_uniform(seed, (uint64_t)(2 * k + 1));
            x_m[k] = x_m[k] + (ux - 0.5) * jitter * dxm;
            y_m[k] = y_m[k] + (uy - 0.5) * jitter * dym;
        }
    }
}

void orc_init_markers(int64_t marker_density, double lx, double ly, double dx, double dy,
                      int64_t nx, int64_t ny, double jitter, uint64_t seed,
                      double* x_m, double* y_m) {
    /* single rank: every boundary flag is true (common.jl:45-48 with dims = (1, 1)) */
    orc_init_markers_rank(marker_density, lx, ly, dx, dy, nx, ny, 0, 0, 1, 1, jitter, seed, x_m, y_m);
}

/* StokesFlow2D_multixpu.jl:387-404 (density / viscosity closures) */
static double plume_eval(const orc_plume_model* m, double x, double y, double a, double mat, double pl) {
    if (y < m->air_height) return a;
    double ddx = x - m->plume_x, ddy = y - m->plume_y;
    if (ddx * ddx + ddy * ddy < m->plume_r * m->plume_r) return pl;
    return mat;
}

/* common.jl:104-110 setInitialMarkerProperties! */
void orc_set_marker_properties(const orc_plume_model* m, const double* x_m, const double* y_m,
                               int64_t nm, double x0, double y0, double* rho_m, double* mu_m) {
    for (int64_t k = 0; k < nm; ++k) {
        double x = x0 + x_m[k], y = y0 + y_m[k];
        rho_m[k] = plume_eval(m, x, y, m->rho_air, m->rho_matrix, m->rho_plume);
        mu_m[k] = plume_eval(m, x, y, m->mu_air, m->mu_matrix, m->mu_plume);
    }
}

/* ------------------------------------------------------------------------ */
/* scripts/MarkerToGrid.jl                                                   */
/* ------------------------------------------------------------------------ */
void orc_bilinear_marker_to_grid(double x_grid_min, double y_grid_min, double* val_grid,
                                 int64_t Nx, int64_t Ny, const double* x_m, const double* y_m,
                                 const double* val_m, int64_t Nm, double dx, double dy,
                                 double* val_wt_sum, double* wt_sum, int64_t ld, int64_t n_sum,
                                 int64_t* n_bad_markers, int64_t* n_empty_nodes) {
    int64_t nbad = 0, nempty = 0;
    /* :24-25 */
    memset(val_wt_sum, 0, sizeof(double) * (size_t)n_sum);
    memset(wt_sum, 0, sizeof(double) * (size_t)n_sum);
    /* :110-155 singleCoreInterpolationCPU!, serial in marker order */
    for (int64_t m = 0; m < Nm; ++m) {
        double xm = x_m[m], ym = y_m[m], val = val_m[m];
        int64_t ix, iy;
        double dxmij, dymij;
        orc_topleft_index_rel_dist(x_grid_min, y_grid_min, xm, ym, dx, dy, &ix, &iy, &dxmij, &dymij);
        if (!(ix >= 0 && ix <= Nx && iy >= 0 && iy <= Ny)) {
            ++nbad; /* "ATTENTION: erroneous marker position" */
            continue;
        }
        if (iy > 0) {
            if (ix > 0) {
                double w = (1.0 - dxmij) * (1.0 - dymij);
                A2(wt_sum, ld, ix, iy) += w;
                A2(val_wt_sum, ld, ix, iy) += w * val;
            }
            if (ix < Nx) {
                double w = dxmij * (1.0 - dymij);
                A2(wt_sum, ld, ix + 1, iy) += w;
                A2(val_wt_sum, ld, ix + 1, iy) += w * val;
            }
        }
        if (iy < Ny) {
            if (ix > 0) {
                double w = (1.0 - dxmij) * dymij;
                A2(wt_sum, ld, ix, iy + 1) += w;
                A2(val_wt_sum, ld, ix, iy + 1) += w * val;
            }
            if (ix < Nx) {
                double w = dxmij * dymij;
                A2(wt_sum, ld, ix + 1, iy + 1) += w;
                A2(val_wt_sum, ld, ix + 1, iy + 1) += w * val;
            }
        }
    }
    /* :164-172 safeDivision over (1:Nx, 1:Ny) */
    for (int64_t iy = 1; iy <= Ny; ++iy)
        for (int64_t ix = 1; ix <= Nx; ++ix) {
            double den = A2(wt_sum, ld, ix, iy);
            if (den != 0.0)
                A2(val_grid, Nx, ix, iy) = A2(val_wt_sum, ld, ix, iy) / den;
            else
                ++nempty; /* value kept, "PROBLEM: no markers close enough" */
        }
    if (n_bad_markers) *n_bad_markers = nbad;
    if (n_empty_nodes) *n_empty_nodes = nempty;
}

int64_t orc_cell_counts(const double* x_m, const double* y_m, int64_t nm, double x_grid_min,
                        double y_grid_min, double dx, double dy, int64_t nx, int64_t ny,
                        int32_t* counts) {
    int64_t nout = 0;
    memset(counts, 0, sizeof(int32_t) * (size_t)((nx + 1) * (ny + 1)));
    for (int64_t m = 0; m < nm; ++m) {
        int64_t ix, iy;
        double a, b;
        orc_topleft_index_rel_dist(x_grid_min, y_grid_min, x_m[m], y_m[m], dx, dy, &ix, &iy, &a, &b);
        if (ix < 0 || ix > nx || iy < 0 || iy > ny) {
            ++nout;
            continue;
        }
        counts[ix + iy * (nx + 1)] += 1;
    }
    return nout;
}

/* ------------------------------------------------------------------------ */
/* scripts/StokesSolver_multixpu.jl                                          */
/* ------------------------------------------------------------------------ */
typedef struct {
    int64_t Nx, Ny;
    double _dx, _dy, g_y;
    int nthreads;
} pt_dims;

/* :128-133 compute_timesteps! (@av_xa(A) = (A[ix,iy] + A[ix+1,iy])*0.5) */
static void compute_timesteps(const pt_dims* d, double* dtVx, double* dtVy, double* dtP,
                              const double* mu_p, double Vsc, double Ptsc, double min_dxy2,
                              double max_nxy) {
    int64_t Nx = d->Nx, Ny = d->Ny;
    int64_t lp = Nx - 1, lx = Nx - 2, ly = Nx - 1;
#pragma omp parallel for num_threads(d->nthreads) schedule(static) if (d->nthreads > 1)
    for (int64_t iy = 1; iy <= Ny - 1; ++iy)
        for (int64_t ix = 1; ix <= Nx - 1; ++ix) {
            if (ix <= Nx - 2 && iy <= Ny - 1)
                A2(dtVx, lx, ix, iy) = Vsc * min_dxy2 / ((A2(mu_p, lp, ix, iy) + A2(mu_p, lp, ix + 1, iy)) * 0.5) / 4.1;
            if (ix <= Nx - 1 && iy <= Ny - 2)
                A2(dtVy, ly, ix, iy) = Vsc * min_dxy2 / ((A2(mu_p, lp, ix, iy) + A2(mu_p, lp, ix, iy + 1)) * 0.5) / 4.1;
            A2(dtP, lp, ix, iy) = Ptsc * 4.1 * A2(mu_p, lp, ix, iy) / max_nxy;
        }
}

/* :140-169 compute_P_tau! ; Vx = Vx_s (Nx, Ny+1), Vy = Vy_s (Nx+1, Ny) */
static void compute_P_tau(const pt_dims* d, double* divV, double* P, const double* Vx,
                          const double* Vy, const double* dtP, double* txx, double* tyy,
                          double* txy, const double* mu_p, const double* mu_b) {
    int64_t Nx = d->Nx, Ny = d->Ny;
    int64_t lp = Nx - 1, lvx = Nx, lvy = Nx + 1, lb = Nx;
    double _dx = d->_dx, _dy = d->_dy;
    int64_t xmax = Nx, ymax = Ny; /* size(txy) */
#pragma omp parallel for num_threads(d->nthreads) schedule(static) if (d->nthreads > 1)
    for (int64_t iy = 1; iy <= ymax; ++iy)
        for (int64_t ix = 1; ix <= xmax; ++ix) {
            double vx0 = A2(Vx, lvx, ix, iy);
            double vx1 = A2(Vx, lvx, ix, iy + 1);
            double vy0 = A2(Vy, lvy, ix, iy);
            double vy1 = A2(Vy, lvy, ix + 1, iy);
            if (ix < xmax && iy < ymax) {
                double vx2 = A2(Vx, lvx, ix + 1, iy + 1);
                double vy2 = A2(Vy, lvy, ix + 1, iy + 1);
                double dVx_dx = (vx2 - vx1) * _dx;
                double dVy_dy = (vy2 - vy1) * _dy;
                double div_V = dVx_dx + dVy_dy;
                A2(divV, lp, ix, iy) = div_V;
                A2(P, lp, ix, iy) = A2(P, lp, ix, iy) - A2(dtP, lp, ix, iy) * div_V;
                double mu = A2(mu_p, lp, ix, iy);
                A2(txx, lp, ix, iy) = 2.0 * mu * (dVx_dx - 1.0 / 3.0 * div_V);
                A2(tyy, lp, ix, iy) = 2.0 * mu * (dVy_dy - 1.0 / 3.0 * div_V);
            }
            double dVx_dy = (vx1 - vx0) * _dy;
            double dVy_dx = (vy1 - vy0) * _dx;
            A2(txy, lb, ix, iy) = 2.0 * A2(mu_b, lb, ix, iy) * 0.5 * (dVx_dy + dVy_dx);
        }
}

/* :176-182 compute_ResX */
static inline double res_x(const pt_dims* d, int64_t ix, int64_t iy, const double* txx,
                           const double* txy, const double* P) {
    int64_t lp = d->Nx - 1, lb = d->Nx;
    return ((A2(txx, lp, ix + 1, iy) - A2(txx, lp, ix, iy)) * d->_dx
            + (A2(txy, lb, ix + 1, iy + 1) - A2(txy, lb, ix + 1, iy)) * d->_dy
            - (A2(P, lp, ix + 1, iy) - A2(P, lp, ix, iy)) * d->_dx);
}

/* :189-202 compute_ResY */
static inline double res_y(const pt_dims* d, int64_t ix, int64_t iy, const double* tyy,
                           const double* txy, const double* P, const double* rho,
                           const double* Vx, const double* Vy, double dt) {
    int64_t Nx = d->Nx;
    int64_t lp = Nx - 1, lb = Nx, lvx = Nx, lvy = Nx + 1, lr = Nx + 1;
    double av_inn_y_Vx = 0.25 * (A2(Vx, lvx, ix, iy + 1) + A2(Vx, lvx, ix + 1, iy + 1)
                                 + A2(Vx, lvx, ix, iy + 2) + A2(Vx, lvx, ix + 1, iy + 2));
    double d_xi_2_rho = A2(rho, lr, ix + 2, iy + 1) - A2(rho, lr, ix, iy + 1);
    double d_yi_2_rho = A2(rho, lr, ix + 1, iy + 2) - A2(rho, lr, ix + 1, iy);
    return ((A2(tyy, lp, ix, iy + 1) - A2(tyy, lp, ix, iy)) * d->_dy
            + (A2(txy, lb, ix + 1, iy + 1) - A2(txy, lb, ix, iy + 1)) * d->_dx
            - (A2(P, lp, ix, iy + 1) - A2(P, lp, ix, iy)) * d->_dy
            + d->g_y * (A2(rho, lr, ix + 1, iy + 1)
                        - dt * (av_inn_y_Vx * d_xi_2_rho * 0.5 * d->_dx
                                + A2(Vy, lvy, ix + 1, iy + 1) * d_yi_2_rho * 0.5 * d->_dy)));
}

/* :209-219 compute_dV! */
static void compute_dV(const pt_dims* d, double* dVxdt, double* dVydt, const double* P,
                       const double* rho, const double* txx, const double* tyy, const double* txy,
                       const double* Vx, const double* Vy, double dampX, double dampY, double dt) {
    int64_t Nx = d->Nx, Ny = d->Ny;
    int64_t lx = Nx - 2, ly = Nx - 1;
#pragma omp parallel for num_threads(d->nthreads) schedule(static) if (d->nthreads > 1)
    for (int64_t iy = 1; iy <= Ny - 1; ++iy)
        for (int64_t ix = 1; ix <= Nx - 1; ++ix) {
            if (ix <= Nx - 2 && iy <= Ny - 1) {
                double r = res_x(d, ix, iy, txx, txy, P);
                A2(dVxdt, lx, ix, iy) = dampX * A2(dVxdt, lx, ix, iy) + r;
            }
            if (ix <= Nx - 1 && iy <= Ny - 2) {
                double r = res_y(d, ix, iy, tyy, txy, P, rho, Vx, Vy, dt);
                A2(dVydt, ly, ix, iy) = dampY * A2(dVydt, ly, ix, iy) + r;
            }
        }
}

/* :226-234 compute_V! followed by the free-slip BCs of :53-56 in order */
static void compute_V_bc(const pt_dims* d, double* Vx, double* Vy, const double* dVxdt,
                         const double* dVydt, const double* dtVx, const double* dtVy) {
    int64_t Nx = d->Nx, Ny = d->Ny;
    int64_t lx = Nx - 2, ly = Nx - 1, lvx = Nx, lvy = Nx + 1;
#pragma omp parallel for num_threads(d->nthreads) schedule(static) if (d->nthreads > 1)
    for (int64_t iy = 1; iy <= Ny - 1; ++iy)
        for (int64_t ix = 1; ix <= Nx - 1; ++ix) {
            if (ix <= Nx - 2 && iy <= Ny - 1)
                A2(Vx, lvx, ix + 1, iy + 1) = A2(Vx, lvx, ix + 1, iy + 1) + A2(dtVx, lx, ix, iy) * A2(dVxdt, lx, ix, iy);
            if (ix <= Nx - 1 && iy <= Ny - 2)
                A2(Vy, lvy, ix + 1, iy + 1) = A2(Vy, lvy, ix + 1, iy + 1) + A2(dtVy, ly, ix, iy) * A2(dVydt, ly, ix, iy);
        }
    /* :299-303 bc_y_noflux!(Vx_s) over ix = 1:size(Vx_s,1) */
    for (int64_t ix = 1; ix <= Nx; ++ix) {
        A2(Vx, lvx, ix, 1) = A2(Vx, lvx, ix, 2);
        A2(Vx, lvx, ix, Ny + 1) = A2(Vx, lvx, ix, Ny);
    }
    /* :256-260 bc_x_zero!(Vx_s) over iy = 1:size(Vx_s,2) */
    for (int64_t iy = 1; iy <= Ny + 1; ++iy) {
        A2(Vx, lvx, 1, iy) = 0.0;
        A2(Vx, lvx, Nx, iy) = 0.0;
    }
    /* :289-293 bc_y_zero!(Vy_s) over ix = 1:size(Vy_s,1) */
    for (int64_t ix = 1; ix <= Nx + 1; ++ix) {
        A2(Vy, lvy, ix, 1) = 0.0;
        A2(Vy, lvy, ix, Ny) = 0.0;
    }
    /* :267-271 bc_x_noflux!(Vy_s) over iy = 1:size(Vy_s,2) */
    for (int64_t iy = 1; iy <= Ny; ++iy) {
        A2(Vy, lvy, 1, iy) = A2(Vy, lvy, 2, iy);
        A2(Vy, lvy, Nx + 1, iy) = A2(Vy, lvy, Nx, iy);
    }
}

/* :241-249 compute_Residuals! */
static void compute_residuals(const pt_dims* d, double* Rx, double* Ry, const double* P,
                              const double* rho, const double* txx, const double* tyy,
                              const double* txy, const double* Vx, const double* Vy, double dt) {
    int64_t Nx = d->Nx, Ny = d->Ny;
    int64_t lx = Nx - 2, ly = Nx - 1;
#pragma omp parallel for num_threads(d->nthreads) schedule(static) if (d->nthreads > 1)
    for (int64_t iy = 1; iy <= Ny - 1; ++iy)
        for (int64_t ix = 1; ix <= Nx - 1; ++ix) {
            if (ix <= Nx - 2 && iy <= Ny - 1) A2(Rx, lx, ix, iy) = res_x(d, ix, iy, txx, txy, P);
            if (ix <= Nx - 1 && iy <= Ny - 2) A2(Ry, ly, ix, iy) = res_y(d, ix, iy, tyy, txy, P, rho, Vx, Vy, dt);
        }
}

static double mean_abs(const double* a, int64_t n) {
    double s = 0.0;
    for (int64_t k = 0; k < n; ++k) s += fabs(a[k]);
    return s / (double)n;
}

static double max_abs(const double* a, int64_t n) {
    double m = 0.0;
    for (int64_t k = 0; k < n; ++k) {
        double v = fabs(a[k]);
        if (v > m) m = v;
    }
    return m;
}

/* :118-121 compute_dt (single rank: Allreduce MIN is the identity) */
double orc_compute_dt(const double* Vx, int64_t nvx, const double* Vy, int64_t nvy,
                      double maxdisp, double dx, double dy) {
    double a = dx / max_abs(Vx, nvx), b = dy / max_abs(Vy, nvy);
    double min_l = (b < a) ? b : a; /* Julia min of two non-NaN doubles */
    if (a != a) min_l = a;
    if (b != b) min_l = b;
    return maxdisp * min_l;
}

/* :103-109 compute_err */
static double compute_err(const double* Rx, int64_t nrx, const double* Ry, int64_t nry,
                          const double* divV, int64_t ndv) {
    double a = mean_abs(Rx, nrx), b = mean_abs(Ry, nry), c = mean_abs(divV, ndv);
    double m = a;
    if (b > m) m = b;
    if (c > m) m = c;
    return m;
}

void orc_solve_stokes(double* P, double* Vx_pad, double* Vy_pad, const double* rho_vy,
                      const double* mu_b, const double* mu_p, double* txx, double* tyy,
                      double* txy, double* divV, double* dtPt, double* Rx, double* Ry,
                      double* dVxdt, double* dVydt, double* dtVx, double* dtVy, double* Vx_s,
                      double* Vy_s, double g_y, double dx, double dy, int64_t Nx, int64_t Ny,
                      double dt, double maxdisp, int use_stab, double eps, int64_t iter_max,
                      int nthreads, orc_solve_result* res) {
    pt_dims d = {Nx, Ny, 1.0 / dx, 1.0 / dy, g_y, nthreads < 1 ? 1 : nthreads};
    /* :17-27 */
    double Vdmp = 4.0, Vsc = 0.45, Ptsc = 1.0 / 2.0;
    double mdxy = dx < dy ? dx : dy;
    double min_dxy2 = mdxy * mdxy;
    double max_nxy = (double)(Nx > Ny ? Nx : Ny);
    double dampX = 1.0 - Vdmp / (double)Nx;
    double dampY = 1.0 - Vdmp / (double)Ny;
    if (!use_stab) dt = 0.0; /* :29-31 */
    compute_timesteps(&d, dtVx, dtVy, dtPt, mu_p, Vsc, Ptsc, min_dxy2, max_nxy);
    int64_t mnxy = Nx < Ny ? Nx : Ny;
    int64_t ncheck = 5 * mnxy < 2000 ? 5 * mnxy : 2000; /* :35 */
    int64_t ndtupdate = 10 * mnxy;                      /* :36 */
    int64_t nvx = Nx * (Ny + 1), nvy = (Nx + 1) * Ny;
    int64_t nrx = (Nx - 2) * (Ny - 1), nry = (Nx - 1) * (Ny - 2), np = (Nx - 1) * (Ny - 1);
    double t1 = 0.0;
    int64_t itert1 = 11;
    double err = 2.0 * eps;
    int64_t iter = 1, niter = 0, nchecks = 0;
    while (err > eps && iter <= iter_max) { /* :43 */
        if (iter == itert1) t1 = wall_s();
        compute_P_tau(&d, divV, P, Vx_s, Vy_s, dtPt, txx, tyy, txy, mu_p, mu_b);
        compute_dV(&d, dVxdt, dVydt, P, rho_vy, txx, tyy, txy, Vx_s, Vy_s, dampX, dampY, dt);
        compute_V_bc(&d, Vx_s, Vy_s, dVxdt, dVydt, dtVx, dtVy);
        if (use_stab && (iter % ndtupdate == 0)) dt = orc_compute_dt(Vx_s, nvx, Vy_s, nvy, maxdisp, dx, dy);
        if (iter % ncheck == 0) {
            double dt_check = use_stab ? orc_compute_dt(Vx_s, nvx, Vy_s, nvy, maxdisp, dx, dy) : 0.0;
            compute_residuals(&d, Rx, Ry, P, rho_vy, txx, tyy, txy, Vx_s, Vy_s, dt_check);
            err = compute_err(Rx, nrx, Ry, nry, divV, np);
            ++nchecks;
        }
        ++iter;
        ++niter;
    }
    double runtime = (niter >= itert1) ? wall_s() - t1 : 0.0;
    /* :89-93 padded velocities with mirror ghost layer */
    for (int64_t iy = 1; iy <= Ny + 1; ++iy)
        for (int64_t ix = 1; ix <= Nx; ++ix) A2(Vx_pad, Nx + 2, ix + 1, iy) = A2(Vx_s, Nx, ix, iy);
    for (int64_t iy = 1; iy <= Ny; ++iy)
        for (int64_t ix = 1; ix <= Nx + 1; ++ix) A2(Vy_pad, Nx + 1, ix, iy + 1) = A2(Vy_s, Nx + 1, ix, iy);
    for (int64_t iy = 1; iy <= Ny + 1; ++iy) { /* :278-282 bc_x_mirror!(Vx_pad) */
        A2(Vx_pad, Nx + 2, 1, iy) = -A2(Vx_pad, Nx + 2, 3, iy);
        A2(Vx_pad, Nx + 2, Nx + 2, iy) = -A2(Vx_pad, Nx + 2, Nx, iy);
    }
    for (int64_t ix = 1; ix <= Nx + 1; ++ix) { /* :309-313 bc_y_mirror!(Vy_pad) */
        A2(Vy_pad, Nx + 1, ix, 1) = -A2(Vy_pad, Nx + 1, ix, 3);
        A2(Vy_pad, Nx + 1, ix, Ny + 2) = -A2(Vy_pad, Nx + 1, ix, Ny);
    }
    if (res) {
        res->dt_out = orc_compute_dt(Vx_s, nvx, Vy_s, nvy, maxdisp, dx, dy); /* :95 */
        res->err = err;
        res->iters = niter;
        res->n_checks = nchecks;
        res->runtime_s = runtime;
    }
}

/* ------------------------------------------------------------------------ */
/* scripts/MoveMarkers.jl                                                    */
/* ------------------------------------------------------------------------ */
/* :181-187 bilinearInterp */
static inline double bilinear_interp(double v1, double v2, double v3, double v4, double dxij, double dyij) {
    double s1 = (1.0 - dxij) * (1.0 - dyij) * v1;
    double s2 = dxij * (1.0 - dyij) * v2;
    double s3 = (1.0 - dxij) * dyij * v3;
    double s4 = dxij * dyij * v4;
    return s1 + s2 + s3 + s4;
}

/* :76-174 interpolateV */
void orc_interpolate_v(double x, double y, const double* Vx, int64_t vx_nx, int64_t vx_ny,
                       const double* Vy, int64_t vy_nx, int64_t vy_ny, double x_vx_min,
                       double y_vx_min, double x_vy_min, double y_vy_min, double dx, double dy,
                       double* vx_out, double* vy_out, int64_t* n_fail) {
    int64_t ix, iy;
    double dxij, dyij;
    int64_t nf = 0;
    /* Vx */
    orc_topleft_index_rel_dist(x_vx_min, y_vx_min, x, y, dx, dy, &ix, &iy, &dxij, &dyij);
    if (ix < 2) { ++nf; ix = 2; dxij = 0.0; }
    if (iy < 1) { ++nf; iy = 1; dyij = 0.0; }
    if (ix >= vx_nx - 1) { ++nf; ix = vx_nx - 2; dxij = 1.0; }
    if (iy >= vx_ny) { ++nf; iy = vx_ny - 1; dyij = 1.0; }
    double v1 = A2(Vx, vx_nx, ix, iy);
    double v2 = A2(Vx, vx_nx, ix + 1, iy);
    double v3 = A2(Vx, vx_nx, ix, iy + 1);
    double v4 = A2(Vx, vx_nx, ix + 1, iy + 1);
    double vx = bilinear_interp(v1, v2, v3, v4, dxij, dyij);
    double correction;
    if (dxij >= 0.5) {
        double v5 = A2(Vx, vx_nx, ix + 2, iy);
        double v6 = A2(Vx, vx_nx, ix + 2, iy + 1);
        double h = dxij - 0.5;
        correction = 0.5 * (h * h) * ((1.0 - dyij) * (v1 - 2.0 * v2 + v5) + dyij * (v3 - 2.0 * v4 + v6));
    } else {
        double v5 = A2(Vx, vx_nx, ix - 1, iy);
        double v6 = A2(Vx, vx_nx, ix - 1, iy + 1);
        double h = dxij - 0.5;
        correction = 0.5 * (h * h) * ((1.0 - dyij) * (v5 - 2.0 * v1 + v2) + dyij * (v6 - 2.0 * v3 + v4));
    }
    vx = vx + correction;
    /* Vy */
    orc_topleft_index_rel_dist(x_vy_min, y_vy_min, x, y, dx, dy, &ix, &iy, &dxij, &dyij);
    if (ix < 1) { ++nf; ix = 1; dxij = 0.0; }
    if (iy < 2) { ++nf; iy = 2; dyij = 0.0; }
    if (ix >= vy_nx) { ++nf; ix = vy_nx - 1; dxij = 1.0; }
    if (iy >= vy_ny - 1) { ++nf; iy = vy_ny - 2; dyij = 1.0; }
    v1 = A2(Vy, vy_nx, ix, iy);
    v2 = A2(Vy, vy_nx, ix + 1, iy);
    v3 = A2(Vy, vy_nx, ix, iy + 1);
    v4 = A2(Vy, vy_nx, ix + 1, iy + 1);
    double vy = bilinear_interp(v1, v2, v3, v4, dxij, dyij);
    if (dyij >= 0.5) {
        double v5 = A2(Vy, vy_nx, ix, iy + 2);
        double v6 = A2(Vy, vy_nx, ix + 1, iy + 2);
        double h = dyij - 0.5;
        correction = 0.5 * (h * h) * ((1.0 - dxij) * (v1 - 2.0 * v3 + v5) + dxij * (v2 - 2.0 * v4 + v6));
    } else {
        double v5 = A2(Vy, vy_nx, ix, iy - 1);
        double v6 = A2(Vy, vy_nx, ix + 1, iy - 1);
        double h = dyij - 0.5;
        correction = 0.5 * (h * h) * ((1.0 - dxij) * (v5 - 2.0 * v1 + v3) + dxij * (v6 - 2.0 * v2 + v4));
    }
    vy = vy + correction;
    *vx_out = vx;
    *vy_out = vy;
    if (n_fail) *n_fail += nf;
}

/* Julia max(x, 0) / min(x, l) for Float64 (-0.0 < 0.0, NaN propagates) */
static inline double jl_max0(double x) {
    if (x != x) return x;
    return (x < 0.0 || (x == 0.0 && signbit(x))) ? 0.0 : x;
}
static inline double jl_min(double x, double l) {
    if (x != x) return x;
    return (l < x) ? l : x;
}

/* :15-69 moveMarkersRK4! / moveMarkersRK4_Kernel! */
void orc_move_markers_rk4(double* x_m, double* y_m, int64_t nm, const double* Vx, int64_t vx_nx,
                          int64_t vx_ny, const double* Vy, int64_t vy_nx, int64_t vy_ny,
                          double x_vx_min, double y_vx_min, double x_vy_min, double y_vy_min,
                          double dt, double lx, double ly, double dx, double dy, int nthreads,
                          int64_t* n_fail) {
    const double rk4_dt[4] = {0.0, 0.5 * dt, 0.5 * dt, dt};
    const double rk4_wt[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};
    int64_t nf_total = 0;
    int nt = nthreads < 1 ? 1 : nthreads;
#pragma omp parallel for num_threads(nt) schedule(static) reduction(+ : nf_total) if (nt > 1)
    for (int64_t m = 0; m < nm; ++m) {
        double x_old = x_m[m], y_old = y_m[m];
        double vx_eff = 0.0, vy_eff = 0.0;
        double vx_rk = 0.0, vy_rk = 0.0;
        int64_t nf = 0;
        for (int it = 0; it < 4; ++it) {
            double x_rk = x_old + rk4_dt[it] * vx_rk;
            double y_rk = y_old + rk4_dt[it] * vy_rk;
            orc_interpolate_v(x_rk, y_rk, Vx, vx_nx, vx_ny, Vy, vy_nx, vy_ny, x_vx_min, y_vx_min,
                              x_vy_min, y_vy_min, dx, dy, &vx_rk, &vy_rk, &nf);
            vx_eff = vx_eff + rk4_wt[it] * vx_rk;
            vy_eff = vy_eff + rk4_wt[it] * vy_rk;
        }
        double x_new = x_old + vx_eff * dt;
        double y_new = y_old + vy_eff * dt;
        x_new = jl_min(jl_max0(x_new), lx);
        y_new = jl_min(jl_max0(y_new), ly);
        x_m[m] = x_new;
        y_m[m] = y_new;
        nf_total += nf;
    }
    if (n_fail) *n_fail = nf_total;
}
