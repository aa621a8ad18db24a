/* One StokesFlow2D timestep through the C ABI alone -- no Python, no torch: the calls a C or Julia host makes.
 * Markers set up on the device, the three deposits of the timestep in one fused call (checked byte for byte
 * against one call per grid), the PT solve to relative residual 1e-6, RK4 advection and the rebin.
 * Built and run by tests/test_gpu_c_abi.py; prints one line and returns 0 on success. */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <cuda_runtime_api.h>

#include "stokesflow_b200.h"

#define CHECK(call)                                                                   \
    do {                                                                              \
        int rc_ = (call);                                                             \
        if (rc_ != SF_OK) {                                                           \
            fprintf(stderr, "%s failed: %s (%s)\n", #call, sf_status_string(rc_),     \
                    sf_last_error());                                                 \
            return 1;                                                                 \
        }                                                                             \
    } while (0)
#define CUDA(call)                                                                    \
    do {                                                                              \
        cudaError_t e_ = (call);                                                      \
        if (e_ != cudaSuccess) {                                                      \
            fprintf(stderr, "%s failed: %s\n", #call, cudaGetErrorString(e_));        \
            return 1;                                                                 \
        }                                                                             \
    } while (0)

static double* dalloc(int64_t n) {
    double* p = NULL;
    if (cudaMalloc((void**)&p, (size_t)(n > 0 ? n : 1) * sizeof(double)) != cudaSuccess) return NULL;
    if (cudaMemset(p, 0, (size_t)(n > 0 ? n : 1) * sizeof(double)) != cudaSuccess) return NULL;
    return p;
}

static int same(const double* a, const double* b, int64_t n) {
    size_t bytes = (size_t)n * sizeof(double);
    double* ha = (double*)malloc(bytes);
    double* hb = (double*)malloc(bytes);
    int eq = ha && hb && cudaMemcpy(ha, a, bytes, cudaMemcpyDeviceToHost) == cudaSuccess &&
             cudaMemcpy(hb, b, bytes, cudaMemcpyDeviceToHost) == cudaSuccess && memcmp(ha, hb, bytes) == 0;
    free(ha);
    free(hb);
    return eq;
}

int main(void) {
    const int64_t Nx = 33, Ny = 33, md = 4;
    const double lx = 1.0, ly = 1.0, dx = lx / (double)(Nx - 1), dy = ly / (double)(Ny - 1);
    sf_ctx* ctx = NULL;
    CHECK(sf_ctx_create(0, &ctx));

    /* markers: initializeMarkersCPU + setInitialMarkerProperties! of the plume model */
    int64_t nmx = 0, nmy = 0;
    CHECK(sf_marker_count(md, Nx, Ny, &nmx, &nmy));
    const int64_t nm = nmx * nmy;
    double *x = dalloc(nm), *y = dalloc(nm), *rho = dalloc(nm), *mu = dalloc(nm);
    if (!x || !y || !rho || !mu) return 1;
    CHECK(sf_init_markers(ctx, md, lx, ly, dx, dy, Nx, Ny, 0.5, 0, x, y, NULL));
    const sf_plume_model model = {0.1, 0.5, 0.75, 0.1, 1e-3, 1.0, 0.9, 1e-2, 1.0, 0.1};
    CHECK(sf_set_marker_properties(ctx, &model, x, y, nm, 0.0, 0.0, rho, mu, NULL));

    /* the three deposits (StokesFlow2D_multixpu.jl:164-166), fused and one call per grid */
    double *rho_vy = dalloc((Nx + 1) * Ny), *mu_b = dalloc(Nx * Ny), *mu_p = dalloc((Nx - 1) * (Ny - 1));
    double *rho1 = dalloc((Nx + 1) * Ny), *mub1 = dalloc(Nx * Ny), *mup1 = dalloc((Nx - 1) * (Ny - 1));
    if (!rho_vy || !mu_b || !mu_p || !rho1 || !mub1 || !mup1) return 1;
    const sf_deposit_grid grids[3] = {{-0.5 * dx, 0.0, rho_vy, Nx + 1, Ny, rho},
                                      {0.0, 0.0, mu_b, Nx, Ny, mu},
                                      {0.5 * dx, 0.5 * dy, mu_p, Nx - 1, Ny - 1, mu}};
    CHECK(sf_bilinear_marker_to_grids(ctx, grids, 3, x, y, nm, dx, dy, NULL, NULL, 0, 0, NULL));
    CHECK(sf_bilinear_marker_to_grid(ctx, -0.5 * dx, 0.0, rho1, Nx + 1, Ny, x, y, rho, nm, dx, dy, NULL, NULL, 0, 0,
                                     NULL));
    CHECK(sf_bilinear_marker_to_grid(ctx, 0.0, 0.0, mub1, Nx, Ny, x, y, mu, nm, dx, dy, NULL, NULL, 0, 0, NULL));
    CHECK(sf_bilinear_marker_to_grid(ctx, 0.5 * dx, 0.5 * dy, mup1, Nx - 1, Ny - 1, x, y, mu, nm, dx, dy, NULL, NULL,
                                     0, 0, NULL));
    CUDA(cudaDeviceSynchronize());
    if (!same(rho_vy, rho1, (Nx + 1) * Ny) || !same(mu_b, mub1, Nx * Ny) || !same(mu_p, mup1, (Nx - 1) * (Ny - 1))) {
        fprintf(stderr, "fused deposit differs from one call per grid\n");
        return 1;
    }

    /* the PT solve from rest to relative residual 1e-6 (the work arrays are optional) */
    double *P = dalloc((Nx - 1) * (Ny - 1)), *Vx_pad = dalloc((Nx + 2) * (Ny + 1)), *Vy_pad = dalloc((Nx + 1) * (Ny + 2));
    double *dVx = dalloc((Nx - 2) * (Ny - 1)), *dVy = dalloc((Nx - 1) * (Ny - 2));
    double *Vx_s = dalloc(Nx * (Ny + 1)), *Vy_s = dalloc((Nx + 1) * Ny);
    if (!P || !Vx_pad || !Vy_pad || !dVx || !dVy || !Vx_s || !Vy_s) return 1;
    const double g_y = 9.81, maxdisp = 0.5;
    double scale = 0.0;
    CHECK(sf_stokes_residual_scale(ctx, rho_vy, Nx, Ny, g_y, NULL, &scale));
    sf_solve_info info;
    CHECK(sf_solve_stokes(ctx, P, Vx_pad, Vy_pad, rho_vy, mu_b, mu_p, NULL, NULL, NULL, NULL, NULL, NULL, NULL, dVx,
                          dVy, NULL, NULL, Vx_s, Vy_s, g_y, dx, dy, Nx, Ny, 0.0, maxdisp, 1, 1e-6 * scale, 0, 100000,
                          NULL, &info));
    if (!info.converged || !(info.dt > 0.0) || info.iters < 1) {
        fprintf(stderr, "solve: converged %d, dt %g, iters %lld\n", info.converged, info.dt, (long long)info.iters);
        return 1;
    }

    /* RK4 advection on the padded velocities (origins of StokesFlow2D_multixpu.jl:121-124), then the rebin */
    CHECK(sf_move_markers_rk4(ctx, x, y, nm, Vx_pad, Nx + 2, Ny + 1, Vy_pad, Nx + 1, Ny + 2, -dx, -0.5 * dy,
                              -0.5 * dx, -dy, info.dt, lx, ly, dx, dy, NULL));
    const int64_t ncells = (Nx + 1) * (Ny + 1);
    int32_t *counts = NULL, *offsets = NULL, *perm = NULL;
    CUDA(cudaMalloc((void**)&counts, (size_t)ncells * 4));
    CUDA(cudaMalloc((void**)&offsets, (size_t)(ncells + 1) * 4));
    CUDA(cudaMalloc((void**)&perm, (size_t)nm * 4));
    CHECK(sf_rebin_markers(ctx, x, y, nm, 0.0, 0.0, dx, dy, Nx, Ny, counts, offsets, perm, NULL));
    CUDA(cudaDeviceSynchronize());
    int32_t total = -1;
    CUDA(cudaMemcpy(&total, offsets + ncells, 4, cudaMemcpyDeviceToHost));
    double* hx = (double*)malloc((size_t)nm * sizeof(double));
    double* hy = (double*)malloc((size_t)nm * sizeof(double));
    if (!hx || !hy) return 1;
    CUDA(cudaMemcpy(hx, x, (size_t)nm * sizeof(double), cudaMemcpyDeviceToHost));
    CUDA(cudaMemcpy(hy, y, (size_t)nm * sizeof(double), cudaMemcpyDeviceToHost));
    for (int64_t m = 0; m < nm; ++m)
        if (!(hx[m] >= 0.0 && hx[m] <= lx && hy[m] >= 0.0 && hy[m] <= ly)) {
            fprintf(stderr, "marker %lld outside the domain after advection\n", (long long)m);
            return 1;
        }
    if (total != (int32_t)nm) {
        fprintf(stderr, "rebin placed %d of %lld markers\n", total, (long long)nm);
        return 1;
    }
    CHECK(sf_ctx_destroy(ctx));
    printf("c abi ok: %lld markers, %lld PT iterations, dt %.6e\n", (long long)nm, (long long)info.iters, info.dt);
    free(hx);
    free(hy);
    return 0;
}
