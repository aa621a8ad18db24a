// sf_advect.cu -- RK4 marker advection (scripts/MoveMarkers.jl:15-187) for
// libstokesflow_b200.so.  One thread per marker; every floating-point
// expression keeps the reference's order and the file is compiled with
// -fmad=false, so positions are bit-identical to the reference's.
//
// The padded velocity arrays (2 x (N+2)(N+1) doubles, 67 MB at N = 2048) sit
// in the 126 MB L2, so the 4 x 12 gathers per marker are L2 hits; HBM traffic
// is the marker read/write (32 B per marker) plus one pass over V.
#include <algorithm>

#include "sf_internal.cuh"

namespace sf {

struct AdvectArgs {
    const double* Vx;
    const double* Vy;
    int64_t vx_nx, vx_ny, vy_nx, vy_ny;
    double x_vx_min, y_vx_min, x_vy_min, y_vy_min;
    double dx, dy;
};

// MoveMarkers.jl:181-187 bilinearInterp
__device__ __forceinline__ double bilinear_interp(double v1, double v2, double v3, double v4, double dxij,
                                                  double dyij) {
    double s1 = (1.0 - dxij) * (1.0 - dyij) * v1;
    double s2 = dxij * (1.0 - dyij) * v2;
    double s3 = (1.0 - dxij) * dyij * v3;
    double s4 = dxij * dyij * v4;
    return s1 + s2 + s3 + s4;
}

#define VXA(i, j) __ldg(&a.Vx[((i) - 1) + ((j) - 1) * a.vx_nx])
#define VYA(i, j) __ldg(&a.Vy[((i) - 1) + ((j) - 1) * a.vy_nx])

// MoveMarkers.jl:76-174 interpolateV.  ix, iy are 1-based as in the reference.
__device__ __forceinline__ void interpolate_v(const AdvectArgs& a, double x, double y, double& vx_out, double& vy_out,
                                              int& nfail) {
    // ---- Vx ----
    TopLeft t = topleft(a.x_vx_min, a.y_vx_min, x, y, a.dx, a.dy);
    double dxij = t.dxij, dyij = t.dyij;
    // clamp the double index before converting (NaN / huge -> failsafe branch, as below)
    int64_t ix, iy;
    {
        double qx = t.qx + 1.0, qy = t.qy + 1.0;
        ix = (qx >= 2.0) ? ((qx < (double)(a.vx_nx - 1)) ? (int64_t)qx : a.vx_nx - 1) : 1;
        iy = (qy >= 1.0) ? ((qy < (double)a.vx_ny) ? (int64_t)qy : a.vx_ny) : 0;
    }
    if (ix < 2) { ++nfail; ix = 2; dxij = 0.0; }
    if (iy < 1) { ++nfail; iy = 1; dyij = 0.0; }
    if (ix >= a.vx_nx - 1) { ++nfail; ix = a.vx_nx - 2; dxij = 1.0; }
    if (iy >= a.vx_ny) { ++nfail; iy = a.vx_ny - 1; dyij = 1.0; }
    double v1 = VXA(ix, iy), v2 = VXA(ix + 1, iy), v3 = VXA(ix, iy + 1), v4 = VXA(ix + 1, iy + 1);
    double vx = bilinear_interp(v1, v2, v3, v4, dxij, dyij);
    double correction;
    if (dxij >= 0.5) {
        double v5 = VXA(ix + 2, iy), v6 = VXA(ix + 2, iy + 1);
        double h = dxij - 0.5;
        correction = 0.5 * (h * h) * ((1.0 - dyij) * (v1 - 2.0 * v2 + v5) + dyij * (v3 - 2.0 * v4 + v6));
    } else {
        double v5 = VXA(ix - 1, iy), v6 = VXA(ix - 1, iy + 1);
        double h = dxij - 0.5;
        correction = 0.5 * (h * h) * ((1.0 - dyij) * (v5 - 2.0 * v1 + v2) + dyij * (v6 - 2.0 * v3 + v4));
    }
    vx = vx + correction;
    // ---- Vy ----
    t = topleft(a.x_vy_min, a.y_vy_min, x, y, a.dx, a.dy);
    dxij = t.dxij;
    dyij = t.dyij;
    {
        double qx = t.qx + 1.0, qy = t.qy + 1.0;
        ix = (qx >= 1.0) ? ((qx < (double)a.vy_nx) ? (int64_t)qx : a.vy_nx) : 0;
        iy = (qy >= 2.0) ? ((qy < (double)(a.vy_ny - 1)) ? (int64_t)qy : a.vy_ny - 1) : 1;
    }
    if (ix < 1) { ++nfail; ix = 1; dxij = 0.0; }
    if (iy < 2) { ++nfail; iy = 2; dyij = 0.0; }
    if (ix >= a.vy_nx) { ++nfail; ix = a.vy_nx - 1; dxij = 1.0; }
    if (iy >= a.vy_ny - 1) { ++nfail; iy = a.vy_ny - 2; dyij = 1.0; }
    v1 = VYA(ix, iy); v2 = VYA(ix + 1, iy); v3 = VYA(ix, iy + 1); v4 = VYA(ix + 1, iy + 1);
    double vy = bilinear_interp(v1, v2, v3, v4, dxij, dyij);
    if (dyij >= 0.5) {
        double v5 = VYA(ix, iy + 2), v6 = VYA(ix + 1, iy + 2);
        double h = dyij - 0.5;
        correction = 0.5 * (h * h) * ((1.0 - dxij) * (v1 - 2.0 * v3 + v5) + dxij * (v2 - 2.0 * v4 + v6));
    } else {
        double v5 = VYA(ix, iy - 1), v6 = VYA(ix + 1, iy - 1);
        double h = dyij - 0.5;
        correction = 0.5 * (h * h) * ((1.0 - dxij) * (v5 - 2.0 * v1 + v3) + dxij * (v6 - 2.0 * v2 + v4));
    }
    vy = vy + correction;
    vx_out = vx;
    vy_out = vy;
}

// MoveMarkers.jl:30-69 moveMarkersRK4_Kernel!
__global__ void __launch_bounds__(256) k_move_markers_rk4(AdvectArgs a, double* __restrict__ x_m,
                                                         double* __restrict__ y_m, int64_t nm, double dt, double lx,
                                                         double ly, unsigned long long* __restrict__ fail_counter) {
    const double rk4_dt[4] = {0.0, 0.5 * dt, 0.5 * dt, dt};
    const double rk4_wt[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};
    int nfail = 0;
    for (int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; m < nm; m += (int64_t)gridDim.x * blockDim.x) {
        double x_old = x_m[m], y_old = y_m[m];
        double vx_eff = 0.0, vy_eff = 0.0, vx_rk = 0.0, vy_rk = 0.0;
#pragma unroll
        for (int it = 0; it < 4; ++it) {
            double x_rk = x_old + rk4_dt[it] * vx_rk;
            double y_rk = y_old + rk4_dt[it] * vy_rk;
            interpolate_v(a, x_rk, y_rk, vx_rk, vy_rk, nfail);
            vx_eff = vx_eff + rk4_wt[it] * vx_rk;
            vy_eff = vy_eff + rk4_wt[it] * vy_rk;
        }
        double x_new = x_old + vx_eff * dt;
        double y_new = y_old + vy_eff * dt;
        x_m[m] = jl_min(jl_max0(x_new), lx);
        y_m[m] = jl_min(jl_max0(y_new), ly);
    }
    if (__any_sync(0xffffffffu, nfail != 0)) {
        for (int o = 16; o > 0; o >>= 1) nfail += __shfl_xor_sync(0xffffffffu, nfail, o);
        if ((threadIdx.x & 31) == 0 && fail_counter) atomicAdd(fail_counter, (unsigned long long)nfail);
    }
}

}  // namespace sf

using namespace sf;

extern "C" {

int sf_move_markers_rk4(sf_ctx* ctx, double* x_m, double* y_m, int64_t nm, const double* Vx, int64_t vx_nx,
                        int64_t vx_ny, const double* Vy, int64_t vy_nx, int64_t vy_ny, double x_vx_min,
                        double y_vx_min, double x_vy_min, double y_vy_min, double dt, double lx, double ly, double dx,
                        double dy, void* stream) {
    SF_REQUIRE(ctx, "sf_move_markers_rk4: ctx is NULL");
    SF_REQUIRE(nm >= 0 && (nm == 0 || (x_m && y_m)), "sf_move_markers_rk4: bad markers");
    SF_REQUIRE(Vx && Vy && vx_nx >= 4 && vx_ny >= 2 && vy_nx >= 2 && vy_ny >= 4,
               "sf_move_markers_rk4: velocity arrays too small (need Vx >= 4x2, Vy >= 2x4)");
    SF_REQUIRE(dx > 0.0 && dy > 0.0, "sf_move_markers_rk4: dx, dy must be positive");
    if (nm == 0) return SF_OK;
    int rc = set_device(ctx);
    if (rc) return rc;
    AdvectArgs a{Vx, Vy, vx_nx, vx_ny, vy_nx, vy_ny, x_vx_min, y_vx_min, x_vy_min, y_vy_min, dx, dy};
    unsigned blocks = (unsigned)std::min<int64_t>(ceil_div(nm, 256), (int64_t)ctx->num_sms * 16);
    k_move_markers_rk4<<<blocks, 256, 0, as_stream(stream)>>>(a, x_m, y_m, nm, dt, lx, ly,
                                                              ctx->d_counters + CNT_INTERP_FAILSAFE);
    SF_LAUNCHED(ctx);
    return SF_OK;
}

}  // extern "C"
