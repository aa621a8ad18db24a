// sf_mixed.cu -- mixed-precision, batched pseudo-transient Stokes solve.
//
// Defect correction around FP32 PT sweeps.  For every instance (one Stokes
// problem of StokesSolver_multixpu.jl:14-96, its own grid size) the FP64 state
// (V, P) is corrected repeatedly:
//
//   1. FP64: dt = maxdisp*min(dx/max|Vx|, dy/max|Vy|) (compute_dt, :118-121),
//      then the residuals R_k = (Rx, Ry, divV) of (V_k, P_k) with the
//      reference's formulas (:140-202) and err_k = max of their mean |.|
//      (compute_err, :103-109).  Stop when err_k <= eps.
//   2. FP32: `fold_every` sweeps of the reference's PT iteration (:128-234,
//      same damping, pseudo-time steps and free-slip BCs) applied to the
//      correction (dV, dP) from zero, with R_k as the constant term -- i.e. the
//      PT iteration of the full problem continued from (V_k, P_k), its damped
//      rates kept across folds (in exact arithmetic the whole sequence is the
//      FP64 iteration; folding often keeps each FP32 increment well above the
//      rounding of the correction it is added to).
//   3. FP64 fold: V_{k+1} = V_k + dV, P_{k+1} = P_k + dP; back to 1.
//
// All instances live in one arena.  Every FP32 sweep is ONE persistent kernel
// launch over a device-resident work list of 32 x 16 tiles from all instances
// in their inner phase, with per-instance tensor maps (TMA, double-buffered,
// no multicast) -- so hundreds of small problems cost one launch per
// iteration instead of hundreds.  The runs of iterations between checks are
// replayed from a captured CUDA graph.  Instances move between phases
// independently, which is what lets a serving loop add and retire instances
// while others run.
//
// The FP32 sweeps are not bit-compatible with the plain FP64 path (nothing can
// be at FP32); their accuracy is measured against the FP64 oracle.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <type_traits>
#include <vector>

#include "sf_internal.cuh"
#include "sf_tma.cuh"

namespace sf {
namespace mx {

constexpr int BX = 32, BY = 16, TY = 8, RPT = BY / TY, NT = BX * TY;
constexpr int TW = 36, TH = BY + 2;   // staged halo box; TW*4 bytes is a multiple of 16
constexpr int W1 = BX + 1, H1 = BY + 1;
constexpr int r128(int b) { return (b + 127) / 128 * 128; }
constexpr int HALO_BYTES = r128(TH * TW * 4);
constexpr int TILE_BYTES = r128(BY * BX * 4);
constexpr int NHALO = 7;  // dVx, dVy, dP (current), mu_b, mu_p, rho, rdiv
constexpr int NTILE = 4;  // rate_x, rate_y, rx, ry
constexpr int STAGE_BYTES = NHALO * HALO_BYTES + NTILE * TILE_BYTES;
constexpr uint32_t STAGE_TX = NHALO * TH * TW * 4 + NTILE * BY * BX * 4;
constexpr int ST1_BYTES = r128(H1 * W1 * 4);
constexpr int NST = 2;
constexpr int SMEM_BYTES = NST * STAGE_BYTES + 4 * ST1_BYTES + 64;
constexpr uint64_t WAIT_BUDGET_NS = 2000000000ull;

// FP32 fields of an instance (each LD32 x rows floats)
enum { G_VXA, G_VXB, G_VYA, G_VYB, G_PA, G_PB, G_RVX, G_RVY, G_MUB, G_MUP, G_RHO, G_RX, G_RY, G_RDIV, G_NUM };
// FP64 fields of an instance (each LD64 x rows doubles)
enum { D_VX, D_VY, D_P, D_RHO, D_MUB, D_MUP, D_NUM };
// tensor maps per instance, in the order a stage is filled
enum { M_VXA, M_VXB, M_VYA, M_VYB, M_PA, M_PB, M_MUB, M_MUP, M_RHO, M_RDIV, M_RVX, M_RVY, M_RX, M_RY, M_NUM };

struct Inst {  // device-side description of one instance
    int Nx, Ny, ntx, nty;
    int64_t LD32, LD64, rows;
    float* f32;             // G_NUM fields
    double* f64;            // D_NUM fields
    int64_t fstride32, fstride64;
    float _dxf, _dyf, dampXf, dampYf, c_vscf, c_ptscf;   // FP32 constants
    float g_dtf;            // g_y * dt for the stabilisation term of the correction
    int parity;             // which dV/dP buffer is "in" at launch parity 0
    double dx, dy, _dx, _dy, g_y, dt, dt_cfl, dt_in, maxdisp;
    int use_stab;
    int pad_;
};

__device__ __forceinline__ float* gf(const Inst& I, int k) { return I.f32 + (int64_t)k * I.fstride32; }
__device__ __forceinline__ double* gd(const Inst& I, int k) { return I.f64 + (int64_t)k * I.fstride64; }

// ---------------------------------------------------------------------------
// FP32 PT sweep over a tile work list (tiles: {instance, tile index})
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(NT, 3) k_pt32(const CUtensorMap* __restrict__ maps, const Inst* __restrict__ insts,
                                               const int2* __restrict__ tiles, const int* __restrict__ ntiles_ptr,
                                               int launch_parity, int* __restrict__ err_flag) {
    extern __shared__ __align__(128) unsigned char smem[];
    typedef float Row1[W1];
    typedef float RowH[TW];
    typedef float RowT[BX];
    Row1* sPn = reinterpret_cast<Row1*>(smem + NST * STAGE_BYTES);
    Row1* sTxx = reinterpret_cast<Row1*>(smem + NST * STAGE_BYTES + ST1_BYTES);
    Row1* sTyy = reinterpret_cast<Row1*>(smem + NST * STAGE_BYTES + 2 * ST1_BYTES);
    Row1* sTxy = reinterpret_cast<Row1*>(smem + NST * STAGE_BYTES + 3 * ST1_BYTES);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + NST * STAGE_BYTES + 4 * ST1_BYTES);

    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * BX + tx;
    const int ntiles = *ntiles_ptr;
    if (tid == 0) {
        for (int k = 0; k < NST; ++k) mbar_init(&bar[k], 1);
        fence_mbar_init();
    }
    __syncthreads();
    auto issue = [&](int t, int s) {  // thread 0 only
        const int2 td = tiles[t];
        const Inst& I = insts[td.x];
        const int i0 = (td.y % I.ntx) * BX, j0 = (td.y / I.ntx) * BY;
        const int in = (I.parity ^ launch_parity) & 1;
        const CUtensorMap* M = maps + (int64_t)td.x * M_NUM;
        unsigned char* st = smem + s * STAGE_BYTES;
        mbar_arrive_expect_tx(&bar[s], STAGE_TX);
        tma_load_2d(st + 0 * HALO_BYTES, &M[in ? M_VXB : M_VXA], &bar[s], i0, j0);
        tma_load_2d(st + 1 * HALO_BYTES, &M[in ? M_VYB : M_VYA], &bar[s], i0, j0);
        tma_load_2d(st + 2 * HALO_BYTES, &M[in ? M_PB : M_PA], &bar[s], i0, j0);
        tma_load_2d(st + 3 * HALO_BYTES, &M[M_MUB], &bar[s], i0, j0);
        tma_load_2d(st + 4 * HALO_BYTES, &M[M_MUP], &bar[s], i0, j0);
        tma_load_2d(st + 5 * HALO_BYTES, &M[M_RHO], &bar[s], i0, j0);
        tma_load_2d(st + 6 * HALO_BYTES, &M[M_RDIV], &bar[s], i0, j0);
        unsigned char* tb = st + NHALO * HALO_BYTES;
        tma_load_2d(tb + 0 * TILE_BYTES, &M[M_RVX], &bar[s], i0, j0);
        tma_load_2d(tb + 1 * TILE_BYTES, &M[M_RVY], &bar[s], i0, j0);
        tma_load_2d(tb + 2 * TILE_BYTES, &M[M_RX], &bar[s], i0, j0);
        tma_load_2d(tb + 3 * TILE_BYTES, &M[M_RY], &bar[s], i0, j0);
    };
    const int G = gridDim.x;
    int t = blockIdx.x;
    if (tid == 0)
        for (int k = 0; k < NST - 1; ++k)
            if (t + k * G < ntiles) issue(t + k * G, k);
    uint32_t phase = 0;
    int s = 0;
    for (; t < ntiles; t += G) {
        const int tn = t + (NST - 1) * G;
        if (tid == 0 && tn < ntiles) issue(tn, (s + NST - 1) % NST);
        const bool ok = mbar_wait(&bar[s], (phase >> s) & 1u, WAIT_BUDGET_NS);
        phase ^= 1u << s;
        if (__syncthreads_or(!ok)) {
            if (tid == 0) {
                atomicExch(err_flag, 1);
                for (int k = 0; k < NST; ++k) {
                    if (t + k * G >= ntiles) break;
                    const int sk = (s + k) % NST;
                    const uint32_t par = (k == 0) ? (((phase >> sk) & 1u) ^ 1u) : ((phase >> sk) & 1u);
                    mbar_wait(&bar[sk], par, WAIT_BUDGET_NS);
                }
            }
            __syncthreads();
            return;
        }
        const int2 td = tiles[t];
        const Inst& I = insts[td.x];
        const int Nx = I.Nx, Ny = I.Ny;
        const int i0 = (td.y % I.ntx) * BX, j0 = (td.y / I.ntx) * BY;
        const int in = (I.parity ^ launch_parity) & 1;
        const int64_t LD = I.LD32;
        const float _dx = I._dxf, _dy = I._dyf;
        unsigned char* st = smem + s * STAGE_BYTES;
        RowH* sVx = reinterpret_cast<RowH*>(st + 0 * HALO_BYTES);
        RowH* sVy = reinterpret_cast<RowH*>(st + 1 * HALO_BYTES);
        RowH* sPo = reinterpret_cast<RowH*>(st + 2 * HALO_BYTES);
        RowH* sMub = reinterpret_cast<RowH*>(st + 3 * HALO_BYTES);
        RowH* sMup = reinterpret_cast<RowH*>(st + 4 * HALO_BYTES);
        RowH* sRho = reinterpret_cast<RowH*>(st + 5 * HALO_BYTES);
        RowH* sRdiv = reinterpret_cast<RowH*>(st + 6 * HALO_BYTES);
        unsigned char* tb = st + NHALO * HALO_BYTES;
        RowT* sRvx = reinterpret_cast<RowT*>(tb + 0 * TILE_BYTES);
        RowT* sRvy = reinterpret_cast<RowT*>(tb + 1 * TILE_BYTES);
        RowT* sRx = reinterpret_cast<RowT*>(tb + 2 * TILE_BYTES);
        RowT* sRy = reinterpret_cast<RowT*>(tb + 3 * TILE_BYTES);
        float* Vx_out = gf(I, in ? G_VXA : G_VXB);
        float* Vy_out = gf(I, in ? G_VYA : G_VYB);
        float* P_out = gf(I, in ? G_PA : G_PB);
        float* Rvx = gf(I, G_RVX);
        float* Rvy = gf(I, G_RVY);

        // ---- stage 1: P and tau of the correction on tile + 1 halo ----
        for (int idx = tid; idx < W1 * H1; idx += NT) {
            const int b = idx / W1, a = idx - b * W1;
            const int i = i0 + a, j = j0 + b;
            if (i < Nx - 1 && j < Ny - 1) {
                float dVx_dx = (sVx[b + 1][a + 1] - sVx[b + 1][a]) * _dx;
                float dVy_dy = (sVy[b + 1][a + 1] - sVy[b][a + 1]) * _dy;
                float div_d = dVx_dx + dVy_dy;
                float div_full = div_d + sRdiv[b][a];          // divV of V_k + dV
                float mu = sMup[b][a];
                sPn[b][a] = sPo[b][a] - I.c_ptscf * mu * div_full;
                sTxx[b][a] = 2.0f * mu * (dVx_dx - (1.0f / 3.0f) * div_d);
                sTyy[b][a] = 2.0f * mu * (dVy_dy - (1.0f / 3.0f) * div_d);
            }
            if (i < Nx && j < Ny) {
                float dVx_dy = (sVx[b + 1][a] - sVx[b][a]) * _dy;
                float dVy_dx = (sVy[b][a + 1] - sVy[b][a]) * _dx;
                sTxy[b][a] = sMub[b][a] * (dVx_dy + dVy_dx);
            }
        }
        __syncthreads();
        // ---- stage 2: damped rates and velocity update of the correction ----
#pragma unroll
        for (int r = 0; r < RPT; ++r) {
            const int a = tx, b = ty + r * TY;
            const int i = i0 + a, j = j0 + b;
            if (i >= Nx - 1 || j >= Ny - 1) continue;
            const int64_t o = i + (int64_t)j * LD;
            P_out[o] = sPn[b][a];
            if (i < Nx - 2) {
                float Rx = (sTxx[b][a + 1] - sTxx[b][a]) * _dx + (sTxy[b + 1][a + 1] - sTxy[b][a + 1]) * _dy -
                           (sPn[b][a + 1] - sPn[b][a]) * _dx + sRx[b][a];
                float dv = I.dampXf * sRvx[b][a] + Rx;
                Rvx[o] = dv;
                float dtau = I.c_vscf / ((sMup[b][a] + sMup[b][a + 1]) * 0.5f);
                float vn = sVx[b + 1][a + 1] + dtau * dv;
                Vx_out[o + 1 + LD] = vn;
                if (j == 0) Vx_out[o + 1] = vn;
                if (j == Ny - 2) Vx_out[o + 1 + 2 * LD] = vn;
            }
            if (j < Ny - 2) {
                float av = 0.25f * (sVx[b + 1][a] + sVx[b + 1][a + 1] + sVx[b + 2][a] + sVx[b + 2][a + 1]);
                float dxr = sRho[b + 1][a + 2] - sRho[b + 1][a];
                float dyr = sRho[b + 2][a + 1] - sRho[b][a + 1];
                float Ry = (sTyy[b + 1][a] - sTyy[b][a]) * _dy + (sTxy[b + 1][a + 1] - sTxy[b + 1][a]) * _dx -
                           (sPn[b + 1][a] - sPn[b][a]) * _dy -
                           I.g_dtf * (av * dxr * 0.5f * _dx + sVy[b + 1][a + 1] * dyr * 0.5f * _dy) + sRy[b][a];
                float dv = I.dampYf * sRvy[b][a] + Ry;
                Rvy[o] = dv;
                float dtau = I.c_vscf / ((sMup[b][a] + sMup[b + 1][a]) * 0.5f);
                float vn = sVy[b + 1][a + 1] + dtau * dv;
                Vy_out[o + 1 + LD] = vn;
                if (i == 0) Vy_out[o + LD] = vn;
                if (i == Nx - 2) Vy_out[o + 2 + LD] = vn;
            }
            if (i == 0 || i == Nx - 2) {
                int ic = (i == 0) ? 0 : Nx - 1;
                Vx_out[ic + (int64_t)(j + 1) * LD] = 0.f;
                if (j == 0) Vx_out[ic] = 0.f;
                if (j == Ny - 2) Vx_out[ic + (int64_t)Ny * LD] = 0.f;
            }
            if (j == 0 || j == Ny - 2) {
                int64_t jr = (j == 0) ? 0 : (int64_t)(Ny - 1) * LD;
                Vy_out[(i + 1) + jr] = 0.f;
                if (i == 0) Vy_out[jr] = 0.f;
                if (i == Nx - 2) Vy_out[Nx + jr] = 0.f;
            }
        }
        __syncthreads();  // stage s and the stage-1 arrays are free again
        s = (s + 1 == NST) ? 0 : s + 1;
    }
}

// ---------------------------------------------------------------------------
// FP64 kernels over tile lists (one CTA per tile)
// ---------------------------------------------------------------------------
constexpr int T64 = 256;

__device__ __forceinline__ double blk_sum(double v, double* sh) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r += sh[w];
    __syncthreads();
    return r;
}
__device__ __forceinline__ double blk_max(double v, double* sh) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r = fmax(r, sh[w]);
    __syncthreads();
    return r;
}

// max |Vx|, |Vy| of the FP64 state per tile (compute_dt's maxima; ghost entries repeat interior values or are 0)
__global__ void __launch_bounds__(T64) k_maxv64(const Inst* __restrict__ insts, const int2* __restrict__ tiles,
                                               double* __restrict__ part) {
    __shared__ double sh[T64 / 32];
    const int2 td = tiles[blockIdx.x];
    const Inst& I = insts[td.x];
    const int i0 = (td.y % I.ntx) * BX, j0 = (td.y / I.ntx) * BY;
    const double* Vx = gd(I, D_VX);
    const double* Vy = gd(I, D_VY);
    double mx = 0.0, my = 0.0;
    for (int k = threadIdx.x; k < BX * BY; k += T64) {
        const int i = i0 + (k % BX), j = j0 + (k / BX);
        if (i < I.Nx - 2 && j < I.Ny - 1) mx = fmax(mx, fabs(Vx[(i + 1) + (int64_t)(j + 1) * I.LD64]));
        if (i < I.Nx - 1 && j < I.Ny - 2) my = fmax(my, fabs(Vy[(i + 1) + (int64_t)(j + 1) * I.LD64]));
    }
    double a = blk_max(mx, sh), b = blk_max(my, sh);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = a;
        part[2 * blockIdx.x + 1] = b;
    }
}

// FP64 residuals of (V, P) (compute_ResX/ResY :176-202 with dt, divV :154-157), FP32 copies for the
// correction's constant term, per-tile sums of |Rx|, |Ry|, |divV|
__global__ void __launch_bounds__(T64) k_resid64(const Inst* __restrict__ insts, const int2* __restrict__ tiles,
                                                double* __restrict__ part) {
    __shared__ double sh[T64 / 32];
    const int2 td = tiles[blockIdx.x];
    const Inst& I = insts[td.x];
    const int Nx = I.Nx, Ny = I.Ny;
    const int i0 = (td.y % I.ntx) * BX, j0 = (td.y / I.ntx) * BY;
    const int64_t L = I.LD64, L32 = I.LD32;
    const double* Vx = gd(I, D_VX);
    const double* Vy = gd(I, D_VY);
    const double* P = gd(I, D_P);
    const double* rho = gd(I, D_RHO);
    const double* mub = gd(I, D_MUB);
    const double* mup = gd(I, D_MUP);
    float* rx = gf(I, G_RX);
    float* ry = gf(I, G_RY);
    float* rdiv = gf(I, G_RDIV);
    const double _dx = I._dx, _dy = I._dy, dt = I.dt;
    // tau at P point (i, j) and tau_xy at node (i, j), from (:154-166)
    auto txx_at = [&](int i, int j, double* tyy) {
        double dVx_dx = (Vx[(i + 1) + (int64_t)(j + 1) * L] - Vx[i + (int64_t)(j + 1) * L]) * _dx;
        double dVy_dy = (Vy[(i + 1) + (int64_t)(j + 1) * L] - Vy[(i + 1) + (int64_t)j * L]) * _dy;
        double d = dVx_dx + dVy_dy;
        double mu = mup[i + (int64_t)j * L];
        *tyy = 2.0 * mu * (dVy_dy - 1.0 / 3.0 * d);
        return 2.0 * mu * (dVx_dx - 1.0 / 3.0 * d);
    };
    auto txy_at = [&](int i, int j) {
        double dVx_dy = (Vx[i + (int64_t)(j + 1) * L] - Vx[i + (int64_t)j * L]) * _dy;
        double dVy_dx = (Vy[(i + 1) + (int64_t)j * L] - Vy[i + (int64_t)j * L]) * _dx;
        return 2.0 * mub[i + (int64_t)j * L] * 0.5 * (dVx_dy + dVy_dx);
    };
    double srx = 0.0, sry = 0.0, sdv = 0.0;
    for (int k = threadIdx.x; k < BX * BY; k += T64) {
        const int i = i0 + (k % BX), j = j0 + (k / BX);
        if (i >= Nx - 1 || j >= Ny - 1) continue;
        const int64_t o = i + (int64_t)j * L, o32 = i + (int64_t)j * L32;
        double tyy0;
        double txx0 = txx_at(i, j, &tyy0);
        {
            double dVx_dx = (Vx[(i + 1) + (int64_t)(j + 1) * L] - Vx[i + (int64_t)(j + 1) * L]) * _dx;
            double dVy_dy = (Vy[(i + 1) + (int64_t)(j + 1) * L] - Vy[(i + 1) + (int64_t)j * L]) * _dy;
            double d = dVx_dx + dVy_dy;
            rdiv[o32] = (float)d;
            sdv += fabs(d);
        }
        if (i < Nx - 2) {
            double tyy1;
            double txx1 = txx_at(i + 1, j, &tyy1);
            double R = (txx1 - txx0) * _dx + (txy_at(i + 1, j + 1) - txy_at(i + 1, j)) * _dy -
                       (P[o + 1] - P[o]) * _dx;
            rx[o32] = (float)R;
            srx += fabs(R);
        }
        if (j < Ny - 2) {
            double tyy1;
            (void)txx_at(i, j + 1, &tyy1);
            double av = 0.25 * (Vx[i + (int64_t)(j + 1) * L] + Vx[(i + 1) + (int64_t)(j + 1) * L] +
                                Vx[i + (int64_t)(j + 2) * L] + Vx[(i + 1) + (int64_t)(j + 2) * L]);
            double dxr = rho[(i + 2) + (int64_t)(j + 1) * L] - rho[i + (int64_t)(j + 1) * L];
            double dyr = rho[(i + 1) + (int64_t)(j + 2) * L] - rho[(i + 1) + (int64_t)j * L];
            double R = (tyy1 - tyy0) * _dy + (txy_at(i + 1, j + 1) - txy_at(i, j + 1)) * _dx - (P[o + L] - P[o]) * _dy +
                       I.g_y * (rho[(i + 1) + (int64_t)(j + 1) * L] -
                                dt * (av * dxr * 0.5 * _dx + Vy[(i + 1) + (int64_t)(j + 1) * L] * dyr * 0.5 * _dy));
            ry[o32] = (float)R;
            sry += fabs(R);
        }
    }
    double a = blk_sum(srx, sh), b = blk_sum(sry, sh), c = blk_sum(sdv, sh);
    if (threadIdx.x == 0) {
        part[3 * blockIdx.x] = a;
        part[3 * blockIdx.x + 1] = b;
        part[3 * blockIdx.x + 2] = c;
    }
}

// per-instance reductions over the instance's contiguous range of tile partials
struct Seg { int inst, begin, end, pad_; };

__global__ void k_inst_dt(Inst* __restrict__ insts, const Seg* __restrict__ segs, const double* __restrict__ part) {
    __shared__ double sh[32];
    const Seg g = segs[blockIdx.x];
    double mx = 0.0, my = 0.0;
    for (int t = g.begin + threadIdx.x; t < g.end; t += blockDim.x) {
        mx = fmax(mx, part[2 * t]);
        my = fmax(my, part[2 * t + 1]);
    }
    double a = blk_max(mx, sh), b = blk_max(my, sh);
    if (threadIdx.x == 0) {
        // compute_dt (:118-121); while V is still zero the CFL dt is infinite and the stabilisation keeps
        // the dt the solve started with (the reference's first dt update comes only once V is non-zero)
        Inst& I = insts[g.inst];
        double x = I.dx / a, y = I.dy / b;
        double m = (y < x) ? y : x;
        if (x != x) m = x;
        if (y != y) m = y;
        I.dt_cfl = I.maxdisp * m;
        I.dt = I.use_stab ? (isfinite(I.dt_cfl) ? I.dt_cfl : I.dt_in) : 0.0;
        I.g_dtf = (float)(I.g_y * I.dt);
    }
}

__global__ void k_inst_err(const Seg* __restrict__ segs, const double* __restrict__ part, const Inst* __restrict__ insts,
                           double* __restrict__ err_out) {
    __shared__ double sh[32];
    const Seg g = segs[blockIdx.x];
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    for (int t = g.begin + threadIdx.x; t < g.end; t += blockDim.x) {
        s0 += part[3 * t];
        s1 += part[3 * t + 1];
        s2 += part[3 * t + 2];
    }
    double a = blk_sum(s0, sh), b = blk_sum(s1, sh), c = blk_sum(s2, sh);
    if (threadIdx.x == 0) {
        const Inst& I = insts[g.inst];
        double nrx = (double)(I.Nx - 2) * (I.Ny - 1), nry = (double)(I.Nx - 1) * (I.Ny - 2),
               ndv = (double)(I.Nx - 1) * (I.Ny - 1);
        double m = a / nrx;
        double bb = b / nry, cc = c / ndv;
        if (bb > m || bb != bb) m = bb;
        if (cc > m || cc != cc) m = cc;
        if (a != a) m = a;
        err_out[blockIdx.x] = m;
    }
}

// V += dV, P += dP (FP64 += FP32) over an instance's padded arrays, then zero the correction.  The damped
// rates are kept: folding the correction into the FP64 state and re-anchoring the constant term on the FP64
// residual leaves the PT iteration itself unchanged (in exact arithmetic it is the FP64 iteration), so its
// accumulated momentum stays valid.  blockIdx.y = position in the instance list.
__global__ void k_accumulate(const Inst* __restrict__ insts, const int* __restrict__ list, int launch_parity) {
    const Inst& I = insts[list[blockIdx.y]];
    const int in = (I.parity ^ launch_parity) & 1;
    const int64_t n = I.LD32 * I.rows;  // every entry; the FP64 and FP32 fields share (i, j) -> i + j*LD
    float* cvx = gf(I, in ? G_VXB : G_VXA);
    float* cvy = gf(I, in ? G_VYB : G_VYA);
    float* cp = gf(I, in ? G_PB : G_PA);
    float* rvx = gf(I, G_RVX);
    float* rvy = gf(I, G_RVY);
    double* Vx = gd(I, D_VX);
    double* Vy = gd(I, D_VY);
    double* P = gd(I, D_P);
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = k % I.LD32, j = k / I.LD32;
        if (i < I.Nx && j < I.Ny + 1) Vx[k] += (double)cvx[k];
        if (i < I.Nx + 1 && j < I.Ny) Vy[k] += (double)cvy[k];
        if (i < I.Nx - 1 && j < I.Ny - 1) P[k] += (double)cp[k];
        cvx[k] = 0.f;
        cvy[k] = 0.f;
        cp[k] = 0.f;
    }
    (void)rvx;
    (void)rvy;
}

__global__ void k_f64_to_f32(float* __restrict__ dst, int64_t ld_dst, const double* __restrict__ src, int64_t ld_src,
                             int64_t nx, int64_t ny) {
    int64_t n = nx * ny;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        int64_t i = k % nx, j = k / nx;
        dst[i + j * ld_dst] = (float)src[i + j * ld_src];
    }
}

__global__ void k_copy64(double* __restrict__ dst, int64_t ld_dst, const double* __restrict__ src, int64_t ld_src,
                         int64_t nx, int64_t ny) {
    int64_t n = nx * ny;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        int64_t i = k % nx, j = k / nx;
        dst[i + j * ld_dst] = src[i + j * ld_src];
    }
}

__global__ void k_pad_vx64(double* __restrict__ pad, const double* __restrict__ Vx, int64_t LD, int Nx, int Ny) {
    int64_t W = Nx + 2, n = W * (Ny + 1);
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        int64_t i = k % W, j = k / W;
        pad[k] = (i == 0) ? -Vx[1 + j * LD] : (i == W - 1) ? -Vx[(Nx - 2) + j * LD] : Vx[(i - 1) + j * LD];
    }
}
__global__ void k_pad_vy64(double* __restrict__ pad, const double* __restrict__ Vy, int64_t LD, int Nx, int Ny) {
    int64_t W = Nx + 1, n = W * (Ny + 2);
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        int64_t i = k % W, j = k / W;
        pad[k] = (j == 0) ? -Vy[i + LD] : (j == Ny + 1) ? -Vy[i + (int64_t)(Ny - 2) * LD] : Vy[i + (j - 1) * LD];
    }
}

__global__ void k_rho_scale64(const double* __restrict__ rho, int Nx, int Ny, double g_y, double* __restrict__ out) {
    __shared__ double sh[32];
    int64_t W = Nx - 1, n = W * (Ny - 2);
    double s = 0.0;
    for (int64_t k = threadIdx.x; k < n; k += blockDim.x) {
        int64_t i = k % W + 1, j = k / W + 1;
        s += fabs(g_y * rho[i + j * (Nx + 1)]);
    }
    double t = blk_sum(s, sh);
    if (threadIdx.x == 0) *out = t / (double)n;
}

}  // namespace mx
}  // namespace sf

// ===========================================================================
// host side: the batch engine
// ===========================================================================
namespace sf {
namespace mx {

enum Phase { PH_OUTER = 0, PH_INNER = 1, PH_DONE = 2 };

struct HostInst {
    sf_batch_instance* user;
    Inst d;                  // device copy source
    int64_t tile0, ntiles;   // tiles of this instance in the full tile list
    int phase = PH_OUTER;
    int cur = 0;             // physical buffer (0 = A, 1 = B) holding the current correction
    int64_t inner_here = 0;  // FP32 sweeps in the current correction
    int64_t inner_total = 0;
    int64_t outer = 0;
    double err = 0.0, target = 0.0, eps = 0.0;
    bool accumulated = true; // nothing to add before the first residual
};

struct Engine {
    sf_ctx* ctx;
    cudaStream_t s;
    sf_mixed_options opt;
    std::vector<HostInst> in;
    // device
    Inst* d_insts = nullptr;
    CUtensorMap* d_maps = nullptr;
    int2* d_tiles = nullptr;
    int* d_ntiles = nullptr;
    double* d_part64 = nullptr;
    Seg* d_segs = nullptr;
    double* d_err = nullptr;
    int* d_list = nullptr;
    double* d_scale = nullptr;
    // host scratch (pinned)
    double* h_err = nullptr;
    int64_t total_tiles = 0;
    int h_ntiles = 0;         // host copy of the sweep tile count (source of an async upload)
    int64_t launches = 0;     // k_pt32 launches so far (their parity alternates)
    int pt_blocks = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    int graph_k = 0;

    ~Engine() {
        if (gexec) cudaGraphExecDestroy(gexec);
        if (graph) cudaGraphDestroy(graph);
    }

    int upload_inst(int b) {
        SF_CUDA(cudaMemcpyAsync(d_insts + b, &in[b].d, sizeof(Inst), cudaMemcpyHostToDevice, s));
        return SF_OK;
    }

    // tile list + segments of the instances in `ids`; returns the number of tiles
    int build_lists(const std::vector<int>& ids, int2* h_tiles, Seg* h_segs, int64_t* ntiles_out) {
        int64_t nt = 0;
        for (size_t q = 0; q < ids.size(); ++q) {
            const HostInst& h = in[ids[q]];
            h_segs[q] = Seg{ids[q], (int)nt, (int)(nt + h.ntiles), 0};
            for (int64_t k = 0; k < h.ntiles; ++k) h_tiles[nt++] = make_int2(ids[q], (int)k);
        }
        *ntiles_out = nt;
        return SF_OK;
    }
};

static unsigned grid1(int64_t n, int per) { return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + per - 1) / per, 65535)); }

}  // namespace mx
}  // namespace sf

using namespace sf;
using namespace sf::mx;

extern "C" int sf_solve_stokes_batch_mixed(sf_ctx* ctx, sf_batch_instance* inst, int n, const sf_mixed_options* o,
                                           void* stream) {
    SF_REQUIRE(ctx && inst && n >= 1, "sf_solve_stokes_batch_mixed: bad arguments");
    int rc = set_device(ctx);
    if (rc) return rc;
    Engine E;
    E.ctx = ctx;
    // the caller's inputs are ready once its stream is; the engine then works on the context's own
    // non-blocking stream, where graph capture is allowed, and synchronises it before returning
    SF_CUDA(cudaStreamSynchronize(as_stream(stream)));
    E.s = ctx->work;
    cudaStream_t s = E.s;
    E.opt = o ? *o : sf_mixed_options{};
    if (!o) {
        E.opt.max_sweeps = 4000000;
        E.opt.fold_every = 400;
        E.opt.use_graphs = 1;
    }
    if (E.opt.fold_every < 2) E.opt.fold_every = 2;
    E.opt.fold_every &= ~1;  // even: the current correction is back in the A buffers at every fold
    // ---- layout ----
    E.in.resize(n);
    int64_t bytes32 = 0, bytes64 = 0, ntiles = 0;
    for (int b = 0; b < n; ++b) {
        sf_batch_instance& u = inst[b];
        SF_REQUIRE(u.Nx >= 4 && u.Ny >= 4 && u.Nx < (1 << 20) && u.Ny < (1 << 20), "sf_solve_stokes_batch_mixed: bad grid");
        SF_REQUIRE(u.P && u.Vx_pad && u.Vy_pad && u.rho_vy && u.mu_b && u.mu_p && u.Vx_s && u.Vy_s,
                   "sf_solve_stokes_batch_mixed: NULL array");
        SF_REQUIRE(u.dx > 0 && u.dy > 0, "sf_solve_stokes_batch_mixed: dx, dy must be positive");
        HostInst& h = E.in[b];
        h.user = &u;
        Inst& I = h.d;
        memset(&I, 0, sizeof(I));
        I.Nx = (int)u.Nx;
        I.Ny = (int)u.Ny;
        I.ntx = (int)ceil_div(u.Nx - 1, BX);
        I.nty = (int)ceil_div(u.Ny - 1, BY);
        I.LD32 = I.LD64 = round_up(u.Nx + 4, 32);
        I.rows = u.Ny + 3;
        I.fstride32 = I.fstride64 = I.LD32 * I.rows;
        h.tile0 = ntiles;
        h.ntiles = (int64_t)I.ntx * I.nty;
        ntiles += h.ntiles;
        bytes32 += (int64_t)G_NUM * I.fstride32 * 4;
        bytes64 += (int64_t)D_NUM * I.fstride64 * 8;
        bytes32 = round_up(bytes32, 256);
        bytes64 = round_up(bytes64, 256);
    }
    E.total_tiles = ntiles;
    // one scratch block: FP32 arena | FP64 arena | maps | insts | tiles | partials | segs | err | list | scale
    const size_t off32 = 0, off64 = round_up(off32 + bytes32, 256);
    const size_t offmap = round_up(off64 + bytes64, 256);
    const size_t offins = round_up(offmap + (size_t)n * M_NUM * sizeof(CUtensorMap), 256);
    const size_t offtil = round_up(offins + (size_t)n * sizeof(Inst), 256);
    const size_t offnt = round_up(offtil + (size_t)ntiles * sizeof(int2), 256);
    const size_t offp32 = round_up(offnt + 256, 256);
    const size_t offp64 = round_up(offp32 + (size_t)ntiles * 3 * 4, 256);
    const size_t offseg = round_up(offp64 + (size_t)ntiles * 3 * 8, 256);
    const size_t offerr = round_up(offseg + (size_t)n * sizeof(Seg), 256);
    const size_t offlst = round_up(offerr + (size_t)n * 8, 256);
    const size_t offscl = round_up(offlst + (size_t)n * 4, 256);
    const size_t total = round_up(offscl + (size_t)n * 8, 256);
    if ((rc = ensure(ctx, ctx->mixed, total))) return rc;
    unsigned char* base = (unsigned char*)ctx->mixed.ptr;
    SF_CUDA(cudaMemsetAsync(base, 0, offmap, s));  // both arenas start at zero (corrections, rates, padding)
    E.d_maps = (CUtensorMap*)(base + offmap);
    E.d_insts = (Inst*)(base + offins);
    E.d_tiles = (int2*)(base + offtil);
    E.d_ntiles = (int*)(base + offnt);
    E.d_part64 = (double*)(base + offp64);
    E.d_segs = (Seg*)(base + offseg);
    E.d_err = (double*)(base + offerr);
    E.d_list = (int*)(base + offlst);
    E.d_scale = (double*)(base + offscl);
    std::vector<double> h_err_v(n), h_scale(n);
    // ---- per-instance fields, constants, maps ----
    std::vector<CUtensorMap> hmaps((size_t)n * M_NUM);
    int64_t o32 = 0, o64 = 0;
    const double Vdmp = 4.0, Vsc = 0.45, Ptsc = 0.5;
    for (int b = 0; b < n; ++b) {
        HostInst& h = E.in[b];
        sf_batch_instance& u = *h.user;
        Inst& I = h.d;
        I.f32 = (float*)(base + off32 + o32);
        I.f64 = (double*)(base + off64 + o64);
        o32 = round_up(o32 + (int64_t)G_NUM * I.fstride32 * 4, 256);
        o64 = round_up(o64 + (int64_t)D_NUM * I.fstride64 * 8, 256);
        const int64_t Nx = u.Nx, Ny = u.Ny, LD = I.LD64;
        const double mdxy = std::min(u.dx, u.dy);
        I.dx = u.dx;
        I.dy = u.dy;
        I._dx = 1.0 / u.dx;
        I._dy = 1.0 / u.dy;
        I.g_y = u.g_y;
        I.maxdisp = u.maxdisp;
        I.use_stab = u.use_free_surface_stabilization ? 1 : 0;
        I.dt_in = I.use_stab ? u.dt : 0.0;
        I.dt = I.dt_in;
        I._dxf = (float)I._dx;
        I._dyf = (float)I._dy;
        I.dampXf = (float)(1.0 - Vdmp / (double)Nx);
        I.dampYf = (float)(1.0 - Vdmp / (double)Ny);
        I.c_vscf = (float)(Vsc * mdxy * mdxy / 4.1);
        I.c_ptscf = (float)(Ptsc * 4.1 / (double)std::max(Nx, Ny));
        I.g_dtf = (float)(I.g_y * I.dt);
        // pack the caller's FP64 arrays
        double* f64 = I.f64;
        struct Pk { int f; const double* src; int64_t nx, ny; } packs[] = {
            {D_VX, u.Vx_s, Nx, Ny + 1}, {D_VY, u.Vy_s, Nx + 1, Ny}, {D_P, u.P, Nx - 1, Ny - 1},
            {D_RHO, u.rho_vy, Nx + 1, Ny}, {D_MUB, u.mu_b, Nx, Ny}, {D_MUP, u.mu_p, Nx - 1, Ny - 1}};
        for (const Pk& k : packs) {
            k_copy64<<<grid1(k.nx * k.ny, 256), 256, 0, s>>>(f64 + (int64_t)k.f * I.fstride64, LD, k.src, k.nx, k.nx, k.ny);
            SF_LAUNCHED(ctx);
        }
        struct Cv { int g, d; int64_t nx, ny; } cvs[] = {{G_MUB, D_MUB, Nx, Ny}, {G_MUP, D_MUP, Nx - 1, Ny - 1},
                                                           {G_RHO, D_RHO, Nx + 1, Ny}};
        for (const Cv& c : cvs) {
            k_f64_to_f32<<<grid1(c.nx * c.ny, 256), 256, 0, s>>>(I.f32 + (int64_t)c.g * I.fstride32, LD,
                                                                 f64 + (int64_t)c.d * I.fstride64, LD, c.nx, c.ny);
            SF_LAUNCHED(ctx);
        }
        if (u.rel_tol > 0) {
            k_rho_scale64<<<1, 1024, 0, s>>>(u.rho_vy, (int)Nx, (int)Ny, u.g_y, E.d_scale + b);
            SF_LAUNCHED(ctx);
        }
        // tensor maps (FP32 fields, LD x rows)
        const int gmap[M_NUM] = {G_VXA, G_VXB, G_VYA, G_VYB, G_PA, G_PB, G_MUB, G_MUP, G_RHO, G_RDIV,
                                 G_RVX, G_RVY, G_RX, G_RY};
        for (int m = 0; m < M_NUM; ++m) {
            const bool halo = m <= M_RDIV;
            if ((rc = encode_tmap_f32(&hmaps[(size_t)b * M_NUM + m], I.f32 + (int64_t)gmap[m] * I.fstride32, LD,
                                      I.rows, halo ? TW : BX, halo ? TH : BY)))
                return rc;
        }
    }
    SF_CUDA(cudaMemcpyAsync(E.d_maps, hmaps.data(), hmaps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice, s));
    SF_CUDA(cudaMemcpyAsync(h_scale.data(), E.d_scale, (size_t)n * 8, cudaMemcpyDeviceToHost, s));
    SF_CUDA(cudaStreamSynchronize(s));
    for (int b = 0; b < n; ++b) {
        HostInst& h = E.in[b];
        h.eps = h.user->rel_tol > 0 ? h.user->rel_tol * h_scale[b] : h.user->eps;
        if ((rc = E.upload_inst(b))) return rc;
    }
    static int per_sm = 0;
    if (!per_sm) {
        SF_CUDA(cudaFuncSetAttribute(k_pt32, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES));
        SF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pt32, NT, SMEM_BYTES));
        if (per_sm < 1) return fail(SF_ERR_CUDA, "k_pt32 does not fit on an SM");
    }
    SF_CUDA(cudaMemsetAsync(ctx->d_flags, 0, sizeof(int), s));
    std::vector<int2> h_tiles((size_t)ntiles);
    std::vector<Seg> h_segs(n);
    std::vector<int> ids;
    ids.reserve(n);
    cudaEvent_t e0 = ctx->ev_a, e1 = ctx->ev_b;
    SF_CUDA(cudaEventRecord(e0, s));

    // ---- the loop: an outer step (fold the correction into V, P -> dt -> FP64 residual) for every
    // instance still iterating, then K FP32 sweeps of all of them.  K is even, so each instance's
    // current correction stays in its A buffers at every fold (no buffer bookkeeping). ----
    const int K = E.opt.fold_every;
    const int blocks = (int)std::min<int64_t>(E.total_tiles, (int64_t)per_sm * ctx->num_sms);
    std::vector<int> sweep_ids_prev;
    bool first = true;
    while (true) {
        ids.clear();
        for (int b = 0; b < n; ++b)
            if (E.in[b].phase != PH_DONE) ids.push_back(b);
        if (ids.empty()) break;
        int64_t nt = 0;
        if (!first) {
            // fold: V += dV, P += dP for every instance that just swept
            SF_CUDA(cudaMemcpyAsync(E.d_list, ids.data(), ids.size() * 4, cudaMemcpyHostToDevice, s));
            k_accumulate<<<dim3(64, (unsigned)ids.size()), 256, 0, s>>>(E.d_insts, E.d_list, 0);
            SF_LAUNCHED(ctx);
        }
        E.build_lists(ids, h_tiles.data(), h_segs.data(), &nt);
        SF_CUDA(cudaMemcpyAsync(E.d_tiles, h_tiles.data(), nt * sizeof(int2), cudaMemcpyHostToDevice, s));
        SF_CUDA(cudaMemcpyAsync(E.d_segs, h_segs.data(), ids.size() * sizeof(Seg), cudaMemcpyHostToDevice, s));
        E.h_ntiles = (int)nt;
        SF_CUDA(cudaMemcpyAsync(E.d_ntiles, &E.h_ntiles, sizeof(int), cudaMemcpyHostToDevice, s));
        k_maxv64<<<(unsigned)nt, T64, 0, s>>>(E.d_insts, E.d_tiles, E.d_part64);
        SF_LAUNCHED(ctx);
        k_inst_dt<<<(unsigned)ids.size(), 256, 0, s>>>(E.d_insts, E.d_segs, E.d_part64);
        SF_LAUNCHED(ctx);
        k_resid64<<<(unsigned)nt, T64, 0, s>>>(E.d_insts, E.d_tiles, E.d_part64);
        SF_LAUNCHED(ctx);
        k_inst_err<<<(unsigned)ids.size(), 256, 0, s>>>(E.d_segs, E.d_part64, E.d_insts, E.d_err);
        SF_LAUNCHED(ctx);
        SF_CUDA(cudaMemcpyAsync(h_err_v.data(), E.d_err, ids.size() * 8, cudaMemcpyDeviceToHost, s));
        SF_CUDA(cudaStreamSynchronize(s));
        int flag = 0;
        SF_CUDA(cudaMemcpy(&flag, ctx->d_flags, sizeof(int), cudaMemcpyDeviceToHost));
        if (flag) return fail(SF_ERR_CUDA, "sf_solve_stokes_batch_mixed: a tile copy did not complete in time");
        first = false;
        std::vector<int> sweep;
        for (size_t q = 0; q < ids.size(); ++q) {
            HostInst& h = E.in[ids[q]];
            h.err = h_err_v[q];
            ++h.outer;
            const bool bad = !(h.err == h.err) || std::isinf(h.err);
            if (bad || h.err <= h.eps || h.inner_total >= E.opt.max_sweeps)
                h.phase = PH_DONE;
            else
                sweep.push_back(ids[q]);
        }
        if (sweep.empty()) continue;
        if (sweep != ids) {
            E.build_lists(sweep, h_tiles.data(), h_segs.data(), &nt);
            SF_CUDA(cudaMemcpyAsync(E.d_tiles, h_tiles.data(), nt * sizeof(int2), cudaMemcpyHostToDevice, s));
            E.h_ntiles = (int)nt;
            SF_CUDA(cudaMemcpyAsync(E.d_ntiles, &E.h_ntiles, sizeof(int), cudaMemcpyHostToDevice, s));
        }
        auto launch_run = [&]() -> int {
            for (int k = 0; k < K; ++k) {
                k_pt32<<<blocks, dim3(BX, TY), SMEM_BYTES, s>>>(E.d_maps, E.d_insts, E.d_tiles, E.d_ntiles, k & 1,
                                                                ctx->d_flags);
                SF_CHECK_LAUNCH();
            }
            return SF_OK;
        };
        if (E.opt.use_graphs) {
            if (!E.gexec) {
                SF_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
                int lrc = launch_run();
                cudaGraph_t g = nullptr;
                cudaError_t ce = cudaStreamEndCapture(s, &g);
                if (lrc) return lrc;
                SF_CUDA(ce);
                E.graph = g;
                SF_CUDA(cudaGraphInstantiate(&E.gexec, g, 0));
            }
            SF_CUDA(cudaGraphLaunch(E.gexec, s));
        } else {
            if ((rc = launch_run())) return rc;
        }
        ctx->launches += K;
        E.launches += K;
        for (int b : sweep) E.in[b].inner_total += K;
    }
    SF_CUDA(cudaEventRecord(e1, s));
    // the device-side instance records hold the last dt computed from the FP64 velocities
    std::vector<Inst> dev_inst(n);
    SF_CUDA(cudaMemcpyAsync(dev_inst.data(), E.d_insts, (size_t)n * sizeof(Inst), cudaMemcpyDeviceToHost, s));
    SF_CUDA(cudaStreamSynchronize(s));
    for (int b = 0; b < n; ++b) E.in[b].d.dt_cfl = dev_inst[b].dt_cfl;
    // ---- unpack (:89-95) ----
    for (int b = 0; b < n; ++b) {
        HostInst& h = E.in[b];
        sf_batch_instance& u = *h.user;
        const Inst& I = h.d;
        const int64_t Nx = u.Nx, Ny = u.Ny, LD = I.LD64;
        struct Uk { double* dst; int f; int64_t nx, ny; } ups[] = {
            {u.Vx_s, D_VX, Nx, Ny + 1}, {u.Vy_s, D_VY, Nx + 1, Ny}, {u.P, D_P, Nx - 1, Ny - 1}};
        for (const Uk& k : ups) {
            k_copy64<<<grid1(k.nx * k.ny, 256), 256, 0, s>>>(k.dst, k.nx, I.f64 + (int64_t)k.f * I.fstride64, LD, k.nx, k.ny);
            SF_LAUNCHED(ctx);
        }
        k_pad_vx64<<<grid1((Nx + 2) * (Ny + 1), 256), 256, 0, s>>>(u.Vx_pad, I.f64 + D_VX * I.fstride64, LD, (int)Nx, (int)Ny);
        SF_LAUNCHED(ctx);
        k_pad_vy64<<<grid1((Nx + 1) * (Ny + 2), 256), 256, 0, s>>>(u.Vy_pad, I.f64 + D_VY * I.fstride64, LD, (int)Nx, (int)Ny);
        SF_LAUNCHED(ctx);
        u.dt_out = I.dt_cfl;   // compute_dt of the final V (:95), from the last outer step
        u.err = h.err;
        u.inner_iters = h.inner_total;
        u.outer_iters = h.outer;
        u.converged = (h.err <= h.eps) ? 1 : 0;
        u.eps_used = h.eps;
        u.status = (h.err == h.err && !std::isinf(h.err)) ? SF_OK : SF_ERR_NONFINITE;
    }
    SF_CUDA(cudaStreamSynchronize(s));
    float ms = 0.f;
    SF_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    for (int b = 0; b < n; ++b) inst[b].batch_ms = ms;
    return SF_OK;
}

extern "C" int sf_solve_stokes_mixed(sf_ctx* ctx, double* P, double* Vx_pad, double* Vy_pad, const double* rho_vy,
                                     const double* mu_b, const double* mu_p, double* Vx_s, double* Vy_s, double g_y,
                                     double dx, double dy, int64_t Nx, int64_t Ny, double dt, double maxdisp,
                                     int use_stab, double eps, double rel_tol, const sf_mixed_options* opt,
                                     void* stream, sf_batch_instance* info) {
    sf_batch_instance u;
    memset(&u, 0, sizeof(u));
    u.P = P;
    u.Vx_pad = Vx_pad;
    u.Vy_pad = Vy_pad;
    u.rho_vy = rho_vy;
    u.mu_b = mu_b;
    u.mu_p = mu_p;
    u.Vx_s = Vx_s;
    u.Vy_s = Vy_s;
    u.Nx = Nx;
    u.Ny = Ny;
    u.g_y = g_y;
    u.dx = dx;
    u.dy = dy;
    u.dt = dt;
    u.maxdisp = maxdisp;
    u.eps = eps;
    u.rel_tol = rel_tol;
    u.use_free_surface_stabilization = use_stab;
    int rc = sf_solve_stokes_batch_mixed(ctx, &u, 1, opt, stream);
    if (info) *info = u;
    if (rc) return rc;
    return u.status;
}
