// sf_solve.cu -- pseudo-transient Stokes solve (scripts/StokesSolver_multixpu.jl)
// for libstokesflow_b200.so.
//
// The reference runs, per PT iteration, compute_P_tau! -> compute_dV! ->
// compute_V! -> four BC kernels (:48-57), with tau, divV, dtau* stored as full
// arrays.  Here one fused kernel does the whole iteration:
//
//   * the domain is cut into BX x BY tiles of points (i, j), 0 <= i < Nx-1,
//     0 <= j < Ny-1 (the pressure index space, which contains the dVx and dVy
//     index spaces); persistent CTAs (4 per SM) walk the tiles;
//   * one thread per CTA brings the next tile's old Vx, Vy, rho, P, mu_p, mu_b
//     (tile + 2 halo) and dVx, dVy (tile) into a second shared-memory stage
//     with bulk-tensor copies (TMA, mbarrier-completed) while the CTA computes
//     the current tile, so the HBM stream never waits for the arithmetic;
//   * per tile it computes P_new, tau_xx, tau_yy, tau_xy on the tile + 1 halo
//     (the halo row/column is recomputed by the neighbouring tile, cheaper
//     than a grid-wide barrier), then the residuals, the damped rates dV and
//     the new velocities of its tile;
//   * tau and divV are stored only on check iterations; dtauVx, dtauVy are
//     computed in the kernel from the staged mu_p with compute_timesteps!'s
//     expression (4 FP64 divisions per point cost less than streaming two
//     precomputed arrays, 16 B per point, and free the shared memory for a
//     fourth CTA per SM);
//   * the free-slip ghost rows / columns of the new velocities are written by
//     the CTAs on the domain edge, in the reference's BC order (:53-56);
//   * V and P are double-buffered (the iteration is Jacobi-like: every read is
//     an old value), dV is updated in place.
//
// HBM bytes per iteration: read Vx, Vy, P, dVx, dVy, rho, mu_b, mu_p and write
// Vx, Vy, P, dVx, dVy -- 13 arrays, ~104 * Nx * Ny bytes, which is all the
// kernel reads and writes.
//
// Fields live in a padded internal layout (one leading dimension LD, a
// multiple of 32 doubles, for every field) packed from / unpacked to the
// caller's Julia-layout arrays once per solve.  Every iteration on the check
// schedule additionally stores tau / divV and runs the residual + norm
// kernels; dt updates (every ndtupdate) run a max|V| reduction whose result
// stays on the device.  The only host synchronisation is the residual test.
//
// All floating-point expressions keep the reference's evaluation order and
// the file is compiled with -fmad=false: the iterates are bit-identical to
// the reference's (only the summation order inside the residual norm differs).
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <functional>
#include <vector>

#include "sf_internal.cuh"
#include "sf_tma.cuh"

namespace sf {

enum {
    F_VXA, F_VXB, F_VYA, F_VYB, F_PA, F_PB, F_DVX, F_DVY, F_RHO, F_MUB, F_MUP,
    F_TXX, F_TYY, F_TXY, F_DIV, F_RX, F_RY, F_NUM
};

struct Layout {
    int64_t Nx, Ny, LD, rows, fstride;
    double* base;
    double* f(int k) const { return base + (int64_t)k * fstride; }
};

struct PTParams {
    const double* __restrict__ Vx_in;
    const double* __restrict__ Vy_in;
    const double* __restrict__ P_in;
    double* __restrict__ Vx_out;
    double* __restrict__ Vy_out;
    double* __restrict__ P_out;
    double* __restrict__ dVx;
    double* __restrict__ dVy;
    const double* __restrict__ rho;
    const double* __restrict__ mub;
    const double* __restrict__ mup;
    double* __restrict__ txx;
    double* __restrict__ tyy;
    double* __restrict__ txy;
    double* __restrict__ divV;
    const double* __restrict__ dt_ptr;
    int Nx, Ny;
    int64_t LD;
    double _dx, _dy, g_y, dampX, dampY;
    double c_vsc;    // Vsc * min_dxy2            (StokesSolver_multixpu.jl:129)
    double c_ptsc;   // Ptsc * 4.1                (:131)
    double max_nxy;  // max(nx_g(), ny_g())       (:21)
    double inv_max_nxy;  // 1/max_nxy, used only when max_nxy is a power of two (then x/max == x*inv exactly)
    int pow2;
    int ntx, nty;        // tiles in x / y
    int* __restrict__ err_flag;  // set when a tile copy did not arrive in time
};

// ---------------------------------------------------------------------------
// fused PT iteration: persistent CTAs, TMA double-buffered tiles
// ---------------------------------------------------------------------------
// Each CTA walks tiles t = blockIdx.x, blockIdx.x + gridDim.x, ...  While it
// computes tile t from shared-memory stage s, one thread has already issued
// the bulk-tensor copies of tile t + gridDim.x into stage s^1, so HBM reads
// overlap the arithmetic without needing high occupancy.  A stage holds the
// old Vx, Vy, rho_vy, P, mu_p, mu_b boxes (tile + 2 halo; the TMA zero-fills
// beyond the arrays) and the dVx, dVy boxes (tile only).
// 32 x 8 tiles: 51 KB of shared memory per CTA, 4 CTAs per SM (32 x 16 tiles allowed 2 before the dtau
// arrays left the stage: same speed at 2048^2, 10% slower at 4096^2)
#ifndef SF_PT_BY
#define SF_PT_BY 8
#endif
#ifndef SF_PT_TY
#define SF_PT_TY 8
#endif
#ifndef SF_PT_STAGES
#define SF_PT_STAGES 2
#endif
constexpr int BX = 32, BY = SF_PT_BY, TY = SF_PT_TY;   // owned tile, threads (BX x TY)
constexpr int NST = SF_PT_STAGES;                      // shared-memory stages (tiles in flight + 1)
static_assert(NST >= 2 && NST <= 8, "2..8 pipeline stages");
static_assert(BY % TY == 0, "tile rows must be a multiple of the thread rows");
constexpr int PT_THREADS = BX * TY;
constexpr int PT_MIN_BLOCKS = (PT_THREADS >= 512) ? 2 : 4;
constexpr int TW = BX + 2, TH = BY + 2;      // staged box (tile + 2 halo); TW*8 is a multiple of 16 bytes
constexpr int W1 = BX + 1, H1 = BY + 1;      // P / tau points computed per tile (tile + 1 halo)
constexpr int RPT = BY / TY;                 // owned rows per thread
constexpr int ARR_BYTES = ((TH * TW * 8 + 127) / 128) * 128;
constexpr int DV_BYTES = ((BY * BX * 8 + 127) / 128) * 128;
constexpr int ST1_BYTES = ((H1 * W1 * 8 + 127) / 128) * 128;
constexpr int STAGE_BYTES = 6 * ARR_BYTES + 2 * DV_BYTES;         // + dVx, dVy boxes
constexpr uint32_t STAGE_TX = 6 * TH * TW * 8 + 2 * BY * BX * 8;  // bytes delivered per stage
constexpr int SMEM_BYTES = NST * STAGE_BYTES + 4 * ST1_BYTES + 64;
constexpr uint64_t WAIT_BUDGET_NS = 2000000000ull;                 // 2 s per stage wait
enum { S_VX = 0, S_VY, S_RHO, S_P, S_MUP, S_MUB };

struct TmaMaps {
    CUtensorMap f[6];  // S_* order
    CUtensorMap dvx, dvy;
};

template <bool STORE>
__global__ void __launch_bounds__(PT_THREADS, PT_MIN_BLOCKS) k_pt_iter(const __grid_constant__ TmaMaps maps,
                                                                      PTParams p) {
    extern __shared__ __align__(128) unsigned char smem[];
    typedef double Row1[W1];
    typedef double Row2[TW];
    typedef double RowD[BX];
    Row1* sPn = reinterpret_cast<Row1*>(smem + NST * STAGE_BYTES);
    Row1* sTxx = reinterpret_cast<Row1*>(smem + NST * STAGE_BYTES + ST1_BYTES);
    Row1* sTyy = reinterpret_cast<Row1*>(smem + NST * STAGE_BYTES + 2 * ST1_BYTES);
    Row1* sTxy = reinterpret_cast<Row1*>(smem + NST * STAGE_BYTES + 3 * ST1_BYTES);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + NST * STAGE_BYTES + 4 * ST1_BYTES);

    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * BX + tx;
    const int Nx = p.Nx, Ny = p.Ny, ntiles = p.ntx * p.nty;
    const int64_t LD = p.LD;
    const double _dx = p._dx, _dy = p._dy;

    if (tid == 0) {
        for (int k = 0; k < NST; ++k) mbar_init(&bar[k], 1);
        fence_mbar_init();
    }
    __syncthreads();
    auto issue = [&](int t, int s) {  // thread 0 only
        const int i0 = (t % p.ntx) * BX, j0 = (t / p.ntx) * BY;
        unsigned char* st = smem + s * STAGE_BYTES;
        mbar_arrive_expect_tx(&bar[s], STAGE_TX);
#pragma unroll
        for (int k = 0; k < 6; ++k) tma_load_2d(st + k * ARR_BYTES, &maps.f[k], &bar[s], i0, j0);
        tma_load_2d(st + 6 * ARR_BYTES, &maps.dvx, &bar[s], i0, j0);
        tma_load_2d(st + 6 * ARR_BYTES + DV_BYTES, &maps.dvy, &bar[s], i0, j0);
    };
    const int G = gridDim.x;
    int t = blockIdx.x;
    // prologue: the first NST-1 tiles of this CTA into stages 0 .. NST-2
    if (tid == 0)
        for (int k = 0; k < NST - 1; ++k)
            if (t + k * G < ntiles) issue(t + k * G, k);
    uint32_t phase = 0;  // bit s: parity of the next completion of stage s
    int s = 0;
    const double dt = *p.dt_ptr;
    for (; t < ntiles; t += G) {
        // refill the stage freed by the previous tile with the tile NST-1 ahead
        const int tn = t + (NST - 1) * G;
        if (tid == 0 && tn < ntiles) issue(tn, (s + NST - 1) % NST);
        // the timeout vote rides on the stage-1 barrier below: stage 1 writes shared memory only (and, in the
        // check variant, tau/divV, which a failed solve discards), so a thread whose copy did not land
        // computes garbage and nothing else before everyone leaves
        const bool ok = mbar_wait(&bar[s], (phase >> s) & 1u, WAIT_BUDGET_NS);
        phase ^= 1u << s;
        unsigned char* st = smem + s * STAGE_BYTES;
        Row2* sVx = reinterpret_cast<Row2*>(st + S_VX * ARR_BYTES);
        Row2* sVy = reinterpret_cast<Row2*>(st + S_VY * ARR_BYTES);
        Row2* sRho = reinterpret_cast<Row2*>(st + S_RHO * ARR_BYTES);
        Row2* sPo = reinterpret_cast<Row2*>(st + S_P * ARR_BYTES);
        Row2* sMup = reinterpret_cast<Row2*>(st + S_MUP * ARR_BYTES);
        Row2* sMub = reinterpret_cast<Row2*>(st + S_MUB * ARR_BYTES);
        RowD* sDvx = reinterpret_cast<RowD*>(st + 6 * ARR_BYTES);
        RowD* sDvy = reinterpret_cast<RowD*>(st + 6 * ARR_BYTES + DV_BYTES);
        const int i0 = (t % p.ntx) * BX, j0 = (t / p.ntx) * BY;
        // interior tiles: every point of the tile and its halo is inside, no boundary node among them
        const bool interior = i0 > 0 && j0 > 0 && i0 + BX + 2 < Nx && j0 + BY + 2 < Ny;

        // ---- stage 1: compute_P_tau! (:140-169) on tile + 1 halo ----
        // the (BX+1) x (BY+1) points are spread evenly over all threads, row by row
        for (int idx = tid; idx < W1 * H1; idx += PT_THREADS) {
            {
                const int b = idx / W1, a = idx - b * W1;
                const int i = i0 + a, j = j0 + b;
                if (interior || (i < Nx - 1 && j < Ny - 1)) {
                    double vx1 = sVx[b + 1][a], vx2 = sVx[b + 1][a + 1];
                    double vy1 = sVy[b][a + 1], vy2 = sVy[b + 1][a + 1];
                    double dVx_dx = (vx2 - vx1) * _dx;
                    double dVy_dy = (vy2 - vy1) * _dy;
                    double div_V = dVx_dx + dVy_dy;
                    double mu = sMup[b][a];
                    // Ptsc*4.1*mu_p/max_nxy (:131); for a power-of-two max_nxy the product by its
                    // reciprocal is the same correctly rounded value
                    double dtP = p.pow2 ? p.c_ptsc * mu * p.inv_max_nxy : p.c_ptsc * mu / p.max_nxy;
                    sPn[b][a] = sPo[b][a] - dtP * div_V;
                    double txx = 2.0 * mu * (dVx_dx - 1.0 / 3.0 * div_V);
                    double tyy = 2.0 * mu * (dVy_dy - 1.0 / 3.0 * div_V);
                    sTxx[b][a] = txx;
                    sTyy[b][a] = tyy;
                    if (STORE && a < BX && b < BY) {
                        int64_t o = i + (int64_t)j * LD;
                        p.divV[o] = div_V;
                        p.txx[o] = txx;
                        p.tyy[o] = tyy;
                    }
                }
                if (interior || (i < Nx && j < Ny)) {
                    double vx0 = sVx[b][a], vx1 = sVx[b + 1][a];
                    double vy0 = sVy[b][a], vy1 = sVy[b][a + 1];
                    double dVx_dy = (vx1 - vx0) * _dy;
                    double dVy_dx = (vy1 - vy0) * _dx;
                    double tv = 2.0 * sMub[b][a] * 0.5 * (dVx_dy + dVy_dx);
                    sTxy[b][a] = tv;
                    if (STORE && (a < BX || i == Nx - 1) && (b < BY || j == Ny - 1)) p.txy[i + (int64_t)j * LD] = tv;
                }
            }
        }
        if (__syncthreads_or(!ok)) {
            // a copy never completed: flag it, give every copy still in flight a bounded chance to land, leave
            if (tid == 0) {
                atomicExch(p.err_flag, 1);
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

        // ---- stage 2: compute_dV! (:209-219), compute_V! (:226-234), BCs (:53-56) ----
        // offsets are taken from the tile corner (i0, j0); in-tile offsets fit 32 bits
        const int64_t tbase = i0 + (int64_t)j0 * LD;
        const int ldi = (int)LD;
        double* const P_t = p.P_out + tbase;
        double* const dVx_t = p.dVx + tbase;
        double* const dVy_t = p.dVy + tbase;
        double* const Vx_t = p.Vx_out + tbase;
        double* const Vy_t = p.Vy_out + tbase;
        auto new_vx = [&](int a, int b, int o) {
            // compute_ResX (:176-182)
            double Rx = (sTxx[b][a + 1] - sTxx[b][a]) * _dx + (sTxy[b + 1][a + 1] - sTxy[b][a + 1]) * _dy
                        - (sPn[b][a + 1] - sPn[b][a]) * _dx;
            double dv = p.dampX * sDvx[b][a] + Rx;
            dVx_t[o] = dv;
            const double dtau = p.c_vsc / ((sMup[b][a] + sMup[b][a + 1]) * 0.5) / 4.1;  // dtauVx (:129)
            return sVx[b + 1][a + 1] + dtau * dv;
        };
        auto new_vy = [&](int a, int b, int o) {
            // compute_ResY (:189-202)
            double av_inn_y_Vx = 0.25 * (sVx[b + 1][a] + sVx[b + 1][a + 1] + sVx[b + 2][a] + sVx[b + 2][a + 1]);
            double d_xi_2_rho = sRho[b + 1][a + 2] - sRho[b + 1][a];
            double d_yi_2_rho = sRho[b + 2][a + 1] - sRho[b][a + 1];
            double Ry = (sTyy[b + 1][a] - sTyy[b][a]) * _dy + (sTxy[b + 1][a + 1] - sTxy[b + 1][a]) * _dx
                        - (sPn[b + 1][a] - sPn[b][a]) * _dy
                        + p.g_y * (sRho[b + 1][a + 1] - dt * (av_inn_y_Vx * d_xi_2_rho * 0.5 * _dx
                                                               + sVy[b + 1][a + 1] * d_yi_2_rho * 0.5 * _dy));
            double dv = p.dampY * sDvy[b][a] + Ry;
            dVy_t[o] = dv;
            const double dtau = p.c_vsc / ((sMup[b][a] + sMup[b + 1][a]) * 0.5) / 4.1;  // dtauVy (:130)
            return sVy[b + 1][a + 1] + dtau * dv;
        };
        if (interior) {
#pragma unroll
            for (int r = 0; r < RPT; ++r) {
                const int a = tx, b = ty + r * TY;
                const int o = a + b * ldi;
                P_t[o] = sPn[b][a];
                Vx_t[o + 1 + ldi] = new_vx(a, b, o);
                Vy_t[o + 1 + ldi] = new_vy(a, b, o);
            }
        } else {
#pragma unroll
            for (int r = 0; r < RPT; ++r) {
                const int a = tx, b = ty + r * TY;
                const int i = i0 + a, j = j0 + b;
                if (i >= Nx - 1 || j >= Ny - 1) continue;
                const int o = a + b * ldi;
                P_t[o] = sPn[b][a];
                if (i < Nx - 2) {
                    double vn = new_vx(a, b, o);
                    Vx_t[o + 1 + ldi] = vn;
                    if (j == 0) Vx_t[o + 1] = vn;                                       // bc_y_noflux!
                    if (j == Ny - 2) Vx_t[o + 1 + 2 * ldi] = vn;
                }
                if (j < Ny - 2) {
                    double vn = new_vy(a, b, o);
                    Vy_t[o + 1 + ldi] = vn;
                    if (i == 0) Vy_t[o + ldi] = vn;                                     // bc_x_noflux!
                    if (i == Nx - 2) Vy_t[o + 2 + ldi] = vn;
                }
                // constant free-slip entries: bc_x_zero!(Vx) and bc_y_zero!(Vy), corners included
                if (i == 0 || i == Nx - 2) {
                    int ac = (i == 0) ? -i0 : Nx - 1 - i0;
                    Vx_t[ac + (b + 1) * ldi] = 0.0;
                    if (j == 0) Vx_t[ac - j0 * ldi] = 0.0;
                    if (j == Ny - 2) Vx_t[ac + (Ny - j0) * ldi] = 0.0;
                }
                if (j == 0 || j == Ny - 2) {
                    int br = (j == 0) ? -j0 : Ny - 1 - j0;
                    Vy_t[(a + 1) + br * ldi] = 0.0;
                    if (i == 0) Vy_t[-i0 + br * ldi] = 0.0;
                    if (i == Nx - 2) Vy_t[Nx - i0 + br * ldi] = 0.0;
                }
            }
        }
        __syncthreads();  // stage s and the stage-1 arrays are free again
        s = (s + 1 == NST) ? 0 : s + 1;
    }
}

// ---------------------------------------------------------------------------
// residuals + norms (compute_Residuals! :241-249, compute_err :103-109)
// ---------------------------------------------------------------------------
constexpr int RES_THREADS = 256;

__device__ __forceinline__ double block_sum(double v, double* sh) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    double r = 0.0;
    if (warp == 0) {
        r = (lane < (int)(blockDim.x >> 5)) ? sh[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
    }
    __syncthreads();
    return r;  // valid in thread 0
}

struct ResParams {
    const double* __restrict__ txx;
    const double* __restrict__ tyy;
    const double* __restrict__ txy;
    const double* __restrict__ P;
    const double* __restrict__ rho;
    const double* __restrict__ Vx;
    const double* __restrict__ Vy;
    const double* __restrict__ divV;
    const double* __restrict__ dt_ptr;
    double* __restrict__ Rx;
    double* __restrict__ Ry;
    double* __restrict__ partials;  // [gridDim.x][3]
    int Nx, Ny;
    int64_t LD;
    double _dx, _dy, g_y;
};

__global__ void __launch_bounds__(RES_THREADS) k_residuals(ResParams p) {
    __shared__ double sh[32];
    const int Nx = p.Nx, Ny = p.Ny;
    const int64_t LD = p.LD, W = Nx - 1, npts = (int64_t)(Nx - 1) * (Ny - 1);
    const double dt = *p.dt_ptr, _dx = p._dx, _dy = p._dy;
    double srx = 0.0, sry = 0.0, sdv = 0.0;
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < npts; n += (int64_t)gridDim.x * blockDim.x) {
        int i = (int)(n % W), j = (int)(n / W);
        int64_t o = i + (int64_t)j * LD;
        sdv += fabs(p.divV[o]);
        if (i < Nx - 2) {
            double Rx = (p.txx[o + 1] - p.txx[o]) * _dx + (p.txy[o + 1 + LD] - p.txy[o + 1]) * _dy
                        - (p.P[o + 1] - p.P[o]) * _dx;
            p.Rx[o] = Rx;
            srx += fabs(Rx);
        }
        if (j < Ny - 2) {
            double av = 0.25 * (p.Vx[o + LD] + p.Vx[o + 1 + LD] + p.Vx[o + 2 * LD] + p.Vx[o + 1 + 2 * LD]);
            double dxr = p.rho[o + 2 + LD] - p.rho[o + LD];
            double dyr = p.rho[o + 1 + 2 * LD] - p.rho[o + 1];
            double Ry = (p.tyy[o + LD] - p.tyy[o]) * _dy + (p.txy[o + 1 + LD] - p.txy[o + LD]) * _dx
                        - (p.P[o + LD] - p.P[o]) * _dy
                        + p.g_y * (p.rho[o + 1 + LD] - dt * (av * dxr * 0.5 * _dx + p.Vy[o + 1 + LD] * dyr * 0.5 * _dy));
            p.Ry[o] = Ry;
            sry += fabs(Ry);
        }
    }
    double a = block_sum(srx, sh), b = block_sum(sry, sh), c = block_sum(sdv, sh);
    if (threadIdx.x == 0) {
        p.partials[blockIdx.x * 3 + 0] = a;
        p.partials[blockIdx.x * 3 + 1] = b;
        p.partials[blockIdx.x * 3 + 2] = c;
    }
}

// single block: sum partials in a fixed order; err = max of the three means
__global__ void k_err_finalize(const double* __restrict__ partials, int nblocks, int64_t nrx, int64_t nry,
                               int64_t ndv, double* __restrict__ scalars) {
    __shared__ double sh[32];
    double s[3] = {0.0, 0.0, 0.0};
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
#pragma unroll
        for (int k = 0; k < 3; ++k) s[k] += partials[b * 3 + k];
    double t0 = block_sum(s[0], sh), t1 = block_sum(s[1], sh), t2 = block_sum(s[2], sh);
    if (threadIdx.x == 0) {
        double a = t0 / (double)nrx, b = t1 / (double)nry, c = t2 / (double)ndv;
        double m = a;
        if (b > m || b != b) m = b;
        if (c > m || c != c) m = c;
        if (a != a) m = a;
        scalars[SC_SUM_RX] = t0;
        scalars[SC_SUM_RY] = t1;
        scalars[SC_SUM_DIV] = t2;
        scalars[SC_ERR] = m;
    }
}

// ---------------------------------------------------------------------------
// max|V| and compute_dt (:118-121)
// ---------------------------------------------------------------------------
__global__ void k_maxabs_v(const double* __restrict__ Vx, const double* __restrict__ Vy, int Nx, int Ny, int64_t LD,
                           unsigned long long* __restrict__ out /* [2] as bits */) {
    __shared__ unsigned long long sh[2][32];
    unsigned long long mx = 0, my = 0;
    const int64_t nvx = (int64_t)Nx * (Ny + 1), nvy = (int64_t)(Nx + 1) * Ny;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nvx; n += stride) {
        int64_t i = n % Nx, j = n / Nx;
        unsigned long long b = (unsigned long long)__double_as_longlong(fabs(Vx[i + j * LD]));
        mx = b > mx ? b : mx;
    }
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nvy; n += stride) {
        int64_t i = n % (Nx + 1), j = n / (Nx + 1);
        unsigned long long b = (unsigned long long)__double_as_longlong(fabs(Vy[i + j * LD]));
        my = b > my ? b : my;
    }
    // non-negative doubles (and +NaN, which sorts above +Inf) order like their bit patterns
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long a = __shfl_down_sync(0xffffffffu, mx, o), c = __shfl_down_sync(0xffffffffu, my, o);
        mx = a > mx ? a : mx;
        my = c > my ? c : my;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) { sh[0][warp] = mx; sh[1][warp] = my; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
            mx = sh[0][w] > mx ? sh[0][w] : mx;
            my = sh[1][w] > my ? sh[1][w] : my;
        }
        atomicMax(&out[0], mx);
        atomicMax(&out[1], my);
    }
}

// dt = maxdisp * min(dx / max|Vx|, dy / max|Vy|); written to every slot in mask
__global__ void k_dt_finalize(const unsigned long long* __restrict__ maxbits, double maxdisp, double dx, double dy,
                              double* __restrict__ scalars, int slot_a, int slot_b) {
    double mvx = __longlong_as_double((long long)maxbits[0]);
    double mvy = __longlong_as_double((long long)maxbits[1]);
    double a = dx / mvx, b = dy / mvy;
    double m = (b < a) ? b : a;
    if (a != a) m = a;
    if (b != b) m = b;
    double dt = maxdisp * m;
    scalars[SC_MAX_VX] = mvx;
    scalars[SC_MAX_VY] = mvy;
    if (slot_a >= 0) scalars[slot_a] = dt;
    if (slot_b >= 0) scalars[slot_b] = dt;
}

__global__ void k_set_scalar(double* __restrict__ p, double v) { *p = v; }

// ---------------------------------------------------------------------------
// pack / unpack between the caller's Julia-layout arrays and the padded layout
// ---------------------------------------------------------------------------
__global__ void k_copy2d(double* __restrict__ dst, int64_t ld_dst, const double* __restrict__ src, int64_t ld_src,
                         int64_t nx, int64_t ny) {
    int64_t n = nx * ny;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        int64_t i = k % nx, j = k / nx;
        dst[i + j * ld_dst] = src[i + j * ld_src];
    }
}

// Vx_pad[2:end-1, :] = Vx_s; Vx_pad[1,:] = -Vx_pad[3,:]; Vx_pad[end,:] = -Vx_pad[end-2,:] (:89-92, :278-282)
__global__ void k_pad_vx(double* __restrict__ pad, const double* __restrict__ Vx, int64_t LD, int Nx, int Ny) {
    int64_t W = Nx + 2, n = W * (Ny + 1);
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        int64_t i = k % W, j = k / W;
        double v;
        if (i == 0) v = -Vx[1 + j * LD];
        else if (i == W - 1) v = -Vx[(Nx - 2) + j * LD];
        else v = Vx[(i - 1) + j * LD];
        pad[k] = v;
    }
}

// Vy_pad[:, 2:end-1] = Vy_s; Vy_pad[:,1] = -Vy_pad[:,3]; Vy_pad[:,end] = -Vy_pad[:,end-2] (:90-92, :309-313)
__global__ void k_pad_vy(double* __restrict__ pad, const double* __restrict__ Vy, int64_t LD, int Nx, int Ny) {
    int64_t W = Nx + 1, n = W * (Ny + 2);
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        int64_t i = k % W, j = k / W;
        double v;
        if (j == 0) v = -Vy[i + 1 * LD];
        else if (j == Ny + 1) v = -Vy[i + (int64_t)(Ny - 2) * LD];
        else v = Vy[i + (j - 1) * LD];
        pad[k] = v;
    }
}

// compute_timesteps! (:128-133): dtVx (Nx-2,Ny-1), dtVy (Nx-1,Ny-2), dtPt (Nx-1,Ny-1) with leading
// dimensions ld_x, ld_y, ld_p (the caller's dense arrays, or the padded internal ones); NULL skips one
__global__ void k_timesteps(const double* __restrict__ mup, int64_t LD, int Nx, int Ny, double c_vsc, double c_ptsc,
                            double max_nxy, double* __restrict__ dtVx, int64_t ld_x, double* __restrict__ dtVy,
                            int64_t ld_y, double* __restrict__ dtPt, int64_t ld_p) {
    int64_t W = Nx - 1, n = W * (Ny - 1);
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        int i = (int)(k % W), j = (int)(k / W);
        int64_t o = i + (int64_t)j * LD;
        if (dtVx && i < Nx - 2) dtVx[i + (int64_t)j * ld_x] = c_vsc / ((mup[o] + mup[o + 1]) * 0.5) / 4.1;
        if (dtVy && j < Ny - 2) dtVy[i + (int64_t)j * ld_y] = c_vsc / ((mup[o] + mup[o + LD]) * 0.5) / 4.1;
        if (dtPt) dtPt[i + (int64_t)j * ld_p] = c_ptsc * mup[o] / max_nxy;
    }
}

// mean |g_y * rho_vy| over the Ry interior rho_vy[2:Nx, 2:Ny-1] (1-based)
__global__ void k_rho_scale(const double* __restrict__ rho, int Nx, int Ny, double g_y, double* __restrict__ partials) {
    __shared__ double sh[32];
    int64_t W = Nx - 1, n = W * (Ny - 2);
    double s = 0.0;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        int64_t i = k % W + 1, j = k / W + 1;
        s += fabs(g_y * rho[i + j * (Nx + 1)]);
    }
    double t = block_sum(s, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = t;
}

__global__ void k_sum_partials(const double* __restrict__ partials, int n, double div, double* __restrict__ out) {
    __shared__ double sh[32];
    double s = 0.0;
    for (int b = threadIdx.x; b < n; b += blockDim.x) s += partials[b];
    double t = block_sum(s, sh);
    if (threadIdx.x == 0) *out = t / div;
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static unsigned copy_blocks(sf_ctx* ctx, int64_t n) {
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(ceil_div(n, 256), (int64_t)ctx->num_sms * 16));
}

// cuTensorMapEncodeTiled through the runtime's driver entry point
typedef CUresult (*PFN_encodeTiled)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                    const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                    CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static int encode_tmap(CUtensorMap* map, CUtensorMapDataType dtype, int esize, const void* base, int64_t ld,
                       int64_t rows, int box_w, int box_h);

int encode_tmap_f64(CUtensorMap* map, const double* base, int64_t ld, int64_t rows, int box_w, int box_h) {
    return encode_tmap(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, base, ld, rows, box_w, box_h);
}

int encode_tmap_f32(CUtensorMap* map, const float* base, int64_t ld, int64_t rows, int box_w, int box_h) {
    return encode_tmap(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, base, ld, rows, box_w, box_h);
}

static int get_encoder(PFN_encodeTiled* out) {
    static PFN_encodeTiled fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        SF_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || !p)
            return fail(SF_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
        fn = (PFN_encodeTiled)p;
    }
    *out = fn;
    return SF_OK;
}

// rank 2 (a field of rows x ld elements) or rank 3 (nfields such fields, fstride elements apart); box depth 1
static int encode_tiled(CUtensorMap* map, CUtensorMapDataType dtype, int esize, const void* base, int64_t ld,
                        int64_t rows, int64_t nfields, int64_t fstride, int box_w, int box_h) {
    PFN_encodeTiled fn = nullptr;
    int rc = get_encoder(&fn);
    if (rc) return rc;
    const cuuint32_t rank = nfields > 0 ? 3 : 2;
    cuuint64_t dims[3] = {(cuuint64_t)ld, (cuuint64_t)rows, (cuuint64_t)(nfields > 0 ? nfields : 1)};
    cuuint64_t strides[2] = {(cuuint64_t)ld * (cuuint64_t)esize, (cuuint64_t)fstride * (cuuint64_t)esize};
    cuuint32_t box[3] = {(cuuint32_t)box_w, (cuuint32_t)box_h, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = fn(map, dtype, rank, (void*)base, dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(SF_ERR_CUDA, "cuTensorMapEncodeTiled failed (code " + std::to_string((int)r) + ")");
    return SF_OK;
}

static int encode_tmap(CUtensorMap* map, CUtensorMapDataType dtype, int esize, const void* base, int64_t ld,
                       int64_t rows, int box_w, int box_h) {
    return encode_tiled(map, dtype, esize, base, ld, rows, 0, 0, box_w, box_h);
}

int encode_tmap_f32_fields(CUtensorMap* map, const float* base, int64_t ld, int64_t rows, int64_t nfields,
                           int64_t fstride, int box_w, int box_h) {
    return encode_tiled(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, base, ld, rows, nfields, fstride, box_w, box_h);
}

struct Solver {
    sf_ctx* ctx;
    cudaStream_t s;
    Layout L;
    PTParams pt;
    ResParams rp;
    TmaMaps maps[2];  // [cur]: inputs read from the A (cur = 0) or B (cur = 1) buffers
    int cur = 0;      // 0: current V/P in A buffers, 1: in B buffers
    int res_blocks = 0;
    int maxv_blocks = 0;
    int pt_blocks = 0;
    double maxdisp, dx, dy;

    int setup_maps() {
        const int64_t LD = L.LD, R = L.rows;
        for (int c = 0; c < 2; ++c) {
            const int fields[6] = {c ? F_VXB : F_VXA, c ? F_VYB : F_VYA, F_RHO, c ? F_PB : F_PA, F_MUP, F_MUB};
            for (int k = 0; k < 6; ++k) {
                int rc = encode_tmap_f64(&maps[c].f[k], L.f(fields[k]), LD, R, TW, TH);
                if (rc) return rc;
            }
            int rc = encode_tmap_f64(&maps[c].dvx, L.f(F_DVX), LD, R, BX, BY);
            if (!rc) rc = encode_tmap_f64(&maps[c].dvy, L.f(F_DVY), LD, R, BX, BY);
            if (rc) return rc;
        }
        static bool attr_set = false;
        if (!attr_set) {
            SF_CUDA(cudaFuncSetAttribute(k_pt_iter<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES));
            SF_CUDA(cudaFuncSetAttribute(k_pt_iter<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES));
            attr_set = true;
        }
        static int per_sm = 0;
        if (!per_sm) {
            SF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pt_iter<false>, PT_THREADS, SMEM_BYTES));
            if (per_sm < 1) return fail(SF_ERR_CUDA, "k_pt_iter does not fit on an SM");
        }
        pt.ntx = (int)ceil_div(L.Nx - 1, BX);
        pt.nty = (int)ceil_div(L.Ny - 1, BY);
        pt_blocks = (int)std::min<int64_t>((int64_t)pt.ntx * pt.nty, (int64_t)per_sm * ctx->num_sms);
        return SF_OK;
    }

    int launch_iter(bool store) {
        pt.Vx_out = L.f(cur ? F_VXA : F_VXB);
        pt.Vy_out = L.f(cur ? F_VYA : F_VYB);
        pt.P_out = L.f(cur ? F_PA : F_PB);
        dim3 block(BX, TY);
        if (store)
            k_pt_iter<true><<<pt_blocks, block, SMEM_BYTES, s>>>(maps[cur], pt);
        else
            k_pt_iter<false><<<pt_blocks, block, SMEM_BYTES, s>>>(maps[cur], pt);
        SF_LAUNCHED(ctx);
        cur ^= 1;
        return SF_OK;
    }

    const double* Vx_cur() const { return L.f(cur ? F_VXB : F_VXA); }
    const double* Vy_cur() const { return L.f(cur ? F_VYB : F_VYA); }
    const double* P_cur() const { return L.f(cur ? F_PB : F_PA); }

    int compute_dt(int slot_a, int slot_b) {
        unsigned long long* bits = (unsigned long long*)(ctx->d_scalars + SC_MAXBITS);
        SF_CUDA(cudaMemsetAsync(bits, 0, 2 * sizeof(unsigned long long), s));
        k_maxabs_v<<<maxv_blocks, 256, 0, s>>>(Vx_cur(), Vy_cur(), (int)L.Nx, (int)L.Ny, L.LD, bits);
        SF_LAUNCHED(ctx);
        k_dt_finalize<<<1, 1, 0, s>>>(bits, maxdisp, dx, dy, ctx->d_scalars, slot_a, slot_b);
        SF_LAUNCHED(ctx);
        return SF_OK;
    }

    int residuals() {
        rp.P = P_cur();
        rp.Vx = Vx_cur();
        rp.Vy = Vy_cur();
        k_residuals<<<res_blocks, RES_THREADS, 0, s>>>(rp);
        SF_LAUNCHED(ctx);
        int64_t Nx = L.Nx, Ny = L.Ny;
        k_err_finalize<<<1, 1024, 0, s>>>(rp.partials, res_blocks, (Nx - 2) * (Ny - 1), (Nx - 1) * (Ny - 2),
                                          (Nx - 1) * (Ny - 1), ctx->d_scalars);
        SF_LAUNCHED(ctx);
        return SF_OK;
    }
};

// the caller's arrays of one solve, in sf_solve_stokes's order (the work arrays may be NULL)
struct SolveArgs {
    double *P, *Vx_pad, *Vy_pad;
    const double *rho_vy, *mu_b, *mu_p;
    double *txx, *tyy, *txy, *divV, *dtPt, *Rx, *Ry, *dVxdt, *dVydt, *dtVx, *dtVy, *Vx_s, *Vy_s;
};

// Layout, scratch, pack, compute_timesteps! and kernel parameters of one (local) grid of Nx x Ny points.
// nx_g, ny_g are the global grid sizes the reference's constants use (nx_g(), ny_g(): :20-22): the local
// ones on a single domain.
static int solver_prepare(Solver& S, sf_ctx* ctx, cudaStream_t s, const SolveArgs& A, int64_t Nx, int64_t Ny,
                          double g_y, double dx, double dy, double dt, double maxdisp, int use_stab, int64_t nx_g,
                          int64_t ny_g) {
    int rc;
    S.ctx = ctx;
    S.s = s;
    S.L.Nx = Nx;
    S.L.Ny = Ny;
    S.L.LD = round_up(Nx + 2, 32);
    S.L.rows = Ny + 3;
    S.L.fstride = S.L.LD * S.L.rows;
    size_t fbytes = (size_t)S.L.fstride * 8 * F_NUM;
    bool fresh = fbytes > ctx->fields.bytes;
    if ((rc = ensure(ctx, ctx->fields, fbytes))) return rc;
    S.L.base = (double*)ctx->fields.ptr;
    if (fresh) SF_CUDA(cudaMemsetAsync(ctx->fields.ptr, 0, ctx->fields.bytes, s));
    S.res_blocks = (int)std::min<int64_t>(ceil_div((Nx - 1) * (Ny - 1), RES_THREADS), (int64_t)ctx->num_sms * 8);
    S.maxv_blocks = (int)std::min<int64_t>(ceil_div(Nx * (Ny + 1), 256), (int64_t)ctx->num_sms * 8);
    if ((rc = ensure(ctx, ctx->partials, (size_t)S.res_blocks * 3 * 8))) return rc;
    S.maxdisp = maxdisp;
    S.dx = dx;
    S.dy = dy;

    // ---- constants (:17-27) ----
    const double Vdmp = 4.0, Vsc = 0.45, Ptsc = 1.0 / 2.0;
    const double mdxy = std::min(dx, dy);
    const double min_dxy2 = mdxy * mdxy;
    const double max_nxy = (double)std::max(nx_g, ny_g);
    const double dampX = 1.0 - Vdmp / (double)nx_g;
    const double dampY = 1.0 - Vdmp / (double)ny_g;
    if (!use_stab) dt = 0.0;  // :29-31

    // ---- pack ----
    const int64_t LD = S.L.LD;
    struct Pk { int f; const double* src; int64_t nx, ny; } packs[] = {
        {F_VXA, A.Vx_s, Nx, Ny + 1}, {F_VYA, A.Vy_s, Nx + 1, Ny}, {F_PA, A.P, Nx - 1, Ny - 1},
        {F_DVX, A.dVxdt, Nx - 2, Ny - 1}, {F_DVY, A.dVydt, Nx - 1, Ny - 2}, {F_RHO, A.rho_vy, Nx + 1, Ny},
        {F_MUB, A.mu_b, Nx, Ny}, {F_MUP, A.mu_p, Nx - 1, Ny - 1}};
    for (const Pk& k : packs) {
        k_copy2d<<<copy_blocks(ctx, k.nx * k.ny), 256, 0, s>>>(S.L.f(k.f), LD, k.src, k.nx, k.nx, k.ny);
        SF_LAUNCHED(ctx);
    }
    k_set_scalar<<<1, 1, 0, s>>>(ctx->d_scalars + SC_DT, dt);
    SF_LAUNCHED(ctx);
    // compute_timesteps! (:34) into the caller's work arrays, if given; the fused kernel computes the same
    // pseudo-time steps from the staged mu_p as it needs them
    if (A.dtVx || A.dtVy || A.dtPt) {
        k_timesteps<<<copy_blocks(ctx, (Nx - 1) * (Ny - 1)), 256, 0, s>>>(S.L.f(F_MUP), LD, (int)Nx, (int)Ny,
                                                                         Vsc * min_dxy2, Ptsc * 4.1, max_nxy,
                                                                         A.dtVx, Nx - 2, A.dtVy, Nx - 1, A.dtPt,
                                                                         Nx - 1);
        SF_LAUNCHED(ctx);
    }

    PTParams& pt = S.pt;
    pt.dVx = S.L.f(F_DVX);
    pt.dVy = S.L.f(F_DVY);
    pt.rho = S.L.f(F_RHO);
    pt.mub = S.L.f(F_MUB);
    pt.mup = S.L.f(F_MUP);
    pt.txx = S.L.f(F_TXX);
    pt.tyy = S.L.f(F_TYY);
    pt.txy = S.L.f(F_TXY);
    pt.divV = S.L.f(F_DIV);
    pt.dt_ptr = ctx->d_scalars + SC_DT;
    pt.Nx = (int)Nx;
    pt.Ny = (int)Ny;
    pt.LD = LD;
    pt._dx = 1.0 / dx;
    pt._dy = 1.0 / dy;
    pt.g_y = g_y;
    pt.dampX = dampX;
    pt.dampY = dampY;
    pt.c_vsc = Vsc * min_dxy2;
    pt.c_ptsc = Ptsc * 4.1;
    pt.max_nxy = max_nxy;
    {
        int e = 0;
        double fr = std::frexp(max_nxy, &e);
        pt.pow2 = (fr == 0.5) ? 1 : 0;
        pt.inv_max_nxy = pt.pow2 ? std::ldexp(1.0, 1 - e) : 0.0;
    }
    pt.err_flag = ctx->d_flags;
    SF_CUDA(cudaMemsetAsync(ctx->d_flags, 0, sizeof(int), s));
    if ((rc = S.setup_maps())) return rc;
    ResParams& rp = S.rp;
    rp.txx = S.L.f(F_TXX);
    rp.tyy = S.L.f(F_TYY);
    rp.txy = S.L.f(F_TXY);
    rp.rho = S.L.f(F_RHO);
    rp.divV = S.L.f(F_DIV);
    rp.dt_ptr = ctx->d_scalars + SC_DT_CHECK;
    rp.Rx = S.L.f(F_RX);
    rp.Ry = S.L.f(F_RY);
    rp.partials = (double*)ctx->partials.ptr;
    rp.Nx = (int)Nx;
    rp.Ny = (int)Ny;
    rp.LD = LD;
    rp._dx = pt._dx;
    rp._dy = pt._dy;
    rp.g_y = g_y;
    return SF_OK;
}

// :89-93: the state back into the caller's arrays, Vx_pad / Vy_pad with the mirrored ghost planes
static int solver_unpack(Solver& S, const SolveArgs& A, int64_t niter, int64_t nchecks) {
    sf_ctx* ctx = S.ctx;
    cudaStream_t s = S.s;
    const int64_t Nx = S.L.Nx, Ny = S.L.Ny, LD = S.L.LD;
    struct Uk { double* dst; const double* src; int64_t nx, ny; } unpacks[] = {
        {A.Vx_s, S.Vx_cur(), Nx, Ny + 1}, {A.Vy_s, S.Vy_cur(), Nx + 1, Ny}, {A.P, S.P_cur(), Nx - 1, Ny - 1},
        {A.dVxdt, S.L.f(F_DVX), Nx - 2, Ny - 1}, {A.dVydt, S.L.f(F_DVY), Nx - 1, Ny - 2},
        {A.txx, S.L.f(F_TXX), Nx - 1, Ny - 1}, {A.tyy, S.L.f(F_TYY), Nx - 1, Ny - 1}, {A.txy, S.L.f(F_TXY), Nx, Ny},
        {A.divV, S.L.f(F_DIV), Nx - 1, Ny - 1},
        {nchecks ? A.Rx : nullptr, S.L.f(F_RX), Nx - 2, Ny - 1}, {nchecks ? A.Ry : nullptr, S.L.f(F_RY), Nx - 1, Ny - 2}};
    for (const Uk& k : unpacks) {
        if (!k.dst || niter == 0 && (k.src == S.L.f(F_TXX) || k.src == S.L.f(F_TYY) || k.src == S.L.f(F_TXY) ||
                                     k.src == S.L.f(F_DIV)))
            continue;
        k_copy2d<<<copy_blocks(ctx, k.nx * k.ny), 256, 0, s>>>(k.dst, k.nx, k.src, LD, k.nx, k.ny);
        SF_LAUNCHED(ctx);
    }
    k_pad_vx<<<copy_blocks(ctx, (Nx + 2) * (Ny + 1)), 256, 0, s>>>(A.Vx_pad, S.Vx_cur(), LD, (int)Nx, (int)Ny);
    SF_LAUNCHED(ctx);
    k_pad_vy<<<copy_blocks(ctx, (Nx + 1) * (Ny + 2)), 256, 0, s>>>(A.Vy_pad, S.Vy_cur(), LD, (int)Nx, (int)Ny);
    SF_LAUNCHED(ctx);
    return SF_OK;
}

// ---------------------------------------------------------------------------
// domain decomposition: update_halo! of ImplicitGlobalGrid (overlap 2) between ranks driven by one thread
// ---------------------------------------------------------------------------
struct Rank {
    sf_ctx* ctx;
    cudaStream_t s;
    cudaEvent_t ev;     // the rank's last finished phase (kernel, x halos, y halos)
    int left, right, down, up;  // neighbour ranks, -1 at a physical boundary
    Solver S;
    SolveArgs A;
};

// one array of every rank for a halo update: entry (i, j) at p[r] + i + j * ld[r]; local size (Nx + sx, Ny + sy)
struct HaloArray {
    std::vector<double*> p;
    std::vector<int64_t> ld;
    int64_t sx, sy;
};

// ImplicitGlobalGrid's overlap of an array along a dimension: the grid overlap (2) plus how much the array is
// larger than the grid there.  With ol = 2 + s and n = N + s entries, the last plane n-1 of a rank is the plane
// ol-1 of its upper neighbour, and the neighbour's first plane 0 is the rank's plane n-ol (0-based).
static int halo_dimension(std::vector<Rank>& R, const std::vector<HaloArray>& arrays, int dim, int64_t Nx,
                          int64_t Ny) {
    for (size_t r = 0; r < R.size(); ++r) {
        const int up = dim == 0 ? R[r].right : R[r].up;
        if (up < 0) continue;
        Rank& a = R[r];
        Rank& b = R[up];
        for (const HaloArray& h : arrays) {
            const int64_t nx = Nx + h.sx, ny = Ny + h.sy, n = dim == 0 ? nx : ny, ol = 2 + (dim == 0 ? h.sx : h.sy);
            // one plane: an x plane is a column of ny entries ld apart, a y plane a row of nx contiguous entries;
            // copied on the receiving rank's device, reading the sender's memory directly when the devices are
            // peers (copy_block)
            auto plane = [&](Rank& from, const double* src, int64_t ld_src, int64_t i_src, Rank& to, double* dst,
                             int64_t ld_dst, int64_t i_dst) -> int {
                if (dim == 0)
                    return copy_block(to.ctx, to.s, dst + i_dst, ld_dst, src + i_src, ld_src, 1, ny,
                                      from.ctx->device);
                return copy_block(to.ctx, to.s, dst + i_dst * ld_dst, ld_dst, src + i_src * ld_src, ld_src, nx, 1,
                                  from.ctx->device);
            };
            int rc;
            // into b's first plane from a's plane n-ol, on b's stream once a's phase is done
            SF_CUDA(cudaSetDevice(b.ctx->device));
            SF_CUDA(cudaStreamWaitEvent(b.s, a.ev, 0));
            if ((rc = plane(a, h.p[r], h.ld[r], n - ol, b, h.p[up], h.ld[up], 0))) return rc;
            // into a's last plane from b's plane ol-1, on a's stream once b's phase is done
            SF_CUDA(cudaSetDevice(a.ctx->device));
            SF_CUDA(cudaStreamWaitEvent(a.s, b.ev, 0));
            if ((rc = plane(b, h.p[up], h.ld[up], ol - 1, a, h.p[r], h.ld[r], n - 1))) return rc;
        }
    }
    for (Rank& k : R) {  // this dimension's incoming planes are in place
        SF_CUDA(cudaSetDevice(k.ctx->device));
        SF_CUDA(cudaEventRecord(k.ev, k.s));
    }
    return SF_OK;
}

static int update_halos(std::vector<Rank>& R, const std::vector<HaloArray>& arrays, int64_t Nx, int64_t Ny) {
    int rc = halo_dimension(R, arrays, 0, Nx, Ny);
    if (!rc) rc = halo_dimension(R, arrays, 1, Nx, Ny);
    return rc;
}

// the current Vx_s, Vy_s of every rank in the padded layout
static std::vector<HaloArray> state_halos(std::vector<Rank>& R) {
    HaloArray vx{{}, {}, 0, 1}, vy{{}, {}, 1, 0};
    for (Rank& k : R) {
        vx.p.push_back(const_cast<double*>(k.S.Vx_cur()));
        vx.ld.push_back(k.S.L.LD);
        vy.p.push_back(const_cast<double*>(k.S.Vy_cur()));
        vy.ld.push_back(k.S.L.LD);
    }
    return {vx, vy};
}

// compute_dt over all ranks (:118-121 with the MIN Allreduce): maxdisp * min(dx / max|Vx|, dy / max|Vy|) with the
// maxima over every rank's local arrays; the division is monotone and correctly rounded, so this is the
// reference's min over ranks of the local values
static int global_dt(std::vector<Rank>& R, double maxdisp, double dx, double dy, double* dt) {
    for (Rank& k : R) {
        SF_CUDA(cudaSetDevice(k.ctx->device));
        int rc = k.S.compute_dt(-1, -1);
        if (rc) return rc;
        SF_CUDA(cudaMemcpyAsync(k.ctx->h_scalars + SC_MAX_VX, k.ctx->d_scalars + SC_MAX_VX, 2 * 8,
                                cudaMemcpyDeviceToHost, k.s));
    }
    double mvx = 0.0, mvy = 0.0;
    bool nan = false;
    for (Rank& k : R) {
        SF_CUDA(cudaSetDevice(k.ctx->device));
        SF_CUDA(cudaStreamSynchronize(k.s));
        const double a = k.ctx->h_scalars[SC_MAX_VX], b = k.ctx->h_scalars[SC_MAX_VY];
        nan = nan || a != a || b != b;
        mvx = std::max(mvx, a);
        mvy = std::max(mvy, b);
    }
    const double a = dx / mvx, b = dy / mvy;
    double m = (b < a) ? b : a;
    *dt = nan ? std::nan("") : maxdisp * m;
    return SF_OK;
}

// Two plain PT iterations of every rank (kernels, their events, the halo updates), captured from the ranks'
// streams into one graph.  Only for ranks that share a device.  The graph starts with every rank's first
// kernel (the launch waits for all earlier work); the second iteration waits on the neighbours' events as the
// direct loop does.  The host-side buffer parity flips twice, so it ends where it started and the graph belongs
// to that parity.  *launches_out: the kernels the graph holds, per rank.  On any failure the capture is ended,
// the parity restored and a status returned: the caller then keeps launching directly.
static int capture_two_iterations(std::vector<Rank>& R, int64_t Nx, int64_t Ny, cudaEvent_t fork,
                                  std::vector<cudaEvent_t>& joins, cudaGraphExec_t* out,
                                  std::vector<int64_t>& launches_out) {
    std::vector<int> parity(R.size());
    std::vector<int64_t> l0(R.size());
    for (size_t k = 0; k < R.size(); ++k) {
        parity[k] = R[k].S.cur;
        l0[k] = R[k].ctx->launches;
    }
    cudaStream_t s0 = R[0].s;
    SF_CUDA(cudaSetDevice(R[0].ctx->device));
    SF_CUDA(cudaStreamBeginCapture(s0, cudaStreamCaptureModeThreadLocal));
    int rc = SF_OK;
    cudaError_t e = cudaEventRecord(fork, s0);
    for (size_t k = 1; k < R.size() && e == cudaSuccess; ++k) e = cudaStreamWaitEvent(R[k].s, fork, 0);
    for (int it = 0; it < 2 && rc == SF_OK && e == cudaSuccess; ++it) {
        if (it == 1)
            for (Rank& k : R)
                for (int n : {k.left, k.right, k.down, k.up})
                    if (n >= 0 && e == cudaSuccess) e = cudaStreamWaitEvent(k.s, R[n].ev, 0);
        for (Rank& k : R) {
            if (rc == SF_OK && e == cudaSuccess) rc = k.S.launch_iter(false);
            if (rc == SF_OK && e == cudaSuccess) e = cudaEventRecord(k.ev, k.s);
        }
        if (rc == SF_OK && e == cudaSuccess) rc = update_halos(R, state_halos(R), Nx, Ny);
    }
    for (size_t k = 1; k < R.size() && e == cudaSuccess; ++k) {
        e = cudaEventRecord(joins[k], R[k].s);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(s0, joins[k], 0);
    }
    cudaGraph_t g = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(s0, &g);
    for (size_t k = 0; k < R.size(); ++k) {
        R[k].S.cur = parity[k];
        launches_out[k] = R[k].ctx->launches - l0[k];
        R[k].ctx->launches = l0[k];
    }
    if (rc == SF_OK && (e != cudaSuccess || ee != cudaSuccess)) rc = fail(SF_ERR_CUDA, "decomposed solve: graph capture");
    if (rc == SF_OK && cudaGraphInstantiate(out, g, 0) != cudaSuccess) rc = fail(SF_ERR_CUDA, "decomposed solve: graph");
    if (g) cudaGraphDestroy(g);
    if (rc != SF_OK) {
        *out = nullptr;
        (void)cudaGetLastError();
    }
    return rc;
}

static int set_scalar_all(std::vector<Rank>& R, int slot, double v) {
    for (Rank& k : R) {
        SF_CUDA(cudaSetDevice(k.ctx->device));
        k_set_scalar<<<1, 1, 0, k.s>>>(k.ctx->d_scalars + slot, v);
        SF_LAUNCHED(k.ctx);
    }
    return SF_OK;
}

}  // namespace sf

using namespace sf;

extern "C" {

int sf_stokes_residual_scale(sf_ctx* ctx, const double* rho_vy, int64_t Nx, int64_t Ny, double g_y, void* stream,
                             double* scale) {
    SF_REQUIRE(ctx && rho_vy && scale, "sf_stokes_residual_scale: NULL argument");
    SF_REQUIRE(Nx >= 3 && Ny >= 3, "sf_stokes_residual_scale: grid too small");
    int rc = set_device(ctx);
    if (rc) return rc;
    cudaStream_t s = as_stream(stream);
    int nb = (int)std::min<int64_t>(ceil_div((Nx - 1) * (Ny - 2), 256), 1024);
    if ((rc = ensure(ctx, ctx->partials, (size_t)nb * 8))) return rc;
    k_rho_scale<<<nb, 256, 0, s>>>(rho_vy, (int)Nx, (int)Ny, g_y, (double*)ctx->partials.ptr);
    SF_LAUNCHED(ctx);
    k_sum_partials<<<1, 1024, 0, s>>>((double*)ctx->partials.ptr, nb, (double)((Nx - 1) * (Ny - 2)),
                                      ctx->d_scalars + SC_SCALE);
    SF_LAUNCHED(ctx);
    SF_CUDA(cudaMemcpyAsync(ctx->h_scalars + SC_SCALE, ctx->d_scalars + SC_SCALE, 8, cudaMemcpyDeviceToHost, s));
    SF_CUDA(cudaStreamSynchronize(s));
    *scale = ctx->h_scalars[SC_SCALE];
    return SF_OK;
}

int sf_solve_stokes(sf_ctx* ctx, double* P, double* Vx_pad, double* Vy_pad, const double* rho_vy, const double* mu_b,
                    const double* mu_p, double* txx, double* tyy, double* txy, double* divV, double* dtPt, double* Rx,
                    double* Ry, double* dVxdt, double* dVydt, double* dtVx, double* dtVy, double* Vx_s, double* Vy_s,
                    double g_y, double dx, double dy, int64_t Nx, int64_t Ny, double dt, double maxdisp,
                    int use_stab, double eps, int print_info, int64_t iter_max, void* stream, sf_solve_info* info) {
    SF_REQUIRE(ctx, "sf_solve_stokes: ctx is NULL");
    SF_REQUIRE(Nx >= 4 && Ny >= 4, "sf_solve_stokes: Nx, Ny must be >= 4");
    SF_REQUIRE(Nx < (1 << 20) && Ny < (1 << 20), "sf_solve_stokes: Nx, Ny too large");
    SF_REQUIRE(P && Vx_pad && Vy_pad && rho_vy && mu_b && mu_p && dVxdt && dVydt && Vx_s && Vy_s,
               "sf_solve_stokes: a state / parameter array is NULL");
    SF_REQUIRE(dx > 0.0 && dy > 0.0, "sf_solve_stokes: dx, dy must be positive");
    int rc = set_device(ctx);
    if (rc) return rc;
    cudaStream_t s = as_stream(stream);

    Solver S;
    const SolveArgs A{P, Vx_pad, Vy_pad, rho_vy, mu_b, mu_p, txx, tyy, txy, divV, dtPt, Rx, Ry, dVxdt, dVydt,
                      dtVx, dtVy, Vx_s, Vy_s};
    if ((rc = solver_prepare(S, ctx, s, A, Nx, Ny, g_y, dx, dy, dt, maxdisp, use_stab, Nx, Ny))) return rc;
    const int64_t mnxy = std::min(Nx, Ny);
    const int64_t ncheck = std::min<int64_t>(5 * mnxy, 2000);  // :35
    const int64_t ndtupdate = 10 * mnxy;                       // :36

    // ---- PT loop (:43-77) ----
    double err = 2.0 * eps;
    int64_t iter = 1, niter = 0, nchecks = 0;
    const int64_t itert1 = 11;
    bool have_t1 = false;
    int64_t fused = 0;
    SF_CUDA(cudaEventRecord(ctx->ev_c, s));
    while (err > eps && iter <= iter_max) {
        // iterations up to and including the next check (or iter_max)
        int64_t next_check = ((iter - 1) / ncheck + 1) * ncheck;
        int64_t last = std::min(next_check, iter_max);
        for (int64_t it = iter; it <= last; ++it) {
            if (it == itert1) {
                SF_CUDA(cudaEventRecord(ctx->ev_a, s));
                have_t1 = true;
            }
            bool store = (it % ncheck == 0) || (it == iter_max);
            if ((rc = S.launch_iter(store))) return rc;
            ++fused;
            bool dt_up = use_stab && (it % ndtupdate == 0);
            bool check = (it % ncheck == 0);
            if (dt_up || (check && use_stab)) {
                if ((rc = S.compute_dt(dt_up ? SC_DT : -1, check ? SC_DT_CHECK : -1))) return rc;
            }
            if (check && !use_stab) {
                k_set_scalar<<<1, 1, 0, s>>>(ctx->d_scalars + SC_DT_CHECK, 0.0);
                SF_LAUNCHED(ctx);
            }
        }
        niter += last - iter + 1;
        iter = last + 1;
        if (last % ncheck == 0) {
            if ((rc = S.residuals())) return rc;
            ++nchecks;
            SF_CUDA(cudaMemcpyAsync(ctx->h_scalars + SC_ERR, ctx->d_scalars + SC_ERR, 8, cudaMemcpyDeviceToHost, s));
            SF_CUDA(cudaStreamSynchronize(s));
            err = ctx->h_scalars[SC_ERR];
            if (!(err == err) || std::isinf(err)) break;
        }
    }
    SF_CUDA(cudaEventRecord(ctx->ev_b, s));

    // ---- unpack (:89-95) ----
    if ((rc = solver_unpack(S, A, niter, nchecks))) return rc;
    if ((rc = S.compute_dt(SC_DT_OUT, -1))) return rc;  // returned dt (:95)
    SF_CUDA(cudaMemcpyAsync(ctx->h_scalars, ctx->d_scalars, SC_N * 8, cudaMemcpyDeviceToHost, s));
    SF_CUDA(cudaStreamSynchronize(s));
    double dt_out = ctx->h_scalars[SC_DT_OUT];

    float ms_loop = 0.f, ms_t1 = 0.f;
    SF_CUDA(cudaEventElapsedTime(&ms_loop, ctx->ev_c, ctx->ev_b));
    if (have_t1) SF_CUDA(cudaEventElapsedTime(&ms_t1, ctx->ev_a, ctx->ev_b));
    double runtime = have_t1 ? ms_t1 * 1e-3 : 0.0;
    double t_it = (niter - itert1 + 1) > 0 ? runtime / (double)(niter - itert1 + 1) : 0.0;
    double A_eff = (3.0 * 2.0) / 1e9 * (double)Nx * (double)Ny * 8.0;
    double T_eff = t_it > 0 ? A_eff / t_it : 0.0;
    // essential bytes: read+write Vx_s, Vy_s, P, dVx, dVy; read rho, mu_b, mu_p
    double bpi = 8.0 * (2.0 * ((double)Nx * (Ny + 1) + (double)(Nx + 1) * Ny + (double)(Nx - 1) * (Ny - 1) +
                               (double)(Nx - 2) * (Ny - 1) + (double)(Nx - 1) * (Ny - 2)) +
                        (double)(Nx + 1) * Ny + (double)Nx * Ny + (double)(Nx - 1) * (Ny - 1));
    if (print_info)
        printf("Total steps = %lld, err = %1.3e, time = %1.3e sec (@ T_eff = %1.2f GB/s) \n", (long long)niter, err,
               runtime, T_eff);
    if (info) {
        info->dt = dt_out;
        info->T_eff = T_eff;
        info->runtime = runtime;
        info->iters = niter;
        info->err = err;
        info->n_checks = nchecks;
        info->converged = (err <= eps) ? 1 : 0;
        info->reserved = 0;
        info->loop_ms = ms_loop;
        info->bytes_per_iter = bpi;
        info->T_eff_essential = ms_loop > 0 ? bpi * (double)niter / (ms_loop * 1e-3) / 1e9 : 0.0;
        info->fused_launches = fused;
        info->fused_ms = 0.0;
    }
    int hflag = 0;
    SF_CUDA(cudaMemcpy(&hflag, ctx->d_flags, sizeof(int), cudaMemcpyDeviceToHost));
    if (hflag) return fail(SF_ERR_CUDA, "sf_solve_stokes: a tile copy into shared memory did not complete in time");
    if (!(err == err) || std::isinf(err)) return fail(SF_ERR_NONFINITE, "sf_solve_stokes: residual is not finite");
    return SF_OK;
}

int sf_solve_stokes_decomposed(sf_domain* domains, int32_t dims_x, int32_t dims_y, int64_t Nx, int64_t Ny,
                               double g_y, double dx, double dy, double dt, double maxdisp, int use_stab, double eps,
                               int64_t iter_max, sf_solve_info* info) {
    SF_REQUIRE(domains && dims_x >= 1 && dims_y >= 1 && dims_x * dims_y <= 4096, "sf_solve_stokes_decomposed: bad dims");
    SF_REQUIRE(Nx >= 4 && Ny >= 4 && Nx < (1 << 20) && Ny < (1 << 20), "sf_solve_stokes_decomposed: bad local grid");
    SF_REQUIRE(dx > 0.0 && dy > 0.0, "sf_solve_stokes_decomposed: dx, dy must be positive");
    const int nr = dims_x * dims_y;
    SF_REQUIRE(distinct_contexts(nr, [&](int i) { return domains[i].ctx; }),
               "sf_solve_stokes_decomposed: every rank needs its own context");
    std::vector<int> at((size_t)nr, -1);  // rank index of each coordinate
    for (int r = 0; r < nr; ++r) {
        const sf_domain& d = domains[r];
        SF_REQUIRE(d.ctx && d.P && d.Vx_pad && d.Vy_pad && d.rho_vy && d.mu_b && d.mu_p && d.dVxdt && d.dVydt &&
                       d.Vx_s && d.Vy_s,
                   "sf_solve_stokes_decomposed: a domain array is NULL");
        SF_REQUIRE(d.coord_x >= 0 && d.coord_x < dims_x && d.coord_y >= 0 && d.coord_y < dims_y,
                   "sf_solve_stokes_decomposed: coordinate outside dims");
        const int c = d.coord_x + d.coord_y * dims_x;
        SF_REQUIRE(at[c] < 0, "sf_solve_stokes_decomposed: two domains have the same coordinates");
        at[c] = r;
    }
    const int64_t nx_g = (int64_t)dims_x * (Nx - 2) + 2, ny_g = (int64_t)dims_y * (Ny - 2) + 2;  // nx_g(), ny_g()
    const int64_t mnxy = std::min(nx_g, ny_g);
    const int64_t ncheck = std::min<int64_t>(5 * mnxy, 2000);  // :35
    const int64_t ndtupdate = 10 * mnxy;                       // :36
    if (!use_stab) dt = 0.0;

    std::vector<Rank> R((size_t)nr);
    int rc;
    for (int r = 0; r < nr; ++r) {
        const sf_domain& d = domains[r];
        Rank& k = R[r];
        k.ctx = d.ctx;
        if ((rc = set_device(k.ctx))) return rc;
        SF_CUDA(cudaDeviceSynchronize());  // the caller's inputs are complete
        k.s = k.ctx->work;
        SF_CUDA(cudaEventCreateWithFlags(&k.ev, cudaEventDisableTiming));
        auto nb = [&](int cx, int cy) { return (cx < 0 || cy < 0 || cx >= dims_x || cy >= dims_y) ? -1 : at[cx + cy * dims_x]; };
        k.left = nb(d.coord_x - 1, d.coord_y);
        k.right = nb(d.coord_x + 1, d.coord_y);
        k.down = nb(d.coord_x, d.coord_y - 1);
        k.up = nb(d.coord_x, d.coord_y + 1);
        k.A = SolveArgs{d.P, d.Vx_pad, d.Vy_pad, d.rho_vy, d.mu_b, d.mu_p, nullptr, nullptr, nullptr, nullptr, nullptr,
                        nullptr, nullptr, d.dVxdt, d.dVydt, nullptr, nullptr, d.Vx_s, d.Vy_s};
        if ((rc = solver_prepare(k.S, k.ctx, k.s, k.A, Nx, Ny, g_y, dx, dy, dt, maxdisp, use_stab, nx_g, ny_g)))
            return rc;
        SF_CUDA(cudaEventRecord(k.ev, k.s));
    }
    auto destroy_events = [&]() {
        for (Rank& k : R)
            if (k.ev) {
                cudaSetDevice(k.ctx->device);
                cudaEventDestroy(k.ev);
            }
    };
    struct Guard { std::function<void()> f; ~Guard() { f(); } } guard{destroy_events};

    // ---- PT loop (:43-77), every rank per iteration, halos after it (:57) ----
    // Ranks that share a device run their plain iterations (no store, dt update or check) two at a time from a
    // captured graph, one per buffer parity: one host launch instead of every rank's kernels, events and halo
    // copies.  Ranks on several devices launch directly.
    bool graphs = nr > 1;
    for (const Rank& k : R) graphs = graphs && k.ctx->device == R[0].ctx->device;
    cudaGraphExec_t gexec[2] = {nullptr, nullptr};
    std::vector<int64_t> glaunches[2] = {std::vector<int64_t>((size_t)nr, 0), std::vector<int64_t>((size_t)nr, 0)};
    cudaEvent_t gfork = nullptr, gdone = nullptr;
    // gjoin are recorded inside the capture only; gpre order the graph launch after every rank's earlier work
    // (an event last recorded inside a capture cannot be waited on outside it)
    std::vector<cudaEvent_t> gjoin((size_t)nr, nullptr), gpre((size_t)nr, nullptr);
    auto destroy_graphs = [&]() {
        for (cudaGraphExec_t& x : gexec)
            if (x) cudaGraphExecDestroy(x);
        if (gfork) cudaEventDestroy(gfork);
        if (gdone) cudaEventDestroy(gdone);
        for (cudaEvent_t ev : gjoin)
            if (ev) cudaEventDestroy(ev);
        for (cudaEvent_t ev : gpre)
            if (ev) cudaEventDestroy(ev);
    };
    struct Guard2 { std::function<void()> f; ~Guard2() { f(); } } guard2{destroy_graphs};
    if (graphs) {
        SF_CUDA(cudaSetDevice(R[0].ctx->device));
        SF_CUDA(cudaEventCreateWithFlags(&gfork, cudaEventDisableTiming));
        SF_CUDA(cudaEventCreateWithFlags(&gdone, cudaEventDisableTiming));
        for (cudaEvent_t& ev : gjoin) SF_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        for (cudaEvent_t& ev : gpre) SF_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    }
    auto plain = [&](int64_t it) {
        return it < iter_max && it % ncheck != 0 && !(use_stab && it % ndtupdate == 0);
    };
    const auto t0 = std::chrono::steady_clock::now();
    double err = 2.0 * eps;
    int64_t iter = 1, niter = 0, nchecks = 0;
    while (err > eps && iter <= iter_max) {
        if (graphs && plain(iter) && plain(iter + 1)) {
            const int par = R[0].S.cur;
            if (!gexec[par] && capture_two_iterations(R, Nx, Ny, gfork, gjoin, &gexec[par], glaunches[par]))
                graphs = false;   // keep launching directly
            if (gexec[par]) {
                SF_CUDA(cudaSetDevice(R[0].ctx->device));
                for (size_t k = 0; k < R.size(); ++k) {   // every rank's earlier work
                    SF_CUDA(cudaEventRecord(gpre[k], R[k].s));
                    SF_CUDA(cudaStreamWaitEvent(R[0].s, gpre[k], 0));
                }
                SF_CUDA(cudaGraphLaunch(gexec[par], R[0].s));
                SF_CUDA(cudaEventRecord(gdone, R[0].s));
                for (size_t k = 0; k < R.size(); ++k) {
                    SF_CUDA(cudaStreamWaitEvent(R[k].s, gdone, 0));
                    SF_CUDA(cudaEventRecord(R[k].ev, R[k].s));
                    R[k].ctx->launches += glaunches[par][k];
                }
                niter += 2;
                iter += 2;
                continue;
            }
        }
        const bool store = (iter % ncheck == 0) || (iter == iter_max);
        for (Rank& k : R) {
            SF_CUDA(cudaSetDevice(k.ctx->device));
            // the neighbours have finished reading this rank's planes of the previous iteration
            for (int n : {k.left, k.right, k.down, k.up})
                if (n >= 0) SF_CUDA(cudaStreamWaitEvent(k.s, R[n].ev, 0));
        }
        for (Rank& k : R) {
            SF_CUDA(cudaSetDevice(k.ctx->device));
            if ((rc = k.S.launch_iter(store))) return rc;
            SF_CUDA(cudaEventRecord(k.ev, k.s));
        }
        if ((rc = update_halos(R, state_halos(R), Nx, Ny))) return rc;
        const bool dt_up = use_stab && (iter % ndtupdate == 0);
        const bool check = (iter % ncheck == 0);
        if (dt_up || (check && use_stab)) {  // :59-61, :64-68
            double d_new = 0.0;
            if ((rc = global_dt(R, maxdisp, dx, dy, &d_new))) return rc;
            if (dt_up && (rc = set_scalar_all(R, SC_DT, d_new))) return rc;
            if (check && (rc = set_scalar_all(R, SC_DT_CHECK, d_new))) return rc;
        } else if (check) {
            if ((rc = set_scalar_all(R, SC_DT_CHECK, 0.0))) return rc;
        }
        if (check) {  // :69-70, compute_err with the SUM Allreduce of the local means (:103-109)
            for (Rank& k : R) {
                SF_CUDA(cudaSetDevice(k.ctx->device));
                if ((rc = k.S.residuals())) return rc;
                SF_CUDA(cudaMemcpyAsync(k.ctx->h_scalars + SC_SUM_RX, k.ctx->d_scalars + SC_SUM_RX, 3 * 8,
                                        cudaMemcpyDeviceToHost, k.s));
            }
            double mean[3] = {0.0, 0.0, 0.0};
            const double cnt[3] = {(double)(Nx - 2) * (Ny - 1), (double)(Nx - 1) * (Ny - 2), (double)(Nx - 1) * (Ny - 1)};
            for (Rank& k : R) {
                SF_CUDA(cudaSetDevice(k.ctx->device));
                SF_CUDA(cudaStreamSynchronize(k.s));
                for (int q = 0; q < 3; ++q) mean[q] += k.ctx->h_scalars[SC_SUM_RX + q] / cnt[q];
            }
            for (int q = 0; q < 3; ++q) mean[q] /= (double)nr;
            double m = mean[0];
            if (mean[1] > m || mean[1] != mean[1]) m = mean[1];
            if (mean[2] > m || mean[2] != mean[2]) m = mean[2];
            if (mean[0] != mean[0]) m = mean[0];
            err = m;
            ++nchecks;
            for (Rank& k : R) {
                SF_CUDA(cudaSetDevice(k.ctx->device));
                SF_CUDA(cudaEventRecord(k.ev, k.s));
            }
        }
        ++niter;
        ++iter;
        if (!(err == err) || std::isinf(err)) break;
    }

    // ---- unpack, Vx_pad / Vy_pad mirrored and their halos updated (:89-93) ----
    HaloArray px{{}, {}, 2, 1}, py{{}, {}, 1, 2};
    for (Rank& k : R) {
        SF_CUDA(cudaSetDevice(k.ctx->device));
        for (int n : {k.left, k.right, k.down, k.up})
            if (n >= 0) SF_CUDA(cudaStreamWaitEvent(k.s, R[n].ev, 0));
        if ((rc = solver_unpack(k.S, k.A, niter, nchecks))) return rc;
        SF_CUDA(cudaEventRecord(k.ev, k.s));
        px.p.push_back(k.A.Vx_pad);
        px.ld.push_back(Nx + 2);
        py.p.push_back(k.A.Vy_pad);
        py.ld.push_back(Nx + 1);
    }
    if ((rc = update_halos(R, {px, py}, Nx, Ny))) return rc;
    double dt_out = 0.0;
    if ((rc = global_dt(R, maxdisp, dx, dy, &dt_out))) return rc;  // :95
    int hflag = 0;
    for (Rank& k : R) {
        SF_CUDA(cudaSetDevice(k.ctx->device));
        SF_CUDA(cudaStreamSynchronize(k.s));
        int f = 0;
        SF_CUDA(cudaMemcpy(&f, k.ctx->d_flags, sizeof(int), cudaMemcpyDeviceToHost));
        hflag |= f;
    }
    const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (info) {
        memset(info, 0, sizeof(*info));
        info->dt = dt_out;
        info->iters = niter;
        info->err = err;
        info->n_checks = nchecks;
        info->converged = (err <= eps) ? 1 : 0;
        info->loop_ms = ms;
        info->fused_launches = niter * nr;
    }
    if (hflag) return fail(SF_ERR_CUDA, "sf_solve_stokes_decomposed: a tile copy into shared memory did not complete in time");
    if (!(err == err) || std::isinf(err)) return fail(SF_ERR_NONFINITE, "sf_solve_stokes_decomposed: residual is not finite");
    return SF_OK;
}

}  // extern "C"
