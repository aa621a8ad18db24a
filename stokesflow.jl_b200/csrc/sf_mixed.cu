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
// launch over a device-resident work list of 32-column tiles from all
// instances in their inner phase, with per-instance tensor maps (TMA,
// double-buffered, no multicast) -- so hundreds of small problems cost one
// launch per iteration instead of hundreds.  The runs of iterations between
// checks are replayed from captured CUDA graphs.  The tile rows (8, 16, 32),
// the order in which the CTAs take the tiles and whether consecutive sweeps
// overlap their launches are chosen per workload class by timing them (the
// tuner); every choice computes the same bits.  Instances move between phases
// independently, which is what lets a serving loop add and retire instances
// while others run.
//
// The FP32 sweeps are not bit-compatible with the plain FP64 path (nothing can
// be at FP32); their accuracy is measured against the FP64 oracle.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <deque>
#include <iterator>
#include <map>
#include <string>
#include <type_traits>
#include <vector>

#include "sf_internal.cuh"
#include "sf_tma.cuh"

namespace sf {
namespace mx {

// Sweep tiles are BX = 32 columns by BY rows, BY one of the shapes below (the autotuner picks it); 8 rows of
// 32 threads, each thread BY/8 rows.  The FP64 kernels keep their own fixed 32 x 16 tiling, so the order of
// their per-tile sums, and with it every residual and stopping decision, does not depend on the sweep shape.
constexpr int BX = 32, TY = 8, NT = BX * TY;
constexpr int BY64 = 16;              // tile rows of the FP64 kernels
constexpr int TW = 36;                // staged halo box width; TW*4 bytes is a multiple of 16
constexpr int W1 = BX + 1;
constexpr int r128(int b) { return (b + 127) / 128 * 128; }
constexpr int NHALO = 7;  // dVx, dVy, dP (current), mu_b, mu_p, rho, rdiv
constexpr int NTILE = 4;  // rate_x, rate_y, rx, ry
constexpr int NST = 2;
template <int BY>
struct Shape {
    static_assert(BY % TY == 0, "tile rows must be a multiple of the thread rows");
    static constexpr int TH = BY + 2, H1 = BY + 1, RPT = BY / TY;
    static constexpr int HALO_BYTES = r128(TH * TW * 4);
    static constexpr int TILE_BYTES = r128(BY * BX * 4);
    static constexpr int STAGE_BYTES = NHALO * HALO_BYTES + NTILE * TILE_BYTES;
    static constexpr uint32_t STAGE_TX = NHALO * TH * TW * 4 + NTILE * BY * BX * 4;
    static constexpr int ST1_BYTES = r128(H1 * W1 * 4);
    static constexpr int SMEM_BYTES = NST * STAGE_BYTES + ST1_BYTES + 64;   // + tau_xy (the others live in the stage)
};
constexpr uint64_t WAIT_BUDGET_NS = 2000000000ull;

// FP32 fields of an instance (each LD32 x rows floats)
enum { G_VXA, G_VXB, G_VYA, G_VYB, G_PA, G_PB, G_RVX, G_RVY, G_MUB, G_MUP, G_RHO, G_RX, G_RY, G_RDIV, G_NUM };
// FP64 fields of an instance (each LD64 x rows doubles)
enum { D_VX, D_VY, D_P, D_RHO, D_MUB, D_MUP, D_NUM };
// tensor maps per instance, in the order a stage is filled
// tensor maps per instance and shape: all G_NUM FP32 fields as one 3-D tensor (the field index is z), read
// through a halo box and through a tile box
enum { M_HALO, M_TILE, M_NUM };

struct Inst {  // device-side description of one instance
    int Nx, Ny;
    int ntx, pad_;          // tiles in x (32 columns for the sweeps and the FP64 kernels alike, whatever the rows)
    int64_t LD32, LD64, rows;
    float* f32;             // G_NUM fields
    double* f64;            // D_NUM fields
    int64_t fstride32, fstride64;
    float _dxf, _dyf, c_vscf, c_ptscf;   // FP32 constants
    // 1 - dampX = Vdmp / Nx and 1 - dampY in FP32: the sweeps damp a rate as r - (Vdmp/Nx) r, which keeps the
    // damping's distance from 1 -- what sets the rates' memory of about Nx/Vdmp sweeps -- accurate to FP32's
    // relative precision; dampX itself rounded to FP32 would be off by up to 3e-8 absolute, a systematic
    // relative error of up to 2e-6 .. 8e-6 in 1 - dampX on grids of 300 .. 1000 points
    float cdampXf, cdampYf;
    float g_dtf;            // g_y * dt for the stabilisation term of the correction
    int pad1_;
    double dx, dy, _dx, _dy, g_y, dt, dt_cfl, dt_in, maxdisp;
    int use_stab;
    int dtau_max;           // pseudo-time step from the stencil's largest viscosity
};

// Per-instance control word, written by host copies between rounds only (never by a kernel):
//   parity  which correction buffer (0: A, 1: B) holds the current correction before the round's first sweep;
//   budget  sweeps the instance runs in this round: it sweeps in launches 0 .. budget-1 of the round and
//           sits out the rest, so that every round ends exactly where the reference's loop has an event
//           (a dt update every ndtupdate iterations, a residual check every ncheck, iterMax);
//   flags   the events at the end of that round (CTL_DT, CTL_CHECK), read by the FP64 kernels of the next.
struct Ctl { int parity, budget, flags, pad_; };
enum { CTL_DT = 1, CTL_CHECK = 2 };

__device__ __forceinline__ float* gf(const Inst& I, int k) { return I.f32 + (int64_t)k * I.fstride32; }
__device__ __forceinline__ double* gd(const Inst& I, int k) { return I.f64 + (int64_t)k * I.fstride64; }

// ---------------------------------------------------------------------------
// FP32 PT sweep over a tile work list (tiles: {instance, tile index})
// ---------------------------------------------------------------------------
// The arithmetic of a point does not depend on BY: the file is compiled without contraction and the fused
// multiply-adds below are written out, so every shape (and a change of shape between sweeps) gives the same bits.
// Launch `launch_idx` of a round sweeps the tiles of the instances whose budget exceeds it; the others' tiles
// are passed over without a copy.
template <int BY, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_pt32(const CUtensorMap* __restrict__ maps, const Inst* __restrict__ insts,
                                                   const Ctl* __restrict__ ctl, const int2* __restrict__ tiles,
                                                   const int* __restrict__ ntiles_ptr, int launch_idx, int chunked,
                                                   int* __restrict__ err_flag) {
    static_assert(NST == 2, "the copy pipeline runs one tile ahead");
    using S = Shape<BY>;
    constexpr int TH = S::TH, H1 = S::H1, RPT = S::RPT, HALO_BYTES = S::HALO_BYTES, TILE_BYTES = S::TILE_BYTES;
    constexpr int STAGE_BYTES = S::STAGE_BYTES, ST1_BYTES = S::ST1_BYTES;
    constexpr uint32_t STAGE_TX = S::STAGE_TX;
    (void)TH;
    extern __shared__ __align__(128) unsigned char smem[];
    typedef float Row1[W1];
    typedef float RowH[TW];
    typedef float RowT[BX];
    Row1* sTxy = reinterpret_cast<Row1*>(smem + NST * STAGE_BYTES);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + NST * STAGE_BYTES + ST1_BYTES);

    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * BX + tx;
    const int ntiles = *ntiles_ptr;
    // schedule: strided (CTA b of G takes tiles b, b + G, ...: neighbouring tiles run side by side) or chunked
    // (CTA b takes a contiguous run of ceil(ntiles / G) tiles: it meets few instances, so it fences few maps)
    const int G = gridDim.x;
    int first, step, end;
    if (chunked) {
        const int chunk = (ntiles + G - 1) / G;
        first = blockIdx.x * chunk;
        step = 1;
        end = min(ntiles, first + chunk);
    } else {
        first = blockIdx.x;
        step = G;
        end = ntiles;
    }
    // the tiles this CTA sweeps in this launch: its share of the list, less those of instances whose budget is
    // used up (every thread walks the same sequence; control words and tile list are host-written)
    auto next_live = [&](int t) {
        for (; t < end; t += step)
            if (ctl[tiles[t].x].budget > launch_idx) break;
        return t;
    };
    // the tile list is ordered by instance, so a CTA meets each instance in one run of tiles: the two maps it
    // reads are fenced when the run starts
    int fenced = -1;
    auto fence_maps = [&](int x) {
        fence_tensormap_acquire(maps + (int64_t)x * M_NUM + M_HALO);
        fence_tensormap_acquire(maps + (int64_t)x * M_NUM + M_TILE);
        fenced = x;
    };
    int t = next_live(first);
    if (tid == 0) {
        for (int k = 0; k < NST; ++k) mbar_init(&bar[k], 1);
        fence_mbar_init();
        // the first instance's maps are fenced before the wait below, while the previous sweep may still run:
        // maps, tile list, tile count and control words are written by host copies before the sweeps, never
        // by a sweep
        if (t < end) fence_maps(tiles[t].x);
    }
    __syncthreads();
    // the previous sweep's corrections and rates are complete and visible from here on
    griddep_wait();
    griddep_launch_dependents();
    const int launch_parity = launch_idx & 1;
    auto issue = [&](int t, int s) {  // thread 0 only
        const int2 td = tiles[t];
        const Inst& I = insts[td.x];
        const int i0 = (td.y % I.ntx) * BX, j0 = (td.y / I.ntx) * BY;
        const int in = (ctl[td.x].parity ^ launch_parity) & 1;
        const CUtensorMap* H = maps + (int64_t)td.x * M_NUM + M_HALO;
        const CUtensorMap* T = maps + (int64_t)td.x * M_NUM + M_TILE;
        if (td.x != fenced) fence_maps(td.x);
        unsigned char* st = smem + s * STAGE_BYTES;
        mbar_arrive_expect_tx(&bar[s], STAGE_TX);
        tma_load_3d(st + 0 * HALO_BYTES, H, &bar[s], i0, j0, in ? G_VXB : G_VXA);
        tma_load_3d(st + 1 * HALO_BYTES, H, &bar[s], i0, j0, in ? G_VYB : G_VYA);
        tma_load_3d(st + 2 * HALO_BYTES, H, &bar[s], i0, j0, in ? G_PB : G_PA);
        tma_load_3d(st + 3 * HALO_BYTES, H, &bar[s], i0, j0, G_MUB);
        tma_load_3d(st + 4 * HALO_BYTES, H, &bar[s], i0, j0, G_MUP);
        tma_load_3d(st + 5 * HALO_BYTES, H, &bar[s], i0, j0, G_RHO);
        tma_load_3d(st + 6 * HALO_BYTES, H, &bar[s], i0, j0, G_RDIV);
        unsigned char* tb = st + NHALO * HALO_BYTES;
        tma_load_3d(tb + 0 * TILE_BYTES, T, &bar[s], i0, j0, G_RVX);
        tma_load_3d(tb + 1 * TILE_BYTES, T, &bar[s], i0, j0, G_RVY);
        tma_load_3d(tb + 2 * TILE_BYTES, T, &bar[s], i0, j0, G_RX);
        tma_load_3d(tb + 3 * TILE_BYTES, T, &bar[s], i0, j0, G_RY);
    };
    if (tid == 0 && t < end) issue(t, 0);
    int tn = (t < end) ? next_live(t + step) : end;   // the tile after t, copied while t is computed
    uint32_t phase = 0;
    int s = 0;
    // a copy never completed: flag it, give every copy still in flight a bounded chance to land (the issuing
    // thread knows their phases: stage s has just been waited on, stage s^1 holds tile tn), leave together
    auto give_up = [&]() {
        if (tid == 0) {
            atomicExch(err_flag, 1);
            mbar_wait(&bar[s], ((phase >> s) & 1u) ^ 1u, WAIT_BUDGET_NS);
            if (tn < end) mbar_wait(&bar[s ^ 1], (phase >> (s ^ 1)) & 1u, WAIT_BUDGET_NS);
        }
        __syncthreads();
    };
    for (; t < end; t = tn, tn = (tn < end) ? next_live(tn + step) : end) {
        if (tid == 0 && tn < end) issue(tn, s ^ 1);
        // the timeout vote rides on the stage-1 barrier below: stage 1 writes shared memory only, so a thread
        // whose copy did not land computes garbage there and nothing else before everyone leaves
        const bool ok = mbar_wait(&bar[s], (phase >> s) & 1u, WAIT_BUDGET_NS);
        phase ^= 1u << s;
        const int2 td = tiles[t];
        const Inst& I = insts[td.x];
        const int Nx = I.Nx, Ny = I.Ny;
        const int i0 = (td.y % I.ntx) * BX, j0 = (td.y / I.ntx) * BY;
        const int in = (ctl[td.x].parity ^ launch_parity) & 1;
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
        // this tile's corner in the fields; in-tile offsets fit 32 bits
        const int64_t tbase = i0 + (int64_t)j0 * LD;
        const int ldi = (int)LD;
        float* Vx_out = gf(I, in ? G_VXA : G_VXB) + tbase;
        float* Vy_out = gf(I, in ? G_VYA : G_VYB) + tbase;
        float* P_out = gf(I, in ? G_PA : G_PB) + tbase;
        float* Rvx = gf(I, G_RVX) + tbase;
        float* Rvy = gf(I, G_RVY) + tbase;
        const float c_pt = I.c_ptscf, cdampX = I.cdampXf, cdampY = I.cdampYf, g_dt = I.g_dtf;
        const float h_dx = 0.5f * _dx, h_dy = 0.5f * _dy;
        // pseudo-time step c_vsc / mu_av = (2 c_vsc) / (mu_0 + mu_1) (the reference's average, :129-130), or
        // c_vsc / (largest viscosity of the node's stencil); the FP32 sweeps only drive the correction, so the
        // fast division is enough
        const float c_vsc = I.c_vscf, c_vsc2 = 2.0f * I.c_vscf;
        const bool dmax = I.dtau_max != 0;
        // interior tiles: every point of the tile and its halo is inside, no boundary node among them
        const bool interior = i0 > 0 && j0 > 0 && i0 + BX + 2 < Nx && j0 + BY + 2 < Ny;

        // ---- stage 1: P and tau of the correction on tile + 1 halo ----
        // stage 2 needs P only through differences next to tau_xx / tau_yy, so stage 1 keeps
        // sigma_xx = tau_xx - P (over the divV-residual box) and sigma_yy = tau_yy - P (over the old P box), each
        // point reading only its own entry of those first, and writes P straight out
        RowH* sSxx = sRdiv;
        RowH* sSyy = sPo;
        auto stage1 = [&](int a, int b) {
            const int i = i0 + a, j = j0 + b;
            if (interior || (i < Nx - 1 && j < Ny - 1)) {
                float dVx_dx = (sVx[b + 1][a + 1] - sVx[b + 1][a]) * _dx;
                float dVy_dy = (sVy[b + 1][a + 1] - sVy[b][a + 1]) * _dy;
                float div_d = dVx_dx + dVy_dy;
                float div_full = div_d + sRdiv[b][a];          // divV of V_k + dV
                float mu = sMup[b][a];
                float pn = fmaf(-(c_pt * mu), div_full, sPo[b][a]);
                float mu2 = 2.0f * mu;
                sSxx[b][a] = fmaf(mu2, fmaf(-(1.0f / 3.0f), div_d, dVx_dx), -pn);
                sSyy[b][a] = fmaf(mu2, fmaf(-(1.0f / 3.0f), div_d, dVy_dy), -pn);
                if (a < BX && b < BY) P_out[a + b * ldi] = pn;
            }
            if (interior || (i < Nx && j < Ny)) {
                float dVx_dy = (sVx[b + 1][a] - sVx[b][a]) * _dy;
                float dVy_dx = (sVy[b][a + 1] - sVy[b][a]) * _dx;
                sTxy[b][a] = sMub[b][a] * (dVx_dy + dVy_dx);
            }
        };
        // the (BX+1) x (BY+1) points spread evenly over all threads, row by row
        for (int idx = tid; idx < W1 * H1; idx += NT) {
            const int b = idx / W1, a = idx - b * W1;
            stage1(a, b);
        }
        if (__syncthreads_or(!ok)) {
            give_up();
            return;
        }
        // ---- stage 2: damped rates and velocity update of the correction ----
        auto rate_x = [&](int a, int b, int o) {
            float Rx = fmaf(sSxx[b][a + 1] - sSxx[b][a], _dx, fmaf(sTxy[b + 1][a + 1] - sTxy[b][a + 1], _dy, sRx[b][a]));
            const float r0 = sRvx[b][a];
            float dv = fmaf(-cdampX, r0, r0) + Rx;   // dampX * r0 + Rx
            Rvx[o] = dv;
            float dtau = dmax ? __fdividef(c_vsc, fmaxf(fmaxf(sMup[b][a], sMup[b][a + 1]),
                                                       fmaxf(sMub[b][a + 1], sMub[b + 1][a + 1])))
                              : __fdividef(c_vsc2, sMup[b][a] + sMup[b][a + 1]);
            return fmaf(dtau, dv, sVx[b + 1][a + 1]);
        };
        auto rate_y = [&](int a, int b, int o) {
            float av = 0.25f * (sVx[b + 1][a] + sVx[b + 1][a + 1] + sVx[b + 2][a] + sVx[b + 2][a + 1]);
            float dxr = sRho[b + 1][a + 2] - sRho[b + 1][a];
            float dyr = sRho[b + 2][a + 1] - sRho[b][a + 1];
            float stab = fmaf(av * dxr, h_dx, (sVy[b + 1][a + 1] * dyr) * h_dy);
            float Ry = fmaf(sSyy[b + 1][a] - sSyy[b][a], _dy,
                            fmaf(sTxy[b + 1][a + 1] - sTxy[b + 1][a], _dx, fmaf(-g_dt, stab, sRy[b][a])));
            const float r0 = sRvy[b][a];
            float dv = fmaf(-cdampY, r0, r0) + Ry;   // dampY * r0 + Ry
            Rvy[o] = dv;
            float dtau = dmax ? __fdividef(c_vsc, fmaxf(fmaxf(sMup[b][a], sMup[b + 1][a]),
                                                       fmaxf(sMub[b + 1][a], sMub[b + 1][a + 1])))
                              : __fdividef(c_vsc2, sMup[b][a] + sMup[b + 1][a]);
            return fmaf(dtau, dv, sVy[b + 1][a + 1]);
        };
        if (interior) {
#pragma unroll
            for (int r = 0; r < RPT; ++r) {
                const int a = tx, b = ty + r * TY;
                const int o = a + b * ldi;
                Vx_out[o + 1 + ldi] = rate_x(a, b, o);
                Vy_out[o + 1 + ldi] = rate_y(a, b, o);
            }
        } else {
#pragma unroll
            for (int r = 0; r < RPT; ++r) {
                const int a = tx, b = ty + r * TY;
                const int i = i0 + a, j = j0 + b;
                if (i >= Nx - 1 || j >= Ny - 1) continue;
                const int o = a + b * ldi;
                if (i < Nx - 2) {
                    float vn = rate_x(a, b, o);
                    Vx_out[o + 1 + ldi] = vn;
                    if (j == 0) Vx_out[o + 1] = vn;
                    if (j == Ny - 2) Vx_out[o + 1 + 2 * ldi] = vn;
                }
                if (j < Ny - 2) {
                    float vn = rate_y(a, b, o);
                    Vy_out[o + 1 + ldi] = vn;
                    if (i == 0) Vy_out[o + ldi] = vn;
                    if (i == Nx - 2) Vy_out[o + 2 + ldi] = vn;
                }
                // free-slip rows / columns: relative to the tile corner (i0, j0)
                if (i == 0 || i == Nx - 2) {
                    int ac = (i == 0) ? -i0 : Nx - 1 - i0;
                    Vx_out[ac + (b + 1) * ldi] = 0.f;
                    if (j == 0) Vx_out[ac - j0 * ldi] = 0.f;
                    if (j == Ny - 2) Vx_out[ac + (Ny - j0) * ldi] = 0.f;
                }
                if (j == 0 || j == Ny - 2) {
                    int br = (j == 0) ? -j0 : Ny - 1 - j0;
                    Vy_out[(a + 1) + br * ldi] = 0.f;
                    if (i == 0) Vy_out[-i0 + br * ldi] = 0.f;
                    if (i == Nx - 2) Vy_out[Nx - i0 + br * ldi] = 0.f;
                }
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

// max |Vx|, |Vy| per tile of V = V64 + correction, the velocity the next fold stores (compute_dt's maxima;
// ghost entries repeat interior values or are 0).  Before an instance's first sweeps the correction is zero.
__global__ void __launch_bounds__(T64) k_maxv64(const Inst* __restrict__ insts, const Ctl* __restrict__ ctl,
                                               const int2* __restrict__ tiles, double* __restrict__ part) {
    __shared__ double sh[T64 / 32];
    const int2 td = tiles[blockIdx.x];
    const Inst& I = insts[td.x];
    const int i0 = (td.y % I.ntx) * BX, j0 = (td.y / I.ntx) * BY64;
    const double* Vx = gd(I, D_VX);
    const double* Vy = gd(I, D_VY);
    const int cur = ctl[td.x].parity & 1;
    const float* cvx = gf(I, cur ? G_VXB : G_VXA);
    const float* cvy = gf(I, cur ? G_VYB : G_VYA);
    double mx = 0.0, my = 0.0;
    for (int k = threadIdx.x; k < BX * BY64; k += T64) {
        const int i = i0 + (k % BX), j = j0 + (k / BX);
        const int64_t o = (i + 1) + (int64_t)(j + 1) * I.LD64;
        if (i < I.Nx - 2 && j < I.Ny - 1) mx = fmax(mx, fabs(Vx[o] + (double)cvx[o]));
        if (i < I.Nx - 1 && j < I.Ny - 2) my = fmax(my, fabs(Vy[o] + (double)cvy[o]));
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
    const int i0 = (td.y % I.ntx) * BX, j0 = (td.y / I.ntx) * BY64;
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
    for (int k = threadIdx.x; k < BX * BY64; k += T64) {
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

// The residual check of the reference's loop at an iteration n that is a multiple of ncheck (:64-73, kernels
// :140-202 and :241-249), evaluated before the fold from the FP64 state plus the two correction buffers:
// divV and tau are those of compute_P_tau! in iteration n, i.e. of V_{n-1} (= V64 + the previous correction);
// P is P_n (= P64 + the current correction); the stabilisation term of Ry uses V_n and dt_check =
// compute_dt(V_n) (Inst::dt_cfl, computed just before).  Per-tile sums of |Rx|, |Ry|, |divV| -> part.  Tiles of
// instances without a check this round leave at once.
__global__ void __launch_bounds__(T64) k_check64(const Inst* __restrict__ insts, const Ctl* __restrict__ ctl,
                                                const int2* __restrict__ tiles, double* __restrict__ part) {
    __shared__ double sh[T64 / 32];
    const int2 td = tiles[blockIdx.x];
    const Ctl c = ctl[td.x];
    if (!(c.flags & CTL_CHECK)) return;
    const Inst& I = insts[td.x];
    const int Nx = I.Nx, Ny = I.Ny;
    const int i0 = (td.y % I.ntx) * BX, j0 = (td.y / I.ntx) * BY64;
    const int64_t L = I.LD64;
    const double* Vx = gd(I, D_VX);
    const double* Vy = gd(I, D_VY);
    const double* P = gd(I, D_P);
    const double* rho = gd(I, D_RHO);
    const double* mub = gd(I, D_MUB);
    const double* mup = gd(I, D_MUP);
    const int cur = c.parity & 1;
    const float* cvx = gf(I, cur ? G_VXB : G_VXA);
    const float* cvy = gf(I, cur ? G_VYB : G_VYA);
    const float* cp = gf(I, cur ? G_PB : G_PA);
    const float* pvx = gf(I, cur ? G_VXA : G_VXB);
    const float* pvy = gf(I, cur ? G_VYA : G_VYB);
    const double _dx = I._dx, _dy = I._dy;
    const double dt = I.use_stab ? I.dt_cfl : 0.0;
    // V_{n-1}, V_n and P_n at an offset (the FP32 and FP64 fields share i + j * LD)
    auto vxp = [&](int64_t o) { return Vx[o] + (double)pvx[o]; };
    auto vyp = [&](int64_t o) { return Vy[o] + (double)pvy[o]; };
    auto vxc = [&](int64_t o) { return Vx[o] + (double)cvx[o]; };
    auto vyc = [&](int64_t o) { return Vy[o] + (double)cvy[o]; };
    auto pc = [&](int64_t o) { return P[o] + (double)cp[o]; };
    auto div_at = [&](int i, int j, double* dvx, double* dvy) {
        *dvx = (vxp((i + 1) + (int64_t)(j + 1) * L) - vxp(i + (int64_t)(j + 1) * L)) * _dx;
        *dvy = (vyp((i + 1) + (int64_t)(j + 1) * L) - vyp((i + 1) + (int64_t)j * L)) * _dy;
        return *dvx + *dvy;
    };
    auto txx_at = [&](int i, int j, double* tyy) {
        double dVx_dx, dVy_dy;
        const double d = div_at(i, j, &dVx_dx, &dVy_dy);
        const double mu = mup[i + (int64_t)j * L];
        *tyy = 2.0 * mu * (dVy_dy - 1.0 / 3.0 * d);
        return 2.0 * mu * (dVx_dx - 1.0 / 3.0 * d);
    };
    auto txy_at = [&](int i, int j) {
        const double dVx_dy = (vxp(i + (int64_t)(j + 1) * L) - vxp(i + (int64_t)j * L)) * _dy;
        const double dVy_dx = (vyp((i + 1) + (int64_t)j * L) - vyp(i + (int64_t)j * L)) * _dx;
        return 2.0 * mub[i + (int64_t)j * L] * 0.5 * (dVx_dy + dVy_dx);
    };
    double srx = 0.0, sry = 0.0, sdv = 0.0;
    for (int k = threadIdx.x; k < BX * BY64; k += T64) {
        const int i = i0 + (k % BX), j = j0 + (k / BX);
        if (i >= Nx - 1 || j >= Ny - 1) continue;
        const int64_t o = i + (int64_t)j * L;
        double dvx, dvy, tyy0;
        sdv += fabs(div_at(i, j, &dvx, &dvy));
        const double txx0 = txx_at(i, j, &tyy0);
        if (i < Nx - 2) {
            double tyy1;
            const double txx1 = txx_at(i + 1, j, &tyy1);
            const double R = (txx1 - txx0) * _dx + (txy_at(i + 1, j + 1) - txy_at(i + 1, j)) * _dy -
                             (pc(o + 1) - pc(o)) * _dx;
            srx += fabs(R);
        }
        if (j < Ny - 2) {
            double tyy1;
            (void)txx_at(i, j + 1, &tyy1);
            const double av = 0.25 * (vxc(i + (int64_t)(j + 1) * L) + vxc((i + 1) + (int64_t)(j + 1) * L) +
                                      vxc(i + (int64_t)(j + 2) * L) + vxc((i + 1) + (int64_t)(j + 2) * L));
            const double dxr = rho[(i + 2) + (int64_t)(j + 1) * L] - rho[i + (int64_t)(j + 1) * L];
            const double dyr = rho[(i + 1) + (int64_t)(j + 2) * L] - rho[(i + 1) + (int64_t)j * L];
            const double R = (tyy1 - tyy0) * _dy + (txy_at(i + 1, j + 1) - txy_at(i, j + 1)) * _dx -
                             (pc(o + L) - pc(o)) * _dy +
                             I.g_y * (rho[(i + 1) + (int64_t)(j + 1) * L] -
                                      dt * (av * dxr * 0.5 * _dx + vyc((i + 1) + (int64_t)(j + 1) * L) * dyr * 0.5 * _dy));
            sry += fabs(R);
        }
    }
    double a = blk_sum(srx, sh), b = blk_sum(sry, sh), cc = blk_sum(sdv, sh);
    if (threadIdx.x == 0) {
        part[3 * blockIdx.x] = a;
        part[3 * blockIdx.x + 1] = b;
        part[3 * blockIdx.x + 2] = cc;
    }
}

// per-instance reductions over the instance's contiguous range of tile partials
struct Seg { int inst, begin, end, pad_; };

// compute_dt (:118-121) of the velocity the fold stores -> Inst::dt_cfl (the check's dt_check and the solve's
// returned dt); at an ndtupdate event (:60-62) it also becomes the stabilisation dt of the iterations that
// follow.  The reference keeps the dt it was called with until then.
__global__ void k_inst_dt(Inst* __restrict__ insts, const Ctl* __restrict__ ctl, const Seg* __restrict__ segs,
                          const double* __restrict__ part) {
    __shared__ double sh[32];
    const Seg g = segs[blockIdx.x];
    double mx = 0.0, my = 0.0;
    for (int t = g.begin + threadIdx.x; t < g.end; t += blockDim.x) {
        mx = fmax(mx, part[2 * t]);
        my = fmax(my, part[2 * t + 1]);
    }
    double a = blk_max(mx, sh), b = blk_max(my, sh);
    if (threadIdx.x == 0) {
        Inst& I = insts[g.inst];
        double x = I.dx / a, y = I.dy / b;
        double m = (y < x) ? y : x;
        if (x != x) m = x;
        if (y != y) m = y;
        I.dt_cfl = I.maxdisp * m;
        // while V is exactly zero the CFL dt is infinite: the stabilisation then keeps its dt
        if ((ctl[g.inst].flags & CTL_DT) && I.use_stab && isfinite(I.dt_cfl)) {
            I.dt = I.dt_cfl;
            I.g_dtf = (float)(I.g_y * I.dt);
        }
    }
}

// err = max of the three means (compute_err, :103-109) of a sum triple
__device__ __forceinline__ double err_of(const Inst& I, double a, double b, double c) {
    const double nrx = (double)(I.Nx - 2) * (I.Ny - 1), nry = (double)(I.Nx - 1) * (I.Ny - 2),
                 ndv = (double)(I.Nx - 1) * (I.Ny - 1);
    double m = a / nrx;
    const double bb = b / nry, cc = c / ndv;
    if (bb > m || bb != bb) m = bb;
    if (cc > m || cc != cc) m = cc;
    if (a != a) m = a;
    return m;
}

// per instance of the round -> out[4 q ..] = {err of the folded state (its residual, which is the constant term of
// the next sweeps; a non-finite value ends the solve), residual scale, dt_cfl, err of the reference's check (when
// the round ended on one, else 0)}
__global__ void k_inst_err(const Seg* __restrict__ segs, const double* __restrict__ part,
                           const double* __restrict__ part_check, const Inst* __restrict__ insts,
                           const Ctl* __restrict__ ctl, const double* __restrict__ scale, double* __restrict__ out) {
    __shared__ double sh[32];
    const Seg g = segs[blockIdx.x];
    const bool check = (ctl[g.inst].flags & CTL_CHECK) != 0;
    double s[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int t = g.begin + threadIdx.x; t < g.end; t += blockDim.x)
        for (int k = 0; k < 3; ++k) {
            s[k] += part[3 * t + k];
            if (check) s[3 + k] += part_check[3 * t + k];
        }
    double r[6];
    for (int k = 0; k < 6; ++k) r[k] = blk_sum(s[k], sh);
    if (threadIdx.x == 0) {
        const Inst& I = insts[g.inst];
        out[4 * blockIdx.x] = err_of(I, r[0], r[1], r[2]);
        out[4 * blockIdx.x + 1] = scale[g.inst];
        out[4 * blockIdx.x + 2] = I.dt_cfl;
        out[4 * blockIdx.x + 3] = check ? err_of(I, r[3], r[4], r[5]) : 0.0;
    }
}

// V += dV, P += dP (FP64 += FP32) over an instance's padded arrays, then zero the correction.  The damped
// rates are kept: folding the correction into the FP64 state and re-anchoring the constant term on the FP64
// residual leaves the PT iteration itself unchanged (in exact arithmetic it is the FP64 iteration), so its
// accumulated momentum stays valid.  The other correction buffer (the previous iterate's) is left as it is:
// the next sweep overwrites it.  blockIdx.y = position in the instance list.
__global__ void k_accumulate(const Inst* __restrict__ insts, const Ctl* __restrict__ ctl, const int* __restrict__ list) {
    const int q = list[blockIdx.y];
    const Inst& I = insts[q];
    const int cur = ctl[q].parity & 1;
    const int64_t n = I.LD32 * I.rows;  // every entry; the FP64 and FP32 fields share (i, j) -> i + j*LD
    float* cvx = gf(I, cur ? G_VXB : G_VXA);
    float* cvy = gf(I, cur ? G_VYB : G_VYA);
    float* cp = gf(I, cur ? G_PB : G_PA);
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
}

__global__ void k_f32_to_f64(double* __restrict__ dst, int64_t ld_dst, const float* __restrict__ src, int64_t ld_src,
                             int64_t nx, int64_t ny) {
    int64_t n = nx * ny;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        int64_t i = k % nx, j = k / nx;
        dst[i + j * ld_dst] = (double)src[i + j * ld_src];
    }
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
// host side: the resident engine
// ===========================================================================
namespace sf {
namespace mx {

static unsigned grid1(int64_t n, int per) { return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + per - 1) / per, 65535)); }

// The sweep shapes the autotuner chooses from: tile rows, and the CTAs per SM that the register budget is
// sized for (the shared memory of a CTA grows with the rows: 31, 56 and 105 KB).
typedef void (*SweepKernel)(const CUtensorMap*, const Inst*, const Ctl*, const int2*, const int*, int, int, int*);
struct SweepShape {
    int rows, minb, smem;
    SweepKernel kern;
};
static const SweepShape kShapes[] = {
    {8, 4, Shape<8>::SMEM_BYTES, k_pt32<8, 4>},
    {16, 4, Shape<16>::SMEM_BYTES, k_pt32<16, 4>},
    {32, 2, Shape<32>::SMEM_BYTES, k_pt32<32, 2>},
};
constexpr int NSHAPES = (int)(sizeof(kShapes) / sizeof(kShapes[0]));
// tile schedules of the persistent sweep kernel: 0 strided, 1 chunked (the kernel's `chunked` argument)
constexpr int NSCHED = 2;
// sweep launches: 0 serialised, 1 overlapped (programmatic dependent launch: a sweep launches and fences its
// first maps while the previous one drains, and waits in the kernel for its results)
constexpr int NLAUNCH = 2;
// the tuner's candidates: shape k, schedule c, launch mode o is candidate (k * NSCHED + c) * NLAUNCH + o
constexpr int NCAND = NSHAPES * NSCHED * NLAUNCH;
static_assert(NCAND == 12, "sf_engine_stats.tune_ns has one entry per candidate");
constexpr int cand_of(int k, int c, int o) { return (k * NSCHED + c) * NLAUNCH + o; }
constexpr int DEFAULT_SHAPE = 1;                      // 32 x 16 rows ...
constexpr int DEFAULT_CAND = cand_of(DEFAULT_SHAPE, 1, 0);  // ... chunked, serialised, until measured
constexpr int TUNE_PASSES = 2;                        // timed pieces per candidate; the fastest counts

static int shape_of_rows(int rows) {
    for (int k = 0; k < NSHAPES; ++k)
        if (kShapes[k].rows == rows) return k;
    return -1;
}

// resident CTAs per SM of each shape on a device (0: not yet queried); the attribute is set per device
static int shape_per_sm(int device, int k, int* out) {
    static int cache[64][NSHAPES] = {};
    if (device < 0 || device >= 64) return fail(SF_ERR_INVALID_ARG, "sf_engine: device index");
    if (!cache[device][k]) {
        const SweepShape& sh = kShapes[k];
        SF_CUDA(cudaFuncSetAttribute((const void*)sh.kern, cudaFuncAttributeMaxDynamicSharedMemorySize, sh.smem));
        int n = 0;
        SF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, (const void*)sh.kern, NT, sh.smem));
        if (n < 1) return fail(SF_ERR_CUDA, "k_pt32 does not fit on an SM");
        cache[device][k] = n;
    }
    *out = cache[device][k];
    return SF_OK;
}

// arena bytes of one instance: FP32 fields, then FP64 fields, each 256-byte aligned
struct Layout {
    int64_t LD, rows, fstride, bytes32, bytes64;
    Layout(int64_t Nx, int64_t Ny) {
        LD = round_up(Nx + 4, 32);
        rows = Ny + 3;
        fstride = LD * rows;
        bytes32 = round_up((int64_t)G_NUM * fstride * 4, 256);
        bytes64 = round_up((int64_t)D_NUM * fstride * 8, 256);
    }
    int64_t bytes() const { return bytes32 + bytes64; }
};

// first-fit allocator over [0, cap) (offsets and sizes multiples of 256), coalescing on release
class ArenaAlloc {
   public:
    void reset(int64_t cap) {
        free_.clear();
        if (cap > 0) free_[0] = cap;
        cap_ = cap;
        used_ = 0;
    }
    int64_t alloc(int64_t bytes) {
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < bytes) continue;
            const int64_t off = it->first, rest = it->second - bytes;
            free_.erase(it);
            if (rest > 0) free_[off + bytes] = rest;
            used_ += bytes;
            peak_ = std::max(peak_, used_);
            return off;
        }
        return -1;
    }
    void release(int64_t off, int64_t bytes) {
        used_ -= bytes;
        auto it = free_.emplace(off, bytes).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
    int64_t cap() const { return cap_; }
    int64_t used() const { return used_; }
    int64_t peak() const { return peak_; }

   private:
    std::map<int64_t, int64_t> free_;
    int64_t cap_ = 0, used_ = 0, peak_ = 0;
};

struct Slot {  // an admitted instance
    sf_batch_instance* user = nullptr;
    int64_t ticket = -1;
    Inst d;                    // source of the device record
    int64_t ntiles[NSHAPES] = {};  // sweep tiles in each shape
    int64_t ntiles64 = 0;      // FP64-kernel tiles
    int64_t off = 0, bytes = 0;
    bool active = false;
    bool swept = false;        // ran sweeps since its last fold
    int budget = 0;            // sweeps of its last round
    int64_t ncheck = 0, ndtupdate = 0;   // the reference's event periods for this grid (:35-36)
    int64_t base = 0;          // inner_total when the current attempt started (a retry starts a new schedule)
    int64_t inner_total = 0, outer = 0;
    double err = 0.0, eps = 0.0;   // err of the last residual check (2 eps before the first, as :40)
    std::chrono::steady_clock::time_point t_submit;
};

static sf_mixed_options normalized(const sf_mixed_options* o) {
    sf_mixed_options r{};
    if (o) {
        r = *o;
    } else {
        r.max_sweeps = 4000000;
        r.fold_every = 400;
        r.use_graphs = 1;
        r.dtau_local_max = 0;
        r.retry_local_max = 1;
        r.tile_rows = 0;
        r.tile_schedule = 0;
        r.overlap_launches = 0;
    }
    if (r.fold_every < 2) r.fold_every = 2;
    r.fold_every &= ~1;  // even: the trial pieces of the tuner run in pairs of sweeps
    return r;
}

}  // namespace mx
}  // namespace sf

using namespace sf;
using namespace sf::mx;

struct sf_engine {
    sf_ctx* ctx = nullptr;
    sf_mixed_options opt{};
    cudaStream_t s = nullptr;            // own non-blocking stream (graph capture needs one)
    unsigned char* arena = nullptr;
    bool arena_owned = false;
    ArenaAlloc alloc;
    std::vector<Slot> slots;
    std::vector<int> free_slots;
    // device tables, one allocation: insts | ctl | maps | segs | out | scale | list | ntiles | flag
    void* tables = nullptr;
    Inst* d_insts = nullptr;
    Ctl* d_ctl = nullptr;                // per-slot control words, uploaded from h_ctl before the kernels read them
    std::vector<Ctl> h_ctl;
    CUtensorMap* d_maps = nullptr;       // [shape][slot][M_NUM]: every slot's maps for every shape
    Seg* d_segs = nullptr;
    double* d_out = nullptr;
    double* d_scale = nullptr;
    int* d_list = nullptr;
    int* d_ntiles = nullptr;             // [shape]
    int* d_flag = nullptr;               // a bounded wait of k_pt32 gave up
    double* h_out = nullptr;             // pinned mirror of d_out
    // the sweep tile list (current shape), and the FP64-kernel tile list with its per-tile partials; grown on demand
    int2* d_tiles[NSHAPES] = {};         // one sweep list per shape (tile counts differ)
    int64_t tile_cap[NSHAPES] = {};
    int2* d_tiles64 = nullptr;
    double* d_part = nullptr;            // 3 per tile: max|V| pairs, then the folded residual's sums ...
    double* d_part_check = nullptr;      // ... and 3 per tile for the check's sums (same allocation)
    int64_t tile64_cap = 0;
    std::vector<int2> h_tiles;
    std::vector<Seg> h_segs;
    int h_ntiles[NSHAPES] = {};          // sources of the tile-count uploads
    std::vector<int2> h_list[NSHAPES];   // sources of the sweep-list uploads
    // one captured run of fold_every sweeps per candidate (shape x schedule), kept while its pointers hold
    cudaGraph_t graph[NCAND] = {};
    cudaGraphExec_t gexec[NCAND] = {};
    int graph_k[NCAND] = {};
    int blocks = 0;                      // persistent CTAs of the current shape
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;
    // the sweep candidate in use (shape, schedule, launch mode) and its tuner: the first round of a workload
    // class the context has not seen starts with short timed pieces of every candidate on the engine stream; the
    // candidate with the fewest ns per point-sweep is then used and recorded in the context for that class
    int shape = DEFAULT_SHAPE;
    int sched = 0;
    int overlap = 0;
    int tune_state = SF_TUNE_MEASURING;
    int tune_trials = 0;                 // pieces timed so far for the class being measured
    int tune_key = -1;                   // workload class of the current sweep set
    double tune_ns[NCAND] = {};          // the last completed measurement, ns per point-sweep (0: not measured)
    int timed_first = 0;                 // the last round timed trials timed_first ...
    int timed_pieces = 0;                // ... up to timed_first + timed_pieces - 1 (candidate = trial % NCAND),
    double timed_points = 0.0;           // each piece over this many point-sweeps
    cudaEvent_t ev_piece[NCAND * TUNE_PASSES + 1] = {};
    int64_t next_ticket = 0, submitted = 0, finished = 0, rounds = 0, sweeps = 0;
    int64_t tune_rounds = 0, tune_hits = 0;   // measuring rounds; class changes answered from the context
    double trial_ns[NCAND] = {};         // the measurement in progress (tune_ns: the last completed one)
    std::deque<int64_t> pending;
};

namespace {

CUtensorMap* maps_of(sf_engine* e, int k) { return e->d_maps + (size_t)k * e->slots.size() * M_NUM; }

void drop_graph(sf_engine* e, int c) {
    if (e->gexec[c]) cudaGraphExecDestroy(e->gexec[c]);
    if (e->graph[c]) cudaGraphDestroy(e->graph[c]);
    e->gexec[c] = nullptr;
    e->graph[c] = nullptr;
}

void drop_graph(sf_engine* e) {
    for (int c = 0; c < NCAND; ++c) drop_graph(e, c);
}

void engine_free(sf_engine* e) {
    if (!e) return;
    if (e->s) cudaStreamSynchronize(e->s);
    drop_graph(e);
    if (e->tables) cudaFree(e->tables);
    for (int2* t : e->d_tiles)
        if (t) cudaFree(t);
    if (e->d_tiles64) cudaFree(e->d_tiles64);
    if (e->d_part) cudaFree(e->d_part);
    if (e->h_out) cudaFreeHost(e->h_out);
    if (e->arena_owned && e->arena) cudaFree(e->arena);
    if (e->ev_in) cudaEventDestroy(e->ev_in);
    if (e->ev_out) cudaEventDestroy(e->ev_out);
    for (cudaEvent_t ev : e->ev_piece)
        if (ev) cudaEventDestroy(ev);
    if (e->s) cudaStreamDestroy(e->s);
    delete e;
}

int configure_tuner(sf_engine* e);

int engine_init(sf_engine* e, sf_ctx* ctx, int slot_cap, const sf_mixed_options* o) {
    e->ctx = ctx;
    e->opt = normalized(o);
    SF_CUDA(cudaStreamCreateWithFlags(&e->s, cudaStreamNonBlocking));
    SF_CUDA(cudaEventCreateWithFlags(&e->ev_in, cudaEventDisableTiming));
    SF_CUDA(cudaEventCreateWithFlags(&e->ev_out, cudaEventDisableTiming));
    for (cudaEvent_t& ev : e->ev_piece) SF_CUDA(cudaEventCreate(&ev));
    const size_t n = (size_t)slot_cap;
    const size_t o_ins = 0, o_ctl = round_up(o_ins + n * sizeof(Inst), 256);
    const size_t o_map = round_up(o_ctl + n * sizeof(Ctl), 256);
    const size_t o_seg = round_up(o_map + (size_t)NSHAPES * n * M_NUM * sizeof(CUtensorMap), 256);
    const size_t o_out = round_up(o_seg + n * sizeof(Seg), 256);
    const size_t o_scl = round_up(o_out + n * 4 * 8, 256);
    const size_t o_lst = round_up(o_scl + n * 8, 256);
    const size_t o_nt = round_up(o_lst + n * 4, 256);
    const size_t o_flg = o_nt + 128;
    const size_t total = o_flg + 128;
    if (cudaMalloc(&e->tables, total) != cudaSuccess) {
        cudaGetLastError();
        return fail(SF_ERR_OOM, "sf_engine: device tables");
    }
    unsigned char* b = (unsigned char*)e->tables;
    e->d_insts = (Inst*)(b + o_ins);
    e->d_ctl = (Ctl*)(b + o_ctl);
    e->d_maps = (CUtensorMap*)(b + o_map);
    e->d_segs = (Seg*)(b + o_seg);
    e->d_out = (double*)(b + o_out);
    e->d_scale = (double*)(b + o_scl);
    e->d_list = (int*)(b + o_lst);
    e->d_ntiles = (int*)(b + o_nt);
    e->d_flag = (int*)(b + o_flg);
    SF_CUDA(cudaMemsetAsync(e->tables, 0, total, e->s));
    SF_CUDA(cudaMallocHost(&e->h_out, n * 4 * 8 + 64));  // 4 results per slot (k_inst_err), then the flag word
    e->slots.assign(n, Slot{});
    e->h_ctl.assign(n, Ctl{0, 0, 0, 0});
    e->free_slots.clear();
    for (int k = slot_cap - 1; k >= 0; --k) e->free_slots.push_back(k);
    return configure_tuner(e);
}

// grows a device tile list (and, for the FP64 list, its per-tile partials: 6 per tile)
int grow_list(sf_engine* e, int64_t need, int2** tiles, double** part, int64_t* cap_io) {
    if (need <= *cap_io) return SF_OK;
    const int64_t cap = std::max<int64_t>({need, 2 * *cap_io, 4096});
    SF_CUDA(cudaStreamSynchronize(e->s));  // the old list may still be read by queued kernels
    if (*tiles) cudaFree(*tiles);
    if (part && *part) cudaFree(*part);
    *tiles = nullptr;
    if (part) *part = nullptr;
    *cap_io = 0;
    if (cudaMalloc(tiles, (size_t)cap * sizeof(int2)) != cudaSuccess ||
        (part && cudaMalloc(part, (size_t)cap * 6 * 8) != cudaSuccess)) {
        cudaGetLastError();
        return fail(SF_ERR_OOM, "sf_engine: tile list");
    }
    *cap_io = cap;
    if ((int64_t)e->h_tiles.size() < cap) e->h_tiles.resize((size_t)cap);
    return SF_OK;
}

// FP64-kernel tile list + segments of the slots in `ids` -> device; returns the tile count in *nt_out
int upload_lists64(sf_engine* e, const std::vector<int>& ids, int64_t* nt_out) {
    int64_t nt = 0;
    for (int q : ids) nt += e->slots[q].ntiles64;
    int rc = grow_list(e, nt, &e->d_tiles64, &e->d_part, &e->tile64_cap);
    if (rc) return rc;
    e->d_part_check = e->d_part + 3 * e->tile64_cap;
    e->h_segs.resize(ids.size());
    int64_t k = 0;
    for (size_t q = 0; q < ids.size(); ++q) {
        const Slot& h = e->slots[ids[q]];
        e->h_segs[q] = Seg{ids[q], (int)k, (int)(k + h.ntiles64), 0};
        for (int64_t t = 0; t < h.ntiles64; ++t) e->h_tiles[k++] = make_int2(ids[q], (int)t);
    }
    // pageable sources: the copies are staged before cudaMemcpyAsync returns, so the host vectors are free again
    SF_CUDA(cudaMemcpyAsync(e->d_tiles64, e->h_tiles.data(), (size_t)nt * sizeof(int2), cudaMemcpyHostToDevice, e->s));
    SF_CUDA(cudaMemcpyAsync(e->d_segs, e->h_segs.data(), ids.size() * sizeof(Seg), cudaMemcpyHostToDevice, e->s));
    *nt_out = nt;
    return SF_OK;
}

// sweep tile list of the slots in `ids` for shape k, and its length -> device
int upload_sweep_list(sf_engine* e, const std::vector<int>& ids, int k) {
    int64_t nt = 0;
    for (int q : ids) nt += e->slots[q].ntiles[k];
    if (nt > e->tile_cap[k])  // the shape's graphs hold the old pointer
        for (int c = cand_of(k, 0, 0); c < cand_of(k + 1, 0, 0); ++c) drop_graph(e, c);
    int rc = grow_list(e, nt, &e->d_tiles[k], nullptr, &e->tile_cap[k]);
    if (rc) return rc;
    std::vector<int2>& h = e->h_list[k];
    h.resize((size_t)nt);
    int64_t n = 0;
    for (int q : ids)
        for (int64_t t = 0; t < e->slots[q].ntiles[k]; ++t) h[(size_t)n++] = make_int2(q, (int)t);
    SF_CUDA(cudaMemcpyAsync(e->d_tiles[k], h.data(), (size_t)nt * sizeof(int2), cudaMemcpyHostToDevice, e->s));
    e->h_ntiles[k] = (int)nt;
    SF_CUDA(cudaMemcpyAsync(e->d_ntiles + k, &e->h_ntiles[k], sizeof(int), cudaMemcpyHostToDevice, e->s));
    return SF_OK;
}

// sweep tilings of slot q: its tile count and its 2 tensor maps (box = tile + halo, or tile) in every shape,
// encoded once at admission, so that a change of shape is a choice of pointers
int encode_maps(sf_engine* e, int q) {
    Slot& h = e->slots[q];
    const Inst& I = h.d;
    CUtensorMap maps[M_NUM];
    for (int k = 0; k < NSHAPES; ++k) {
        const int rows = kShapes[k].rows;
        h.ntiles[k] = (int64_t)I.ntx * ceil_div(I.Ny - 1, rows);
        int rc = encode_tmap_f32_fields(&maps[M_HALO], I.f32, I.LD32, I.rows, G_NUM, I.fstride32, TW, rows + 2);
        if (rc || (rc = encode_tmap_f32_fields(&maps[M_TILE], I.f32, I.LD32, I.rows, G_NUM, I.fstride32, BX, rows)))
            return rc;
        // pageable source: staged before the call returns, so `maps` is free again
        SF_CUDA(cudaMemcpyAsync(maps_of(e, k) + (size_t)q * M_NUM, maps, sizeof(maps), cudaMemcpyHostToDevice, e->s));
    }
    return SF_OK;
}

// switches the sweeps to a candidate: its shape k (persistent grid size; the maps and lists are per shape),
// schedule and launch mode
int use_cand(sf_engine* e, int cand) {
    const int k = cand / (NSCHED * NLAUNCH), c = (cand / NLAUNCH) % NSCHED;
    e->overlap = cand % NLAUNCH;
    int per_sm = 0;
    int rc = shape_per_sm(e->ctx->device, k, &per_sm);
    if (rc) return rc;
    const int blocks = per_sm * e->ctx->num_sms;  // persistent: one wave; CTAs beyond the tile count exit at once
    e->shape = k;  // each candidate's graph was captured with its own grid, maps and list
    e->sched = c;
    e->blocks = blocks;
    return SF_OK;
}

// the caller's tile_rows (and tile_schedule) fix the sweeps; tile_rows 0 lets the tuner choose both
int configure_tuner(sf_engine* e) {
    int cand = DEFAULT_CAND;
    const int sc = e->opt.tile_schedule, ov = e->opt.overlap_launches;
    if (e->opt.tile_rows != 0) {
        const int k = shape_of_rows(e->opt.tile_rows);
        if (k < 0) return fail(SF_ERR_INVALID_ARG, "sf_mixed_options.tile_rows must be 0, 8, 16 or 32");
        if (sc < 0 || sc > NSCHED) return fail(SF_ERR_INVALID_ARG, "sf_mixed_options.tile_schedule must be 0, 1 or 2");
        if (ov < 0 || ov > 1) return fail(SF_ERR_INVALID_ARG, "sf_mixed_options.overlap_launches must be 0 or 1");
        cand = cand_of(k, sc == 2 ? 1 : 0, ov);
        e->tune_state = SF_TUNE_FIXED;
    } else {
        if (sc != 0 || ov != 0)
            return fail(SF_ERR_INVALID_ARG, "sf_mixed_options.tile_schedule and overlap_launches need tile_rows");
        e->tune_state = SF_TUNE_MEASURING;
    }
    e->tune_trials = 0;
    e->tune_key = -1;
    e->timed_pieces = 0;
    e->tune_rounds = e->tune_hits = 0;
    for (double& v : e->tune_ns) v = 0.0;
    for (double& v : e->trial_ns) v = 0.0;
    return use_cand(e, cand);
}

// workload class of a sweep set: half-octaves of the mean points per instance, octaves of the total points
int workload_key(const sf_engine* e, const std::vector<int>& ids, double* points) {
    double tot = 0.0;
    for (int q : ids) tot += (double)(e->slots[q].d.Nx - 1) * (e->slots[q].d.Ny - 1);
    *points = tot;
    const int a = (int)std::floor(2.0 * std::log2(std::max(1.0, tot / (double)ids.size())));
    const int b = (int)std::floor(std::log2(std::max(1.0, tot)));
    return a * 128 + b;
}

// reads the timings of the last round's trial pieces (the stream has been synchronised); once every candidate
// has had TUNE_PASSES pieces, keeps the fastest and records it for the workload class
int tuner_collect(sf_engine* e) {
    if (e->timed_pieces == 0) return SF_OK;
    for (int i = 0; i < e->timed_pieces; ++i) {
        float ms = 0.f;
        SF_CUDA(cudaEventElapsedTime(&ms, e->ev_piece[i], e->ev_piece[i + 1]));
        const double ns = (double)ms * 1e6 / std::max(1.0, e->timed_points);
        double& seen = e->trial_ns[(e->timed_first + i) % NCAND];
        if (seen == 0.0 || ns < seen) seen = ns;
    }
    e->tune_trials += e->timed_pieces;
    e->timed_pieces = 0;
    if (e->tune_trials < NCAND * TUNE_PASSES) return SF_OK;
    int best = DEFAULT_CAND;
    for (int k = 0; k < NCAND; ++k)
        if (e->trial_ns[k] > 0.0 && e->trial_ns[k] < e->trial_ns[best]) best = k;
    for (int k = 0; k < NCAND; ++k) e->tune_ns[k] = e->trial_ns[k];
    e->tune_state = SF_TUNE_MEASURED;
    e->ctx->sweep_shapes[e->tune_key] = best;
    return use_cand(e, best);
}

// `n` sweeps (launch indices k0, k0 + 1, ... of the round) over the uploaded sweep list of the current shape
int launch_direct(sf_engine* e, int k0, int n) {
    const int sk = e->shape;
    const SweepShape& sh = kShapes[sk];
    // overlapped: each sweep may launch while the previous one drains; it waits in the kernel for its results
    for (int k = k0; k < k0 + n; ++k)
        SF_CUDA(launch_overlapped(e->overlap != 0, sh.kern, dim3(e->blocks), dim3(BX, TY), (size_t)sh.smem, e->s,
                                  maps_of(e, sk), (const Inst*)e->d_insts, (const Ctl*)e->d_ctl,
                                  (const int2*)e->d_tiles[sk], (const int*)(e->d_ntiles + sk), k, e->sched,
                                  e->d_flag));
    return SF_OK;
}

// a measuring round: its first sweeps run as short timed pieces, one per trial still to run (P sweeps each, P
// even so that the launch parities run on), the rest in the default candidate; all launched directly, after
// the lists of every shape are uploaded, so that nothing but sweeps lies between the events.  The pieces stay
// within the smallest budget of the round, so each covers every instance of the set.
int launch_trials(sf_engine* e, const std::vector<int>& ids, double points) {
    const int K = e->opt.fold_every;
    const int P = std::min(8, std::max(2, (K / (2 * NCAND)) & ~1));
    int min_budget = K;
    for (int q : ids) min_budget = std::min(min_budget, e->slots[q].budget);
    const int pieces = std::min(NCAND * TUNE_PASSES - e->tune_trials, min_budget / P);
    const int prev = cand_of(e->shape, e->sched, e->overlap);
    int rc, k = 0;
    ++e->tune_rounds;
    for (int sk = 0; sk < NSHAPES; ++sk)
        if ((rc = upload_sweep_list(e, ids, sk))) return rc;
    SF_CUDA(cudaEventRecord(e->ev_piece[0], e->s));
    for (int i = 0; i < pieces; ++i, k += P) {
        const int cand = (e->tune_trials + i) % NCAND;
        if ((rc = use_cand(e, cand))) return rc;
        if ((rc = launch_direct(e, k, P))) return rc;
        SF_CUDA(cudaEventRecord(e->ev_piece[i + 1], e->s));
    }
    e->timed_first = e->tune_trials;
    e->timed_pieces = pieces;
    e->timed_points = points * P;
    if (k < K) {  // the rest in the choice made before (the previous class's, or the default)
        if ((rc = use_cand(e, prev))) return rc;
        if ((rc = launch_direct(e, k, K - k))) return rc;
    }
    return SF_OK;
}

// one fold's worth of sweeps over the sweep set `ids`, in the shape the tuner (or the caller) chose
int launch_sweeps(sf_engine* e, const std::vector<int>& ids) {
    const int K = e->opt.fold_every;
    int rc;
    if (e->tune_state != SF_TUNE_FIXED) {
        // the workload class of this round's sweep set; a new class takes the context's recorded choice, or
        // is measured now (a batch that drains and a serving mix move through classes)
        double points = 0.0;
        const int key = workload_key(e, ids, &points);
        if (key != e->tune_key) {
            e->tune_key = key;
            e->tune_trials = 0;
            for (double& v : e->trial_ns) v = 0.0;
            auto it = e->ctx->sweep_shapes.find(key);
            if (it != e->ctx->sweep_shapes.end()) {
                e->tune_state = SF_TUNE_CACHED;
                ++e->tune_hits;
                if ((rc = use_cand(e, it->second))) return rc;
            } else {
                e->tune_state = SF_TUNE_MEASURING;
            }
        }
        if (e->tune_state == SF_TUNE_MEASURING) {
            if ((rc = launch_trials(e, ids, points))) return rc;
            e->ctx->launches += K;
            e->sweeps += K;
            return SF_OK;
        }
    }
    if ((rc = upload_sweep_list(e, ids, e->shape))) return rc;
    if (e->opt.use_graphs) {
        const int c = cand_of(e->shape, e->sched, e->overlap);
        if (e->gexec[c] && e->graph_k[c] != K) drop_graph(e, c);
        if (!e->gexec[c]) {
            SF_CUDA(cudaStreamBeginCapture(e->s, cudaStreamCaptureModeThreadLocal));
            int lrc = launch_direct(e, 0, K);
            cudaGraph_t g = nullptr;
            cudaError_t ce = cudaStreamEndCapture(e->s, &g);
            if (lrc) {
                if (g) cudaGraphDestroy(g);
                return lrc;
            }
            SF_CUDA(ce);
            e->graph[c] = g;
            SF_CUDA(cudaGraphInstantiate(&e->gexec[c], g, 0));
            e->graph_k[c] = K;
        }
        SF_CUDA(cudaGraphLaunch(e->gexec[c], e->s));
    } else {
        if ((rc = launch_direct(e, 0, K))) return rc;
    }
    e->ctx->launches += K;
    e->sweeps += K;
    return SF_OK;
}

// packs the caller's arrays of slot q into the arena and fills its device record and tensor maps
int admit(sf_engine* e, int q, sf_batch_instance& u, int dtau_max) {
    sf_ctx* ctx = e->ctx;
    cudaStream_t s = e->s;
    Slot& h = e->slots[q];
    Inst& I = h.d;
    memset(&I, 0, sizeof(I));
    const Layout L(u.Nx, u.Ny);
    I.Nx = (int)u.Nx;
    I.Ny = (int)u.Ny;
    I.ntx = (int)ceil_div(u.Nx - 1, BX);
    I.LD32 = I.LD64 = L.LD;
    I.rows = L.rows;
    I.fstride32 = I.fstride64 = L.fstride;
    I.f32 = (float*)(e->arena + h.off);
    I.f64 = (double*)(e->arena + h.off + L.bytes32);
    h.ntiles64 = (int64_t)I.ntx * ceil_div(u.Ny - 1, BY64);
    const double Vdmp = 4.0, Vsc = 0.45, Ptsc = 0.5;  // StokesSolver_multixpu.jl:17-19
    const int64_t Nx = u.Nx, Ny = u.Ny, LD = L.LD;
    const double mdxy = std::min(u.dx, u.dy);
    I.dx = u.dx;
    I.dy = u.dy;
    I._dx = 1.0 / u.dx;
    I._dy = 1.0 / u.dy;
    I.g_y = u.g_y;
    I.maxdisp = u.maxdisp;
    I.use_stab = u.use_free_surface_stabilization ? 1 : 0;
    I.dtau_max = dtau_max;
    I.dt_in = I.use_stab ? u.dt : 0.0;
    I.dt = I.dt_in;
    I._dxf = (float)I._dx;
    I._dyf = (float)I._dy;
    I.cdampXf = (float)(Vdmp / (double)Nx);   // dampX = 1 - Vdmp / nx_g (:22)
    I.cdampYf = (float)(Vdmp / (double)Ny);
    I.c_vscf = (float)(Vsc * mdxy * mdxy / 4.1);
    I.c_ptscf = (float)(Ptsc * 4.1 / (double)std::max(Nx, Ny));
    I.g_dtf = (float)(I.g_y * I.dt);
    // corrections, rates and every padding entry start at zero
    SF_CUDA(cudaMemsetAsync(e->arena + h.off, 0, (size_t)h.bytes, s));
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
    // the damped rates the solve starts from: the caller's (solveStokes! keeps dVxdtau, dVydtau from one call
    // to the next), or zero; rate (i, j) sits at the offset of point (i, j)
    struct Rt { int g; const double* src; int64_t nx, ny; } rts[] = {{G_RVX, u.dVxdt, Nx - 2, Ny - 1},
                                                                     {G_RVY, u.dVydt, Nx - 1, Ny - 2}};
    for (const Rt& r : rts) {
        if (!r.src) continue;
        k_f64_to_f32<<<grid1(r.nx * r.ny, 256), 256, 0, s>>>(I.f32 + (int64_t)r.g * I.fstride32, LD, r.src, r.nx,
                                                             r.nx, r.ny);
        SF_LAUNCHED(ctx);
    }
    // the reference's event periods (:35-36; nx_g, ny_g are the grid's own on one domain); the correction
    // starts in the A buffers, no sweeps yet
    const int64_t mn = std::min(Nx, Ny);
    h.ncheck = std::min<int64_t>(5 * mn, 2000);
    h.ndtupdate = 10 * mn;
    h.budget = 0;
    e->h_ctl[q] = Ctl{0, 0, 0, 0};
    if (u.rel_tol > 0) {
        k_rho_scale64<<<1, 1024, 0, s>>>(u.rho_vy, (int)Nx, (int)Ny, u.g_y, e->d_scale + q);
        SF_LAUNCHED(ctx);
    }
    int rc = encode_maps(e, q);  // sweep tilings in every shape
    if (rc) return rc;
    SF_CUDA(cudaMemcpyAsync(e->d_insts + q, &I, sizeof(Inst), cudaMemcpyHostToDevice, s));
    return SF_OK;
}

// writes the FP64 state of slot q back to the caller's arrays (:89-95) and its results into the struct
int write_back(sf_engine* e, int q, double dt_cfl) {
    sf_ctx* ctx = e->ctx;
    cudaStream_t s = e->s;
    Slot& h = e->slots[q];
    sf_batch_instance& u = *h.user;
    const Inst& I = h.d;
    const int64_t Nx = u.Nx, Ny = u.Ny, LD = I.LD64;
    struct Uk { double* dst; int f; int64_t nx, ny; } ups[] = {
        {u.Vx_s, D_VX, Nx, Ny + 1}, {u.Vy_s, D_VY, Nx + 1, Ny}, {u.P, D_P, Nx - 1, Ny - 1}};
    for (const Uk& k : ups) {
        k_copy64<<<grid1(k.nx * k.ny, 256), 256, 0, s>>>(k.dst, k.nx, I.f64 + (int64_t)k.f * I.fstride64, LD, k.nx, k.ny);
        SF_LAUNCHED(ctx);
    }
    struct Rt { double* dst; int g; int64_t nx, ny; } rts[] = {{u.dVxdt, G_RVX, Nx - 2, Ny - 1},
                                                               {u.dVydt, G_RVY, Nx - 1, Ny - 2}};
    for (const Rt& r : rts) {
        if (!r.dst) continue;
        k_f32_to_f64<<<grid1(r.nx * r.ny, 256), 256, 0, s>>>(r.dst, r.nx, I.f32 + (int64_t)r.g * I.fstride32, LD, r.nx,
                                                             r.ny);
        SF_LAUNCHED(ctx);
    }
    k_pad_vx64<<<grid1((Nx + 2) * (Ny + 1), 256), 256, 0, s>>>(u.Vx_pad, I.f64 + D_VX * I.fstride64, LD, (int)Nx, (int)Ny);
    SF_LAUNCHED(ctx);
    k_pad_vy64<<<grid1((Nx + 1) * (Ny + 2), 256), 256, 0, s>>>(u.Vy_pad, I.f64 + D_VY * I.fstride64, LD, (int)Nx, (int)Ny);
    SF_LAUNCHED(ctx);
    u.dt_out = dt_cfl;  // compute_dt of the final V (:95), from the last outer step
    u.err = h.err;
    u.inner_iters = h.inner_total;
    u.outer_iters = h.outer;
    u.converged = (h.err <= h.eps) ? 1 : 0;
    u.eps_used = h.eps;
    u.status = (h.err == h.err && !std::isinf(h.err)) ? SF_OK : SF_ERR_NONFINITE;
    u.batch_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - h.t_submit).count();
    return SF_OK;
}

int validate(const sf_batch_instance& u, const char* who) {
    const std::string w(who);
    SF_REQUIRE(u.Nx >= 4 && u.Ny >= 4 && u.Nx < (1 << 20) && u.Ny < (1 << 20), (w + ": bad grid").c_str());
    SF_REQUIRE(u.P && u.Vx_pad && u.Vy_pad && u.rho_vy && u.mu_b && u.mu_p && u.Vx_s && u.Vy_s,
               (w + ": NULL array").c_str());
    SF_REQUIRE(u.dx > 0 && u.dy > 0, (w + ": dx, dy must be positive").c_str());
    return SF_OK;
}

int engine_submit(sf_engine* e, sf_batch_instance* u, cudaStream_t caller, int64_t* ticket) {
    int rc = validate(*u, "sf_engine_submit");
    if (rc) return rc;
    const int64_t bytes = Layout(u->Nx, u->Ny).bytes();
    if (bytes > e->alloc.cap())
        return fail(SF_ERR_TOO_LARGE, "sf_engine_submit: the instance needs " + std::to_string(bytes) +
                                          " arena bytes, more than the engine has");
    if (e->free_slots.empty()) return fail(SF_ERR_BUSY, "sf_engine_submit: instance table full");
    const int64_t off = e->alloc.alloc(bytes);
    if (off < 0) return fail(SF_ERR_BUSY, "sf_engine_submit: arena full");
    const int q = e->free_slots.back();
    e->free_slots.pop_back();
    Slot& h = e->slots[q];
    h = Slot{};
    h.user = u;
    h.off = off;
    h.bytes = bytes;
    h.t_submit = std::chrono::steady_clock::now();
    // the inputs are ready once the work queued on the caller's stream is done
    SF_CUDA(cudaEventRecord(e->ev_in, caller));
    SF_CUDA(cudaStreamWaitEvent(e->s, e->ev_in, 0));
    u->retried = 0;
    if ((rc = admit(e, q, *u, e->opt.dtau_local_max ? 1 : 0))) {
        e->alloc.release(off, bytes);
        e->free_slots.push_back(q);
        return rc;
    }
    h.active = true;
    h.ticket = e->next_ticket++;
    ++e->submitted;
    if (ticket) *ticket = h.ticket;
    return SF_OK;
}

// one round: [max|V| -> dt -> the reference's check where one is due] -> fold -> FP64 residual -> stopping test ->
// write-back of the finished -> sweeps of the rest.  Each instance's rounds end exactly on its iterations
// with an event in the reference's loop (:43-77): a dt update every ndtupdate iterations, a residual check
// every ncheck, iterMax; a round of fold_every sweeps is cut short for an instance whose next event comes
// sooner (its budget), so the sequence of dt values, the checks and the iteration it stops at are the FP64
// solver's.
int engine_round(sf_engine* e, cudaStream_t caller) {
    sf_ctx* ctx = e->ctx;
    cudaStream_t s = e->s;
    std::vector<int> ids, swept;
    bool any_check = false;
    for (int q = 0; q < (int)e->slots.size(); ++q)
        if (e->slots[q].active) {
            ids.push_back(q);
            Slot& h = e->slots[q];
            if (h.swept) {
                swept.push_back(q);
                // an odd budget leaves the current correction in the other buffer
                if (h.budget & 1) e->h_ctl[q].parity ^= 1;
                any_check = any_check || (e->h_ctl[q].flags & CTL_CHECK);
            }
        }
    if (ids.empty()) return SF_OK;
    ++e->rounds;
    int rc;
    // pageable source: staged before the call returns
    SF_CUDA(cudaMemcpyAsync(e->d_ctl, e->h_ctl.data(), e->h_ctl.size() * sizeof(Ctl), cudaMemcpyHostToDevice, s));
    int64_t nt = 0;
    if ((rc = upload_lists64(e, ids, &nt))) return rc;
    k_maxv64<<<(unsigned)nt, T64, 0, s>>>(e->d_insts, e->d_ctl, e->d_tiles64, e->d_part);
    SF_LAUNCHED(ctx);
    k_inst_dt<<<(unsigned)ids.size(), 256, 0, s>>>(e->d_insts, e->d_ctl, e->d_segs, e->d_part);
    SF_LAUNCHED(ctx);
    if (any_check) {
        k_check64<<<(unsigned)nt, T64, 0, s>>>(e->d_insts, e->d_ctl, e->d_tiles64, e->d_part_check);
        SF_LAUNCHED(ctx);
    }
    if (!swept.empty()) {  // V += dV, P += dP for every instance that ran sweeps
        SF_CUDA(cudaMemcpyAsync(e->d_list, swept.data(), swept.size() * 4, cudaMemcpyHostToDevice, s));
        // blocks per instance: enough to cover the largest one, at least 64, the whole launch around 8 per SM
        int64_t most = 0;
        for (int q : swept) most = std::max(most, e->slots[q].d.LD32 * e->slots[q].d.rows);
        const int64_t gx = std::max<int64_t>(
            1, std::min<int64_t>(ceil_div(most, 256),
                                 std::max<int64_t>(64, (int64_t)ctx->num_sms * 8 / (int64_t)swept.size())));
        k_accumulate<<<dim3((unsigned)gx, (unsigned)swept.size()), 256, 0, s>>>(e->d_insts, e->d_ctl, e->d_list);
        SF_LAUNCHED(ctx);
    }
    k_resid64<<<(unsigned)nt, T64, 0, s>>>(e->d_insts, e->d_tiles64, e->d_part);
    SF_LAUNCHED(ctx);
    k_inst_err<<<(unsigned)ids.size(), 256, 0, s>>>(e->d_segs, e->d_part, e->d_part_check, e->d_insts, e->d_ctl,
                                                    e->d_scale, e->d_out);
    SF_LAUNCHED(ctx);
    SF_CUDA(cudaMemcpyAsync(e->h_out, e->d_out, ids.size() * 4 * 8, cudaMemcpyDeviceToHost, s));
    SF_CUDA(cudaMemcpyAsync(e->h_out + ids.size() * 4, e->d_flag, sizeof(int), cudaMemcpyDeviceToHost, s));
    SF_CUDA(cudaStreamSynchronize(s));
    int flag = 0;
    memcpy(&flag, e->h_out + ids.size() * 4, sizeof(int));
    if (flag) return fail(SF_ERR_CUDA, "sf_engine: a tile copy did not complete in time");
    if ((rc = tuner_collect(e))) return rc;
    const int K = e->opt.fold_every;
    const int64_t max_sweeps = e->opt.max_sweeps;
    std::vector<int> sweep;
    bool any_done = false;
    for (size_t k = 0; k < ids.size(); ++k) {
        const int q = ids[k];
        Slot& h = e->slots[q];
        Ctl& c = e->h_ctl[q];
        const double err_fold = e->h_out[4 * k];
        if (h.outer == 0) {
            h.eps = h.user->rel_tol > 0 ? h.user->rel_tol * e->h_out[4 * k + 1] : h.user->eps;
            h.err = 2.0 * h.eps;  // :40, before the first check
        }
        ++h.outer;
        const bool at_check = (c.flags & CTL_CHECK) != 0;
        if (at_check) h.err = e->h_out[4 * k + 3];
        h.swept = false;
        c.flags = 0;
        const bool bad = !(err_fold == err_fold) || std::isinf(err_fold) || !(h.err == h.err) || std::isinf(h.err);
        if (bad && e->opt.retry_local_max && !h.d.dtau_max && h.inner_total < max_sweeps) {
            // restart from the caller's inputs (untouched until write-back) with the stencil-maximum
            // pseudo-time step; its sweeps keep counting, the first check comes after ncheck more
            const int64_t done = h.inner_total, outer = h.outer;
            if ((rc = admit(e, q, *h.user, 1))) return rc;
            h.inner_total = done;
            h.base = done;
            h.outer = outer;
            h.err = 2.0 * h.eps;
            h.user->retried = 1;
            continue;
        }
        if (bad) h.err = (h.err == h.err && !std::isinf(h.err)) ? err_fold : h.err;
        if (bad || (at_check && h.err <= h.eps) || h.inner_total >= max_sweeps) {
            if ((rc = write_back(e, q, e->h_out[4 * k + 2]))) return rc;
            h.active = false;
            e->alloc.release(h.off, h.bytes);
            e->free_slots.push_back(q);
            e->pending.push_back(h.ticket);
            ++e->finished;
            any_done = true;
        } else {
            sweep.push_back(q);
        }
    }
    if (any_done) {  // the caller's later work sees the written-back arrays
        SF_CUDA(cudaEventRecord(e->ev_out, s));
        SF_CUDA(cudaStreamWaitEvent(caller, e->ev_out, 0));
    }
    if (sweep.empty()) return SF_OK;
    // budgets: up to the next event of each instance, at most fold_every.  Events are counted from the start
    // of the current attempt (a restarted instance runs the schedule of a fresh solve); max_sweeps counts the
    // sweeps of every attempt.
    for (int q : sweep) {
        Slot& h = e->slots[q];
        Ctl& c = e->h_ctl[q];
        const int64_t it = h.inner_total - h.base;
        int64_t b = std::min<int64_t>(K, h.ncheck - it % h.ncheck);
        const bool stab = h.d.use_stab != 0;
        if (stab) b = std::min<int64_t>(b, h.ndtupdate - it % h.ndtupdate);
        b = std::max<int64_t>(1, std::min<int64_t>(b, max_sweeps - h.inner_total));
        const int64_t end = it + b;
        c.budget = (int)b;
        c.flags = ((end % h.ncheck == 0) ? CTL_CHECK : 0) | ((stab && end % h.ndtupdate == 0) ? CTL_DT : 0);
        h.budget = (int)b;
    }
    SF_CUDA(cudaMemcpyAsync(e->d_ctl, e->h_ctl.data(), e->h_ctl.size() * sizeof(Ctl), cudaMemcpyHostToDevice, s));
    if ((rc = launch_sweeps(e, sweep))) return rc;
    for (int q : sweep) {
        e->slots[q].inner_total += e->slots[q].budget;
        e->slots[q].swept = true;
    }
    return SF_OK;
}

int active_count(const sf_engine* e) {
    int n = 0;
    for (const Slot& h : e->slots) n += h.active ? 1 : 0;
    return n;
}

}  // namespace

void sf::mixed_engine_release(sf_ctx* ctx) {
    if (ctx && ctx->batch_engine) {
        engine_free(ctx->batch_engine);
        ctx->batch_engine = nullptr;
    }
}

// ---------------------------------------------------------------------------
// C ABI: engine
// ---------------------------------------------------------------------------
extern "C" int sf_engine_instance_bytes(int64_t Nx, int64_t Ny, int64_t* bytes) {
    SF_REQUIRE(bytes && Nx >= 4 && Ny >= 4 && Nx < (1 << 20) && Ny < (1 << 20), "sf_engine_instance_bytes: bad arguments");
    *bytes = Layout(Nx, Ny).bytes();
    return SF_OK;
}

extern "C" int sf_engine_create(sf_ctx* ctx, int64_t arena_bytes, int32_t max_instances, const sf_mixed_options* opt,
                                sf_engine** out) {
    SF_REQUIRE(ctx && out && arena_bytes > 0 && max_instances >= 1, "sf_engine_create: bad arguments");
    *out = nullptr;
    int rc = set_device(ctx);
    if (rc) return rc;
    sf_engine* e = new sf_engine();
    if ((rc = engine_init(e, ctx, max_instances, opt))) {
        engine_free(e);
        return rc;
    }
    const int64_t cap = round_up(arena_bytes, 256);
    if (cudaMalloc(&e->arena, (size_t)cap) != cudaSuccess) {
        cudaGetLastError();
        e->arena = nullptr;
        engine_free(e);
        return fail(SF_ERR_OOM, "sf_engine_create: arena of " + std::to_string(cap) + " bytes");
    }
    e->arena_owned = true;
    e->alloc.reset(cap);
    *out = e;
    return SF_OK;
}

extern "C" int sf_engine_destroy(sf_engine* e) {
    if (!e) return SF_OK;
    cudaSetDevice(e->ctx->device);
    engine_free(e);
    return SF_OK;
}

extern "C" int sf_engine_submit(sf_engine* e, sf_batch_instance* inst, void* stream, int64_t* ticket) {
    SF_REQUIRE(e && inst, "sf_engine_submit: NULL argument");
    int rc = set_device(e->ctx);
    if (rc) return rc;
    return engine_submit(e, inst, as_stream(stream), ticket);
}

extern "C" int sf_engine_step(sf_engine* e, void* stream, int64_t* finished, int32_t cap, int32_t* n_finished,
                              int32_t* n_active) {
    SF_REQUIRE(e && (cap <= 0 || finished), "sf_engine_step: bad arguments");
    int rc = set_device(e->ctx);
    if (rc) return rc;
    if ((rc = engine_round(e, as_stream(stream)))) return rc;
    int32_t k = 0;
    while (k < cap && !e->pending.empty()) {
        finished[k++] = e->pending.front();
        e->pending.pop_front();
    }
    if (n_finished) *n_finished = k;
    if (n_active) *n_active = active_count(e);
    return SF_OK;
}

extern "C" int sf_engine_get_stats(sf_engine* e, sf_engine_stats* st) {
    SF_REQUIRE(e && st, "sf_engine_get_stats: NULL argument");
    memset(st, 0, sizeof(*st));
    st->arena_bytes = e->alloc.cap();
    st->arena_used = e->alloc.used();
    st->arena_peak = e->alloc.peak();
    st->submitted = e->submitted;
    st->finished = e->finished;
    st->rounds = e->rounds;
    st->sweeps = e->sweeps;
    st->active = active_count(e);
    st->pending_results = (int32_t)e->pending.size();
    st->tile_rows = kShapes[e->shape].rows;
    st->tile_schedule = e->sched + 1;
    st->overlap_launches = e->overlap;
    st->tune_state = e->tune_state;
    st->tune_classes = (int32_t)e->ctx->sweep_shapes.size();
    st->tune_rounds = e->tune_rounds;
    st->tune_hits = e->tune_hits;
    for (int k = 0; k < NCAND; ++k) st->tune_ns[k] = e->tune_ns[k];
    return SF_OK;
}

extern "C" int sf_ctx_batch_stats(sf_ctx* ctx, sf_engine_stats* st) {
    SF_REQUIRE(ctx && st, "sf_ctx_batch_stats: NULL argument");
    SF_REQUIRE(ctx->batch_engine, "sf_ctx_batch_stats: no batched solve has run in this context");
    return sf_engine_get_stats(ctx->batch_engine, st);
}

extern "C" int sf_solve_stokes_batch_mixed(sf_ctx* ctx, sf_batch_instance* inst, int n, const sf_mixed_options* o,
                                           void* stream) {
    SF_REQUIRE(ctx && inst && n >= 1, "sf_solve_stokes_batch_mixed: bad arguments");
    int rc = set_device(ctx);
    if (rc) return rc;
    int64_t total = 0;
    for (int b = 0; b < n; ++b) {
        if ((rc = validate(inst[b], "sf_solve_stokes_batch_mixed"))) return rc;
        total += Layout(inst[b].Nx, inst[b].Ny).bytes();
    }
    // the context keeps one engine for this call (tables, graph); its arena is the context's scratch,
    // sized to the batch, so every instance is admitted at once
    sf_engine* e = ctx->batch_engine;
    if (e && (int)e->slots.size() < n) {
        mixed_engine_release(ctx);
        e = nullptr;
    }
    if (!e) {
        e = new sf_engine();
        if ((rc = engine_init(e, ctx, std::max(n, 64), o))) {
            engine_free(e);
            return rc;
        }
        ctx->batch_engine = e;
    }
    e->opt = normalized(o);
    if ((rc = configure_tuner(e))) return rc;
    if ((rc = ensure(ctx, ctx->mixed, (size_t)total))) return rc;
    e->arena = (unsigned char*)ctx->mixed.ptr;
    e->alloc.reset(total);
    auto run = [&]() -> int {
        int r;
        cudaStream_t caller = as_stream(stream);
        SF_CUDA(cudaEventRecord(ctx->ev_a, caller));
        SF_CUDA(cudaStreamWaitEvent(e->s, ctx->ev_a, 0));
        SF_CUDA(cudaEventRecord(ctx->ev_b, e->s));
        for (int b = 0; b < n; ++b)
            if ((r = engine_submit(e, &inst[b], caller, nullptr))) return r;
        while (active_count(e) > 0)
            if ((r = engine_round(e, caller))) return r;
        e->pending.clear();
        SF_CUDA(cudaEventRecord(ctx->ev_c, e->s));
        SF_CUDA(cudaStreamSynchronize(e->s));
        float ms = 0.f;
        SF_CUDA(cudaEventElapsedTime(&ms, ctx->ev_b, ctx->ev_c));
        for (int b = 0; b < n; ++b) inst[b].batch_ms = ms;
        return SF_OK;
    };
    if ((rc = run())) {
        mixed_engine_release(ctx);  // its state is unknown after an error
        return rc;
    }
    return SF_OK;
}
extern "C" int sf_solve_stokes_mixed(sf_ctx* ctx, double* P, double* Vx_pad, double* Vy_pad, const double* rho_vy,
                                     const double* mu_b, const double* mu_p, double* Vx_s, double* Vy_s,
                                     double* dVxdt, double* dVydt, double g_y,
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
    u.dVxdt = dVxdt;
    u.dVydt = dVydt;
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
