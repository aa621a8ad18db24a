// sf_domains.cu -- the parts of a decomposed StokesFlow2D timestep besides
// the solve (which is sf_solve_stokes_decomposed in sf_solve.cu):
//
//   * sf_sum_overlapping_values: sumOverlappingValues! (MarkerToGrid.jl:183-269),
//     the deposit's weight / value sums added across the ranks' overlap;
//   * sf_safe_division: safeDivision (MarkerToGrid.jl:164-172) over a grid;
//   * sf_exchange_markers: exchangeMarkers (MarkerExchange.jl:8-163), the
//     markers near an edge shared with a neighbour moved to that neighbour.
//
// All ranks are driven from one host thread, each on its own context (device
// and work stream).  Data crosses between ranks on the receiving rank's
// device: blocks of the overlap sums by a copy kernel that reads the
// neighbour's memory directly when the two devices are peers (copy_block,
// which enables peer access on first use; other pairs go through
// cudaMemcpy2DAsync), the exchanged markers as contiguous peer copies
// (cudaMemcpyDefault), all ordered by events.  Compiled like the other FP64 files (-fmad=false): the one
// arithmetic step of the exchange, x - (lx - dx) * shift, rounds as Julia's.
#include <algorithm>
#include <vector>

#include "sf_internal.cuh"

namespace sf {
namespace dd {

__global__ void k_add_block(double* __restrict__ dst, int64_t ld_dst, const double* __restrict__ src, int64_t ld_src,
                            int64_t w, int64_t h) {
    const int64_t n = w * h;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = k % w, j = k / w;
        dst[i + j * ld_dst] = dst[i + j * ld_dst] + src[i + j * ld_src];   // A .+= received (own + remote)
    }
}

__global__ void k_safe_division(double* __restrict__ val, int64_t nx, int64_t ny, const double* __restrict__ num,
                                const double* __restrict__ den, int64_t ld, unsigned long long* __restrict__ empty) {
    const int64_t n = nx * ny;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = k % nx, j = k / nx;
        const double d = den[i + j * ld];
        if (d != 0.0)
            val[k] = num[i + j * ld] / d;
        else
            atomicAdd(empty, 1ull);
    }
}

// ---------------------------------------------------------------------------
// marker exchange
// ---------------------------------------------------------------------------
constexpr int XT = 256;              // threads per block
constexpr int XITEMS = 16;           // markers per thread per block: a block owns XT * XITEMS consecutive markers
constexpr int NDIR = 9;              // 0: stays, 1..8: the neighbour directions of MarkerExchange.jl:12-18
__constant__ int c_sx[NDIR] = {0, -1, 0, 1, 1, 1, 0, -1, -1};   // neighbourIdxToShift (:187-196)
__constant__ int c_sy[NDIR] = {0, -1, -1, -1, 0, 1, 1, 1, 0};

struct RankGeom {
    double lx, ly, hx, hy;   // local domain size and half a cell (the dx/2, dy/2 of :66)
    int cx, cy, dimx, dimy;
};

// posToNeighbourIdx (:204-222) with dx, dy = half a cell
__device__ __forceinline__ int marker_dir(double x, double y, const RankGeom& g) {
    if (y < g.hy && g.cy != 0) {
        if (x < g.hx && g.cx != 0) return 1;
        if (x > g.lx - g.hx && g.cx != g.dimx - 1) return 3;
        return 2;
    }
    if (y > g.ly - g.hy && g.cy != g.dimy - 1) {
        if (x < g.hx && g.cx != 0) return 7;
        if (x > g.lx - g.hx && g.cx != g.dimx - 1) return 5;
        return 6;
    }
    if (x < g.hx && g.cx != 0) return 8;
    if (x > g.lx - g.hx && g.cx != g.dimx - 1) return 4;
    return 0;
}

// pass 1: each marker's direction, per-block counts per direction
__global__ void __launch_bounds__(XT) k_exch_count(const double* __restrict__ x, const double* __restrict__ y, int64_t n,
                                                   RankGeom g, uint8_t* __restrict__ dir, int32_t* __restrict__ counts) {
    __shared__ int32_t sc[NDIR];
    if (threadIdx.x < NDIR) sc[threadIdx.x] = 0;
    __syncthreads();
    const int64_t b0 = (int64_t)blockIdx.x * XT * XITEMS;
    for (int k = 0; k < XITEMS; ++k) {
        const int64_t m = b0 + (int64_t)k * XT + threadIdx.x;
        if (m < n) {
            const int d = marker_dir(x[m], y[m], g);
            dir[m] = (uint8_t)d;
            atomicAdd(&sc[d], 1);
        }
    }
    __syncthreads();
    if (threadIdx.x < NDIR) counts[(int64_t)blockIdx.x * NDIR + threadIdx.x] = sc[threadIdx.x];
}

// pass 2: stable scatter.  Direction 0 goes to the rank's own output at off[block][0] + rank among the block's
// kept markers so far; direction d > 0 to the send buffer at off[block][d] + ..., shifted by (lx - dx, ly - dy)
// times the direction's step (:77-79).  Order within a direction is marker order: sub-chunks of XT markers in
// sequence, lanes ranked by __match_any_sync, warps by a prefix over the block.
__global__ void __launch_bounds__(XT) k_exch_scatter(const double* __restrict__ x, const double* __restrict__ y,
                                                     const double* __restrict__ rho, const double* __restrict__ mu,
                                                     int64_t n, const uint8_t* __restrict__ dir,
                                                     const int64_t* __restrict__ off, double shift_x, double shift_y,
                                                     double* __restrict__ kx, double* __restrict__ ky,
                                                     double* __restrict__ krho, double* __restrict__ kmu,
                                                     double* __restrict__ sx, double* __restrict__ sy,
                                                     double* __restrict__ srho, double* __restrict__ smu) {
    constexpr int NW = XT / 32;
    __shared__ int32_t warp_cnt[NW][NDIR];
    __shared__ int32_t warp_pre[NW][NDIR];
    __shared__ int32_t total[NDIR];
    __shared__ int64_t base[NDIR];   // next position of each direction for this block
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x < NDIR) base[threadIdx.x] = off[(int64_t)blockIdx.x * NDIR + threadIdx.x];
    const int64_t b0 = (int64_t)blockIdx.x * XT * XITEMS;
    for (int k = 0; k < XITEMS; ++k) {
        for (int q = threadIdx.x; q < NW * NDIR; q += XT) warp_cnt[q / NDIR][q % NDIR] = 0;
        __syncthreads();
        const int64_t m = b0 + (int64_t)k * XT + threadIdx.x;
        const bool live = m < n;
        const int d = live ? dir[m] : NDIR;   // NDIR: no marker in this slot
        const unsigned same = __match_any_sync(0xffffffffu, d);
        const int r = __popc(same & ((1u << lane) - 1u));   // earlier lanes of this warp with the same direction
        if (live && r == 0) warp_cnt[warp][d] = __popc(same);
        __syncthreads();
        if (threadIdx.x < NDIR) {   // per direction: prefix over the warps of this sub-chunk
            int32_t acc = 0;
            for (int w = 0; w < NW; ++w) {
                warp_pre[w][threadIdx.x] = acc;
                acc += warp_cnt[w][threadIdx.x];
            }
            total[threadIdx.x] = acc;
        }
        __syncthreads();
        if (live) {
            const int64_t pos = base[d] + warp_pre[warp][d] + r;
            if (d == 0) {
                kx[pos] = x[m];
                ky[pos] = y[m];
                krho[pos] = rho[m];
                kmu[pos] = mu[m];
            } else {
                sx[pos] = x[m] - shift_x * (double)c_sx[d];   // x_m[i] -= (localDomain[1] - dx) * shift[1]
                sy[pos] = y[m] - shift_y * (double)c_sy[d];
                srho[pos] = rho[m];
                smu[pos] = mu[m];
            }
        }
        __syncthreads();
        if (threadIdx.x < NDIR) base[threadIdx.x] += total[threadIdx.x];
    }
}

static unsigned grid_for(sf_ctx* ctx, int64_t n, int threads) {
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(ceil_div(n, threads), (int64_t)ctx->num_sms * 32));
}

}  // namespace dd
}  // namespace sf

using namespace sf;
using namespace sf::dd;

extern "C" {

int sf_safe_division(sf_ctx* ctx, double* val_grid, int64_t nx, int64_t ny, const double* val_wt_sum,
                     const double* wt_sum, int64_t ld_sum, void* stream) {
    SF_REQUIRE(ctx && val_grid && val_wt_sum && wt_sum && nx >= 1 && ny >= 1 && ld_sum >= nx,
               "sf_safe_division: bad arguments");
    int rc = set_device(ctx);
    if (rc) return rc;
    k_safe_division<<<grid_for(ctx, nx * ny, 256), 256, 0, as_stream(stream)>>>(
        val_grid, nx, ny, val_wt_sum, wt_sum, ld_sum, ctx->d_counters + CNT_EMPTY_NODES);
    SF_LAUNCHED(ctx);
    return SF_OK;
}

int sf_sum_overlapping_values(sf_rank_array* ranks, int32_t dims_x, int32_t dims_y, int64_t Nx, int64_t Ny,
                              int64_t nx, int64_t ny) {
    SF_REQUIRE(ranks && dims_x >= 1 && dims_y >= 1 && dims_x * dims_y <= 4096, "sf_sum_overlapping_values: bad dims");
    const int64_t ox = 2 + nx - Nx, oy = 2 + ny - Ny;
    SF_REQUIRE(nx >= 1 && ny >= 1 && ox >= 0 && oy >= 0, "sf_sum_overlapping_values: bad sizes");
    SF_REQUIRE(2 * ox <= nx && 2 * oy <= ny, "sf_sum_overlapping_values: total overlap is bigger than the array");
    const int nr = dims_x * dims_y;
    SF_REQUIRE(distinct_contexts(nr, [&](int i) { return ranks[i].ctx; }),
               "sf_sum_overlapping_values: every rank needs its own context");
    std::vector<int> at((size_t)nr, -1);
    for (int r = 0; r < nr; ++r) {
        const sf_rank_array& k = ranks[r];
        SF_REQUIRE(k.ctx && k.a && k.coord_x >= 0 && k.coord_x < dims_x && k.coord_y >= 0 && k.coord_y < dims_y,
                   "sf_sum_overlapping_values: bad rank");
        const int c = k.coord_x + k.coord_y * dims_x;
        SF_REQUIRE(at[c] < 0, "sf_sum_overlapping_values: two ranks have the same coordinates");
        at[c] = r;
    }
    auto nb = [&](int r, int ddx, int ddy) {
        const int cx = ranks[r].coord_x + ddx, cy = ranks[r].coord_y + ddy;
        return (cx < 0 || cy < 0 || cx >= dims_x || cy >= dims_y) ? -1 : at[cx + cy * dims_x];
    };
    const int64_t tmp_elems = std::max(ox * ny, nx * oy);
    std::vector<double*> lo((size_t)nr), hi((size_t)nr);     // received from the lower / upper neighbour
    std::vector<cudaEvent_t> ev((size_t)nr, nullptr);
    int rc = SF_OK;
    for (int r = 0; r < nr; ++r) {
        sf_ctx* c = ranks[r].ctx;
        if ((rc = set_device(c))) break;
        SF_CUDA(cudaDeviceSynchronize());   // the ranks' deposits are complete
        if ((rc = ensure(c, c->exch, (size_t)tmp_elems * 2 * 8))) break;
        lo[r] = (double*)c->exch.ptr;
        hi[r] = lo[r] + tmp_elems;
        SF_CUDA(cudaEventCreateWithFlags(&ev[r], cudaEventDisableTiming));
    }
    auto cleanup = [&]() {
        for (int r = 0; r < nr; ++r)
            if (ev[r]) {
                cudaSetDevice(ranks[r].ctx->device);
                cudaEventDestroy(ev[r]);
            }
    };
    if (rc) {
        cleanup();
        return rc;
    }
    // one dimension: copy every neighbour block first (pre-pass values), then add (x, then y: :223-266)
    auto pass = [&](int dim) -> int {
        const int64_t o = dim == 0 ? ox : oy;
        if (o <= 0) return SF_OK;
        for (int r = 0; r < nr; ++r) {
            sf_rank_array& k = ranks[r];
            cudaStream_t s = k.ctx->work;
            SF_CUDA(cudaSetDevice(k.ctx->device));
            const int l = dim == 0 ? nb(r, -1, 0) : nb(r, 0, -1), u = dim == 0 ? nb(r, 1, 0) : nb(r, 0, 1);
            for (int q : {l, u})
                if (q >= 0) SF_CUDA(cudaStreamWaitEvent(s, ev[q], 0));
            // copied on this rank's device, reading the neighbour's memory directly when the devices are peers
            if (dim == 0) {
                // the lower neighbour's last ox planes, the upper neighbour's first ox planes
                if (l >= 0 && (rc = copy_block(k.ctx, s, lo[r], ox, ranks[l].a + (nx - ox), nx, ox, ny,
                                               ranks[l].ctx->device)))
                    return rc;
                if (u >= 0 && (rc = copy_block(k.ctx, s, hi[r], ox, ranks[u].a, nx, ox, ny, ranks[u].ctx->device)))
                    return rc;
            } else {
                if (l >= 0 && (rc = copy_block(k.ctx, s, lo[r], nx, ranks[l].a + (ny - oy) * nx, nx, nx, oy,
                                               ranks[l].ctx->device)))
                    return rc;
                if (u >= 0 && (rc = copy_block(k.ctx, s, hi[r], nx, ranks[u].a, nx, nx, oy, ranks[u].ctx->device)))
                    return rc;
            }
            SF_CUDA(cudaEventRecord(ev[r], s));
        }
        for (int r = 0; r < nr; ++r) {
            sf_rank_array& k = ranks[r];
            cudaStream_t s = k.ctx->work;
            SF_CUDA(cudaSetDevice(k.ctx->device));
            const int l = dim == 0 ? nb(r, -1, 0) : nb(r, 0, -1), u = dim == 0 ? nb(r, 1, 0) : nb(r, 0, 1);
            // the neighbours have read this rank's blocks before it adds to them
            for (int q : {l, u})
                if (q >= 0) SF_CUDA(cudaStreamWaitEvent(s, ev[q], 0));
            const int64_t w = dim == 0 ? ox : nx, h = dim == 0 ? ny : oy;
            const unsigned g = grid_for(k.ctx, w * h, 256);
            if (l >= 0) {
                k_add_block<<<g, 256, 0, s>>>(k.a, nx, lo[r], w, w, h);
                SF_LAUNCHED(k.ctx);
            }
            if (u >= 0) {
                double* dst = dim == 0 ? k.a + (nx - ox) : k.a + (ny - oy) * nx;
                k_add_block<<<g, 256, 0, s>>>(dst, nx, hi[r], w, w, h);
                SF_LAUNCHED(k.ctx);
            }
        }
        for (int r = 0; r < nr; ++r) {
            SF_CUDA(cudaSetDevice(ranks[r].ctx->device));
            SF_CUDA(cudaEventRecord(ev[r], ranks[r].ctx->work));
        }
        return SF_OK;
    };
    if (!(rc = pass(0))) rc = pass(1);
    for (int r = 0; r < nr && !rc; ++r) {
        if ((rc = set_device(ranks[r].ctx))) break;
        cudaError_t e = cudaStreamSynchronize(ranks[r].ctx->work);
        if (e != cudaSuccess) rc = cuda_fail(e, "sf_sum_overlapping_values", __FILE__, __LINE__);
    }
    cleanup();
    return rc;
}

int sf_exchange_markers(sf_marker_rank* ranks, int32_t dims_x, int32_t dims_y, double lx, double ly, double dx,
                        double dy) {
    SF_REQUIRE(ranks && dims_x >= 1 && dims_y >= 1 && dims_x * dims_y <= 4096, "sf_exchange_markers: bad dims");
    SF_REQUIRE(lx > 0 && ly > 0 && dx > 0 && dy > 0, "sf_exchange_markers: bad domain");
    const int nr = dims_x * dims_y;
    SF_REQUIRE(distinct_contexts(nr, [&](int i) { return ranks[i].ctx; }),
               "sf_exchange_markers: every rank needs its own context");
    std::vector<int> at((size_t)nr, -1);
    for (int r = 0; r < nr; ++r) {
        const sf_marker_rank& k = ranks[r];
        SF_REQUIRE(k.ctx && k.n >= 0 && k.n < (int64_t)INT32_MAX, "sf_exchange_markers: bad rank");
        SF_REQUIRE(k.n == 0 || (k.x && k.y && k.rho && k.mu), "sf_exchange_markers: NULL marker array");
        SF_REQUIRE(k.capacity >= 0 && (k.capacity == 0 || (k.x_out && k.y_out && k.rho_out && k.mu_out)),
                   "sf_exchange_markers: NULL output array");
        SF_REQUIRE(k.coord_x >= 0 && k.coord_x < dims_x && k.coord_y >= 0 && k.coord_y < dims_y,
                   "sf_exchange_markers: coordinate outside dims");
        const int c = k.coord_x + k.coord_y * dims_x;
        SF_REQUIRE(at[c] < 0, "sf_exchange_markers: two ranks have the same coordinates");
        at[c] = r;
    }
    static const int sxh[NDIR] = {0, -1, 0, 1, 1, 1, 0, -1, -1}, syh[NDIR] = {0, -1, -1, -1, 0, 1, 1, 1, 0};
    auto nb = [&](int r, int d) {
        const int cx = ranks[r].coord_x + sxh[d], cy = ranks[r].coord_y + syh[d];
        return (cx < 0 || cy < 0 || cx >= dims_x || cy >= dims_y) ? -1 : at[cx + cy * dims_x];
    };
    auto opposite = [](int i) { return i >= 5 ? (i + 4) % 9 + 1 : i + 4; };   // dstToSrcIdx (:198-202)
    const double hx = dx / 2, hy = dy / 2;     // :66
    const double shift_x = lx - dx, shift_y = ly - dy;

    struct Work {
        int64_t nblk = 0;
        uint8_t* dir = nullptr;
        int32_t* counts = nullptr;
        int64_t* off = nullptr;
        double *sx = nullptr, *sy = nullptr, *srho = nullptr, *smu = nullptr;
        std::vector<int32_t> h_counts;
        int64_t tot[NDIR] = {0};
        int64_t send_base[NDIR] = {0};
        cudaEvent_t ev = nullptr;
    };
    std::vector<Work> W((size_t)nr);
    auto cleanup = [&]() {
        for (int r = 0; r < nr; ++r)
            if (W[r].ev) {
                cudaSetDevice(ranks[r].ctx->device);
                cudaEventDestroy(W[r].ev);
            }
    };
    int rc = SF_OK;
    // ---- pass 1 on every rank: directions and per-block counts ----
    for (int r = 0; r < nr && !rc; ++r) {
        sf_marker_rank& k = ranks[r];
        Work& w = W[r];
        sf_ctx* c = k.ctx;
        if ((rc = set_device(c))) break;
        SF_CUDA(cudaDeviceSynchronize());   // the caller's markers are complete
        SF_CUDA(cudaEventCreateWithFlags(&w.ev, cudaEventDisableTiming));
        w.nblk = ceil_div(std::max<int64_t>(k.n, 1), (int64_t)XT * XITEMS);
        const size_t o_dir = 0, o_cnt = round_up(o_dir + (size_t)k.n + 1, 256);
        const size_t o_off = round_up(o_cnt + (size_t)w.nblk * NDIR * 4, 256);
        const size_t o_snd = round_up(o_off + (size_t)w.nblk * NDIR * 8, 256);
        const size_t total = o_snd + (size_t)std::max<int64_t>(k.n, 1) * 8 * 4;
        if ((rc = ensure(c, c->exch, total))) break;
        unsigned char* b = (unsigned char*)c->exch.ptr;
        w.dir = (uint8_t*)(b + o_dir);
        w.counts = (int32_t*)(b + o_cnt);
        w.off = (int64_t*)(b + o_off);
        w.sx = (double*)(b + o_snd);
        w.sy = w.sx + std::max<int64_t>(k.n, 1);
        w.srho = w.sy + std::max<int64_t>(k.n, 1);
        w.smu = w.srho + std::max<int64_t>(k.n, 1);
        RankGeom g{lx, ly, hx, hy, k.coord_x, k.coord_y, dims_x, dims_y};
        SF_CUDA(cudaMemsetAsync(w.counts, 0, (size_t)w.nblk * NDIR * 4, c->work));
        if (k.n > 0) {
            k_exch_count<<<(unsigned)w.nblk, XT, 0, c->work>>>(k.x, k.y, k.n, g, w.dir, w.counts);
            SF_LAUNCHED(c);
        }
        w.h_counts.assign((size_t)w.nblk * NDIR, 0);
        SF_CUDA(cudaMemcpyAsync(w.h_counts.data(), w.counts, (size_t)w.nblk * NDIR * 4, cudaMemcpyDeviceToHost,
                                c->work));
    }
    for (int r = 0; r < nr && !rc; ++r) {
        SF_CUDA(cudaSetDevice(ranks[r].ctx->device));
        SF_CUDA(cudaStreamSynchronize(ranks[r].ctx->work));
        Work& w = W[r];
        for (int64_t bk = 0; bk < w.nblk; ++bk)
            for (int d = 0; d < NDIR; ++d) w.tot[d] += w.h_counts[(size_t)bk * NDIR + d];
        int64_t acc = 0;
        for (int d = 1; d < NDIR; ++d) {
            w.send_base[d] = acc;
            acc += w.tot[d];
        }
    }
    if (rc) {
        cleanup();
        return rc;
    }
    // ---- sizes after the exchange; nothing is written unless every rank has room ----
    bool fits = true;
    for (int r = 0; r < nr; ++r) {
        int64_t n_out = W[r].tot[0];
        for (int i = 1; i < NDIR; ++i) {
            const int src = nb(r, opposite(i));
            if (src >= 0) n_out += W[src].tot[i];
        }
        ranks[r].n_out = n_out;
        fits = fits && n_out <= ranks[r].capacity;
    }
    if (!fits) {
        cleanup();
        return fail(SF_ERR_TOO_LARGE, "sf_exchange_markers: an output capacity is too small (n_out holds the sizes needed)");
    }
    // ---- pass 2: stable scatter of the kept markers and the send buffers ----
    for (int r = 0; r < nr && !rc; ++r) {
        sf_marker_rank& k = ranks[r];
        Work& w = W[r];
        sf_ctx* c = k.ctx;
        SF_CUDA(cudaSetDevice(c->device));
        std::vector<int64_t> h_off((size_t)w.nblk * NDIR);
        int64_t run[NDIR];
        for (int d = 0; d < NDIR; ++d) run[d] = d == 0 ? 0 : w.send_base[d];
        for (int64_t bk = 0; bk < w.nblk; ++bk)
            for (int d = 0; d < NDIR; ++d) {
                h_off[(size_t)bk * NDIR + d] = run[d];
                run[d] += w.h_counts[(size_t)bk * NDIR + d];
            }
        // pageable source: staged before cudaMemcpyAsync returns
        SF_CUDA(cudaMemcpyAsync(w.off, h_off.data(), h_off.size() * 8, cudaMemcpyHostToDevice, c->work));
        if (k.n > 0) {
            k_exch_scatter<<<(unsigned)w.nblk, XT, 0, c->work>>>(k.x, k.y, k.rho, k.mu, k.n, w.dir, w.off, shift_x,
                                                                 shift_y, k.x_out, k.y_out, k.rho_out, k.mu_out,
                                                                 w.sx, w.sy, w.srho, w.smu);
            SF_LAUNCHED(c);
        }
        SF_CUDA(cudaEventRecord(w.ev, c->work));
    }
    // ---- received markers: neighbour index 1..8, each from the neighbour opposite that direction (:150-157) ----
    for (int r = 0; r < nr && !rc; ++r) {
        sf_marker_rank& k = ranks[r];
        sf_ctx* c = k.ctx;
        SF_CUDA(cudaSetDevice(c->device));
        int64_t pos = W[r].tot[0];
        for (int i = 1; i < NDIR; ++i) {
            const int src = nb(r, opposite(i));
            if (src < 0) continue;
            const Work& ws = W[src];
            const int64_t cnt = ws.tot[i];
            if (cnt == 0) continue;
            SF_CUDA(cudaStreamWaitEvent(c->work, ws.ev, 0));
            // a direct peer copy when the sender's device is a peer of this one (enabled on first use)
            bool direct = false;
            if ((rc = peer_access(c->device, ranks[src].ctx->device, &direct))) break;
            const int64_t o = ws.send_base[i];
            SF_CUDA(cudaMemcpyAsync(k.x_out + pos, ws.sx + o, cnt * 8, cudaMemcpyDefault, c->work));
            SF_CUDA(cudaMemcpyAsync(k.y_out + pos, ws.sy + o, cnt * 8, cudaMemcpyDefault, c->work));
            SF_CUDA(cudaMemcpyAsync(k.rho_out + pos, ws.srho + o, cnt * 8, cudaMemcpyDefault, c->work));
            SF_CUDA(cudaMemcpyAsync(k.mu_out + pos, ws.smu + o, cnt * 8, cudaMemcpyDefault, c->work));
            pos += cnt;
        }
    }
    for (int r = 0; r < nr && !rc; ++r) {   // every copy out of every send buffer is done
        if ((rc = set_device(ranks[r].ctx))) break;
        cudaError_t e = cudaStreamSynchronize(ranks[r].ctx->work);
        if (e != cudaSuccess) rc = cuda_fail(e, "sf_exchange_markers", __FILE__, __LINE__);
    }
    cleanup();
    return rc;
}

}  // extern "C"
