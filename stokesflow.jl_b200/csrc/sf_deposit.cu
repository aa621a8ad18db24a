// sf_deposit.cu -- marker->grid deposit (scripts/MarkerToGrid.jl:18-172) and
// marker->cell rebinning for libstokesflow_b200.so.
//
// Design: the reference scatters 8 floating-point adds per marker (serial on
// the CPU, CUDA.@atomic on the GPU, MarkerToGrid.jl:58-155).  Here the adds
// become a gather with no floating-point atomics:
//   1. k_cell_keys     cell (ix, iy) of every marker for this grid, exactly
//                      topleftIndexRelDist (common.jl:22-33); per-cell counts
//                      with warp-aggregated integer atomics.
//   2. exclusive scan  counts -> cell offsets.
//   3. k_scatter       marker indices into their cell's segment (in no
//                      particular order inside it).
//   4. segment sort    every segment ascending by marker index, which makes
//                      the whole a stable counting sort:
//                      k_long_cells + k_sort_long sort the cells holding more
//                      than SORT_LONG markers in place (a block-wide LSD radix
//                      sort per cell, stable, linear in the cell's count, so a
//                      cell where markers pile up costs no more than its
//                      size); k_sort_cells sorts the others in shared memory,
//                      a window of consecutive cells at a time.
//   5. k_gather_sorted one thread per node merges the four adjacent cells'
//                      segments by marker index and accumulates w and w*val in
//                      ascending marker order -- the reference CPU loop's
//                      order, so each node's sums are bit-identical to it --
//                      then divides (safeDivision, :164-172).
// For the deposit, step 4 writes each sorted entry as a payload record
// {dxij, dyij, val, m} (the marker's relative position in its cell, computed
// once with topleftIndexRelDist's IEEE divisions, its value and its index), so
// the gather streams contiguous records of neighbouring cells instead of
// chasing marker indices into x, y and val.  Steps 1-4 with the permutation as
// output are the rebin (sf_rebin_markers).
#include <algorithm>

#include "sf_internal.cuh"

namespace sf {

constexpr int DEP_THREADS = 256;
constexpr int SORT_THREADS = 256;
constexpr int SORT_CPB = 256;     // cells per block of k_sort_cells
constexpr int SORT_CAP = 4096;    // entries of a k_sort_cells window in shared memory
constexpr int SORT_LONG = 64;     // cells with more markers are sorted by k_sort_long

// A sorted deposit entry: the marker's relative position in its cell (topleftIndexRelDist's dxij, dyij), its
// value and its index.  32 bytes: one sector.
struct __align__(32) Payload {
    double dxij, dyij, val;
    int32_t m, pad_;
};

// 1. cell key of every marker; counts[key]++ (warp-aggregated).
__global__ void k_cell_keys(const double* __restrict__ x, const double* __restrict__ y, int64_t nm, double xmin,
                            double ymin, double dx, double dy, int64_t nx, int64_t ny, int32_t* __restrict__ keys,
                            int32_t* __restrict__ counts, unsigned long long* __restrict__ bad_counter) {
    const int lane = threadIdx.x & 31;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < nm; base += stride) {
        int64_t m = base + threadIdx.x;
        int32_t key = -1;
        if (m < nm) {
            TopLeft t = topleft(xmin, ymin, x[m], y[m], dx, dy);
            // MarkerToGrid.jl:66: accept iff 0 <= ix <= Nx && 0 <= iy <= Ny (ix = qx + 1)
            if (t.qx >= -1.0 && t.qx <= (double)(nx - 1) && t.qy >= -1.0 && t.qy <= (double)(ny - 1))
                key = (int32_t)((int64_t)t.qx + 1 + ((int64_t)t.qy + 1) * (nx + 1));
            keys[m] = key;
        }
        unsigned active = __ballot_sync(0xffffffffu, m < nm);
        if (m < nm) {
            unsigned peers = __match_any_sync(active, key);
            int leader = __ffs(peers) - 1;
            if (lane == leader) {
                int n = __popc(peers);
                if (key >= 0)
                    atomicAdd(&counts[key], n);
                else if (bad_counter)
                    atomicAdd(bad_counter, (unsigned long long)n);
            }
        }
    }
}

// 1 for several grids over the same markers (the three deposits of a timestep): each marker's position is read
// once, and every grid gets its own keys and counts, exactly as k_cell_keys computes them.
struct GridKeys {
    double xmin[SF_MAX_GRIDS], ymin[SF_MAX_GRIDS];
    int64_t nx[SF_MAX_GRIDS], ny[SF_MAX_GRIDS];
    int32_t* keys[SF_MAX_GRIDS];
    int32_t* counts[SF_MAX_GRIDS];
    int n;
};

__global__ void k_cell_keys_grids(const double* __restrict__ x, const double* __restrict__ y, int64_t nm, double dx,
                                  double dy, const GridKeys g, unsigned long long* __restrict__ bad_counter) {
    const int lane = threadIdx.x & 31;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < nm; base += stride) {
        const int64_t m = base + threadIdx.x;
        const bool live = m < nm;
        const double xm = live ? x[m] : 0.0, ym = live ? y[m] : 0.0;
        const unsigned active = __ballot_sync(0xffffffffu, live);
#pragma unroll
        for (int k = 0; k < SF_MAX_GRIDS; ++k) {
            if (k >= g.n) break;
            if (!live) continue;
            int32_t key = -1;
            const TopLeft t = topleft(g.xmin[k], g.ymin[k], xm, ym, dx, dy);
            // MarkerToGrid.jl:66: accept iff 0 <= ix <= Nx && 0 <= iy <= Ny (ix = qx + 1)
            if (t.qx >= -1.0 && t.qx <= (double)(g.nx[k] - 1) && t.qy >= -1.0 && t.qy <= (double)(g.ny[k] - 1))
                key = (int32_t)((int64_t)t.qx + 1 + ((int64_t)t.qy + 1) * (g.nx[k] + 1));
            g.keys[k][m] = key;
            const unsigned peers = __match_any_sync(active, key);
            if (lane == __ffs(peers) - 1) {
                const int n = __popc(peers);
                if (key >= 0)
                    atomicAdd(&g.counts[k][key], n);
                else if (bad_counter)
                    atomicAdd(bad_counter, (unsigned long long)n);
            }
        }
    }
}

// 3. scatter marker indices into their cells (order within a cell arbitrary).
__global__ void k_scatter(const int32_t* __restrict__ keys, int64_t nm, const int32_t* __restrict__ offsets,
                          int32_t* __restrict__ cursor, int32_t* __restrict__ perm) {
    const int lane = threadIdx.x & 31;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < nm; base += stride) {
        int64_t m = base + threadIdx.x;
        int32_t key = (m < nm) ? keys[m] : -1;
        unsigned active = __ballot_sync(0xffffffffu, key >= 0);
        if (key >= 0) {
            unsigned peers = __match_any_sync(active, key);
            int leader = __ffs(peers) - 1;
            int32_t pos0 = 0;
            if (lane == leader) pos0 = atomicAdd(&cursor[key], __popc(peers));
            pos0 = __shfl_sync(peers, pos0, leader);
            int rank = __popc(peers & ((1u << lane) - 1u));
            perm[offsets[key] + pos0 + rank] = (int32_t)m;
        }
    }
}

// The allocation-free deposit's per-cell sort of short segments (one thread per cell; its long segments are
// sorted by k_sort_long first, and are skipped here).
__global__ void k_sort_segments(const int32_t* __restrict__ offsets, int64_t ncells, int32_t* __restrict__ perm) {
    int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (c >= ncells) return;
    int32_t b = offsets[c], e = offsets[c + 1];
    if (e - b > SORT_LONG) return;
    for (int32_t i = b + 1; i < e; ++i) {
        int32_t v = perm[i];
        int32_t j = i - 1;
        if (perm[j] <= v) continue;
        while (j >= b && perm[j] > v) {
            perm[j + 1] = perm[j];
            --j;
        }
        perm[j + 1] = v;
    }
}

// 4a. the cells holding more than SORT_LONG markers -> list[0 .. *n_list)
__global__ void k_long_cells(const int32_t* __restrict__ offsets, int64_t ncells, int32_t* __restrict__ list,
                             int32_t* __restrict__ n_list) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ncells; c += (int64_t)gridDim.x * blockDim.x)
        if (offsets[c + 1] - offsets[c] > SORT_LONG) list[atomicAdd(n_list, 1)] = (int32_t)c;
}

// 4b. each long cell's segment sorted ascending in place by a block-wide LSD radix sort on 8-bit digits of the
// marker index (indices are non-negative 31-bit values: 4 digits), stable, through `tmp` at the same offsets.
// A digit on which the whole segment agrees moves nothing and is skipped.  Tiles of SORT_THREADS entries are
// ranked in order: lanes within a warp by __match_any_sync, warps by their per-digit counts.
__global__ void __launch_bounds__(SORT_THREADS) k_sort_long(const int32_t* __restrict__ offsets,
                                                            const int32_t* __restrict__ list,
                                                            const int32_t* __restrict__ n_list, int32_t* perm,
                                                            int32_t* tmp) {
    constexpr int NW = SORT_THREADS / 32;
    __shared__ int hist[256];
    __shared__ int base[256];
    __shared__ int wcnt[NW][256];
    __shared__ int skip;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int n_long = *n_list;
    for (int li = blockIdx.x; li < n_long; li += gridDim.x) {
        const int c = list[li];
        const int32_t b = offsets[c], n = offsets[c + 1] - b;
        int32_t* src = perm + b;
        int32_t* dst = tmp + b;
        for (int shift = 0; shift < 32; shift += 8) {
            hist[tid] = 0;
            __syncthreads();
            for (int i = tid; i < n; i += SORT_THREADS) atomicAdd(&hist[(src[i] >> shift) & 255], 1);
            __syncthreads();
            if (tid == 0) {
                int run = 0, same = 0;
                for (int d = 0; d < 256; ++d) {
                    base[d] = run;
                    run += hist[d];
                    same |= (hist[d] == n);
                }
                skip = same;
            }
            __syncthreads();
            if (skip) continue;
            for (int t0 = 0; t0 < n; t0 += SORT_THREADS) {
                for (int k = tid; k < NW * 256; k += SORT_THREADS) (&wcnt[0][0])[k] = 0;
                __syncthreads();
                const int i = t0 + tid;
                const bool valid = i < n;
                const int32_t v = valid ? src[i] : 0;
                const int d = (v >> shift) & 255;
                const unsigned act = __ballot_sync(0xffffffffu, valid);
                int rank = 0;
                if (valid) {
                    const unsigned peers = __match_any_sync(act, d);
                    rank = __popc(peers & ((1u << lane) - 1u));
                    if (lane == __ffs(peers) - 1) wcnt[warp][d] = __popc(peers);
                }
                __syncthreads();
                if (valid) {
                    int off = base[d] + rank;
                    for (int w = 0; w < warp; ++w) off += wcnt[w][d];
                    dst[off] = v;
                }
                __syncthreads();
                int sum = 0;
                for (int w = 0; w < NW; ++w) sum += wcnt[w][tid];
                base[tid] += sum;
                __syncthreads();
            }
            int32_t* t = src;
            src = dst;
            dst = t;
        }
        if (src != perm + b)
            for (int i = tid; i < n; i += SORT_THREADS) perm[b + i] = src[i];
        __syncthreads();
    }
}

// 4c. every short segment sorted ascending; long segments (sorted by k_sort_long) pass through in order.  A
// block takes SORT_CPB consecutive cells and works through them in windows of consecutive cells holding at most
// SORT_CAP entries: it loads a window's marker indices into shared memory, ranks each entry within its cell by
// counting the smaller indices there, and writes it to its sorted place -- back into perm (the rebin), or as a
// payload record (the deposit: topleftIndexRelDist of the marker and its value, once per marker).
template <bool PAYLOAD>
__global__ void __launch_bounds__(SORT_THREADS) k_sort_cells(const int32_t* __restrict__ offsets, int64_t ncells,
                                                             int32_t* perm, Payload* __restrict__ out,
                                                             const double* __restrict__ x, const double* __restrict__ y,
                                                             const double* __restrict__ val, double xmin, double ymin,
                                                             double dx, double dy) {
    __shared__ int32_t soff[SORT_CPB + 1];
    __shared__ int32_t sm[SORT_CAP];
    const int tid = threadIdx.x;
    const int64_t c0 = (int64_t)blockIdx.x * SORT_CPB;
    if (c0 >= ncells) return;
    const int nc = (int)min((int64_t)SORT_CPB, ncells - c0);
    for (int i = tid; i <= nc; i += SORT_THREADS) soff[i] = offsets[c0 + i];
    __syncthreads();
    auto emit = [&](int32_t pos, int32_t m) {
        if (PAYLOAD) {
            const TopLeft t = topleft(xmin, ymin, x[m], y[m], dx, dy);
            Payload p;
            p.dxij = t.dxij;
            p.dyij = t.dyij;
            p.val = val[m];
            p.m = m;
            p.pad_ = 0;
            out[pos] = p;
        } else {
            perm[pos] = m;
        }
    };
    int w0 = 0;
    while (w0 < nc) {
        // the largest w1 with soff[w1] - soff[w0] <= SORT_CAP (w1 == w0: cell w0 alone holds more)
        int lo = w0, hi = nc;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (soff[mid] - soff[w0] <= SORT_CAP) lo = mid; else hi = mid - 1;
        }
        const int w1 = lo;
        if (w1 == w0) {  // a long cell, sorted already: pass it through
            if (PAYLOAD)
                for (int32_t pos = soff[w0] + tid; pos < soff[w0 + 1]; pos += SORT_THREADS) emit(pos, perm[pos]);
            ++w0;
            continue;
        }
        const int32_t e0 = soff[w0];
        const int ne = soff[w1] - e0;
        for (int i = tid; i < ne; i += SORT_THREADS) sm[i] = perm[e0 + i];
        __syncthreads();
        for (int i = tid; i < ne; i += SORT_THREADS) {
            // the entry's cell k: the last one in [w0, w1) starting at or before it
            int a = w0, z = w1 - 1;
            while (a < z) {
                const int mid = (a + z + 1) >> 1;
                if (soff[mid] - e0 <= i) a = mid; else z = mid - 1;
            }
            const int cb = soff[a] - e0, ce = soff[a + 1] - e0;
            int rank = i - cb;
            if (ce - cb <= SORT_LONG) {
                const int32_t v = sm[i];
                rank = 0;
                for (int j = cb; j < ce; ++j) rank += (sm[j] < v) ? 1 : 0;
            }
            emit(e0 + cb + rank, sm[i]);
        }
        __syncthreads();
        w0 = w1;
    }
}

// 5. per-node gather over the sorted payload.  Node (I, J), 1-based.  A marker in cell (ix, iy) contributes to
// node (ix, iy) with (1-dx)(1-dy), (ix+1, iy) with dx(1-dy), (ix, iy+1) with (1-dx)dy and (ix+1, iy+1) with dx*dy
// (MarkerToGrid.jl:124-151), so node (I, J) merges the cells (I,J), (I-1,J), (I,J-1), (I-1,J-1), whose records
// are sorted by marker index: taking the smallest head each time visits the node's markers in ascending
// index order, the reference's serial order.
//
// Each list's head record is held in registers, so a visit reads its record once, with one 32-byte load (the
// four threads that use a record read it from L2).  The merge gallops: once the smallest head is chosen, the
// records of its list that stay below the other lists' smallest head are the merge's next picks, in order,
// and are taken in an inner loop without comparing the four heads again.  Markers keep much of their initial
// lattice order, so these runs are several records long.
constexpr int GT_NONE = 0x7fffffff;   // head of an exhausted list
constexpr int GT_X = 32, GT_Y = 4;    // nodes of a block: one warp per node row, 4 rows that share cell rows
// (launched 8 blocks per SM: 64 registers, more warps in flight than a spill-free 68)

__global__ void __launch_bounds__(GT_X * GT_Y, 8) k_gather_sorted(const Payload* __restrict__ pl,
                                                               const int32_t* __restrict__ offsets, int64_t nx,
                                                               int64_t ny, double* __restrict__ val_grid,
                                                               double* __restrict__ val_wt_sum,
                                                               double* __restrict__ wt_sum, int64_t ld_sum,
                                                               unsigned long long* __restrict__ empty_counter) {
    const int64_t ntx = (nx + GT_X - 1) / GT_X;
    const int64_t I = (int64_t)(blockIdx.x % ntx) * GT_X + (threadIdx.x % GT_X) + 1;
    const int64_t J = (int64_t)(blockIdx.x / ntx) * GT_Y + (threadIdx.x / GT_X) + 1;
    if (I > nx || J > ny) return;
    const int64_t ldc = nx + 1;
    // corner k: 0 = marker's top-left node (cell I,J), 1 = top-right (cell I-1,J),
    //           2 = bottom-left (cell I,J-1), 3 = bottom-right (cell I-1,J-1)
    int32_t cur[4], end[4], hm[4];
    double hdx[4], hdy[4], hv[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int64_t key = (I - (k & 1)) + (J - (k >> 1)) * ldc;
        cur[k] = offsets[key];
        end[k] = offsets[key + 1];
        hdx[k] = hdy[k] = hv[k] = 0.0;
        hm[k] = GT_NONE;
        if (cur[k] < end[k]) {
            const Payload p = pl[cur[k]];
            hdx[k] = p.dxij;
            hdy[k] = p.dyij;
            hv[k] = p.val;
            hm[k] = p.m;
        }
    }
    double ws = 0.0, vs = 0.0;
    while (true) {
        int kb = 0;
        int32_t best = hm[0];
#pragma unroll
        for (int k = 1; k < 4; ++k)
            if (hm[k] < best) {
                best = hm[k];
                kb = k;
            }
        if (best == GT_NONE) break;
        int32_t t = GT_NONE;   // the smallest head of the other lists
        int32_t c = 0, e = 0;
        double dx = 0.0, dy = 0.0, v = 0.0;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (k != kb && hm[k] < t) t = hm[k];
            if (k == kb) {
                c = cur[k];
                e = end[k];
                dx = hdx[k];
                dy = hdy[k];
                v = hv[k];
            }
        }
        const bool fx = kb & 1, fy = kb >> 1;
        int32_t h;
        do {   // list kb's run below t
            const double wx = fx ? dx : (1.0 - dx);
            const double wy = fy ? dy : (1.0 - dy);
            const double w = wx * wy;
            ws = ws + w;
            vs = vs + w * v;
            ++c;
            h = GT_NONE;
            if (c < e) {
                const Payload p = pl[c];
                dx = p.dxij;
                dy = p.dyij;
                v = p.val;
                h = p.m;
            }
        } while (h < t);
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (k == kb) {
                cur[k] = c;
                hm[k] = h;
                hdx[k] = dx;
                hdy[k] = dy;
                hv[k] = v;
            }
    }
    if (wt_sum) {
        wt_sum[(I - 1) + (J - 1) * ld_sum] = ws;
        val_wt_sum[(I - 1) + (J - 1) * ld_sum] = vs;
    }
    if (ws != 0.0)
        val_grid[(I - 1) + (J - 1) * nx] = vs / ws;   // safeDivision (MarkerToGrid.jl:164-172)
    else if (empty_counter)
        atomicAdd(empty_counter, 1ull);
}

// The allocation-free deposit's gather (its scratch holds no payload): the same merge of node (I, J)'s cells
// (I,J), (I-1,J), (I,J-1), (I-1,J-1) in ascending marker index, reading each marker's position and value
// through the sorted permutation.
__global__ void k_gather(const double* __restrict__ x, const double* __restrict__ y, const double* __restrict__ val,
                         const int32_t* __restrict__ offsets, const int32_t* __restrict__ perm, int64_t nx,
                         int64_t ny, double xmin, double ymin, double dx, double dy, double* __restrict__ val_grid,
                         double* __restrict__ val_wt_sum, double* __restrict__ wt_sum, int64_t ld_sum,
                         unsigned long long* __restrict__ empty_counter) {
    int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t nnodes = nx * ny;
    bool live = n < nnodes;
    int64_t I = live ? n % nx + 1 : 1, J = live ? n / nx + 1 : 1;
    int32_t cur[4], end[4];
    const int64_t ldc = nx + 1;
    // corner k: 0 = marker's top-left node (cell I,J), 1 = top-right (cell I-1,J),
    //           2 = bottom-left (cell I,J-1), 3 = bottom-right (cell I-1,J-1)
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        int64_t ci = I - (k & 1), cj = J - (k >> 1);
        int64_t key = ci + cj * ldc;
        cur[k] = live ? offsets[key] : 0;
        end[k] = live ? offsets[key + 1] : 0;
    }
    double ws = 0.0, vs = 0.0;
    while (true) {
        int32_t best = 0x7fffffff;
        int kb = -1;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (cur[k] < end[k]) {
                int32_t m = perm[cur[k]];
                if (m < best) { best = m; kb = k; }
            }
        }
        if (kb < 0) break;
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (k == kb) ++cur[k];
        TopLeft t = topleft(xmin, ymin, x[best], y[best], dx, dy);
        double wx = (kb & 1) ? t.dxij : (1.0 - t.dxij);
        double wy = (kb >> 1) ? t.dyij : (1.0 - t.dyij);
        double w = wx * wy;
        ws = ws + w;
        vs = vs + w * val[best];
    }
    if (!live) return;
    if (wt_sum) {
        wt_sum[(I - 1) + (J - 1) * ld_sum] = ws;
        val_wt_sum[(I - 1) + (J - 1) * ld_sum] = vs;
    }
    if (ws != 0.0)
        val_grid[(I - 1) + (J - 1) * nx] = vs / ws;
    else if (empty_counter)
        atomicAdd(empty_counter, 1ull);
}

static unsigned grid_for(sf_ctx* ctx, int64_t n, int threads) {
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(ceil_div(n, threads), (int64_t)ctx->num_sms * 32));
}

// Steps 2-4 from cell keys and per-cell counts already computed (step 1): the stable counting sort of markers by
// cell -> ctx->offsets, and either the cell-ordered permutation in ctx->perm or (with val) the cell-ordered
// payload records in ctx->payload.  keys is spent afterwards: it is the radix sort's second buffer.
static int sort_from_keys(sf_ctx* ctx, int32_t* keys, const int32_t* counts, const double* x, const double* y,
                          const double* val, int64_t nm, double xmin, double ymin, double dx, double dy, int64_t nx,
                          int64_t ny, cudaStream_t s) {
    int64_t ncells = (nx + 1) * (ny + 1);
    int rc;
    if ((rc = ensure(ctx, ctx->perm, (size_t)std::max<int64_t>(nm, 1) * 4))) return rc;
    if ((rc = ensure(ctx, ctx->offsets, (size_t)(ncells + 1) * 4))) return rc;
    if ((rc = ensure(ctx, ctx->cursor, (size_t)(ncells + 1) * 4))) return rc;
    if ((rc = ensure(ctx, ctx->longs, (size_t)(ncells + 1) * 4))) return rc;
    if (val && (rc = ensure(ctx, ctx->payload, (size_t)std::max<int64_t>(nm, 1) * sizeof(Payload)))) return rc;
    int32_t* offsets = (int32_t*)ctx->offsets.ptr;
    int32_t* cursor = (int32_t*)ctx->cursor.ptr;
    int32_t* perm = (int32_t*)ctx->perm.ptr;
    int32_t* n_long = (int32_t*)ctx->longs.ptr;   // the count, then the list
    SF_CUDA(cudaMemsetAsync(cursor, 0, (size_t)(ncells + 1) * 4, s));
    SF_CUDA(cudaMemsetAsync(n_long, 0, 4, s));
    if ((rc = exclusive_scan_i32(ctx, counts, offsets, ncells, offsets + ncells, s))) return rc;
    if (nm > 0) {
        k_scatter<<<grid_for(ctx, nm, DEP_THREADS), DEP_THREADS, 0, s>>>(keys, nm, offsets, cursor, perm);
        SF_LAUNCHED(ctx);
        k_long_cells<<<grid_for(ctx, ncells, DEP_THREADS), DEP_THREADS, 0, s>>>(offsets, ncells, n_long + 1, n_long);
        SF_LAUNCHED(ctx);
        // the keys are spent: they are the radix sort's second buffer
        k_sort_long<<<(unsigned)ctx->num_sms * 2, SORT_THREADS, 0, s>>>(offsets, n_long + 1, n_long, perm, keys);
        SF_LAUNCHED(ctx);
        const unsigned blocks = (unsigned)ceil_div(ncells, SORT_CPB);
        if (val)
            k_sort_cells<true><<<blocks, SORT_THREADS, 0, s>>>(offsets, ncells, perm, (Payload*)ctx->payload.ptr, x, y,
                                                               val, xmin, ymin, dx, dy);
        else
            k_sort_cells<false><<<blocks, SORT_THREADS, 0, s>>>(offsets, ncells, perm, nullptr, x, y, val, xmin, ymin,
                                                                dx, dy);
        SF_LAUNCHED(ctx);
    }
    return SF_OK;
}

// Steps 1-4 for one grid: cell keys and counts into ctx->keys / ctx->counts, then the sort.
static int sort_by_cell(sf_ctx* ctx, const double* x, const double* y, const double* val, int64_t nm, double xmin,
                        double ymin, double dx, double dy, int64_t nx, int64_t ny, unsigned long long* bad_counter,
                        cudaStream_t s) {
    int64_t ncells = (nx + 1) * (ny + 1);
    int rc;
    if ((rc = ensure(ctx, ctx->keys, (size_t)std::max<int64_t>(nm, 1) * 4))) return rc;
    if ((rc = ensure(ctx, ctx->counts, (size_t)(ncells + 1) * 4))) return rc;
    int32_t* keys = (int32_t*)ctx->keys.ptr;
    int32_t* counts = (int32_t*)ctx->counts.ptr;
    SF_CUDA(cudaMemsetAsync(counts, 0, (size_t)(ncells + 1) * 4, s));
    if (nm > 0) {
        k_cell_keys<<<grid_for(ctx, nm, DEP_THREADS), DEP_THREADS, 0, s>>>(x, y, nm, xmin, ymin, dx, dy, nx, ny, keys,
                                                                             counts, bad_counter);
        SF_LAUNCHED(ctx);
    }
    return sort_from_keys(ctx, keys, counts, x, y, val, nm, xmin, ymin, dx, dy, nx, ny, s);
}

static void launch_gather(sf_ctx* ctx, int64_t nx, int64_t ny, double* val_grid, double* val_wt_sum, double* wt_sum,
                          int64_t ld_sum, cudaStream_t s) {
    k_gather_sorted<<<(unsigned)(ceil_div(nx, GT_X) * ceil_div(ny, GT_Y)), GT_X * GT_Y, 0, s>>>(
        (const Payload*)ctx->payload.ptr, (const int32_t*)ctx->offsets.ptr, nx, ny, val_grid, val_wt_sum, wt_sum,
        ld_sum, ctx->d_counters + CNT_EMPTY_NODES);
}

}  // namespace sf

using namespace sf;

extern "C" {

int sf_bilinear_marker_to_grid(sf_ctx* ctx, double x_grid_min, double y_grid_min, double* val_grid, int64_t nx,
                               int64_t ny, const double* x_m, const double* y_m, const double* val_m, int64_t nm,
                               double dx, double dy, double* val_wt_sum, double* wt_sum, int64_t ld_sum,
                               int64_t n_sum, void* stream) {
    SF_REQUIRE(ctx, "sf_bilinear_marker_to_grid: ctx is NULL");
    SF_REQUIRE(val_grid && nx >= 1 && ny >= 1, "sf_bilinear_marker_to_grid: bad grid");
    SF_REQUIRE(nm >= 0 && (nm == 0 || (x_m && y_m && val_m)), "sf_bilinear_marker_to_grid: bad markers");
    SF_REQUIRE(nm < (int64_t)INT32_MAX, "sf_bilinear_marker_to_grid: more than 2^31-1 markers");
    SF_REQUIRE((nx + 1) * (ny + 1) < (int64_t)INT32_MAX, "sf_bilinear_marker_to_grid: grid too large");
    SF_REQUIRE(dx > 0.0 && dy > 0.0, "sf_bilinear_marker_to_grid: dx, dy must be positive");
    SF_REQUIRE((val_wt_sum == nullptr) == (wt_sum == nullptr), "sf_bilinear_marker_to_grid: give both sum arrays or neither");
    if (wt_sum) SF_REQUIRE(ld_sum >= nx && n_sum >= ld_sum * (ny - 1) + nx, "sf_bilinear_marker_to_grid: sum arrays too small");
    int rc = set_device(ctx);
    if (rc) return rc;
    cudaStream_t s = as_stream(stream);
    if ((rc = sort_by_cell(ctx, x_m, y_m, val_m, nm, x_grid_min, y_grid_min, dx, dy, nx, ny,
                           ctx->d_counters + CNT_BAD_MARKERS, s)))
        return rc;
    if (wt_sum) {
        SF_CUDA(cudaMemsetAsync(wt_sum, 0, (size_t)n_sum * 8, s));
        SF_CUDA(cudaMemsetAsync(val_wt_sum, 0, (size_t)n_sum * 8, s));
    }
    launch_gather(ctx, nx, ny, val_grid, val_wt_sum, wt_sum, ld_sum, s);
    SF_LAUNCHED(ctx);
    return SF_OK;
}

int sf_bilinear_marker_to_grids(sf_ctx* ctx, const sf_deposit_grid* grids, int n_grids, const double* x_m,
                                const double* y_m, int64_t nm, double dx, double dy, double* val_wt_sum,
                                double* wt_sum, int64_t ld_sum, int64_t n_sum, void* stream) {
    SF_REQUIRE(ctx, "sf_bilinear_marker_to_grids: ctx is NULL");
    SF_REQUIRE(grids && n_grids >= 1 && n_grids <= SF_MAX_GRIDS, "sf_bilinear_marker_to_grids: 1 to SF_MAX_GRIDS grids");
    SF_REQUIRE(nm >= 0 && (nm == 0 || (x_m && y_m)), "sf_bilinear_marker_to_grids: bad markers");
    SF_REQUIRE(nm < (int64_t)INT32_MAX, "sf_bilinear_marker_to_grids: more than 2^31-1 markers");
    SF_REQUIRE(dx > 0.0 && dy > 0.0, "sf_bilinear_marker_to_grids: dx, dy must be positive");
    SF_REQUIRE((val_wt_sum == nullptr) == (wt_sum == nullptr), "sf_bilinear_marker_to_grids: give both sum arrays or neither");
    int64_t total_cells = 0;
    for (int g = 0; g < n_grids; ++g) {
        const sf_deposit_grid& d = grids[g];
        SF_REQUIRE(d.val_grid && d.nx >= 1 && d.ny >= 1, "sf_bilinear_marker_to_grids: bad grid");
        SF_REQUIRE(nm == 0 || d.val_m, "sf_bilinear_marker_to_grids: bad marker values");
        SF_REQUIRE((d.nx + 1) * (d.ny + 1) < (int64_t)INT32_MAX, "sf_bilinear_marker_to_grids: grid too large");
        if (wt_sum)
            SF_REQUIRE(ld_sum >= d.nx && n_sum >= ld_sum * (d.ny - 1) + d.nx,
                       "sf_bilinear_marker_to_grids: sum arrays too small");
        total_cells += (d.nx + 1) * (d.ny + 1) + 1;
    }
    int rc = set_device(ctx);
    if (rc) return rc;
    cudaStream_t s = as_stream(stream);
    const int64_t nmk = std::max<int64_t>(nm, 1);
    if ((rc = ensure(ctx, ctx->keys, (size_t)(n_grids * nmk) * 4))) return rc;
    if ((rc = ensure(ctx, ctx->counts, (size_t)total_cells * 4))) return rc;
    int32_t* keys = (int32_t*)ctx->keys.ptr;
    int32_t* counts = (int32_t*)ctx->counts.ptr;
    SF_CUDA(cudaMemsetAsync(counts, 0, (size_t)total_cells * 4, s));
    GridKeys gk{};
    gk.n = n_grids;
    int64_t off = 0;
    for (int g = 0; g < n_grids; ++g) {
        gk.xmin[g] = grids[g].x_grid_min;
        gk.ymin[g] = grids[g].y_grid_min;
        gk.nx[g] = grids[g].nx;
        gk.ny[g] = grids[g].ny;
        gk.keys[g] = keys + g * nmk;
        gk.counts[g] = counts + off;
        off += (grids[g].nx + 1) * (grids[g].ny + 1) + 1;
    }
    if (nm > 0) {
        k_cell_keys_grids<<<grid_for(ctx, nm, DEP_THREADS), DEP_THREADS, 0, s>>>(x_m, y_m, nm, dx, dy, gk,
                                                                                   ctx->d_counters + CNT_BAD_MARKERS);
        SF_LAUNCHED(ctx);
    }
    for (int g = 0; g < n_grids; ++g) {
        const sf_deposit_grid& d = grids[g];
        if ((rc = sort_from_keys(ctx, gk.keys[g], gk.counts[g], x_m, y_m, d.val_m, nm, d.x_grid_min, d.y_grid_min, dx,
                                 dy, d.nx, d.ny, s)))
            return rc;
        // as after one call per grid in order: the sum arrays hold the last grid's sums
        const bool last = g == n_grids - 1;
        if (wt_sum && last) {
            SF_CUDA(cudaMemsetAsync(wt_sum, 0, (size_t)n_sum * 8, s));
            SF_CUDA(cudaMemsetAsync(val_wt_sum, 0, (size_t)n_sum * 8, s));
        }
        launch_gather(ctx, d.nx, d.ny, d.val_grid, last ? val_wt_sum : nullptr, last ? wt_sum : nullptr, ld_sum, s);
        SF_LAUNCHED(ctx);
    }
    return SF_OK;
}

int sf_rebin_markers(sf_ctx* ctx, const double* x_m, const double* y_m, int64_t nm, double x_grid_min,
                     double y_grid_min, double dx, double dy, int64_t nx, int64_t ny, int32_t* counts,
                     int32_t* offsets, int32_t* perm, void* stream) {
    SF_REQUIRE(ctx, "sf_rebin_markers: ctx is NULL");
    SF_REQUIRE(nx >= 1 && ny >= 1 && dx > 0.0 && dy > 0.0, "sf_rebin_markers: bad grid");
    SF_REQUIRE(nm >= 0 && (nm == 0 || (x_m && y_m)), "sf_rebin_markers: bad markers");
    SF_REQUIRE(nm < (int64_t)INT32_MAX && (nx + 1) * (ny + 1) < (int64_t)INT32_MAX, "sf_rebin_markers: too large");
    int rc = set_device(ctx);
    if (rc) return rc;
    cudaStream_t s = as_stream(stream);
    if ((rc = sort_by_cell(ctx, x_m, y_m, nullptr, nm, x_grid_min, y_grid_min, dx, dy, nx, ny,
                           ctx->d_counters + CNT_OUTSIDE, s)))
        return rc;
    int64_t ncells = (nx + 1) * (ny + 1);
    if (counts) SF_CUDA(cudaMemcpyAsync(counts, ctx->counts.ptr, (size_t)ncells * 4, cudaMemcpyDeviceToDevice, s));
    if (offsets) SF_CUDA(cudaMemcpyAsync(offsets, ctx->offsets.ptr, (size_t)(ncells + 1) * 4, cudaMemcpyDeviceToDevice, s));
    if (perm && nm > 0) SF_CUDA(cudaMemcpyAsync(perm, ctx->perm.ptr, (size_t)nm * 4, cudaMemcpyDeviceToDevice, s));
    return SF_OK;
}

}  // extern "C"

// ==========================================================================
// Allocation-free deposit
// ==========================================================================
// Some callers cannot let a library call cudaMalloc / cudaFree: hosts whose
// runtime owns the device memory through its own pool (for example Julia's
// CUDA.jl or PyTorch with the rest of the GPU reserved), where an allocation
// outside the pool fails or forces an eviction; latency-critical stream loops,
// where cudaMalloc / cudaFree synchronise the whole device and stall the other
// streams; and processes held to a fixed memory budget after start-up.  For
// them sf_bilinear_marker_to_grid_noalloc runs the same deposit with all of
// its scratch in the file-scope array below, which every GPU that loads the
// library holds (about 11 MB) until the process exits.
#include <mutex>

namespace sf {

constexpr int64_t NA_MAX_MARKERS = SF_NOALLOC_MAX_MARKERS;
constexpr int64_t NA_MAX_CELLS = SF_NOALLOC_MAX_CELLS;          // (nx + 1) * (ny + 1)
constexpr int64_t NA_SCAN_TILES = (NA_MAX_CELLS + 1 + 8191) / 8192;
// layout (bytes): keys | perm | counts | offsets | cursor | scan tiles | counters
constexpr size_t NA_OFF_KEYS = 0;
constexpr size_t NA_OFF_PERM = NA_OFF_KEYS + 4 * NA_MAX_MARKERS;
constexpr size_t NA_OFF_COUNTS = NA_OFF_PERM + 4 * NA_MAX_MARKERS;
constexpr size_t NA_OFF_OFFSETS = NA_OFF_COUNTS + 4 * (NA_MAX_CELLS + 64);
constexpr size_t NA_OFF_CURSOR = NA_OFF_OFFSETS + 4 * (NA_MAX_CELLS + 64);
constexpr size_t NA_OFF_TILES = NA_OFF_CURSOR + 4 * (NA_MAX_CELLS + 64);
constexpr size_t NA_OFF_COUNTERS = NA_OFF_TILES + 4 * ((NA_SCAN_TILES + 63) / 64 * 64);
constexpr size_t NA_BYTES = NA_OFF_COUNTERS + 4 * sizeof(unsigned long long);   // 2 counters, the long-cell count

static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_BYTES];

constexpr int NA_MAX_DEVICES = 64;
static unsigned char* g_noalloc_ptr[NA_MAX_DEVICES] = {};
static int g_noalloc_sms[NA_MAX_DEVICES] = {};
static std::mutex g_noalloc_mutex;

// Device address of g_noalloc_scratch and the SM count of the current device.
// In host code the array's name is only a host-side stand-in, so the address
// is looked up once per device (with that device current) and cached, with
// the SM count that sizes the marker kernels' grids.  A device reset
// invalidates the cache (documented at the declaration).
static int noalloc_scratch(unsigned char** out, int* num_sms) {
    int dev = 0;
    SF_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= NA_MAX_DEVICES) return fail(SF_ERR_NO_DEVICE, "noalloc deposit: device index too large");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
        int sms = 0;
        SF_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            (void)cudaGetLastError();
            return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)", __FILE__, __LINE__);
        }
        g_noalloc_sms[dev] = std::max(1, sms);
        g_noalloc_ptr[dev] = (unsigned char*)p;
    }
    *out = g_noalloc_ptr[dev];
    *num_sms = g_noalloc_sms[dev];
    return SF_OK;
}

}  // namespace sf

extern "C" int sf_bilinear_marker_to_grid_noalloc(double x_grid_min, double y_grid_min, double* val_grid, int64_t nx,
                                                  int64_t ny, const double* x_m, const double* y_m, const double* val_m,
                                                  int64_t nm, double dx, double dy, void* stream) {
    SF_REQUIRE(val_grid && nx >= 1 && ny >= 1, "sf_bilinear_marker_to_grid_noalloc: bad grid");
    SF_REQUIRE(nm >= 0 && (nm == 0 || (x_m && y_m && val_m)), "sf_bilinear_marker_to_grid_noalloc: bad markers");
    SF_REQUIRE(dx > 0.0 && dy > 0.0, "sf_bilinear_marker_to_grid_noalloc: dx, dy must be positive");
    if (nm > NA_MAX_MARKERS)
        return fail(SF_ERR_TOO_LARGE, "sf_bilinear_marker_to_grid_noalloc: " + std::to_string(nm) +
                                          " markers exceed the fixed scratch (at most " +
                                          std::to_string(NA_MAX_MARKERS) + ")");
    if (nx > NA_MAX_CELLS || ny > NA_MAX_CELLS || (nx + 1) * (ny + 1) > NA_MAX_CELLS)
        return fail(SF_ERR_TOO_LARGE, "sf_bilinear_marker_to_grid_noalloc: a " + std::to_string(nx) + " x " +
                                          std::to_string(ny) + " grid exceeds the fixed scratch (at most " +
                                          std::to_string(NA_MAX_CELLS) + " cells (nx+1)*(ny+1))");
    unsigned char* base = nullptr;
    int num_sms = 0;
    int rc = noalloc_scratch(&base, &num_sms);
    if (rc) return rc;
    cudaStream_t s = as_stream(stream);
    int32_t* keys = (int32_t*)(base + NA_OFF_KEYS);
    int32_t* perm = (int32_t*)(base + NA_OFF_PERM);
    int32_t* counts = (int32_t*)(base + NA_OFF_COUNTS);
    int32_t* offsets = (int32_t*)(base + NA_OFF_OFFSETS);
    int32_t* cursor = (int32_t*)(base + NA_OFF_CURSOR);
    int32_t* tiles = (int32_t*)(base + NA_OFF_TILES);
    unsigned long long* counters = (unsigned long long*)(base + NA_OFF_COUNTERS);
    const int64_t ncells = (nx + 1) * (ny + 1);
    int32_t* n_long = (int32_t*)(counters + 2);
    // the array keeps the previous call's contents: clear what must start at zero
    SF_CUDA(cudaMemsetAsync(counts, 0, (size_t)(ncells + 1) * 4, s));
    SF_CUDA(cudaMemsetAsync(cursor, 0, (size_t)(ncells + 1) * 4, s));
    SF_CUDA(cudaMemsetAsync(counters, 0, 4 * sizeof(unsigned long long), s));
    // grid-stride marker kernels: up to 32 blocks per SM of this device
    const unsigned blocks =
        (unsigned)std::max<int64_t>(1, std::min<int64_t>(ceil_div(nm, DEP_THREADS), (int64_t)num_sms * 32));
    if (nm > 0) {
        k_cell_keys<<<blocks, DEP_THREADS, 0, s>>>(x_m, y_m, nm, x_grid_min, y_grid_min, dx, dy, nx, ny, keys, counts,
                                                   counters + 0);
        SF_CHECK_LAUNCH();
    }
    if ((rc = exclusive_scan_i32_into(counts, offsets, ncells, offsets + ncells, tiles, s))) return rc;
    if (nm > 0) {
        k_scatter<<<blocks, DEP_THREADS, 0, s>>>(keys, nm, offsets, cursor, perm);
        SF_CHECK_LAUNCH();
        // long segments by the radix sort (the spent cursors hold their list, the spent keys are its buffer),
        // the others one thread per cell
        k_long_cells<<<blocks, DEP_THREADS, 0, s>>>(offsets, ncells, cursor, n_long);
        SF_CHECK_LAUNCH();
        k_sort_long<<<(unsigned)num_sms * 2, SORT_THREADS, 0, s>>>(offsets, cursor, n_long, perm, keys);
        SF_CHECK_LAUNCH();
    }
    k_sort_segments<<<(unsigned)ceil_div(ncells, 128), 128, 0, s>>>(offsets, ncells, perm);
    SF_CHECK_LAUNCH();
    k_gather<<<(unsigned)ceil_div(nx * ny, DEP_THREADS), DEP_THREADS, 0, s>>>(
        x_m, y_m, val_m, offsets, perm, nx, ny, x_grid_min, y_grid_min, dx, dy, val_grid, nullptr, nullptr, 0,
        counters + 1);
    SF_CHECK_LAUNCH();
    return SF_OK;
}
