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
//   3. k_scatter       marker indices into their cell's segment.
//   4. k_sort_segments each segment sorted ascending (insertion sort; a cell
//                      holds ~16-25 markers), giving a stable counting sort.
//   5. k_gather        one thread per node merges the four adjacent cells'
//                      segments by marker index and accumulates w and w*val in
//                      ascending marker order -- the reference CPU loop's
//                      order, so each node's sums are bit-identical to it --
//                      then divides (safeDivision, :164-172).
// Steps 1-4 are also the rebin (sf_rebin_markers).
#include <algorithm>

#include "sf_internal.cuh"

namespace sf {

constexpr int DEP_THREADS = 256;

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

// 4. sort every cell segment ascending (one thread per cell).
__global__ void k_sort_segments(const int32_t* __restrict__ offsets, int64_t ncells, int32_t* __restrict__ perm) {
    int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (c >= ncells) return;
    int32_t b = offsets[c], e = offsets[c + 1];
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

// 5. per-node gather.  Node (I, J), 1-based.  A marker in cell (ix, iy)
// contributes to node (ix, iy) with (1-dx)(1-dy), (ix+1, iy) with dx(1-dy),
// (ix, iy+1) with (1-dx)dy and (ix+1, iy+1) with dx*dy (MarkerToGrid.jl:124-151),
// so node (I, J) merges the cells (I,J), (I-1,J), (I,J-1), (I-1,J-1).
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

// Steps 1-4: stable counting sort of markers by cell -> ctx->counts/offsets/perm.
static int sort_by_cell(sf_ctx* ctx, const double* x, const double* y, int64_t nm, double xmin, double ymin,
                        double dx, double dy, int64_t nx, int64_t ny, unsigned long long* bad_counter,
                        cudaStream_t s) {
    int64_t ncells = (nx + 1) * (ny + 1);
    int rc;
    if ((rc = ensure(ctx, ctx->keys, (size_t)std::max<int64_t>(nm, 1) * 4))) return rc;
    if ((rc = ensure(ctx, ctx->perm, (size_t)std::max<int64_t>(nm, 1) * 4))) return rc;
    if ((rc = ensure(ctx, ctx->counts, (size_t)(ncells + 1) * 4))) return rc;
    if ((rc = ensure(ctx, ctx->offsets, (size_t)(ncells + 1) * 4))) return rc;
    if ((rc = ensure(ctx, ctx->cursor, (size_t)(ncells + 1) * 4))) return rc;
    int32_t* keys = (int32_t*)ctx->keys.ptr;
    int32_t* counts = (int32_t*)ctx->counts.ptr;
    int32_t* offsets = (int32_t*)ctx->offsets.ptr;
    int32_t* cursor = (int32_t*)ctx->cursor.ptr;
    int32_t* perm = (int32_t*)ctx->perm.ptr;
    SF_CUDA(cudaMemsetAsync(counts, 0, (size_t)(ncells + 1) * 4, s));
    SF_CUDA(cudaMemsetAsync(cursor, 0, (size_t)(ncells + 1) * 4, s));
    if (nm > 0) {
        k_cell_keys<<<grid_for(ctx, nm, DEP_THREADS), DEP_THREADS, 0, s>>>(x, y, nm, xmin, ymin, dx, dy, nx, ny, keys,
                                                                             counts, bad_counter);
        SF_LAUNCHED(ctx);
    }
    if ((rc = exclusive_scan_i32(ctx, counts, offsets, ncells, offsets + ncells, s))) return rc;
    if (nm > 0) {
        k_scatter<<<grid_for(ctx, nm, DEP_THREADS), DEP_THREADS, 0, s>>>(keys, nm, offsets, cursor, perm);
        SF_LAUNCHED(ctx);
    }
    k_sort_segments<<<(unsigned)ceil_div(ncells, 128), 128, 0, s>>>(offsets, ncells, perm);
    SF_LAUNCHED(ctx);
    return SF_OK;
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
    if ((rc = sort_by_cell(ctx, x_m, y_m, nm, x_grid_min, y_grid_min, dx, dy, nx, ny,
                           ctx->d_counters + CNT_BAD_MARKERS, s)))
        return rc;
    if (wt_sum) {
        SF_CUDA(cudaMemsetAsync(wt_sum, 0, (size_t)n_sum * 8, s));
        SF_CUDA(cudaMemsetAsync(val_wt_sum, 0, (size_t)n_sum * 8, s));
    }
    int64_t nnodes = nx * ny;
    k_gather<<<(unsigned)ceil_div(nnodes, DEP_THREADS), DEP_THREADS, 0, s>>>(
        x_m, y_m, val_m, (const int32_t*)ctx->offsets.ptr, (const int32_t*)ctx->perm.ptr, nx, ny, x_grid_min,
        y_grid_min, dx, dy, val_grid, val_wt_sum, wt_sum, ld_sum, ctx->d_counters + CNT_EMPTY_NODES);
    SF_LAUNCHED(ctx);
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
    if ((rc = sort_by_cell(ctx, x_m, y_m, nm, x_grid_min, y_grid_min, dx, dy, nx, ny, ctx->d_counters + CNT_OUTSIDE,
                           s)))
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
constexpr size_t NA_BYTES = NA_OFF_COUNTERS + 2 * sizeof(unsigned long long);

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
    // the array keeps the previous call's contents: clear what must start at zero
    SF_CUDA(cudaMemsetAsync(counts, 0, (size_t)(ncells + 1) * 4, s));
    SF_CUDA(cudaMemsetAsync(cursor, 0, (size_t)(ncells + 1) * 4, s));
    SF_CUDA(cudaMemsetAsync(counters, 0, 2 * sizeof(unsigned long long), s));
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
    }
    k_sort_segments<<<(unsigned)ceil_div(ncells, 128), 128, 0, s>>>(offsets, ncells, perm);
    SF_CHECK_LAUNCH();
    k_gather<<<(unsigned)ceil_div(nx * ny, DEP_THREADS), DEP_THREADS, 0, s>>>(
        x_m, y_m, val_m, offsets, perm, nx, ny, x_grid_min, y_grid_min, dx, dy, val_grid, nullptr, nullptr, 0,
        counters + 1);
    SF_CHECK_LAUNCH();
    return SF_OK;
}
