// sf_internal.cuh -- shared internals of libstokesflow_b200.so: the context,
// status/error plumbing, grow-only scratch buffers and the small device
// helpers that every kernel file uses.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>
#include <map>
#include <utility>
#include <string>

#include "stokesflow_b200.h"

namespace sf {

// --------------------------------------------------------------------------
// errors
// --------------------------------------------------------------------------
void set_error(const std::string& msg);
int fail(int status, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what, const char* file, int line);

#define SF_CUDA(call)                                                   \
    do {                                                                \
        cudaError_t e_ = (call);                                        \
        if (e_ != cudaSuccess) return ::sf::cuda_fail(e_, #call, __FILE__, __LINE__); \
    } while (0)

#define SF_CHECK_LAUNCH() SF_CUDA(cudaGetLastError())

// after every kernel launch: check it and count it on the context
#define SF_LAUNCHED(c)        \
    do {                      \
        SF_CHECK_LAUNCH();    \
        ++(c)->launches;      \
    } while (0)

#define SF_REQUIRE(cond, msg)                                           \
    do {                                                                \
        if (!(cond)) return ::sf::fail(SF_ERR_INVALID_ARG, msg);        \
    } while (0)

// --------------------------------------------------------------------------
// scratch: a grow-only device buffer owned by the context
// --------------------------------------------------------------------------
struct Scratch {
    void* ptr = nullptr;
    size_t bytes = 0;
};

// device-side warning counters, in the order of sf_warnings
enum { CNT_BAD_MARKERS = 0, CNT_EMPTY_NODES = 1, CNT_INTERP_FAILSAFE = 2, CNT_OUTSIDE = 3, CNT_N = 4 };

// device scalars used by the PT solve
// SC_DT: dt used by the stabilisation term; SC_DT_CHECK: dt of the residual
// check; SC_DT_OUT: dt returned by the solve; SC_MAXBITS (2 slots): max|Vx|,
// max|Vy| as ordered bit patterns during a reduction.
enum { SC_DT = 0, SC_DT_CHECK = 1, SC_ERR = 2, SC_SUM_RX = 3, SC_SUM_RY = 4, SC_SUM_DIV = 5,
       SC_MAX_VX = 6, SC_MAX_VY = 7, SC_SCALE = 8, SC_DT_OUT = 9, SC_MAXBITS = 12, SC_N = 16 };

}  // namespace sf

struct sf_ctx {
    int device = 0;
    int num_sms = 148;
    // deposit / rebin scratch: cell keys, counts, offsets, scatter cursors, the cell-ordered permutation, scan
    // tiles, the deposit's sorted payload records and the list of long cells
    sf::Scratch keys, counts, offsets, cursor, perm, scan_tmp, payload, longs;
    // PT solve: padded internal fields, reduction partials; mixed/batched engine arena
    sf::Scratch fields, partials, mixed;
    // decomposed timestep: marker-exchange and overlap-sum staging
    sf::Scratch exch;
    cudaStream_t work = nullptr;  // private non-blocking stream (graph capture needs a non-legacy stream)
    // device counters (unsigned long long[CNT_N]) and scalars (double[SC_N])
    unsigned long long* d_counters = nullptr;
    double* d_scalars = nullptr;
    double* h_scalars = nullptr;  // pinned mirror
    int* d_flags = nullptr;       // device error flags (int[4]); [0]: a bounded wait timed out
    cudaEvent_t ev_a = nullptr, ev_b = nullptr, ev_c = nullptr, ev_d = nullptr;
    int64_t launches = 0;         // kernels launched through this context
    sf_engine* batch_engine = nullptr;  // the engine sf_solve_stokes_batch_mixed reuses across calls
    // sweep shapes the engines' autotuner measured best, by workload class (sf_mixed.cu)
    std::map<int, int> sweep_shapes;
};

namespace sf {

// Ensures `s` holds at least `bytes`; contents are not preserved.
int ensure(sf_ctx* ctx, Scratch& s, size_t bytes);
int set_device(sf_ctx* ctx);
// Whether device `dev` can read and write `peer`'s memory directly (NVLink / PCIe peer access), enabling it on
// first use; *ok is true for dev == peer.  Pairs without peer access copy through the runtime instead.
int peer_access(int dev, int peer, bool* ok);
// A w x h block of doubles (rows of w contiguous entries, leading dimensions ld_dst / ld_src) from src, which
// lives on src_device, to dst on ctx's device, queued on stream s of that device (current).  With peer access
// (or one device) a copy kernel on ctx's device reads src directly -- plain loads, no multicast; otherwise
// cudaMemcpy2DAsync does it.
int copy_block(sf_ctx* ctx, cudaStream_t s, double* dst, int64_t ld_dst, const double* src, int64_t ld_src,
               int64_t w, int64_t h, int src_device);
// frees the context's cached batch engine (sf_mixed.cu)
void mixed_engine_release(sf_ctx* ctx);

// true when no two of the n contexts (reached through get(i)) are the same: a rank's scratch is its own
template <typename Get>
bool distinct_contexts(int n, Get get) {
    for (int i = 0; i < n; ++i)
        for (int j = i + 1; j < n; ++j)
            if (get(i) == get(j)) return false;
    return true;
}
inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// launches `kern`; with `overlap`, under programmatic stream serialization: it may begin (launch, prologue)
// while the previous kernel on `s` drains, and must call griddep_wait() before it touches that kernel's
// results (sf_tma.cuh)
template <typename... Params, typename... Args>
cudaError_t launch_overlapped(bool overlap, void (*kern)(Params...), dim3 grid, dim3 block, size_t smem,
                              cudaStream_t s, Args&&... args) {
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = overlap ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }
inline int64_t round_up(int64_t a, int64_t b) { return ceil_div(a, b) * b; }

// exclusive scan of n int32 values (in may alias out); total -> *d_total (device)
int exclusive_scan_i32(sf_ctx* ctx, const int32_t* in, int32_t* out, int64_t n, int32_t* d_total,
                       cudaStream_t stream);
// the same with a caller-provided tile buffer of ceil(n / 8192) ints; allocates nothing
int exclusive_scan_i32_into(const int32_t* in, int32_t* out, int64_t n, int32_t* d_total, int32_t* tiles,
                            cudaStream_t stream);

// --------------------------------------------------------------------------
// device helpers
// --------------------------------------------------------------------------

// scripts/common.jl:22-33 topleftIndexRelDist.  ix, iy are 1-based like the
// reference; q is floor((x - x_grid_min)/dx) kept in double so that NaN and
// huge values can be classified without undefined conversions.
struct TopLeft {
    double qx, qy;     // floor((x - xmin)/dx) = ix - 1
    double dxij, dyij;
};

__device__ __forceinline__ TopLeft topleft(double xmin, double ymin, double x, double y, double dx,
                                           double dy) {
    TopLeft t;
    t.qx = floor((x - xmin) / dx);
    t.qy = floor((y - ymin) / dy);
    double x_ix = xmin + t.qx * dx;   // x_grid_min + (ix - 1) * dx
    double y_iy = ymin + t.qy * dy;
    t.dxij = (x - x_ix) / dx;
    t.dyij = (y - y_iy) / dy;
    return t;
}

// SplitMix64 finaliser; sf_uniform(seed, k) = top 53 bits of
// mix(mix(seed) ^ k*C) / 2^53.
__host__ __device__ __forceinline__ uint64_t splitmix64_mix(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__host__ __device__ __forceinline__ double uniform01(uint64_t seed, uint64_t counter) {
    uint64_t z = splitmix64_mix(splitmix64_mix(seed) ^ (counter * 0xD1B54A32D192ED03ull));
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

// Julia max(x, 0) and min(x, l) for Float64: -0.0 < 0.0, NaN propagates.
__host__ __device__ __forceinline__ double jl_max0(double x) {
    if (x != x) return x;
    return (x < 0.0 || (x == 0.0 && std::signbit(x))) ? 0.0 : x;
}
__host__ __device__ __forceinline__ double jl_min(double x, double l) {
    if (x != x) return x;
    return (l < x) ? l : x;
}

}  // namespace sf
