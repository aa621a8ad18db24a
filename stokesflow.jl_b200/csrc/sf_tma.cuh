// sf_tma.cuh -- thin wrappers over the sm_90+/sm_100 bulk-tensor copy (TMA)
// and shared-memory mbarrier PTX used by the persistent PT kernel, plus the
// host-side tensor-map encoder (cuTensorMapEncodeTiled fetched through the
// runtime's driver entry point, so the library needs no link to libcuda).
//
// Every wait is bounded: mbar_wait() gives up after a wall-clock budget
// (%globaltimer) and reports failure instead of spinning forever.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace sf {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Programmatic dependent launch.  A kernel launched with programmatic stream serialization may start while
// the previous kernel in the stream is still running; griddep_wait() returns once that kernel has completed
// and its memory operations are visible, so nothing it writes may be read (or overwritten) before it.
// griddep_launch_dependents() lets the next such kernel start its own launch and prologue.  Both are no-ops
// for a kernel launched without the attribute.
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void griddep_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t global_timer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Wait for phase `parity` of `bar` for at most budget_ns; false on timeout.
// The clock is read only every 256 polls so that waiting warps stay cheap.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint64_t budget_ns) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_timer_ns();
    for (uint32_t k = 1;; ++k) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((k & 255u) == 0u && global_timer_ns() - t0 > budget_ns) return false;
    }
}

// A tensor map that the host copied into global memory (between launches) is seen by this thread's
// bulk-tensor copies only after this fence; once per thread block and map, until the map changes again.
// System scope, because the host wrote the map (device scope measured no cheaper).
__device__ __forceinline__ void fence_tensormap_acquire(const CUtensorMap* map) {
    asm volatile("fence.proxy.tensormap::generic.acquire.sys [%0], 128;" ::"l"((uint64_t)map) : "memory");
}

// 2-D tiled bulk-tensor load global -> shared, completion counted on `bar`.
// No multicast: the tile lands in this CTA's shared memory only.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
        ::"r"(smem_u32(dst)), "l"((uint64_t)map), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}

// 3-D tiled bulk-tensor load (x, y, z) global -> shared, completion counted on `bar`; no multicast
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y, int z) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];"
        ::"r"(smem_u32(dst)), "l"((uint64_t)map), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
        : "memory");
}

// host: encode a 2-D FP64 tensor map over a (rows x ld) row-major buffer
// (inner dimension ld elements, row pitch ld*8 bytes), box = box_w x box_h.
int encode_tmap_f64(CUtensorMap* map, const double* base, int64_t ld, int64_t rows, int box_w, int box_h);
int encode_tmap_f32(CUtensorMap* map, const float* base, int64_t ld, int64_t rows, int box_w, int box_h);
// host: a 3-D FP32 tensor map over nfields such buffers, fstride elements apart (the field is the z
// coordinate), box = box_w x box_h x 1
int encode_tmap_f32_fields(CUtensorMap* map, const float* base, int64_t ld, int64_t rows, int64_t nfields,
                           int64_t fstride, int box_w, int box_h);

}  // namespace sf
