// Tensor-memory-access (TMA) bulk copies into shared memory, completed on an mbarrier.
//
// Only the plain tiled load of this GPU's own memory is used: cp.async.bulk.tensor with no
// cluster multicast, issued by one thread, its bytes counted on a shared-memory mbarrier that
// the consuming threads wait on. Every wait is bounded: after kWaitLimit polls the waiter gives
// up and reports it, so a copy that never lands cannot hang the kernel.
//
// Tensor maps are encoded on the host through the driver's cuTensorMapEncodeTiled, reached with
// cudaGetDriverEntryPoint (the library links only the runtime). The map of a [planes][rows][cols]
// float2 array views it as float32 elements (2 per complex value), so a box of 4 complex columns
// is 8 floats = 32 bytes wide: the innermost coordinate (2·col) times 4 bytes is a multiple of
// 16 whenever col is a multiple of 4, as a tiled copy requires.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace zc {

constexpr uint32_t kWaitLimit = 1u << 20;  // mbarrier polls before a wait gives up (a copy takes microseconds)

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// make the initialised barrier visible to the async proxy (the TMA unit) and to the cluster of one
__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// order this thread's earlier shared-memory accesses before later async-proxy copies into it
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// true once the barrier's phase `parity` has completed; false after kWaitLimit polls
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    const uint32_t a = smem_addr(bar);
    for (uint32_t i = 0; i < kWaitLimit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// 3-D tiled load of box (x, y, z) of `map` into shared memory at dst, counted on bar
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
            smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
        : "memory");
}

// Host: a 3-D tiled tensor map over `planes` planes of `rows` rows of `cols` float2 values, rows
// `pitch` float2 apart and planes `pstride` float2 apart, with boxes of box_cols complex columns
// (a multiple of 2) × box_rows rows × 1 plane. Columns past `cols` read as zero. false when the
// driver refuses the map (e.g. misaligned base or strides).
bool encode_cplx_map(CUtensorMap* out, const void* base, int cols, int rows, int planes, size_t pitch, size_t pstride,
                     int box_cols, int box_rows);

}  // namespace zc
