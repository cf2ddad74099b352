// Tensor-memory-accelerator (TMA) tile loads for the fine-grid transposes of the NUFFT, on
// sm_100a: 2-D tiled `cp.async.bulk.tensor` loads of this GPU's own memory into shared memory
// (no cluster multicast), completed on an mbarrier whose wait is bounded.
#pragma once
#include <cuda.h>  // CUtensorMap and its enums; the encoder is fetched from the driver at run time
#include <cuda_runtime.h>

#include <cstdint>

namespace pf {

// counts the tile loads that did not complete within their wait limit (read by tma_timeouts();
// the kernel then skips the tile and returns); one counter per translation unit including this
static __device__ int g_tma_timeouts = 0;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    // make the initialised barrier visible to the asynchronous (TMA) proxy
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}

// one 2-D tile of `map` at element coordinates (x, y) into dst (1024-byte aligned for the
// 128-byte swizzle); completion is counted on bar
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar,
                                            int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%2, %3}], [%4];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}" : "=r"(ok) : "r"(smem_addr(bar)), "r"(parity) : "memory");
    return ok != 0;
}

// Waits for phase `parity` of bar for at most `limit` tries (each try may suspend the thread for
// a short hardware-chosen time). On giving up it records the timeout, waits once more for the
// copy in flight (again bounded) and returns false.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int limit) {
    for (int i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    atomicAdd(&g_tma_timeouts, 1);
    for (int i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, parity)) break;
    return false;
}

// Byte offset of element (line, byte offset b within the line) in a tile of 128-byte lines
// loaded with CU_TENSOR_MAP_SWIZZLE_128B: the 16-byte chunk index is XORed with line mod 8.
__device__ __forceinline__ int swz128(int line, int b) {
    return line * 128 + ((((b >> 4) ^ (line & 7)) << 4) | (b & 15));
}

// host: a 2-D tensor map over a column-major array of `inner` x `outer` elements of esize bytes
// (row pitch inner * esize), tiles of box_inner x box_outer elements, 128-byte swizzle. Returns
// 0 on success; non-zero when the driver has no encoder or rejects the map (callers then use
// their plain-load kernels).
int make_tile_map(CUtensorMap* map, void* base, int esize, int64_t inner, int64_t outer,
                  int box_inner, int box_outer);

}  // namespace pf
