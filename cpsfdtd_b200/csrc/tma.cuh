// tma.cuh -- thin PTX wrappers for mbarriers and TMA bulk-tensor loads
// (sm_90+ PTX, used here on sm_100a), and the tensor maps of a grid.
#pragma once

#include <cuda.h>
#include <stdint.h>

namespace cps {

// Tensor maps of the six field arrays and the ID array of one grid, x fastest:
//   halo[c]: box 36 x (BY+1) x 1   own[c]: box 32 x BY x 1   id: box 32 x BY x 1
// c = 0..5 for Ex Ey Ez Hx Hy Hz.
//   gain: FP32 segment-dense gain words, dims {32 lanes, 15 words, segments,
//         ny+1 rows, nz+1 planes}, box 32 x 15 x 1 x BY x 1 (grids with gain)
struct TmaMaps {
    CUtensorMap halo[6];
    CUtensorMap own[6];
    CUtensorMap id;
    CUtensorMap gain;
};

// Tensor maps of the one-pass step sweep over one field buffer, x fastest:
//   e[c]: Ex Ey Ez, box 40 x (BY+2) x 1 (from x0-4, y0-1)
//   h[c]: Hx Hy Hz, box 36 x (BY+1) x 1 (from x0-4, y0-1)
//   id:   uint8 IDs, box 48 x (BY+1) x 1 (from x0-16, y0-1)
struct StepMaps {
    CUtensorMap e[3];
    CUtensorMap h[3];
    CUtensorMap id;
};

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t phase)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(phase)
        : "memory");
    return ok != 0;
}

// 3-D tiled load into this CTA's shared memory, completion counted on bar.
// The x coordinate times the element size must be a multiple of 16 bytes.
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y, int z)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
        : "memory");
}

// 5-D tiled load (the segment-dense gain words), completion counted on bar
__device__ __forceinline__ void tma_load_5d(void *dst, const CUtensorMap *map, uint64_t *bar, int c0, int c1, int c2,
                                            int c3, int c4)
{
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4, %5, %6, %7}], [%2];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4)
        : "memory");
}

}  // namespace cps
