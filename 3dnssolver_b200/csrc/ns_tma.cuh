// ns_tma.cuh -- Tensor Memory Accelerator loads of halo'd W tiles (sm_100a,
// inline PTX): the 4D tiled load (no multicast) that completes on an
// mbarrier, and the transaction-count arrival that arms it.
#pragma once

#include <cuda.h>

#include <cstdint>

namespace nsb {

// polls of an mbarrier wait before a TMA kernel gives up and reports it
constexpr uint32_t kTilePolls = 1u << 24;

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// 4D tiled load of the box at (c0, c1, c2, c3) into dst; completion is
// signalled on the mbarrier at bar
__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5}], [%6];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar)
        : "memory");
}

}  // namespace nsb
