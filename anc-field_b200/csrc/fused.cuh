// Streaming interior kernel for sm_100a (the HBM-bound part of a step).
//
// The grid is cut into TX x TY tiles in (x, y) and z-chunks of up to DZ
// planes; persistent blocks take work items (tile, chunk, batch member)
// from a counter and march through the chunk's planes (2.5-D z-marching).
// A producer thread streams, per plane, the p^n tile with a one-cell halo
// (x widened to 4 cells so every TMA box starts on a 16-byte boundary) and
// the p^{n-1} tile into a ring of STAGES shared-memory stages with
// cp.async.bulk.tensor (no multicast), signalling mbarriers. Eight consumer
// warps compute four consecutive x cells per thread from the staged planes
// and store float4 rows. Every mbarrier wait is bounded in time: on expiry
// the kernel sets bit 1 of the watchdog flag and returns instead of
// spinning.
#pragma once

#include <cuda.h>
#include <cstdint>

#include "device.cuh"

namespace afd {

constexpr int FT_X = 64;                 // tile width in x (cells)
constexpr int FT_Y = 16;                 // tile height in y
constexpr int FH_X = FT_X + 8;           // halo tile width (4-cell aligned halo each side)
constexpr int FH_Y = FT_Y + 2;
constexpr int F_STAGES = 8;
constexpr int F_PN_BYTES = FH_X * FH_Y * 4;                 // 5184
constexpr int F_PN_PAD = (F_PN_BYTES + 127) / 128 * 128;    // 5248
constexpr int F_PO_BYTES = FT_X * FT_Y * 4;                 // 4096
constexpr int F_STAGE_BYTES = F_PN_PAD + F_PO_BYTES;        // 9344
constexpr int F_TX_BYTES = F_PN_BYTES + F_PO_BYTES;         // bytes each stage receives
constexpr int F_CONSUMERS = 256;
constexpr int F_THREADS = F_CONSUMERS + 32;
constexpr size_t F_SMEM = (size_t)F_STAGES * F_STAGE_BYTES + 2 * F_STAGES * 8 + F_STAGES * 4 + 128;
constexpr unsigned long long kWaitLimitNs = 2000000000ull;   // 2 s

// Stage layout per storage type. FP16 levels: 128-cell tiles (a stage
// holds the same bytes as an FP32 one), the halo box starts 8 cells before
// the tile (x times 2 bytes stays a multiple of 16) and is 144 cells wide.
template <typename T>
struct Tile;
// W: tile width in cells; CPT: cells per consumer thread (16 threads per
// row, 16 rows).
template <>
struct Tile<float> {
    static constexpr int W = FT_X, CPT = 4;
    static constexpr int HX = FH_X, XOFF = 4, PN_PAD = F_PN_PAD, STAGE = F_STAGE_BYTES, TX = F_TX_BYTES;
    static constexpr size_t SMEM = F_SMEM;
};
template <>
struct Tile<__half> {
    static constexpr int W = 2 * FT_X, CPT = 8;
    static constexpr int HX = W + 16, XOFF = 8;
    static constexpr int PN_BYTES = HX * FH_Y * 2;                               // 5184
    static constexpr int PN_PAD = (PN_BYTES + 127) / 128 * 128;                  // 5248
    static constexpr int PO_BYTES = W * FT_Y * 2;                                // 4096
    static constexpr int STAGE = (PN_PAD + PO_BYTES + 127) / 128 * 128;          // 9344
    static constexpr int TX = PN_BYTES + PO_BYTES;                               // 9280
    static constexpr size_t SMEM = (size_t)F_STAGES * STAGE + 2 * F_STAGES * 8 + F_STAGES * 4 + 128;
};

// Work decomposition of the streaming kernel.
struct FusedDev {
    int32_t tiles_x, tiles_y, dz, n_chunks;
    int* work;          // work-item counters, one per launch of a chunk
    const int* items;   // null: every item; else the n_items items to run (ascending)
    int32_t n_items;
    const uint32_t* owned;  // null, or 1 bit per cell ([z][y][owned_wpr] words): cells not to store
    int32_t owned_wpr;
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Bounded wait: false after kWaitLimitNs without the phase completing.
// The clock is read once per 16 polls, so waiting warps issue few
// instructions beside the ones that compute.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    if (mbar_try(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    for (;;) {
#pragma unroll 1
        for (int i = 0; i < 16; ++i)
            if (mbar_try(bar, parity)) return true;
        if (global_ns() - t0 > kWaitLimitNs) return false;
    }
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
        : "memory");
}
// Barrier over the 256 consumer threads (named barrier 1).
__device__ __forceinline__ void consumer_sync() { asm volatile("bar.sync 1, 256;" ::: "memory"); }
// Same barrier, returning the AND of `ok` over the consumers.
__device__ __forceinline__ bool consumer_all(bool ok) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred pi, po;\n\t"
        "setp.ne.u32 pi, %1, 0;\n\t"
        "bar.red.and.pred po, 1, 256, pi;\n\t"
        "selp.u32 %0, 1, 0, po;\n}\n"
        : "=r"(r)
        : "r"((uint32_t)ok)
        : "memory");
    return r != 0;
}

struct FusedItem {
    int tx, ty, b, z0, z1;
};

__device__ __forceinline__ FusedItem fused_item(const FusedDev& f, int item, int nz) {
    FusedItem it;
    it.tx = item % f.tiles_x;
    int r = item / f.tiles_x;
    it.ty = r % f.tiles_y;
    r /= f.tiles_y;
    const int chunk = r % f.n_chunks;
    it.b = r / f.n_chunks;
    it.z0 = 1 + chunk * f.dz;
    it.z1 = min(it.z0 + f.dz, nz - 1);
    return it;
}

}  // namespace afd
