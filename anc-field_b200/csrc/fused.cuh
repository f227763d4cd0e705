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

constexpr int FT_X = 64;                 // default tile width in x (cells, FP32 storage)
constexpr int FT_Y = 16;                 // default tile height in y
constexpr int F_CONSUMERS = 256;
constexpr int F_THREADS = F_CONSUMERS + 32;
constexpr unsigned long long kWaitLimitNs = 2000000000ull;   // 2 s

// Tile shapes of the streaming kernel (a plan parameter the autotuner
// varies): S = 0: 64 x 16, 1: 128 x 8, 2: 32 x 32 cells for FP32 storage;
// FP16 storage doubles the width (the same bytes per row).
constexpr int kTileShapes = 3;
__host__ __device__ constexpr int shape_w32(int S) { return S == 0 ? 64 : (S == 1 ? 128 : 32); }
__host__ __device__ constexpr int shape_h(int S) { return S == 0 ? 16 : (S == 1 ? 8 : 32); }

// Stage layout per storage type and shape. W: tile width in cells; H: rows;
// CPT: cells per consumer thread; TPR = W / CPT consumer threads per row
// (TPR x H = 256). The p^n box is the tile with a one-cell halo in y and a
// halo of XOFF cells in x (x times the element size stays a multiple of 16
// bytes, as TMA requires), followed by the p^{n-1} box of the tile. The
// 64 x 16 shape keeps 8 stages; the others, whose halo boxes are larger,
// keep 7 so that three blocks still fit an SM's shared memory.
template <typename T, int S = 0>
struct Tile {
    static constexpr int ES = (int)sizeof(T);
    static constexpr int CPT = ES == 4 ? 4 : 8;
    static constexpr int W = shape_w32(S) * (4 / ES);
    static constexpr int H = shape_h(S);
    static constexpr int TPR = W / CPT;
    static constexpr int XOFF = 16 / ES;
    static constexpr int HX = W + 2 * XOFF;
    static constexpr int PN_BYTES = HX * (H + 2) * ES;
    static constexpr int PN_PAD = (PN_BYTES + 127) / 128 * 128;
    static constexpr int PO_BYTES = W * H * ES;
    static constexpr int STAGE = (PN_PAD + PO_BYTES + 127) / 128 * 128;
    static constexpr int TX = PN_BYTES + PO_BYTES;  // bytes each stage receives
    static constexpr int STAGES = S == 0 ? 8 : 7;
    static constexpr size_t SMEM = (size_t)STAGES * STAGE + 2 * STAGES * 8 + STAGES * 4 + 128;
    static_assert(TPR * H == F_CONSUMERS, "256 consumer threads cover the tile");
};
static_assert(Tile<float, 0>::STAGE == 9344 && Tile<float, 0>::TX == 9280, "64 x 16 FP32 stage");

// Work decomposition of the streaming kernel.
struct FusedDev {
    int32_t tiles_x, tiles_y, dz, n_chunks;
    int* work;          // work-item counters, one per launch of a chunk
    const int* items;   // null: every item; else the n_items items to run (ascending)
    int32_t n_items;
    const uint32_t* owned;  // null, or 1 bit per cell ([z][y][owned_wpr] words): cells not to store
    int32_t owned_wpr;
    unsigned long long* tail;  // tail-warp work counters, one per step of a chunk
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
// A consumer's release of a stage: its shared-memory reads of the stage go
// through the generic proxy, the TMA load that refills the stage once the
// producer sees the release writes through the async proxy. The proxy fence
// orders this thread's reads before those writes; without it a refill could
// land before a read of the old plane completed (seen as one-unit differences
// between runs of the FP16 kernel, whose consumers release a plane early).
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
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
