// Learned impulse-response surrogate: a Fourier-feature MLP trained and
// evaluated with hand-written tcgen05 BF16 GEMMs (FP32 accumulation in
// TMEM) on sm_100a. No counterpart in the reference; the FDTD engine of
// this library generates its training data and measures its error.
//
// Network: x (n_in values in [0, 1]) -> [sin(2 pi x B), cos(2 pi x B)]
// (B: n_in x n_freq, N(0, sigma^2)) -> (n_layers - 1) x [Linear + ReLU] ->
// Linear -> n_out samples. Weights kept in FP32 (Adam) with BF16 copies in
// both orientations for the GEMMs; activations and their gradients in BF16.
//
// GEMM: C[M][N] = A[M][K] * B[N][K]^T, both operands K-major BF16, K in
// steps of 64 through a ring of TMA stages. Warp 0 (one thread) streams
// tiles, warp 1 allocates TMEM and one of its threads issues tcgen05.mma
// (K = 16 per instruction) and commits stage releases, warps 2-5 read the
// accumulator with tcgen05.ld and run the epilogue. Two forms:
//   k_gemm_p  N a multiple of 256: persistent, one CTA per SM looping over
//             128 x 256 output tiles, 4-stage ring of 48 KB, two 256-column
//             TMEM accumulators so that the epilogue of one tile overlaps
//             the MMAs of the next;
//   k_gemm_pair  M and N multiples of 256: the same, by CTA pairs (clusters
//             of two): 256 x 256 tiles, each CTA loading 128 rows of A and
//             128 rows of B per k-step (32 KB, 6-stage ring) and the even CTA
//             issuing tcgen05.mma.cta_group::2 M 256 N 256 over both CTAs'
//             shared memory, so a CTA pulls a third less from L2 per FLOP;
//   k_gemm    otherwise: one 128 x 128 tile per CTA, 3-stage ring, two CTAs
//             per SM.
// Every wait is bounded; on expiry the kernel records it in the error flag,
// drains and frees TMEM.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "../../include/afd_surrogate.h"
#include "tc.cuh"

namespace afd {
namespace mlp {

using bf16 = __nv_bfloat16;

struct Err : std::runtime_error {
    int code;
    Err(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define MCK(call)                                                                                  \
    do {                                                                                           \
        cudaError_t e__ = (call);                                                                  \
        if (e__ != cudaSuccess) throw Err(AFD_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e__)); \
    } while (0)

constexpr int TM = 128, TN = 128, TK = 64, NST = 3;
constexpr int A_BYTES = TM * TK * 2, B_BYTES = TN * TK * 2, STAGE_BYTES = A_BYTES + B_BYTES;
constexpr int GEMM_THREADS = 192;
constexpr size_t GEMM_SMEM = 1024 + (size_t)NST * STAGE_BYTES + 256;
// persistent form
constexpr int PTN = 256, PNST = 4;
constexpr int PSTAGE = A_BYTES + 2 * B_BYTES;  // A 128 x 64, B 256 x 64 (two 128-row TMA boxes)
constexpr size_t PGEMM_SMEM = 1024 + (size_t)PNST * PSTAGE + 256;
// pair form
constexpr int QNST = 6;
constexpr int QSTAGE = A_BYTES + B_BYTES;  // 128 rows of A and 128 rows of B, 64 deep
constexpr size_t QGEMM_SMEM = 1024 + (size_t)QNST * QSTAGE + 256;

enum Epi : int {
    EPI_F32 = 0,   // c32[row][col] = acc (+ bias[col])
    EPI_RELU = 1,  // h = relu(acc + bias): c16[row][col] and c16t[col][row]
    EPI_MASK = 2,  // g = acc * (mask[row][col] > 0): c16[row][col] and c16t[col][row]
};

struct GemmOut {
    int M, N, K;
    const float* bias;
    float* c32;
    int ldc;
    bf16* c16;
    bf16* c16t;
    int ld16, ld16t;
    const bf16* mask;
    int ldmask;
    int* flag;  // bit 0: a wait expired
};

// 32 accumulator columns col0 .. col0+31 of output row `row` through the
// epilogue EPI.
template <int EPI>
__device__ __forceinline__ void epilogue32(const GemmOut& g, float v[32], int row, int col0) {
    if (g.bias) {
#pragma unroll
        for (int j = 0; j < 32; ++j) v[j] += __ldg(g.bias + col0 + j);
    }
    if constexpr (EPI == EPI_F32) {
        float4* dst = reinterpret_cast<float4*>(g.c32 + (size_t)row * g.ldc + col0);
#pragma unroll
        for (int j = 0; j < 8; ++j) dst[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
    } else {
        if constexpr (EPI == EPI_RELU) {
#pragma unroll
            for (int j = 0; j < 32; ++j) v[j] = fmaxf(v[j], 0.0f);
        } else {
            const uint4* mk = reinterpret_cast<const uint4*>(g.mask + (size_t)row * g.ldmask + col0);
#pragma unroll
            for (int j4 = 0; j4 < 4; ++j4) {
                const uint4 w = __ldg(mk + j4);
                const uint32_t ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
                for (int h = 0; h < 4; ++h) {
                    const __nv_bfloat162 p = *reinterpret_cast<const __nv_bfloat162*>(&ws[h]);
                    if (!(__low2float(p) > 0.0f)) v[8 * j4 + 2 * h] = 0.0f;
                    if (!(__high2float(p) > 0.0f)) v[8 * j4 + 2 * h + 1] = 0.0f;
                }
            }
        }
        uint32_t packed[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const __nv_bfloat162 p = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
            packed[j] = *reinterpret_cast<const uint32_t*>(&p);
        }
        uint4* dst = reinterpret_cast<uint4*>(g.c16 + (size_t)row * g.ld16 + col0);
#pragma unroll
        for (int j = 0; j < 4; ++j)
            dst[j] = make_uint4(packed[4 * j], packed[4 * j + 1], packed[4 * j + 2], packed[4 * j + 3]);
        if (g.c16t) {
#pragma unroll
            for (int j = 0; j < 32; ++j) g.c16t[(size_t)(col0 + j) * g.ld16t + row] = __float2bfloat16_rn(v[j]);
        }
    }
}

// Two CTAs per SM (99 KB of shared memory and 128 TMEM columns each): one
// CTA's epilogue and set-up overlap the other's MMAs.
template <int EPI>
__global__ void __launch_bounds__(GEMM_THREADS, 2)
    k_gemm(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, const GemmOut g) {
    extern __shared__ unsigned char raw[];
    unsigned char* sm = (unsigned char*)(((uintptr_t)raw + 1023) & ~(uintptr_t)1023);
    uint64_t* full = reinterpret_cast<uint64_t*>(sm + NST * STAGE_BYTES);
    uint64_t* empty = full + NST;
    uint64_t* done = empty + NST;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(done + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.y * TM, n0 = blockIdx.x * TN;
    const int KT = g.K / TK;
    if (threadIdx.x == 0) {
        for (int s = 0; s < NST; ++s) {
            tc::bar_init(&full[s], 1);
            tc::bar_init(&empty[s], 1);
        }
        tc::bar_init(done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) tc::tmem_alloc(tslot, TN);
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = *tslot;

    if (warp == 0) {
        if (lane == 0) {
            int issued = 0;
            for (int kt = 0; kt < KT; ++kt) {
                const int s = kt % NST;
                if (kt >= NST && !tc::bar_wait(&empty[s], ((kt / NST) - 1) & 1)) {
                    atomicOr(g.flag, 1);
                    break;
                }
                unsigned char* st = sm + s * STAGE_BYTES;
                tc::bar_expect_tx(&full[s], STAGE_BYTES);
                tc::tma_2d(st, &ta, kt * TK, m0, &full[s]);
                tc::tma_2d(st + A_BYTES, &tb, kt * TK, n0, &full[s]);
                ++issued;
            }
            // the copies still in flight complete before the block leaves
            for (int s = 0; s < NST && s < issued; ++s) {
                const int last = issued - 1 - ((issued - 1 - s) % NST);
                tc::bar_wait(&full[s], (last / NST) & 1);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t idesc = tc::bf16_f32_idesc(TM, TN);
            for (int kt = 0; kt < KT; ++kt) {
                const int s = kt % NST;
                if (!tc::bar_wait(&full[s], (kt / NST) & 1)) {
                    atomicOr(g.flag, 1);
                    break;
                }
                tc::fence_after();
                const uint32_t a0 = tc::smem_u32(sm + s * STAGE_BYTES), b0 = a0 + A_BYTES;
#pragma unroll
                for (int ks = 0; ks < TK / 16; ++ks)  // 16 BF16 = 32 bytes along K inside the swizzled row
                    tc::umma_bf16(tmem, tc::sw128_kmajor_desc(a0 + ks * 32), tc::sw128_kmajor_desc(b0 + ks * 32),
                                  idesc, (kt | ks) != 0);
                tc::umma_commit(&empty[s]);  // stage free once these MMAs have read it
            }
            tc::umma_commit(done);  // accumulator complete (or the issued part of it)
        }
    } else {
        // epilogue: warp w reads TMEM lanes 32 (w % 4) .. +31 = tile rows
        const int q = warp & 3;
        const int row = m0 + 32 * q + lane;
        const bool ok = __all_sync(0xffffffffu, tc::bar_wait(done, 0));  // warp-uniform for tcgen05.ld
        if (!ok && lane == 0) atomicOr(g.flag, 1);
        tc::fence_after();
        if (ok) {
#pragma unroll 1
            for (int c = 0; c < TN / 32; ++c) {
                float v[32];
                tc::tmem_ld32(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(32 * c), v);
                epilogue32<EPI>(g, v, row, n0 + 32 * c);
            }
        }
    }
    tc::fence_before();
    __syncthreads();
    if (warp == 1) {
        __syncwarp();
        tc::fence_after();
        tc::tmem_dealloc(tmem, TN);
    }
}

// Output tile t of the persistent form: groups of 16 row panels, columns
// outer inside a group, so that the ~148 tiles in flight share their A and
// B panels in L2.
constexpr int RASTER_M = 16;
__device__ __forceinline__ void tile_of(int t, int tiles_m, int tiles_n, int tile_h, int& m0, int& n0) {
    const int per_group = RASTER_M * tiles_n;
    const int first = (t / per_group) * RASTER_M;
    const int gm = min(tiles_m - first, RASTER_M);
    const int w = t % per_group;
    m0 = (first + w % gm) * tile_h;
    n0 = (w / gm) * PTN;
}

// Persistent form, one CTA per SM (194 KB of shared memory, all 512 TMEM
// columns), tiles t = blockIdx.x + i gridDim.x placed by tile_of. Barrier
// phases count uses: stage s is used for the u-th k-step of the CTA with
// s = u mod 4, accumulator ab for the it-th tile with ab = it & 1.
template <int EPI>
__global__ void __launch_bounds__(GEMM_THREADS, 1)
    k_gemm_p(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, const GemmOut g) {
    extern __shared__ unsigned char raw[];
    unsigned char* sm = (unsigned char*)(((uintptr_t)raw + 1023) & ~(uintptr_t)1023);
    uint64_t* full = reinterpret_cast<uint64_t*>(sm + PNST * PSTAGE);
    uint64_t* empty = full + PNST;
    uint64_t* acc_full = empty + PNST;   // [2] MMAs of a tile done
    uint64_t* acc_empty = acc_full + 2;  // [2] its four epilogue warps done reading
    uint64_t* drain = acc_empty + 2;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(drain + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tiles_m = g.M / TM, tiles_n = g.N / PTN, tiles = tiles_m * tiles_n;
    const int KT = g.K / TK;
    if (threadIdx.x == 0) {
        for (int s = 0; s < PNST; ++s) {
            tc::bar_init(&full[s], 1);
            tc::bar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            tc::bar_init(&acc_full[b], 1);
            tc::bar_init(&acc_empty[b], 4);
        }
        tc::bar_init(drain, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) tc::tmem_alloc(tslot, 2 * PTN);
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = *tslot;

    if (warp == 0) {
        if (lane == 0) {
            uint32_t u = 0;
            bool ok = true;
            for (int t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
                int m0, n0;
                tile_of(t, tiles_m, tiles_n, TM, m0, n0);
                for (int kt = 0; kt < KT; ++kt, ++u) {
                    const uint32_t s = u % PNST;
                    if (u >= (uint32_t)PNST && !tc::bar_wait(&empty[s], ((u / PNST) - 1) & 1)) {
                        atomicOr(g.flag, 1);
                        ok = false;
                        break;
                    }
                    unsigned char* st = sm + s * PSTAGE;
                    tc::bar_expect_tx(&full[s], PSTAGE);
                    tc::tma_2d(st, &ta, kt * TK, m0, &full[s]);
                    tc::tma_2d(st + A_BYTES, &tb, kt * TK, n0, &full[s]);
                    tc::tma_2d(st + A_BYTES + B_BYTES, &tb, kt * TK, n0 + 128, &full[s]);
                }
            }
            // the copies still in flight complete before the block leaves
            for (uint32_t s = 0; s < (uint32_t)PNST && s < u; ++s) {
                const uint32_t last = u - 1 - ((u - 1 - s) % PNST);
                tc::bar_wait(&full[s], (last / PNST) & 1);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t idesc = tc::bf16_f32_idesc(TM, PTN);
            uint32_t u = 0;
            int it = 0;
            bool ok = true;
            for (int t = blockIdx.x; t < tiles && ok; t += gridDim.x, ++it) {
                const int ab = it & 1;
                if (it >= 2 && !tc::bar_wait(&acc_empty[ab], ((it >> 1) - 1) & 1)) {
                    atomicOr(g.flag, 1);
                    break;
                }
                tc::fence_after();
                const uint32_t d = tmem + (uint32_t)(ab * PTN);
                for (int kt = 0; kt < KT; ++kt, ++u) {
                    const uint32_t s = u % PNST;
                    if (!tc::bar_wait(&full[s], (u / PNST) & 1)) {
                        atomicOr(g.flag, 1);
                        ok = false;
                        break;
                    }
                    tc::fence_after();
                    const uint32_t a0 = tc::smem_u32(sm + s * PSTAGE), b0 = a0 + A_BYTES;
#pragma unroll
                    for (int ks = 0; ks < TK / 16; ++ks)
                        tc::umma_bf16(d, tc::sw128_kmajor_desc(a0 + ks * 32), tc::sw128_kmajor_desc(b0 + ks * 32),
                                      idesc, (kt | ks) != 0);
                    tc::umma_commit(&empty[s]);
                }
                if (ok) tc::umma_commit(&acc_full[ab]);
            }
            // every MMA issued has completed once this arrives
            tc::umma_commit(drain);
            tc::bar_wait(drain, 0);
        }
    } else {
        // epilogue: warp w reads TMEM lanes 32 (w % 4) .. +31 = tile rows
        const int q = warp & 3;
        int it = 0;
        for (int t = blockIdx.x; t < tiles; t += gridDim.x, ++it) {
            const int ab = it & 1;
            const bool ok = __all_sync(0xffffffffu, tc::bar_wait(&acc_full[ab], (it >> 1) & 1));
            if (!ok) {
                if (lane == 0) atomicOr(g.flag, 1);
                break;
            }
            tc::fence_after();
            int m0, n0;
            tile_of(t, tiles_m, tiles_n, TM, m0, n0);
            const int row = m0 + 32 * q + lane;
#pragma unroll 1
            for (int c = 0; c < PTN / 32; ++c) {
                float v[32];
                tc::tmem_ld32(tmem + (uint32_t)(ab * PTN) + ((uint32_t)(32 * q) << 16) + (uint32_t)(32 * c), v);
                epilogue32<EPI>(g, v, row, n0 + 32 * c);
            }
            tc::fence_before();
            __syncwarp();
            if (lane == 0) tc::bar_arrive(&acc_empty[ab]);
        }
    }
    tc::fence_before();
    __syncthreads();
    if (warp == 1) {
        __syncwarp();
        tc::fence_after();
        tc::tmem_dealloc(tmem, 2 * PTN);
    }
}

// Pair form: clusters of two CTAs, one per SM, over 256 x 256 tiles placed
// by tile_of (pair p takes tiles p, p + pairs, ...). Rank r loads rows
// m0 + 128 r of A and n0 + 128 r of B into its own ring; both loads count
// on rank 0's full barrier (64 KB per stage). Rank 0's MMA thread issues the
// pair's MMAs and commits every stage release, accumulator completion and
// the final drain to the barrier of the same offset in both CTAs. Each CTA's
// epilogue drains its own TMEM rows and arrives on rank 0's acc_empty
// (eight warps per use). Every path reaches both cluster barriers once.
template <int EPI>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(GEMM_THREADS, 1)
    k_gemm_pair(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, const GemmOut g) {
    extern __shared__ unsigned char raw[];
    unsigned char* sm = (unsigned char*)(((uintptr_t)raw + 1023) & ~(uintptr_t)1023);
    uint64_t* full = reinterpret_cast<uint64_t*>(sm + QNST * QSTAGE);
    uint64_t* empty = full + QNST;
    uint64_t* acc_full = empty + QNST;
    uint64_t* acc_empty = acc_full + 2;
    uint64_t* drain = acc_empty + 2;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(drain + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rank = tc::cluster_rank();
    const int pair = (int)(blockIdx.x >> 1), pairs = (int)(gridDim.x >> 1);
    const int tiles_m = g.M / (2 * TM), tiles_n = g.N / PTN, tiles = tiles_m * tiles_n;
    const int KT = g.K / TK;
    if (threadIdx.x == 0) {
        for (int s = 0; s < QNST; ++s) {
            tc::bar_init(&full[s], 1);
            tc::bar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            tc::bar_init(&acc_full[b], 1);
            tc::bar_init(&acc_empty[b], 8);
        }
        tc::bar_init(drain, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) tc::tmem_alloc_pair(tslot, 2 * PTN);
    tc::fence_before();
    __syncthreads();
    tc::cluster_sync();  // both CTAs' barriers initialised and TMEM allocated
    tc::fence_after();
    const uint32_t tmem = *tslot;

    if (warp == 0) {
        if (lane == 0) {
            uint32_t u = 0;
            bool ok = true;
            for (int t = pair; t < tiles && ok; t += pairs) {
                int m0, n0;
                tile_of(t, tiles_m, tiles_n, 2 * TM, m0, n0);
                const int am = m0 + (int)rank * TM, bn = n0 + (int)rank * TN;
                for (int kt = 0; kt < KT; ++kt, ++u) {
                    const uint32_t s = u % QNST;
                    if (u >= (uint32_t)QNST && !tc::bar_wait(&empty[s], ((u / QNST) - 1) & 1)) {
                        atomicOr(g.flag, 1);
                        ok = false;
                        break;
                    }
                    if (rank == 0) tc::bar_expect_tx(&full[s], 2 * QSTAGE);
                    const uint32_t fb = tc::mapa(tc::smem_u32(&full[s]), 0);
                    unsigned char* st = sm + s * QSTAGE;
                    tc::tma_2d_pair(st, &ta, kt * TK, am, fb);
                    tc::tma_2d_pair(st + A_BYTES, &tb, kt * TK, bn, fb);
                }
            }
            // rank 0 sees the pair's copies complete; rank 1's land on the
            // same barriers
            if (rank == 0)
                for (uint32_t s = 0; s < (uint32_t)QNST && s < u; ++s) {
                    const uint32_t last = u - 1 - ((u - 1 - s) % QNST);
                    tc::bar_wait(&full[s], (last / QNST) & 1);
                }
        }
    } else if (warp == 1) {
        if (lane == 0 && rank == 0) {
            const uint32_t idesc = tc::bf16_f32_idesc(2 * TM, PTN);
            uint32_t u = 0;
            int it = 0;
            bool ok = true;
            for (int t = pair; t < tiles && ok; t += pairs, ++it) {
                const int ab = it & 1;
                if (it >= 2 && !tc::bar_wait(&acc_empty[ab], ((it >> 1) - 1) & 1)) {
                    atomicOr(g.flag, 1);
                    break;
                }
                tc::fence_after();
                const uint32_t d = tmem + (uint32_t)(ab * PTN);
                for (int kt = 0; kt < KT; ++kt, ++u) {
                    const uint32_t s = u % QNST;
                    if (!tc::bar_wait(&full[s], (u / QNST) & 1)) {
                        atomicOr(g.flag, 1);
                        ok = false;
                        break;
                    }
                    tc::fence_after();
                    const uint32_t a0 = tc::smem_u32(sm + s * QSTAGE), b0 = a0 + A_BYTES;
#pragma unroll
                    for (int ks = 0; ks < TK / 16; ++ks)
                        tc::umma_bf16_pair(d, tc::sw128_kmajor_desc(a0 + ks * 32),
                                           tc::sw128_kmajor_desc(b0 + ks * 32), idesc, (kt | ks) != 0);
                    tc::umma_commit_pair(&empty[s], 3);
                }
                if (ok) tc::umma_commit_pair(&acc_full[ab], 3);
            }
            tc::umma_commit_pair(drain, 3);
        }
    } else {
        const int q = warp & 3;
        int it = 0;
        for (int t = pair; t < tiles; t += pairs, ++it) {
            const int ab = it & 1;
            const bool ok = __all_sync(0xffffffffu, tc::bar_wait(&acc_full[ab], (it >> 1) & 1));
            if (!ok) {
                if (lane == 0) atomicOr(g.flag, 1);
                break;
            }
            tc::fence_after();
            int m0, n0;
            tile_of(t, tiles_m, tiles_n, 2 * TM, m0, n0);
            const int row = m0 + (int)rank * TM + 32 * q + lane;
#pragma unroll 1
            for (int c = 0; c < PTN / 32; ++c) {
                float v[32];
                tc::tmem_ld32(tmem + (uint32_t)(ab * PTN) + ((uint32_t)(32 * q) << 16) + (uint32_t)(32 * c), v);
                epilogue32<EPI>(g, v, row, n0 + 32 * c);
            }
            tc::fence_before();
            __syncwarp();
            if (lane == 0) tc::bar_arrive_cluster(tc::mapa(tc::smem_u32(&acc_empty[ab]), 0));
        }
    }
    // every MMA of the pair has completed (rank 0 commits the drain to both)
    if (warp == 1 && lane == 0) tc::bar_wait(drain, 0);
    tc::fence_before();
    __syncthreads();
    tc::cluster_sync();  // neither CTA leaves while the other may still use its memory
    if (warp == 1) {
        __syncwarp();
        tc::fence_after();
        tc::tmem_dealloc_pair(tmem, 2 * PTN);
    }
}

// ---- small kernels ---------------------------------------------------------
// Fourier features: f[r][j] = sin(2 pi <x_r, B_j>) (j < n_freq) and the
// cosine at j + n_freq; rows r >= n are zero.
__global__ void k_fourier(const float* x, int n, int n_in, const float* Bf, int n_freq, int rows, bf16* f,
                          bf16* ft) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (r >= rows) return;
    float s = 0.0f, c = 0.0f;
    if (r < n) {
        float a = 0.0f;
        for (int i = 0; i < n_in; ++i) a += x[(size_t)r * n_in + i] * Bf[(size_t)i * n_freq + j];
        const float ph = 6.283185307179586f * a;
        s = sinf(ph);
        c = cosf(ph);
    }
    const int F = 2 * n_freq;
    f[(size_t)r * F + j] = __float2bfloat16_rn(s);
    f[(size_t)r * F + j + n_freq] = __float2bfloat16_rn(c);
    ft[(size_t)j * rows + r] = __float2bfloat16_rn(s);
    ft[(size_t)(j + n_freq) * rows + r] = __float2bfloat16_rn(c);
}

// Loss gradient of the mean squared error over n valid rows:
// d = 2 (pred - y) / (n * n_out); rows >= n get zero. Loss partial sums per
// warp (FP32; the loss value is for reporting).
__global__ void k_mse_grad(const float* pred, const float* y, int n, int n_out, int rows, float scale, bf16* d,
                           bf16* dt, float* loss_acc) {
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = blockIdx.y;
    if (col >= n_out) return;
    float e = 0.0f;
    if (r < n) e = pred[(size_t)r * n_out + col] - y[(size_t)r * n_out + col];
    const bf16 v = __float2bfloat16_rn(scale * e);
    d[(size_t)r * n_out + col] = v;
    dt[(size_t)col * rows + r] = v;
    float sq = e * e;
    for (int o = 16; o > 0; o >>= 1) sq += __shfl_down_sync(0xffffffffu, sq, o);
    if ((threadIdx.x & 31) == 0 && sq != 0.0f) atomicAdd(loss_acc, sq);
}

// Bias gradient: db[o] = sum_r d[r][o], from the transposed copy (rows of
// dt contiguous), summed in order by one warp per output.
__global__ void k_bias_grad(const bf16* dt, int outs, int rows, float* db) {
    const int o = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    const int lane = threadIdx.x & 31;
    if (o >= outs) return;
    float s = 0.0f;
    for (int r = lane; r < rows; r += 32) s += __bfloat162float(dt[(size_t)o * rows + r]);
    for (int k = 16; k > 0; k >>= 1) s += __shfl_down_sync(0xffffffffu, s, k);
    if (lane == 0) db[o] = s;
}

// Adam on FP32 master weights; refreshes the BF16 copies w16 ([out][in])
// and w16t ([in][out]) of a weight matrix (w16 null for a bias vector).
__global__ void k_adam(float* w, const float* gw, float* m, float* v, int64_t n, int in, float lr, float b1,
                       float b2, float eps, float c1, float c2, bf16* w16, bf16* w16t, int outs) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float gg = gw[i];
        const float mm = b1 * m[i] + (1.0f - b1) * gg;
        const float vv = b2 * v[i] + (1.0f - b2) * gg * gg;
        m[i] = mm;
        v[i] = vv;
        const float wn = w[i] - lr * (mm / c1) / (sqrtf(vv / c2) + eps);
        w[i] = wn;
        if (w16) {
            const bf16 b = __float2bfloat16_rn(wn);
            w16[i] = b;
            const int o = (int)(i / in), c = (int)(i % in);
            w16t[(size_t)c * outs + o] = b;
        }
    }
}

__global__ void k_f32_to_bf16_both(const float* w, int outs, int in, bf16* w16, bf16* w16t) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)outs * in) return;
    const bf16 b = __float2bfloat16_rn(w[i]);
    w16[i] = b;
    w16t[(size_t)(i % in) * outs + i / in] = b;
}

// ---- host ------------------------------------------------------------------
template <typename T>
struct Dev {
    T* p = nullptr;
    size_t n = 0;
    Dev() = default;
    Dev(const Dev&) = delete;
    Dev& operator=(const Dev&) = delete;
    ~Dev() {
        if (p) cudaFree(p);
    }
    void alloc(size_t count) {
        if (p) cudaFree(p);
        p = nullptr;
        n = count;
        if (count) {
            MCK(cudaMalloc(&p, count * sizeof(T)));
            // the zeroing runs on the legacy stream, which the surrogate's
            // non-blocking stream does not wait for: finished before return
            MCK(cudaMemset(p, 0, count * sizeof(T)));
            MCK(cudaStreamSynchronize(cudaStreamLegacy));
        }
    }
};

typedef CUresult (*EncodeFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                             const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                             CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeFn encoder() {
    static EncodeFn fn = nullptr;
    if (!fn) {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        MCK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q));
        if (!f || q != cudaDriverEntryPointSuccess) throw Err(AFD_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
        fn = (EncodeFn)f;
    }
    return fn;
}

// K-major BF16 operand [rows][K] (row stride K): 64 x 128 boxes, 128-byte swizzle.
static CUtensorMap operand_map(const bf16* base, int rows, int K) {
    if (rows % 128 || K % 64 || ((uintptr_t)base & 15)) throw Err(AFD_ERR_ARG, "GEMM operand not tile-aligned");
    CUtensorMap m;
    const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)K * 2};
    const cuuint32_t box[2] = {TK, 128}, estr[2] = {1, 1};
    CUresult r = encoder()(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, (void*)base, dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw Err(AFD_ERR_CUDA, "tensor map encoding failed");
    return m;
}

struct Gemm {
    CUtensorMap ta, tb;
    GemmOut o;
    int epi;
};

// Shared-memory limits of the GEMM kernels and the SM count, per device
// (function attributes belong to the current device).
struct DeviceGemm {
    bool ready = false;
    int sms = 0;
};

static std::mutex g_gemm_mu;  // guards the per-device tables below

static int set_smem_attr() {
    static DeviceGemm devs[64];
    std::lock_guard<std::mutex> lock(g_gemm_mu);
    int dev = 0;
    MCK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) throw Err(AFD_ERR_ARG, "device ordinal out of range");
    DeviceGemm& d = devs[dev];
    if (d.ready) return d.sms;
    const int s1 = (int)GEMM_SMEM, s2 = (int)PGEMM_SMEM, s3 = (int)QGEMM_SMEM;
    MCK(cudaFuncSetAttribute((const void*)k_gemm<EPI_F32>, cudaFuncAttributeMaxDynamicSharedMemorySize, s1));
    MCK(cudaFuncSetAttribute((const void*)k_gemm<EPI_RELU>, cudaFuncAttributeMaxDynamicSharedMemorySize, s1));
    MCK(cudaFuncSetAttribute((const void*)k_gemm<EPI_MASK>, cudaFuncAttributeMaxDynamicSharedMemorySize, s1));
    MCK(cudaFuncSetAttribute((const void*)k_gemm_p<EPI_F32>, cudaFuncAttributeMaxDynamicSharedMemorySize, s2));
    MCK(cudaFuncSetAttribute((const void*)k_gemm_p<EPI_RELU>, cudaFuncAttributeMaxDynamicSharedMemorySize, s2));
    MCK(cudaFuncSetAttribute((const void*)k_gemm_p<EPI_MASK>, cudaFuncAttributeMaxDynamicSharedMemorySize, s2));
    MCK(cudaFuncSetAttribute((const void*)k_gemm_pair<EPI_F32>, cudaFuncAttributeMaxDynamicSharedMemorySize, s3));
    MCK(cudaFuncSetAttribute((const void*)k_gemm_pair<EPI_RELU>, cudaFuncAttributeMaxDynamicSharedMemorySize, s3));
    MCK(cudaFuncSetAttribute((const void*)k_gemm_pair<EPI_MASK>, cudaFuncAttributeMaxDynamicSharedMemorySize, s3));
    MCK(cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev));
    d.ready = true;
    return d.sms;
}

static void launch(const Gemm& G, cudaStream_t st) {
    const int sms = set_smem_attr();
    if (G.o.M % (2 * TM) == 0 && G.o.N % PTN == 0 && sms >= 2) {
        const int tiles = (G.o.M / (2 * TM)) * (G.o.N / PTN);
        const unsigned grid = 2u * (unsigned)std::max(1, std::min(tiles, sms / 2));
        switch (G.epi) {
            case EPI_F32: k_gemm_pair<EPI_F32><<<grid, GEMM_THREADS, QGEMM_SMEM, st>>>(G.ta, G.tb, G.o); break;
            case EPI_RELU: k_gemm_pair<EPI_RELU><<<grid, GEMM_THREADS, QGEMM_SMEM, st>>>(G.ta, G.tb, G.o); break;
            default: k_gemm_pair<EPI_MASK><<<grid, GEMM_THREADS, QGEMM_SMEM, st>>>(G.ta, G.tb, G.o); break;
        }
    } else if (G.o.N % PTN == 0) {
        const int tiles = (G.o.M / TM) * (G.o.N / PTN);
        const unsigned grid = (unsigned)std::max(1, std::min(tiles, sms));
        switch (G.epi) {
            case EPI_F32: k_gemm_p<EPI_F32><<<grid, GEMM_THREADS, PGEMM_SMEM, st>>>(G.ta, G.tb, G.o); break;
            case EPI_RELU: k_gemm_p<EPI_RELU><<<grid, GEMM_THREADS, PGEMM_SMEM, st>>>(G.ta, G.tb, G.o); break;
            default: k_gemm_p<EPI_MASK><<<grid, GEMM_THREADS, PGEMM_SMEM, st>>>(G.ta, G.tb, G.o); break;
        }
    } else {
        const dim3 grid((unsigned)(G.o.N / TN), (unsigned)(G.o.M / TM));
        switch (G.epi) {
            case EPI_F32: k_gemm<EPI_F32><<<grid, GEMM_THREADS, GEMM_SMEM, st>>>(G.ta, G.tb, G.o); break;
            case EPI_RELU: k_gemm<EPI_RELU><<<grid, GEMM_THREADS, GEMM_SMEM, st>>>(G.ta, G.tb, G.o); break;
            default: k_gemm<EPI_MASK><<<grid, GEMM_THREADS, GEMM_SMEM, st>>>(G.ta, G.tb, G.o); break;
        }
    }
    MCK(cudaGetLastError());
}

static Gemm make_gemm(int epi, const bf16* A, const bf16* B, int M, int N, int K, int* flag) {
    if (M % TM || N % TN || K % TK || K <= 0) throw Err(AFD_ERR_ARG, "GEMM sizes must be multiples of 128 x 128 x 64");
    Gemm G;
    G.ta = operand_map(A, M, K);
    G.tb = operand_map(B, N, K);
    std::memset(&G.o, 0, sizeof(G.o));
    G.o.M = M;
    G.o.N = N;
    G.o.K = K;
    G.o.flag = flag;
    G.epi = epi;
    return G;
}

struct Layer {
    int in = 0, out = 0;
    Dev<float> w, b, gw, gb, mw, vw, mb, vb;
    Dev<bf16> w16, w16t;
};

}  // namespace mlp
}  // namespace afd

using namespace afd::mlp;

struct afd_mlp {
    afd_mlp_params prm{};
    std::string err;
    int device = 0;
    cudaStream_t own = nullptr, stream = nullptr;
    int rows = 0, F = 0;
    std::vector<Layer*> L;
    Dev<float> fourier;             // [n_in][n_freq]
    Dev<float> xin, yin;            // staging copies of inputs / targets
    Dev<bf16> feat, featT;          // [rows][F], [F][rows]
    std::vector<Dev<bf16>*> H, HT;  // hidden activations per hidden layer: [rows][hidden], [hidden][rows]
    std::vector<Dev<bf16>*> G, GT;  // gradients w.r.t. each layer's output (pre-activation)
    Dev<float> pred;                // [rows][n_out]
    Dev<float> loss;                // 1
    Dev<int> flag;
    int64_t step = 0;
    std::vector<Gemm> fwd, bwd_w, bwd_x;

    ~afd_mlp() {
        if (stream) cudaStreamSynchronize(stream);
        for (auto* l : L) delete l;
        for (auto* p : H) delete p;
        for (auto* p : HT) delete p;
        for (auto* p : G) delete p;
        for (auto* p : GT) delete p;
        if (own) cudaStreamDestroy(own);
    }

    const bf16* layer_input(int l) const { return l == 0 ? feat.p : H[l - 1]->p; }
    const bf16* layer_input_t(int l) const { return l == 0 ? featT.p : HT[l - 1]->p; }

    void build() {
        const afd_mlp_params& p = prm;
        if (p.n_in < 1 || p.n_freq < 32 || (2 * p.n_freq) % 128 || p.hidden % 128 || p.n_out % 128 ||
            p.n_layers < 2 || p.n_layers > 16 || p.batch < 128 || p.batch % 128)
            throw Err(AFD_ERR_ARG, "surrogate sizes: 2*n_freq, hidden, n_out and batch must be multiples of 128");
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) throw Err(AFD_ERR_CUDA, "no CUDA device available");
        device = p.device;
        MCK(cudaSetDevice(device));
        MCK(cudaStreamCreateWithFlags(&own, cudaStreamNonBlocking));
        stream = own;
        set_smem_attr();
        rows = p.batch;
        F = 2 * p.n_freq;
        std::mt19937_64 rng(p.seed);
        std::normal_distribution<double> nd(0.0, 1.0);
        std::vector<float> fb((size_t)p.n_in * p.n_freq);
        for (auto& v : fb) v = (float)(nd(rng) * p.fourier_sigma);
        fourier.alloc(fb.size());
        MCK(cudaMemcpyAsync(fourier.p, fb.data(), fb.size() * 4, cudaMemcpyHostToDevice, stream));
        MCK(cudaStreamSynchronize(stream));
        for (int l = 0; l < p.n_layers; ++l) {
            Layer* ly = new Layer;
            L.push_back(ly);
            ly->in = l == 0 ? F : p.hidden;
            ly->out = l == p.n_layers - 1 ? p.n_out : p.hidden;
            const size_t nw = (size_t)ly->in * ly->out;
            // He-uniform initialisation from the seed
            std::vector<float> w(nw);
            const double a = std::sqrt(6.0 / ly->in);
            std::uniform_real_distribution<double> ud(-a, a);
            for (auto& v : w) v = (float)ud(rng);
            ly->w.alloc(nw);
            MCK(cudaMemcpyAsync(ly->w.p, w.data(), nw * 4, cudaMemcpyHostToDevice, stream));
            MCK(cudaStreamSynchronize(stream));
            ly->b.alloc(ly->out);
            ly->gw.alloc(nw);
            ly->gb.alloc(ly->out);
            ly->mw.alloc(nw);
            ly->vw.alloc(nw);
            ly->mb.alloc(ly->out);
            ly->vb.alloc(ly->out);
            ly->w16.alloc(nw);
            ly->w16t.alloc(nw);
            refresh_bf16(l);
        }
        xin.alloc((size_t)rows * p.n_in);
        yin.alloc((size_t)rows * p.n_out);
        feat.alloc((size_t)rows * F);
        featT.alloc((size_t)rows * F);
        for (int l = 0; l + 1 < p.n_layers; ++l) {
            H.push_back(new Dev<bf16>);
            H.back()->alloc((size_t)rows * p.hidden);
            HT.push_back(new Dev<bf16>);
            HT.back()->alloc((size_t)rows * p.hidden);
        }
        for (int l = 0; l < p.n_layers; ++l) {
            const int o = L[(size_t)l]->out;
            G.push_back(new Dev<bf16>);
            G.back()->alloc((size_t)rows * o);
            GT.push_back(new Dev<bf16>);
            GT.back()->alloc((size_t)rows * o);
        }
        pred.alloc((size_t)rows * p.n_out);
        loss.alloc(1);
        flag.alloc(1);
        // the GEMMs of one training step, with their tensor maps
        for (int l = 0; l < p.n_layers; ++l) {
            Layer& ly = *L[(size_t)l];
            const bool last = l == p.n_layers - 1;
            Gemm f = make_gemm(last ? EPI_F32 : EPI_RELU, layer_input(l), ly.w16.p, rows, ly.out, ly.in, flag.p);
            f.o.bias = ly.b.p;
            if (last) {
                f.o.c32 = pred.p;
                f.o.ldc = ly.out;
            } else {
                f.o.c16 = H[(size_t)l]->p;
                f.o.c16t = HT[(size_t)l]->p;
                f.o.ld16 = ly.out;
                f.o.ld16t = rows;
            }
            fwd.push_back(f);
            // dW = G^T (out x rows) * X^T (in x rows)^T
            Gemm w = make_gemm(EPI_F32, GT[(size_t)l]->p, layer_input_t(l), ly.out, ly.in, rows, flag.p);
            w.o.c32 = ly.gw.p;
            w.o.ldc = ly.in;
            bwd_w.push_back(w);
            if (l > 0) {
                // dX = G (rows x out) * W^T-as-[in][out] -> masked by the ReLU of layer l-1
                Gemm x = make_gemm(EPI_MASK, G[(size_t)l]->p, ly.w16t.p, rows, ly.in, ly.out, flag.p);
                x.o.c16 = G[(size_t)l - 1]->p;
                x.o.c16t = GT[(size_t)l - 1]->p;
                x.o.ld16 = ly.in;
                x.o.ld16t = rows;
                x.o.mask = H[(size_t)l - 1]->p;
                x.o.ldmask = ly.in;
                bwd_x.push_back(x);
            }
        }
    }

    void refresh_bf16(int l) {
        Layer& ly = *L[(size_t)l];
        const int64_t n = (int64_t)ly.in * ly.out;
        k_f32_to_bf16_both<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(ly.w.p, ly.out, ly.in, ly.w16.p, ly.w16t.p);
        MCK(cudaGetLastError());
    }

    void check_flag() {
        int f = 0;
        MCK(cudaMemcpyAsync(&f, flag.p, 4, cudaMemcpyDeviceToHost, stream));
        MCK(cudaStreamSynchronize(stream));
        if (f) throw Err(AFD_ERR_CUDA, "surrogate GEMM pipeline wait timed out");
    }

    void features(const float* x_dev, int n) {
        if (n < 1 || n > rows) throw Err(AFD_ERR_ARG, "row count outside 1..batch");
        MCK(cudaMemcpyAsync(xin.p, x_dev, (size_t)n * prm.n_in * 4, cudaMemcpyDefault, stream));
        const dim3 grd((unsigned)((rows + 127) / 128), (unsigned)prm.n_freq);
        k_fourier<<<grd, 128, 0, stream>>>(xin.p, n, prm.n_in, fourier.p, prm.n_freq, rows, feat.p, featT.p);
        MCK(cudaGetLastError());
    }

    void forward() {
        for (auto& g : fwd) launch(g, stream);
    }

    void backward(const float* y_dev, int n) {
        MCK(cudaMemcpyAsync(yin.p, y_dev, (size_t)n * prm.n_out * 4, cudaMemcpyDefault, stream));
        MCK(cudaMemsetAsync(loss.p, 0, 4, stream));
        const int nl = prm.n_layers;
        const float scale = 2.0f / ((float)n * (float)prm.n_out);
        const dim3 grd((unsigned)((prm.n_out + 255) / 256), (unsigned)rows);
        k_mse_grad<<<grd, 256, 0, stream>>>(pred.p, yin.p, n, prm.n_out, rows, scale, G[(size_t)nl - 1]->p,
                                            GT[(size_t)nl - 1]->p, loss.p);
        MCK(cudaGetLastError());
        for (int l = nl - 1; l >= 0; --l) {
            launch(bwd_w[(size_t)l], stream);
            Layer& ly = *L[(size_t)l];
            k_bias_grad<<<(unsigned)((ly.out + 7) / 8), 256, 0, stream>>>(GT[(size_t)l]->p, ly.out, rows, ly.gb.p);
            MCK(cudaGetLastError());
            if (l > 0) launch(bwd_x[(size_t)l - 1], stream);
        }
    }

    void adam() {
        ++step;
        const float b1 = prm.beta1, b2 = prm.beta2;
        const float c1 = 1.0f - (float)std::pow((double)b1, (double)step);
        const float c2 = 1.0f - (float)std::pow((double)b2, (double)step);
        for (auto* lp : L) {
            Layer& ly = *lp;
            const int64_t nw = (int64_t)ly.in * ly.out;
            k_adam<<<592, 256, 0, stream>>>(ly.w.p, ly.gw.p, ly.mw.p, ly.vw.p, nw, ly.in, prm.lr, b1, b2, prm.eps, c1,
                                            c2, ly.w16.p, ly.w16t.p, ly.out);
            k_adam<<<4, 256, 0, stream>>>(ly.b.p, ly.gb.p, ly.mb.p, ly.vb.p, ly.out, 1, prm.lr, b1, b2, prm.eps, c1, c2,
                                          nullptr, nullptr, 1);
            MCK(cudaGetLastError());
        }
    }
};

namespace {

template <typename F>
int mguard(afd_mlp* m, F&& f) {
    try {
        f();
        return AFD_OK;
    } catch (const Err& e) {
        if (m) m->err = e.what();
        return e.code;
    } catch (const std::exception& e) {
        if (m) m->err = e.what();
        return AFD_ERR_STATE;
    }
}

thread_local std::string g_create_err;

}  // namespace

extern "C" {

void afd_mlp_default_params(afd_mlp_params* p) {
    std::memset(p, 0, sizeof(*p));
    p->n_in = 10;
    p->n_freq = 128;
    p->hidden = 512;
    p->n_layers = 5;
    p->n_out = 2048;
    p->batch = 1024;
    p->device = 0;
    p->fourier_sigma = 1.0f;
    p->seed = 1;
    p->lr = 1e-3f;
    p->beta1 = 0.9f;
    p->beta2 = 0.999f;
    p->eps = 1e-8f;
}

int afd_mlp_create(afd_mlp** out, const afd_mlp_params* p) {
    if (!out || !p) return AFD_ERR_ARG;
    *out = nullptr;
    afd_mlp* m = new afd_mlp;
    m->prm = *p;
    const int st = mguard(m, [&] { m->build(); });
    if (st != AFD_OK) {
        g_create_err = m->err;
        delete m;
        return st;
    }
    *out = m;
    return AFD_OK;
}

void afd_mlp_destroy(afd_mlp* m) { delete m; }

const char* afd_mlp_last_error(const afd_mlp* m) { return m ? m->err.c_str() : g_create_err.c_str(); }

int afd_mlp_set_stream(afd_mlp* m, void* stream) {
    if (!m) return AFD_ERR_ARG;
    return mguard(m, [&] {
        MCK(cudaStreamSynchronize(m->stream));
        m->stream = stream ? (cudaStream_t)stream : m->own;
    });
}

int afd_mlp_train_step(afd_mlp* m, const float* x, const float* y, int32_t n, float* loss) {
    if (!m || !x || !y) return AFD_ERR_ARG;
    return mguard(m, [&] {
        MCK(cudaSetDevice(m->device));
        m->features(x, n);
        m->forward();
        m->backward(y, n);
        m->adam();
        if (loss) {
            float s = 0.0f;
            MCK(cudaMemcpyAsync(&s, m->loss.p, 4, cudaMemcpyDeviceToHost, m->stream));
            m->check_flag();
            *loss = s / ((float)n * (float)m->prm.n_out);
        }
    });
}

int afd_mlp_gradients(afd_mlp* m, const float* x, const float* y, int32_t n, float* loss) {
    if (!m || !x || !y) return AFD_ERR_ARG;
    return mguard(m, [&] {
        MCK(cudaSetDevice(m->device));
        m->features(x, n);
        m->forward();
        m->backward(y, n);
        float s = 0.0f;
        MCK(cudaMemcpyAsync(&s, m->loss.p, 4, cudaMemcpyDeviceToHost, m->stream));
        m->check_flag();
        if (loss) *loss = s / ((float)n * (float)m->prm.n_out);
    });
}

int afd_mlp_predict(afd_mlp* m, const float* x, int32_t n, float* out) {
    if (!m || !x || !out) return AFD_ERR_ARG;
    return mguard(m, [&] {
        MCK(cudaSetDevice(m->device));
        m->features(x, n);
        m->forward();
        MCK(cudaMemcpyAsync(out, m->pred.p, (size_t)n * m->prm.n_out * 4, cudaMemcpyDefault, m->stream));
        m->check_flag();
    });
}

int afd_mlp_sync(afd_mlp* m) {
    if (!m) return AFD_ERR_ARG;
    return mguard(m, [&] { m->check_flag(); });
}

int afd_mlp_get(afd_mlp* m, int32_t what, int32_t layer, float* out, int64_t cap) {
    if (!m || !out) return AFD_ERR_ARG;
    return mguard(m, [&] {
        MCK(cudaSetDevice(m->device));
        MCK(cudaStreamSynchronize(m->stream));
        if (what == AFD_MLP_FOURIER) {
            if (cap < (int64_t)m->fourier.n) throw Err(AFD_ERR_ARG, "output buffer too small");
            MCK(cudaMemcpy(out, m->fourier.p, m->fourier.n * 4, cudaMemcpyDeviceToHost));
            return;
        }
        if (what == AFD_MLP_FEATURES) {
            const size_t n = (size_t)m->rows * m->F;
            if (cap < (int64_t)n) throw Err(AFD_ERR_ARG, "output buffer too small");
            std::vector<bf16> h(n);
            MCK(cudaMemcpy(h.data(), m->feat.p, n * 2, cudaMemcpyDeviceToHost));
            for (size_t i = 0; i < n; ++i) out[i] = __bfloat162float(h[i]);
            return;
        }
        if (layer < 0 || layer >= (int)m->L.size()) throw Err(AFD_ERR_ARG, "layer index out of range");
        Layer& ly = *m->L[(size_t)layer];
        const Dev<float>* src = what == AFD_MLP_WEIGHT ? &ly.w : what == AFD_MLP_BIAS ? &ly.b
                                : what == AFD_MLP_GRAD_WEIGHT ? &ly.gw : what == AFD_MLP_GRAD_BIAS ? &ly.gb : nullptr;
        if (!src) throw Err(AFD_ERR_ARG, "unknown tensor");
        if (cap < (int64_t)src->n) throw Err(AFD_ERR_ARG, "output buffer too small");
        MCK(cudaMemcpy(out, src->p, src->n * 4, cudaMemcpyDeviceToHost));
    });
}

int afd_mlp_set_weights(afd_mlp* m, int32_t layer, const float* w, const float* b) {
    if (!m || !w || !b) return AFD_ERR_ARG;
    return mguard(m, [&] {
        MCK(cudaSetDevice(m->device));
        if (layer < 0 || layer >= (int)m->L.size()) throw Err(AFD_ERR_ARG, "layer index out of range");
        Layer& ly = *m->L[(size_t)layer];
        MCK(cudaMemcpyAsync(ly.w.p, w, ly.w.n * 4, cudaMemcpyHostToDevice, m->stream));
        MCK(cudaMemcpyAsync(ly.b.p, b, ly.b.n * 4, cudaMemcpyHostToDevice, m->stream));
        m->refresh_bf16(layer);
        MCK(cudaStreamSynchronize(m->stream));
    });
}

int afd_gemm_bf16_async(const void* a, const void* b, float* c, int32_t M, int32_t N, int32_t K, void* stream,
                        int32_t* status) {
    try {
        if (!a || !b || !c || !status) throw Err(AFD_ERR_ARG, "null pointer");
        Gemm g = make_gemm(EPI_F32, (const bf16*)a, (const bf16*)b, M, N, K, status);
        g.o.c32 = c;
        g.o.ldc = N;
        launch(g, (cudaStream_t)stream);
        return AFD_OK;
    } catch (const Err& e) {
        g_create_err = e.what();
        return e.code;
    } catch (const std::exception& e) {
        g_create_err = e.what();
        return AFD_ERR_STATE;
    }
}

int afd_gemm_bf16(const void* a, const void* b, float* c, int32_t M, int32_t N, int32_t K, void* stream) {
    try {
        if (!a || !b || !c) throw Err(AFD_ERR_ARG, "null pointer");
        int dev = 0;
        MCK(cudaGetDevice(&dev));
        if (dev < 0 || dev >= 64) throw Err(AFD_ERR_ARG, "device ordinal out of range");
        static Dev<int> flags[64];  // the wait-expired flag of each device, kept for the process
        Dev<int>& flag = flags[dev];
        {
            std::lock_guard<std::mutex> lock(g_gemm_mu);
            if (!flag.p) flag.alloc(1);
        }
        Gemm g = make_gemm(EPI_F32, (const bf16*)a, (const bf16*)b, M, N, K, flag.p);
        g.o.c32 = c;
        g.o.ldc = N;
        cudaStream_t st = (cudaStream_t)stream;
        // one flag per device: concurrent calls on one device share it
        MCK(cudaMemsetAsync(flag.p, 0, sizeof(int), st));
        launch(g, st);
        int f = 0;
        MCK(cudaMemcpyAsync(&f, flag.p, 4, cudaMemcpyDeviceToHost, st));
        MCK(cudaStreamSynchronize(st));
        if (f) throw Err(AFD_ERR_CUDA, "GEMM pipeline wait timed out");
        return AFD_OK;
    } catch (const Err& e) {
        g_create_err = e.what();
        return e.code;
    } catch (const std::exception& e) {
        g_create_err = e.what();
        return AFD_ERR_STATE;
    }
}

}  // extern "C"
