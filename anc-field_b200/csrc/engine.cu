// Simulation engine: device memory, compact lists, step kernels and the
// chunked step loop (per-step launches or replayed CUDA graphs).
//
// Per time step (simulation.hpp:358-393) the reference runs leapfrog, 26
// LRS groups, the PML kernel, source and mic. Here a step is
//   fused:   the streaming interior kernel (k_stream, TMA z-marching), then
//            the boundary list and, in FIXED mode, the PML pressure boxes
//            (side by side inside a CUDA graph), the per-axis PML auxiliary
//            updates and the source/receiver kernel;
//   unfused: one-thread-per-cell interior kernel, boundary, PML and
//            source/receiver kernels in turn.
// REF mode with a PML runs the reference's PML order (k_pml_ref_*), because
// the reference PML kernel reads the boundary-updated pressure of its
// neighbours (pml.cl:124-137).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <stdexcept>
#include <string>
#include <vector>

#include "device.cuh"
#include "engine.hpp"
#include "fused.cuh"
#include "geometry.hpp"

namespace afd {

#define CK(call)                                                                        \
    do {                                                                                \
        cudaError_t err__ = (call);                                                     \
        if (err__ != cudaSuccess)                                                       \
            throw Error(AFD_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(err__)); \
    } while (0)

template <typename T>
struct DBuf {
    T* ptr = nullptr;
    size_t n = 0;
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    ~DBuf() { release(); }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        n = 0;
    }
    void alloc(size_t count, bool zero = true) {
        release();
        if (count == 0) return;
        CK(cudaMalloc(&ptr, count * sizeof(T)));
        n = count;
        // the engine's streams are non-blocking and do not wait for the
        // legacy stream the zeroing runs on: finished before return
        if (zero) {
            CK(cudaMemset(ptr, 0, count * sizeof(T)));
            CK(cudaStreamSynchronize(cudaStreamLegacy));
        }
    }
    void upload(const std::vector<T>& v) {
        alloc(v.size(), false);
        if (v.empty()) return;
        // a copy from pageable memory may return before its DMA lands
        CK(cudaMemcpy(ptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
        CK(cudaStreamSynchronize(cudaStreamLegacy));
    }
};

// ---------------------------------------------------------------------------
// Unfused kernels (one launch per sub-step, the reference's order)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void watch(int* flag, float v) {
    if (!(fabsf(v) < 1e30f)) atomicOr(flag, 1);
}

// leapfrog.cl:34-55 over 1 <= x,y,z <= n-2 of every batch member. FP16
// storage: the update on stored values and the largest |p^n| gathered per
// warp, as in k_stream.
template <typename T>
__global__ void __launch_bounds__(256) k_interior(StepArgs a, int j) {
    const long long g = *a.d_step + j;
    const TlMark tl(a, 0, g, blockIdx.z < (unsigned)(a.g.nz - 2));
    const int x = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int y = 1 + blockIdx.y * blockDim.y + threadIdx.y;
    const int zn = a.g.nz - 2;
    const int b = blockIdx.z / zn;
    const int z = 1 + blockIdx.z % zn;
    const size_t base = (size_t)b * a.g.vol;
    const int64_t i = (int64_t)z * a.g.plane + (int64_t)y * a.g.pitch + x;
    if constexpr (sizeof(T) == 4) {
        if (x > a.g.nx - 2 || y > a.g.ny - 2) return;
        float* pn = a.p[buf_new(g)] + base;
        const float* pc = a.p[buf_cur(g)] + base;
        const float* po = a.p[buf_old(g)] + base;
        const float v = slf_update(a.lambda2, a.cint, pc[i + 1], pc[i - 1], pc[i + a.g.pitch],
                                   pc[i - a.g.pitch], pc[i + a.g.plane], pc[i - a.g.plane], pc[i], po[i]);
        pn[i] = v;
        watch(a.flag, v);
    } else {
        if (blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 && threadIdx.x == 0 && threadIdx.y == 0)
            for (int m = 0; m < a.batch; ++m) a.f16.mx[(size_t)m * 5 + max_slot(g)] = 0u;
        const bool in = x <= a.g.nx - 2 && y <= a.g.ny - 2;
        const StepScales sc = step_scales(a.f16, b, g);
        uint32_t amax = 0;
        if (in) {
            __half* pn = a.f16.h[buf_new(g)] + base;
            const __half* pc = a.f16.h[buf_cur(g)] + base;
            const __half* po = a.f16.h[buf_old(g)] + base;
            const float v = slf_update_scaled(
                a.lambda2, sc.s_new * sc.inv_cur, sc.s_new * sc.inv_old, __half2float(pc[i + 1]),
                __half2float(pc[i - 1]), __half2float(pc[i + a.g.pitch]), __half2float(pc[i - a.g.pitch]),
                __half2float(pc[i + a.g.plane]), __half2float(pc[i - a.g.plane]), __half2float(pc[i]),
                __half2float(po[i]));
            pn[i] = __float2half_rn(v);
            if (!f16_finite(v)) atomicOr(a.flag, 1);
            amax = __half_as_ushort(pc[i]) & 0x7fffu;
        }
        const uint32_t wmax = __reduce_max_sync(0xffffffffu, amax);
        if ((threadIdx.x & 31) == 0 && wmax)
            atomicMax(a.f16.mx + (size_t)b * 5 + max_slot(g - 1),
                      __float_as_uint(__half2float(__ushort_as_half((unsigned short)wmax)) * sc.inv_cur));
    }
}

// The 26 lrs_k launches of simulation.hpp:366-370 as one launch over the
// compact list.
// KT: filter length fixed at compile time (1..4), 0 for any length.
// T: level storage (FP16 only with the FIXED scheme).
// Memory-latency-bound gathers: 5 blocks per SM (48 registers, no spills
// for the FIXED variants) keep more loads in flight than 4.
// One boundary point e of batch member b at global step g: reads p^n and
// p^{n-1} around the cell, writes p^{n+1} of the cell and its filter state.
template <bool REF, int KT, typename T>
__device__ __forceinline__ void lrs_update(const StepArgs& a, int b, int e, long long g) {
    const size_t base = (size_t)b * a.g.vol;
    T* pn = level_ptr<T>(a, buf_new(g)) + base;
    const T* pc = level_ptr<T>(a, buf_cur(g)) + base;
    const T* po = level_ptr<T>(a, buf_old(g)) + base;
    float s_new = 1.0f, ic = 1.0f, io = 1.0f;
    if constexpr (sizeof(T) == 2) {
        const StepScales sc = step_scales(a.f16, b, g);
        s_new = sc.s_new;
        ic = sc.inv_cur;
        io = sc.inv_old;
    }
    const int64_t c = __ldg(a.lrs.cell + e);
    const uint32_t info = __ldg(a.lrs.info + e);
    const float nb[6] = {fldg(pc + c + 1, ic), fldg(pc + c - 1, ic), fldg(pc + c + a.g.pitch, ic),
                         fldg(pc + c - a.g.pitch, ic), fldg(pc + c + a.g.plane, ic), fldg(pc + c - a.g.plane, ic)};
    const int grp = (int)(info & 31u);
    const int ix_buf = ring_index(g, a.lrs.K);
    float v;
    if (grp < 6) {
        v = lrs_face<KT>(a.lrs, e, b, grp, (int)((info >> 5) & 255u), nb, fldg(pc + c, ic), fldg(po + c, io),
                         ix_buf);
    } else {
        const float pint = (REF && grp == 25) ? fld(pn + c, 1.0f) : 0.0f;
        v = lrs_point<REF, KT>(a.lrs, e, b, info, nb, fldg(pc + c, ic), fldg(po + c, io), pint, ix_buf);
    }
    fst(pn + c, v, s_new);
    if constexpr (sizeof(T) == 2) {
        if (!f16_finite(v * s_new)) atomicOr(a.flag, 1);
    }
}

template <bool REF, int KT, typename T>
__global__ void __launch_bounds__(256, 5) k_lrs(const __grid_constant__ StepArgs a, int j) {
    const long long g = *a.d_step + j;
    const TlMark tl(a, 1, g, blockIdx.y == 0);
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= a.lrs.n) return;
    lrs_update<REF, KT, T>(a, (int)blockIdx.y, e, g);
}

template <bool REF, typename T>
static void launch_lrs(const StepArgs& a, int j, dim3 grd, cudaStream_t st) {
    switch (a.lrs.K) {
        case 1: k_lrs<REF, 1, T><<<grd, 256, 0, st>>>(a, j); break;
        case 2: k_lrs<REF, 2, T><<<grd, 256, 0, st>>>(a, j); break;
        case 3: k_lrs<REF, 3, T><<<grd, 256, 0, st>>>(a, j); break;
        case 4: k_lrs<REF, 4, T><<<grd, 256, 0, st>>>(a, j); break;
        default: k_lrs<REF, 0, T><<<grd, 256, 0, st>>>(a, j); break;
    }
}

// ---- PML -------------------------------------------------------------------
// Face averages of pml.cl:74-122 (fi_*_avg, p_*_avg, psi_*_avg share one
// pattern each): x-faces average over (y, y+1) x (z, z+1), y-faces over
// (x, x+1) x (z, z+1), z-faces over (x, x+1) x (y, y+1). `own` replaces the
// value of cell `self` when it is one of the four (the reference kernel's
// own write becomes visible to its later reads, pml.cl:185-188).
struct Avg {
    const float* f;
    int64_t self;
    float own;
    bool subst;
    __device__ __forceinline__ float v(int64_t i) const { return (subst && i == self) ? own : f[i]; }
    __device__ __forceinline__ float ax(int64_t i, int64_t pitch, int64_t plane) const {
        return 0.25f * (((v(i) + v(i + plane)) + v(i + pitch)) + v(i + pitch + plane));
    }
    __device__ __forceinline__ float ay(int64_t i, int64_t pitch, int64_t plane) const {
        return 0.25f * (((v(i) + v(i + plane)) + v(i + 1)) + v(i + 1 + plane));
    }
    __device__ __forceinline__ float az(int64_t i, int64_t pitch, int64_t plane) const {
        return 0.25f * (((v(i) + v(i + pitch)) + v(i + 1)) + v(i + 1 + pitch));
    }
};

// PML pressure update, pml.cl:185-207. Returns p^{n+1}; psi_new receives
// psi^{n+1/2} = dt*p^n + psi^{n-1/2}.
__device__ __forceinline__ float pml_pressure(const StepArgs& a, const float* pc, const float* po,
                                              const float* fx1, const float* fy1, const float* fz1,
                                              const float* psimh, int x, int y, int z, int64_t i,
                                              float* psi_new) {
    const PmlDev& P = a.pml;
    const int64_t pitch = a.g.pitch, plane = a.g.plane;
    const float kx = P.ksi[0][x], ky = P.ksi[1][y], kz = P.ksi[2][z];
    const float pm1 = pc[i];
    const float ps = P.dt * pm1 + psimh[i];
    *psi_new = ps;
    float s = pc[i + 1] + pc[i - 1];
    s = s + pc[i + pitch];
    s = s + pc[i - pitch];
    s = s + pc[i + plane];
    s = s + pc[i - plane];
    s = s - 6.0f * pm1;
    const float A = P.cc_dxdx * s;
    const Avg FX{fx1, -1, 0.0f, false}, FY{fy1, -1, 0.0f, false}, FZ{fz1, -1, 0.0f, false};
    float d = FX.ax(i + 1, pitch, plane) - FX.ax(i, pitch, plane);
    d = d + FY.ay(i + pitch, pitch, plane);
    d = d - FY.ay(i, pitch, plane);
    d = d + FZ.az(i + plane, pitch, plane);
    d = d - FZ.az(i, pitch, plane);
    const float B = P.inv_dx * d;
    const float C = kx * ky * kz * 0.5f * (ps + psimh[i]);
    const float D = P.inv_dt2 * (po[i] - 2.0f * pm1);
    const float E = (kx * ky + ky * kz + kz * kx) * pm1;
    const float F = (kx + ky + kz) / P.two_dt * po[i];
    const float num = A + B - C - D - E + F;
    return num / (P.inv_dt2 + (kx + ky + kz) / P.two_dt);
}

// Auxiliary field updates of pml.cl:231-262 for one cell. REF: `p` reads
// see the cell's own new pressure and the other cells' values before the
// PML pass; the x-derivative's last term reads p (pml.cl:126) and fi_y's
// psi coefficient reads ksi_x at y (pml.cl:247). FIXED: both corrected.
template <bool REF>
__device__ __forceinline__ void pml_aux(const StepArgs& a, unsigned axes, const float* pnew,
                                        const float* pc, const float* psiph, float p_own,
                                        float psi_own, const float* fx1, const float* fy1,
                                        const float* fz1, float* fx, float* fy, float* fz, int x,
                                        int y, int z, int64_t i) {
    const PmlDev& P = a.pml;
    const int64_t pitch = a.g.pitch, plane = a.g.plane;
    const Avg Pn{pnew, i, p_own, REF}, Pm{pc, -1, 0.0f, false}, Ps{psiph, i, psi_own, REF};
    const Avg& Plast = REF ? Pn : Pm;
    const float kax = 0.5f * (P.ksi[0][x] + P.ksi[0][x + 1]);
    const float kay = 0.5f * (P.ksi[1][y] + P.ksi[1][y + 1]);
    const float kaz = 0.5f * (P.ksi[2][z] + P.ksi[2][z + 1]);
    const bool psi = REF || P.psi_on;
    if (axes & 1u) {
        const float dxp = P.half_inv_dx * (Pn.ax(i + 1, pitch, plane) - Pn.ax(i, pitch, plane) +
                                           Pm.ax(i + 1, pitch, plane) - Plast.ax(i, pitch, plane));
        const float dxpsi = psi ? P.inv_dx * (Ps.ax(i + 1, pitch, plane) - Ps.ax(i, pitch, plane)) : 0.0f;
        const float f1 = fx1[i];
        fx[i] = (-0.5f * kax * f1 + (kay + kaz - kax) * dxp + (kay * kaz) * dxpsi + P.inv_dt * f1) /
                (P.inv_dt + kax * 0.5f);
    }
    if (axes & 2u) {
        const float dyp = P.half_inv_dx * (Pn.ay(i + pitch, pitch, plane) - Pn.ay(i, pitch, plane) +
                                           Pm.ay(i + pitch, pitch, plane) - Plast.ay(i, pitch, plane));
        const float dypsi = psi ? P.inv_dx * (Ps.ay(i + pitch, pitch, plane) - Ps.ay(i, pitch, plane)) : 0.0f;
        const float kx_coef = REF ? 0.5f * (P.ksi[0][y] + P.ksi[0][y + 1]) : kax;
        const float f1 = fy1[i];
        fy[i] = (-0.5f * kay * f1 + (kax + kaz - kay) * dyp + (kx_coef * kaz) * dypsi + P.inv_dt * f1) /
                (P.inv_dt + kay * 0.5f);
    }
    if (axes & 4u) {
        const float dzp = P.half_inv_dx * (Pn.az(i + plane, pitch, plane) - Pn.az(i, pitch, plane) +
                                           Pm.az(i + plane, pitch, plane) - Plast.az(i, pitch, plane));
        const float dzpsi = psi ? P.inv_dx * (Ps.az(i + plane, pitch, plane) - Ps.az(i, pitch, plane)) : 0.0f;
        const float f1 = fz1[i];
        fz[i] = (-0.5f * kaz * f1 + (kax + kay - kaz) * dzp + (kax * kay) * dzpsi + P.inv_dt * f1) /
                (P.inv_dt + kaz * 0.5f);
    }
}

__device__ __forceinline__ int pml_level(const StepArgs& a, long long g) {
    return (int)((g - a.pml.g0 + 1) & 1);
}

// REF pass 1: auxiliary fields of every cell 2..n-3, using the cell's own
// new pressure and psi recomputed locally (nothing written that is read).
__global__ void __launch_bounds__(256) k_pml_ref_aux(StepArgs a, int j) {
    const long long g = *a.d_step + j;
    const TlMark tl(a, 3, g, blockIdx.z < (unsigned)(a.g.nz - 4));
    const int x = 2 + blockIdx.x * blockDim.x + threadIdx.x;
    const int y = 2 + blockIdx.y * blockDim.y + threadIdx.y;
    const int zn = a.g.nz - 4;
    const int b = blockIdx.z / zn;
    const int z = 2 + blockIdx.z % zn;
    if (x > a.g.nx - 3 || y > a.g.ny - 3) return;
    const int W = a.pml.width;
    unsigned axes = 0;
    if (x < W || x > a.g.nx - W - 1) axes |= 1u;
    if (y < W || y > a.g.ny - W - 1) axes |= 2u;
    if (z < W || z > a.g.nz - W - 1) axes |= 4u;
    if (!axes) return;
    const size_t base = (size_t)b * a.g.vol;
    const float* pn = a.p[buf_new(g)] + base;
    const float* pc = a.p[buf_cur(g)] + base;
    const float* po = a.p[buf_old(g)] + base;
    const int lv = pml_level(a, g);
    const float* fx1 = a.pml.fi[0][lv ^ 1] + base;
    const float* fy1 = a.pml.fi[1][lv ^ 1] + base;
    const float* fz1 = a.pml.fi[2][lv ^ 1] + base;
    const float* psiph = a.pml.psi[lv] + base;
    const float* psimh = a.pml.psi[lv ^ 1] + base;
    const int64_t i = (int64_t)z * a.g.plane + (int64_t)y * a.g.pitch + x;
    float psi_new;
    const float p_new = pml_pressure(a, pc, po, fx1, fy1, fz1, psimh, x, y, z, i, &psi_new);
    pml_aux<true>(a, axes, pn, pc, psiph, p_new, psi_new, fx1, fy1, fz1, a.pml.fi[0][lv] + base,
                  a.pml.fi[1][lv] + base, a.pml.fi[2][lv] + base, x, y, z, i);
}

// REF pass 2: pressure and psi of every cell 2..n-3 (pml.cl:182-207).
__global__ void __launch_bounds__(256) k_pml_ref_p(StepArgs a, int j) {
    const long long g = *a.d_step + j;
    const TlMark tl(a, 2, g, blockIdx.z < (unsigned)(a.g.nz - 4));
    const int x = 2 + blockIdx.x * blockDim.x + threadIdx.x;
    const int y = 2 + blockIdx.y * blockDim.y + threadIdx.y;
    const int zn = a.g.nz - 4;
    const int b = blockIdx.z / zn;
    const int z = 2 + blockIdx.z % zn;
    if (x > a.g.nx - 3 || y > a.g.ny - 3) return;
    const size_t base = (size_t)b * a.g.vol;
    float* pn = a.p[buf_new(g)] + base;
    const float* pc = a.p[buf_cur(g)] + base;
    const float* po = a.p[buf_old(g)] + base;
    const int lv = pml_level(a, g);
    const int64_t i = (int64_t)z * a.g.plane + (int64_t)y * a.g.pitch + x;
    float psi_new;
    const float v = pml_pressure(a, pc, po, a.pml.fi[0][lv ^ 1] + base, a.pml.fi[1][lv ^ 1] + base,
                                 a.pml.fi[2][lv ^ 1] + base, a.pml.psi[lv ^ 1] + base, x, y, z, i,
                                 &psi_new);
    a.pml.psi[lv][base + i] = psi_new;
    pn[i] = v;
}

// ---- FIXED-mode PML over dense slab boxes ----------------------------------
// Axes whose enabled slab meets the coordinate ranges (inclusive): for one
// cell, the auxiliary fields it updates; for a cell's 2x2x2 cube, the fields
// its pressure update can read as nonzero.
__device__ __forceinline__ unsigned slab_axes(const StepArgs& a, int x0, int x1, int y0, int y1, int z0,
                                              int z1) {
    const uint32_t F = a.pml.faces;
    const int W = a.pml.width;
    unsigned ax = 0;
    if (((F & AFD_FACE_XM) && x0 < W) || ((F & AFD_FACE_XP) && x1 > a.g.nx - W - 1)) ax |= 1u;
    if (((F & AFD_FACE_YM) && y0 < W) || ((F & AFD_FACE_YP) && y1 > a.g.ny - W - 1)) ax |= 2u;
    const int zg0 = z0 + a.pml.zoff, zg1 = z1 + a.pml.zoff;
    if (((F & AFD_FACE_ZM) && zg0 < W) || ((F & AFD_FACE_ZP) && zg1 > a.pml.nz_glob - W - 1)) ax |= 4u;
    return ax;
}

// The four cells x..x+3 (x a multiple of 4) of row (y, z) that are PML
// cells (inside 2..n-3, in an enabled slab, plain air), as a bit mask.
__device__ __forceinline__ unsigned pml_mask4(const StepArgs& a, int x, int y, int z) {
    const PmlDev& P = a.pml;
    return (__ldg(P.cells + ((int64_t)z * a.g.ny + y) * P.words_per_row + (x >> 5)) >> (x & 31)) & 15u;
}

// Values x..x+4 of a row (x a multiple of 4). hi = false: the fifth value
// is not needed (the unit's last cell is not updated) and not loaded; at the
// end of a row it would cost a DRAM sector of the next row for one value.
__device__ __forceinline__ void row5(const float* p, float r[5], bool hi = true) {
    const float4 v = __ldg(reinterpret_cast<const float4*>(p));
    r[0] = v.x;
    r[1] = v.y;
    r[2] = v.z;
    r[3] = v.w;
    r[4] = hi ? __ldg(p + 4) : 0.0f;
}

__device__ __forceinline__ void store4(float* p, const float v[4], unsigned m) {
    if (m == 15u) {
        *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
    } else {
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (m & (1u << q)) p[q] = v[q];
    }
}

// The same for a pressure level of either storage: FP16 rows decode with
// 1/s (eight-byte loads of four values) and stores encode v * s.
template <typename T>
__device__ __forceinline__ void row5t(const T* p, float r[5], float inv, bool fifth = true) {
    if constexpr (sizeof(T) == 4) {
        (void)inv;
        row5(p, r, fifth);
    } else {
        const uint2 w = __ldg(reinterpret_cast<const uint2*>(p));
        const float2 lo = __half22float2(*reinterpret_cast<const __half2*>(&w.x));
        const float2 hi = __half22float2(*reinterpret_cast<const __half2*>(&w.y));
        r[0] = lo.x * inv;
        r[1] = lo.y * inv;
        r[2] = hi.x * inv;
        r[3] = hi.y * inv;
        r[4] = fifth ? __half2float(__ldg(p + 4)) * inv : 0.0f;
    }
}

template <typename T>
__device__ __forceinline__ void store4t(T* p, const float v[4], unsigned m, float s) {
    if constexpr (sizeof(T) == 4) {
        (void)s;
        store4(p, v, m);
    } else if (m == 15u) {
        const __half2 lo = __floats2half2_rn(v[0] * s, v[1] * s), hi = __floats2half2_rn(v[2] * s, v[3] * s);
        uint2 w;
        w.x = *reinterpret_cast<const uint32_t*>(&lo);
        w.y = *reinterpret_cast<const uint32_t*>(&hi);
        *reinterpret_cast<uint2*>(p) = w;
    } else {
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (m & (1u << q)) p[q] = __float2half_rn(v[q] * s);
    }
}

// Pressure of the PML cells (pml.cl:185-207 restricted to the slab cells)
// of one 4-cell unit x..x+3 of row (y, z). Fields outside the read axes are
// identically zero there and are not loaded; PSI: psi is kept (PML faces on
// all three axes). s_new, ic, io: FP16 scales of the new level and inverse
// scales of p^n and p^{n-1} (1 for FP32 storage).
template <bool PSI, typename T>
__device__ __forceinline__ void pml_p_unit(const StepArgs& a, int b, int x, int y, int z, long long g,
                                           float s_new, float ic, float io) {
    // The mask gates only the stores and the flag: the loads below issue
    // without waiting for it (every unit of a box lies in planes and rows
    // 2..n-3, so x-1 .. x+4, y+-1 and z+-1 stay inside the level and field
    // arrays even for a unit with no PML cell, whose results are dropped).
    const unsigned m = pml_mask4(a, x, y, z);
    const PmlDev& P = a.pml;
    const size_t base = (size_t)b * a.g.vol;
    const int64_t pitch = a.g.pitch, plane = a.g.plane;
    const int64_t i = (int64_t)z * plane + (int64_t)y * pitch + x;
    const T* pc = level_ptr<T>(a, buf_cur(g)) + base;
    const T* po = level_ptr<T>(a, buf_old(g)) + base;
    T* pn = level_ptr<T>(a, buf_new(g)) + base;
    const int lv = pml_level(a, g);
    // x+4 is read only where it lies in the row (the unit's last cell can be
    // a PML cell only then)
    const bool hi = x + 4 < a.g.pitch;
    float c[5], ym4[5], yp4[5], zm4[5], zp4[5], o[5];
    row5t(pc + i, c, ic, hi);
    const float xm = x >= 1 ? fldg(pc + i - 1, ic) : 0.0f;
    row5t(pc + i - pitch, ym4, ic, false);
    row5t(pc + i + pitch, yp4, ic, false);
    row5t(pc + i - plane, zm4, ic, false);
    row5t(pc + i + plane, zp4, ic, false);
    row5t(po + i, o, io, false);
    const float4 kx4 = __ldg(reinterpret_cast<const float4*>(P.ksi[0] + x));
    const float kxv[4] = {kx4.x, kx4.y, kx4.z, kx4.w};
    const float ky = __ldg(P.ksi[1] + y), kz = __ldg(P.ksi[2] + z);
    const unsigned ra = slab_axes(a, x, x + 4, y, y + 1, z, z + 1);
    float d[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    if (ra & 1u) {
        const float* f = P.fi[0][lv ^ 1] + base + i;
        float r00[5], r01[5], r10[5], r11[5], av[5];
        row5(f, r00, hi);
        row5(f + plane, r01, hi);
        row5(f + pitch, r10, hi);
        row5(f + pitch + plane, r11, hi);
#pragma unroll
        for (int q = 0; q < 5; ++q) av[q] = 0.25f * (((r00[q] + r01[q]) + r10[q]) + r11[q]);
#pragma unroll
        for (int q = 0; q < 4; ++q) d[q] = av[q + 1] - av[q];
    }
    if (ra & 2u) {
        const float* f = P.fi[1][lv ^ 1] + base + i;
        float r00[5], r01[5], r10[5], r11[5];
        row5(f, r00, hi);
        row5(f + plane, r01, hi);
        row5(f + pitch, r10, hi);
        row5(f + pitch + plane, r11, hi);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const float a1 = 0.25f * (((r10[q] + r11[q]) + r10[q + 1]) + r11[q + 1]);
            const float a0 = 0.25f * (((r00[q] + r01[q]) + r00[q + 1]) + r01[q + 1]);
            d[q] = d[q] + a1;
            d[q] = d[q] - a0;
        }
    }
    if (ra & 4u) {
        const float* f = P.fi[2][lv ^ 1] + base + i;
        float r00[5], r01[5], r10[5], r11[5];
        row5(f, r00, hi);
        row5(f + plane, r01, hi);
        row5(f + pitch, r10, hi);
        row5(f + pitch + plane, r11, hi);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const float a1 = 0.25f * (((r01[q] + r11[q]) + r01[q + 1]) + r11[q + 1]);
            const float a0 = 0.25f * (((r00[q] + r10[q]) + r00[q + 1]) + r10[q + 1]);
            d[q] = d[q] + a1;
            d[q] = d[q] - a0;
        }
    }
    float ps[4] = {0.0f, 0.0f, 0.0f, 0.0f}, pmh[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    if (PSI) {
        const float4 h = *reinterpret_cast<const float4*>(P.psi[lv ^ 1] + base + i);
        pmh[0] = h.x;
        pmh[1] = h.y;
        pmh[2] = h.z;
        pmh[3] = h.w;
#pragma unroll
        for (int q = 0; q < 4; ++q) ps[q] = P.dt * c[q] + pmh[q];
        store4(P.psi[lv] + base + i, ps, m);
    }
    float v[4];
    // ks depends on kx only within the row: one division when the four agree
    float ksq[4];
    if (kxv[0] == kxv[1] && kxv[1] == kxv[2] && kxv[2] == kxv[3]) {
        const float k0 = (kxv[0] + ky + kz) / P.two_dt;
        ksq[0] = ksq[1] = ksq[2] = ksq[3] = k0;
    } else {
#pragma unroll
        for (int q = 0; q < 4; ++q) ksq[q] = (kxv[q] + ky + kz) / P.two_dt;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float xmq = q == 0 ? xm : c[q - 1];
        float s6 = c[q + 1] + xmq;
        s6 = s6 + yp4[q];
        s6 = s6 + ym4[q];
        s6 = s6 + zp4[q];
        s6 = s6 + zm4[q];
        const float kx = kxv[q];
        const float ks = ksq[q];
        const float A = P.cc_dxdx * (s6 - 6.0f * c[q]);
        const float B = P.inv_dx * d[q];
        const float C = kx * ky * kz * 0.5f * (ps[q] + pmh[q]);
        const float D = P.inv_dt2 * (o[q] - 2.0f * c[q]);
        const float E = (kx * ky + ky * kz + kz * kx) * c[q];
        const float F = ks * o[q];
        const float num = A + B - C - D - E + F;
        v[q] = num / (P.inv_dt2 + ks);
        if constexpr (sizeof(T) == 4) {
            if ((m >> q) & 1u) watch(a.flag, v[q]);
        } else {
            if (((m >> q) & 1u) && !f16_finite(v[q] * s_new)) atomicOr(a.flag, 1);
        }
    }
    store4t(pn + i, v, m, s_new);
}

// Auxiliary field AX of the PML cells of one 4-cell unit (pml.cl:231-262
// with the derivative and ksi index corrected). The derivatives of the new
// and previous pressure along every axis come from the same four rows
// (y, y+1) x (z, z+1), x..x+4. in_, ic: FP16 inverse scales of the new
// level and of p^n (1 for FP32 storage).
template <int AX, bool PSI, typename T>
__device__ __forceinline__ void pml_aux_unit(const StepArgs& a, int b, int x, int y, int z, long long g,
                                             float in_, float ic) {
    // loads issue without waiting for the mask, as in pml_p_unit
    const unsigned m = pml_mask4(a, x, y, z);
    const PmlDev& P = a.pml;
    const size_t base = (size_t)b * a.g.vol;
    const int64_t pitch = a.g.pitch, plane = a.g.plane;
    const int64_t i = (int64_t)z * plane + (int64_t)y * pitch + x;
    const T* pn = level_ptr<T>(a, buf_new(g)) + base + i;
    const T* pc = level_ptr<T>(a, buf_cur(g)) + base + i;
    const int lv = pml_level(a, g);
    const bool hi = x + 4 < a.g.pitch;  // x+4 is read only where it lies in the row
    float n00[5], n01[5], n10[5], n11[5], m00[5], m01[5], m10[5], m11[5];
    row5t(pn, n00, in_, hi);
    row5t(pn + plane, n01, in_, hi);
    row5t(pn + pitch, n10, in_, hi);
    row5t(pn + pitch + plane, n11, in_, hi);
    row5t(pc, m00, ic, hi);
    row5t(pc + plane, m01, ic, hi);
    row5t(pc + pitch, m10, ic, hi);
    row5t(pc + pitch + plane, m11, ic, hi);
    float s00[5] = {0}, s01[5] = {0}, s10[5] = {0}, s11[5] = {0};
    if (PSI) {
        const float* ps = P.psi[lv] + base + i;
        row5(ps, s00, hi);
        row5(ps + plane, s01, hi);
        row5(ps + pitch, s10, hi);
        row5(ps + pitch + plane, s11, hi);
    }
    float kxs[5];
    row5(P.ksi[0] + x, kxs, hi);
    const float kay = 0.5f * (__ldg(P.ksi[1] + y) + __ldg(P.ksi[1] + y + 1));
    const float kaz = 0.5f * (__ldg(P.ksi[2] + z) + __ldg(P.ksi[2] + z + 1));
    const float4 f14 = *reinterpret_cast<const float4*>(P.fi[AX][lv ^ 1] + base + i);
    const float f1v[4] = {f14.x, f14.y, f14.z, f14.w};
    float out[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float kax = 0.5f * (kxs[q] + kxs[q + 1]);
        const float f1 = f1v[q];
        if (AX == 0) {
            const float an1 = 0.25f * (((n00[q + 1] + n01[q + 1]) + n10[q + 1]) + n11[q + 1]);
            const float an0 = 0.25f * (((n00[q] + n01[q]) + n10[q]) + n11[q]);
            const float am1 = 0.25f * (((m00[q + 1] + m01[q + 1]) + m10[q + 1]) + m11[q + 1]);
            const float am0 = 0.25f * (((m00[q] + m01[q]) + m10[q]) + m11[q]);
            const float dxp = P.half_inv_dx * (an1 - an0 + am1 - am0);
            float dxpsi = 0.0f;
            if (PSI) {
                const float as1 = 0.25f * (((s00[q + 1] + s01[q + 1]) + s10[q + 1]) + s11[q + 1]);
                const float as0 = 0.25f * (((s00[q] + s01[q]) + s10[q]) + s11[q]);
                dxpsi = P.inv_dx * (as1 - as0);
            }
            out[q] = (-0.5f * kax * f1 + (kay + kaz - kax) * dxp + (kay * kaz) * dxpsi + P.inv_dt * f1) /
                     (P.inv_dt + kax * 0.5f);
        } else if (AX == 1) {
            const float an1 = 0.25f * (((n10[q] + n11[q]) + n10[q + 1]) + n11[q + 1]);
            const float an0 = 0.25f * (((n00[q] + n01[q]) + n00[q + 1]) + n01[q + 1]);
            const float am1 = 0.25f * (((m10[q] + m11[q]) + m10[q + 1]) + m11[q + 1]);
            const float am0 = 0.25f * (((m00[q] + m01[q]) + m00[q + 1]) + m01[q + 1]);
            const float dyp = P.half_inv_dx * (an1 - an0 + am1 - am0);
            float dypsi = 0.0f;
            if (PSI) {
                const float as1 = 0.25f * (((s10[q] + s11[q]) + s10[q + 1]) + s11[q + 1]);
                const float as0 = 0.25f * (((s00[q] + s01[q]) + s00[q + 1]) + s01[q + 1]);
                dypsi = P.inv_dx * (as1 - as0);
            }
            out[q] = (-0.5f * kay * f1 + (kax + kaz - kay) * dyp + (kax * kaz) * dypsi + P.inv_dt * f1) /
                     (P.inv_dt + kay * 0.5f);
        } else {
            const float an1 = 0.25f * (((n01[q] + n11[q]) + n01[q + 1]) + n11[q + 1]);
            const float an0 = 0.25f * (((n00[q] + n10[q]) + n00[q + 1]) + n10[q + 1]);
            const float am1 = 0.25f * (((m01[q] + m11[q]) + m01[q + 1]) + m11[q + 1]);
            const float am0 = 0.25f * (((m00[q] + m10[q]) + m00[q + 1]) + m10[q + 1]);
            const float dzp = P.half_inv_dx * (an1 - an0 + am1 - am0);
            float dzpsi = 0.0f;
            if (PSI) {
                const float as1 = 0.25f * (((s01[q] + s11[q]) + s01[q + 1]) + s11[q + 1]);
                const float as0 = 0.25f * (((s00[q] + s10[q]) + s00[q + 1]) + s10[q + 1]);
                dzpsi = P.inv_dx * (as1 - as0);
            }
            out[q] = (-0.5f * kaz * f1 + (kax + kay - kaz) * dzp + (kax * kay) * dzpsi + P.inv_dt * f1) /
                     (P.inv_dt + kaz * 0.5f);
        }
    }
    store4(P.fi[AX][lv] + base + i, out, m);
}

// One launch over several PML boxes: a flat grid whose blocks are dealt to
// the boxes in order (start[k] .. start[k+1]-1 to entry k). Within an entry
// a block holds w units across (w = min(units, 32)) and 256 / w rows, and
// every thread marches zc planes of its column; the planes (times the batch
// members) are split into chunks of zc.
constexpr int kMaxLaunchBoxes = 9;
struct BoxLaunch {
    int32_t n, zc;
    PmlBox box[kMaxLaunchBoxes];
    int32_t axis[kMaxLaunchBoxes];  // auxiliary launches: the field of the entry
    int32_t w[kMaxLaunchBoxes], gx[kMaxLaunchBoxes], gy[kMaxLaunchBoxes], gzc[kMaxLaunchBoxes];
    int32_t start[kMaxLaunchBoxes + 1];
};

struct BoxThread {
    int k, b, x, y, z0, z1;
    bool ok;
};

__device__ __forceinline__ BoxThread box_thread(const BoxLaunch& L) {
    BoxThread t;
    int k = 0;
    while (k + 1 < L.n && (int)blockIdx.x >= L.start[k + 1]) ++k;
    t.k = k;
    const PmlBox& bx = L.box[k];
    const int w = L.w[k], rows = 256 / w;
    int r = (int)blockIdx.x - L.start[k];
    const int bxi = r % L.gx[k];
    r /= L.gx[k];
    const int byi = r % L.gy[k];
    r /= L.gy[k];
    const int zci = r % L.gzc[k];
    t.b = r / L.gzc[k];
    const int ux = bxi * w + (int)threadIdx.x % w, yy = byi * rows + (int)threadIdx.x / w;
    t.ok = (int)threadIdx.x < w * rows && ux < bx.units && yy < bx.height;
    t.x = bx.x0 + 4 * ux;
    t.y = bx.y0 + yy;
    t.z0 = bx.z0 + zci * L.zc;
    t.z1 = min(t.z0 + L.zc, bx.z0 + bx.depth);
    return t;
}

// PML pressure over every box of the disjoint box cover in one launch. Four
// blocks per SM (64 registers in every variant).
template <bool PSI, typename T>
__global__ void __launch_bounds__(256, 3) k_pml_p_all(const __grid_constant__ StepArgs a,
                                                      const __grid_constant__ BoxLaunch L, int j) {
    const long long g = *a.d_step + j;
    const BoxThread t = box_thread(L);
    const TlMark tl(a, 2, g, t.b == 0);
    if (!t.ok) return;
    float s_new = 1.0f, ic = 1.0f, io = 1.0f;
    if constexpr (sizeof(T) == 2) {
        const StepScales sc = step_scales(a.f16, t.b, g);
        s_new = sc.s_new;
        ic = sc.inv_cur;
        io = sc.inv_old;
    }
#pragma unroll 1
    for (int z = t.z0; z < t.z1; ++z) pml_p_unit<PSI, T>(a, t.b, t.x, t.y, z, g, s_new, ic, io);
}

// The auxiliary fields of every (axis, slab box) pair in one launch: the
// fields are disjoint outputs and read only the new pressure, p^n, the new
// psi and their own previous level.
template <bool PSI, typename T>
__global__ void __launch_bounds__(256, 3) k_pml_aux_all(const __grid_constant__ StepArgs a,
                                                        const __grid_constant__ BoxLaunch L, int j) {
    const long long g = *a.d_step + j;
    const BoxThread t = box_thread(L);
    const int ax = L.axis[t.k];
    const TlMark tl(a, 3 + ax, g, t.b == 0);
    if (!t.ok) return;
    float in_ = 1.0f, ic = 1.0f;
    if constexpr (sizeof(T) == 2) {
        const StepScales sc = step_scales(a.f16, t.b, g);
        in_ = sc.inv_new;
        ic = sc.inv_cur;
    }
    if (ax == 0) {
#pragma unroll 1
        for (int z = t.z0; z < t.z1; ++z) pml_aux_unit<0, PSI, T>(a, t.b, t.x, t.y, z, g, in_, ic);
    } else if (ax == 1) {
#pragma unroll 1
        for (int z = t.z0; z < t.z1; ++z) pml_aux_unit<1, PSI, T>(a, t.b, t.x, t.y, z, g, in_, ic);
    } else {
#pragma unroll 1
        for (int z = t.z0; z < t.z1; ++z) pml_aux_unit<2, PSI, T>(a, t.b, t.x, t.y, z, g, in_, ic);
    }
}

// Eight binary16 values (one 16-byte word) as FP32 numbers.
__device__ __forceinline__ void cvt8(const uint4 w, float v[8]) {
    const uint32_t ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&ws[q]));
        v[2 * q] = f.x;
        v[2 * q + 1] = f.y;
    }
}

// Interior SLF update of every cell 1..n-2 (leapfrog.cl:34-55) streamed
// through shared memory; see fused.cuh. Consumer warps wait on the stage
// barriers independently (no block-wide barrier), so a slow warp delays
// only its own rows. T = __half: FP16 levels, the update evaluated on the
// stored values (slf_update_scaled) and the largest |p^n| of every work
// item gathered for the scale of level g + 1.
// The tail warps of the streaming kernel (FP32 storage, FIXED scheme): the
// step's boundary points and PML pressure units, taken 32 at a time from a
// per-step counter, while the other warps stream the interior (which skips
// those cells through the owned-cell mask). Both read only p^n, p^{n-1},
// the filter state and the previous auxiliary fields, and write disjoint
// cells; the order of the work items does not change any result.
constexpr int kTailWarps = 4;

__device__ __forceinline__ void stream_tail(const StepArgs& a, const FusedDev& f, int j, long long g) {
    const int lane = threadIdx.x & 31;
    const long long B = a.batch;
    const long long n_lrs = (long long)a.lrs.n * B;
    const bool pml = a.mode != AFD_MODE_REF && a.pml.width > 0 && a.pml.n_units > 0;
    const long long total = n_lrs + (pml ? a.pml.n_units * B : 0);
    const int K = a.lrs.K;
    const bool psi = a.pml.psi_on != 0;
    for (;;) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(f.tail + j, 32ull);
        base = __shfl_sync(0xffffffffu, base, 0);
        if ((long long)base >= total) break;
        const long long u = (long long)base + lane;
        if (u < n_lrs) {
            const int b = (int)(u / a.lrs.n), e = (int)(u - (long long)b * a.lrs.n);
            switch (K) {
                case 1: lrs_update<false, 1, float>(a, b, e, g); break;
                case 2: lrs_update<false, 2, float>(a, b, e, g); break;
                case 3: lrs_update<false, 3, float>(a, b, e, g); break;
                case 4: lrs_update<false, 4, float>(a, b, e, g); break;
                default: lrs_update<false, 0, float>(a, b, e, g); break;
            }
        } else if (u < total) {
            const PmlDev& P = a.pml;
            long long r = u - n_lrs;
            const int b = (int)(r / P.n_units);
            r -= (long long)b * P.n_units;
            int k = 0;
            while (k + 1 < P.n_boxes && r >= P.boxes[k + 1].first) ++k;
            const PmlBox& bx = P.boxes[k];
            r -= bx.first;
            const int ux = (int)(r % bx.units);
            r /= bx.units;
            const int yy = (int)(r % bx.height), zz = (int)(r / bx.height);
            if (psi) pml_p_unit<true, float>(a, b, bx.x0 + 4 * ux, bx.y0 + yy, bx.z0 + zz, g, 1.0f, 1.0f, 1.0f);
            else pml_p_unit<false, float>(a, b, bx.x0 + 4 * ux, bx.y0 + yy, bx.z0 + zz, g, 1.0f, 1.0f, 1.0f);
        }
    }
}

template <typename T, int S, bool TAIL = false>
__global__ void __launch_bounds__(TAIL ? F_THREADS + 32 * kTailWarps : F_THREADS, 2)
    k_stream(const __grid_constant__ CUtensorMap tm_halo, const __grid_constant__ CUtensorMap tm_own,
             const __grid_constant__ StepArgs a, const __grid_constant__ FusedDev f, int j) {
    const TlMark tl(a, 0, *a.d_step + j, true);
    using TL = Tile<T, S>;
    constexpr int F_STAGES = TL::STAGES;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + F_STAGES * TL::STAGE);
    uint64_t* empty = full + F_STAGES;
    int* slot = reinterpret_cast<int*>(empty + F_STAGES);  // work item of the stage that starts it
    const int tid = threadIdx.x;
    if (tid == 0) {
        for (int s = 0; s < F_STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], F_CONSUMERS / 32);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const long long g = *a.d_step + j;
    const int B = a.batch, nz = a.g.nz;
    const int n_items = f.items ? f.n_items : f.tiles_x * f.tiles_y * f.n_chunks * B;
    const int wn = buf_new(g), wc = buf_cur(g), wo = buf_old(g);
    if constexpr (TAIL && sizeof(T) == 4) {
        if (tid >= F_THREADS) {
            stream_tail(a, f, j, g);
            return;
        }
    }

    if (tid >= F_CONSUMERS) {
        // producer: takes work items from the launch's counter and streams
        // their planes; a stage with item -1 tells the consumers to stop
        if (tid == F_CONSUMERS) {
            if constexpr (sizeof(T) == 2) {
                // level g's maximum is gathered by the next step
                if (blockIdx.x == 0)
                    for (int b = 0; b < B; ++b) a.f16.mx[(size_t)b * 5 + max_slot(g)] = 0u;
            }
            uint32_t k = 0;
            bool ok = true;
            while (ok) {
                const int s0 = (int)(k % F_STAGES);
                if (k >= (uint32_t)F_STAGES && !mbar_wait(&empty[s0], ((k / F_STAGES) - 1) & 1)) {
                    atomicOr(a.flag, 2);
                    break;
                }
                const int taken = atomicAdd(f.work + j, 1);
                if (taken >= n_items) {
                    slot[s0] = -1;
                    mbar_arrive(&full[s0]);
                    ++k;
                    break;
                }
                const int item = f.items ? __ldg(f.items + taken) : taken;
                slot[s0] = item;
                const FusedItem it = fused_item(f, item, nz);
                const int x0 = it.tx * TL::W, y0 = it.ty * TL::H;
                const int zc = (wc * B + it.b) * nz, zo = (wo * B + it.b) * nz;
                for (int z = it.z0 - 1; z <= it.z1; ++z, ++k) {
                    const int s = (int)(k % F_STAGES);
                    if (z > it.z0 - 1 && k >= (uint32_t)F_STAGES &&
                        !mbar_wait(&empty[s], ((k / F_STAGES) - 1) & 1)) {
                        ok = false;
                        atomicOr(a.flag, 2);
                        break;
                    }
                    unsigned char* st = smem + s * TL::STAGE;
                    mbar_expect_tx(&full[s], TL::TX);
                    tma_load_3d(st, &tm_halo, x0 - TL::XOFF, y0 - 1, zc + z, &full[s]);
                    tma_load_3d(st + TL::PN_PAD, &tm_own, x0, y0, zo + z, &full[s]);
                }
            }
            // wait for the last copy issued into every stage before leaving
            for (uint32_t s = 0; s < (uint32_t)F_STAGES && s < k; ++s) {
                const uint32_t last = k - 1 - ((k - 1 - s) % F_STAGES);
                mbar_wait(&full[s], (last / F_STAGES) & 1);
            }
        }
        return;
    }

    const int lane = tid & 31;
    const int cx = (tid % TL::TPR) * TL::CPT, cy = tid / TL::TPR;
    const float L2 = a.lambda2, CI = a.cint;
    // FP16: the level scales of the current member, loaded again only when
    // a work item of another member comes (items of one member are
    // consecutive in the list), so the L2 load is off most items' path
    // (kept as the three factors the update uses: s_new / s_cur, s_cur /
    // s_old and 1 / s_cur)
    int sc_b = -1;
    float sc_rc = 1.0f, sc_ro = 1.0f, sc_ic = 1.0f;
    uint32_t k = 0;
    while (true) {
        if (!mbar_wait(&full[k % F_STAGES], (k / F_STAGES) & 1)) {
            if (lane == 0) atomicOr(a.flag, 2);
            return;
        }
        const int item = slot[k % F_STAGES];
        if (item < 0) break;
        const FusedItem it = fused_item(f, item, nz);
        const int x = it.tx * TL::W + cx, y = it.ty * TL::H + cy;
        T* pn = level_ptr<T>(a, wn) + (size_t)it.b * a.g.vol + (int64_t)y * a.g.pitch + x;
        const bool yok = (y >= 1 && y <= a.g.ny - 2);
        const bool xfull = (x >= 1 && x + TL::CPT - 1 <= a.g.nx - 2);
        const int planes = it.z1 - it.z0;
        if (!mbar_wait(&full[(k + 1) % F_STAGES], ((k + 1) / F_STAGES) & 1)) {
            if (lane == 0) atomicOr(a.flag, 2);
            return;
        }
        bool bad = false;
        if constexpr (sizeof(T) == 4) {
            for (int pl = 0; pl < planes; ++pl) {
                const int z = it.z0 + pl;
                const uint32_t kc = k + 1 + pl, kp = kc + 1, km = kc - 1;
                if (!mbar_wait(&full[kp % F_STAGES], (kp / F_STAGES) & 1)) {
                    if (lane == 0) atomicOr(a.flag, 2);
                    return;
                }
                const float* P0 = reinterpret_cast<const float*>(smem + (kc % F_STAGES) * TL::STAGE);
                const float* Pm = reinterpret_cast<const float*>(smem + (km % F_STAGES) * TL::STAGE);
                const float* Pp = reinterpret_cast<const float*>(smem + (kp % F_STAGES) * TL::STAGE);
                const float* O = reinterpret_cast<const float*>(smem + (kc % F_STAGES) * TL::STAGE + TL::PN_PAD);
                const int s0 = (cy + 1) * TL::HX + cx + TL::XOFF;
                const float4 c = *reinterpret_cast<const float4*>(P0 + s0);
                const float xm = P0[s0 - 1], xp = P0[s0 + 4];
                const float4 ym = *reinterpret_cast<const float4*>(P0 + s0 - TL::HX);
                const float4 yp = *reinterpret_cast<const float4*>(P0 + s0 + TL::HX);
                const float4 zm = *reinterpret_cast<const float4*>(Pm + s0);
                const float4 zp = *reinterpret_cast<const float4*>(Pp + s0);
                const float4 o = *reinterpret_cast<const float4*>(O + cy * TL::W + cx);
                __syncwarp();
                fence_async_smem();
                if (lane == 0) mbar_arrive(&empty[km % F_STAGES]);  // plane z-1 no longer read
                float4 v;
                v.x = slf_update(L2, CI, c.y, xm, yp.x, ym.x, zp.x, zm.x, c.x, o.x);
                v.y = slf_update(L2, CI, c.z, c.x, yp.y, ym.y, zp.y, zm.y, c.y, o.y);
                v.z = slf_update(L2, CI, c.w, c.y, yp.z, ym.z, zp.z, zm.z, c.z, o.z);
                v.w = slf_update(L2, CI, xp, c.z, yp.w, ym.w, zp.w, zm.w, c.w, o.w);
                bad |= !(fabsf(v.x) < 1e30f && fabsf(v.y) < 1e30f && fabsf(v.z) < 1e30f && fabsf(v.w) < 1e30f);
                if (yok) {
                    // cells owned by the boundary/PML kernels are left to them
                    const unsigned own =
                        f.owned && x <= a.g.nx - 2
                            ? (__ldg(f.owned + ((int64_t)z * a.g.ny + y) * f.owned_wpr + (x >> 5)) >> (x & 31)) & 0xFu
                            : 0u;
                    float* dst = pn + (int64_t)z * a.g.plane;
                    if (xfull && !own) {
                        __stcs(reinterpret_cast<float4*>(dst), v);
                    } else {
                        const float vv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                        for (int m = 0; m < 4; ++m)
                            if (x + m >= 1 && x + m <= a.g.nx - 2 && !((own >> m) & 1u)) dst[m] = vv[m];
                    }
                }
            }
        } else {
            // FP16: 8 cells per thread. p^n of planes z-1 and z stays in
            // registers from plane to plane: each plane loads and converts
            // only z+1, y+-1 and p^{n-1}. The update runs on stored values
            // of level g-1 (scale s_cur) and is rescaled once at the end.
            if (it.b != sc_b) {
                const StepScales sc = step_scales(a.f16, it.b, g);
                sc_rc = sc.s_new * sc.inv_cur;
                sc_ro = sc.s_cur * sc.inv_old;
                sc_ic = sc.inv_cur;
                sc_b = it.b;
            }
            const float rc = sc_rc, ro = sc_ro;
            uint32_t vmask[4];
#pragma unroll
            for (int w = 0; w < 4; ++w) {
                const int x0c = x + 2 * w;
                vmask[w] = (yok && x0c >= 1 && x0c <= a.g.nx - 2 ? 0x7fffu : 0u) |
                           (yok && x0c + 1 >= 1 && x0c + 1 <= a.g.nx - 2 ? 0x7fff0000u : 0u);
            }
            const int s0 = (cy + 1) * TL::HX + cx + TL::XOFF;
            const int so = cy * TL::W + cx;
            float ra[8], rb[8], rcv[8];
            uint4 wa, wb, wc;  // raw words of the rows in ra, rb, rcv
            {
                const __half* Pm = reinterpret_cast<const __half*>(smem + (k % F_STAGES) * TL::STAGE);
                const __half* P0 = reinterpret_cast<const __half*>(smem + ((k + 1) % F_STAGES) * TL::STAGE);
                wa = *reinterpret_cast<const uint4*>(Pm + s0);
                wb = *reinterpret_cast<const uint4*>(P0 + s0);
                cvt8(wa, ra);
                cvt8(wb, rb);
            }
            __syncwarp();
            fence_async_smem();
            if (lane == 0) mbar_arrive(&empty[k % F_STAGES]);  // plane z0-1 now in registers
            uint32_t amax = 0, omax = 0;
            // one plane: zm, c, zp rotate through ra, rb, rcv
            auto plane = [&](int pl, float (&zm)[8], float (&c)[8], float (&zp)[8], const uint4& cw,
                             uint4& zpw) -> bool {
                const int z = it.z0 + pl;
                const uint32_t kc = k + 1 + pl, kp = kc + 1;
                if (!mbar_wait(&full[kp % F_STAGES], (kp / F_STAGES) & 1)) return false;
                const __half* P0 = reinterpret_cast<const __half*>(smem + (kc % F_STAGES) * TL::STAGE);
                const __half* Pp = reinterpret_cast<const __half*>(smem + (kp % F_STAGES) * TL::STAGE);
                const __half* O =
                    reinterpret_cast<const __half*>(smem + (kc % F_STAGES) * TL::STAGE + TL::PN_PAD);
                const uint4 ymw = *reinterpret_cast<const uint4*>(P0 + s0 - TL::HX);
                const uint4 ypw = *reinterpret_cast<const uint4*>(P0 + s0 + TL::HX);
                zpw = *reinterpret_cast<const uint4*>(Pp + s0);
                const uint4 ow = *reinterpret_cast<const uint4*>(O + so);
                const float xm = __half2float(P0[s0 - 1]), xp = __half2float(P0[s0 + 8]);
                __syncwarp();
                fence_async_smem();
                if (lane == 0) mbar_arrive(&empty[kc % F_STAGES]);  // plane z read
                amax = __vmaxu2(amax, __vmaxu2(__vmaxu2(cw.x & vmask[0], cw.y & vmask[1]),
                                               __vmaxu2(cw.z & vmask[2], cw.w & vmask[3])));
                float ym[8], yp[8], o[8];
                cvt8(ymw, ym);
                cvt8(ypw, yp);
                cvt8(zpw, zp);
                cvt8(ow, o);
                uint32_t outw[4];
#pragma unroll
                for (int w = 0; w < 4; ++w) {
                    float v2[2];
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int m = 2 * w + h;
                        const float xl = m == 0 ? xm : c[m - 1];
                        const float xr = m == 7 ? xp : c[m + 1];
                        float s = xr + xl;
                        s = s + yp[m];
                        s = s + ym[m];
                        s = s + zp[m];
                        s = s + zm[m];
                        // c and o are decoded binary16 values (at most 11
                        // significant bits) and ro a power of two, so o * ro
                        // and 6 * c are exact: the fused forms round once,
                        // as the separate product and difference do
                        const float inc = __fmaf_rn(-o[m], ro, c[m]);   // c - o * ro
                        const float lap = __fmaf_rn(-6.0f, c[m], s);    // s - 6 c
                        v2[h] = (c[m] + (inc + L2 * lap)) * rc;
                    }
                    const __half2 hv = __floats2half2_rn(v2[0], v2[1]);
                    outw[w] = *reinterpret_cast<const uint32_t*>(&hv);
                    omax = __vmaxu2(omax, outw[w] & 0x7fff7fffu);
                }
                if (yok) {
                    const unsigned own =
                        f.owned && x <= a.g.nx - 2
                            ? (__ldg(f.owned + ((int64_t)z * a.g.ny + y) * f.owned_wpr + (x >> 5)) >> (x & 31)) & 0xFFu
                            : 0u;
                    __half* dst = pn + (int64_t)z * a.g.plane;
                    if (xfull && !own) {
                        __stcs(reinterpret_cast<uint4*>(dst), make_uint4(outw[0], outw[1], outw[2], outw[3]));
                    } else {
#pragma unroll
                        for (int m = 0; m < 8; ++m)
                            if (x + m >= 1 && x + m <= a.g.nx - 2 && !((own >> m) & 1u))
                                reinterpret_cast<unsigned short*>(dst)[m] =
                                    (unsigned short)(outw[m >> 1] >> (16 * (m & 1)));
                    }
                }
                return true;
            };
            bool ok = true;
            for (int pl = 0; pl < planes && ok; pl += 3) {
                ok = plane(pl, ra, rb, rcv, wb, wc);
                if (ok && pl + 1 < planes) ok = plane(pl + 1, rb, rcv, ra, wc, wa);
                if (ok && pl + 2 < planes) ok = plane(pl + 2, rcv, ra, rb, wa, wb);
            }
            if (!ok) {
                if (lane == 0) atomicOr(a.flag, 2);
                return;
            }
            // the plane z1 loaded last is the next item's halo: release it
            // together with the others below
            const uint32_t gmax = __reduce_max_sync(0xffffffffu, max(amax & 0xffffu, amax >> 16));
            if (lane == 0 && gmax) {
                const float mv = __half2float(__ushort_as_half((unsigned short)gmax)) * sc_ic;
                atomicMax(a.f16.mx + (size_t)it.b * 5 + max_slot(g - 1), __float_as_uint(mv));
            }
            // a stored binary16 infinity or NaN (magnitude bits >= 0x7c00)
            // in a grid-interior cell means the field left the range
            const uint32_t om = max(omax & 0xffffu, omax >> 16);
            bad = om >= 0x7c00u;
            __syncwarp();
            fence_async_smem();
            if (lane == 0) mbar_arrive(&empty[(k + planes + 1) % F_STAGES]);
            if (__any_sync(0xffffffffu, bad && yok && x <= a.g.nx - 2) && lane == 0) atomicOr(a.flag, 1);
            k += (uint32_t)planes + 2;
            continue;
        }
        __syncwarp();
        fence_async_smem();
        if (lane == 0) {
            mbar_arrive(&empty[(k + planes) % F_STAGES]);
            mbar_arrive(&empty[(k + planes + 1) % F_STAGES]);
        }
        if (__any_sync(0xffffffffu, bad && yok && x <= a.g.nx - 2) && lane == 0) atomicOr(a.flag, 1);
        k += (uint32_t)planes + 2;
    }
}

// Host view of a streaming-kernel instance: tile width and height in cells,
// halo box width, shared memory per block and the kernel. FP16 storage has
// no 128x8 instance: its halo box would be 272 cells wide, past the 256 a
// TMA box allows.
struct StreamShape {
    int w, h, hx, threads;
    size_t smem;
    const void* kern;
};
template <typename T, int S, bool TAIL = false>
static StreamShape stream_shape_t() {
    using TL = Tile<T, S>;
    static_assert(TL::HX <= 256 && TL::H + 2 <= 256, "TMA box dimensions are at most 256");
    return StreamShape{TL::W, TL::H, TL::HX, TAIL ? F_THREADS + 32 * kTailWarps : F_THREADS, TL::SMEM,
                       (const void*)k_stream<T, S, TAIL>};
}
static bool shape_valid(bool f16, int S) { return S >= 0 && S < kTileShapes && !(f16 && S == 1); }
// tail: the instance with tail warps (FP32 storage only)
static StreamShape stream_shape(bool f16, int S, bool tail = false) {
    if (f16) return S == 2 ? stream_shape_t<__half, 2>() : stream_shape_t<__half, 0>();
    if (tail)
        return S == 1 ? stream_shape_t<float, 1, true>()
                      : (S == 2 ? stream_shape_t<float, 2, true>() : stream_shape_t<float, 0, true>());
    return S == 1 ? stream_shape_t<float, 1>() : (S == 2 ? stream_shape_t<float, 2>() : stream_shape_t<float, 0>());
}
template <typename T>
static void launch_stream(int S, bool tail, int grid, cudaStream_t st, const CUtensorMap& th, const CUtensorMap& to,
                          const StepArgs& a, const FusedDev& f, int j) {
    if constexpr (sizeof(T) == 2) {
        if (S == 2) k_stream<T, 2><<<grid, F_THREADS, Tile<T, 2>::SMEM, st>>>(th, to, a, f, j);
        else k_stream<T, 0><<<grid, F_THREADS, Tile<T, 0>::SMEM, st>>>(th, to, a, f, j);
    } else if (tail) {
        constexpr int TT = F_THREADS + 32 * kTailWarps;
        if (S == 1) k_stream<T, 1, true><<<grid, TT, Tile<T, 1>::SMEM, st>>>(th, to, a, f, j);
        else if (S == 2) k_stream<T, 2, true><<<grid, TT, Tile<T, 2>::SMEM, st>>>(th, to, a, f, j);
        else k_stream<T, 0, true><<<grid, TT, Tile<T, 0>::SMEM, st>>>(th, to, a, f, j);
    } else {
        if (S == 1) k_stream<T, 1><<<grid, F_THREADS, Tile<T, 1>::SMEM, st>>>(th, to, a, f, j);
        else if (S == 2) k_stream<T, 2><<<grid, F_THREADS, Tile<T, 2>::SMEM, st>>>(th, to, a, f, j);
        else k_stream<T, 0><<<grid, F_THREADS, Tile<T, 0>::SMEM, st>>>(th, to, a, f, j);
    }
}

// Scale and inverse scale of level g for member b (1 for FP32 storage).
template <typename T>
__device__ __forceinline__ float2 new_level_scale(const StepArgs& a, int b, long long g) {
    if constexpr (sizeof(T) == 4) {
        return make_float2(1.0f, 1.0f);
    } else {
        const int k = level_scale_exp(ld_slot(a.f16.mx + (size_t)b * 5 + max_slot(g - 2)), __ldg(a.f16.src_max + b));
        return make_float2(pow2_exact(k), pow2_exact(-k));
    }
}

// source.cl:32-40 then mic.cl:32-41 for one batch member per block.
// Sources landing on one cell are added in insertion order.
template <typename T>
__global__ void k_src_rcv(StepArgs a, int j, int do_src, int do_rcv) {
    const long long g = *a.d_step + j;
    const TlMark tl(a, 6, g, blockIdx.x == 0);
    const int b = blockIdx.x;
    T* pn = level_ptr<T>(a, buf_new(g)) + (size_t)b * a.g.vol;
    const float2 sc = new_level_scale<T>(a, b, g);
    if (do_src && threadIdx.x == 0) {
        for (int s = a.src.begin[b]; s < a.src.begin[b + 1]; ++s) {
            const float v = (g < a.src.len[s]) ? a.src.data[a.src.off[s] + g] : 0.0f;
            T* c = pn + a.src.cell[s];
            fst(c, fld(c, sc.y) + v, sc.x);
        }
    }
    __syncthreads();
    if (!do_rcv) return;
    for (int r = threadIdx.x; r < a.rcv.n; r += blockDim.x) {
        const float v = fld(pn + a.rcv.cell[r], sc.y);
        a.rcv.out[((size_t)b * a.rcv.n + r) * a.rcv.cap + g] = v;
        if constexpr (sizeof(T) == 4) watch(a.flag, v);
        else if (!f16_finite(v * sc.x)) atomicOr(a.flag, 1);
    }
}

// Sources and receivers with their cells passed as kernel parameters (no
// dependent metadata loads): source.cl:32-40 then mic.cl:32-41.
constexpr int kInlineSrc = 64, kInlineRcv = 256;
struct SrcRcvInline {
    int32_t n_src, n_rcv;
    int32_t src_cell[kInlineSrc];
    int32_t src_batch[kInlineSrc];
    int64_t src_len[kInlineSrc];
    const float* src_ptr[kInlineSrc];
    int32_t rcv_cell[kInlineRcv];
};

template <typename T>
__global__ void k_src_rcv_inline(const __grid_constant__ StepArgs a, const __grid_constant__ SrcRcvInline q,
                                 int j) {
    const long long g = *a.d_step + j;
    const TlMark tl(a, 6, g, blockIdx.x == 0);
    const int b = blockIdx.x;
    T* pn = level_ptr<T>(a, buf_new(g)) + (size_t)b * a.g.vol;
    const float2 sc = new_level_scale<T>(a, b, g);
    if (threadIdx.x == 0) {
        for (int s = 0; s < q.n_src; ++s) {
            if (q.src_batch[s] != b) continue;
            const float v = (g < q.src_len[s]) ? __ldg(q.src_ptr[s] + g) : 0.0f;
            T* c = pn + q.src_cell[s];
            fst(c, fld(c, sc.y) + v, sc.x);
        }
    }
    __syncthreads();
    for (int r = threadIdx.x; r < q.n_rcv; r += blockDim.x) {
        const float v = fld(pn + q.rcv_cell[r], sc.y);
        a.rcv.out[((size_t)b * q.n_rcv + r) * a.rcv.cap + g] = v;
        if constexpr (sizeof(T) == 4) watch(a.flag, v);
        else if (!f16_finite(v * sc.x)) atomicOr(a.flag, 1);
    }
}

// Headless visualisation: copy_plane.cl:29-34 (the y plane of the newest
// level, copied after every third step of a run by simulation.hpp:393-400)
// for any axis, into a device ring of frames. Runs after the step's source
// and receiver updates; copies when the run-local step index is a multiple
// of `every` (decided on the device, so one graph serves every chunk).
struct CaptureDev {
    int32_t batch, axis, index, every, max_frames, rows, cols;
    float* frames;             // [max_frames][rows][cols]
    long long* frame_step;     // [max_frames] global step of each frame
    const long long* run0;     // [0] global step at the start of the run, [1] frames captured before it
};

template <typename T>
__global__ void k_capture(const __grid_constant__ StepArgs a, const CaptureDev c, int j) {
    const long long g = *a.d_step + j;
    const long long i = g - c.run0[0];
    if (i % c.every) return;
    const long long n = c.run0[1] + i / c.every;
    const int slot = (int)(n % c.max_frames);
    const float2 sc = new_level_scale<T>(a, c.batch, g);
    const T* p = level_ptr<T>(a, buf_new(g)) + (size_t)c.batch * a.g.vol;
    float* out = c.frames + (size_t)slot * c.rows * c.cols;
    const int total = c.rows * c.cols;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
        const int r = e / c.cols, q = e % c.cols;
        int64_t idx;
        if (c.axis == 0) idx = (int64_t)r * a.g.plane + (int64_t)q * a.g.pitch + c.index;        // [nz][ny] at x
        else if (c.axis == 1) idx = (int64_t)r * a.g.plane + (int64_t)c.index * a.g.pitch + q;   // [nz][nx] at y
        else idx = (int64_t)c.index * a.g.plane + (int64_t)r * a.g.pitch + q;                    // [ny][nx] at z
        out[e] = fld(p + idx, sc.y);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) c.frame_step[slot] = g;
}

__global__ void k_advance(long long* d_step, int n) { *d_step += n; }

// Solid cell of the model (cells outside the model or the grid are air).
__device__ __forceinline__ bool cell_solid(const SolidBits& s, int x, int y, int z) {
    if (!s.bits || x < 0 || y < 0 || z < 0 || x >= s.nx || y >= s.ny || z >= s.nz) return false;
    return (__ldg(s.bits + ((int64_t)z * s.ny + y) * s.w + (x >> 5)) >> (x & 31)) & 1u;
}

// Walls of a cell: bit d set when its neighbour in direction d (x+, x-, y+,
// y-, z+, z-) is solid.
__device__ __forceinline__ unsigned wall_bits(const SolidBits& s, int x, int y, int z) {
    return (unsigned)cell_solid(s, x + 1, y, z) | (unsigned)cell_solid(s, x - 1, y, z) << 1 |
           (unsigned)cell_solid(s, x, y + 1, z) << 2 | (unsigned)cell_solid(s, x, y - 1, z) << 3 |
           (unsigned)cell_solid(s, x, y, z + 1) << 4 | (unsigned)cell_solid(s, x, y, z - 1) << 5;
}

// 1/2 for every axis among `axes_mask` (two bits per axis) that has a bit set.
__device__ __forceinline__ double half_per_axis(unsigned m, int skip_axis) {
    double w = 1.0;
#pragma unroll
    for (int b = 0; b < 3; ++b)
        if (b != skip_axis && ((m >> (2 * b)) & 3u)) w *= 0.5;
    return w;
}

// Discrete SLF energy between the two latest levels u1 (newest) and u0, in
// FP64, over the air cells 1..n-2: 1/2 sum w_i (u1_i-u0_i)^2 + lambda2/2 sum
// over edges between air cells of w_e (u1_i-u1_j)(u0_i-u0_j) (edges to the
// fixed outer faces included once). A boundary cell's update mirrors its
// neighbour across each wall, which makes it a half cell per walled axis:
// w_i = 1/2 per axis with a wall, and an edge lying along walls takes 1/2
// for each other axis on which both ends have the same wall. With walls of
// frequency-independent admittance beta >= 0 around a convex air region the
// energy changes by minus the wall loss each step (non-increasing; constant
// for rigid walls); without a model every cell is air and every weight 1.
template <typename T>
__global__ void k_energy(const T* u1_, const T* u0_, float inv1, float inv0, GridDev g, SolidBits sb,
                         double lambda2, double* out) {
    auto u1 = [&](int64_t k) { return (double)fld(u1_ + k, inv1); };
    auto u0 = [&](int64_t k) { return (double)fld(u0_ + k, inv0); };
    const int x = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int y = 1 + blockIdx.y * blockDim.y + threadIdx.y;
    const int z = 1 + blockIdx.z;
    double acc = 0.0;
    if (x <= g.nx - 2 && y <= g.ny - 2 && !cell_solid(sb, x, y, z)) {
        const int64_t i = (int64_t)z * g.plane + (int64_t)y * g.pitch + x;
        const unsigned mi = wall_bits(sb, x, y, z);
        const double d = u1(i) - u0(i);
        acc = 0.5 * half_per_axis(mi, -1) * d * d;
        const int64_t off[3] = {1, g.pitch, g.plane};
        const int c[3] = {x, y, z};
        double pot = 0.0;
        for (int ax = 0; ax < 3; ++ax) {
            for (int sgn = 1; sgn >= -1; sgn -= 2) {
                if (sgn < 0 && c[ax] != 1) break;  // the low edge only toward the outer face
                int q[3] = {x, y, z};
                q[ax] += sgn;
                if (cell_solid(sb, q[0], q[1], q[2])) continue;
                const int64_t j = i + sgn * off[ax];
                const double we = half_per_axis(mi & wall_bits(sb, q[0], q[1], q[2]), ax);
                pot += we * (u1(i) - u1(j)) * (u0(i) - u0(j));
            }
        }
        acc += 0.5 * lambda2 * pot;
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, acc);
}

// FP16 level -> FP32 values (reads of the field by the host).
__global__ void k_decode(const __half* in, float* out, int64_t n, float inv) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = __half2float(in[i]) * inv;
}

// ---------------------------------------------------------------------------
// Engine implementation
// ---------------------------------------------------------------------------
namespace {

void check_cell(const int32_t ijk[3], int32_t nx, int32_t ny, int32_t nz, const char* what) {
    if (ijk[0] < 0 || ijk[0] >= nx || ijk[1] < 0 || ijk[1] >= ny || ijk[2] < 0 || ijk[2] >= nz) {
        char buf[200];
        std::snprintf(buf, sizeof buf, "%s cell (%d,%d,%d) lies outside the %dx%dx%d grid", what,
                      ijk[0], ijk[1], ijk[2], nx, ny, nz);
        throw Error(AFD_ERR_ARG, buf);
    }
}

}  // namespace

struct Source {
    int32_t batch;
    int32_t ijk[3];
    std::vector<float> sig;
};

struct Engine::Impl {
    afd_params prm{};
    // geometry
    bool have_model = false;
    Model model;  // dimensions, materials and filters; the voxels stay on the device
    DBuf<uint32_t> model_solid;  // solid cells of the model, rows of row_words(model.nx) words
    std::vector<BoundaryPoint> boundary;
    int64_t boundary_counts[kNumGroups] = {};  // points per group, counted when the list is set
    int32_t min_size[3] = {0, 0, 0};
    int32_t nx = 0, ny = 0, nz = 0;
    int64_t pitch = 0, plane = 0, vol = 0;
    bool initialized = false;
    int64_t group_counts[kNumGroups] = {};
    // PML configuration (applied at the next run)
    int32_t pml_width = 0;
    uint32_t pml_faces = 0;
    std::vector<float> ksi[3];
    bool pml_dirty = false;
    int64_t pml_g0 = 0;
    // sources / receivers
    std::vector<Source> sources;
    std::vector<std::array<int32_t, 3>> receivers;
    bool src_dirty = true;
    int64_t steps_done = 0;

    // device state
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    DBuf<float> fields;  // 3 * batch * vol values (FP32, or FP16 in half the floats)
    DBuf<uint32_t> f16_mx;   // FP16 storage: level maxima [batch][5]
    DBuf<float> f16_smax;    // FP16 storage: largest |source sample| per member
    std::vector<float> smax_host;
    DBuf<float> decoded;     // FP16 storage: one decoded level for host reads
    DBuf<int32_t> lrs_cell;
    DBuf<uint32_t> lrs_info;
    DBuf<float> lrs_in, lrs_out;
    DBuf<float> coef_a, coef_b;
    DBuf<float> fi[3][2], psi[2];
    DBuf<float> ksi_dev[3];
    std::vector<PmlBox> pml_boxes;
    std::vector<PmlBox> pml_axis_boxes[3];
    // the launches over all pressure boxes and over all (axis, slab box) pairs
    BoxLaunch pml_p_all{}, pml_aux_all{};
    // z-slab of a larger grid (slab_nz > 0): local plane z is global plane
    // z + slab_z0 of slab_nz planes; planes 0 and nz-1 are halos filled by
    // the caller between step phases
    int32_t slab_z0 = 0, slab_nz = 0;
    int step_phase = 0;       // 0: whole steps; 1, 2: the halves of a split step
    bool phase_open = false;  // the first half of a split step has run
    int pml_p_blocks = 0, pml_aux_blocks = 0;
    int pml_zc = 2;  // planes each PML thread marches
    int64_t pml_units = 0;
    int64_t n_pml_cells = 0;
    DBuf<int32_t> src_cell, src_begin;
    DBuf<int64_t> src_off, src_len;
    DBuf<float> src_data;
    DBuf<int32_t> rcv_cell;
    DBuf<float> rcv_out;
    int64_t rcv_cap = 0;
    int32_t rcv_n_dev = 0;
    DBuf<long long> d_step;
    // headless visualisation (afd_set_capture)
    int32_t cap_batch = 0, cap_axis = 1, cap_index = 0, cap_every = 0, cap_max = 0;
    bool cap_dirty = false;
    int64_t cap_total = 0;  // frames captured so far
    DBuf<float> cap_frames;
    DBuf<long long> cap_steps, cap_run0;
    // step timeline (afd_set_timeline)
    DBuf<unsigned long long> tl_start, tl_end;
    long long tl_first = 0;
    int32_t tl_steps = 0;
    bool tl_dirty = false;
    CaptureDev cap{};
    void advance_done(int64_t n) {
        if (cap_every > 0 && n > 0) cap_total += (n + cap_every - 1) / cap_every;
        steps_done += n;
    }
    void plane_dims(int32_t axis, int64_t* rows, int64_t* cols) const {
        if (axis == 0) { *rows = nz; *cols = ny; }
        else if (axis == 1) { *rows = nz; *cols = nx; }
        else { *rows = ny; *cols = nx; }
    }
    DBuf<int> d_flag;
    DBuf<double> d_energy;

    // fused step plan
    FusedDev fdev{};
    DBuf<int4> f_offs;
    DBuf<int> f_work;
    DBuf<unsigned long long> f_tail;  // tail-warp counters, one per step of a chunk
    // compact work lists of the streaming kernel (FIXED scheme), one per plan
    struct PlanItems {
        std::array<int64_t, 7> key{{-1, -1, -1, -1, -1, -1, -1}};
        int64_t n = -1;  // -1: every item
        DBuf<int> buf;
    };
    std::map<int, PlanItems> plan_items;
    // FIXED scheme: 1 bit per cell (rows of pitch / 32 words) for the
    // boundary cells, the PML cells, and their union: the cells whose new
    // value comes from the boundary or PML kernels, which the streaming
    // kernel then skips so that those kernels can run beside it
    DBuf<uint32_t> lrs_bits, pml_owned, owned;
    bool owned_dirty = true;
    // streaming plan: tile shape (0: 64x16, 1: 128x8, 2: 32x32 cells for
    // FP32 storage), resident blocks per SM (0: as many as fit) and z-chunk
    // depth (0: the rule in build_fused); the online autotuner picks them
    struct Plan {
        int per_sm, dz;
        bool beside;  // boundary and PML pressure kernels beside the streaming kernel
        int shape;
        bool tail;    // boundary and PML pressure work in the streaming kernel's tail warps
    };
    Plan plan{0, 0, false, 0, false};
    std::vector<Plan> tune_cands;
    std::vector<float> tune_ms;
    size_t tune_next = 0;
    bool tuned = false;
    int plan_id = 0;             // index of `plan` in tune_cands (graph cache key), 0 before tuning
    int64_t tune_gen = -1;       // model_gen the candidates were made for
    cudaEvent_t tev0 = nullptr, tev1 = nullptr;
    bool tune_active() const { return use_fused() && prm.graphs && !prm.profile && !tuned; }
    void apply_plan(int id) {
        plan = id == 0 ? Plan{0, 0, false, 0, false} : tune_cands[(size_t)id - 1];
        plan_id = id;
        fused_dirty = true;
        build_fused();
    }
    // candidates: for each tile shape the streaming kernel with all resident
    // blocks per SM and z-chunk depth {rule, rule / 4} (and rule / 2 for the
    // 64x16 tile), followed by the boundary and PML kernels; every candidate
    // gives the results of the serial order. Made once per model and grid
    // (the plan then restarts from the default).
    void ensure_candidates() {
        if (use_fused() && tune_gen != model_gen) {
            make_candidates();
            apply_plan(forced ? 1 : 0);
        }
    }
    // a plan fixed by afd_set_plan: the only candidate, tuning off
    bool forced = false;
    Plan forced_plan{0, 0, false, 0, false};
    // resident blocks per SM that fit and the z-chunk depth rule of a shape
    void shape_limits(int shape, bool tail, int* per_sm_max, int* dz_rule);
    void make_candidates() {
        tune_cands.clear();
        if (forced) {
            tune_cands.push_back(forced_plan);
            tune_ms.assign(1, 0.0f);
            tune_next = 1;
            tuned = true;
            tune_gen = model_gen;
            return;
        }
        auto add = [&](int ps, int d, bool bs, int sh, bool tl) {
            if (ps < 1 || d < 8) return;
            for (const Plan& q : tune_cands)
                if (q.per_sm == ps && q.dz == d && q.beside == bs && q.shape == sh && q.tail == tl) return;
            tune_cands.push_back(Plan{ps, d, bs, sh, tl});
        };
        for (int sh = 0; sh < kTileShapes; ++sh) {
            if (!shape_valid(f16(), sh)) continue;
            int ps = 0, rule = 0;
            shape_limits(sh, false, &ps, &rule);
            add(ps, rule, false, sh, false);
            if (sh == 0) add(ps, rule / 2, false, sh, false);
            add(ps, rule / 4, false, sh, false);
            // the beside and tail-warp orders (afd_set_plan) give the same
            // results but measured slower on every workload here, so the
            // tuner does not spend chunks on them
        }
        tune_ms.assign(tune_cands.size(), 0.0f);
        tune_next = 0;
        tuned = false;
        tune_gen = model_gen;
    }
    std::vector<uint8_t> air_flags;  // [z][tile] air within the widened footprint (per model and tiling)
    SolidBits solid_view() const {
        SolidBits sb;
        if (have_model && model_solid.ptr) {
            sb.bits = model_solid.ptr;
            sb.nx = model.nx;
            sb.ny = model.ny;
            sb.nz = model.nz;
            sb.w = row_words(model.nx);
        }
        return sb;
    }
    std::array<int64_t, 5> flags_key{{-1, -1, -1, -1, -1}};
    int64_t model_gen = 0;  // counts init_device calls (a new model or grid)
    CUtensorMap tm_halo{}, tm_own{};
    int fused_grid = 0;
    int max_per_sm = 0, rule_dz = 0, stream_per_sm = 0;
    bool fused_dirty = true;
    int tiles_x = 0, tiles_y = 0, tile_w = 0, tile_h = 0;

    StepArgs args{};
    SrcRcvInline inl{};
    bool inline_ok = false;
    bool src_beside_aux = false;  // see build_args
    std::map<int64_t, cudaGraphExec_t> graphs;
    double last_ms = 0.0;
    int64_t launches = 0;
    std::vector<KernelStat> kstats;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_pool;
    std::vector<int> ev_kind;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;

    bool ref() const { return prm.mode == AFD_MODE_REF; }
    bool f16() const { return prm.storage == AFD_STORE_FP16; }
    // scale of level L of member b from the device maxima (host copy of the
    // rule the kernels apply)
    float host_level_scale(int32_t b, long long L) {
        uint32_t m = 0;
        float smax = 0.0f;
        CK(cudaMemcpy(&m, f16_mx.ptr + (size_t)b * 5 + max_slot(L - 2), 4, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(&smax, f16_smax.ptr + b, 4, cudaMemcpyDeviceToHost));
        return level_scale(m, smax);
    }
    float lambda2() const {
        const float t = prm.dt * prm.c / prm.dx;
        return t * t;
    }
    void drop_graphs() {
        for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
        graphs.clear();
    }
    void grid_dims(int32_t dims[3]) const {
        if (initialized) {
            dims[0] = nx;
            dims[1] = ny;
            dims[2] = nz;
            return;
        }
        const int32_t md[3] = {have_model ? model.nx : 0, have_model ? model.ny : 0,
                               have_model ? model.nz : 0};
        for (int k = 0; k < 3; ++k) dims[k] = std::max(md[k], min_size[k]);
    }

    void init_device();
    void adopt_model(Model&& hdr, const int32_t* d_vox);
    // page-locked host staging for strided device-to-host copies, grown on
    // demand and kept for the engine's life
    float* pinned = nullptr;
    size_t pinned_n = 0;
    float* pinned_floats(size_t n) {
        if (n > pinned_n) {
            if (pinned) cudaFreeHost(pinned);
            pinned = nullptr;
            pinned_n = 0;
            CK(cudaHostAlloc((void**)&pinned, n * sizeof(float), cudaHostAllocDefault));
            pinned_n = n;
        }
        return pinned;
    }
    void build_fused();
    void encode_maps(int shape);
    int maps_shape = -1;  // shape of tm_halo / tm_own (-1: none yet for these buffers)
    bool use_fused() const { return prm.fused != 0; }
    // FIXED scheme in graphs: the boundary and PML pressure kernels run
    // beside the streaming kernel (which skips the cells they own)
    bool lists_beside() const {
        return plan.beside && !ref() && use_fused() && prm.graphs && !prm.profile && owned.ptr;
    }
    // FIXED scheme, FP32 storage: the boundary and PML pressure updates run
    // in the streaming kernel's tail warps (with or without graphs)
    bool tail_active() const { return plan.tail && !plan.beside && !ref() && !f16() && use_fused() && owned.ptr; }
    // (FT_X x FT_Y tile, plane) of a cell, in tile-major order
    int64_t tile_key(int x, int y, int z) const {
        return ((int64_t)(y / FT_Y) * ((nx + FT_X - 1) / FT_X) + x / FT_X) * nz + z;
    }
    void setup_pml();
    void upload_sources();
    void ensure_receivers(int64_t t_end);
    void build_args();
    void launch_step(int j, bool profile);
    // Runs independent launches concurrently: the first on `stream`, the
    // others on side streams forked from it and joined back to it.
    std::vector<cudaStream_t> side;
    std::vector<cudaEvent_t> side_ev;
    cudaEvent_t fork_ev = nullptr;
    void run_side_by_side(const std::vector<std::function<void(cudaStream_t)>>& work) {
        if (work.empty()) return;
        const size_t extra = std::min<size_t>(work.size() - 1, 4);
        while (side.size() < extra) {
            cudaStream_t s;
            cudaEvent_t e;
            CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
            CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            side.push_back(s);
            side_ev.push_back(e);
        }
        if (!fork_ev) CK(cudaEventCreateWithFlags(&fork_ev, cudaEventDisableTiming));
        if (extra) {
            CK(cudaEventRecord(fork_ev, stream));
            for (size_t k = 0; k < extra; ++k) CK(cudaStreamWaitEvent(side[k], fork_ev, 0));
        }
        for (size_t w = 0; w < work.size(); ++w) work[w](w == 0 ? stream : side[(w - 1) % std::max<size_t>(extra, 1)]);
        for (size_t k = 0; k < extra; ++k) {
            CK(cudaEventRecord(side_ev[k], side[k]));
            CK(cudaStreamWaitEvent(stream, side_ev[k], 0));
        }
    }
    template <typename T>
    void launch_step_t(int j, bool profile);
    int64_t kernels_per_step() const;
    void launch_step_count_only(int64_t n) { launches += kernels_per_step() * n + 1; }
    cudaGraphExec_t graph_for(int64_t n);
    void run_chunk(int64_t n);
    void setup_run(int64_t steps);
    void build_owned_mask();
    void collect_profile();
};

// Simulation::Init (simulation.hpp:201-231) plus the device copy of
// LrsData (lrs-data.hpp:116-215): fixes the grid, allocates the three
// pressure levels and uploads the compact boundary list.
void Engine::Impl::init_device() {
    int32_t dims[3];
    grid_dims(dims);
    if (dims[0] < 3 || dims[1] < 3 || dims[2] < 3)
        throw Error(AFD_ERR_STATE, "no grid: load a model or set minsize before run");
    nx = dims[0];
    ny = dims[1];
    nz = dims[2];
    pitch = ((int64_t)nx + 31) / 32 * 32;
    plane = pitch * ny;
    vol = plane * nz;
    if (vol * 3 > (int64_t)1 << 31 && vol > ((int64_t)1 << 31) - 1)
        throw Error(AFD_ERR_ARG, "grid too large for 32-bit cell indices");
    CK(cudaSetDevice(device));
    fields.alloc((size_t)vol * 3 * prm.batch / (f16() ? 2 : 1));  // vol is a multiple of 32
    if (f16()) {
        f16_mx.alloc((size_t)prm.batch * 5);
        if (!f16_smax.ptr) f16_smax.alloc((size_t)prm.batch);
    }

    // boundary list, sorted by (tile, plane, position in tile) so that the
    // boundary kernel's neighbour reads stay local; every order gives the
    // same results. The list arrives in z-y-x scan order, in which the cells
    // of one tile and plane already come by position in the tile, so a
    // stable counting sort by tile_key suffices.
    {
        const int64_t nkey = (int64_t)((ny + FT_Y - 1) / FT_Y) * ((nx + FT_X - 1) / FT_X) * nz;
        std::vector<int64_t> start((size_t)nkey + 1, 0);
        for (const BoundaryPoint& b : boundary) start[(size_t)tile_key(b.x, b.y, b.z) + 1]++;
        for (int64_t k = 0; k < nkey; ++k) start[(size_t)k + 1] += start[(size_t)k];
        std::vector<BoundaryPoint> sorted(boundary.size());
        for (const BoundaryPoint& b : boundary) sorted[(size_t)start[(size_t)tile_key(b.x, b.y, b.z)]++] = b;
        boundary.swap(sorted);
    }
    std::vector<int32_t> cell;
    std::vector<uint32_t> info;
    std::fill(group_counts, group_counts + kNumGroups, 0);
    for (const BoundaryPoint& b : boundary) {
        cell.push_back((int32_t)(b.z * plane + b.y * pitch + b.x));
        uint32_t w = (uint32_t)b.group;
        for (int f = 0; f < 3; ++f)
            if (b.mat[f] >= 0) w |= (uint32_t)b.mat[f] << (5 + 8 * f);
        info.push_back(w);
        group_counts[b.group]++;
    }
    lrs_cell.upload(cell);
    lrs_info.upload(info);
    lrs_bits.alloc((size_t)nz * ny * (pitch / 32), false);
    boundary_bits_device(lrs_cell.ptr, (int64_t)cell.size(), (int64_t)lrs_bits.n, lrs_bits.ptr, stream);
    CK(cudaStreamSynchronize(stream));
    const int K = have_model ? model.ncoef : 1;
    const size_t S = 3 * (size_t)K;
    lrs_in.alloc(cell.size() * S * prm.batch);
    lrs_out.alloc(cell.size() * S * prm.batch);
    if (have_model) {
        coef_a.upload(model.a);
        coef_b.upload(model.b);
    }
    maps_shape = -1;  // the tensor maps cover the new field buffers once build_fused encodes them
    initialized = true;
    fused_dirty = true;
    owned_dirty = true;
    ++model_gen;
}

// The owned-cell mask of the FIXED scheme: boundary cells and PML cells.
void Engine::Impl::build_owned_mask() {
    owned.release();
    owned_dirty = false;
    fused_dirty = true;
    if (ref()) return;
    if (n_pml_cells == 0 && boundary.empty()) return;
    const size_t words = (size_t)nz * ny * (pitch / 32);
    owned.alloc(words, false);
    or_masks_device(pml_owned.n == words ? pml_owned.ptr : nullptr, lrs_bits.ptr, owned.ptr, (int64_t)words, stream);
    CK(cudaStreamSynchronize(stream));
}

// Tensor maps over the three field levels seen as one stack of
// 3 * batch * nz planes: the halo box of p^n and the own box of p^{n-1} of
// a tile of the given shape.
void Engine::Impl::encode_maps(int shape) {
    typedef CUresult (*EncodeFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    CK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
    if (!fn || q != cudaDriverEntryPointSuccess) throw Error(AFD_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    EncodeFn enc = (EncodeFn)fn;
    const StreamShape sh = stream_shape(f16(), shape);
    const cuuint64_t es = f16() ? 2 : 4;
    const CUtensorMapDataType dt = f16() ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    const cuuint64_t dims[3] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)(3 * prm.batch * nz)};
    const cuuint64_t strides[2] = {(cuuint64_t)pitch * es, (cuuint64_t)plane * es};
    const cuuint32_t box_h[3] = {(cuuint32_t)sh.hx, (cuuint32_t)(sh.h + 2), 1},
                     box_o[3] = {(cuuint32_t)sh.w, (cuuint32_t)sh.h, 1}, estr[3] = {1, 1, 1};
    CUresult r1 = enc(&tm_halo, dt, 3, fields.ptr, dims, strides, box_h, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                      CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    CUresult r2 = enc(&tm_own, dt, 3, fields.ptr, dims, strides, box_o, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                      CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r1 != CUDA_SUCCESS || r2 != CUDA_SUCCESS) throw Error(AFD_ERR_CUDA, "tensor map encoding failed");
    maps_shape = shape;
}

// z-chunk depth: enough work items for every resident block to take a few,
// with the two halo planes a small share of each chunk.
static int chunk_rule(int64_t tiles, int nz, int64_t resident) {
    int dz = 64;
    while (dz > 8 && tiles * ((nz - 2 + dz - 1) / dz) < 4 * resident) dz /= 2;
    return dz;
}

void Engine::Impl::shape_limits(int shape, bool tail, int* per_sm_max, int* dz_rule) {
    const StreamShape sh = stream_shape(f16(), shape, tail);
    int per_sm = 0, sms = 0;
    CK(cudaFuncSetAttribute(sh.kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh.smem));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sh.kern, sh.threads, sh.smem));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    per_sm = std::max(per_sm, 1);
    const int64_t tiles = (int64_t)((nx + sh.w - 1) / sh.w) * ((ny + sh.h - 1) / sh.h) * prm.batch;
    *per_sm_max = per_sm;
    *dz_rule = chunk_rule(tiles, nz, (int64_t)per_sm * sms);
}

// Work decomposition of the streaming kernel: tiles, z-chunk depth and the
// persistent grid size.
void Engine::Impl::build_fused() {
    FusedDev& F = fdev;
    F = FusedDev{};
    if (!shape_valid(f16(), plan.shape)) plan.shape = 0;
    const StreamShape sh = stream_shape(f16(), plan.shape, tail_active());
    tile_w = sh.w;
    tile_h = sh.h;
    tiles_x = (nx + sh.w - 1) / sh.w;
    tiles_y = (ny + sh.h - 1) / sh.h;
    if (maps_shape != plan.shape) encode_maps(plan.shape);
    F.tiles_x = tiles_x;
    F.tiles_y = tiles_y;
    int per_sm = 0;
    CK(cudaFuncSetAttribute(sh.kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh.smem));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sh.kern, sh.threads, sh.smem));
    int sms = 0;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    max_per_sm = std::max(per_sm, 1);
    if (plan.per_sm > 0) per_sm = std::min(per_sm, plan.per_sm);
    stream_per_sm = std::max(per_sm, 1);
    const int64_t resident = (int64_t)stream_per_sm * sms;
    F.owned = lists_beside() || tail_active() ? owned.ptr : nullptr;
    F.owned_wpr = (int32_t)(pitch / 32);
    if (!f_tail.ptr) f_tail.alloc(256);
    F.tail = f_tail.ptr;
    const int64_t tiles = (int64_t)tiles_x * tiles_y * prm.batch;
    int dz = chunk_rule(tiles, nz, resident);
    rule_dz = dz;
    if (plan.dz > 0) dz = plan.dz;
    F.dz = dz;
    F.n_chunks = (nz - 2 + dz - 1) / dz;
    if (!f_work.ptr) f_work.alloc(256);
    F.work = f_work.ptr;
    int64_t n_items = tiles * F.n_chunks;
    // FIXED scheme: no air cell reads the value of a solid cell that is not
    // within one cell of air, so items whose region widened by one cell on
    // every side holds no air are left out (uneven rooms packed into one
    // grid, thick walls). REF keeps every item: its X_M_Y_M_Z_M corner reads
    // solid neighbours' leapfrog values.
    // the work list depends on the model, the tiling, the batch and the
    // plan's z-chunk depth; one device copy per plan lives as long as the
    // engine, because the graphs of every tried plan keep its address
    const std::array<int64_t, 7> key = {model_gen, tiles_x, tiles_y, dz, prm.batch, f16() ? 1 : 0, plan.shape};
    PlanItems& pi = plan_items[plan_id];
    if (pi.key != key && !ref() && have_model) {
        pi.key = key;
        pi.n = -1;
        const int W = sh.w;
        const int64_t ntile = (int64_t)tiles_x * tiles_y;
        const std::array<int64_t, 5> fkey = {model_gen, tiles_x, tiles_y, W, sh.h};
        if (fkey != flags_key) {
            flags_key = fkey;
            air_flags.assign((size_t)(ntile * nz), 0);
            DBuf<uint8_t> fl;
            fl.alloc(air_flags.size(), false);
            air_flags_device(solid_view(), nx, ny, nz, W, sh.h, tiles_x, tiles_y, fl.ptr, stream);
            CK(cudaMemcpyAsync(air_flags.data(), fl.ptr, air_flags.size(), cudaMemcpyDeviceToHost, stream));
            CK(cudaStreamSynchronize(stream));
        }
        std::vector<int> items;
        for (int b = 0; b < prm.batch; ++b)
            for (int c = 0; c < F.n_chunks; ++c) {
                const int z0 = 1 + c * dz, z1 = std::min(z0 + dz, nz - 1);
                for (int64_t t = 0; t < ntile; ++t) {
                    bool need = false;
                    for (int z = std::max(0, z0 - 1); z <= std::min(z1, nz - 1) && !need; ++z)
                        need = air_flags[(size_t)z * ntile + t] != 0;
                    if (need) items.push_back((int)((((int64_t)b * F.n_chunks + c) * tiles_y) * tiles_x + t));
                }
            }
        if ((int64_t)items.size() < n_items) {
            if (pi.buf.ptr) throw Error(AFD_ERR_STATE, "work list of a plan changed while graphs may use it");
            pi.buf.upload(items);
            pi.n = (int64_t)items.size();
        }
    }
    if (pi.n >= 0) {
        F.items = pi.buf.ptr;
        F.n_items = (int32_t)pi.n;
        n_items = pi.n;
    }
    fused_grid = (int)std::max<int64_t>(1, std::min<int64_t>(n_items, resident));
    fused_dirty = false;
}

// The flat launch over `entries` (box, axis): blocks of 256 threads, w =
// min(units, 32) units across, zc planes per thread; *blocks receives the
// grid size.
static BoxLaunch make_box_launch(const std::vector<std::pair<PmlBox, int>>& entries, int batch, int zc,
                                 int* blocks) {
    if ((int)entries.size() > kMaxLaunchBoxes) throw Error(AFD_ERR_ARG, "too many PML boxes for one launch");
    BoxLaunch L{};
    L.n = (int32_t)entries.size();
    L.zc = zc;
    int64_t start = 0;
    for (size_t k = 0; k < entries.size(); ++k) {
        const PmlBox& bx = entries[k].first;
        const int w = std::min(bx.units, 32), rows = 256 / w;
        L.box[k] = bx;
        L.axis[k] = entries[k].second;
        L.w[k] = w;
        L.gx[k] = (bx.units + w - 1) / w;
        L.gy[k] = (bx.height + rows - 1) / rows;
        L.gzc[k] = (bx.depth + zc - 1) / zc;
        L.start[k] = (int32_t)start;
        start += (int64_t)L.gx[k] * L.gy[k] * L.gzc[k] * batch;
    }
    if (start >= ((int64_t)1 << 31)) throw Error(AFD_ERR_ARG, "PML launch too large");
    L.start[entries.size()] = (int32_t)start;
    *blocks = (int)start;
    return L;
}

// SetPml (simulation.hpp:233-277) applied on the device: fresh auxiliary
// fields, ksi profiles and, in FIXED mode, the PML cell list.
void Engine::Impl::setup_pml() {
    pml_owned.release();
    owned_dirty = true;
    for (int a = 0; a < 3; ++a) {
        fi[a][0].release();
        fi[a][1].release();
        ksi_dev[a].release();
    }
    psi[0].release();
    psi[1].release();
    pml_boxes.clear();
    for (auto& v : pml_axis_boxes) v.clear();
    pml_p_all = BoxLaunch{};
    pml_aux_all = BoxLaunch{};
    pml_p_blocks = pml_aux_blocks = 0;
    pml_units = 0;
    n_pml_cells = 0;
    fused_dirty = true;
    pml_g0 = steps_done;
    pml_dirty = false;
    if (pml_width <= 0) return;
    for (int a = 0; a < 3; ++a)
        for (int l = 0; l < 2; ++l) fi[a][l].alloc((size_t)vol * prm.batch);
    psi[0].alloc((size_t)vol * prm.batch);
    psi[1].alloc((size_t)vol * prm.batch);
    // padded so that the reference's ksi_x[y] read (pml.cl:247) stays in bounds
    const int32_t kmax = std::max(nx, std::max(ny, nz)) + 8;
    const int32_t dims[3] = {nx, ny, nz};
    for (int a = 0; a < 3; ++a) {
        std::vector<float> k((size_t)kmax, 0.0f);
        for (int32_t i = 0; i < dims[a] && i < (int32_t)ksi[a].size(); ++i) k[(size_t)i] = ksi[a][(size_t)i];
        ksi_dev[a].upload(k);
    }
    if (!ref()) {
        // FIXED: PML cells are the plain air cells (not solid, not boundary)
        // with 2 <= x, y, z <= n-3 inside an enabled face slab. The kernels
        // walk disjoint boxes covering the slabs and test a 1-bit air mask.
        // (both masks built on the device from the solid and boundary bits)
        const int W = pml_width;
        const uint32_t F = pml_faces;
        const int wpr = (int)(pitch / 32);
        pml_owned.alloc((size_t)nz * ny * wpr, false);
        const int zoff = slab_nz > 0 ? slab_z0 : 0, nzg = slab_nz > 0 ? slab_nz : nz;
        n_pml_cells = pml_masks_device(solid_view(), lrs_bits.ptr, nx, ny, nz, wpr, W, F, pml_owned.ptr, stream,
                                       zoff, nzg);
        // disjoint boxes: z slabs take whole planes, y slabs the remaining
        // planes, x slabs the remaining rows
        pml_boxes.clear();
        auto add = [&](int x0, int x1, int y0, int y1, int z0, int z1) {
            if (x0 > x1 || y0 > y1 || z0 > z1) return;
            PmlBox bx{};
            bx.x0 = x0 & ~3;
            bx.units = (x1 - bx.x0) / 4 + 1;
            bx.y0 = y0;
            bx.height = y1 - y0 + 1;
            bx.z0 = z0;
            bx.depth = z1 - z0 + 1;
            pml_boxes.push_back(bx);
        };
        // local coordinates; along z the grid may be a slab of a larger one
        // (global plane = local + zoff), and the PML rules are global: cells
        // 2..n-3 of the global grid, slabs of W planes at its global faces
        const int off[3] = {0, 0, zoff};
        const int dims3[3] = {nx, ny, nzg};
        int lo[3] = {2, 2, std::max(2 - zoff, 1)}, hi[3] = {nx - 3, ny - 3, std::min(nzg - 3 - zoff, nz - 2)};
        int rest_lo[3] = {lo[0], lo[1], lo[2]}, rest_hi[3] = {hi[0], hi[1], hi[2]};
        for (int ax = 2; ax >= 0; --ax) {
            const bool m_face = F & (1u << (2 * ax)), p_face = F & (2u << (2 * ax));
            int mlo = lo[ax], mhi = std::min(W - 1 - off[ax], hi[ax]);
            int plo = std::max(dims3[ax] - W - off[ax], lo[ax]), phi = hi[ax];
            if (m_face && p_face && plo <= mhi) plo = mhi + 1;
            int box_lo[3], box_hi[3];
            for (int k = 0; k < 3; ++k) {
                box_lo[k] = k > ax ? rest_lo[k] : lo[k];
                box_hi[k] = k > ax ? rest_hi[k] : hi[k];
            }
            if (m_face) {
                box_lo[ax] = mlo;
                box_hi[ax] = mhi;
                add(box_lo[0], box_hi[0], box_lo[1], box_hi[1], box_lo[2], box_hi[2]);
                rest_lo[ax] = std::max(rest_lo[ax], mhi + 1);
            }
            if (p_face) {
                box_lo[ax] = plo;
                box_hi[ax] = phi;
                add(box_lo[0], box_hi[0], box_lo[1], box_hi[1], box_lo[2], box_hi[2]);
                rest_hi[ax] = std::min(rest_hi[ax], plo - 1);
            }
        }
        int64_t first = 0;
        for (PmlBox& bx : pml_boxes) {
            bx.first = first;
            first += (int64_t)bx.units * bx.height * bx.depth;
        }
        pml_units = first;
        // per-axis slab boxes for the auxiliary fields (a cell in two slabs
        // updates one field in each)
        for (int ax = 0; ax < 3; ++ax) {
            pml_axis_boxes[ax].clear();
            const bool m_face = F & (1u << (2 * ax)), p_face = F & (2u << (2 * ax));
            const int mhi = std::min(W - 1 - off[ax], hi[ax]);
            int plo = std::max(dims3[ax] - W - off[ax], lo[ax]);
            if (m_face && p_face && plo <= mhi) plo = mhi + 1;
            auto push = [&](int alo, int ahi) {
                int l3[3] = {lo[0], lo[1], lo[2]}, h3[3] = {hi[0], hi[1], hi[2]};
                l3[ax] = alo;
                h3[ax] = ahi;
                if (l3[0] > h3[0] || l3[1] > h3[1] || l3[2] > h3[2]) return;
                PmlBox bx{};
                bx.x0 = l3[0] & ~3;
                bx.units = (h3[0] - bx.x0) / 4 + 1;
                bx.y0 = l3[1];
                bx.height = h3[1] - l3[1] + 1;
                bx.z0 = l3[2];
                bx.depth = h3[2] - l3[2] + 1;
                pml_axis_boxes[ax].push_back(bx);
            };
            if (m_face) push(lo[ax], mhi);
            if (p_face) push(plo, hi[ax]);
        }
        if ((int)pml_boxes.size() > kMaxPmlBoxes) throw Error(AFD_ERR_ARG, "too many PML boxes");
        std::vector<std::pair<PmlBox, int>> pe, ae;
        for (const PmlBox& bx : pml_boxes) pe.emplace_back(bx, 0);
        for (int ax = 0; ax < 3; ++ax)
            for (const PmlBox& bx : pml_axis_boxes[ax]) ae.emplace_back(bx, ax);
        pml_p_all = make_box_launch(pe, prm.batch, pml_zc, &pml_p_blocks);
        pml_aux_all = make_box_launch(ae, prm.batch, pml_zc, &pml_aux_blocks);
    }
}

void Engine::Impl::upload_sources() {
    std::vector<int32_t> cell, begin((size_t)prm.batch + 1, 0);
    std::vector<int64_t> off, len;
    std::vector<float> data;
    for (int32_t b = 0; b < prm.batch; ++b) {
        begin[(size_t)b] = (int32_t)cell.size();
        for (const Source& s : sources) {
            if (s.batch != b) continue;
            check_cell(s.ijk, nx, ny, nz, "source");
            cell.push_back((int32_t)(s.ijk[2] * plane + s.ijk[1] * pitch + s.ijk[0]));
            off.push_back((int64_t)data.size());
            len.push_back((int64_t)s.sig.size());
            data.insert(data.end(), s.sig.begin(), s.sig.end());
        }
    }
    begin[(size_t)prm.batch] = (int32_t)cell.size();
    if (f16()) {
        smax_host.assign((size_t)prm.batch, 0.0f);
        for (const Source& s : sources)
            for (float v : s.sig) smax_host[(size_t)s.batch] = std::max(smax_host[(size_t)s.batch], std::fabs(v));
        f16_smax.upload(smax_host);
    }
    src_cell.upload(cell);
    src_begin.upload(begin);
    src_off.upload(off);
    src_len.upload(len);
    if (data.empty()) data.push_back(0.0f);
    src_data.upload(data);
    src_dirty = false;
    fused_dirty = true;
}

// CheckVariables (simulation.hpp:436-447): the receiver record grows to the
// new end time; recorded samples keep their place.
void Engine::Impl::ensure_receivers(int64_t t_end) {
    const int32_t nr = (int32_t)receivers.size();
    if (nr == rcv_n_dev && rcv_cap >= t_end && rcv_out.ptr) return;
    std::vector<int32_t> cell;
    for (auto& r : receivers) {
        check_cell(r.data(), nx, ny, nz, "receiver");
        cell.push_back((int32_t)(r[2] * plane + r[1] * pitch + r[0]));
    }
    int64_t cap = std::max<int64_t>(t_end, 1);
    cap = std::max(cap, rcv_cap);
    DBuf<float> fresh;
    fresh.alloc((size_t)prm.batch * std::max(nr, 1) * cap);
    if (rcv_out.ptr && rcv_cap > 0 && steps_done > 0) {
        // copy the rows of the receivers that existed before
        for (int32_t b = 0; b < prm.batch; ++b)
            CK(cudaMemcpy2D(fresh.ptr + (size_t)b * nr * cap, cap * sizeof(float),
                            rcv_out.ptr + (size_t)b * rcv_n_dev * rcv_cap, rcv_cap * sizeof(float),
                            steps_done * sizeof(float), (size_t)rcv_n_dev, cudaMemcpyDeviceToDevice));
    }
    std::swap(rcv_out.ptr, fresh.ptr);
    std::swap(rcv_out.n, fresh.n);
    rcv_cap = cap;
    rcv_n_dev = nr;
    rcv_cell.upload(cell);
    drop_graphs();
    fused_dirty = true;
}

void Engine::Impl::build_args() {
    // the source/receiver kernel may run beside the FIXED-scheme auxiliary
    // updates when no source cell lies where they read the new pressure (a
    // unit of 4 cells at (x, y, z) reads x..x+4, y..y+1, z..z+1): the
    // auxiliary updates read the pressure before injection, write only the
    // auxiliary fields, and recording reads the injected values
    src_beside_aux = !ref() && pml_width > 0;
    for (const Source& src : sources)
        for (int ax = 0; ax < 3 && src_beside_aux; ++ax)
            for (const PmlBox& bx : pml_axis_boxes[ax]) {
                const int x = src.ijk[0], y = src.ijk[1], z = src.ijk[2];
                if (x >= bx.x0 && x <= bx.x0 + 4 * bx.units && y >= bx.y0 && y <= bx.y0 + bx.height &&
                    z >= bx.z0 && z <= bx.z0 + bx.depth) {
                    src_beside_aux = false;
                    break;
                }
            }
    StepArgs& a = args;
    a = StepArgs{};
    a.g = GridDev{nx, ny, nz, pitch, plane, vol};
    a.batch = prm.batch;
    a.mode = prm.mode;
    if (f16()) {
        for (int k = 0; k < 3; ++k) a.f16.h[k] = reinterpret_cast<__half*>(fields.ptr) + (size_t)k * vol * prm.batch;
        a.f16.mx = f16_mx.ptr;
        a.f16.src_max = f16_smax.ptr;
    } else {
        for (int k = 0; k < 3; ++k) a.p[k] = fields.ptr + (size_t)k * vol * prm.batch;
    }
    a.d_step = d_step.ptr;
    a.lambda2 = lambda2();
    a.cint = 2.0f * (1.0f - 3.0f * a.lambda2);
    a.lrs.n = (int32_t)lrs_cell.n;
    a.lrs.K = have_model ? model.ncoef : 1;
    a.lrs.S = 3 * a.lrs.K;
    a.lrs.cell = lrs_cell.ptr;
    a.lrs.info = lrs_info.ptr;
    a.lrs.st_in = lrs_in.ptr;
    a.lrs.st_out = lrs_out.ptr;
    a.lrs.ca = coef_a.ptr;
    a.lrs.cb = coef_b.ptr;
    // REF: simulation.hpp:368-369 passes lambda^2 as l (lrs_1.cl:58,78)
    a.lrs.l = ref() ? a.lambda2 : prm.dt * prm.c / prm.dx;
    a.lrs.l2 = a.lrs.l * a.lrs.l;
    a.lrs.c2 = 2.0f * (1.0f - 3.0f * a.lrs.l2);
    PmlDev& P = a.pml;
    P.width = pml_width > 0 && psi[0].ptr ? pml_width : 0;
    P.faces = pml_faces;
    P.g0 = pml_g0;
    for (int x = 0; x < 3; ++x) {
        P.fi[x][0] = fi[x][0].ptr;
        P.fi[x][1] = fi[x][1].ptr;
        P.ksi[x] = ksi_dev[x].ptr;
    }
    P.psi[0] = psi[0].ptr;
    P.psi[1] = psi[1].ptr;
    const float c = prm.c, dx = prm.dx, dt = prm.dt;
    P.dt = dt;
    P.cc_dxdx = c * c / (dx * dx);
    P.inv_dx = 1.0f / dx;
    P.half_inv_dx = 0.5f / dx;
    P.inv_dt2 = 1.0f / (dt * dt);
    P.two_dt = 2.0f * dt;
    P.inv_dt = 1.0f / dt;
    P.psi_on = ref() || ((pml_faces & 3u) && (pml_faces & 12u) && (pml_faces & 48u)) ? 1 : 0;
    P.n_boxes = (int32_t)pml_boxes.size();
    for (size_t k = 0; k < pml_boxes.size(); ++k) P.boxes[k] = pml_boxes[k];
    P.n_units = pml_units;
    P.cells = pml_owned.ptr;
    P.words_per_row = (int32_t)(pitch / 32);
    P.zoff = slab_nz > 0 ? slab_z0 : 0;
    P.nz_glob = slab_nz > 0 ? slab_nz : nz;
    a.src.n = (int32_t)src_cell.n;
    a.src.cell = src_cell.ptr;
    a.src.begin = src_begin.ptr;
    a.src.off = src_off.ptr;
    a.src.len = src_len.ptr;
    a.src.data = src_data.ptr;
    a.rcv.n = rcv_n_dev;
    a.rcv.cell = rcv_cell.ptr;
    a.rcv.out = rcv_out.ptr;
    a.rcv.cap = rcv_cap;
    a.flag = d_flag.ptr;
    a.tl_start = tl_steps > 0 ? tl_start.ptr : nullptr;
    a.tl_end = tl_steps > 0 ? tl_end.ptr : nullptr;
    a.tl_g0 = tl_first;
    a.tl_steps = tl_steps;
    // inline source/receiver table (device order of upload_sources)
    inline_ok = (int64_t)sources.size() <= kInlineSrc && (int64_t)receivers.size() <= kInlineRcv;
    inl = SrcRcvInline{};
    if (inline_ok) {
        int64_t off = 0;
        int k = 0;
        for (int32_t bm = 0; bm < prm.batch; ++bm)
            for (const Source& q : sources) {
                if (q.batch != bm) continue;
                inl.src_cell[k] = (int32_t)(q.ijk[2] * plane + q.ijk[1] * pitch + q.ijk[0]);
                inl.src_batch[k] = bm;
                inl.src_len[k] = (int64_t)q.sig.size();
                inl.src_ptr[k] = src_data.ptr + off;
                off += (int64_t)q.sig.size();
                ++k;
            }
        inl.n_src = k;
        inl.n_rcv = (int32_t)receivers.size();
        for (size_t r = 0; r < receivers.size(); ++r)
            inl.rcv_cell[r] = (int32_t)(receivers[r][2] * plane + receivers[r][1] * pitch + receivers[r][0]);
    }
}

enum KernelKind { KK_INTERIOR, KK_LRS, KK_PML_AUX, KK_PML_P, KK_SRC_RCV, KK_FUSED, KK_COUNT };
static const char* kKernelNames[KK_COUNT] = {"interior", "boundary", "pml_aux", "pml_pressure",
                                             "source_receiver", "interior_stream"};

void Engine::Impl::launch_step(int j, bool profile) {
    if (f16()) launch_step_t<__half>(j, profile);
    else launch_step_t<float>(j, profile);
}

// One time step, global step = *d_step + j (simulation.hpp:358-392).
template <typename T>
void Engine::Impl::launch_step_t(int j, bool profile) {
    const StepArgs& a = args;
    auto begin = [&](int kind) {
        if (!profile) return;
        if (ev_kind.size() >= ev_pool.size()) {
            cudaEvent_t e0, e1;
            CK(cudaEventCreate(&e0));
            CK(cudaEventCreate(&e1));
            ev_pool.emplace_back(e0, e1);
        }
        CK(cudaEventRecord(ev_pool[ev_kind.size()].first, stream));
        ev_kind.push_back(kind);
    };
    auto end = [&]() {
        if (!profile) return;
        CK(cudaEventRecord(ev_pool[ev_kind.size() - 1].second, stream));
    };
    const dim3 blk(64, 4, 1);
    const bool tail = tail_active() && step_phase == 0;
    auto stream_launch = [&](cudaStream_t st) {
        launch_stream<T>(plan.shape, tail, fused_grid, st, tm_halo, tm_own, a, fdev, j);
        ++launches;
    };
    // a split step (z-slab runs): phase 1 runs the interior, boundary and
    // PML pressure updates, phase 2 the PML auxiliary fields and the
    // source/receiver and capture kernels, in the serial order
    const bool phA = step_phase != 2, phB = step_phase != 1;
    const bool beside = lists_beside() && fdev.owned && step_phase == 0;
    if (!beside && phA) {
        if (use_fused()) {
            begin(KK_FUSED);
            stream_launch(stream);
            end();
        } else {
            const dim3 grd((unsigned)((nx - 2 + 63) / 64), (unsigned)((ny - 2 + 3) / 4),
                           (unsigned)((nz - 2) * prm.batch));
            begin(KK_INTERIOR);
            k_interior<T><<<grd, blk, 0, stream>>>(a, j);
            end();
            ++launches;
        }
    }
    auto lrs_launch = [&](cudaStream_t st) {
        const dim3 grd((unsigned)((a.lrs.n + 255) / 256), (unsigned)prm.batch);
        if constexpr (sizeof(T) == 4) {
            if (ref()) launch_lrs<true, float>(a, j, grd, st);
            else launch_lrs<false, float>(a, j, grd, st);
        } else {
            launch_lrs<false, T>(a, j, grd, st);
        }
        ++launches;
    };
    const bool psi = a.pml.psi_on != 0;
    // every pressure box in one launch, every (axis, slab box) pair in another
    auto pml_p_launch = [&](cudaStream_t st) {
        if (psi) k_pml_p_all<true, T><<<pml_p_blocks, 256, 0, st>>>(a, pml_p_all, j);
        else k_pml_p_all<false, T><<<pml_p_blocks, 256, 0, st>>>(a, pml_p_all, j);
        ++launches;
    };
    auto pml_aux_launch = [&](cudaStream_t st) {
        if (psi) k_pml_aux_all<true, T><<<pml_aux_blocks, 256, 0, st>>>(a, pml_aux_all, j);
        else k_pml_aux_all<false, T><<<pml_aux_blocks, 256, 0, st>>>(a, pml_aux_all, j);
        ++launches;
    };
    bool src_done = false;  // the source/receiver kernel already queued beside the auxiliary updates
    auto src_rcv_launch = [&](cudaStream_t st) {
        if (inline_ok) k_src_rcv_inline<T><<<(unsigned)prm.batch, 256, 0, st>>>(a, inl, j);
        else k_src_rcv<T><<<(unsigned)prm.batch, 128, 0, st>>>(a, j, 1, 1);
        ++launches;
    };
    const bool fixed_pml = !ref() && a.pml.width > 0 && a.pml.n_units > 0;
    if (beside) {
        // FIXED scheme in graphs: the streaming kernel skips the cells of
        // the boundary and PML kernels, which run beside it (they read only
        // levels n and n-1, filter state and the old auxiliary fields); the
        // auxiliary updates read the new level of every cell and follow.
        std::vector<std::function<void(cudaStream_t)>> g1, g2;
        g1.push_back(stream_launch);
        if (a.lrs.n > 0) g1.push_back(lrs_launch);
        if (fixed_pml) g1.push_back(pml_p_launch);
        if (fixed_pml) g2.push_back(pml_aux_launch);
        run_side_by_side(g1);
        run_side_by_side(g2);
    } else if (fixed_pml && !profile && prm.graphs && step_phase == 0) {  // inside CUDA graphs: no host cost per step
        // FIXED scheme: the boundary update and the PML pressure boxes write
        // disjoint cells and read only levels n and n-1 and the old
        // auxiliary fields, so they run side by side; the auxiliary updates
        // (one per axis, disjoint outputs) follow once both are done.
        std::vector<std::function<void(cudaStream_t)>> g1, g2;
        if (a.lrs.n > 0 && !tail) g1.push_back(lrs_launch);
        if (!tail) g1.push_back(pml_p_launch);
        if (src_beside_aux && (a.src.n > 0 || a.rcv.n > 0)) {
            // queued first: its one block then starts at once instead of
            // waiting for the auxiliary updates' blocks to be dispatched
            g2.push_back([&](cudaStream_t st) { src_rcv_launch(st); });
            src_done = true;
        }
        g2.push_back(pml_aux_launch);
        run_side_by_side(g1);
        run_side_by_side(g2);
    } else {
        if (a.lrs.n > 0 && phA && !tail) {
            begin(KK_LRS);
            lrs_launch(stream);
            end();
        }
        if (a.pml.width > 0) {
            if (ref()) {
                if (sizeof(T) == 4 && nx > 4 && ny > 4 && nz > 4) {
                    const dim3 grd((unsigned)((nx - 4 + 63) / 64), (unsigned)((ny - 4 + 3) / 4),
                                   (unsigned)((nz - 4) * prm.batch));
                    begin(KK_PML_AUX);
                    k_pml_ref_aux<<<grd, blk, 0, stream>>>(a, j);
                    end();
                    begin(KK_PML_P);
                    k_pml_ref_p<<<grd, blk, 0, stream>>>(a, j);
                    end();
                    launches += 2;
                }
            } else if (a.pml.n_units > 0) {
                if (phA && !tail) {
                    begin(KK_PML_P);
                    pml_p_launch(stream);
                    end();
                }
                if (phB) {
                    begin(KK_PML_AUX);
                    pml_aux_launch(stream);
                    end();
                }
            }
        }
    }
    if ((a.src.n > 0 || a.rcv.n > 0) && !src_done && phB) {
        begin(KK_SRC_RCV);
        src_rcv_launch(stream);
        end();
    }
    if (cap_every > 0 && phB) {
        const int total = cap.rows * cap.cols;
        k_capture<T><<<(unsigned)std::min(592, (total + 255) / 256), 256, 0, stream>>>(a, cap, j);
        ++launches;
    }
}

cudaGraphExec_t Engine::Impl::graph_for(int64_t n) {
    const int64_t key = n + ((int64_t)plan_id << 32);  // one graph per chunk length and streaming plan
    auto it = graphs.find(key);
    if (it != graphs.end()) return it->second;
    cudaGraph_t graph;
    const int64_t saved = launches;
    CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    if (use_fused()) CK(cudaMemsetAsync(f_work.ptr, 0, (size_t)n * sizeof(int), stream));
    if (tail_active()) CK(cudaMemsetAsync(f_tail.ptr, 0, (size_t)n * sizeof(unsigned long long), stream));
    for (int64_t j = 0; j < n; ++j) launch_step((int)j, false);
    k_advance<<<1, 1, 0, stream>>>(d_step.ptr, (int)n);
    CK(cudaStreamEndCapture(stream, &graph));
    launches = saved;
    cudaGraphExec_t exec;
    CK(cudaGraphInstantiate(&exec, graph, 0));
    cudaGraphDestroy(graph);
    graphs[key] = exec;
    return exec;
}

void Engine::Impl::run_chunk(int64_t n) {
    const bool profile = prm.profile != 0;
    if (prm.graphs && !profile) {
        cudaGraphExec_t g = graph_for(n);
        CK(cudaGraphLaunch(g, stream));
        // the graph holds n steps of kernels plus the step-counter advance
        launch_step_count_only(n);
    } else {
        if (use_fused()) CK(cudaMemsetAsync(f_work.ptr, 0, (size_t)n * sizeof(int), stream));
        if (tail_active()) CK(cudaMemsetAsync(f_tail.ptr, 0, (size_t)n * sizeof(unsigned long long), stream));
        for (int64_t j = 0; j < n; ++j) launch_step((int)j, profile);
        k_advance<<<1, 1, 0, stream>>>(d_step.ptr, (int)n);
        ++launches;
    }
    CK(cudaGetLastError());
}

void Engine::Impl::collect_profile() {
    if (ev_kind.empty()) return;
    CK(cudaStreamSynchronize(stream));
    for (size_t k = 0; k < ev_kind.size(); ++k) {
        float ms = 0.0f;
        CK(cudaEventElapsedTime(&ms, ev_pool[k].first, ev_pool[k].second));
        KernelStat& st = kstats[(size_t)ev_kind[k]];
        st.launches += 1;
        st.ms += ms;
    }
    ev_kind.clear();
}

int64_t Engine::Impl::kernels_per_step() const {
    const StepArgs& a = args;
    int64_t k = 1;
    const bool tail = tail_active();
    if (a.lrs.n > 0 && !tail) ++k;
    if (a.pml.width > 0) {
        if (ref()) k += (nx > 4 && ny > 4 && nz > 4) ? 2 : 0;
        else if (a.pml.n_units > 0)
            k += tail ? 1 : 2;
    }
    if (a.src.n > 0 || a.rcv.n > 0) ++k;
    if (cap_every > 0) ++k;
    return k;
}

// ---------------------------------------------------------------------------
// Engine public methods
// ---------------------------------------------------------------------------
Engine::Engine(const afd_params& p) : d_(new Impl) {
    Impl& D = *d_;
    D.prm = p;
    if (!(p.dx > 0.0f) || !(p.c > 0.0f) || !(p.dt > 0.0f))
        throw Error(AFD_ERR_ARG, "dx, c and dt must be positive");
    if (p.batch < 1 || p.batch > 4096) throw Error(AFD_ERR_ARG, "batch must be in 1..4096");
    if (p.mode != AFD_MODE_REF && p.mode != AFD_MODE_FIXED) throw Error(AFD_ERR_ARG, "unknown mode");
    if (p.storage != AFD_STORE_FP32 && p.storage != AFD_STORE_FP16) throw Error(AFD_ERR_ARG, "unsupported storage");
    if (p.storage == AFD_STORE_FP16 && p.mode != AFD_MODE_FIXED)
        throw Error(AFD_ERR_ARG, "FP16 storage requires the FIXED scheme");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        throw Error(AFD_ERR_CUDA, "no CUDA device available");
    if (p.device < 0 || p.device >= ndev) throw Error(AFD_ERR_ARG, "device ordinal out of range");
    D.device = p.device;
    CK(cudaSetDevice(D.device));
    CK(cudaStreamCreateWithFlags(&D.own_stream, cudaStreamNonBlocking));
    D.stream = D.own_stream;
    CK(cudaEventCreate(&D.ev0));
    CK(cudaEventCreate(&D.ev1));
    D.d_step.alloc(1);
    D.d_flag.alloc(1);
    D.d_energy.alloc(1);
    CK(cudaMemcpyToSymbol(c_group_mask, kGroupMask, sizeof(kGroupMask)));
    CK(cudaStreamSynchronize(cudaStreamLegacy));  // before any launch on the non-blocking stream
    for (int k = 0; k < KK_COUNT; ++k) D.kstats.push_back(KernelStat{kKernelNames[k], 0, 0.0});
}

Engine::~Engine() {
    Impl& D = *d_;
    cudaSetDevice(D.device);
    if (D.stream) cudaStreamSynchronize(D.stream);
    D.drop_graphs();
    for (auto& e : D.ev_pool) {
        cudaEventDestroy(e.first);
        cudaEventDestroy(e.second);
    }
    if (D.ev0) cudaEventDestroy(D.ev0);
    if (D.ev1) cudaEventDestroy(D.ev1);
    if (D.pinned) cudaFreeHost(D.pinned);
    for (auto st : D.side) cudaStreamDestroy(st);
    for (auto e : D.side_ev) cudaEventDestroy(e);
    if (D.fork_ev) cudaEventDestroy(D.fork_ev);
    if (D.tev0) cudaEventDestroy(D.tev0);
    if (D.tev1) cudaEventDestroy(D.tev1);
    if (D.own_stream) cudaStreamDestroy(D.own_stream);
}

float Engine::cell_size() const { return d_->prm.dx; }

void Engine::set_stream(void* stream) {
    Impl& D = *d_;
    CK(cudaSetDevice(D.device));
    cudaStream_t s = stream ? (cudaStream_t)stream : D.own_stream;
    if (s != D.stream) {
        CK(cudaStreamSynchronize(D.stream));
        D.drop_graphs();
        D.stream = s;
    }
}

void Engine::set_slab(int32_t z_offset, int32_t nz_global) {
    Impl& D = *d_;
    if (D.phase_open) throw Error(AFD_ERR_STATE, "a split step is open");
    if (nz_global == 0) {
        D.slab_z0 = D.slab_nz = 0;
    } else {
        if (D.ref()) throw Error(AFD_ERR_STATE, "z-slabs need the FIXED scheme");
        if (D.f16()) throw Error(AFD_ERR_STATE, "z-slabs need FP32 storage (FP16 scales are per grid)");
        if (z_offset < 0 || nz_global < 3) throw Error(AFD_ERR_ARG, "bad slab placement");
        D.slab_z0 = z_offset;
        D.slab_nz = nz_global;
    }
    D.pml_dirty = true;  // the PML cells and boxes follow global planes
}

// Half of one time step (z-slab runs): phase 1 runs the interior, boundary
// and PML pressure updates of step steps_done; phase 2 the PML auxiliary
// updates, sources, receivers and capture, and completes the step. Between
// them and after phase 2 the caller refreshes the halo planes (afd_halo).
void Engine::step(int32_t phase) {
    Impl& D = *d_;
    if (phase != 1 && phase != 2) throw Error(AFD_ERR_ARG, "phase must be 1 or 2");
    if ((phase == 1) == D.phase_open) throw Error(AFD_ERR_STATE, phase == 1 ? "phase 2 of the previous step is due"
                                                                            : "phase 1 of this step has not run");
    if (D.ref()) throw Error(AFD_ERR_STATE, "split steps need the FIXED scheme");
    if (phase == 1) {
        D.setup_run(1);
        if (D.use_fused()) CK(cudaMemsetAsync(D.f_work.ptr, 0, sizeof(int), D.stream));
        CK(cudaMemsetAsync(D.d_flag.ptr, 0, sizeof(int), D.stream));
    }
    D.step_phase = phase;
    try {
        D.launch_step(0, false);
    } catch (...) {
        D.step_phase = 0;
        throw;
    }
    D.step_phase = 0;
    if (phase == 2) {
        k_advance<<<1, 1, 0, D.stream>>>(D.d_step.ptr, 1);
        ++D.launches;
    }
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(D.stream));
    int flag = 0;
    CK(cudaMemcpy(&flag, D.d_flag.ptr, sizeof(int), cudaMemcpyDeviceToHost));
    D.phase_open = phase == 1;
    if (phase == 2) D.advance_done(1);
    if (flag & 2) throw Error(AFD_ERR_CUDA, "step kernel pipeline wait timed out");
    if (flag && D.prm.watchdog)
        throw Error(AFD_ERR_NUMERIC, "pressure left the finite bound |p| < 1e30 by step " + std::to_string(D.steps_done));
}

// One plane of every batch member between the engine and a caller device
// buffer ([batch][ny][pitch] floats): side 0 the low-z end, 1 the high-z
// end; dir 0 reads the outermost interior plane of that end (local 1 or
// nz-2), dir 1 writes the halo plane (local 0 or nz-1). field 0: the
// pressure level of the open or last completed step; 1..3: that step's new
// PML auxiliary field of axis x, y, z; 4: its new psi.
void Engine::halo(int32_t side, int32_t dir, int32_t field, void* dev, int64_t cap) {
    Impl& D = *d_;
    if (!D.initialized || D.steps_done + (D.phase_open ? 1 : 0) == 0) throw Error(AFD_ERR_STATE, "no step has run");
    if (side < 0 || side > 1 || dir < 0 || dir > 1 || field < 0 || field > 4) throw Error(AFD_ERR_ARG, "bad halo selector");
    if (D.f16()) throw Error(AFD_ERR_STATE, "halo planes are FP32 levels");
    const int64_t need = (int64_t)D.prm.batch * D.plane;
    if (!dev || cap < need) throw Error(AFD_ERR_ARG, "halo buffer too small (batch * ny * pitch floats)");
    const long long g = D.phase_open ? D.steps_done : D.steps_done - 1;
    float* base = nullptr;
    if (field == 0) {
        base = D.fields.ptr + (size_t)buf_new(g) * D.vol * D.prm.batch;
    } else {
        if (D.pml_width <= 0 || !D.psi[0].ptr) throw Error(AFD_ERR_STATE, "no PML fields");
        const int lv = (int)((g - D.pml_g0 + 1) & 1);
        base = field == 4 ? D.psi[lv].ptr : D.fi[field - 1][lv].ptr;
    }
    const int64_t z = dir == 0 ? (side == 0 ? 1 : D.nz - 2) : (side == 0 ? 0 : D.nz - 1);
    CK(cudaSetDevice(D.device));
    float* d = static_cast<float*>(dev);
    for (int32_t b = 0; b < D.prm.batch; ++b) {
        float* lvl = base + (size_t)b * D.vol + (size_t)z * D.plane;
        float* buf = d + (size_t)b * D.plane;
        if (dir == 0) CK(cudaMemcpyAsync(buf, lvl, (size_t)D.plane * sizeof(float), cudaMemcpyDeviceToDevice, D.stream));
        else CK(cudaMemcpyAsync(lvl, buf, (size_t)D.plane * sizeof(float), cudaMemcpyDeviceToDevice, D.stream));
    }
    CK(cudaStreamSynchronize(D.stream));
}

void Engine::set_plan(const afd_plan* p) {
    Impl& D = *d_;
    int shape = 0;
    if (p) {
        shape = -1;
        if (p->tile_x == 0 && p->tile_y == 0) shape = 0;
        for (int sh = 0; sh < kTileShapes && shape < 0; ++sh)
            if (shape_valid(D.f16(), sh) && p->tile_x == shape_w32(sh) * (D.f16() ? 2 : 1) && p->tile_y == shape_h(sh))
                shape = sh;
        if (shape < 0)
            throw Error(AFD_ERR_ARG, D.f16() ? "unsupported streaming tile (FP16 storage: 128x16 or 64x32)"
                                             : "unsupported streaming tile (64x16, 128x8 or 32x32)");
        if (p->per_sm < 0 || p->per_sm > 32) throw Error(AFD_ERR_ARG, "per_sm out of range (0..32)");
        if (p->dz < 0 || p->dz > 1024) throw Error(AFD_ERR_ARG, "dz out of range (0..1024)");
    }
    CK(cudaSetDevice(D.device));
    CK(cudaStreamSynchronize(D.stream));
    // no graph may keep the addresses of the per-plan work lists freed here
    D.drop_graphs();
    D.plan_items.clear();
    D.forced = p != nullptr;
    if (p) D.forced_plan = Impl::Plan{p->per_sm, p->dz, p->beside != 0, shape, p->tail != 0};
    D.tuned = false;
    D.tune_gen = -1;  // candidates are made again by the next run or prepare
    D.plan = Impl::Plan{0, 0, false, 0, false};
    D.plan_id = 0;
    D.fused_dirty = true;
}

void Engine::set_min_size(float x, float y, float z) {
    Impl& D = *d_;
    if (D.initialized) throw Error(AFD_ERR_STATE, "the grid is fixed after the first run");
    const float v[3] = {x, y, z};
    int32_t out[3];
    for (int k = 0; k < 3; ++k) {
        if (!(v[k] >= 0.0f) || !(v[k] / D.prm.dx < 65536.0f)) throw Error(AFD_ERR_ARG, "minsize out of range");
        out[k] = (int32_t)round_to((uint32_t)(cell_of(v[k], D.prm.dx) + 1), 32);
    }
    std::copy(out, out + 3, D.min_size);
}

static void check_model_header(const Model& m) {
    if (m.nx < 3 || m.ny < 3 || m.nz < 3) throw Error(AFD_ERR_ARG, "model grid must be at least 3x3x3");
    if ((int64_t)m.vox.size() != m.cells() && !m.vox.empty()) throw Error(AFD_ERR_ARG, "voxel count mismatch");
    if (m.nmat < 1 || m.nmat > 256) throw Error(AFD_ERR_ARG, "1..256 materials are supported");
    if (m.ncoef < 1 || m.ncoef > 64) throw Error(AFD_ERR_ARG, "filters must have 1..64 coefficients");
}

// Simulation::Load's LrsData (simulation.hpp:176): the voxel range check and
// the boundary classification run on the device (geometry.cu).
void Engine::set_model(const Model& m) {
    Impl& D = *d_;
    if (D.initialized) throw Error(AFD_ERR_STATE, "the model cannot change after the first run");
    check_model_header(m);
    if (m.vox.empty()) throw Error(AFD_ERR_ARG, "voxel count mismatch");
    CK(cudaSetDevice(D.device));
    DBuf<int32_t> dv;
    dv.alloc((size_t)m.cells(), false);
    CK(cudaMemcpyAsync(dv.ptr, m.vox.data(), (size_t)m.cells() * sizeof(int32_t), cudaMemcpyHostToDevice, D.stream));
    Model hdr;
    hdr.nx = m.nx;
    hdr.ny = m.ny;
    hdr.nz = m.nz;
    hdr.nmat = m.nmat;
    hdr.ncoef = m.ncoef;
    hdr.a = m.a;
    hdr.b = m.b;
    hdr.material_names = m.material_names;
    D.adopt_model(std::move(hdr), dv.ptr);
}

// The boundary list and the solid bits of the voxels at d_vox (on the
// engine's stream); the model keeps no host voxels.
void Engine::Impl::adopt_model(Model&& hdr, const int32_t* d_vox) {
    std::vector<BoundaryPoint> pts = classify_device(d_vox, hdr.nx, hdr.ny, hdr.nz, hdr.nmat, stream);
    DBuf<uint32_t> bits;
    bits.alloc((size_t)hdr.ny * hdr.nz * row_words(hdr.nx), false);
    solid_bits_device(d_vox, hdr.nx, hdr.ny, hdr.nz, bits.ptr, stream);
    CK(cudaStreamSynchronize(stream));
    hdr.vox.clear();
    model = std::move(hdr);
    std::swap(model_solid.ptr, bits.ptr);
    std::swap(model_solid.n, bits.n);
    boundary.swap(pts);
    std::fill(boundary_counts, boundary_counts + kNumGroups, 0);
    for (const BoundaryPoint& bp : boundary) boundary_counts[bp.group]++;
    have_model = true;
}

// Simulation::Load (simulation.hpp:173-176): the scene is parsed on the host,
// rasterised and classified on the device.
void Engine::load_kerkythea(const std::string& xml_path) {
    Impl& D = *d_;
    if (D.initialized) throw Error(AFD_ERR_STATE, "the model cannot change after the first run");
    Scene sc = parse_kerkythea(xml_path, D.prm.dx);
    check_model_header(sc.model);
    CK(cudaSetDevice(D.device));
    DBuf<int32_t> dv;
    dv.alloc((size_t)sc.model.cells(), false);
    rasterize_device(sc, dv.ptr, D.stream);
    D.adopt_model(std::move(sc.model), dv.ptr);
}

void Engine::set_pml(int32_t width, uint32_t faces, const float* kx, const float* ky, const float* kz) {
    Impl& D = *d_;
    if (width < 0) throw Error(AFD_ERR_ARG, "PML width must be >= 0");
    int32_t dims[3];
    D.grid_dims(dims);
    if (width > 0 && (dims[0] < 3 || dims[1] < 3 || dims[2] < 3))
        throw Error(AFD_ERR_STATE, "load a model or set minsize before pml");
    const float* src[3] = {kx, ky, kz};
    for (int k = 0; k < 3; ++k) {
        D.ksi[k].assign((size_t)std::max(dims[k], 0), 0.0f);
        if (src[k] && dims[k] > 0) std::copy(src[k], src[k] + dims[k], D.ksi[k].begin());
    }
    D.pml_width = width;
    D.pml_faces = faces & 63u;
    D.pml_dirty = true;
}

void Engine::set_pml_profile(int32_t width, const float* prof, int32_t len) {
    Impl& D = *d_;
    if (len < 0 || (len > 0 && !prof)) throw Error(AFD_ERR_ARG, "bad PML profile");
    int32_t dims[3];
    D.grid_dims(dims);
    if (dims[0] < 3 || dims[1] < 3 || dims[2] < 3)
        throw Error(AFD_ERR_STATE, "load a model or set minsize before pml");
    std::vector<float> k3[3];
    for (int k = 0; k < 3; ++k) {
        k3[k].assign((size_t)dims[k], 0.0f);
        // simulation.hpp:268-276: ksi[i] = ksi[n-1-i] = prof[L-1-i]
        for (int32_t i = 0; i < len; ++i) {
            if (i >= dims[k]) throw Error(AFD_ERR_ARG, "PML profile longer than the grid");
            k3[k][(size_t)i] = prof[len - 1 - i];
            k3[k][(size_t)(dims[k] - i - 1)] = prof[len - 1 - i];
        }
    }
    set_pml(width, 63u, k3[0].data(), k3[1].data(), k3[2].data());
}

void Engine::add_source_cell(int32_t batch, const int32_t ijk[3], const float* sig, int64_t len) {
    Impl& D = *d_;
    if (batch < 0 || batch >= D.prm.batch) throw Error(AFD_ERR_ARG, "batch index out of range");
    if (len < 0 || (len > 0 && !sig)) throw Error(AFD_ERR_ARG, "bad source signal");
    int32_t dims[3];
    D.grid_dims(dims);
    if (dims[0] > 0 && dims[1] > 0 && dims[2] > 0) check_cell(ijk, dims[0], dims[1], dims[2], "source");
    Source s;
    s.batch = batch;
    std::copy(ijk, ijk + 3, s.ijk);
    s.sig.assign(sig, sig + len);
    D.sources.push_back(std::move(s));
    D.src_dirty = true;
}

void Engine::add_source_pos(int32_t batch, const float pos[3], const float* sig, int64_t len) {
    // (cl_int)(pos / res_), simulation.hpp:322
    int32_t ijk[3];
    for (int k = 0; k < 3; ++k) {
        const float q = pos[k] / d_->prm.dx;
        if (!(q > -2.0e9f && q < 2.0e9f)) throw Error(AFD_ERR_ARG, "source position out of range");
        ijk[k] = (int32_t)q;
    }
    add_source_cell(batch, ijk, sig, len);
}

void Engine::add_receiver_cell(const int32_t ijk[3]) {
    Impl& D = *d_;
    int32_t dims[3];
    D.grid_dims(dims);
    if (dims[0] > 0 && dims[1] > 0 && dims[2] > 0) check_cell(ijk, dims[0], dims[1], dims[2], "receiver");
    D.receivers.push_back({ijk[0], ijk[1], ijk[2]});
}

void Engine::add_receiver_pos(const float pos[3]) {
    // (cl_int)(pos / res_), simulation.hpp:338
    int32_t ijk[3];
    for (int k = 0; k < 3; ++k) {
        const float q = pos[k] / d_->prm.dx;
        if (!(q > -2.0e9f && q < 2.0e9f)) throw Error(AFD_ERR_ARG, "receiver position out of range");
        ijk[k] = (int32_t)q;
    }
    add_receiver_cell(ijk);
}

// Simulation::Run (simulation.hpp:342-434). Chunks end where the reference
// reports progress (step 0 and every 200th step), so a chunk is one
// captured graph replay; the REF-mode PML fields are zeroed after every
// 8000th step of the run (simulation.hpp:411-430).
// Device state for a run of `steps` more steps: model, PML, sources,
// receiver record, streaming plan and kernel arguments.
void Engine::Impl::setup_run(int64_t steps) {
    if (steps < 0) throw Error(AFD_ERR_ARG, "steps must be >= 0");
    CK(cudaSetDevice(device));
    if (!initialized) init_device();
    if (pml_dirty) {
        setup_pml();
        drop_graphs();
    }
    if (src_dirty) {
        upload_sources();
        drop_graphs();
    }
    ensure_receivers(steps_done + steps);
    if (owned_dirty) build_owned_mask();
    if (use_fused() && fused_dirty) {
        build_fused();
        drop_graphs();
    }
    if (cap_dirty) {
        if (cap_every > 0) {
            const int32_t dims[3] = {nx, ny, nz};
            if (cap_batch < 0 || cap_batch >= prm.batch || cap_axis < 0 || cap_axis > 2 || cap_index < 0 ||
                cap_index >= dims[cap_axis])
                throw Error(AFD_ERR_ARG, "capture plane outside the grid");
            int64_t rows, cols;
            plane_dims(cap_axis, &rows, &cols);
            cap_frames.alloc((size_t)cap_max * rows * cols);
            cap_steps.alloc((size_t)cap_max);
            if (!cap_run0.ptr) cap_run0.alloc(2);
            cap = CaptureDev{cap_batch, cap_axis, cap_index, cap_every, cap_max, (int32_t)rows, (int32_t)cols,
                             cap_frames.ptr, cap_steps.ptr, cap_run0.ptr};
        }
        cap_total = 0;
        cap_dirty = false;
        drop_graphs();
    }
    if (tl_dirty) {
        if (tl_steps > 0) {
            const size_t n = (size_t)tl_steps * TL_SLOTS;
            tl_start.alloc(n);
            tl_end.alloc(n);
            CK(cudaMemsetAsync(tl_start.ptr, 0xff, n * sizeof(unsigned long long), stream));
            CK(cudaMemsetAsync(tl_end.ptr, 0, n * sizeof(unsigned long long), stream));
        }
        tl_dirty = false;
        drop_graphs();  // the kernels' arguments carry the timeline buffers
    }
    if (cap_every > 0) {
        const long long r0[2] = {(long long)steps_done, (long long)cap_total};
        CK(cudaMemcpyAsync(cap_run0.ptr, r0, sizeof(r0), cudaMemcpyHostToDevice, stream));
        CK(cudaStreamSynchronize(stream));
    }
    build_args();
}

// Chunks of a run: step 0 alone, then up to 200 steps (the progress
// points of simulation.hpp:403-409).
static std::vector<int64_t> run_chunks(int64_t steps) {
    std::vector<int64_t> out;
    for (int64_t i = 0; i < steps;) {
        const int64_t n = (i == 0) ? 1 : std::min<int64_t>(200, steps - i);
        out.push_back(n);
        i += n;
    }
    return out;
}

// The graphs of every chunk length of a run of `steps`, for the current
// plan and, while the autotuner still has candidates to try, for each of
// them, so that the run itself only replays graphs.
void Engine::prepare(int64_t steps) {
    Impl& D = *d_;
    D.setup_run(steps);
    if (!D.prm.graphs || D.prm.profile) return;
    D.ensure_candidates();
    std::vector<int64_t> lens = run_chunks(steps);
    std::sort(lens.begin(), lens.end());
    lens.erase(std::unique(lens.begin(), lens.end()), lens.end());
    if (D.tune_active() && D.tune_next < D.tune_cands.size()) {
        const int cur = D.plan_id;
        for (size_t c = D.tune_next; c < D.tune_cands.size(); ++c) {
            D.apply_plan((int)c + 1);
            for (int64_t n : lens) D.graph_for(n);
        }
        D.apply_plan(cur);
    }
    for (int64_t n : lens) D.graph_for(n);
}

int Engine::run(int64_t steps, afd_progress_fn cb, void* user) {
    Impl& D = *d_;
    D.setup_run(steps);
    D.ensure_candidates();
    if (D.tune_active() && !D.tev0) {
        CK(cudaEventCreate(&D.tev0));
        CK(cudaEventCreate(&D.tev1));
    }
    D.launches = 0;
    for (auto& st : D.kstats) {
        st.launches = 0;
        st.ms = 0.0;
    }
    CK(cudaMemsetAsync(D.d_flag.ptr, 0, sizeof(int), D.stream));
    CK(cudaEventRecord(D.ev0, D.stream));
    int status = AFD_OK;
    int64_t i = 0;
    while (i < steps) {
        const int64_t n = (i == 0) ? 1 : std::min<int64_t>(200, steps - i);
        // online autotuning: each full chunk of the first runs uses the next
        // candidate plan, timed on the device; then the fastest is kept
        const bool measure = D.tune_active() && n == 200 && D.tune_next < D.tune_cands.size();
        if (measure) {
            // the candidate's graph is captured, instantiated and uploaded
            // before the clock starts: host work inside the timed region
            // would leave the GPU idle and bias the choice
            D.apply_plan((int)D.tune_next + 1);
            CK(cudaGraphUpload(D.graph_for(n), D.stream));
            CK(cudaEventRecord(D.tev0, D.stream));
        }
        D.run_chunk(n);
        if (measure) CK(cudaEventRecord(D.tev1, D.stream));
        i += n;
        const int64_t last = i - 1;
        if (measure) {
            CK(cudaEventSynchronize(D.tev1));
            float ms = 0.0f;
            CK(cudaEventElapsedTime(&ms, D.tev0, D.tev1));
            D.tune_ms[D.tune_next++] = ms;
            if (D.tune_next == D.tune_cands.size()) {
                size_t best = 0;
                for (size_t c = 1; c < D.tune_ms.size(); ++c)
                    if (D.tune_ms[c] < D.tune_ms[best]) best = c;
                D.tuned = true;
                D.apply_plan((int)best + 1);
            }
        }
        if (D.ref() && D.args.pml.width > 0 && last % 8000 == 0) {
            const size_t bytes = (size_t)D.vol * D.prm.batch * sizeof(float);
            for (int a = 0; a < 3; ++a)
                for (int l = 0; l < 2; ++l) CK(cudaMemsetAsync(D.fi[a][l].ptr, 0, bytes, D.stream));
            CK(cudaMemsetAsync(D.psi[0].ptr, 0, bytes, D.stream));
            CK(cudaMemsetAsync(D.psi[1].ptr, 0, bytes, D.stream));
        }
        if (last % 200 == 0) {
            if (D.prm.profile) D.collect_profile();
            CK(cudaStreamSynchronize(D.stream));
            int flag = 0;
            CK(cudaMemcpy(&flag, D.d_flag.ptr, sizeof(int), cudaMemcpyDeviceToHost));
            if (flag & 2) {
                D.advance_done(i);
                throw Error(AFD_ERR_CUDA, "step kernel pipeline wait timed out");
            }
            if (flag && D.prm.watchdog) {
                D.advance_done(i);
                throw Error(AFD_ERR_NUMERIC, std::string(D.f16() ? "pressure left the FP16 storage range"
                                                                 : "pressure left the finite bound |p| < 1e30") +
                                                 " by step " + std::to_string(D.steps_done));
            }
            if (cb && cb(last, steps, user) != 0) {
                status = AFD_ERR_ABORTED;
                break;
            }
        }
    }
    CK(cudaEventRecord(D.ev1, D.stream));
    if (D.prm.profile) D.collect_profile();
    CK(cudaEventSynchronize(D.ev1));
    float ms = 0.0f;
    CK(cudaEventElapsedTime(&ms, D.ev0, D.ev1));
    D.last_ms = ms;
    CK(cudaGetLastError());
    int flag = 0;
    CK(cudaMemcpy(&flag, D.d_flag.ptr, sizeof(int), cudaMemcpyDeviceToHost));
    D.advance_done(i);
    if (flag & 2) throw Error(AFD_ERR_CUDA, "step kernel pipeline wait timed out");
    if (flag && D.prm.watchdog)
        throw Error(AFD_ERR_NUMERIC, std::string(D.f16() ? "pressure left the FP16 storage range"
                                                         : "pressure left the finite bound |p| < 1e30") +
                                         " by step " + std::to_string(D.steps_done));
    if (status == AFD_OK && cb) cb(steps, steps, user);
    return status;
}

void Engine::get_receivers(int32_t batch, float* out, int64_t cap) {
    Impl& D = *d_;
    if (batch < 0 || batch >= D.prm.batch) throw Error(AFD_ERR_ARG, "batch index out of range");
    const int64_t nr = (int64_t)D.receivers.size();
    const int64_t need = nr * D.steps_done;
    if (cap < need) throw Error(AFD_ERR_ARG, "output buffer too small: need " + std::to_string(need));
    if (need == 0) return;
    if (D.rcv_n_dev != nr) throw Error(AFD_ERR_STATE, "receivers were added after the last run");
    CK(cudaSetDevice(D.device));
    float* stage = D.pinned_floats((size_t)need);
    CK(cudaMemcpy2DAsync(stage, D.steps_done * sizeof(float),
                         D.rcv_out.ptr + (size_t)batch * nr * D.rcv_cap, D.rcv_cap * sizeof(float),
                         D.steps_done * sizeof(float), (size_t)nr, cudaMemcpyDeviceToHost, D.stream));
    CK(cudaStreamSynchronize(D.stream));
    std::memcpy(out, stage, (size_t)need * sizeof(float));
}

void Engine::get_receivers_range(int32_t batch, int64_t t0, int64_t t1, float* out, int64_t cap) {
    Impl& D = *d_;
    if (batch < 0 || batch >= D.prm.batch) throw Error(AFD_ERR_ARG, "batch index out of range");
    if (t0 < 0 || t1 < t0 || t1 > D.steps_done) throw Error(AFD_ERR_ARG, "time range outside the run");
    const int64_t nr = (int64_t)D.receivers.size();
    const int64_t n = t1 - t0;
    if (cap < nr * n) throw Error(AFD_ERR_ARG, "output buffer too small");
    if (nr == 0 || n == 0) return;
    if (D.rcv_n_dev != nr) throw Error(AFD_ERR_STATE, "receivers were added after the last run");
    CK(cudaSetDevice(D.device));
    // one strided copy into page-locked staging (a strided copy into
    // pageable memory goes row by row), then into the caller's buffer
    float* stage = D.pinned_floats((size_t)(nr * n));
    CK(cudaMemcpy2DAsync(stage, n * sizeof(float), D.rcv_out.ptr + (size_t)batch * nr * D.rcv_cap + t0,
                         D.rcv_cap * sizeof(float), n * sizeof(float), (size_t)nr, cudaMemcpyDeviceToHost,
                         D.stream));
    CK(cudaStreamSynchronize(D.stream));
    std::memcpy(out, stage, (size_t)(nr * n) * sizeof(float));
}

// Replaces samples t0.. of one source. When the device copy already holds
// the source at a sufficient length the new samples are copied in place
// (stream-ordered with the steps already queued); otherwise the source
// list is rebuilt at the next run.
void Engine::update_source(int64_t index, int64_t t0, const float* sig, int64_t len) {
    Impl& D = *d_;
    if (index < 0 || index >= (int64_t)D.sources.size()) throw Error(AFD_ERR_ARG, "source index out of range");
    if (t0 < 0) throw Error(AFD_ERR_ARG, "t0 must be >= 0");
    Source& s = D.sources[(size_t)index];
    const bool grows = (int64_t)s.sig.size() < t0 + len;
    if (grows) s.sig.resize((size_t)(t0 + len), 0.0f);
    std::copy(sig, sig + len, s.sig.begin() + t0);
    if (grows || D.src_dirty || !D.src_data.ptr) {
        D.src_dirty = true;
        return;
    }
    if (D.f16() && D.f16_smax.ptr && (size_t)s.batch < D.smax_host.size()) {
        // the scale rule's source maximum follows larger new samples from
        // the next queued step on
        float& cur = D.smax_host[(size_t)s.batch];
        float m = cur;
        for (int64_t k = 0; k < len; ++k) m = std::max(m, std::fabs(sig[k]));
        if (m > cur) {
            cur = m;
            CK(cudaSetDevice(D.device));
            CK(cudaMemcpyAsync(D.f16_smax.ptr + s.batch, &cur, 4, cudaMemcpyHostToDevice, D.stream));
        }
    }
    // device position of this source: sources are stored grouped by batch member
    int64_t off = 0;
    for (int32_t b = 0; b < D.prm.batch; ++b)
        for (const Source& q : D.sources) {
            if (q.batch != b) continue;
            if (&q == &s) {
                CK(cudaSetDevice(D.device));
                CK(cudaMemcpyAsync(D.src_data.ptr + off + t0, sig, (size_t)len * sizeof(float),
                                   cudaMemcpyHostToDevice, D.stream));
                return;
            }
            off += (int64_t)q.sig.size();
        }
}

// The newest level of one member as FP32 values on the device (FP16
// storage: decoded into a scratch buffer).
static const float* latest_field(Engine::Impl& D, int32_t batch) {
    if (D.steps_done == 0) return nullptr;
    const long long g = D.steps_done - 1;
    if (!D.f16()) return D.fields.ptr + (size_t)buf_new(g) * D.vol * D.prm.batch + (size_t)batch * D.vol;
    const __half* h = reinterpret_cast<const __half*>(D.fields.ptr) + (size_t)buf_new(g) * D.vol * D.prm.batch +
                      (size_t)batch * D.vol;
    if (D.decoded.n != (size_t)D.vol) D.decoded.alloc((size_t)D.vol);
    const float inv = 1.0f / D.host_level_scale(batch, g);
    k_decode<<<1184, 256, 0, D.stream>>>(h, D.decoded.ptr, D.vol, inv);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(D.stream));
    return D.decoded.ptr;
}

void Engine::get_field(int32_t batch, float* out, int64_t cap) {
    Impl& D = *d_;
    if (!D.initialized) throw Error(AFD_ERR_STATE, "no field before the first run");
    if (batch < 0 || batch >= D.prm.batch) throw Error(AFD_ERR_ARG, "batch index out of range");
    const int64_t need = (int64_t)D.nx * D.ny * D.nz;
    if (cap < need) throw Error(AFD_ERR_ARG, "output buffer too small");
    CK(cudaSetDevice(D.device));
    CK(cudaStreamSynchronize(D.stream));
    const float* f = latest_field(D, batch);
    if (!f) {
        std::fill(out, out + need, 0.0f);
        return;
    }
    CK(cudaMemcpy2D(out, D.nx * sizeof(float), f, D.pitch * sizeof(float), D.nx * sizeof(float),
                    (size_t)D.ny * D.nz, cudaMemcpyDeviceToHost));
}

void Engine::set_capture(int32_t batch, int32_t axis, int32_t index, int32_t every, int32_t max_frames) {
    Impl& D = *d_;
    if (every > 0 && (max_frames < 1 || max_frames > 1 << 20)) throw Error(AFD_ERR_ARG, "max_frames must be in 1..2^20");
    if (axis < 0 || axis > 2) throw Error(AFD_ERR_ARG, "axis must be 0, 1 or 2");
    D.cap_batch = batch;
    D.cap_axis = axis;
    D.cap_index = index;
    D.cap_every = every > 0 ? every : 0;
    D.cap_max = every > 0 ? max_frames : 0;
    D.cap_dirty = true;
}

void Engine::set_timeline(int64_t first, int32_t steps) {
    Impl& D = *d_;
    if (steps > 4096) throw Error(AFD_ERR_ARG, "timeline steps must be at most 4096");
    if (first < 0) throw Error(AFD_ERR_ARG, "first step must be >= 0");
    D.tl_first = first;
    D.tl_steps = steps > 0 ? steps : 0;
    D.tl_dirty = true;
}

int32_t Engine::get_timeline(double* out, int64_t cap) {
    Impl& D = *d_;
    if (D.tl_steps <= 0 || D.tl_dirty || !D.tl_start.ptr) return 0;
    const size_t n = (size_t)D.tl_steps * TL_SLOTS;
    if (out && cap < (int64_t)(2 * n)) throw Error(AFD_ERR_ARG, "output buffer too small: need " + std::to_string(2 * n));
    CK(cudaSetDevice(D.device));
    CK(cudaStreamSynchronize(D.stream));
    std::vector<unsigned long long> st(n), en(n);
    CK(cudaMemcpy(st.data(), D.tl_start.ptr, n * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(en.data(), D.tl_end.ptr, n * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
    unsigned long long t0 = ~0ull;
    for (size_t k = 0; k < n; ++k) t0 = std::min(t0, st[k]);
    if (out)
        for (size_t k = 0; k < n; ++k) {
            const bool ok = st[k] != ~0ull && en[k] >= st[k];
            out[2 * k] = ok ? (double)(st[k] - t0) : -1.0;
            out[2 * k + 1] = ok ? (double)(en[k] - t0) : -1.0;
        }
    return D.tl_steps;
}

int32_t Engine::get_frames(float* out, int64_t cap, int64_t* steps, int64_t steps_cap) {
    Impl& D = *d_;
    if (D.cap_every <= 0 || !D.cap_frames.ptr || D.cap_dirty) return 0;
    const int64_t n = std::min<int64_t>(D.cap_total, D.cap_max);
    const int64_t fsz = (int64_t)D.cap.rows * D.cap.cols;
    if (out && cap < n * fsz) throw Error(AFD_ERR_ARG, "output buffer too small: need " + std::to_string(n * fsz));
    if (steps && steps_cap < n) throw Error(AFD_ERR_ARG, "steps buffer too small");
    CK(cudaSetDevice(D.device));
    CK(cudaStreamSynchronize(D.stream));
    std::vector<long long> st((size_t)D.cap_max);
    CK(cudaMemcpy(st.data(), D.cap_steps.ptr, st.size() * sizeof(long long), cudaMemcpyDeviceToHost));
    for (int64_t k = 0; k < n; ++k) {
        const int64_t slot = (D.cap_total - n + k) % D.cap_max;  // oldest first
        if (out)
            CK(cudaMemcpy(out + k * fsz, D.cap_frames.ptr + slot * fsz, (size_t)fsz * sizeof(float),
                          cudaMemcpyDeviceToHost));
        if (steps) steps[k] = st[(size_t)slot];
    }
    return (int32_t)n;
}

void Engine::get_plane(int32_t batch, int32_t axis, int32_t index, float* out, int64_t cap) {
    Impl& D = *d_;
    if (!D.initialized) throw Error(AFD_ERR_STATE, "no field before the first run");
    if (batch < 0 || batch >= D.prm.batch) throw Error(AFD_ERR_ARG, "batch index out of range");
    const int32_t dims[3] = {D.nx, D.ny, D.nz};
    if (axis < 0 || axis > 2 || index < 0 || index >= dims[axis]) throw Error(AFD_ERR_ARG, "bad plane");
    CK(cudaSetDevice(D.device));
    CK(cudaStreamSynchronize(D.stream));
    const float* f = latest_field(D, batch);
    int64_t rows, cols;
    if (axis == 0) { rows = D.nz; cols = D.ny; }
    else if (axis == 1) { rows = D.nz; cols = D.nx; }
    else { rows = D.ny; cols = D.nx; }
    if (cap < rows * cols) throw Error(AFD_ERR_ARG, "output buffer too small");
    if (!f) {
        std::fill(out, out + rows * cols, 0.0f);
        return;
    }
    if (axis == 1) {
        // copy_plane.cl:29-34: to[x, z] = from[x, level, z]
        CK(cudaMemcpy2D(out, D.nx * sizeof(float), f + (size_t)index * D.pitch, D.plane * sizeof(float),
                        D.nx * sizeof(float), (size_t)D.nz, cudaMemcpyDeviceToHost));
    } else if (axis == 2) {
        CK(cudaMemcpy2D(out, D.nx * sizeof(float), f + (size_t)index * D.plane, D.pitch * sizeof(float),
                        D.nx * sizeof(float), (size_t)D.ny, cudaMemcpyDeviceToHost));
    } else {
        CK(cudaMemcpy2D(out, sizeof(float), f + index, D.pitch * sizeof(float), sizeof(float),
                        (size_t)D.ny * D.nz, cudaMemcpyDeviceToHost));
    }
}

void Engine::get_info(afd_info* info) {
    Impl& D = *d_;
    std::memset(info, 0, sizeof(*info));
    int32_t dims[3];
    D.grid_dims(dims);
    info->nx = dims[0];
    info->ny = dims[1];
    info->nz = dims[2];
    info->ncoef = D.have_model ? D.model.ncoef : 0;
    info->nmat = D.have_model ? D.model.nmat : 0;
    info->batch = D.prm.batch;
    info->steps_done = D.steps_done;
    info->n_sources = (int64_t)D.sources.size();
    info->n_receivers = (int64_t)D.receivers.size();
    info->n_boundary = (int64_t)D.boundary.size();
    for (int g = 0; g < kNumGroups; ++g) info->group_counts[g] = D.boundary_counts[g];
    info->n_pml_cells = D.n_pml_cells;
    info->lambda2 = D.lambda2();
    info->mode = D.prm.mode;
    info->storage = D.prm.storage;
    info->last_run_ms = D.last_ms;
    info->kernel_launches = D.launches;
    info->tile_x = D.tile_w;
    info->tile_y = D.tile_h;
    info->tile_z = D.fdev.dz;
    info->stream_blocks = D.fused_grid;
    info->stream_beside = D.lists_beside() ? 1 : 0;
    info->stream_per_sm = D.stream_per_sm;
    info->stream_tail = D.tail_active() ? 1 : 0;
    info->tuned = D.tuned ? 1 : 0;
}

int Engine::kernel_stats(int32_t idx, char* name, int64_t cap, int64_t* launches, double* ms) {
    Impl& D = *d_;
    if (idx < 0 || idx >= (int32_t)D.kstats.size()) return AFD_ERR_ARG;
    const KernelStat& st = D.kstats[(size_t)idx];
    if (name && cap > 0) {
        std::strncpy(name, st.name.c_str(), (size_t)cap - 1);
        name[cap - 1] = '\0';
    }
    if (launches) *launches = st.launches;
    if (ms) *ms = st.ms;
    return AFD_OK;
}

double Engine::energy(int32_t batch) {
    Impl& D = *d_;
    if (!D.initialized) throw Error(AFD_ERR_STATE, "no field before the first run");
    if (batch < 0 || batch >= D.prm.batch) throw Error(AFD_ERR_ARG, "batch index out of range");
    if (D.steps_done == 0) return 0.0;
    CK(cudaSetDevice(D.device));
    const long long g = D.steps_done - 1;
    const size_t base = (size_t)batch * D.vol;
    const size_t stride = (size_t)D.vol * D.prm.batch;
    CK(cudaMemsetAsync(D.d_energy.ptr, 0, sizeof(double), D.stream));
    const dim3 blk(64, 4, 1);
    const dim3 grd((unsigned)((D.nx - 2 + 63) / 64), (unsigned)((D.ny - 2 + 3) / 4), (unsigned)(D.nz - 2));
    const GridDev gd{D.nx, D.ny, D.nz, D.pitch, D.plane, D.vol};
    if (D.f16()) {
        const __half* h = reinterpret_cast<const __half*>(D.fields.ptr);
        const float inv1 = 1.0f / D.host_level_scale(batch, g), inv0 = 1.0f / D.host_level_scale(batch, g - 1);
        k_energy<__half><<<grd, blk, 0, D.stream>>>(h + (size_t)buf_new(g) * stride + base,
                                                    h + (size_t)buf_cur(g) * stride + base, inv1, inv0, gd,
                                                    D.solid_view(), (double)D.lambda2(), D.d_energy.ptr);
    } else {
        k_energy<float><<<grd, blk, 0, D.stream>>>(D.fields.ptr + (size_t)buf_new(g) * stride + base,
                                                   D.fields.ptr + (size_t)buf_cur(g) * stride + base, 1.0f, 1.0f,
                                                   gd, D.solid_view(), (double)D.lambda2(), D.d_energy.ptr);
    }
    CK(cudaGetLastError());
    double e = 0.0;
    CK(cudaMemcpyAsync(&e, D.d_energy.ptr, sizeof(double), cudaMemcpyDeviceToHost, D.stream));
    CK(cudaStreamSynchronize(D.stream));
    return e;
}

}  // namespace afd
