// Device-side data layout and the per-cell update arithmetic shared by the
// step kernels. Every expression keeps the evaluation order of the
// reference OpenCL kernels it restates; the engine is compiled with
// -fmad=false so no multiply-add contraction changes a rounding, which makes
// the FP32 results reproducible operation by operation on the CPU.
#pragma once

#include <cstdint>
#include <cstring>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

namespace afd {

// Field layout of one batch member: x-fastest rows padded to `pitch`
// floats, index = z*plane + y*pitch + x.
struct GridDev {
    int32_t nx, ny, nz;
    int64_t pitch, plane, vol;
};

// Compact boundary (LRS) list. Entry e: linear cell index, packed info
// (group | mat0 << 5 | mat1 << 13 | mat2 << 21) and filter state
// st_in/st_out[(b*S + slot)*n + e], S = 3*K slots per entry.
struct LrsDev {
    int32_t n;
    int32_t K, S;
    const int32_t* cell;
    const uint32_t* info;
    float* st_in;
    float* st_out;
    const float* ca;  // [nmat][K]
    const float* cb;  // [nmat][K]
    float l, l2, c2;  // coefficient l, l*l and 2(1-3*l*l)
};

// One dense box of PML work (FIXED mode): 4-cell units in x starting at
// x0, rows y0.., planes z0..; `first` is the running unit count before it.
struct PmlBox {
    int32_t x0, units, y0, height, z0, depth;
    int64_t first;
};
constexpr int kMaxPmlBoxes = 6;

// PML state. Full-grid auxiliary fields (two time levels each) per batch
// member; ksi profiles padded with zeros to kmax entries.
struct PmlDev {
    int32_t width;     // 0: PML off
    uint32_t faces;    // FIXED-mode face mask
    int64_t g0;        // global step at which the PML was enabled
    float* fi[3][2];   // [axis][level]
    float* psi[2];
    const float* ksi[3];
    // scalars, each computed on the host in FP32 exactly as the reference
    // kernel expression would compute it (pml.cl:185-262)
    float dt, cc_dxdx, inv_dx, half_inv_dx, inv_dt2, two_dt, inv_dt;
    int32_t psi_on;    // psi is kept (REF always; FIXED with faces on all three axes)
    // FIXED mode: disjoint boxes covering the slabs, and a 1-bit mask of the
    // PML cells (plain air, not boundary, inside 2..n-3 and an enabled
    // slab), pitch/32 words per row
    int32_t n_boxes;
    PmlBox boxes[kMaxPmlBoxes];
    int64_t n_units;
    const uint32_t* cells;
    int32_t words_per_row;
    // z-slab of a larger grid: local plane z is global plane z + zoff of
    // nz_glob planes; the PML cell rule and the z slabs use global planes
    int32_t zoff, nz_glob;
};

struct SrcDev {
    int32_t n;
    const int32_t* cell;
    const int32_t* begin;   // [batch+1] range of sources of each member
    const int64_t* off;
    const int64_t* len;
    const float* data;
};

struct RcvDev {
    int32_t n;
    const int32_t* cell;
    float* out;      // [batch][n][cap]
    int64_t cap;
};

// FP16 field storage (AFD_STORE_FP16, FIXED scheme): the three levels as
// binary16 holding p * s, one power-of-two scale s per stored level and
// batch member. The scale of level L (written at global step L) follows
// from the largest magnitude of level L - 2, which the interior kernel of
// step L - 1 gathers while it reads that level as p^n (no extra pass):
// mx[b * 5 + slot(L)] holds the float bits of max |level L| (atomicMax),
// slot(L) = L mod 5. Step g gathers slot g - 1, reads slots g - 2 .. g - 4
// and clears slot g for the next step.
struct F16Dev {
    __half* h[3];             // the three levels, each [batch][vol]
    uint32_t* mx;             // [batch][5]
    const float* src_max;     // [batch] largest |source sample| of the member
};

struct StepArgs {
    GridDev g;
    int32_t batch;
    int32_t mode;             // AFD_MODE_REF / AFD_MODE_FIXED
    float* p[3];              // three rotating field buffers, each [batch][vol]
    F16Dev f16;
    const long long* d_step;  // global step index at the start of the chunk
    float lambda2, cint;      // interior: lambda^2 and 2(1-3 lambda^2)
    LrsDev lrs;
    PmlDev pml;
    SrcDev src;
    RcvDev rcv;
    int* flag;                // watchdog flag (bit0: |p| left the bound)
    // step timeline (off when tl_start is null): for global steps
    // tl_g0 .. tl_g0 + tl_steps - 1 and each of TL_SLOTS kernel kinds, the
    // start of the first and the end of the last recording block (%globaltimer)
    unsigned long long* tl_start;
    unsigned long long* tl_end;
    long long tl_g0;
    int32_t tl_steps;
};

// Timeline slots: streaming or interior kernel, boundary, PML pressure,
// PML auxiliary x, y, z, source/receiver.
constexpr int TL_SLOTS = 7;

// Marks one block of a kernel in the step timeline: thread 0 of a recording
// block takes the start at construction and the end when it leaves the
// kernel (every return path). `rec`: the block belongs to batch member 0
// (the kernels with one block column per member) or to every member.
struct TlMark {
    unsigned long long* end = nullptr;
    __device__ __forceinline__ static unsigned long long now() {
        unsigned long long t;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        return t;
    }
    __device__ __forceinline__ TlMark(const StepArgs& a, int slot, long long g, bool rec) {
        if (!a.tl_start || !rec || (threadIdx.x | threadIdx.y | threadIdx.z)) return;
        const long long d = g - a.tl_g0;
        if (d < 0 || d >= a.tl_steps) return;
        const size_t k = (size_t)d * TL_SLOTS + slot;
        atomicMin(a.tl_start + k, now());
        end = a.tl_end + k;
    }
    __device__ __forceinline__ ~TlMark() {
        if (end) atomicMax(end, now());
    }
};

// Buffer roles of global step g, following the pointer rotation of
// simulation.hpp:360 (three buffers rotated right by one per step):
// the new level is written into buffer (2 + 2g) mod 3.
__host__ __device__ inline int buf_new(long long g) { return (int)((2 + 2 * (g % 3)) % 3); }
__host__ __device__ inline int buf_cur(long long g) { return (buf_new(g) + 1) % 3; }
__host__ __device__ inline int buf_old(long long g) { return (buf_new(g) + 2) % 3; }

// Ring slot written at global step g (simulation.hpp:365: decremented
// before every step, starting from 0).
__host__ __device__ inline int ring_index(long long g, int K) { return K - 1 - (int)(g % K); }

// ---- FP16 storage ----------------------------------------------------------
__host__ __device__ inline int max_slot(long long L) { return (int)(((L % 5) + 5) % 5); }

// Scale of a level from the largest magnitude m of the level two steps
// before it and the member's largest source sample smax: 2^(10 - e) with
// m' = max(m, smax) < 2^e (frexp's exponent), 1 when m' is 0, exponent
// clamped to [-60, 60]. The 2^6 headroom below the binary16 maximum covers
// the growth of two steps.
__host__ __device__ inline int level_scale_exp(uint32_t mbits, float smax) {
    float m;
    memcpy(&m, &mbits, 4);
    const float a = m > smax ? m : smax;
    if (!(a > 0.0f)) return 0;
    uint32_t ab;
    memcpy(&ab, &a, 4);
    const int e = (int)((ab >> 23) & 0xffu) - 126;  // frexp exponent of a normal a
    const int k = 10 - e;
    return k > 60 ? 60 : (k < -60 ? -60 : k);
}

// 2^k for |k| <= 60 (a normal float, built from its exponent bits).
__host__ __device__ inline float pow2_exact(int k) {
    const uint32_t sb = (uint32_t)(k + 127) << 23;
    float v;
    memcpy(&v, &sb, 4);
    return v;
}

__host__ __device__ inline float level_scale(uint32_t mbits, float smax) {
    return pow2_exact(level_scale_exp(mbits, smax));
}

// Scales of the levels step g reads and writes for member b.
struct StepScales {
    float s_new, inv_new;  // level g
    float s_cur, inv_cur;  // level g - 1 (p^n)
    float s_old, inv_old;  // level g - 2 (p^{n-1})
};

// Slot load through L2 only (ld.global.cg): the slots are written inside
// the same CUDA graph by the interior kernels of earlier steps (step g
// writes slot g-1 and clears slot g) while other kernels of a step may read
// the neighbouring slots of the same sector, so they are never read through
// the SM's non-coherent read-only cache, which could keep a sector fetched
// before its slots were final.
__device__ __forceinline__ uint32_t ld_slot(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.global.cg.u32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}

// Scales of levels g, g-1, g-2 from the slots of levels g-2..g-4. 1/s is
// 2^-k exactly (what 1.0f / s gives for a power of two).
__device__ __forceinline__ StepScales step_scales(const F16Dev& f, int b, long long g) {
    const uint32_t* mx = f.mx + (size_t)b * 5;
    const float smax = __ldg(f.src_max + b);
    const int kn = level_scale_exp(ld_slot(mx + max_slot(g - 2)), smax);
    const int kc = level_scale_exp(ld_slot(mx + max_slot(g - 3)), smax);
    const int ko = level_scale_exp(ld_slot(mx + max_slot(g - 4)), smax);
    StepScales s;
    s.s_new = pow2_exact(kn);
    s.s_cur = pow2_exact(kc);
    s.s_old = pow2_exact(ko);
    s.inv_new = pow2_exact(-kn);
    s.inv_cur = pow2_exact(-kc);
    s.inv_old = pow2_exact(-ko);
    return s;
}

// Loads and stores of a level as FP32 values: FP32 storage reads and
// writes the value; FP16 storage decodes with 1/s and encodes v * s
// (round to nearest even, exact scaling by a power of two).
template <typename T>
__device__ __forceinline__ float fld(const T* p, float inv) {
    if constexpr (sizeof(T) == 4) {
        (void)inv;
        return *p;
    } else {
        return __half2float(*p) * inv;
    }
}

template <typename T>
__device__ __forceinline__ float fldg(const T* p, float inv) {
    if constexpr (sizeof(T) == 4) {
        (void)inv;
        return __ldg(p);
    } else {
        return __half2float(__ldg(p)) * inv;
    }
}

template <typename T>
__device__ __forceinline__ void fst(T* p, float v, float s) {
    if constexpr (sizeof(T) == 4) {
        (void)s;
        *p = v;
    } else {
        *p = __float2half_rn(v * s);
    }
}

// A stored FP16 value is finite when |v * s| < 65520 (binary16 overflow
// threshold under round to nearest even).
__device__ __forceinline__ bool f16_finite(float scaled) { return fabsf(scaled) < 65520.0f; }

template <typename T>
__device__ __forceinline__ T* level_ptr(const StepArgs& a, int buf) {
    if constexpr (sizeof(T) == 4) return a.p[buf];
    else return a.f16.h[buf];
}

// Interior SLF update, leapfrog.cl:41-53.
__device__ __forceinline__ float slf_update(float lambda2, float cint, float xp, float xm, float yp,
                                            float ym, float zp, float zm, float c, float old) {
    float s = xp + xm;
    s = s + yp;
    s = s + ym;
    s = s + zp;
    s = s + zm;
    return lambda2 * s + cint * c - old;
}

// The same update for FP16 storage, on stored values: c, the six
// neighbours and old are p^n * s_cur and p^{n-1} * s_old; rc = s_new /
// s_cur and ro = s_new / s_old are powers of two, so each operation equals
// its unscaled counterpart times s_new exactly. Evaluated as
// p + ((p - p^{n-1}) + lambda^2 (S - 6p)): the increment is formed before
// it is added to the level.
__device__ __forceinline__ float slf_update_scaled(float lambda2, float rc, float ro, float xp, float xm,
                                                   float yp, float ym, float zp, float zm, float c,
                                                   float old) {
    float s = xp + xm;
    s = s + yp;
    s = s + ym;
    s = s + zp;
    s = s + zm;
    const float S = s * rc, p = c * rc, o = old * ro;
    return p + ((p - o) + lambda2 * (S - 6.0f * p));
}

// Neighbour sum of a boundary cell: axes in x, y, z order; a wall on the +
// side contributes 2*p(-1), on the - side 2*p(+1), none p(+1) + p(-1)
// (lrs_1.cl:80-120, lrs_2.cl:89-207, lrs_3.cl:96-174).
__device__ __forceinline__ float lrs_neighbour_sum(unsigned mask, const float nb[6]) {
    // nb: p at x+1, x-1, y+1, y-1, z+1, z-1
    float s;
    bool first = true;
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        float t0, t1;
        int n;
        if (mask & (1u << (2 * ax))) {          // wall on the + side
            t0 = 2.0f * nb[2 * ax + 1];
            n = 1;
        } else if (mask & (1u << (2 * ax + 1))) {  // wall on the - side
            t0 = 2.0f * nb[2 * ax];
            n = 1;
        } else {
            t0 = nb[2 * ax];
            t1 = nb[2 * ax + 1];
            n = 2;
        }
        if (first) {
            s = t0;
            first = false;
        } else {
            s = s + t0;
        }
        if (n == 2) s = s + t1;
    }
    return s;
}

__constant__ uint8_t c_group_mask[26];

// One boundary point update. Returns p^{n+1} of the cell and writes the
// filter state of every face. `pint` is the interior (leapfrog) value of
// the cell, kept by the corner group that the reference never updates
// (group 25 in REF mode). `pc`, `pold`: p^n and p^{n-1} of the cell.
// REF semantics: lrs_1.cl:61-124, lrs_2.cl:61-215, lrs_3.cl:61-186 with the
// host call of simulation.hpp:368-369. FIXED: l is the Courant number,
// corners use all three filters with a ring of K slots each, group 25 is a
// regular corner.
// KT > 0 fixes the filter length at compile time (the tap loop unrolls and
// all state loads issue together); KT = 0 reads it from L.K.
template <bool REF, int KT = 0>
__device__ __forceinline__ float lrs_point(const LrsDev& L, int e, int b, uint32_t info,
                                           const float nb[6], float pc, float pold, float pint,
                                           int ix_buf) {
    const int group = (int)(info & 31u);
    const int nf = group < 6 ? 1 : (group < 18 ? 2 : 3);
    const int K = KT > 0 ? KT : L.K;
    int mat[3] = {(int)((info >> 5) & 255u), (int)((info >> 13) & 255u), (int)((info >> 21) & 255u)};
    // ring width per filter: K, except REF corners (lrs_3.cl:70, size_a_0/2)
    const int size_f = (REF && nf == 3) ? K / 2 : K;
    const size_t n = (size_t)L.n;
    float* sin_ = L.st_in + (size_t)b * L.S * n + e;
    float* sout = L.st_out + (size_t)b * L.S * n + e;

    float a0[3], b0[3], gn[3];
#pragma unroll
    for (int f = 0; f < 3; ++f) {
        gn[f] = 0.0f;
        a0[f] = 1.0f;
        b0[f] = 1.0f;
        if (f < nf) {
            a0[f] = __ldg(L.ca + mat[f] * K);
            b0[f] = __ldg(L.cb + mat[f] * K);
        }
    }
    auto tap = [&](int i) {
#pragma unroll
        for (int f = 0; f < 3; ++f) {
            if (f < nf) {
                const int slot = (ix_buf + i) % size_f + f * size_f;
                const float bi = __ldg(L.cb + mat[f] * K + i);
                const float ai = __ldg(L.ca + mat[f] * K + i);
                gn[f] += bi * sin_[(size_t)slot * n] - ai * sout[(size_t)slot * n];
            }
        }
    };
    if constexpr (KT > 0) {
#pragma unroll
        for (int i = 1; i < KT; ++i) tap(i);
    } else {
        for (int i = 1; i < K; ++i) tap(i);
    }

    const float l = L.l, l2 = L.l2;
    const float S = lrs_neighbour_sum(c_group_mask[group], nb);
    float pn;
    if (nf == 1) {
        pn = (l2 * S + L.c2 * pc + l2 / b0[0] * gn[0] + (l * a0[0] / b0[0] - 1.0f) * pold) /
             (1.0f + l * a0[0] / b0[0]);
    } else if (nf == 2 || REF) {
        if (REF && group == 25) {
            pn = pint;  // no variant define reaches lrs_3.cl for this group
        } else {
            pn = (l2 * S + l2 * (gn[0] / b0[0] + gn[1] / b0[1]) + L.c2 * pc +
                  (l * a0[0] / b0[0] + l * a0[1] / b0[1] - 1.0f) * pold) /
                 (1.0f + l * a0[0] / b0[0] + l * a0[1] / b0[1]);
        }
    } else {
        pn = (l2 * S + l2 * (gn[0] / b0[0] + gn[1] / b0[1] + gn[2] / b0[2]) + L.c2 * pc +
              (l * a0[0] / b0[0] + l * a0[1] / b0[1] + l * a0[2] / b0[2] - 1.0f) * pold) /
             (1.0f + l * a0[0] / b0[0] + l * a0[1] / b0[1] + l * a0[2] / b0[2]);
    }
#pragma unroll
    for (int f = 0; f < 3; ++f) {
        if (f < nf) {
            const float xn = a0[f] / (l * b0[f]) * (pn - pold) - gn[f] / b0[f];
            const int slot = ix_buf + f * size_f;
            sin_[(size_t)slot * n] = xn;
            sout[(size_t)slot * n] = 1.0f / a0[f] * (b0[f] * xn + gn[f]);
        }
    }
    return pn;
}

// Boundary cell with one solid neighbour in direction d (groups 0-5,
// lrs_1.cl:61-124): the same arithmetic as lrs_point for one filter, with
// the neighbour sum and the ring slots resolved without the general
// pattern handling.
template <int KT>
__device__ __forceinline__ float lrs_face(const LrsDev& L, int e, int b, int d, int mat, const float nb[6],
                                          float pc, float pold, int ix_buf) {
    const int K = KT > 0 ? KT : L.K;
    const size_t n = (size_t)L.n;
    float* sin_ = L.st_in + (size_t)b * L.S * n + e;
    float* sout = L.st_out + (size_t)b * L.S * n + e;
    const float* ca = L.ca + mat * K;
    const float* cb = L.cb + mat * K;
    const float a0 = __ldg(ca), b0 = __ldg(cb);
    float gn = 0.0f;
    auto tap = [&](int i) {
        int s = ix_buf + i;
        if (s >= K) s -= K;
        gn += __ldg(cb + i) * sin_[(size_t)s * n] - __ldg(ca + i) * sout[(size_t)s * n];
    };
    if constexpr (KT > 0) {
#pragma unroll
        for (int i = 1; i < KT; ++i) tap(i);
    } else {
        for (int i = 1; i < K; ++i) tap(i);
    }
    // nb: x+1, x-1, y+1, y-1, z+1, z-1; the wall side's term is replaced by
    // twice the opposite neighbour, axes summed in x, y, z order
    float S;
    if (d < 2) {
        S = 2.0f * nb[d == 0 ? 1 : 0];
        S = S + nb[2];
        S = S + nb[3];
        S = S + nb[4];
        S = S + nb[5];
    } else if (d < 4) {
        S = nb[0] + nb[1];
        S = S + 2.0f * nb[d == 2 ? 3 : 2];
        S = S + nb[4];
        S = S + nb[5];
    } else {
        S = nb[0] + nb[1];
        S = S + nb[2];
        S = S + nb[3];
        S = S + 2.0f * nb[d == 4 ? 5 : 4];
    }
    const float l = L.l, l2 = L.l2;
    const float pn = (l2 * S + L.c2 * pc + l2 / b0 * gn + (l * a0 / b0 - 1.0f) * pold) / (1.0f + l * a0 / b0);
    const float xn = a0 / (l * b0) * (pn - pold) - gn / b0;
    sin_[(size_t)ix_buf * n] = xn;
    sout[(size_t)ix_buf * n] = 1.0f / a0 * (b0 * xn + gn);
    return pn;
}

}  // namespace afd
