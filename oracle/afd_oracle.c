/*
 * afd_oracle.c - CPU restatement of the anc-field FDTD time step.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the checker the parity tests,
 * __graft_entry__.smoke() and the CPU-baseline leg of bench.py compare the
 * CUDA engine against; the product path never calls it.
 *
 * It restates, in plain C with OpenMP, the per-step sequence of
 * Simulation::Run (anc-field/src/simulation.hpp:342-434) and the kernels it
 * launches:
 *   leapfrog.cl:34-55          interior standard-leapfrog update
 *   lrs_1.cl:49-125            boundary cells with one solid neighbour
 *   lrs_2.cl:49-216            ... two solid neighbours
 *   lrs_3.cl:49-187            ... three solid neighbours
 *   pml.cl:74-265              PML pressure and auxiliary fields
 *   source.cl:32-40, mic.cl:32-41
 * Two semantics (mode): 0 = REF, the reference kernels' arithmetic with its
 * quirks (l = lambda^2 in the boundary kernels, the corner kernel's ring
 * index and unused third filter, the X_M_Y_M_Z_M corner left at its
 * leapfrog value, the PML over the whole interior with the derivative and
 * ksi typos, the 8000-step PML reset); 1 = FIXED, the intended scheme.
 * Every expression keeps the reference's evaluation order; built with
 * -ffp-contract=off the FP32 build rounds exactly as the kernels specify.
 *
 * The same source compiled with -DORA_REAL=double is the FP64 version of
 * each scheme. The FP32 build also exports ora_simulate_f16, the FIXED
 * scheme with FP16 field storage (the engine's AFD_STORE_FP16 option, which
 * has no counterpart in the reference): FP32 arithmetic on values that are
 * rounded to binary16 times a power-of-two scale whenever a pressure level
 * is stored, the scale of each level chosen by level_scale() below.
 *
 * Parity of this restatement is pinned against the reference's own kernel
 * sources compiled in oracle/ref_harness.c (outputs under oracle/_ref/).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifndef ORA_REAL
#define ORA_REAL float
#endif
typedef ORA_REAL real;

/* ---- FP16 storage ------------------------------------------------------
 * IEEE 754 binary32 -> binary16 with round to nearest even, and back. */
static inline uint16_t f32_to_f16(float f) {
    uint32_t x;
    memcpy(&x, &f, 4);
    const uint32_t sign = (x >> 16) & 0x8000u, ax = x & 0x7fffffffu;
    if (ax > 0x7f800000u) return (uint16_t)(sign | 0x7e00u);     /* NaN */
    if (ax >= 0x477ff000u) return (uint16_t)(sign | 0x7c00u);    /* >= 65520 rounds to inf */
    if (ax < 0x38800000u) {                                      /* below 2^-14: subnormal */
        float a;
        memcpy(&a, &ax, 4);
        return (uint16_t)(sign | (uint32_t)rintf(a * 16777216.0f)); /* units of 2^-24 */
    }
    const uint32_t r = ax + 0x0fffu + ((ax >> 13) & 1u);         /* round the low 13 bits */
    return (uint16_t)(sign | ((r - (112u << 23)) >> 13));        /* rebias 127 -> 15 */
}

static inline float f16_to_f32(uint16_t h) {
    const uint32_t sign = (uint32_t)(h & 0x8000u) << 16, e = (h >> 10) & 0x1fu, m = h & 0x3ffu;
    uint32_t x;
    float r;
    if (e == 0) {
        r = (float)m * 5.9604644775390625e-8f;                   /* m * 2^-24, exact */
        return sign ? -r : r;
    }
    x = sign | (e == 31 ? 0x7f800000u | (m << 13) : ((e + 112u) << 23) | (m << 13));
    memcpy(&r, &x, 4);
    return r;
}

/* The value a stored level holds: v * s rounded to binary16, times 1/s. */
static inline float q16(float v, float s, float inv) { return f16_to_f32(f32_to_f16(v * s)) * inv; }

/* Scale of the level written at step g: 2^(10 - e) with 2^e above the
 * largest magnitude m of level g - 2 (the last level complete when the
 * step starts, other than the one it reads as p^n) and of the batch
 * member's source samples smax; 1 when both are zero; exponent clamped to
 * [-60, 60]. Two steps of the scheme grow a field by far less than the
 * 2^6 headroom this leaves below the binary16 maximum. */
static float level_scale(float m, float smax) {
    const float a = m > smax ? m : smax;
    if (!(a > 0.0f)) return 1.0f;
    int e;
    frexpf(a, &e);
    int k = 10 - e;
    k = k > 60 ? 60 : (k < -60 ? -60 : k);
    return ldexpf(1.0f, k);
}

#ifndef ORA_NAME
#define ORA_NAME ora_simulate_f32
#endif

/* Group masks in the group numbering of lrs-data.hpp:53-78; bit d is the
 * solid neighbour in direction d = X_P, X_M, Y_P, Y_M, Z_P, Z_M. */
static const unsigned kMask[26] = {
    1, 2, 4, 8, 16, 32,
    1 | 4, 1 | 8, 1 | 16, 1 | 32, 2 | 4, 2 | 8, 2 | 16, 2 | 32, 4 | 16, 4 | 32, 8 | 16, 8 | 32,
    1 | 4 | 16, 1 | 4 | 32, 1 | 8 | 16, 1 | 8 | 32, 2 | 4 | 16, 2 | 4 | 32, 2 | 8 | 16, 2 | 8 | 32};

static int group_of(unsigned m) {
    for (int g = 0; g < 26; ++g)
        if (kMask[g] == m) return g;
    return -1;
}

typedef struct {
    int64_t cell;  /* linear index in the simulation grid */
    int group;
    int mat[3];
} Bpt;

/* LrsData::Init, lrs-data.hpp:154-210: air cells 1..n-2 of the model grid
 * with solid face neighbours, z-y-x scan order, materials in direction
 * order. Returns -1 on an unphysical pattern. */
static int64_t classify(const int32_t* v, int mx, int my, int mz, int64_t pitch, int64_t plane,
                        Bpt* out) {
    int64_t n = 0;
    for (int z = 1; z < mz - 1; ++z)
        for (int y = 1; y < my - 1; ++y)
            for (int x = 1; x < mx - 1; ++x) {
                const int64_t i = ((int64_t)z * my + y) * mx + x;
                if (v[i] != -1) continue;
                const int32_t nb[6] = {v[i + 1], v[i - 1], v[i + mx], v[i - mx],
                                       v[i + (int64_t)mx * my], v[i - (int64_t)mx * my]};
                unsigned m = 0;
                for (int d = 0; d < 6; ++d)
                    if (nb[d] != -1) m |= 1u << d;
                if (!m) continue;
                const int g = group_of(m);
                if (g < 0) return -1;
                if (out) {
                    Bpt* b = &out[n];
                    b->cell = (int64_t)z * plane + (int64_t)y * pitch + x;
                    b->group = g;
                    int k = 0;
                    b->mat[0] = b->mat[1] = b->mat[2] = -1;
                    for (int d = 0; d < 6; ++d)
                        if (m & (1u << d)) b->mat[k++] = nb[d];
                }
                ++n;
            }
    return n;
}

/* Neighbour sum of a boundary cell (lrs_1.cl:80-120 and the edge and
 * corner variants): axes x, y, z in turn; a wall on the + side gives
 * 2*p(-1), on the - side 2*p(+1), no wall p(+1) + p(-1). */
static real lrs_sum(unsigned m, const real* p, int64_t i, int64_t pitch, int64_t plane) {
    const int64_t off[3] = {1, pitch, plane};
    real s = 0;
    int first = 1;
    for (int ax = 0; ax < 3; ++ax) {
        real t0, t1 = 0;
        int two = 0;
        if (m & (1u << (2 * ax))) t0 = (real)2.0f * p[i - off[ax]];
        else if (m & (1u << (2 * ax + 1))) t0 = (real)2.0f * p[i + off[ax]];
        else {
            t0 = p[i + off[ax]];
            t1 = p[i - off[ax]];
            two = 1;
        }
        s = first ? t0 : s + t0;
        first = 0;
        if (two) s = s + t1;
    }
    return s;
}

/* One boundary point (lrs_1.cl:61-124 / lrs_2.cl:61-215 / lrs_3.cl:61-186).
 * in/out: the point's ring buffers, width 3K. */
static void lrs_point(int mode, const Bpt* b, real* pn, const real* pc, const real* po,
                      const real* ca, const real* cb, int K, real* in, real* out, int ix_buf,
                      real l, real l2, real c2, int64_t pitch, int64_t plane) {
    const int nf = b->group < 6 ? 1 : (b->group < 18 ? 2 : 3);
    const int size_f = (mode == 0 && nf == 3) ? K / 2 : K;
    real a0[3], b0[3], gn[3];
    for (int f = 0; f < nf; ++f) {
        a0[f] = ca[b->mat[f] * K];
        b0[f] = cb[b->mat[f] * K];
        gn[f] = 0;
    }
    for (int i = 1; i < K; ++i)
        for (int f = 0; f < nf; ++f) {
            const int s = (ix_buf + i) % size_f + f * size_f;
            gn[f] += cb[b->mat[f] * K + i] * in[s] - ca[b->mat[f] * K + i] * out[s];
        }
    const int64_t c = b->cell;
    const real S = lrs_sum(kMask[b->group], pc, c, pitch, plane);
    real v;
    if (nf == 1) {
        v = (l2 * S + c2 * pc[c] + l2 / b0[0] * gn[0] + (l * a0[0] / b0[0] - (real)1.0f) * po[c]) /
            ((real)1.0f + l * a0[0] / b0[0]);
    } else if (nf == 2 || mode == 0) {
        if (mode == 0 && b->group == 25)
            v = pn[c]; /* no variant define reaches the kernel (simulation.hpp:452) */
        else
            v = (l2 * S + l2 * (gn[0] / b0[0] + gn[1] / b0[1]) + c2 * pc[c] +
                 (l * a0[0] / b0[0] + l * a0[1] / b0[1] - (real)1.0f) * po[c]) /
                ((real)1.0f + l * a0[0] / b0[0] + l * a0[1] / b0[1]);
    } else {
        v = (l2 * S + l2 * (gn[0] / b0[0] + gn[1] / b0[1] + gn[2] / b0[2]) + c2 * pc[c] +
             (l * a0[0] / b0[0] + l * a0[1] / b0[1] + l * a0[2] / b0[2] - (real)1.0f) * po[c]) /
            ((real)1.0f + l * a0[0] / b0[0] + l * a0[1] / b0[1] + l * a0[2] / b0[2]);
    }
    pn[c] = v;
    for (int f = 0; f < nf; ++f) {
        const real xn = a0[f] / (l * b0[f]) * (v - po[c]) - gn[f] / b0[f];
        in[ix_buf + f * size_f] = xn;
        out[ix_buf + f * size_f] = (real)1.0f / a0[f] * (b0[f] * xn + gn[f]);
    }
}

/* ---- PML (pml.cl) ------------------------------------------------------ */
typedef struct {
    const real* f;
    int64_t self;
    real own;
    int subst;
} Avg;

static real av(const Avg* A, int64_t i) { return (A->subst && i == A->self) ? A->own : A->f[i]; }
/* pml.cl:74-122 face averages */
static real avx(const Avg* A, int64_t i, int64_t pitch, int64_t plane) {
    return (real)0.25f * (((av(A, i) + av(A, i + plane)) + av(A, i + pitch)) + av(A, i + pitch + plane));
}
static real avy(const Avg* A, int64_t i, int64_t pitch, int64_t plane) {
    (void)pitch;
    return (real)0.25f * (((av(A, i) + av(A, i + plane)) + av(A, i + 1)) + av(A, i + 1 + plane));
}
static real avz(const Avg* A, int64_t i, int64_t pitch, int64_t plane) {
    (void)plane;
    return (real)0.25f * (((av(A, i) + av(A, i + pitch)) + av(A, i + 1)) + av(A, i + 1 + pitch));
}

typedef struct {
    real dt, cc_dxdx, inv_dx, half_inv_dx, inv_dt2, two_dt, inv_dt;
    const real* ksi[3];
} PmlK;

/* pml.cl:185-207 */
static real pml_p(const PmlK* K, const real* pc, const real* po, const real* fx1, const real* fy1,
                  const real* fz1, const real* psimh, int x, int y, int z, int64_t i, int64_t pitch,
                  int64_t plane, real* psi_new) {
    const real kx = K->ksi[0][x], ky = K->ksi[1][y], kz = K->ksi[2][z];
    const real pm1 = pc[i];
    const real ps = K->dt * pm1 + psimh[i];
    *psi_new = ps;
    real s = pc[i + 1] + pc[i - 1];
    s = s + pc[i + pitch];
    s = s + pc[i - pitch];
    s = s + pc[i + plane];
    s = s + pc[i - plane];
    s = s - (real)6.0f * pm1;
    const real A = K->cc_dxdx * s;
    const Avg FX = {fx1, -1, 0, 0}, FY = {fy1, -1, 0, 0}, FZ = {fz1, -1, 0, 0};
    real d = avx(&FX, i + 1, pitch, plane) - avx(&FX, i, pitch, plane);
    d = d + avy(&FY, i + pitch, pitch, plane);
    d = d - avy(&FY, i, pitch, plane);
    d = d + avz(&FZ, i + plane, pitch, plane);
    d = d - avz(&FZ, i, pitch, plane);
    const real B = K->inv_dx * d;
    const real C = kx * ky * kz * (real)0.5f * (ps + psimh[i]);
    const real D = K->inv_dt2 * (po[i] - (real)2.0f * pm1);
    const real E = (kx * ky + ky * kz + kz * kx) * pm1;
    const real F = (kx + ky + kz) / K->two_dt * po[i];
    const real num = A + B - C - D - E + F;
    return num / (K->inv_dt2 + (kx + ky + kz) / K->two_dt);
}

/* pml.cl:231-262. REF: reads of p see this cell's new value and every other
 * cell before the PML pass (the kernel's serial work-item order); Dxp's last
 * term reads p (pml.cl:126) and fi_y's psi coefficient ksi_x at y (:247). */
static void pml_aux(int mode, const PmlK* K, unsigned axes, const real* pnew, const real* pc,
                    const real* psiph, real p_own, real psi_own, const real* fx1, const real* fy1,
                    const real* fz1, real* fx, real* fy, real* fz, int x, int y, int z, int64_t i,
                    int64_t pitch, int64_t plane) {
    const int ref = mode == 0;
    const Avg Pn = {pnew, i, p_own, ref}, Pm = {pc, -1, 0, 0}, Ps = {psiph, i, psi_own, ref};
    const Avg* Pl = ref ? &Pn : &Pm;
    const real kax = (real)0.5f * (K->ksi[0][x] + K->ksi[0][x + 1]);
    const real kay = (real)0.5f * (K->ksi[1][y] + K->ksi[1][y + 1]);
    const real kaz = (real)0.5f * (K->ksi[2][z] + K->ksi[2][z + 1]);
    if (axes & 1u) {
        const real dxp = K->half_inv_dx * (avx(&Pn, i + 1, pitch, plane) - avx(&Pn, i, pitch, plane) +
                                           avx(&Pm, i + 1, pitch, plane) - avx(Pl, i, pitch, plane));
        const real dxpsi = K->inv_dx * (avx(&Ps, i + 1, pitch, plane) - avx(&Ps, i, pitch, plane));
        const real f1 = fx1[i];
        fx[i] = (-(real)0.5f * kax * f1 + (kay + kaz - kax) * dxp + (kay * kaz) * dxpsi + K->inv_dt * f1) /
                (K->inv_dt + kax * (real)0.5f);
    }
    if (axes & 2u) {
        const real dyp = K->half_inv_dx * (avy(&Pn, i + pitch, pitch, plane) - avy(&Pn, i, pitch, plane) +
                                           avy(&Pm, i + pitch, pitch, plane) - avy(Pl, i, pitch, plane));
        const real dypsi = K->inv_dx * (avy(&Ps, i + pitch, pitch, plane) - avy(&Ps, i, pitch, plane));
        const real kxc = ref ? (real)0.5f * (K->ksi[0][y] + K->ksi[0][y + 1]) : kax;
        const real f1 = fy1[i];
        fy[i] = (-(real)0.5f * kay * f1 + (kax + kaz - kay) * dyp + (kxc * kaz) * dypsi + K->inv_dt * f1) /
                (K->inv_dt + kay * (real)0.5f);
    }
    if (axes & 4u) {
        const real dzp = K->half_inv_dx * (avz(&Pn, i + plane, pitch, plane) - avz(&Pn, i, pitch, plane) +
                                           avz(&Pm, i + plane, pitch, plane) - avz(Pl, i, pitch, plane));
        const real dzpsi = K->inv_dx * (avz(&Ps, i + plane, pitch, plane) - avz(&Ps, i, pitch, plane));
        const real f1 = fz1[i];
        fz[i] = (-(real)0.5f * kaz * f1 + (kax + kay - kaz) * dzp + (kax * kay) * dzpsi + K->inv_dt * f1) /
                (K->inv_dt + kaz * (real)0.5f);
    }
}

/*
 * Runs one simulation (one batch member).
 *   mode            0 REF, 1 FIXED
 *   nx, ny, nz      simulation grid
 *   mx, my, mz, vox model grid and voxels (-1 air); mx = 0 for no model
 *   nmat, K, a, b   filter coefficients [nmat][K]
 *   dx, c, dt       scalars (rounded to `real` first)
 *   pml_width, faces, ksi_x/y/z (nx, ny, nz values; faces used by FIXED)
 *   sources: nsrc cells src_ijk[3*s], signals src_data[src_off[s] ..+ src_len[s]]
 *   receivers: nrcv cells rcv_ijk[3*r]
 *   n_runs, run_steps: consecutive run calls (the REF PML reset counts
 *                      steps per run)
 *   rcv_out [nrcv][total steps] (float), field_out [nz][ny][nx] of the
 *   last level or NULL.
 * Returns 0, or -1 on bad input / unphysical geometry, -2 on no memory.
 */
static int simulate(int mode, int nx, int ny, int nz, int mx, int my, int mz, const int32_t* vox, int nmat,
                    int K, const double* a, const double* b, double dx, double c, double dt, int pml_width,
                    unsigned faces, const float* ksi_x, const float* ksi_y, const float* ksi_z, int nsrc,
                    const int32_t* src_ijk, const int64_t* src_off, const int64_t* src_len,
                    const float* src_data, int nrcv, const int32_t* rcv_ijk, int n_runs,
                    const int64_t* run_steps, float* rcv_out, float* field_out, int f16) {
    if (nx < 3 || ny < 3 || nz < 3 || K < 1 || (mx && (mx > nx || my > ny || mz > nz))) return -1;
    if (f16 && (mode != 1 || sizeof(real) != sizeof(float))) return -1;
    float smax = 0.0f;
    for (int s = 0; s < nsrc; ++s)
        for (int64_t k = 0; k < src_len[s]; ++k) {
            const float v = fabsf(src_data[src_off[s] + k]);
            smax = v > smax ? v : smax;
        }
    const int64_t pitch = nx, plane = (int64_t)nx * ny, vol = plane * nz;
    int64_t total = 0;
    for (int r = 0; r < n_runs; ++r) total += run_steps[r];

    /* boundary list */
    int64_t nb = mx ? classify(vox, mx, my, mz, pitch, plane, NULL) : 0;
    if (nb < 0) return -1;
    Bpt* bp = nb ? (Bpt*)malloc(sizeof(Bpt) * (size_t)nb) : NULL;
    if (nb) classify(vox, mx, my, mz, pitch, plane, bp);
    const int S = 3 * K;
    real* ring_in = (real*)calloc((size_t)(nb ? nb : 1) * S, sizeof(real));
    real* ring_out = (real*)calloc((size_t)(nb ? nb : 1) * S, sizeof(real));
    real* ca = (real*)malloc(sizeof(real) * (size_t)(nmat > 0 ? nmat : 1) * K);
    real* cb = (real*)malloc(sizeof(real) * (size_t)(nmat > 0 ? nmat : 1) * K);
    for (int k = 0; k < nmat * K; ++k) {
        ca[k] = (real)(float)a[k];
        cb[k] = (real)(float)b[k];
    }
    real* buf = (real*)calloc((size_t)vol * 3, sizeof(real));
    if (!ring_in || !ring_out || !buf || !ca || !cb) return -2;
    real* P[3] = {buf, buf + vol, buf + 2 * vol};

    const real rdx = (real)dx, rc = (real)c, rdt = (real)dt;
    const real t = rdt * rc / rdx;
    const real lambda2 = t * t;
    const real cint = (real)2.0f * ((real)1.0f - (real)3.0f * lambda2);
    const real l = mode == 0 ? lambda2 : t; /* simulation.hpp:368-369 passes lambda^2 */
    const real l2 = l * l;
    const real c2 = (real)2.0f * ((real)1.0f - (real)3.0f * l2);

    /* PML */
    real *fi[3][2] = {{0}}, *psi[2] = {0}, *ksi[3] = {0};
    int64_t npml = 0;
    int64_t* pml_cells = NULL;
    unsigned char* pml_flags = NULL;
    PmlK PK;
    if (pml_width > 0) {
        const int kmax = (nx > ny ? (nx > nz ? nx : nz) : (ny > nz ? ny : nz)) + 1;
        for (int ax = 0; ax < 3; ++ax) {
            fi[ax][0] = (real*)calloc((size_t)vol, sizeof(real));
            fi[ax][1] = (real*)calloc((size_t)vol, sizeof(real));
            ksi[ax] = (real*)calloc((size_t)kmax, sizeof(real));
            const float* src = ax == 0 ? ksi_x : ax == 1 ? ksi_y : ksi_z;
            const int n = ax == 0 ? nx : ax == 1 ? ny : nz;
            for (int k = 0; k < n; ++k) ksi[ax][k] = (real)src[k];
            PK.ksi[ax] = ksi[ax];
        }
        psi[0] = (real*)calloc((size_t)vol, sizeof(real));
        psi[1] = (real*)calloc((size_t)vol, sizeof(real));
        PK.dt = rdt;
        PK.cc_dxdx = rc * rc / (rdx * rdx);
        PK.inv_dx = (real)1.0f / rdx;
        PK.half_inv_dx = (real)0.5f / rdx;
        PK.inv_dt2 = (real)1.0f / (rdt * rdt);
        PK.two_dt = (real)2.0f * rdt;
        PK.inv_dt = (real)1.0f / rdt;
        if (mode == 1) {
            unsigned char* lrs = (unsigned char*)calloc((size_t)vol, 1);
            for (int64_t e = 0; e < nb; ++e) lrs[bp[e].cell] = 1;
            pml_cells = (int64_t*)malloc(sizeof(int64_t) * (size_t)vol);
            pml_flags = (unsigned char*)malloc((size_t)vol);
            const int W = pml_width;
            for (int z = 2; z <= nz - 3; ++z)
                for (int y = 2; y <= ny - 3; ++y)
                    for (int x = 2; x <= nx - 3; ++x) {
                        unsigned ax = 0;
                        if (((faces & 1u) && x < W) || ((faces & 2u) && x > nx - W - 1)) ax |= 1u;
                        if (((faces & 4u) && y < W) || ((faces & 8u) && y > ny - W - 1)) ax |= 2u;
                        if (((faces & 16u) && z < W) || ((faces & 32u) && z > nz - W - 1)) ax |= 4u;
                        if (!ax) continue;
                        const int64_t i = (int64_t)z * plane + (int64_t)y * pitch + x;
                        if (lrs[i]) continue;
                        if (mx && x < mx && y < my && z < mz && vox[((int64_t)z * my + y) * mx + x] != -1)
                            continue;
                        pml_cells[npml] = i;
                        pml_flags[npml] = (unsigned char)ax;
                        ++npml;
                    }
            free(lrs);
        }
    }

    int64_t g = 0;
    for (int r = 0; r < n_runs; ++r) {
        for (int64_t it = 0; it < run_steps[r]; ++it, ++g) {
            /* simulation.hpp:360: the three levels rotate right by one */
            const int w = (int)((2 + 2 * (g % 3)) % 3);
            real* pn = P[w];
            const real* pc = P[(w + 1) % 3];
            real* po = P[(w + 2) % 3];
            float sp = 1.0f, isp = 1.0f;
            if (f16) {
                float m = 0.0f;
#pragma omp parallel for schedule(static) reduction(max : m)
                for (int64_t i = 0; i < vol; ++i) m = fabsf(po[i]) > m ? fabsf(po[i]) : m;
                sp = level_scale(m, smax);
                isp = 1.0f / sp;
            }
            /* leapfrog.cl:40-53; FP16 storage evaluates the same update as
             * p + ((p - p^{n-1}) + lambda^2 (S - 6p)), the increment formed
             * before it meets the stored level */
#pragma omp parallel for schedule(static)
            for (int z = 1; z <= nz - 2; ++z)
                for (int y = 1; y <= ny - 2; ++y)
                    for (int x = 1; x <= nx - 2; ++x) {
                        const int64_t i = (int64_t)z * plane + (int64_t)y * pitch + x;
                        real s = pc[i + 1] + pc[i - 1];
                        s = s + pc[i + pitch];
                        s = s + pc[i - pitch];
                        s = s + pc[i + plane];
                        s = s + pc[i - plane];
                        if (!f16)
                            pn[i] = lambda2 * s + cint * pc[i] - po[i];
                        else
                            pn[i] = pc[i] + ((pc[i] - po[i]) + lambda2 * (s - (real)6.0f * pc[i]));
                    }
            /* simulation.hpp:365 */
            const int ix_buf = K - 1 - (int)(g % K);
#pragma omp parallel for schedule(static)
            for (int64_t e = 0; e < nb; ++e)
                lrs_point(mode, &bp[e], pn, pc, po, ca, cb, K, ring_in + e * S, ring_out + e * S,
                          ix_buf, l, l2, c2, pitch, plane);
            if (pml_width > 0) {
                const int lv = (int)((g + 1) & 1);
                real* fx = fi[0][lv]; real* fy = fi[1][lv]; real* fz = fi[2][lv];
                const real* fx1 = fi[0][lv ^ 1]; const real* fy1 = fi[1][lv ^ 1]; const real* fz1 = fi[2][lv ^ 1];
                real* psiph = psi[lv];
                const real* psimh = psi[lv ^ 1];
                if (mode == 0) {
                    /* pml.cl:182-262 over 2..n-3; auxiliary fields first
                     * (they read the pre-pass pressure and psi of every other
                     * cell), then pressure and psi. */
                    const int W = pml_width;
#pragma omp parallel for schedule(static)
                    for (int z = 2; z <= nz - 3; ++z)
                        for (int y = 2; y <= ny - 3; ++y)
                            for (int x = 2; x <= nx - 3; ++x) {
                                unsigned ax = 0;
                                if (x < W || x > nx - W - 1) ax |= 1u;
                                if (y < W || y > ny - W - 1) ax |= 2u;
                                if (z < W || z > nz - W - 1) ax |= 4u;
                                if (!ax) continue;
                                const int64_t i = (int64_t)z * plane + (int64_t)y * pitch + x;
                                real ps;
                                const real pv = pml_p(&PK, pc, po, fx1, fy1, fz1, psimh, x, y, z, i, pitch, plane, &ps);
                                pml_aux(0, &PK, ax, pn, pc, psiph, pv, ps, fx1, fy1, fz1, fx, fy, fz, x, y, z, i,
                                        pitch, plane);
                            }
#pragma omp parallel for schedule(static)
                    for (int z = 2; z <= nz - 3; ++z)
                        for (int y = 2; y <= ny - 3; ++y)
                            for (int x = 2; x <= nx - 3; ++x) {
                                const int64_t i = (int64_t)z * plane + (int64_t)y * pitch + x;
                                real ps;
                                const real pv = pml_p(&PK, pc, po, fx1, fy1, fz1, psimh, x, y, z, i, pitch, plane, &ps);
                                psiph[i] = ps;
                                pn[i] = pv;
                            }
                } else {
#pragma omp parallel for schedule(static)
                    for (int64_t e = 0; e < npml; ++e) {
                        const int64_t i = pml_cells[e];
                        const int z = (int)(i / plane), y = (int)((i % plane) / pitch), x = (int)(i % pitch);
                        real ps;
                        const real pv = pml_p(&PK, pc, po, fx1, fy1, fz1, psimh, x, y, z, i, pitch, plane, &ps);
                        psiph[i] = ps;
                        pn[i] = pv;
                    }
                }
            }
            if (f16) {
                /* the store of the new level to the FP16 grid of scale sp */
#pragma omp parallel for schedule(static)
                for (int z = 1; z <= nz - 2; ++z)
                    for (int y = 1; y <= ny - 2; ++y)
                        for (int x = 1; x <= nx - 2; ++x) {
                            const int64_t i = (int64_t)z * plane + (int64_t)y * pitch + x;
                            pn[i] = q16(pn[i], sp, isp);
                        }
            }
            if (pml_width > 0 && mode == 1) {
                const int lv = (int)((g + 1) & 1);
                real* fx = fi[0][lv]; real* fy = fi[1][lv]; real* fz = fi[2][lv];
                const real* fx1 = fi[0][lv ^ 1]; const real* fy1 = fi[1][lv ^ 1]; const real* fz1 = fi[2][lv ^ 1];
                real* psiph = psi[lv];
                {
#pragma omp parallel for schedule(static)
                    for (int64_t e = 0; e < npml; ++e) {
                        const int64_t i = pml_cells[e];
                        const int z = (int)(i / plane), y = (int)((i % plane) / pitch), x = (int)(i % pitch);
                        pml_aux(1, &PK, pml_flags[e], pn, pc, psiph, 0, 0, fx1, fy1, fz1, fx, fy, fz, x, y, z, i,
                                pitch, plane);
                    }
                }
            }
            /* source.cl:32-40, in source order */
            for (int s = 0; s < nsrc; ++s) {
                const int64_t i = (int64_t)src_ijk[3 * s + 2] * plane + (int64_t)src_ijk[3 * s + 1] * pitch +
                                  src_ijk[3 * s];
                const real v = (g < src_len[s]) ? (real)src_data[src_off[s] + g] : (real)0.0f;
                pn[i] = f16 ? q16(pn[i] + v, sp, isp) : pn[i] + v;
            }
            /* mic.cl:32-41 */
            for (int m = 0; m < nrcv; ++m) {
                const int64_t i = (int64_t)rcv_ijk[3 * m + 2] * plane + (int64_t)rcv_ijk[3 * m + 1] * pitch +
                                  rcv_ijk[3 * m];
                rcv_out[(size_t)m * total + g] = (float)pn[i];
            }
            /* simulation.hpp:411-430: REF zeroes the PML fields every 8000 run steps */
            if (mode == 0 && pml_width > 0 && it % 8000 == 0) {
                for (int ax = 0; ax < 3; ++ax) {
                    memset(fi[ax][0], 0, sizeof(real) * (size_t)vol);
                    memset(fi[ax][1], 0, sizeof(real) * (size_t)vol);
                }
                memset(psi[0], 0, sizeof(real) * (size_t)vol);
                memset(psi[1], 0, sizeof(real) * (size_t)vol);
            }
        }
    }
    if (field_out) {
        const real* last = total > 0 ? P[(int)((2 + 2 * ((total - 1) % 3)) % 3)] : P[0];
        for (int64_t i = 0; i < vol; ++i) field_out[i] = (float)last[i];
    }
    free(bp);
    free(ring_in);
    free(ring_out);
    free(ca);
    free(cb);
    free(buf);
    for (int ax = 0; ax < 3; ++ax) {
        free(fi[ax][0]);
        free(fi[ax][1]);
        free(ksi[ax]);
    }
    free(psi[0]);
    free(psi[1]);
    free(pml_cells);
    free(pml_flags);
    return 0;
}

int ORA_NAME(int mode, int nx, int ny, int nz, int mx, int my, int mz, const int32_t* vox, int nmat,
             int K, const double* a, const double* b, double dx, double c, double dt, int pml_width,
             unsigned faces, const float* ksi_x, const float* ksi_y, const float* ksi_z, int nsrc,
             const int32_t* src_ijk, const int64_t* src_off, const int64_t* src_len,
             const float* src_data, int nrcv, const int32_t* rcv_ijk, int n_runs,
             const int64_t* run_steps, float* rcv_out, float* field_out) {
    return simulate(mode, nx, ny, nz, mx, my, mz, vox, nmat, K, a, b, dx, c, dt, pml_width, faces, ksi_x,
                    ksi_y, ksi_z, nsrc, src_ijk, src_off, src_len, src_data, nrcv, rcv_ijk, n_runs, run_steps,
                    rcv_out, field_out, 0);
}

#ifndef ORA_NO_F16
/* The storage rounding and the level scale rule, for the tests that pin
 * them: out[i] = q16(in[i], s, 1/s); scales[i] = level_scale(m[i], smax). */
void ora_f16_round(const float* in, float* out, int64_t n, float s) {
    for (int64_t i = 0; i < n; ++i) out[i] = q16(in[i], s, 1.0f / s);
}

void ora_level_scale(const float* m, float* scales, int64_t n, float smax) {
    for (int64_t i = 0; i < n; ++i) scales[i] = level_scale(m[i], smax);
}

/* FIXED scheme with FP16 storage of the three pressure levels. */
int ora_simulate_f16(int mode, int nx, int ny, int nz, int mx, int my, int mz, const int32_t* vox, int nmat,
                     int K, const double* a, const double* b, double dx, double c, double dt, int pml_width,
                     unsigned faces, const float* ksi_x, const float* ksi_y, const float* ksi_z, int nsrc,
                     const int32_t* src_ijk, const int64_t* src_off, const int64_t* src_len,
                     const float* src_data, int nrcv, const int32_t* rcv_ijk, int n_runs,
                     const int64_t* run_steps, float* rcv_out, float* field_out) {
    return simulate(mode, nx, ny, nz, mx, my, mz, vox, nmat, K, a, b, dx, c, dt, pml_width, faces, ksi_x,
                    ksi_y, ksi_z, nsrc, src_ijk, src_off, src_len, src_data, nrcv, rcv_ijk, n_runs, run_steps,
                    rcv_out, field_out, 1);
}
#endif
