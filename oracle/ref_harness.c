/*
 * ref_harness.c - runs the reference's own OpenCL kernel sources on the CPU.
 *
 * TEST INFRASTRUCTURE ONLY (the CPU baseline and the pin of the oracle
 * restatement). The kernels are #included from the reference tree where
 * they lie; this file supplies the OpenCL-to-C shim, the size and index
 * macros that clh generates at JIT time (anc-field/clh/clh-kernel.hpp:
 * 215-251, 334-378: size_<arg>_<d> and ix_<arg>(...) with x fastest), and a
 * replay of Simulation::Run (anc-field/src/simulation.hpp:342-434): buffer
 * rotation, the ring index, the 26 boundary launches, the PML launch, the
 * source and mic launches and the 8000-step PML reset.
 *
 * Build (oracle/build_oracle.py): gcc -std=c11 -O2 -ffp-contract=off
 * -fopenmp -DKS_LEAPFROG=\"<reference>/anc-field/src/leapfrog.cl\" ...;
 * -DREF_FP64 (float read as double) gives the FP64 version of the same
 * kernels. The 26th boundary kernel gets no
 * variant define, as in the reference (simulation.hpp:452 has no "=1", and
 * the clh define regex at clh-kernel.hpp:336 requires one).
 *
 * Work-items of leapfrog and of the boundary kernels are independent and
 * run in parallel; the PML kernel writes cells that other work-items read
 * (pml.cl:188 vs :124-137), so it runs its NDRange serially in x-fastest
 * order, one legal schedule of the kernel. For timing only,
 * ref_set_pml_parallel(1) runs that NDRange over all host threads the way a
 * CPU OpenCL device would (its results then depend on the schedule, as the
 * reference's do on a device); ref_last_loop_seconds() gives the wall time
 * of the last call's step loop, set-up excluded.
 */
#include <omp.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* The ABI keeps FP32 arrays in both builds; `real_t` is the kernels' type. */
typedef __typeof__(1.0f) f32;
#ifdef REF_FP64
#define float double
#endif
typedef float real_t;

/* Kernel file paths arrive as string literals: -DKS_LEAPFROG="\".../leapfrog.cl\"" */

/* OpenCL C -> C */
#define __kernel
#define __global
#define __constant const
static _Thread_local size_t g_gid[3];
static size_t g_gsz[3];
#define get_global_id(d) (g_gid[d])
#define get_global_size(d) (g_gsz[d])

/* clh-generated macros; sizes are runtime values here */
static size_t G_NX, G_NY, G_NZ, G_POSW, G_K, G_BUFW, G_T;
#define CLH_SIZES 1
#define size_p_0 G_NX
#define size_p_1 G_NY
#define size_p_2 G_NZ
#define size_p_p1_0 G_NX
#define size_p_p1_1 G_NY
#define size_p_d1_0 G_NX
#define size_p_d1_1 G_NY
#define size_p_d2_0 G_NX
#define size_p_d2_1 G_NY
#define size_pm1_0 G_NX
#define size_pm1_1 G_NY
#define size_pm2_0 G_NX
#define size_pm2_1 G_NY
#define size_pos_0 G_POSW
#define size_a_0 G_K
#define size_b_0 G_K
#define size_buf_in_0 G_BUFW
#define size_buf_out_0 G_BUFW
#define size_source_0 G_T
#define size_mic_0 G_T
#define IX3(x, y, z) ((z) * G_NY * G_NX + (y) * G_NX + (x))
#define ix_p(x, y, z) IX3(x, y, z)
#define ix_p_p1(x, y, z) IX3(x, y, z)
#define ix_p_d1(x, y, z) IX3(x, y, z)
#define ix_p_d2(x, y, z) IX3(x, y, z)
#define ix_pm1(x, y, z) IX3(x, y, z)
#define ix_pm2(x, y, z) IX3(x, y, z)
#define ix_fi_x(x, y, z) IX3(x, y, z)
#define ix_fi_xm1(x, y, z) IX3(x, y, z)
#define ix_fi_y(x, y, z) IX3(x, y, z)
#define ix_fi_ym1(x, y, z) IX3(x, y, z)
#define ix_fi_z(x, y, z) IX3(x, y, z)
#define ix_fi_zm1(x, y, z) IX3(x, y, z)
#define ix_psiph(x, y, z) IX3(x, y, z)
#define ix_psimh(x, y, z) IX3(x, y, z)
#define ix_pos(x, y) ((y) * size_pos_0 + (x))
#define ix_a(x, y) ((y) * size_a_0 + (x))
#define ix_b(x, y) ((y) * size_b_0 + (x))
#define ix_buf_in(x, y) ((y) * size_buf_in_0 + (x))
#define ix_buf_out(x, y) ((y) * size_buf_out_0 + (x))
#define ix_source(x, y) ((y) * size_source_0 + (x))
#define ix_mic(x, y) ((y) * size_mic_0 + (x))

#include KS_LEAPFROG
#include KS_SOURCE
#include KS_MIC
#include KS_PML

/* The boundary kernels, one compiled copy per variant define. */
#define lrs_1 ref_lrs_X_P
#define X_P 1
#include KS_LRS1
#undef X_P
#undef lrs_1
#define lrs_1 ref_lrs_X_M
#define X_M 1
#include KS_LRS1
#undef X_M
#undef lrs_1
#define lrs_1 ref_lrs_Y_P
#define Y_P 1
#include KS_LRS1
#undef Y_P
#undef lrs_1
#define lrs_1 ref_lrs_Y_M
#define Y_M 1
#include KS_LRS1
#undef Y_M
#undef lrs_1
#define lrs_1 ref_lrs_Z_P
#define Z_P 1
#include KS_LRS1
#undef Z_P
#undef lrs_1
#define lrs_1 ref_lrs_Z_M
#define Z_M 1
#include KS_LRS1
#undef Z_M
#undef lrs_1

#define lrs_2 ref_lrs_X_P_Y_P
#define X_P_Y_P 1
#include KS_LRS2
#undef X_P_Y_P
#undef lrs_2
#define lrs_2 ref_lrs_X_P_Y_M
#define X_P_Y_M 1
#include KS_LRS2
#undef X_P_Y_M
#undef lrs_2
#define lrs_2 ref_lrs_X_P_Z_P
#define X_P_Z_P 1
#include KS_LRS2
#undef X_P_Z_P
#undef lrs_2
#define lrs_2 ref_lrs_X_P_Z_M
#define X_P_Z_M 1
#include KS_LRS2
#undef X_P_Z_M
#undef lrs_2
#define lrs_2 ref_lrs_X_M_Y_P
#define X_M_Y_P 1
#include KS_LRS2
#undef X_M_Y_P
#undef lrs_2
#define lrs_2 ref_lrs_X_M_Y_M
#define X_M_Y_M 1
#include KS_LRS2
#undef X_M_Y_M
#undef lrs_2
#define lrs_2 ref_lrs_X_M_Z_P
#define X_M_Z_P 1
#include KS_LRS2
#undef X_M_Z_P
#undef lrs_2
#define lrs_2 ref_lrs_X_M_Z_M
#define X_M_Z_M 1
#include KS_LRS2
#undef X_M_Z_M
#undef lrs_2
#define lrs_2 ref_lrs_Y_P_Z_P
#define Y_P_Z_P 1
#include KS_LRS2
#undef Y_P_Z_P
#undef lrs_2
#define lrs_2 ref_lrs_Y_P_Z_M
#define Y_P_Z_M 1
#include KS_LRS2
#undef Y_P_Z_M
#undef lrs_2
#define lrs_2 ref_lrs_Y_M_Z_P
#define Y_M_Z_P 1
#include KS_LRS2
#undef Y_M_Z_P
#undef lrs_2
#define lrs_2 ref_lrs_Y_M_Z_M
#define Y_M_Z_M 1
#include KS_LRS2
#undef Y_M_Z_M
#undef lrs_2

#define lrs_3 ref_lrs_X_P_Y_P_Z_P
#define X_P_Y_P_Z_P 1
#include KS_LRS3
#undef X_P_Y_P_Z_P
#undef lrs_3
#define lrs_3 ref_lrs_X_P_Y_P_Z_M
#define X_P_Y_P_Z_M 1
#include KS_LRS3
#undef X_P_Y_P_Z_M
#undef lrs_3
#define lrs_3 ref_lrs_X_P_Y_M_Z_P
#define X_P_Y_M_Z_P 1
#include KS_LRS3
#undef X_P_Y_M_Z_P
#undef lrs_3
#define lrs_3 ref_lrs_X_P_Y_M_Z_M
#define X_P_Y_M_Z_M 1
#include KS_LRS3
#undef X_P_Y_M_Z_M
#undef lrs_3
#define lrs_3 ref_lrs_X_M_Y_P_Z_P
#define X_M_Y_P_Z_P 1
#include KS_LRS3
#undef X_M_Y_P_Z_P
#undef lrs_3
#define lrs_3 ref_lrs_X_M_Y_P_Z_M
#define X_M_Y_P_Z_M 1
#include KS_LRS3
#undef X_M_Y_P_Z_M
#undef lrs_3
#define lrs_3 ref_lrs_X_M_Y_M_Z_P
#define X_M_Y_M_Z_P 1
#include KS_LRS3
#undef X_M_Y_M_Z_P
#undef lrs_3
/* group 25: no variant define reaches the kernel */
#define lrs_3 ref_lrs_X_M_Y_M_Z_M
#include KS_LRS3
#undef lrs_3

typedef void (*lrs_fn)(float*, const float*, const float*, const unsigned*, const float*,
                       const float*, float*, float*, const float, const unsigned);
static const lrs_fn kLrs[26] = {
    ref_lrs_X_P, ref_lrs_X_M, ref_lrs_Y_P, ref_lrs_Y_M, ref_lrs_Z_P, ref_lrs_Z_M,
    ref_lrs_X_P_Y_P, ref_lrs_X_P_Y_M, ref_lrs_X_P_Z_P, ref_lrs_X_P_Z_M, ref_lrs_X_M_Y_P,
    ref_lrs_X_M_Y_M, ref_lrs_X_M_Z_P, ref_lrs_X_M_Z_M, ref_lrs_Y_P_Z_P, ref_lrs_Y_P_Z_M,
    ref_lrs_Y_M_Z_P, ref_lrs_Y_M_Z_M, ref_lrs_X_P_Y_P_Z_P, ref_lrs_X_P_Y_P_Z_M,
    ref_lrs_X_P_Y_M_Z_P, ref_lrs_X_P_Y_M_Z_M, ref_lrs_X_M_Y_P_Z_P, ref_lrs_X_M_Y_P_Z_M,
    ref_lrs_X_M_Y_M_Z_P, ref_lrs_X_M_Y_M_Z_M};

#include "classify.h"

#ifndef REF_NAME
#define REF_NAME ref_simulate_f32
#endif

static int g_pml_parallel = 0;
static double g_loop_seconds = 0.0;

void ref_set_pml_parallel(int on) { g_pml_parallel = on != 0; }
double ref_last_loop_seconds(void) { return g_loop_seconds; }

/*
 * Same arguments as the oracle restatement's ora_simulate_*; mode must be 0
 * (the reference has only its own semantics) and faces is ignored.
 */
int REF_NAME(int mode, int nx, int ny, int nz, int mx, int my, int mz, const int32_t* vox, int nmat,
             int K, const double* a, const double* b, double dx, double c, double dt, int pml_width,
             unsigned faces, const f32* ksi_x, const f32* ksi_y, const f32* ksi_z, int nsrc,
             const int32_t* src_ijk, const int64_t* src_off, const int64_t* src_len,
             const f32* src_data, int nrcv, const int32_t* rcv_ijk, int n_runs,
             const int64_t* run_steps, f32* rcv_out, f32* field_out) {
    (void)faces;
    if (mode != 0 || nx < 3 || ny < 3 || nz < 3 || K < 1) return -1;
    if (mx && (mx > nx || my > ny || mz > nz)) return -1;
    const size_t vol = (size_t)nx * ny * nz;
    int64_t total = 0;
    for (int r = 0; r < n_runs; ++r) total += run_steps[r];

    /* LrsData: per-group point lists {x,y,z,mat...} and zeroed state */
    int64_t cnt[26];
    int32_t* pos[26];
    float *bin[26], *bout[26];
    if (cls_count(vox, mx, my, mz, cnt) < 0) return -1;
    for (int gix = 0; gix < 26; ++gix) {
        const int w = cls_faces(gix);
        pos[gix] = (int32_t*)malloc(sizeof(int32_t) * (size_t)(cnt[gix] ? cnt[gix] : 1) * (3 + w));
        bin[gix] = (float*)calloc((size_t)(cnt[gix] ? cnt[gix] : 1) * w * K, sizeof(float));
        bout[gix] = (float*)calloc((size_t)(cnt[gix] ? cnt[gix] : 1) * w * K, sizeof(float));
    }
    cls_fill(vox, mx, my, mz, pos);

    float* ca = (float*)malloc(sizeof(float) * (size_t)(nmat > 0 ? nmat : 1) * K);
    float* cb = (float*)malloc(sizeof(float) * (size_t)(nmat > 0 ? nmat : 1) * K);
    for (int k = 0; k < nmat * K; ++k) {
        /* coefficients are FP32 values in both builds (kerkythea.hpp:166-175) */
        ca[k] = (float)(f32)a[k];
        cb[k] = (float)(f32)b[k];
    }
    /* Simulation::Simulation, simulation.hpp:162-166 */
    const float c_ = (float)c, dx_ = (float)dx, dt_ = (float)dt;
    const float lambda2 = (dt_ * c_ / dx_) * (dt_ * c_ / dx_);

    float* data = (float*)calloc(vol * 3, sizeof(float));
    float* P[3] = {data, data + vol, data + 2 * vol};

    float *fi[3][2] = {{0}}, *psi[2] = {0}, *ksi[3] = {0};
    if (pml_width > 0) {
        const int kmax = (nx > ny ? (nx > nz ? nx : nz) : (ny > nz ? ny : nz)) + 1;
        for (int ax = 0; ax < 3; ++ax) {
            fi[ax][0] = (float*)calloc(vol, sizeof(float));
            fi[ax][1] = (float*)calloc(vol, sizeof(float));
            ksi[ax] = (float*)calloc((size_t)kmax, sizeof(float));
            const f32* s = ax == 0 ? ksi_x : ax == 1 ? ksi_y : ksi_z;
            const int n = ax == 0 ? nx : ax == 1 ? ny : nz;
            for (int k = 0; k < n; ++k) ksi[ax][k] = s[k];
        }
        psi[0] = (float*)calloc(vol, sizeof(float));
        psi[1] = (float*)calloc(vol, sizeof(float));
    }

    /* sources and mics as clh vectors {T, n} (simulation.hpp:436-447) */
    float* src = (float*)calloc((size_t)(total ? total : 1) * (nsrc ? nsrc : 1), sizeof(float));
    for (int s = 0; s < nsrc; ++s)
        for (int64_t t = 0; t < total && t < src_len[s]; ++t) src[(size_t)s * total + t] = src_data[src_off[s] + t];
    float* mic_rec = (float*)calloc((size_t)(total ? total : 1) * (nrcv ? nrcv : 1), sizeof(float));
    int32_t* spos = (int32_t*)malloc(sizeof(int32_t) * 3 * (size_t)(nsrc ? nsrc : 1));
    int32_t* mpos = (int32_t*)malloc(sizeof(int32_t) * 3 * (size_t)(nrcv ? nrcv : 1));
    memcpy(spos, src_ijk, sizeof(int32_t) * 3 * (size_t)nsrc);
    memcpy(mpos, rcv_ijk, sizeof(int32_t) * 3 * (size_t)nrcv);

    G_NX = (size_t)nx;
    G_NY = (size_t)ny;
    G_NZ = (size_t)nz;
    G_K = (size_t)K;
    G_T = (size_t)total;
    g_gsz[0] = (size_t)nx;
    g_gsz[1] = (size_t)ny;
    g_gsz[2] = (size_t)nz;

    unsigned ix_buf = 0, sim_cnt = 0;
    const double t_loop = omp_get_wtime();
    for (int r = 0; r < n_runs; ++r) {
        for (int64_t i = 0; i < run_steps[r]; ++i) {
            { float* t0 = P[2]; P[2] = P[1]; P[1] = P[0]; P[0] = t0; } /* rotate(begin, begin+2) */
            g_gsz[0] = (size_t)nx; g_gsz[1] = (size_t)ny; g_gsz[2] = (size_t)nz;
#pragma omp parallel for schedule(static)
            for (int z = 0; z < nz; ++z)
                for (int y = 0; y < ny; ++y)
                    for (int x = 0; x < nx; ++x) {
                        g_gid[0] = (size_t)x; g_gid[1] = (size_t)y; g_gid[2] = (size_t)z;
                        leapfrog(P[0], P[1], P[2], lambda2);
                    }
            if (mx) {
                if (ix_buf == 0) ix_buf = (unsigned)K - 1; else ix_buf -= 1;
                for (int gix = 0; gix < 26; ++gix) {
                    const int w = cls_faces(gix);
                    G_POSW = (size_t)(3 + w);
                    G_BUFW = (size_t)(w * K);
                    g_gsz[0] = (size_t)cnt[gix];
                    const int64_t n = cnt[gix];
#pragma omp parallel for schedule(static)
                    for (int64_t id = 0; id < n; ++id) {
                        g_gid[0] = (size_t)id;
                        kLrs[gix](P[0], P[1], P[2], (const unsigned*)pos[gix], ca, cb, bin[gix], bout[gix],
                                  lambda2, ix_buf);
                    }
                }
            }
            if (pml_width > 0) {
                for (int ax = 0; ax < 3; ++ax) { float* t0 = fi[ax][0]; fi[ax][0] = fi[ax][1]; fi[ax][1] = t0; }
                { float* t0 = psi[0]; psi[0] = psi[1]; psi[1] = t0; }
                g_gsz[0] = (size_t)nx; g_gsz[1] = (size_t)ny; g_gsz[2] = (size_t)nz;
#pragma omp parallel for schedule(static) if (g_pml_parallel)
                for (int z = 0; z < nz; ++z)
                    for (int y = 0; y < ny; ++y)
                        for (int x = 0; x < nx; ++x) {
                            g_gid[0] = (size_t)x; g_gid[1] = (size_t)y; g_gid[2] = (size_t)z;
                            calculate_pml(P[0], P[1], P[2], fi[0][0], fi[0][1], fi[1][0], fi[1][1], fi[2][0],
                                          fi[2][1], psi[0], psi[1], ksi[0], ksi[1], ksi[2], c_, dx_, dt_,
                                          pml_width);
                        }
            }
            G_POSW = 3;
            for (int s = 0; s < nsrc; ++s) {
                g_gid[0] = (size_t)s;
                source(P[0], spos, src, (unsigned)(sim_cnt + i));
            }
            for (int m = 0; m < nrcv; ++m) {
                g_gid[0] = (size_t)m;
                mic(P[0], mpos, mic_rec, (unsigned)(sim_cnt + i));
            }
            if (pml_width > 0 && i % 8000 == 0) {
                for (int ax = 0; ax < 3; ++ax) {
                    memset(fi[ax][0], 0, vol * sizeof(float));
                    memset(fi[ax][1], 0, vol * sizeof(float));
                }
                memset(psi[0], 0, vol * sizeof(float));
                memset(psi[1], 0, vol * sizeof(float));
            }
        }
        sim_cnt += (unsigned)run_steps[r];
    }
    g_loop_seconds = omp_get_wtime() - t_loop;
    for (int m = 0; m < nrcv; ++m)
        for (int64_t t = 0; t < total; ++t) rcv_out[(size_t)m * total + t] = (f32)mic_rec[(size_t)m * total + t];
    if (field_out)
        for (size_t i = 0; i < vol; ++i) field_out[i] = (f32)P[0][i];
    for (int gix = 0; gix < 26; ++gix) {
        free(pos[gix]);
        free(bin[gix]);
        free(bout[gix]);
    }
    free(ca); free(cb); free(data); free(src); free(mic_rec); free(spos); free(mpos);
    for (int ax = 0; ax < 3; ++ax) { free(fi[ax][0]); free(fi[ax][1]); free(ksi[ax]); }
    free(psi[0]); free(psi[1]);
    return 0;
}
