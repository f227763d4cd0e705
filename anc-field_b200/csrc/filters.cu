// FP64 filter checks: polynomial roots by Durand-Kerner iteration and the
// real part of the admittance on a dense frequency grid, one CUDA thread per
// (material, frequency) and per material for the roots.
#include <cuda_runtime.h>

#include <cmath>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/afd.h"
#include "filters.hpp"
#include "model.hpp"

namespace afd {

namespace {

struct C {
    double re, im;
};
__host__ __device__ inline C cadd(C x, C y) { return {x.re + y.re, x.im + y.im}; }
__host__ __device__ inline C csub(C x, C y) { return {x.re - y.re, x.im - y.im}; }
__host__ __device__ inline C cmul(C x, C y) { return {x.re * y.re - x.im * y.im, x.re * y.im + x.im * y.re}; }
__host__ __device__ inline C cdiv(C x, C y) {
    const double d = y.re * y.re + y.im * y.im;
    return {(x.re * y.re + x.im * y.im) / d, (x.im * y.re - x.re * y.im) / d};
}
__host__ __device__ inline double cabs_(C x) { return sqrt(x.re * x.re + x.im * x.im); }

constexpr int kMaxCoef = 64;

// Largest root magnitude of c[0] z^n + c[1] z^(n-1) + ... + c[n], n = K-1.
__host__ __device__ double max_root_of(const double* c, int K) {
    const int n = K - 1;
    if (n <= 0) return 0.0;
    if (c[0] == 0.0) return INFINITY;
    C z[kMaxCoef];
    double mono[kMaxCoef];
    for (int k = 0; k <= n; ++k) mono[k] = c[k] / c[0];
    C seed{0.4, 0.9}, p{1.0, 0.0};
    for (int k = 0; k < n; ++k) {
        z[k] = p;
        p = cmul(p, seed);
    }
    for (int it = 0; it < 2000; ++it) {
        double moved = 0.0;
        for (int k = 0; k < n; ++k) {
            C v{1.0, 0.0};  // Horner on the monic polynomial
            for (int q = 1; q <= n; ++q) v = cadd(cmul(v, z[k]), C{mono[q], 0.0});
            C den{1.0, 0.0};
            for (int q = 0; q < n; ++q)
                if (q != k) den = cmul(den, csub(z[k], z[q]));
            const C step = cdiv(v, den);
            z[k] = csub(z[k], step);
            moved = fmax(moved, cabs_(step));
        }
        if (moved < 1e-15) break;
    }
    double m = 0.0;
    for (int k = 0; k < n; ++k) m = fmax(m, cabs_(z[k]));
    return m;
}

// Re{A(e^jw)/B(e^jw)}, coefficients in powers of z^-1.
__host__ __device__ double re_admittance(const double* a, const double* b, int K, double w) {
    C A{0.0, 0.0}, B{0.0, 0.0};
    for (int k = 0; k < K; ++k) {
        const C e{cos(-w * k), sin(-w * k)};
        A = cadd(A, C{a[k] * e.re, a[k] * e.im});
        B = cadd(B, C{b[k] * e.re, b[k] * e.im});
    }
    return cdiv(A, B).re;
}

__global__ void k_roots(const double* b, int nmat, int K, double* out) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m < nmat) out[m] = max_root_of(b + (size_t)m * K, K);
}

__global__ void k_passive(const double* a, const double* b, int nmat, int K, int nf, double* out) {
    const int m = blockIdx.y;
    double lo = INFINITY;
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < nf; f += gridDim.x * blockDim.x) {
        const double w = 3.141592653589793 * (double)f / (double)(nf - 1);
        lo = fmin(lo, re_admittance(a + (size_t)m * K, b + (size_t)m * K, K, w));
    }
    for (int o = 16; o > 0; o >>= 1) lo = fmin(lo, __shfl_down_sync(0xffffffffu, lo, o));
    __shared__ double part[32];
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = lo;
    __syncthreads();
    if (threadIdx.x == 0) {
        double v = part[0];
        for (int k = 1; k < (int)(blockDim.x >> 5); ++k) v = fmin(v, part[k]);
        // atomic min on a double through its bit pattern is valid only for
        // one sign, so each block writes its own slot
        out[(size_t)m * gridDim.x + blockIdx.x] = v;
    }
}

// The same two checks for at most MAXC coefficients without local memory
// (no per-thread stack to reserve at launch): the Durand-Kerner iterates of
// the root kernel live in shared memory, one row per thread, and the
// passivity kernel evaluates e^{-jwk} with sincospi (w = pi f / (nf - 1), so
// the argument is the exact fraction -k f / (nf - 1) and needs no reduction
// table). Same iteration as max_root_of; the frequency grid of k_passive.
template <int MAXC>
__global__ void __launch_bounds__(64) k_roots_static(const double* b, int nmat, int K, double* out) {
    __shared__ C zs[64][MAXC];
    __shared__ double ms[64][MAXC];
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nmat) return;
    C* z = zs[threadIdx.x];
    double* mono = ms[threadIdx.x];
    const double* c = b + (size_t)m * K;
    const int n = K - 1;
    if (n <= 0) {
        out[m] = 0.0;
        return;
    }
    if (c[0] == 0.0) {
        out[m] = INFINITY;
        return;
    }
    for (int k = 0; k <= n; ++k) mono[k] = c[k] / c[0];
    C seed{0.4, 0.9}, p{1.0, 0.0};
    for (int k = 0; k < n; ++k) {
        z[k] = p;
        p = cmul(p, seed);
    }
    for (int it = 0; it < 2000; ++it) {
        double moved = 0.0;
        for (int k = 0; k < n; ++k) {
            C v{1.0, 0.0};
            for (int q = 1; q <= n; ++q) v = cadd(cmul(v, z[k]), C{mono[q], 0.0});
            C den{1.0, 0.0};
            for (int q = 0; q < n; ++q)
                if (q != k) den = cmul(den, csub(z[k], z[q]));
            const C step = cdiv(v, den);
            z[k] = csub(z[k], step);
            moved = fmax(moved, cabs_(step));
        }
        if (moved < 1e-15) break;
    }
    double mr = 0.0;
    for (int k = 0; k < n; ++k) mr = fmax(mr, cabs_(z[k]));
    out[m] = mr;
}

__global__ void k_passive_static(const double* a, const double* b, int nmat, int K, int nf, double* out) {
    const int m = blockIdx.y;
    double lo = INFINITY;
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < nf; f += gridDim.x * blockDim.x) {
        C A{0.0, 0.0}, B{0.0, 0.0};
        for (int k = 0; k < K; ++k) {
            double sn, cs;
            sincospi(-(double)(k * f) / (double)(nf - 1), &sn, &cs);
            A = cadd(A, C{a[(size_t)m * K + k] * cs, a[(size_t)m * K + k] * sn});
            B = cadd(B, C{b[(size_t)m * K + k] * cs, b[(size_t)m * K + k] * sn});
        }
        lo = fmin(lo, cdiv(A, B).re);
    }
    for (int o = 16; o > 0; o >>= 1) lo = fmin(lo, __shfl_down_sync(0xffffffffu, lo, o));
    __shared__ double part[32];
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = lo;
    __syncthreads();
    if (threadIdx.x == 0) {
        double v = part[0];
        for (int k = 1; k < (int)(blockDim.x >> 5); ++k) v = fmin(v, part[k]);
        out[(size_t)m * gridDim.x + blockIdx.x] = v;
    }
}

#define CKF(call)                                                                        \
    do {                                                                                 \
        cudaError_t e__ = (call);                                                        \
        if (e__ != cudaSuccess) throw Error(AFD_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e__)); \
    } while (0)

}  // namespace

void check_filters(int32_t nmat, int32_t K, const double* a, const double* b, int32_t nf, int32_t* status,
                   double* min_real, double* max_root) {
    if (K > kMaxCoef) throw Error(AFD_ERR_ARG, "at most 64 filter coefficients");
    std::vector<double> roots((size_t)nmat), lows((size_t)nmat, INFINITY);
    int ndev = 0;
    const bool gpu = cudaGetDeviceCount(&ndev) == cudaSuccess && ndev > 0;
    if (gpu) {
        const int blocks = 8;
        // freed on every path, a failed allocation included
        struct Bufs {
            double *a = nullptr, *b = nullptr, *r = nullptr, *l = nullptr;
            ~Bufs() {
                cudaFree(a);
                cudaFree(b);
                cudaFree(r);
                cudaFree(l);
            }
        } m;
        const size_t nab = (size_t)nmat * K;
        CKF(cudaMalloc(&m.a, nab * sizeof(double)));
        CKF(cudaMalloc(&m.b, nab * sizeof(double)));
        CKF(cudaMalloc(&m.r, (size_t)nmat * sizeof(double)));
        CKF(cudaMalloc(&m.l, (size_t)nmat * blocks * sizeof(double)));
        double *da = m.a, *db = m.b, *dr = m.r, *dl = m.l;
        CKF(cudaMemcpy(da, a, nab * sizeof(double), cudaMemcpyHostToDevice));
        CKF(cudaMemcpy(db, b, nab * sizeof(double), cudaMemcpyHostToDevice));
        k_roots<<<(nmat + 63) / 64, 64>>>(db, nmat, K, dr);
        k_passive<<<dim3(blocks, nmat), 256>>>(da, db, nmat, K, nf, dl);
        CKF(cudaGetLastError());
        std::vector<double> part((size_t)nmat * blocks);
        CKF(cudaMemcpy(roots.data(), dr, (size_t)nmat * sizeof(double), cudaMemcpyDeviceToHost));
        CKF(cudaMemcpy(part.data(), dl, part.size() * sizeof(double), cudaMemcpyDeviceToHost));
        for (int i = 0; i < nmat; ++i)
            for (int k = 0; k < blocks; ++k) lows[(size_t)i] = std::fmin(lows[(size_t)i], part[(size_t)i * blocks + k]);
    } else {
        // no CUDA device: the same FP64 arithmetic on the host (a coefficient
        // check before a run, not part of the step)
        for (int m = 0; m < nmat; ++m) {
            roots[(size_t)m] = max_root_of(b + (size_t)m * K, K);
            for (int f = 0; f < nf; ++f) {
                const double w = 3.141592653589793 * (double)f / (double)(nf - 1);
                lows[(size_t)m] = std::fmin(lows[(size_t)m], re_admittance(a + (size_t)m * K, b + (size_t)m * K, K, w));
            }
        }
    }
    for (int m = 0; m < nmat; ++m) {
        int st = 0;
        if (!(roots[(size_t)m] < 1.0)) st |= 1;
        if (!(lows[(size_t)m] >= 0.0)) st |= 2;
        status[m] = st;
        if (min_real) min_real[m] = lows[(size_t)m];
        if (max_root) max_root[m] = roots[(size_t)m];
    }
}

// ---------------------------------------------------------------------------
// Allocation-free variant of the filter check.
//
// For callers that must not allocate device memory: a process that runs
// under a fixed GPU memory budget set by its host application (which has
// reserved the device memory for itself), or a setup path that re-checks
// filter coefficients after the simulations have taken the rest of the
// device and a cudaMalloc could fail. The scratch lives in one file-scope
// device array; inputs and outputs stay host arrays.
// Limits: nmat <= kStaticMaxMat materials, ncoef <= kStaticMaxCoef.
// Every call reuses the same array, so calls that overlap on the GPU (from
// several host threads on one device) race and must be serialised by the
// caller. The copies are synchronous cudaMemcpy calls and the kernels go to
// the legacy default stream, so a call waits for work queued on that
// device's blocking streams (the simulation engine's own streams are
// non-blocking). Each call looks up the array's device address
// (cudaGetSymbolAddress) with the device current: an address kept from an
// earlier call would be stale after a cudaDeviceReset. The first call on a
// device loads the module there; make it before any stream capture.
// ---------------------------------------------------------------------------
constexpr int kStaticMaxMat = 64;
constexpr int kStaticMaxCoef = 16;
constexpr int kStaticBlocks = 8;
constexpr int kStaticDoubles =
    2 * kStaticMaxMat * kStaticMaxCoef + kStaticMaxMat + kStaticMaxMat * kStaticBlocks;
static __device__ __align__(256) double g_filter_scratch[kStaticDoubles];

// Device address of g_filter_scratch on the current device.
static double* scratch_on_current_device() {
    void* ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_filter_scratch);
    if (e != cudaSuccess || !ptr)
        throw Error(AFD_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    return static_cast<double*>(ptr);
}

void check_filters_static(int32_t nmat, int32_t K, const double* a, const double* b, int32_t nf,
                          int32_t* status, double* min_real, double* max_root) {
    if (nmat > kStaticMaxMat || K > kStaticMaxCoef)
        throw Error(AFD_ERR_ARG, "afd_check_filters_static: at most " + std::to_string(kStaticMaxMat) +
                                     " materials of " + std::to_string(kStaticMaxCoef) +
                                     " coefficients fit its fixed scratch (got " + std::to_string(nmat) + " x " +
                                     std::to_string(K) + ")");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        throw Error(AFD_ERR_CUDA, "afd_check_filters_static needs a CUDA device");
    double* base = scratch_on_current_device();
    double* da = base;
    double* db = base + kStaticMaxMat * kStaticMaxCoef;
    double* dr = base + 2 * kStaticMaxMat * kStaticMaxCoef;
    double* dl = dr + kStaticMaxMat;
    const size_t nab = (size_t)nmat * K;
    CKF(cudaMemcpy(da, a, nab * sizeof(double), cudaMemcpyHostToDevice));
    CKF(cudaMemcpy(db, b, nab * sizeof(double), cudaMemcpyHostToDevice));
    // every result slot read below is written by this call's kernels; the
    // slots are cleared anyway so that a failed launch cannot hand back the
    // previous call's values
    CKF(cudaMemset(dr, 0, (size_t)(kStaticMaxMat + kStaticMaxMat * kStaticBlocks) * sizeof(double)));
    k_roots_static<kStaticMaxCoef><<<(nmat + 63) / 64, 64>>>(db, nmat, K, dr);
    k_passive_static<<<dim3(kStaticBlocks, nmat), 256>>>(da, db, nmat, K, nf, dl);
    CKF(cudaGetLastError());
    double roots[kStaticMaxMat];
    double part[kStaticMaxMat * kStaticBlocks];
    CKF(cudaMemcpy(roots, dr, (size_t)nmat * sizeof(double), cudaMemcpyDeviceToHost));
    CKF(cudaMemcpy(part, dl, (size_t)nmat * kStaticBlocks * sizeof(double), cudaMemcpyDeviceToHost));
    for (int m = 0; m < nmat; ++m) {
        double lo = INFINITY;
        for (int k = 0; k < kStaticBlocks; ++k) lo = std::fmin(lo, part[m * kStaticBlocks + k]);
        int st = 0;
        if (!(roots[m] < 1.0)) st |= 1;
        if (!(lo >= 0.0)) st |= 2;
        status[m] = st;
        if (min_real) min_real[m] = lo;
        if (max_root) max_root[m] = roots[m];
    }
}

int device_name(int32_t index, std::string* name) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return AFD_ERR_CUDA;
    if (index < 0 || index >= ndev) return AFD_ERR_ARG;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, index) != cudaSuccess) return AFD_ERR_CUDA;
    *name = prop.name;
    return AFD_OK;
}

}  // namespace afd
