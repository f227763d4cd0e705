// LMS impulse-response estimation on the GPU: the estimator of
// anc_field_py/ancutil.py:24-37 (EstimateIr), which the reference runs as a
// Python loop over samples ("takes hours" for the 10 s, 64000-tap case).
//
// The reference's recursion, per pass over the samples (delay line u
// cleared at the start of each pass, weights w kept):
//     u <- [x_k, u_0 .. u_{N-2}],  e_k = d_k - w.u,  w <- w + (2 mu e_k) u.
// Over a block of B samples k0 .. k0+B-1 the weights seen by sample k are
// the block-start weights plus the updates of the block's earlier samples,
// so  e_k = d_k - (y0_k + 2 mu sum_{m<k} e_m R(m, k))  with
//   y0_k = sum_j w_j x_{k-j}                 (block-start weights)
//   R(m, k) = sum_{j<N} x_{m-j} x_{k-j}       (sliding-window correlation)
// and R(m, m+l) = r_l(m) follows from r_l(m-1) by adding x_m x_{m+l} and
// removing x_{m-N} x_{m+l-N}. This is the same recursion reassociated; the
// N-tap work becomes three parallel passes per block:
//   k_lms_y0     y0 for the block, taps and samples split over CTAs
//                (partial sums per tap chunk)
//   k_lms_solve  one CTA: y0 from the partials, R by lag, the errors
//   k_lms_update w_j <- w_j + (2 mu e_m) x_{m-j} in sample order, per tap
// All arithmetic is FP64, as in the reference.
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/afd_lms.h"

namespace afd {
namespace lms {

constexpr int B = 128;       // samples per block
constexpr int J = 4096;      // taps per CTA of k_lms_y0
constexpr int SPC = 16;      // samples per CTA of k_lms_y0 (16 x 8 = 128 CTAs at 64000 taps)
constexpr int Y0_THREADS = 256;
constexpr size_t Y0_SMEM = (size_t)(2 * J + SPC) * sizeof(double);

// CTA (c, g): taps j0 = c J .. j0 + J - 1 of samples k0 + g SPC .. +SPC-1.
// xs[o + t] = x_t for 0 <= t < steps, zero elsewhere (o = N + J + B).
__global__ void __launch_bounds__(Y0_THREADS) k_lms_y0(const double* __restrict__ w, const double* __restrict__ xs,
                                                       int64_t o, int N, int64_t k0, int nb, double* partial) {
    extern __shared__ double y0_smem[];
    double* ws = y0_smem;      // [J]
    double* xw = ws + J;       // [J + SPC - 1]
    const int j0 = blockIdx.x * J, s0 = blockIdx.y * SPC;
    if (s0 >= nb) return;  // whole CTA
    const int nj = min(J, N - j0);
    for (int t = threadIdx.x; t < nj; t += blockDim.x) ws[t] = w[j0 + t];
    // x_{k-j} for k in [k0+s0, k0+s0+SPC), j in [j0, j0+J): xw[q] = x_{k0+s0-j0-(J-1)+q}
    const int64_t base = o + k0 + s0 - j0 - (J - 1);
    for (int t = threadIdx.x; t < J + SPC - 1; t += blockDim.x) xw[t] = xs[base + t];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = warp; i < SPC && s0 + i < nb; i += Y0_THREADS / 32) {
        double acc = 0.0;
        // x_{k0+s0+i-j0-jj} = xw[(J - 1) + i - jj]
        for (int jj = lane; jj < nj; jj += 32) acc += ws[jj] * xw[(J - 1) + i - jj];
        for (int s = 16; s > 0; s >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, s);
        if (lane == 0) partial[(size_t)blockIdx.x * B + s0 + i] = acc;
    }
}

// One CTA of B threads. r_state[l]: r_l at the last sample of the previous
// block (zero at the start of a pass). The two windows of x the lag sums
// read (x_{k0 ..}, x_{k0-N ..}, 2 B - 1 values each) are staged in shared
// memory first, so the sequential sums wait on shared, not global, loads.
constexpr int XW = 2 * B;  // window length (2 B - 1 used)
__global__ void __launch_bounds__(B) k_lms_solve(const double* __restrict__ xs, int64_t o, int N, int64_t k0,
                                                 int nb, const double* __restrict__ partial, int nchunk,
                                                 const double* __restrict__ d, double mu, double* r_state,
                                                 double* e_out) {
    extern __shared__ double smem[];
    double* R = smem;          // R[i * B + l] = r_l(k0 + i)
    double* y0 = R + B * B;    // [B]
    double* e = y0 + B;        // [B]
    double* xa = e + B;        // [XW]: x_{k0 + q}
    double* xb = xa + XW;      // [XW]: x_{k0 - N + q}
    double* dd = xb + XW;      // [B]: d_{k0 + i}
    const int t = threadIdx.x;
    for (int q = t; q < nb + B - 1; q += B) {
        xa[q] = xs[o + k0 + q];
        xb[q] = xs[o + k0 - N + q];
    }
    if (t < nb) {
        dd[t] = d[k0 + t];
        // the partials in chunk order; unrolled so that the loads overlap
        double s = 0.0;
        int c = 0;
        for (; c + 8 <= nchunk; c += 8) {
            double v[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) v[u] = partial[(size_t)(c + u) * B + t];
#pragma unroll
            for (int u = 0; u < 8; ++u) s += v[u];
        }
        for (; c < nchunk; ++c) s += partial[(size_t)c * B + t];
        y0[t] = s;
    }
    __syncthreads();
    if (t >= 1) {
        double r = r_state[t];
        for (int i = 0; i < nb; ++i) {
            r += xa[i] * xa[i + t] - xb[i] * xb[i + t];
            R[i * B + t] = r;
        }
        r_state[t] = r;
    }
    __syncthreads();
    // e_i = d_i - (y0_i + 2 mu sum_{m<i} e_m R(m, i)), forward substitution
    // by one warp over sub-blocks of 32 samples: lane j of a sub-block first
    // takes the earlier sub-blocks' errors, then each error of its own
    // sub-block as the owning lane finalises it (one shuffle per sample);
    // every sum runs in sample order.
    if (t < 32) {
        const double c2 = 2 * mu;
        for (int b0 = 0; b0 < nb; b0 += 32) {
            const int j = b0 + t;
            double acc = 0.0;
            if (j < nb)
                for (int m = 0; m < b0; ++m) acc += e[m] * R[m * B + (j - m)];
            const int b1 = min(b0 + 32, nb);
            for (int i = b0; i < b1; ++i) {
                double ei = 0.0;
                if (j == i) {
                    ei = dd[i] - (y0[i] + c2 * acc);
                    e[i] = ei;
                }
                ei = __shfl_sync(0xffffffffu, ei, i - b0);
                if (j > i && j < nb) acc += ei * R[i * B + (j - i)];
            }
            __syncwarp();
        }
    }
    __syncthreads();
    if (t < nb) e_out[t] = e[t];
}

// w_j <- w_j + (2 mu e_m) x_{m-j} for the block's samples in order. The
// CTA's taps j0 .. j0+255 read x_{k0-j0-255} .. x_{k0-j0+nb-1}, staged in
// shared memory first.
constexpr int UPD_THREADS = 256;
__global__ void __launch_bounds__(UPD_THREADS) k_lms_update(double* w, const double* __restrict__ xs, int64_t o,
                                                            int N, int64_t k0, int nb,
                                                            const double* __restrict__ e_in, double mu) {
    __shared__ double c[B];
    __shared__ double win[UPD_THREADS + B];
    const int tid = threadIdx.x;
    const int j0 = blockIdx.x * UPD_THREADS;
    if (tid < nb) c[tid] = 2 * mu * e_in[tid];
    const int64_t base = o + k0 - j0 - (UPD_THREADS - 1);
    for (int q = tid; q < UPD_THREADS - 1 + nb; q += UPD_THREADS) win[q] = xs[base + q];
    __syncthreads();
    const int j = j0 + tid;
    if (j >= N) return;
    double v = w[j];
    const double* xp = win + (UPD_THREADS - 1 - tid);  // xp[i] = x_{k0 + i - j}
    for (int i = 0; i < nb; ++i) v = v + c[i] * xp[i];
    w[j] = v;
}

struct Err : std::runtime_error {
    int code;
    Err(int cd, const std::string& m) : std::runtime_error(m), code(cd) {}
};

#define LCK(call)                                                                                   \
    do {                                                                                            \
        cudaError_t e__ = (call);                                                                   \
        if (e__ != cudaSuccess) throw Err(AFD_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e__)); \
    } while (0)

template <typename T>
struct Buf {
    T* p = nullptr;
    ~Buf() {
        if (p) cudaFree(p);
    }
    void alloc(size_t n) {
        LCK(cudaMalloc(&p, n * sizeof(T)));
        // zeroed on the legacy stream, which the non-blocking work stream
        // does not wait for: finished before return
        LCK(cudaMemset(p, 0, n * sizeof(T)));
        LCK(cudaStreamSynchronize(cudaStreamLegacy));
    }
};

thread_local std::string g_err;

void estimate(const double* x, int64_t nx, const double* d, int64_t nd, int32_t taps, double mu, int32_t epochs,
              int32_t device, double* w_out) {
    if (!x || !d || !w_out) throw Err(AFD_ERR_ARG, "null pointer");
    if (taps < 1 || taps > (1 << 26)) throw Err(AFD_ERR_ARG, "taps must be in 1 .. 2^26");
    if (nx < 0 || nd < 0 || epochs < 0) throw Err(AFD_ERR_ARG, "negative length or epoch count");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) throw Err(AFD_ERR_CUDA, "no CUDA device available");
    if (device < 0 || device >= ndev) throw Err(AFD_ERR_ARG, "device ordinal out of range");
    LCK(cudaSetDevice(device));
    const int N = taps;
    const int64_t steps = std::min(nx, nd);
    const int64_t o = (int64_t)N + J + B;  // zero padding in front of x_0 (k_lms_y0 stages J + B values)
    const size_t nxs = (size_t)(o + steps + 2 * B);
    std::vector<double> hx(nxs, 0.0);
    std::memcpy(hx.data() + o, x, (size_t)steps * sizeof(double));
    Buf<double> xs, dd, w, partial, e, r;
    const int nchunk = (N + J - 1) / J;
    xs.alloc(nxs);
    dd.alloc((size_t)std::max<int64_t>(steps, 1));
    w.alloc((size_t)N);
    partial.alloc((size_t)nchunk * B);
    e.alloc(B);
    r.alloc(B);
    cudaStream_t st;
    LCK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    try {
        LCK(cudaMemcpyAsync(xs.p, hx.data(), nxs * sizeof(double), cudaMemcpyHostToDevice, st));
        if (steps) LCK(cudaMemcpyAsync(dd.p, d, (size_t)steps * sizeof(double), cudaMemcpyHostToDevice, st));
        const size_t solve_smem = (size_t)(B * B + 3 * B + 2 * XW) * sizeof(double);
        LCK(cudaFuncSetAttribute((const void*)k_lms_solve, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)solve_smem));
        LCK(cudaFuncSetAttribute((const void*)k_lms_y0, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)Y0_SMEM));
        // one pass over the samples: the delay line emptied, then per block
        // of B samples its outputs, errors and weight update
        auto pass = [&]() {
            LCK(cudaMemsetAsync(r.p, 0, B * sizeof(double), st));
            for (int64_t k0 = 0; k0 < steps; k0 += B) {
                const int nb = (int)std::min<int64_t>(B, steps - k0);
                k_lms_y0<<<dim3((unsigned)nchunk, (unsigned)((nb + SPC - 1) / SPC)), Y0_THREADS, Y0_SMEM, st>>>(
                    w.p, xs.p, o, N, k0, nb, partial.p);
                k_lms_solve<<<1, B, solve_smem, st>>>(xs.p, o, N, k0, nb, partial.p, nchunk, dd.p, mu, r.p, e.p);
                k_lms_update<<<(N + UPD_THREADS - 1) / UPD_THREADS, UPD_THREADS, 0, st>>>(w.p, xs.p, o, N, k0, nb,
                                                                                        e.p, mu);
            }
        };
        if (epochs >= 2 && steps > 0) {
            // every pass launches the same kernels with the same arguments:
            // captured once as a graph and replayed per pass
            cudaGraph_t graph = nullptr;
            cudaGraphExec_t exec = nullptr;
            LCK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            try {
                pass();
            } catch (...) {
                cudaStreamEndCapture(st, &graph);  // leave the stream out of capture mode
                if (graph) cudaGraphDestroy(graph);
                throw;
            }
            const cudaError_t ce = cudaStreamEndCapture(st, &graph);
            if (ce != cudaSuccess) {
                if (graph) cudaGraphDestroy(graph);
                LCK(ce);
            }
            const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
            cudaGraphDestroy(graph);
            LCK(ie);
            cudaError_t le = cudaSuccess;
            for (int ep = 0; ep < epochs && le == cudaSuccess; ++ep) le = cudaGraphLaunch(exec, st);
            const cudaError_t se = cudaStreamSynchronize(st);
            cudaGraphExecDestroy(exec);
            LCK(le);
            LCK(se);
        } else {
            for (int ep = 0; ep < epochs; ++ep) pass();
        }
        LCK(cudaGetLastError());
        LCK(cudaMemcpyAsync(w_out, w.p, (size_t)N * sizeof(double), cudaMemcpyDeviceToHost, st));
        LCK(cudaStreamSynchronize(st));
    } catch (...) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
        throw;
    }
    cudaStreamDestroy(st);
}

}  // namespace lms
}  // namespace afd

extern "C" {

int afd_lms_estimate(const double* x, int64_t nx, const double* d, int64_t nd, int32_t taps, double mu,
                     int32_t epochs, int32_t device, double* w) {
    try {
        afd::lms::estimate(x, nx, d, nd, taps, mu, epochs, device, w);
        return AFD_OK;
    } catch (const afd::lms::Err& e) {
        afd::lms::g_err = e.what();
        return e.code;
    } catch (const std::exception& e) {
        afd::lms::g_err = e.what();
        return AFD_ERR_STATE;
    }
}

const char* afd_lms_last_error(void) { return afd::lms::g_err.c_str(); }

}  // extern "C"
