// FP64 admittance-filter preprocessing checks (stability and passivity).
#pragma once
#include <cstdint>
#include <string>

namespace afd {

// For each material m with coefficients a[m][0..ncoef), b[m][0..ncoef):
// the boundary recursion computes the filter input from b (lrs_1.cl:73-76,
// 122-124: b0*in_n = a0*out_n - sum_{i>=1}(b_i*in_{n-i} - a_i*out_{n-i})),
// so its poles are the roots of b0 z^(K-1) + b1 z^(K-2) + ... + b_{K-1};
// the wall admittance is Y(z) = A(z)/B(z). status bit0: some root has
// |z| >= 1; bit1: Re{Y(e^jw)} < 0 at some of n_freq frequencies in [0, pi].
// Runs on the current CUDA device when one is present, else on the host.
void check_filters(int32_t nmat, int32_t ncoef, const double* a, const double* b, int32_t n_freq,
                   int32_t* status, double* min_real, double* max_root);

// Same check with its device scratch in a fixed file-scope array instead
// of cudaMalloc'd buffers (nmat <= 64, ncoef <= 16); needs a CUDA device.
void check_filters_static(int32_t nmat, int32_t ncoef, const double* a, const double* b, int32_t n_freq,
                          int32_t* status, double* min_real, double* max_root);

// Name of CUDA device `index`; AFD_ERR_ARG past the end, AFD_ERR_CUDA
// without a device.
int device_name(int32_t index, std::string* name);

}  // namespace afd
