// Shared helpers of the cdftb library: status plumbing, launch checks and small device utilities.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/cdftb.h"

namespace cdftb {

// The last failed CUDA call's error, per host thread (cdftb_last_cuda_error).
extern thread_local int g_last_cuda_error;
// Kernels this library has launched in this process (cdftb_launch_count).
extern unsigned long long g_launch_count;

inline int check_launch() {
    __atomic_fetch_add(&g_launch_count, 1ull, __ATOMIC_RELAXED);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        g_last_cuda_error = static_cast<int>(e);
        return CDFTB_ERR_LAUNCH;
    }
    return CDFTB_OK;
}

inline int check(cudaError_t e) {
    if (e != cudaSuccess) {
        g_last_cuda_error = static_cast<int>(e);
        return CDFTB_ERR_LAUNCH;
    }
    return CDFTB_OK;
}

inline cudaStream_t as_stream(cdftb_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }

inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

template <typename T>
__device__ __forceinline__ T load_as(const void* p, int dtype, int64_t i);

template <>
__device__ __forceinline__ double load_as<double>(const void* p, int dtype, int64_t i) {
    return dtype == CDFTB_F64 ? static_cast<const double*>(p)[i]
                              : static_cast<double>(static_cast<const float*>(p)[i]);
}

template <>
__device__ __forceinline__ float load_as<float>(const void* p, int dtype, int64_t i) {
    return dtype == CDFTB_F64 ? static_cast<float>(static_cast<const double*>(p)[i])
                              : static_cast<const float*>(p)[i];
}

template <typename T>
__device__ __forceinline__ void store_as(void* p, int dtype, int64_t i, T v) {
    if (dtype == CDFTB_F64)
        static_cast<double*>(p)[i] = static_cast<double>(v);
    else
        static_cast<float*>(p)[i] = static_cast<float>(v);
}

// Staggered first-derivative weights onto a face from `accuracy` nodes (k = -p .. p-1), the exact
// rationals of src/cdft/operators/divergence.py:31-74 rounded to double. Filled on the host.
struct StaggeredTaps {
    double c[8];
    int half;
};

StaggeredTaps staggered_taps(int accuracy);

// The two Chebyshev filter paths behind cdftb_chebyshev_filter (stencil.cu, filter.cu).
int generic_chebyshev_filter(const cdftb_operator* op, const void* block, int in_dtype, void* out, int out_dtype,
                             void* work, int64_t batch, const double* coefficients, int degree, cdftb_stream_t stream);
int64_t slab_filter_work_bytes(const cdftb_operator* op, int64_t batch);
int generic_cusp_apply(const cdftb_operator* op, const void* phi, int in_dtype, void* out, int out_dtype,
                       int64_t batch, int kinetic_only, cdftb_stream_t stream);
bool slab_filter_applies(const cdftb_operator* op);
int slab_chebyshev_filter(const cdftb_operator* op, const void* block, int in_dtype, void* out, int out_dtype,
                          void* work, int64_t batch, const double* coefficients, int degree, cudaStream_t stream);

}  // namespace cdftb
