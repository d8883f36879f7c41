// Library-level entry points: version, status text, the CUDA error of the last failure, the
// staggered weights, and the double/float cast at the precision boundary.

#include "common.cuh"

namespace cdftb {

thread_local int g_last_cuda_error = 0;
unsigned long long g_launch_count = 0;

StaggeredTaps staggered_taps(int accuracy) {
    // The exact rationals solving sum_k c_k (k + 1/2)^m = delta_{m,1}, k = -p .. p-1
    // (src/cdft/operators/divergence.py:31-74), each rounded once by an IEEE division of two
    // exactly representable integers, which is what float(Fraction) gives.
    StaggeredTaps t{};
    switch (accuracy) {
        case 2: {
            const double c[2] = {-1.0, 1.0};
            for (int k = 0; k < 2; ++k) t.c[k] = c[k];
            t.half = 1;
            break;
        }
        case 4: {
            const double c[4] = {1.0 / 24.0, -9.0 / 8.0, 9.0 / 8.0, -1.0 / 24.0};
            for (int k = 0; k < 4; ++k) t.c[k] = c[k];
            t.half = 2;
            break;
        }
        case 6: {
            const double c[6] = {-3.0 / 640.0, 25.0 / 384.0, -75.0 / 64.0, 75.0 / 64.0, -25.0 / 384.0, 3.0 / 640.0};
            for (int k = 0; k < 6; ++k) t.c[k] = c[k];
            t.half = 3;
            break;
        }
        case 8: {
            const double c[8] = {5.0 / 7168.0,    -49.0 / 5120.0,  245.0 / 3072.0, -1225.0 / 1024.0,
                                 1225.0 / 1024.0, -245.0 / 3072.0, 49.0 / 5120.0,  -5.0 / 7168.0};
            for (int k = 0; k < 8; ++k) t.c[k] = c[k];
            t.half = 4;
            break;
        }
        default:
            t.half = 0;
    }
    return t;
}

namespace {

template <typename TI, typename TO>
__global__ void cast_kernel(const TI* in, TO* out, int64_t count) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < count;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        out[i] = static_cast<TO>(in[i]);
}

}  // namespace

}  // namespace cdftb

using namespace cdftb;

extern "C" int cdftb_version(void) { return 1 * 10000 + 0 * 100 + 0; }

extern "C" const char* cdftb_status_string(int status) {
    switch (status) {
        case CDFTB_OK: return "ok";
        case CDFTB_ERR_ARGUMENT: return "invalid argument (shape, pointer, order or dtype)";
        case CDFTB_ERR_LAUNCH: return "CUDA launch or runtime failure";
        case CDFTB_ERR_NOT_POSITIVE: return "Gram matrix not positive definite";
        case CDFTB_ERR_TIMEOUT: return "bounded device-side wait expired";
        case CDFTB_ERR_CAPACITY: return "size exceeds a compiled limit";
        default: return "unknown status";
    }
}

extern "C" int cdftb_last_cuda_error(void) { return g_last_cuda_error; }

extern "C" unsigned long long cdftb_launch_count(void) { return __atomic_load_n(&g_launch_count, __ATOMIC_RELAXED); }

extern "C" int cdftb_cast(const void* in, int in_dtype, void* out, int out_dtype, int64_t count,
                          cdftb_stream_t stream) {
    if (count < 0 || (count > 0 && (!in || !out))) return CDFTB_ERR_ARGUMENT;
    if (count == 0) return CDFTB_OK;
    const int threads = 256;
    const int blocks = static_cast<int>(count / threads + 1 < 148 * 16 ? count / threads + 1 : 148 * 16);
    cudaStream_t s = as_stream(stream);
    if (in_dtype == CDFTB_F64 && out_dtype == CDFTB_F32)
        cast_kernel<double, float><<<blocks, threads, 0, s>>>(static_cast<const double*>(in), static_cast<float*>(out), count);
    else if (in_dtype == CDFTB_F32 && out_dtype == CDFTB_F64)
        cast_kernel<float, double><<<blocks, threads, 0, s>>>(static_cast<const float*>(in), static_cast<double*>(out), count);
    else if (in_dtype == CDFTB_F64 && out_dtype == CDFTB_F64)
        return check(cudaMemcpyAsync(out, in, count * 8, cudaMemcpyDeviceToDevice, s));
    else if (in_dtype == CDFTB_F32 && out_dtype == CDFTB_F32)
        return check(cudaMemcpyAsync(out, in, count * 4, cudaMemcpyDeviceToDevice, s));
    else
        return CDFTB_ERR_ARGUMENT;
    return check_launch();
}
