// Reciprocal-space filters of a field on the box, by a periodic transform of the box itself (not
// zero-padded), q from the box's own frequencies (2 pi fftfreq(n, h) per axis):
//   (s2) the Kerker preconditioner of the density mixers (src/cdft/scf/mixing.py:35-56),
//        F(q) q^2 / (q^2 + q0^2);
//   (f4) the Teter--Payne--Allan kinetic preconditioner of LOBPCG (src/cdft/eigen/lobpcg.py:160-189),
//        P(x) / (P(x) + 16 x^4), P = 27 + 18 x + 12 x^2 + 8 x^3, x = (q^2 / 2) / E_ref.
//
// The box edge is any length (65 = 5 x 13 at He 65^3), so the transforms are direct sums along
// each axis with a twiddle table built per line in shared memory from the exact index (j k mod n):
// O(n) per output, about 6 n N complex multiply-adds per call -- 0.1 GFLOP at 65^3, a small cost
// once per SCF iteration, and only when the Kerker option is on. Five launches: z forward (real
// in), y forward, x forward x filter x x inverse (one line in shared memory), y inverse, z inverse
// (real part out, scaled by 1/N). Each CTA takes one line of one spin channel.

#include "common.cuh"

namespace cdftb {
namespace {

enum class Pass : int { ZForward = 0, YForward = 1, XFilter = 2, YInverse = 3, ZInverse = 4 };

constexpr int kMaxEdge = 1024;  // shared memory: 3 lines of complex doubles + the twiddles

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// frequency index of bin i of an n-point transform (numpy's fftfreq order)
__device__ __forceinline__ int freq_index(int i, int n) { return i < (n + 1) / 2 ? i : i - n; }

// out[k] = sum_j in[j] w[(j k) mod n], w[m] = exp(sign 2 pi i m / n), for the k this thread owns
__device__ __forceinline__ void line_dft(const double2* in, double2* out, const double2* w, int n) {
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        double2 acc = make_double2(0.0, 0.0);
        int m = 0;  // (j k) mod n, advanced by k each step
        for (int j = 0; j < n; ++j) {
            const double2 t = cmul(in[j], w[m]);
            acc.x += t.x;
            acc.y += t.y;
            m += k;
            if (m >= n) m -= n;
        }
        out[k] = acc;
    }
}

__device__ __forceinline__ void twiddles(double2* w, int n, double sign) {
    for (int m = threadIdx.x; m < n; m += blockDim.x) {
        double s, c;
        sincospi(2.0 * m / n, &s, &c);
        w[m] = make_double2(c, sign * s);
    }
}

// One line per CTA. Box (nx, ny, nz) in C order; blockIdx.y is the spin channel.
// the filter of kind `kind` at q^2: 0 Kerker (param q0), 1 Teter--Payne--Allan (param E_ref)
__device__ __forceinline__ double reciprocal_filter(int kind, double q2, double param) {
    if (kind == 0) return q2 / (q2 + param * param);
    const double x = (0.5 * q2) / param;
    const double poly = 27.0 + 18.0 * x + 12.0 * (x * x) + 8.0 * (x * x * x);
    return poly / (poly + 16.0 * (x * x * x * x));
}

template <Pass P>
__global__ void kerker_pass_kernel(const double* __restrict__ real_in, double2* __restrict__ a,
                                   double2* __restrict__ b, double* __restrict__ real_out, int nx, int ny, int nz,
                                   double spacing, int kind, double q0, double scale) {
    extern __shared__ double2 sm[];
    const int64_t npts = int64_t(nx) * ny * nz;
    const int64_t chan = blockIdx.y * npts;
    int n;
    int64_t base, stride;
    int line = blockIdx.x;
    if (P == Pass::ZForward || P == Pass::ZInverse) {
        n = nz;
        base = int64_t(line) * nz;  // line = x * ny + y
        stride = 1;
    } else if (P == Pass::YForward || P == Pass::YInverse) {
        n = ny;
        const int x = line / nz, z = line - x * nz;
        base = int64_t(x) * ny * nz + z;
        stride = nz;
    } else {
        n = nx;
        base = line;  // line = y * nz + z
        stride = int64_t(ny) * nz;
    }
    double2* w = sm;
    double2* l0 = sm + n;
    double2* l1 = l0 + n;
    const bool inverse = P == Pass::YInverse || P == Pass::ZInverse;
    twiddles(w, n, inverse ? 1.0 : -1.0);
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        const int64_t p = chan + base + j * stride;
        // buffers: z forward real -> a, y forward a -> b, x filter b -> a, y inverse a -> b, z inverse b -> real
        l0[j] = P == Pass::ZForward ? make_double2(real_in[p], 0.0)
                                    : (P == Pass::YForward || P == Pass::YInverse ? a[p] : b[p]);
    }
    __syncthreads();
    line_dft(l0, l1, w, n);
    __syncthreads();
    if (P == Pass::XFilter) {
        // multiply by the filter and transform back along x
        const int y = line / nz, z = line - y * nz;
        const double two_pi = 2.0 * 3.141592653589793;
        const double ky = two_pi * (double(freq_index(y, ny)) / (ny * spacing));
        const double kz = two_pi * (double(freq_index(z, nz)) / (nz * spacing));
        for (int i = threadIdx.x; i < nx; i += blockDim.x) {
            const double kx = two_pi * (double(freq_index(i, nx)) / (nx * spacing));
            const double q2 = kx * kx + ky * ky + kz * kz;
            const double f = reciprocal_filter(kind, q2, q0);
            l1[i] = make_double2(l1[i].x * f, l1[i].y * f);
        }
        __syncthreads();
        twiddles(w, n, 1.0);
        __syncthreads();
        line_dft(l1, l0, w, n);
        __syncthreads();
        for (int j = threadIdx.x; j < n; j += blockDim.x) a[chan + base + j * stride] = l0[j];
    } else {
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            const int64_t p = chan + base + j * stride;
            if (P == Pass::ZInverse)
                real_out[p] = l1[j].x * scale;
            else if (P == Pass::ZForward)
                a[p] = l1[j];
            else
                b[p] = l1[j];  // y forward, y inverse
        }
    }
}

template <Pass P>
int launch_pass(const double* in, double2* a, double2* b, double* out, int nx, int ny, int nz, int channels,
                double spacing, int kind, double q0, double scale, cudaStream_t st) {
    const int lines = P == Pass::ZForward || P == Pass::ZInverse ? nx * ny
                      : P == Pass::YForward || P == Pass::YInverse ? nx * nz
                                                                     : ny * nz;
    const int n = P == Pass::ZForward || P == Pass::ZInverse ? nz : P == Pass::YForward || P == Pass::YInverse ? ny : nx;
    const int threads = n >= 128 ? 128 : (n + 31) / 32 * 32;
    const size_t smem = size_t(3) * n * sizeof(double2);
    dim3 grid(static_cast<unsigned>(lines), static_cast<unsigned>(channels));
    kerker_pass_kernel<P><<<grid, threads, smem, st>>>(in, a, b, out, nx, ny, nz, spacing, kind, q0, scale);
    return check_launch();
}

}  // namespace
}  // namespace cdftb

extern "C" int64_t cdftb_kerker_work_bytes(int nx, int ny, int nz, int channels) {
    if (nx <= 0 || ny <= 0 || nz <= 0 || channels <= 0) return -1;
    return int64_t(2) * channels * nx * ny * nz * int64_t(sizeof(double2));
}

extern "C" int cdftb_reciprocal_filter_f64(const double* field, int channels, int nx, int ny, int nz, double spacing,
                                           int kind, double param, double* out, void* work, int64_t work_bytes,
                                           cdftb_stream_t stream) {
    using namespace cdftb;
    if (!field || !out || !work || channels <= 0 || nx <= 0 || ny <= 0 || nz <= 0 || !(spacing > 0.0) ||
        nx > kMaxEdge || ny > kMaxEdge || nz > kMaxEdge || int64_t(nx) * ny > 0x7fffffff || int64_t(nx) * nz > 0x7fffffff ||
        int64_t(ny) * nz > 0x7fffffff || channels > 65535 || (kind != 0 && kind != 1) || !(param > 0.0))
        return CDFTB_ERR_ARGUMENT;
    if (work_bytes < cdftb_kerker_work_bytes(nx, ny, nz, channels)) return CDFTB_ERR_ARGUMENT;
    cudaStream_t st = as_stream(stream);
    double2* a = static_cast<double2*>(work);
    double2* b = a + int64_t(channels) * nx * ny * nz;
    const double scale = 1.0 / (double(nx) * ny * nz);
    int rc = launch_pass<Pass::ZForward>(field, a, b, out, nx, ny, nz, channels, spacing, kind, param, scale, st);
    if (rc == CDFTB_OK)
        rc = launch_pass<Pass::YForward>(field, a, b, out, nx, ny, nz, channels, spacing, kind, param, scale, st);
    if (rc == CDFTB_OK)
        rc = launch_pass<Pass::XFilter>(field, a, b, out, nx, ny, nz, channels, spacing, kind, param, scale, st);
    if (rc == CDFTB_OK)
        rc = launch_pass<Pass::YInverse>(field, a, b, out, nx, ny, nz, channels, spacing, kind, param, scale, st);
    if (rc == CDFTB_OK)
        rc = launch_pass<Pass::ZInverse>(field, a, b, out, nx, ny, nz, channels, spacing, kind, param, scale, st);
    return rc;
}

extern "C" int cdftb_kerker_precondition_f64(const double* residual, int channels, int nx, int ny, int nz,
                                             double spacing, double q0, double* out, void* work, int64_t work_bytes,
                                             cdftb_stream_t stream) {
    return cdftb_reciprocal_filter_f64(residual, channels, nx, ny, nz, spacing, 0, q0, out, work, work_bytes, stream);
}
