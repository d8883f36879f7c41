// (c) The Coulomb-cutoff Poisson solve (src/cdft/operators/poisson.py:21-107) as five pruned
// axis-wise FFT passes on the device, with the truncated kernel K(G) fused into the x pass. Passes
// 2-4 use the four-step register kernels below when the axis length has a factor pair (A, B), the
// shared-memory Stockham kernels otherwise.
//
// The density occupies the first n of the N = fft_friendly(ceil(pad n)) points of every padded
// axis and only the first n outputs are read back, so each pass transforms only lines that can be
// non-zero and keeps only the outputs a later pass reads:
//   pass 1  z, real -> half complex      rho[x][y][z]        -> A[x][y][kz]    (x < nx, y < ny)
//   pass 2  y, forward                   A[x][y][kz]         -> B[x][ky][kz]   (x < nx)
//   pass 3  x, forward, * K, inverse     B[x][ky][kz]        -> B[x][ky][kz]   (in place, x < nx)
//   pass 4  y, inverse                   B[x][ky][kz]        -> A[x][y][kz]    (y < ny)
//   pass 5  z, half complex -> real      A[x][y][kz]         -> v[x][y][z]     (z < nz), / (Nx Ny Nz)
// Every pass is one CTA per L lines: the lines are staged in shared memory as [element][line] (row
// stride L + 1, so that both the FFT stages and the transposed loads and stores avoid bank
// conflicts) and transformed by a mixed-radix Stockham FFT (radices 4, 2, 3, 5; each stage reads
// one buffer and writes the other, in natural order, with per-stage twiddle tables made on the host
// in double precision). The result is rfftn / *K / irfftn of the zero-padded box up to round-off.

#include <math.h>

#include "common.cuh"

namespace cdftb {

namespace {

struct cplx {
    double re, im;
};

__device__ __forceinline__ cplx operator+(cplx a, cplx b) { return {a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ cplx operator-(cplx a, cplx b) { return {a.re - b.re, a.im - b.im}; }
__device__ __forceinline__ cplx scale(cplx a, double s) { return {a.re * s, a.im * s}; }
__device__ __forceinline__ cplx cmul(cplx a, cplx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
__device__ __forceinline__ cplx cmulc(cplx a, cplx b) { return {a.re * b.re + a.im * b.im, a.im * b.re - a.re * b.im}; }
// i * sign * a
__device__ __forceinline__ cplx rot(cplx a, int sign) { return sign < 0 ? cplx{a.im, -a.re} : cplx{-a.im, a.re}; }

constexpr int MAX_STAGES = 16;

// One axis: N = product of radix[0..nst); stage st has stride s (product of the earlier radices),
// m = N / (s * radix) and twiddles tw[tw_off + p * (radix - 1) + k - 1] = exp(-2 pi i p k / (N / s)).
struct FftPlan {
    int n;
    int nst;
    int radix[MAX_STAGES];
    int stride[MAX_STAGES];
    int m[MAX_STAGES];
    int tw_off[MAX_STAGES];
    const cplx* tw;
};

// Radix-R DFT with the rotation exp(sign 2 pi i / R) (sign -1 forward, +1 inverse).
template <int R>
__device__ __forceinline__ void dft_radix(cplx* a, int sign);

template <>
__device__ __forceinline__ void dft_radix<2>(cplx* a, int) {
    const cplx t = a[0] - a[1];
    a[0] = a[0] + a[1];
    a[1] = t;
}

template <>
__device__ __forceinline__ void dft_radix<4>(cplx* a, int sign) {
    const cplx t0 = a[0] + a[2], t1 = a[0] - a[2], t2 = a[1] + a[3], t3 = rot(a[1] - a[3], sign);
    a[0] = t0 + t2;
    a[1] = t1 + t3;
    a[2] = t0 - t2;
    a[3] = t1 - t3;
}

template <>
__device__ __forceinline__ void dft_radix<3>(cplx* a, int sign) {
    constexpr double s3 = 0.86602540378443864676;  // sqrt(3) / 2
    const cplx t = a[1] + a[2];
    const cplx v = rot(scale(a[1] - a[2], s3), sign);
    const cplx h = {a[0].re - 0.5 * t.re, a[0].im - 0.5 * t.im};
    a[0] = a[0] + t;
    a[1] = h + v;
    a[2] = h - v;
}

template <>
__device__ __forceinline__ void dft_radix<5>(cplx* a, int sign) {
    constexpr double c1 = 0.30901699437494742410;   // cos(2 pi / 5)
    constexpr double c2 = -0.80901699437494742410;  // cos(4 pi / 5)
    constexpr double s1 = 0.95105651629515357212;   // sin(2 pi / 5)
    constexpr double s2 = 0.58778525229247312917;   // sin(4 pi / 5)
    const cplx t1 = a[1] + a[4], t2 = a[2] + a[3], t3 = a[1] - a[4], t4 = a[2] - a[3];
    const cplx x1 = {a[0].re + c1 * t1.re + c2 * t2.re, a[0].im + c1 * t1.im + c2 * t2.im};
    const cplx x2 = {a[0].re + c2 * t1.re + c1 * t2.re, a[0].im + c2 * t1.im + c1 * t2.im};
    const cplx y1 = rot({s1 * t3.re + s2 * t4.re, s1 * t3.im + s2 * t4.im}, sign);
    const cplx y2 = rot({s2 * t3.re - s1 * t4.re, s2 * t3.im - s1 * t4.im}, sign);
    a[0] = a[0] + t1 + t2;
    a[1] = x1 + y1;
    a[2] = x2 + y2;
    a[3] = x2 - y2;
    a[4] = x1 - y1;
}

template <int R>
__device__ __forceinline__ void stage_radix(const cplx* __restrict__ x, cplx* __restrict__ y, int s, int m,
                                            const cplx* __restrict__ tw, int sign, int lp, int lane, int ty, int nty,
                                            int nb) {
    for (int b = ty; b < nb; b += nty) {
        const int p = b / s;
        const int q = b - p * s;
        cplx a[R];
#pragma unroll
        for (int j = 0; j < R; ++j) a[j] = x[(q + s * (p + j * m)) * lp + lane];
        dft_radix<R>(a, sign);
        const cplx* w = tw + p * (R - 1);
        y[(q + s * R * p) * lp + lane] = a[0];
#pragma unroll
        for (int k = 1; k < R; ++k) {
            const cplx wk = w[k - 1];
            y[(q + s * (R * p + k)) * lp + lane] = sign < 0 ? cmul(a[k], wk) : cmulc(a[k], wk);
        }
    }
}

// The FFT of the lines held in x ([N][lp]); y is scratch of the same size. Returns the buffer that
// holds the result. Called by every thread of the CTA (it synchronises after each stage).
__device__ cplx* fft_lines(cplx* x, cplx* y, const FftPlan& P, int sign, int lp, int lane, int ty, int nty) {
    for (int st = 0; st < P.nst; ++st) {
        const int R = P.radix[st];
        const int s = P.stride[st];
        const int m = P.m[st];
        const cplx* tw = P.tw + P.tw_off[st];
        const int nb = P.n / R;
        switch (R) {
            case 4: stage_radix<4>(x, y, s, m, tw, sign, lp, lane, ty, nty, nb); break;
            case 2: stage_radix<2>(x, y, s, m, tw, sign, lp, lane, ty, nty, nb); break;
            case 3: stage_radix<3>(x, y, s, m, tw, sign, lp, lane, ty, nty, nb); break;
            default: stage_radix<5>(x, y, s, m, tw, sign, lp, lane, ty, nty, nb); break;
        }
        __syncthreads();
        cplx* t = x;
        x = y;
        y = t;
    }
    return x;
}

// ---------------------------------------------------------------------------------------------
// Four-step transforms in registers, for line lengths N = A B with A, B in {8, 9, 10, 12, 15, 16,
// 18, 20}. For n = B n1 + n2 and k = k1 + A k2:
//   X[k1 + A k2] = sum_n2 W_B^(n2 k2) W_N^(n2 k1) sum_n1 x[B n1 + n2] W_A^(n1 k1),
// so a thread does one A-point DFT (over n1, fixed n2) and, after an in-place exchange through
// shared memory, one B-point DFT (over n2, fixed k1), each entirely in registers. The small DFTs
// are nested radix 2/3/4/5 butterflies with their internal twiddles from a constant table of the
// 720th roots of unity (every size here divides 720); W_N comes from a per-axis table.

__constant__ cplx kUnit720[720];  // exp(-2 pi i j / 720)

template <int R>
__device__ __forceinline__ cplx unit_root(int m, int sign) {
    const cplx w = kUnit720[(m % R) * (720 / R)];
    return sign < 0 ? w : cplx{w.re, -w.im};
}

template <int R>
struct FirstFactor {
    static constexpr int value = R % 4 == 0 ? 4 : (R % 2 == 0 ? 2 : (R % 3 == 0 ? 3 : 5));
};

// In-place DFT of R values held in registers (natural order in and out), sign -1 forward.
template <int R>
__device__ __forceinline__ void small_dft(cplx* a, int sign) {
    if constexpr (R == 2 || R == 3 || R == 4 || R == 5) {
        dft_radix<R>(a, sign);
    } else {
        constexpr int P = FirstFactor<R>::value;
        constexpr int Q = R / P;
        static_assert(P * Q == R && 720 % R == 0, "small DFT sizes divide 720");
        cplx b[R];
#pragma unroll
        for (int n2 = 0; n2 < Q; ++n2) {
            cplx c[P];
#pragma unroll
            for (int n1 = 0; n1 < P; ++n1) c[n1] = a[Q * n1 + n2];
            small_dft<P>(c, sign);
#pragma unroll
            for (int k1 = 0; k1 < P; ++k1) b[k1 * Q + n2] = (n2 * k1 == 0) ? c[k1] : cmul(c[k1], unit_root<R>(n2 * k1, sign));
        }
#pragma unroll
        for (int k1 = 0; k1 < P; ++k1) {
            cplx c[Q];
#pragma unroll
            for (int n2 = 0; n2 < Q; ++n2) c[n2] = b[k1 * Q + n2];
            small_dft<Q>(c, sign);
#pragma unroll
            for (int k2 = 0; k2 < Q; ++k2) a[k1 + P * k2] = c[k2];
        }
    }
}

constexpr int kLines4 = 8;     // lines per CTA of the four-step kernels
constexpr int kThreads4 = 128;

// Step 1 of a forward (sign -1) or inverse (+1) transform of the L lines in buf ([N][L+1]): per
// (line, n2), the A-point DFT over n1 of x[B n1 + n2], times W_N^(+-n2 k1), back in place.
template <int A, int B>
__device__ __forceinline__ void fourstep_first(cplx* buf, const cplx* __restrict__ twn, int sign) {
    constexpr int N = A * B, L = kLines4, LP = L + 1;
    for (int task = threadIdx.x; task < B * L; task += kThreads4) {
        const int line = task % L, n2 = task / L;
        cplx v[A];
#pragma unroll
        for (int n1 = 0; n1 < A; ++n1) v[n1] = buf[(B * n1 + n2) * LP + line];
        small_dft<A>(v, sign);
#pragma unroll
        for (int k1 = 0; k1 < A; ++k1) {
            const cplx w = twn[(n2 * k1) % N];
            buf[(B * k1 + n2) * LP + line] = sign < 0 ? cmul(v[k1], w) : cmulc(v[k1], w);
        }
    }
}

// Pass 3, four-step: the x lines of one system ([nx][inner]) -- forward, times K, inverse -- with
// the K multiply and the first inverse step on the registers of the second forward step.
template <int A, int B>
__global__ void __launch_bounds__(kThreads4) fft_x_fourstep_kernel(cplx* __restrict__ data, int nx, int64_t inner,
                                                                  const double* __restrict__ kernel,
                                                                  const cplx* __restrict__ twn) {
    constexpr int N = A * B, L = kLines4, LP = L + 1;
    __shared__ cplx buf[N * LP];
    const int64_t c0 = int64_t(blockIdx.x) * L;
    cplx* col = data + int64_t(blockIdx.y) * nx * inner + c0;
#pragma unroll 4
    for (int idx = threadIdx.x; idx < N * L; idx += kThreads4) {
        const int line = idx % L, x = idx / L;
        buf[x * LP + line] = (x < nx && c0 + line < inner) ? col[int64_t(x) * inner + line] : cplx{0.0, 0.0};
    }
    __syncthreads();
    fourstep_first<A, B>(buf, twn, -1);
    __syncthreads();
    for (int task = threadIdx.x; task < A * L; task += kThreads4) {
        const int line = task % L, k1 = task / L;
        const bool live = c0 + line < inner;
        cplx v[B];
#pragma unroll
        for (int n2 = 0; n2 < B; ++n2) v[n2] = buf[(B * k1 + n2) * LP + line];
        small_dft<B>(v, -1);  // X[k1 + A k2] = v[k2]
#pragma unroll
        for (int k2 = 0; k2 < B; ++k2)
            v[k2] = scale(v[k2], live ? kernel[int64_t(k1 + A * k2) * inner + c0 + line] : 0.0);
        small_dft<B>(v, +1);  // inverse, first step: Z[k1][n2] = v[n2]
#pragma unroll
        for (int n2 = 0; n2 < B; ++n2) buf[(B * k1 + n2) * LP + line] = cmulc(v[n2], twn[(n2 * k1) % N]);
    }
    __syncthreads();
    for (int task = threadIdx.x; task < B * L; task += kThreads4) {
        const int line = task % L, n2 = task / L;
        cplx v[A];
#pragma unroll
        for (int k1 = 0; k1 < A; ++k1) v[k1] = buf[(B * k1 + n2) * LP + line];
        small_dft<A>(v, +1);
        if (c0 + line < inner) {
#pragma unroll
            for (int n1 = 0; n1 < A; ++n1) {
                const int x = B * n1 + n2;
                if (x < nx) col[int64_t(x) * inner + line] = v[n1];
            }
        }
    }
}

// Passes 2 and 4, four-step: middle-axis lines of [outer][n][inner]; reads n_in elements per line
// (zero beyond), transforms (sign), writes the first n_out.
template <int A, int B>
__global__ void __launch_bounds__(kThreads4) fft_middle_fourstep_kernel(const cplx* __restrict__ in,
                                                                       int64_t in_outer_stride, int n_in,
                                                                       cplx* __restrict__ out,
                                                                       int64_t out_outer_stride, int n_out,
                                                                       int64_t inner, const cplx* __restrict__ twn,
                                                                       int sign) {
    constexpr int N = A * B, L = kLines4, LP = L + 1;
    __shared__ cplx buf[N * LP];
    const int64_t o = blockIdx.x;
    const int64_t c0 = int64_t(blockIdx.y) * L;
    const cplx* src = in + o * in_outer_stride + c0;
#pragma unroll 4
    for (int idx = threadIdx.x; idx < N * L; idx += kThreads4) {
        const int line = idx % L, j = idx / L;
        buf[j * LP + line] = (j < n_in && c0 + line < inner) ? src[int64_t(j) * inner + line] : cplx{0.0, 0.0};
    }
    __syncthreads();
    fourstep_first<A, B>(buf, twn, sign);
    __syncthreads();
    cplx* dst = out + o * out_outer_stride + c0;
    for (int task = threadIdx.x; task < A * L; task += kThreads4) {
        const int line = task % L, k1 = task / L;
        cplx v[B];
#pragma unroll
        for (int n2 = 0; n2 < B; ++n2) v[n2] = buf[(B * k1 + n2) * LP + line];
        small_dft<B>(v, sign);
        if (c0 + line < inner) {
#pragma unroll
            for (int k2 = 0; k2 < B; ++k2) {
                const int k = k1 + A * k2;
                if (k < n_out) dst[int64_t(k) * inner + line] = v[k2];
            }
        }
    }
}

// The factor pair (A, B) of a length the four-step kernels take, A * B = n; false otherwise.
bool fourstep_pair(int n, int* a, int* b) {
    static const int pairs[][3] = {{64, 8, 8},     {72, 8, 9},     {80, 8, 10},   {90, 9, 10},    {96, 8, 12},
                                   {100, 10, 10},  {108, 9, 12},   {120, 10, 12}, {128, 8, 16},   {135, 9, 15},
                                   {144, 12, 12},  {150, 10, 15},  {160, 10, 16}, {162, 9, 18},   {180, 12, 15},
                                   {192, 12, 16},  {200, 10, 20},  {216, 12, 18}, {225, 15, 15},  {240, 15, 16},
                                   {256, 16, 16},  {270, 15, 18},  {288, 16, 18}, {300, 15, 20},  {320, 16, 20}};
    for (const auto& q : pairs)
        if (q[0] == n) {
            *a = q[1];
            *b = q[2];
            return true;
        }
    return false;
}

#define CDFTB_FOURSTEP_PAIRS(X)                                                                                    \
    X(8, 8) X(8, 9) X(8, 10) X(9, 10) X(8, 12) X(10, 10) X(9, 12) X(10, 12) X(8, 16) X(9, 15) X(12, 12) X(10, 15) \
        X(10, 16) X(9, 18) X(12, 15) X(12, 16) X(10, 20) X(12, 18) X(15, 15) X(15, 16) X(16, 16) X(15, 18)        \
            X(16, 18) X(15, 20) X(16, 20)

// Pass 1: z lines (contiguous, nz real values zero-padded to N) -> half spectrum kz < nk.
template <int L>
__global__ void __launch_bounds__(256) fft_z_forward_kernel(const double* __restrict__ rho, int64_t lines, int nz,
                                                            cplx* __restrict__ out, int nk, const FftPlan P) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int LP = L + 1;
    cplx* b0 = reinterpret_cast<cplx*>(smem_raw);
    cplx* b1 = b0 + P.n * LP;
    const int tid = threadIdx.y * L + threadIdx.x;
    const int nthreads = L * blockDim.y;
    const int64_t l0 = int64_t(blockIdx.x) * L;
    for (int idx = tid; idx < L * P.n; idx += nthreads) {
        const int line = idx / P.n;
        const int z = idx - line * P.n;
        const double v = (z < nz && l0 + line < lines) ? rho[(l0 + line) * nz + z] : 0.0;
        b0[z * LP + line] = {v, 0.0};
    }
    __syncthreads();
    const cplx* r = fft_lines(b0, b1, P, -1, LP, threadIdx.x, threadIdx.y, blockDim.y);
    for (int idx = tid; idx < L * nk; idx += nthreads) {
        const int line = idx / nk;
        const int k = idx - line * nk;
        if (l0 + line < lines) out[(l0 + line) * nk + k] = r[k * LP + line];
    }
}

// Passes 2 and 4: middle-axis lines of data viewed as [outer][n][inner], inner contiguous; reads
// n_in elements per line (zero beyond), transforms with length P.n, writes n_out elements.
template <int L>
__global__ void __launch_bounds__(256) fft_middle_kernel(const cplx* __restrict__ in, int64_t in_outer_stride, int n_in,
                                                         cplx* __restrict__ out, int64_t out_outer_stride, int n_out,
                                                         int64_t inner, const FftPlan P, int sign) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int LP = L + 1;
    cplx* b0 = reinterpret_cast<cplx*>(smem_raw);
    cplx* b1 = b0 + P.n * LP;
    const int64_t o = blockIdx.x;
    const int64_t c = int64_t(blockIdx.y) * L + threadIdx.x;
    const bool live = c < inner;
    const cplx* src = in + o * in_outer_stride + c;
    for (int j = threadIdx.y; j < P.n; j += blockDim.y)
        b0[j * LP + threadIdx.x] = (j < n_in && live) ? src[int64_t(j) * inner] : cplx{0.0, 0.0};
    __syncthreads();
    const cplx* r = fft_lines(b0, b1, P, sign, LP, threadIdx.x, threadIdx.y, blockDim.y);
    if (!live) return;
    cplx* dst = out + o * out_outer_stride + c;
    for (int j = threadIdx.y; j < n_out; j += blockDim.y) dst[int64_t(j) * inner] = r[j * LP + threadIdx.x];
}

// Pass 3: x lines of one system ([nx][inner], inner = N1 * nk contiguous): forward FFT of the nx
// non-zero values, times K[kx][ky][kz], inverse FFT, the first nx values written back in place.
template <int L>
__global__ void __launch_bounds__(256) fft_x_fused_kernel(cplx* __restrict__ data, int nx, int64_t inner,
                                                          const double* __restrict__ kernel, const FftPlan P) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int LP = L + 1;
    cplx* b0 = reinterpret_cast<cplx*>(smem_raw);
    cplx* b1 = b0 + P.n * LP;
    const int64_t c = int64_t(blockIdx.x) * L + threadIdx.x;
    const bool live = c < inner;
    cplx* col = data + int64_t(blockIdx.y) * nx * inner + c;
    for (int j = threadIdx.y; j < P.n; j += blockDim.y)
        b0[j * LP + threadIdx.x] = (j < nx && live) ? col[int64_t(j) * inner] : cplx{0.0, 0.0};
    __syncthreads();
    cplx* r = fft_lines(b0, b1, P, -1, LP, threadIdx.x, threadIdx.y, blockDim.y);
    for (int j = threadIdx.y; j < P.n; j += blockDim.y) {
        const double kv = live ? kernel[int64_t(j) * inner + c] : 0.0;
        r[j * LP + threadIdx.x] = scale(r[j * LP + threadIdx.x], kv);
    }
    __syncthreads();
    const cplx* v = fft_lines(r, r == b0 ? b1 : b0, P, +1, LP, threadIdx.x, threadIdx.y, blockDim.y);
    if (!live) return;
    for (int j = threadIdx.y; j < nx; j += blockDim.y) col[int64_t(j) * inner] = v[j * LP + threadIdx.x];
}

// Pass 5: half spectrum -> real z lines (z < nz), with the 1/(Nx Ny Nz) of irfftn. The full
// spectrum is the Hermitian extension X[N-k] = conj(X[k]); the real part of its inverse is irfft
// (the imaginary parts of the k = 0 and Nyquist terms drop out, as in irfft).
template <int L>
__global__ void __launch_bounds__(256) fft_z_inverse_kernel(const cplx* __restrict__ in, int64_t lines, int nk,
                                                            double* __restrict__ v, int nz, const FftPlan P,
                                                            double norm) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int LP = L + 1;
    cplx* b0 = reinterpret_cast<cplx*>(smem_raw);
    cplx* b1 = b0 + P.n * LP;
    const int tid = threadIdx.y * L + threadIdx.x;
    const int nthreads = L * blockDim.y;
    const int64_t l0 = int64_t(blockIdx.x) * L;
    const int N = P.n;
    for (int idx = tid; idx < L * nk; idx += nthreads) {
        const int line = idx / nk;
        const int k = idx - line * nk;
        const cplx a = (l0 + line < lines) ? in[(l0 + line) * nk + k] : cplx{0.0, 0.0};
        b0[k * LP + line] = a;
        if (k > 0 && N - k >= nk) b0[(N - k) * LP + line] = {a.re, -a.im};
    }
    __syncthreads();
    const cplx* r = fft_lines(b0, b1, P, +1, LP, threadIdx.x, threadIdx.y, blockDim.y);
    for (int idx = tid; idx < L * nz; idx += nthreads) {
        const int line = idx / nz;
        const int z = idx - line * nz;
        if (l0 + line < lines) v[(l0 + line) * nz + z] = r[z * LP + line].re * norm;
    }
}

// The truncated kernel K(G) = 4 pi (1 - cos(G R)) / G^2, K(0) = 2 pi R^2 (poisson.py:43-64) on the
// half-spectrum grid (Nx, Ny, Nz/2+1), laid out [kx][ky][kz].
__global__ void kernel_table_kernel(double* __restrict__ out, int n0, int n1, int n2, int nk2, double spacing,
                                    double radius) {
    const int64_t total = static_cast<int64_t>(n0) * n1 * nk2;
    for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < total;
         idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int i2 = static_cast<int>(idx % nk2);
        const int i1 = static_cast<int>((idx / nk2) % n1);
        const int i0 = static_cast<int>(idx / (static_cast<int64_t>(nk2) * n1));
        // fftfreq: i / (n d) for i < ceil(n/2), (i - n) / (n d) above; times 2 pi.
        const double two_pi = 6.283185307179586;
        const double f0 = (i0 < (n0 + 1) / 2 ? i0 : i0 - n0) / (n0 * spacing);
        const double f1 = (i1 < (n1 + 1) / 2 ? i1 : i1 - n1) / (n1 * spacing);
        const double f2 = i2 / (n2 * spacing);
        const double kx = two_pi * f0, ky = two_pi * f1, kz = two_pi * f2;
        const double g_sq = kx * kx + ky * ky + kz * kz;
        double v;
        if (g_sq > 0.0) {
            const double g = sqrt(g_sq);
            v = 4.0 * 3.141592653589793 * (1.0 - cos(g * radius)) / g_sq;
        } else {
            v = 2.0 * 3.141592653589793 * radius * radius;
        }
        out[idx] = v;
    }
}

constexpr int kPoissonSmem = 200 * 1024;
constexpr int kThreads = 256;

// Lines per CTA for transforms of length n: 8 while two [n][9] complex buffers fit, else 4. (At
// n = 180, 32 systems: 8 lines 3.0 ms per solve, 16 lines 3.8 ms -- two CTAs per SM instead of
// four -- and 4 lines 3.9 ms.)
int lines_for(int n) { return size_t(2) * n * 9 * sizeof(cplx) <= size_t(kPoissonSmem) ? 8 : 4; }

size_t smem_for(int n, int L) { return size_t(2) * n * (L + 1) * sizeof(cplx); }

template <int L>
int configure_lines() {
    int st = check(cudaFuncSetAttribute(fft_z_forward_kernel<L>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        kPoissonSmem));
    if (st == CDFTB_OK)
        st = check(cudaFuncSetAttribute(fft_middle_kernel<L>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        kPoissonSmem));
    if (st == CDFTB_OK)
        st = check(cudaFuncSetAttribute(fft_x_fused_kernel<L>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        kPoissonSmem));
    if (st == CDFTB_OK)
        st = check(cudaFuncSetAttribute(fft_z_inverse_kernel<L>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        kPoissonSmem));
    return st;
}

int configure_poisson_kernels() {
    int st = configure_lines<16>();
    if (st == CDFTB_OK) st = configure_lines<8>();
    if (st == CDFTB_OK) st = configure_lines<4>();
    return st;
}

int fft_friendly(int n) {
    for (int c = n;; ++c) {
        int r = c;
        for (int p : {2, 3, 5})
            while (r % p == 0) r /= p;
        if (r == 1) return c;
    }
}

// Stage list and twiddle table (host, double) of a length-n transform; false if n is not 2,3,5-smooth
// or has too many stages.
bool make_fft_plan(int n, FftPlan* plan, cplx** device_tw) {
    FftPlan P{};
    P.n = n;
    int rem = n;
    int radices[MAX_STAGES];
    int count = 0;
    for (int r : {4, 2, 3, 5}) {
        while (rem % r == 0 && count < MAX_STAGES) {
            radices[count++] = r;
            rem /= r;
        }
    }
    if (rem != 1) return false;
    P.nst = count;
    int total = 0;
    int stride = 1;
    for (int st = 0; st < count; ++st) {
        const int r = radices[st];
        const int len = n / stride;
        P.radix[st] = r;
        P.stride[st] = stride;
        P.m[st] = len / r;
        P.tw_off[st] = total;
        total += P.m[st] * (r - 1);
        stride *= r;
    }
    cplx* host = new cplx[total > 0 ? total : 1];
    for (int st = 0; st < count; ++st) {
        const int r = P.radix[st];
        const int len = n / P.stride[st];
        for (int p = 0; p < P.m[st]; ++p)
            for (int k = 1; k < r; ++k) {
                // exp(-2 pi i p k / len), the angle reduced exactly in integers first
                const long long num = static_cast<long long>(p) * k % len;
                const double t = -2.0 * 3.14159265358979323846 * static_cast<double>(num) / static_cast<double>(len);
                host[P.tw_off[st] + p * (r - 1) + k - 1] = {cos(t), sin(t)};
            }
    }
    cplx* dev = nullptr;
    bool ok = cudaMalloc(&dev, sizeof(cplx) * (total > 0 ? total : 1)) == cudaSuccess &&
              cudaMemcpy(dev, host, sizeof(cplx) * (total > 0 ? total : 1), cudaMemcpyHostToDevice) == cudaSuccess;
    delete[] host;
    if (!ok) {
        cudaFree(dev);
        return false;
    }
    P.tw = dev;
    *plan = P;
    *device_tw = dev;
    return true;
}

// exp(-2 pi i j / n) for j < n on the device (the angle reduced exactly in integers first).
bool make_root_table(int n, cplx** device) {
    cplx* host = new cplx[n];
    for (int j = 0; j < n; ++j) {
        const double t = -2.0 * 3.14159265358979323846 * static_cast<double>(j) / static_cast<double>(n);
        host[j] = {cos(t), sin(t)};
    }
    cplx* dev = nullptr;
    const bool ok = cudaMalloc(&dev, sizeof(cplx) * n) == cudaSuccess &&
                    cudaMemcpy(dev, host, sizeof(cplx) * n, cudaMemcpyHostToDevice) == cudaSuccess;
    delete[] host;
    if (!ok) {
        cudaFree(dev);
        return false;
    }
    *device = dev;
    return true;
}

// The small-DFT roots of unity in constant memory (this device's copy of the module).
int load_unit_roots() {
    cplx host[720];
    for (int j = 0; j < 720; ++j) {
        const double t = -2.0 * 3.14159265358979323846 * static_cast<double>(j) / 720.0;
        host[j] = {cos(t), sin(t)};
    }
    return check(cudaMemcpyToSymbol(kUnit720, host, sizeof(host)));
}

}  // namespace

}  // namespace cdftb

using namespace cdftb;

// A plan: padded shape, the kernel table, the FFT plan of each axis, and the two transform buffers.
struct cdftb_poisson_plan {
    int n[3];
    int pad[3];
    int nk;  // pad[2]/2 + 1
    double spacing;
    double radius;
    double* kernel;  // [pad0][pad1][nk]
    FftPlan fft[3];
    cplx* tw[3];
    cplx* twn[3];  // W_N^j, j < pad[d] (the four-step kernels' outer twiddles)
    int four[3][2];  // the four-step factor pair of each axis, {0, 0} if its length has none
    cplx* a;  // [batch][n0][n1][nk]
    cplx* b;  // [batch][n0][pad1][nk]
    int max_batch;
};

static void free_plan(cdftb_poisson_plan* p) {
    cudaFree(p->kernel);
    for (int d = 0; d < 3; ++d) cudaFree(p->tw[d]);
    for (int d = 0; d < 3; ++d) cudaFree(p->twn[d]);
    cudaFree(p->a);
    cudaFree(p->b);
    delete p;
}

extern "C" int cdftb_poisson_plan_create(int nx, int ny, int nz, double spacing, double pad_factor, int max_batch,
                                         void** plan_out, int* padded_shape_out, double* cutoff_radius_out) {
    if (!plan_out || nx <= 0 || ny <= 0 || nz <= 0 || !(spacing > 0.0) || pad_factor < 2.0 || max_batch < 1)
        return CDFTB_ERR_ARGUMENT;
    auto* p = new cdftb_poisson_plan{};
    p->n[0] = nx;
    p->n[1] = ny;
    p->n[2] = nz;
    for (int d = 0; d < 3; ++d) p->pad[d] = fft_friendly(static_cast<int>(ceil(pad_factor * p->n[d])));
    p->nk = p->pad[2] / 2 + 1;
    p->spacing = spacing;
    double r = 1e300;
    for (int d = 0; d < 3; ++d) r = fmin(r, p->pad[d] * spacing);
    p->radius = 0.5 * r;
    p->max_batch = max_batch;
    for (int d = 0; d < 3; ++d)
        if (smem_for(p->pad[d], lines_for(p->pad[d])) > size_t(kPoissonSmem)) {
            delete p;
            return CDFTB_ERR_CAPACITY;
        }
    const int64_t nkern = static_cast<int64_t>(p->pad[0]) * p->pad[1] * p->nk;
    int st = configure_poisson_kernels();
    if (st != CDFTB_OK) {
        delete p;
        return st;
    }
    st = check(cudaMalloc(&p->kernel, nkern * sizeof(double)));
    for (int d = 0; d < 3 && st == CDFTB_OK; ++d)
        if (!make_fft_plan(p->pad[d], &p->fft[d], &p->tw[d])) st = CDFTB_ERR_LAUNCH;
    for (int d = 0; d < 3 && st == CDFTB_OK; ++d) {
        if (!fourstep_pair(p->pad[d], &p->four[d][0], &p->four[d][1])) {
            p->four[d][0] = p->four[d][1] = 0;
            continue;
        }
        if (!make_root_table(p->pad[d], &p->twn[d])) st = CDFTB_ERR_LAUNCH;
    }
    if (st == CDFTB_OK) st = load_unit_roots();
    if (st == CDFTB_OK)
        st = check(cudaMalloc(&p->a, static_cast<int64_t>(max_batch) * nx * ny * p->nk * sizeof(cplx)));
    if (st == CDFTB_OK)
        st = check(cudaMalloc(&p->b, static_cast<int64_t>(max_batch) * nx * p->pad[1] * p->nk * sizeof(cplx)));
    if (st == CDFTB_OK) {
        kernel_table_kernel<<<static_cast<unsigned>(ceil_div(nkern, 256)), 256>>>(p->kernel, p->pad[0], p->pad[1],
                                                                                  p->pad[2], p->nk, spacing, p->radius);
        st = check_launch();
        if (st == CDFTB_OK) st = check(cudaDeviceSynchronize());
    }
    if (st != CDFTB_OK) {
        free_plan(p);
        return st;
    }
    if (padded_shape_out)
        for (int d = 0; d < 3; ++d) padded_shape_out[d] = p->pad[d];
    if (cutoff_radius_out) *cutoff_radius_out = p->radius;
    *plan_out = p;
    return CDFTB_OK;
}

extern "C" int cdftb_poisson_plan_destroy(void* plan) {
    auto* p = static_cast<cdftb_poisson_plan*>(plan);
    if (!p) return CDFTB_OK;
    free_plan(p);
    return CDFTB_OK;
}

extern "C" int cdftb_poisson_kernel_table(void* plan, const double** table_out) {
    auto* p = static_cast<cdftb_poisson_plan*>(plan);
    if (!p || !table_out) return CDFTB_ERR_ARGUMENT;
    *table_out = p->kernel;
    return CDFTB_OK;
}

namespace {

template <int L>
int run_passes(cdftb_poisson_plan* p, const double* density, double* potential, int batch, cudaStream_t s, int which) {
    const int nx = p->n[0], ny = p->n[1], nz = p->n[2];
    const int N0 = p->pad[0], N1 = p->pad[1], N2 = p->pad[2], nk = p->nk;
    const int64_t lines = static_cast<int64_t>(batch) * nx * ny;
    const dim3 blk(L, kThreads / L);
    switch (which) {
        case 1:
            fft_z_forward_kernel<L><<<static_cast<unsigned>(ceil_div(lines, L)), blk, smem_for(N2, L), s>>>(
                density, lines, nz, p->a, nk, p->fft[2]);
            break;
        case 2: {
            dim3 grid(static_cast<unsigned>(batch * nx), static_cast<unsigned>(ceil_div(nk, L)));
            fft_middle_kernel<L><<<grid, blk, smem_for(N1, L), s>>>(p->a, static_cast<int64_t>(ny) * nk, ny, p->b,
                                                                   static_cast<int64_t>(N1) * nk, N1, nk, p->fft[1], -1);
            break;
        }
        case 3: {
            const int64_t inner = static_cast<int64_t>(N1) * nk;
            dim3 grid(static_cast<unsigned>(ceil_div(inner, L)), static_cast<unsigned>(batch));
            fft_x_fused_kernel<L><<<grid, blk, smem_for(N0, L), s>>>(p->b, nx, inner, p->kernel, p->fft[0]);
            break;
        }
        case 4: {
            dim3 grid(static_cast<unsigned>(batch * nx), static_cast<unsigned>(ceil_div(nk, L)));
            fft_middle_kernel<L><<<grid, blk, smem_for(N1, L), s>>>(p->b, static_cast<int64_t>(N1) * nk, N1, p->a,
                                                                   static_cast<int64_t>(ny) * nk, ny, nk, p->fft[1], +1);
            break;
        }
        default: {
            const double norm = 1.0 / (static_cast<double>(N0) * N1 * N2);
            fft_z_inverse_kernel<L><<<static_cast<unsigned>(ceil_div(lines, L)), blk, smem_for(N2, L), s>>>(
                p->a, lines, nk, potential, nz, p->fft[2], norm);
            break;
        }
    }
    return check_launch();
}

// Passes 2-4 with the four-step kernels (the axis length has a factor pair).
int run_fourstep(cdftb_poisson_plan* p, int batch, cudaStream_t s, int pass) {
    const int nx = p->n[0], ny = p->n[1];
    const int N1 = p->pad[1], nk = p->nk;
    const int d = pass == 3 ? 0 : 1;
    const int A = p->four[d][0], B = p->four[d][1];
    const dim3 blk(kThreads4);
    if (pass == 3) {
        const int64_t inner = static_cast<int64_t>(N1) * nk;
        const dim3 grid(static_cast<unsigned>(ceil_div(inner, kLines4)), static_cast<unsigned>(batch));
#define CDFTB_X4(A_, B_)                                                                                     \
    if (A == A_ && B == B_) {                                                                                \
        fft_x_fourstep_kernel<A_, B_><<<grid, blk, 0, s>>>(p->b, nx, inner, p->kernel, p->twn[0]);           \
        return check_launch();                                                                               \
    }
        CDFTB_FOURSTEP_PAIRS(CDFTB_X4)
#undef CDFTB_X4
        return CDFTB_ERR_ARGUMENT;
    }
    const dim3 grid(static_cast<unsigned>(batch * nx), static_cast<unsigned>(ceil_div(nk, kLines4)));
    const cplx* in = pass == 2 ? p->a : p->b;
    cplx* out = pass == 2 ? p->b : p->a;
    const int64_t in_stride = pass == 2 ? static_cast<int64_t>(ny) * nk : static_cast<int64_t>(N1) * nk;
    const int64_t out_stride = pass == 2 ? static_cast<int64_t>(N1) * nk : static_cast<int64_t>(ny) * nk;
    const int n_in = pass == 2 ? ny : N1;
    const int n_out = pass == 2 ? N1 : ny;
    const int sign = pass == 2 ? -1 : +1;
#define CDFTB_M4(A_, B_)                                                                                      \
    if (A == A_ && B == B_) {                                                                                 \
        fft_middle_fourstep_kernel<A_, B_><<<grid, blk, 0, s>>>(in, in_stride, n_in, out, out_stride, n_out, nk, \
                                                                p->twn[1], sign);                             \
        return check_launch();                                                                                \
    }
    CDFTB_FOURSTEP_PAIRS(CDFTB_M4)
#undef CDFTB_M4
    return CDFTB_ERR_ARGUMENT;
}

}  // namespace

extern "C" int cdftb_poisson_solve(void* plan, const double* density, double* potential, int batch,
                                   cdftb_stream_t stream) {
    auto* p = static_cast<cdftb_poisson_plan*>(plan);
    if (!p || !density || !potential || batch < 1 || batch > p->max_batch) return CDFTB_ERR_ARGUMENT;
    if (static_cast<int64_t>(batch) * p->n[0] > 0x7fffffff) return CDFTB_ERR_CAPACITY;
    cudaStream_t s = as_stream(stream);
    const int axis_of_pass[6] = {0, 2, 1, 0, 1, 2};
    for (int pass = 1; pass <= 5; ++pass) {
        if (pass >= 2 && pass <= 4 && p->four[axis_of_pass[pass]][0] != 0) {
            const int st = run_fourstep(p, batch, s, pass);
            if (st != CDFTB_OK) return st;
            continue;
        }
        const int n = p->pad[axis_of_pass[pass]];
        const int lines = lines_for(n);
        const int st = lines == 16  ? run_passes<16>(p, density, potential, batch, s, pass)
                       : lines == 8 ? run_passes<8>(p, density, potential, batch, s, pass)
                                    : run_passes<4>(p, density, potential, batch, s, pass);
        if (st != CDFTB_OK) return st;
    }
    return CDFTB_OK;
}
