// (c) The Coulomb-cutoff Poisson solve (src/cdft/operators/poisson.py:21-107) as five pruned
// axis-wise transforms on the device, with the truncated kernel K(G) fused into the x pass.
//
// The density occupies the first n of the N = fft_friendly(ceil(2.5 n)) points of every padded
// axis and only the first n outputs are read back, so each pass transforms exactly the non-zero
// lines and computes only the needed outputs:
//   pass 1  z, real -> half complex      rho[x][y][z]        -> A[x][y][kz]    (x < nx, y < ny)
//   pass 2  y, forward                   A[x][y][kz]         -> B[x][ky][kz]   (x < nx)
//   pass 3  x, forward, * K, inverse     B[x][ky][kz]        -> B[x][ky][kz]   (in place, x < nx)
//   pass 4  y, inverse                   B[x][ky][kz]        -> A[x][y][kz]    (y < ny)
//   pass 5  z, half complex -> real      A[x][y][kz]         -> v[x][y][z]     (z < nz), / (Nx Ny Nz)
// Each pass stages the lines it transforms in shared memory and sums against a table of the N-th
// roots of unity (a direct pruned DFT per line). The result is what rfftn / *K / irfftn of the
// zero-padded box gives, up to round-off (pocketfft / cuFFT re-associate differently).

#include <math.h>

#include "common.cuh"

namespace cdftb {

namespace {

struct cplx {
    double re, im;
};

__device__ __forceinline__ cplx cmul(cplx a, cplx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }

constexpr int LANES = 32;

// Middle-axis transform: data viewed as [outer][n][inner]; for every (outer, inner) line computes
// out[outer][k][inner] = sum_{j < n_in} in[outer][j][inner] * root^(sign * j * k), k < n_out.
// One CTA per (outer, 32 consecutive inner); the line segment lives in shared memory.
__global__ void dft_middle_kernel(const cplx* __restrict__ in, int64_t in_outer_stride, int n_in, cplx* __restrict__ out,
                                  int64_t out_outer_stride, int n_out, int64_t inner, const cplx* __restrict__ roots,
                                  int n_fft, int sign) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx* s_in = reinterpret_cast<cplx*>(smem_raw);  // [n_in][LANES]
    cplx* s_root = s_in + static_cast<int64_t>(n_in) * LANES;
    const int64_t o = blockIdx.y;
    const int64_t i0 = static_cast<int64_t>(blockIdx.x) * LANES;
    const int tx = threadIdx.x;
    const int ty = threadIdx.y;
    const int tid = ty * LANES + tx;
    const int nthreads = LANES * blockDim.y;
    for (int r = tid; r < n_fft; r += nthreads) s_root[r] = roots[r];
    const cplx* src = in + o * in_outer_stride;
    for (int idx = tid; idx < n_in * LANES; idx += nthreads) {
        const int j = idx / LANES;
        const int l = idx - j * LANES;
        const int64_t ii = i0 + l;
        s_in[idx] = (ii < inner) ? src[static_cast<int64_t>(j) * inner + ii] : cplx{0.0, 0.0};
    }
    __syncthreads();
    const int64_t ii = i0 + tx;
    if (ii >= inner) return;
    cplx* dst = out + o * out_outer_stride;
    for (int k = ty; k < n_out; k += blockDim.y) {
        double re = 0.0, im = 0.0;
        int idx = 0;  // (j * k) mod n_fft, advanced incrementally
        for (int j = 0; j < n_in; ++j) {
            cplx w = s_root[idx];
            if (sign < 0) w.im = -w.im;
            const cplx x = s_in[j * LANES + tx];
            re += x.re * w.re - x.im * w.im;
            im += x.re * w.im + x.im * w.re;
            idx += k;
            if (idx >= n_fft) idx -= n_fft;
        }
        dst[static_cast<int64_t>(k) * inner + ii] = {re, im};
    }
}

// Pass 3: along x for 32 (ky, kz) lines per CTA: forward (nx -> Nx), times K, inverse (Nx -> nx),
// written back in place.
__global__ void dft_x_kernel_fused(cplx* __restrict__ data, int nx, int64_t inner, const double* __restrict__ kernel,
                                   const cplx* __restrict__ roots, int n_fft) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx* s_in = reinterpret_cast<cplx*>(smem_raw);        // [nx][LANES]
    cplx* s_mid = s_in + static_cast<int64_t>(nx) * LANES;  // [n_fft][LANES]
    cplx* s_root = s_mid + static_cast<int64_t>(n_fft) * LANES;
    const int64_t b = blockIdx.y;
    const int64_t i0 = static_cast<int64_t>(blockIdx.x) * LANES;
    const int tx = threadIdx.x;
    const int ty = threadIdx.y;
    const int tid = ty * LANES + tx;
    const int nthreads = LANES * blockDim.y;
    cplx* col = data + b * static_cast<int64_t>(nx) * inner;
    for (int r = tid; r < n_fft; r += nthreads) s_root[r] = roots[r];
    for (int idx = tid; idx < nx * LANES; idx += nthreads) {
        const int j = idx / LANES;
        const int l = idx - j * LANES;
        const int64_t ii = i0 + l;
        s_in[idx] = (ii < inner) ? col[static_cast<int64_t>(j) * inner + ii] : cplx{0.0, 0.0};
    }
    __syncthreads();
    const int64_t ii = i0 + tx;
    const bool live = ii < inner;
    for (int k = ty; k < n_fft; k += blockDim.y) {
        double re = 0.0, im = 0.0;
        int idx = 0;
        for (int j = 0; j < nx; ++j) {
            cplx w = s_root[idx];
            w.im = -w.im;
            const cplx x = s_in[j * LANES + tx];
            re += x.re * w.re - x.im * w.im;
            im += x.re * w.im + x.im * w.re;
            idx += k;
            if (idx >= n_fft) idx -= n_fft;
        }
        const double kv = live ? kernel[static_cast<int64_t>(k) * inner + ii] : 0.0;
        s_mid[k * LANES + tx] = {re * kv, im * kv};
    }
    __syncthreads();
    if (!live) return;
    for (int x = ty; x < nx; x += blockDim.y) {
        double re = 0.0, im = 0.0;
        int idx = 0;
        for (int k = 0; k < n_fft; ++k) {
            const cplx w = s_root[idx];
            const cplx v = s_mid[k * LANES + tx];
            re += v.re * w.re - v.im * w.im;
            im += v.re * w.im + v.im * w.re;
            idx += x;
            if (idx >= n_fft) idx -= n_fft;
        }
        col[static_cast<int64_t>(x) * inner + ii] = {re, im};
    }
}

// Pass 1: z lines (contiguous, length nz, zero-padded to N) -> half spectrum kz <= N/2.
// One CTA per LANES consecutive (x, y) lines; lines staged transposed [z][line].
__global__ void dft_z_r2c_kernel(const double* __restrict__ rho, int64_t lines, int nz, cplx* __restrict__ out, int nk,
                                 const cplx* __restrict__ roots, int n_fft) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* s_line = reinterpret_cast<double*>(smem_raw);  // [nz][LANES]
    cplx* s_root = reinterpret_cast<cplx*>(s_line + static_cast<int64_t>(nz) * LANES);
    const int64_t l0 = static_cast<int64_t>(blockIdx.x) * LANES;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int tid = ty * LANES + tx;
    const int nthreads = LANES * blockDim.y;
    for (int r = tid; r < n_fft; r += nthreads) s_root[r] = roots[r];
    for (int idx = tid; idx < nz * LANES; idx += nthreads) {
        const int l = idx / nz;
        const int z = idx - l * nz;
        const int64_t line = l0 + l;
        s_line[z * LANES + l] = (line < lines) ? rho[line * nz + z] : 0.0;
    }
    __syncthreads();
    const int64_t line = l0 + tx;
    if (line >= lines) return;
    for (int k = ty; k < nk; k += blockDim.y) {
        double re = 0.0, im = 0.0;
        int idx = 0;
        for (int z = 0; z < nz; ++z) {
            const cplx w = s_root[idx];
            const double x = s_line[z * LANES + tx];
            re += x * w.re;
            im -= x * w.im;
            idx += k;
            if (idx >= n_fft) idx -= n_fft;
        }
        out[line * nk + k] = {re, im};
    }
}

// Pass 5: half spectrum -> real z lines, z < nz, with the 1/(Nx Ny Nz) normalisation of irfftn.
// out[z] = A0.re + (-1)^z A_{N/2}.re + 2 sum_{0<k<N/2} Re(A_k w^{kz}) for even N.
__global__ void dft_z_c2r_kernel(const cplx* __restrict__ in, int64_t lines, int nk, double* __restrict__ v, int nz,
                                 const cplx* __restrict__ roots, int n_fft, double scale) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx* s_line = reinterpret_cast<cplx*>(smem_raw);  // [nk][LANES]
    cplx* s_root = s_line + static_cast<int64_t>(nk) * LANES;
    const int64_t l0 = static_cast<int64_t>(blockIdx.x) * LANES;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int tid = ty * LANES + tx;
    const int nthreads = LANES * blockDim.y;
    for (int r = tid; r < n_fft; r += nthreads) s_root[r] = roots[r];
    for (int idx = tid; idx < nk * LANES; idx += nthreads) {
        const int l = idx / nk;
        const int k = idx - l * nk;
        const int64_t line = l0 + l;
        s_line[k * LANES + l] = (line < lines) ? in[line * nk + k] : cplx{0.0, 0.0};
    }
    __syncthreads();
    const int64_t line = l0 + tx;
    if (line >= lines) return;
    const bool even = (n_fft % 2) == 0;
    const int k_last = even ? n_fft / 2 : -1;  // the Nyquist term (real part only)
    for (int z = ty; z < nz; z += blockDim.y) {
        double acc = s_line[tx].re;  // k = 0, real part only
        int idx = z;                 // (k * z) mod n_fft for k = 1
        if (idx >= n_fft) idx -= n_fft;
        double sum = 0.0;
        for (int k = 1; k < nk; ++k) {
            const cplx a = s_line[k * LANES + tx];
            const cplx w = s_root[idx];
            if (k == k_last)
                acc += a.re * w.re;  // (-1)^z, imaginary part ignored
            else
                sum += a.re * w.re - a.im * w.im;
            idx += z;
            if (idx >= n_fft) idx -= n_fft;
        }
        v[line * nz + z] = (acc + 2.0 * sum) * scale;
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

int configure_poisson_kernels() {
    int st = check(cudaFuncSetAttribute(dft_x_kernel_fused, cudaFuncAttributeMaxDynamicSharedMemorySize, kPoissonSmem));
    if (st == CDFTB_OK)
        st = check(cudaFuncSetAttribute(dft_middle_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kPoissonSmem));
    if (st == CDFTB_OK)
        st = check(cudaFuncSetAttribute(dft_z_r2c_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kPoissonSmem));
    if (st == CDFTB_OK)
        st = check(cudaFuncSetAttribute(dft_z_c2r_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kPoissonSmem));
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

}  // namespace

}  // namespace cdftb

using namespace cdftb;

// A plan: padded shape, the kernel table, roots of unity per axis, and the two transform buffers.
struct cdftb_poisson_plan {
    int n[3];
    int pad[3];
    int nk;  // pad[2]/2 + 1
    double spacing;
    double radius;
    double* kernel;  // [pad0][pad1][nk]
    cplx* roots[3];  // N-th roots of unity per axis
    cplx* a;         // [batch][n0][n1][nk]
    cplx* b;         // [batch][n0][pad1][nk]
    int max_batch;
};

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
    const int64_t nkern = static_cast<int64_t>(p->pad[0]) * p->pad[1] * p->nk;
    int st = configure_poisson_kernels();
    if (st != CDFTB_OK) {
        delete p;
        return st;
    }
    st = check(cudaMalloc(&p->kernel, nkern * sizeof(double)));
    for (int d = 0; d < 3 && st == CDFTB_OK; ++d) {
        const int N = p->pad[d];
        cplx* host = new cplx[N];
        for (int j = 0; j < N; ++j) {
            // exp(+2 pi i j / N); the sign is applied per pass
            const double t = 2.0 * 3.14159265358979323846 * static_cast<double>(j) / static_cast<double>(N);
            host[j] = {cos(t), sin(t)};
        }
        st = check(cudaMalloc(&p->roots[d], N * sizeof(cplx)));
        if (st == CDFTB_OK) st = check(cudaMemcpy(p->roots[d], host, N * sizeof(cplx), cudaMemcpyHostToDevice));
        delete[] host;
    }
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
        cudaFree(p->kernel);
        for (int d = 0; d < 3; ++d) cudaFree(p->roots[d]);
        cudaFree(p->a);
        cudaFree(p->b);
        delete p;
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
    cudaFree(p->kernel);
    for (int d = 0; d < 3; ++d) cudaFree(p->roots[d]);
    cudaFree(p->a);
    cudaFree(p->b);
    delete p;
    return CDFTB_OK;
}

extern "C" int cdftb_poisson_kernel_table(void* plan, const double** table_out) {
    auto* p = static_cast<cdftb_poisson_plan*>(plan);
    if (!p || !table_out) return CDFTB_ERR_ARGUMENT;
    *table_out = p->kernel;
    return CDFTB_OK;
}

extern "C" int cdftb_poisson_solve(void* plan, const double* density, double* potential, int batch,
                                   cdftb_stream_t stream) {
    auto* p = static_cast<cdftb_poisson_plan*>(plan);
    if (!p || !density || !potential || batch < 1 || batch > p->max_batch) return CDFTB_ERR_ARGUMENT;
    cudaStream_t s = as_stream(stream);
    const int nx = p->n[0], ny = p->n[1], nz = p->n[2];
    const int N0 = p->pad[0], N1 = p->pad[1], N2 = p->pad[2], nk = p->nk;
    const int64_t lines = static_cast<int64_t>(batch) * nx * ny;
    const dim3 blk(LANES, 8);
    // pass 1
    {
        const size_t sm = static_cast<size_t>(nz) * LANES * sizeof(double) + N2 * sizeof(cplx);
        dft_z_r2c_kernel<<<static_cast<unsigned>(ceil_div(lines, LANES)), blk, sm, s>>>(density, lines, nz, p->a, nk,
                                                                                        p->roots[2], N2);
        int st = check_launch();
        if (st != CDFTB_OK) return st;
    }
    // pass 2: [b*nx][ny][nk] -> [b*nx][N1][nk]
    {
        const size_t sm = static_cast<size_t>(ny) * LANES * sizeof(cplx) + N1 * sizeof(cplx);
        dim3 grid(static_cast<unsigned>(ceil_div(nk, LANES)), static_cast<unsigned>(batch * nx));
        dft_middle_kernel<<<grid, blk, sm, s>>>(p->a, static_cast<int64_t>(ny) * nk, ny, p->b,
                                                static_cast<int64_t>(N1) * nk, N1, nk, p->roots[1], N1, -1);
        int st = check_launch();
        if (st != CDFTB_OK) return st;
    }
    // pass 3: per batch, [nx][N1*nk] columns
    {
        const size_t sm = (static_cast<size_t>(nx) * LANES + static_cast<size_t>(N0) * LANES + N0) * sizeof(cplx);
        if (sm > kPoissonSmem) return CDFTB_ERR_CAPACITY;
        const int64_t inner = static_cast<int64_t>(N1) * nk;
        dim3 grid(static_cast<unsigned>(ceil_div(inner, LANES)), static_cast<unsigned>(batch));
        dft_x_kernel_fused<<<grid, blk, sm, s>>>(p->b, nx, inner, p->kernel, p->roots[0], N0);
        int st = check_launch();
        if (st != CDFTB_OK) return st;
    }
    // pass 4: [b*nx][N1][nk] -> [b*nx][ny][nk]
    {
        const size_t sm = static_cast<size_t>(N1) * LANES * sizeof(cplx) + N1 * sizeof(cplx);
        dim3 grid(static_cast<unsigned>(ceil_div(nk, LANES)), static_cast<unsigned>(batch * nx));
        dft_middle_kernel<<<grid, blk, sm, s>>>(p->b, static_cast<int64_t>(N1) * nk, N1, p->a,
                                                static_cast<int64_t>(ny) * nk, ny, nk, p->roots[1], N1, +1);
        int st = check_launch();
        if (st != CDFTB_OK) return st;
    }
    // pass 5
    {
        const size_t sm = static_cast<size_t>(nk) * LANES * sizeof(cplx) + N2 * sizeof(cplx);
        const double scale = 1.0 / (static_cast<double>(N0) * N1 * N2);
        dft_z_c2r_kernel<<<static_cast<unsigned>(ceil_div(lines, LANES)), blk, sm, s>>>(p->a, lines, nk, potential, nz,
                                                                                        p->roots[2], N2, scale);
        int st = check_launch();
        if (st != CDFTB_OK) return st;
    }
    return CDFTB_OK;
}
