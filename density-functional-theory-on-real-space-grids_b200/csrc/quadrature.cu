// (d4) The cusp-aware quadrature's degree-7 tensor-product Lagrange interpolant L (nodes x grid)
// and its transpose ("lift"), without storing L's values: every node keeps its stencil corner and
// its three 8-point one-dimensional weight vectors, and a tap's value is (wx * wy) * wz, the
// product the reference stores in its CSR (src/cdft/operators/quadrature.py:56-93, 506-650).
//
// interpolate: one warp per node gathers its 512 taps (8 contiguous z values per row).
// lift: the transpose as a gather over grid points: a CSR of L^T holding only node indices, sorted
//       by (grid point, node) on the device (a radix sort of 64-bit keys), one warp per grid point,
//       entries in node order, fixed-order lane reduction -- deterministic, no atomics.

#include <cub/cub.cuh>

#include "common.cuh"

namespace cdftb {

namespace {

constexpr int KTAP = 8;  // degree + 1
constexpr int HALFD = 3; // degree / 2

// Lagrange basis at offset t over nodes -3..4, products in the reference's order (quadrature.py:77).
__device__ __forceinline__ void lagrange8(double t, double* w) {
    double x[KTAP];
#pragma unroll
    for (int m = 0; m < KTAP; ++m) x[m] = t - static_cast<double>(m - HALFD);
#pragma unroll
    for (int j = 0; j < KTAP; ++j) {
        double v = 1.0;
#pragma unroll
        for (int m = 0; m < KTAP; ++m) {
            if (m == j) continue;
            v = v * x[m] / static_cast<double>(j - m);
        }
        w[j] = v;
    }
}

__global__ void stencil_kernel(const double* __restrict__ points, int64_t m, int nx, int ny, int nz, double ox,
                               double oy, double oz, double h, int* __restrict__ base, double* __restrict__ w1d,
                               int* __restrict__ bad) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= m) return;
    const double o[3] = {ox, oy, oz};
    const int n[3] = {nx, ny, nz};
    for (int d = 0; d < 3; ++d) {
        const double frac = (points[i * 3 + d] - o[d]) / h;
        const double fl = floor(frac);
        const double t = frac - fl;
        const int b = static_cast<int>(fl);
        if (b - HALFD < 0 || b - HALFD + KTAP > n[d]) atomicOr(bad, 1);
        base[i * 3 + d] = b;
        double w[KTAP];
        lagrange8(t, w);
        for (int k = 0; k < KTAP; ++k) w1d[i * 24 + d * 8 + k] = w[k];
    }
}

__global__ void tap_keys_kernel(const int* __restrict__ base, int64_t m, int ny, int nz,
                                unsigned long long* __restrict__ keys, int* __restrict__ counts) {
    const int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (e >= m * 512) return;
    const int64_t node = e >> 9;
    const int t = static_cast<int>(e & 511);
    const int a = t >> 6, b = (t >> 3) & 7, c = t & 7;
    const int64_t ix = base[node * 3 + 0] - HALFD + a;
    const int64_t iy = base[node * 3 + 1] - HALFD + b;
    const int64_t iz = base[node * 3 + 2] - HALFD + c;
    const int64_t point = (ix * ny + iy) * nz + iz;
    keys[e] = (static_cast<unsigned long long>(point) << 32) | static_cast<unsigned long long>(node);
    atomicAdd(&counts[point], 1);
}

__global__ void low_bits_kernel(const unsigned long long* __restrict__ keys, int64_t count, int* __restrict__ col) {
    const int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (e < count) col[e] = static_cast<int>(keys[e] & 0xffffffffull);
}

// out[f][node] = sum_taps (wx wy wz) field[f][tap], one warp per node.
__global__ void interpolate_kernel(const int* __restrict__ base, const double* __restrict__ w1d, int64_t m, int ny,
                                   int nz, const double* __restrict__ fields, int nf, int64_t field_stride,
                                   double* __restrict__ out, int64_t out_stride) {
    // fields are processed five at a time, chunk blockIdx.y
    const int64_t warp = (blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= m) return;
    const int64_t node = warp;
    const int f0 = blockIdx.y * 5;
    nf = min(5, nf - f0);
    fields += f0 * field_stride;
    out += f0 * out_stride;
    const int bx = base[node * 3 + 0] - HALFD, by = base[node * 3 + 1] - HALFD, bz = base[node * 3 + 2] - HALFD;
    const double* w = w1d + node * 24;
    double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (int t = lane; t < 512; t += 32) {
        const int a = t >> 6, b = (t >> 3) & 7, c = t & 7;
        const double v = (w[a] * w[8 + b]) * w[16 + c];
        const int64_t idx = (static_cast<int64_t>(bx + a) * ny + (by + b)) * nz + (bz + c);
        for (int f = 0; f < nf; ++f) acc[f] += v * fields[f * field_stride + idx];
    }
    for (int f = 0; f < nf; ++f) {
        double s = acc[f];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
        if (lane == 0) out[f * out_stride + node] = s;
    }
}

// out[f][j] = sum_{entries e of row j} x[f][node_e] * (wx wy wz)(node_e, j), one warp per grid point.
__global__ void lift_kernel(const int* __restrict__ base, const double* __restrict__ w1d,
                            const long long* __restrict__ row_ptr, const int* __restrict__ col, int64_t n_points, int ny,
                            int nz, const double* __restrict__ x, int nf, int64_t x_stride, double* __restrict__ out,
                            int64_t out_stride) {
    const int64_t row = (blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= n_points) return;
    const int f0 = blockIdx.y * 5;
    nf = min(5, nf - f0);
    x += f0 * x_stride;
    out += f0 * out_stride;
    const long long e0 = row_ptr[row], e1 = row_ptr[row + 1];
    double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (e1 > e0) {
        const int jx = static_cast<int>(row / (static_cast<int64_t>(ny) * nz));
        const int jy = static_cast<int>((row / nz) % ny);
        const int jz = static_cast<int>(row % nz);
        for (long long e = e0 + lane; e < e1; e += 32) {
            const int node = col[e];
            const int a = jx - (base[node * 3 + 0] - HALFD);
            const int b = jy - (base[node * 3 + 1] - HALFD);
            const int c = jz - (base[node * 3 + 2] - HALFD);
            const double* w = w1d + static_cast<int64_t>(node) * 24;
            const double v = (w[a] * w[8 + b]) * w[16 + c];
            for (int f = 0; f < nf; ++f) acc[f] += x[f * x_stride + node] * v;
        }
    }
    for (int f = 0; f < nf; ++f) {
        double s = acc[f];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
        if (lane == 0) out[f * out_stride + row] = s;
    }
}

struct LiftScratch {
    size_t keys_a, keys_b, counts, sort_temp, scan_temp, total;
};

LiftScratch lift_scratch_layout(int64_t m, int64_t n_points) {
    LiftScratch s{};
    const int64_t e = m * 512;
    auto align = [](size_t v) { return (v + 255) & ~static_cast<size_t>(255); };
    size_t sort_bytes = 0, scan_bytes = 0;
    cub::DeviceRadixSort::SortKeys(nullptr, sort_bytes, static_cast<unsigned long long*>(nullptr),
                                   static_cast<unsigned long long*>(nullptr), static_cast<int>(e));
    cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, static_cast<long long*>(nullptr),
                                  static_cast<long long*>(nullptr), static_cast<int>(n_points + 1));
    s.keys_a = 0;
    s.keys_b = align(s.keys_a + e * 8);
    s.counts = align(s.keys_b + e * 8);
    s.sort_temp = align(s.counts + (n_points + 1) * 8);
    s.scan_temp = align(s.sort_temp + sort_bytes);
    s.total = align(s.scan_temp + scan_bytes);
    return s;
}

__global__ void widen_counts_kernel(const int* __restrict__ counts32, long long* __restrict__ counts64, int64_t n) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i <= n) counts64[i] = (i < n) ? counts32[i] : 0;
}

inline unsigned blocks_for(int64_t n, int threads) { return static_cast<unsigned>(ceil_div(n, threads)); }

}  // namespace

}  // namespace cdftb

using namespace cdftb;

extern "C" int cdftb_quadrature_stencils(const double* points, int64_t m, int nx, int ny, int nz, double ox, double oy,
                                         double oz, double spacing, int* base, double* w1d, int* bad_flag,
                                         cdftb_stream_t stream) {
    if (m < 0 || !(spacing > 0.0) || (m > 0 && (!points || !base || !w1d || !bad_flag))) return CDFTB_ERR_ARGUMENT;
    if (m == 0) return CDFTB_OK;
    cudaStream_t s = as_stream(stream);
    stencil_kernel<<<blocks_for(m, 128), 128, 0, s>>>(points, m, nx, ny, nz, ox, oy, oz, spacing, base, w1d, bad_flag);
    return check_launch();
}

extern "C" int64_t cdftb_lift_plan_scratch_bytes(int64_t m, int64_t n_points) {
    if (m <= 0 || n_points <= 0 || m * 512 >= (1ll << 31)) return 0;
    return static_cast<int64_t>(lift_scratch_layout(m, n_points).total);
}

extern "C" int cdftb_lift_plan_build(const int* base, int64_t m, int nx, int ny, int nz, long long* row_ptr, int* col,
                                     void* scratch, int64_t scratch_bytes, cdftb_stream_t stream) {
    const int64_t n_points = static_cast<int64_t>(nx) * ny * nz;
    if (!base || !row_ptr || !col || m <= 0 || n_points <= 0 || n_points >= (1ll << 32)) return CDFTB_ERR_ARGUMENT;
    if (m * 512 >= (1ll << 31)) return CDFTB_ERR_CAPACITY;
    LiftScratch lay = lift_scratch_layout(m, n_points);
    if (!scratch || scratch_bytes < static_cast<int64_t>(lay.total)) return CDFTB_ERR_ARGUMENT;
    cudaStream_t s = as_stream(stream);
    char* sc = static_cast<char*>(scratch);
    auto* keys_a = reinterpret_cast<unsigned long long*>(sc + lay.keys_a);
    auto* keys_b = reinterpret_cast<unsigned long long*>(sc + lay.keys_b);
    auto* counts32 = reinterpret_cast<int*>(sc + lay.counts);
    const int64_t e = m * 512;
    int st = check(cudaMemsetAsync(counts32, 0, (n_points + 1) * sizeof(int), s));
    if (st != CDFTB_OK) return st;
    tap_keys_kernel<<<blocks_for(e, 256), 256, 0, s>>>(base, m, ny, nz, keys_a, counts32);
    if ((st = check_launch()) != CDFTB_OK) return st;
    int end_bit = 32;
    while (end_bit < 64 && (1ll << (end_bit - 32)) < n_points) ++end_bit;
    size_t sort_bytes = lay.scan_temp - lay.sort_temp;
    if ((st = check(cub::DeviceRadixSort::SortKeys(sc + lay.sort_temp, sort_bytes, keys_a, keys_b, static_cast<int>(e), 0,
                                                   end_bit, s))) != CDFTB_OK)
        return st;
    low_bits_kernel<<<blocks_for(e, 256), 256, 0, s>>>(keys_b, e, col);
    if ((st = check_launch()) != CDFTB_OK) return st;
    // counts -> row_ptr (int64) by an exclusive scan over n_points + 1 entries; keys_a is free now
    auto* counts64 = reinterpret_cast<long long*>(keys_a);
    widen_counts_kernel<<<blocks_for(n_points + 1, 256), 256, 0, s>>>(counts32, counts64, n_points);
    if ((st = check_launch()) != CDFTB_OK) return st;
    size_t scan_bytes = lay.total - lay.scan_temp;
    return check(cub::DeviceScan::ExclusiveSum(sc + lay.scan_temp, scan_bytes, counts64, row_ptr,
                                               static_cast<int>(n_points + 1), s));
}

extern "C" int cdftb_quadrature_interpolate_f64(const int* base, const double* w1d, int64_t m, int nx, int ny, int nz,
                                                const double* fields, int nf, int64_t field_stride, double* out,
                                                int64_t out_stride, cdftb_stream_t stream) {
    (void)nx;
    if (m < 0 || nf < 1 || nf > 5 * 65535 || (m > 0 && (!base || !w1d || !fields || !out))) return CDFTB_ERR_ARGUMENT;
    if (m == 0) return CDFTB_OK;
    dim3 grid(blocks_for(m * 32, 256), static_cast<unsigned>(ceil_div(nf, 5)));
    interpolate_kernel<<<grid, 256, 0, as_stream(stream)>>>(base, w1d, m, ny, nz, fields, nf, field_stride, out,
                                                            out_stride);
    return check_launch();
}

extern "C" int cdftb_quadrature_lift_f64(const int* base, const double* w1d, const long long* row_ptr, const int* col,
                                         int nx, int ny, int nz, const double* node_values, int nf, int64_t x_stride,
                                         double* out, int64_t out_stride, cdftb_stream_t stream) {
    const int64_t n_points = static_cast<int64_t>(nx) * ny * nz;
    if (nf < 1 || nf > 5 * 65535 || !base || !w1d || !row_ptr || !col || !node_values || !out || n_points <= 0)
        return CDFTB_ERR_ARGUMENT;
    dim3 grid(blocks_for(n_points * 32, 256), static_cast<unsigned>(ceil_div(nf, 5)));
    lift_kernel<<<grid, 256, 0, as_stream(stream)>>>(base, w1d, row_ptr, col, n_points, ny, nz, node_values, nf, x_stride,
                                                     out, out_stride);
    return check_launch();
}
