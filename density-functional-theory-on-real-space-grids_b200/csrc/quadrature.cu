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
                            const long long* __restrict__ row_ptr, const int* __restrict__ col,
                            const double* __restrict__ values, int64_t n_points, int ny, int nz,
                            const double* __restrict__ x, int nf, int64_t x_stride, double* __restrict__ out,
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
            double v;
            if (values) {
                v = values[e];
            } else {
                const int a = jx - (base[node * 3 + 0] - HALFD);
                const int b = jy - (base[node * 3 + 1] - HALFD);
                const int c = jz - (base[node * 3 + 2] - HALFD);
                const double* w = w1d + static_cast<int64_t>(node) * 24;
                v = (w[a] * w[8 + b]) * w[16 + c];
            }
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
    // Only the grid point (the high word) is sorted on. The keys enter in entry order, so their low
    // words (the nodes) already rise, and the radix sort is stable: the order is the full keys'
    // (point, node) order in 3 digit passes instead of 7 at ~2^18 points.
    const int begin_bit = end_bit > 32 ? 32 : 0;
    size_t sort_bytes = lay.scan_temp - lay.sort_temp;
    if ((st = check(cub::DeviceRadixSort::SortKeys(sc + lay.sort_temp, sort_bytes, keys_a, keys_b, static_cast<int>(e),
                                                   begin_bit, end_bit, s))) != CDFTB_OK)
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
                                         const double* values, int nx, int ny, int nz, const double* node_values,
                                         int nf, int64_t x_stride, double* out, int64_t out_stride,
                                         cdftb_stream_t stream) {
    const int64_t n_points = static_cast<int64_t>(nx) * ny * nz;
    if (nf < 1 || nf > 5 * 65535 || !base || !w1d || !row_ptr || !col || !node_values || !out || n_points <= 0)
        return CDFTB_ERR_ARGUMENT;
    dim3 grid(blocks_for(n_points * 32, 256), static_cast<unsigned>(ceil_div(nf, 5)));
    lift_kernel<<<grid, 256, 0, as_stream(stream)>>>(base, w1d, row_ptr, col, values, n_points, ny, nz, node_values, nf,
                                                     x_stride, out, out_stride);
    return check_launch();
}

// ---------------------------------------------------------------------------------------------
// Many fields at once (the batched systems): L and L^T for up to 32 fields per pass with one lane
// per field. The fields are first copied into point-major rows of 32 (scratch), so that the value of
// every field at one grid point (or node) is one coalesced 256-byte row; a warp then walks one node's
// 512 stencil points (interpolate) or one grid point's CSR row (lift) once for all fields, instead
// of once per 5 fields. Results pass through a shared tile so that the field-major stores coalesce.

namespace cdftb {
namespace {

constexpr int MANY = 32;
constexpr int kLiftSegment = 256;  // CSR entries per warp task of the many-field lift

// src[f * stride + i] (f < nf, i < n) -> dst[i * 32 + f], zero for f >= nf.
__global__ void fields_to_rows_kernel(const double* __restrict__ src, int nf, int64_t stride, int64_t n,
                                      double* __restrict__ dst) {
    __shared__ double tile[MANY][MANY + 1];
    const int64_t i0 = int64_t(blockIdx.x) * MANY;
    for (int f = threadIdx.y; f < MANY; f += blockDim.y) {
        const int64_t i = i0 + threadIdx.x;
        tile[f][threadIdx.x] = (f < nf && i < n) ? src[f * stride + i] : 0.0;
    }
    __syncthreads();
    for (int r = threadIdx.y; r < MANY; r += blockDim.y) {
        const int64_t i = i0 + r;
        if (i < n) dst[i * MANY + threadIdx.x] = tile[threadIdx.x][r];
    }
}

// A CTA of 8 warps handles 32 consecutive outputs (nodes or grid points), 4 per warp; tile[j][f].
__device__ __forceinline__ void store_tile(double (*tile)[MANY + 1], int64_t j0, int64_t count, int nf,
                                           double* __restrict__ out, int64_t out_stride) {
    __syncthreads();
    const int lane = threadIdx.x & 31;
    for (int f = threadIdx.x >> 5; f < nf; f += blockDim.x >> 5)
        if (j0 + lane < count) out[f * out_stride + j0 + lane] = tile[lane][f];
}

__global__ void __launch_bounds__(256) interpolate_many_kernel(const int* __restrict__ base,
                                                               const double* __restrict__ w1d, int64_t m, int ny,
                                                               int nz, const double* __restrict__ rows, int nf,
                                                               double* __restrict__ out, int64_t out_stride) {
    __shared__ double tile[MANY][MANY + 1];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int64_t j0 = int64_t(blockIdx.x) * MANY;
    for (int r = warp; r < MANY; r += 8) {
        const int64_t node = j0 + r;
        if (node >= m) break;
        const int bx = base[node * 3 + 0] - HALFD, by = base[node * 3 + 1] - HALFD, bz = base[node * 3 + 2] - HALFD;
        const double* w = w1d + node * 24;
        const double wl = w[lane < 24 ? lane : 0];  // the 24 1-D weights, one per lane, then shuffled
        double wz[KTAP], wy[KTAP];
#pragma unroll
        for (int c = 0; c < KTAP; ++c) {
            wy[c] = __shfl_sync(0xffffffffu, wl, 8 + c);
            wz[c] = __shfl_sync(0xffffffffu, wl, 16 + c);
        }
        // separable contraction: z sums of the 8 rows of each (a, b) are independent chains, then y, then x
        double acc = 0.0;
        for (int a = 0; a < KTAP; ++a) {
            const double* plane = rows + (int64_t(bx + a) * ny + by) * int64_t(nz) * MANY + int64_t(bz) * MANY + lane;
            double sa = 0.0;
#pragma unroll
            for (int b = 0; b < KTAP; ++b) {
                const double* row = plane + int64_t(b) * nz * MANY;
                double t = 0.0;
#pragma unroll
                for (int c = 0; c < KTAP; ++c) t = fma(wz[c], row[c * MANY], t);
                sa = fma(wy[b], t, sa);
            }
            acc = fma(__shfl_sync(0xffffffffu, wl, a), sa, acc);
        }
        tile[r][lane] = acc;
    }
    store_tile(tile, j0, m, nf, out, out_stride);
}

// The interpolant for nodes grouped by their base cell: the nodes of a group read the same 8 x 8 x 8
// box, so one warp reads each box row once for up to GROUP_BATCH nodes (a cell near a nucleus holds
// ~6 nodes at He 65^3) instead of once per node. Each node's sums run in the same order as in
// interpolate_many_kernel (z, then y, then x, each a chain of fmas from zero), so the results are the
// same bit for bit. One warp per group, lanes over the fields of the row layout.
constexpr int GROUP_BATCH = 4;

__global__ void __launch_bounds__(256, 2) interpolate_grouped_kernel(const int* __restrict__ base,
                                                                  const double* __restrict__ w1d,
                                                                  const int* __restrict__ group_nodes,
                                                                  const int* __restrict__ group_ptr, int64_t groups,
                                                                  int ny, int nz, const double* __restrict__ rows,
                                                                  int nf, double* __restrict__ out,
                                                                  int64_t out_stride) {
    const int lane = threadIdx.x & 31;
    const int64_t g = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    if (g >= groups) return;
    const int first = group_ptr[g], last = group_ptr[g + 1];
    const int lead = group_nodes[first];
    const int bx = base[lead * 3 + 0] - HALFD, by = base[lead * 3 + 1] - HALFD, bz = base[lead * 3 + 2] - HALFD;
    for (int b0 = first; b0 < last; b0 += GROUP_BATCH) {
        const int count = last - b0 < GROUP_BATCH ? last - b0 : GROUP_BATCH;
        int node[GROUP_BATCH];
        double wz[GROUP_BATCH][KTAP], acc[GROUP_BATCH];
#pragma unroll
        for (int j = 0; j < GROUP_BATCH; ++j) {
            node[j] = group_nodes[b0 + (j < count ? j : 0)];  // a short batch repeats its first node
            const double* w = w1d + int64_t(node[j]) * 24;
#pragma unroll
            for (int c = 0; c < KTAP; ++c) wz[j][c] = __ldg(w + 16 + c);
            acc[j] = 0.0;
        }
        for (int a = 0; a < KTAP; ++a) {
            const double* plane = rows + (int64_t(bx + a) * ny + by) * int64_t(nz) * MANY + int64_t(bz) * MANY + lane;
            double sa[GROUP_BATCH];
#pragma unroll
            for (int j = 0; j < GROUP_BATCH; ++j) sa[j] = 0.0;
#pragma unroll 1
            for (int b = 0; b < KTAP; ++b) {
                const double* row = plane + int64_t(b) * nz * MANY;
                double v[KTAP];
#pragma unroll
                for (int c = 0; c < KTAP; ++c) v[c] = row[c * MANY];
#pragma unroll
                for (int j = 0; j < GROUP_BATCH; ++j) {
                    double t = 0.0;
#pragma unroll
                    for (int c = 0; c < KTAP; ++c) t = fma(wz[j][c], v[c], t);
                    sa[j] = fma(__ldg(w1d + int64_t(node[j]) * 24 + 8 + b), t, sa[j]);
                }
            }
#pragma unroll
            for (int j = 0; j < GROUP_BATCH; ++j) acc[j] = fma(__ldg(w1d + int64_t(node[j]) * 24 + a), sa[j], acc[j]);
        }
        if (lane < nf) {
#pragma unroll
            for (int j = 0; j < GROUP_BATCH; ++j)
                if (j < count) out[lane * out_stride + node[j]] = acc[j];
        }
    }
}

int fields_to_rows(const double* src, int nf, int64_t stride, int64_t n, double* dst, cudaStream_t s) {
    fields_to_rows_kernel<<<static_cast<unsigned>(ceil_div(n, MANY)), dim3(MANY, 8), 0, s>>>(src, nf, stride, n, dst);
    return check_launch();
}

}  // namespace
}  // namespace cdftb

extern "C" int64_t cdftb_lift_segments_capacity(int64_t m, int64_t n_points) {
    if (m < 0 || n_points < 0) return 0;
    return m * 512 / cdftb::kLiftSegment + n_points + 1;
}

extern "C" int64_t cdftb_quadrature_many_scratch_bytes(int64_t m, int64_t n_points) {
    if (m < 0 || n_points < 0) return 0;
    const int64_t lift = m + cdftb_lift_segments_capacity(m, n_points);  // node rows + segment partials
    return (lift > n_points ? lift : n_points) * cdftb::MANY * 8;
}

extern "C" int cdftb_quadrature_interpolate_many_f64(const int* base, const double* w1d, int64_t m, int nx, int ny,
                                                     int nz, const double* fields, int nf, int64_t field_stride,
                                                     double* out, int64_t out_stride, void* scratch,
                                                     int64_t scratch_bytes, cdftb_stream_t stream) {
    const int64_t n_points = int64_t(nx) * ny * nz;
    if (m < 0 || nf < 1 || n_points <= 0 || (m > 0 && (!base || !w1d || !fields || !out || !scratch)))
        return CDFTB_ERR_ARGUMENT;
    if (scratch_bytes < n_points * cdftb::MANY * 8) return CDFTB_ERR_ARGUMENT;
    if (m == 0) return CDFTB_OK;
    cudaStream_t s = as_stream(stream);
    double* rows = static_cast<double*>(scratch);
    for (int f0 = 0; f0 < nf; f0 += cdftb::MANY) {
        const int count = nf - f0 < cdftb::MANY ? nf - f0 : cdftb::MANY;
        int st = cdftb::fields_to_rows(fields + f0 * field_stride, count, field_stride, n_points, rows, s);
        if (st != CDFTB_OK) return st;
        cdftb::interpolate_many_kernel<<<static_cast<unsigned>(ceil_div(m, cdftb::MANY)), 256, 0, s>>>(
            base, w1d, m, ny, nz, rows, count, out + f0 * out_stride, out_stride);
        st = check_launch();
        if (st != CDFTB_OK) return st;
    }
    return CDFTB_OK;
}

extern "C" int cdftb_quadrature_interpolate_grouped_f64(const int* base, const double* w1d, int64_t m, int nx,
                                                        int ny, int nz, const int* group_nodes, const int* group_ptr,
                                                        int64_t groups, const double* fields, int nf,
                                                        int64_t field_stride, double* out, int64_t out_stride,
                                                        void* scratch, int64_t scratch_bytes, cdftb_stream_t stream) {
    const int64_t n_points = int64_t(nx) * ny * nz;
    if (m < 0 || nf < 1 || n_points <= 0 || groups < 0 || groups > m ||
        (m > 0 && (!base || !w1d || !group_nodes || !group_ptr || !fields || !out || !scratch)))
        return CDFTB_ERR_ARGUMENT;
    if (scratch_bytes < n_points * cdftb::MANY * 8) return CDFTB_ERR_ARGUMENT;
    if (m == 0 || groups == 0) return CDFTB_OK;
    cudaStream_t s = as_stream(stream);
    double* rows = static_cast<double*>(scratch);
    for (int f0 = 0; f0 < nf; f0 += cdftb::MANY) {
        const int count = nf - f0 < cdftb::MANY ? nf - f0 : cdftb::MANY;
        int st = cdftb::fields_to_rows(fields + f0 * field_stride, count, field_stride, n_points, rows, s);
        if (st != CDFTB_OK) return st;
        cdftb::interpolate_grouped_kernel<<<static_cast<unsigned>(ceil_div(groups, 8)), 256, 0, s>>>(
            base, w1d, group_nodes, group_ptr, groups, ny, nz, rows, count, out + f0 * out_stride, out_stride);
        st = check_launch();
        if (st != CDFTB_OK) return st;
    }
    return CDFTB_OK;
}

// The weight of every CSR entry of L^T (the same product as the lift kernels form on the fly).
namespace cdftb {
namespace {
__global__ void lift_values_kernel(const int* __restrict__ base, const double* __restrict__ w1d,
                                   const long long* __restrict__ row_ptr, const int* __restrict__ col, int64_t n_points,
                                   int ny, int nz, double* __restrict__ values) {
    const int64_t row = (blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= n_points) return;
    const int jx = static_cast<int>(row / (static_cast<int64_t>(ny) * nz));
    const int jy = static_cast<int>((row / nz) % ny);
    const int jz = static_cast<int>(row % nz);
    for (long long e = row_ptr[row] + lane; e < row_ptr[row + 1]; e += 32) {
        const int node = col[e];
        const int a = jx - (base[node * 3 + 0] - HALFD);
        const int b = jy - (base[node * 3 + 1] - HALFD);
        const int c = jz - (base[node * 3 + 2] - HALFD);
        const double* w = w1d + static_cast<int64_t>(node) * 24;
        values[e] = (w[a] * w[8 + b]) * w[16 + c];
    }
}
}  // namespace
}  // namespace cdftb

extern "C" int cdftb_lift_plan_values_f64(const int* base, const double* w1d, const long long* row_ptr, const int* col,
                                          int nx, int ny, int nz, double* values, cdftb_stream_t stream) {
    const int64_t n_points = static_cast<int64_t>(nx) * ny * nz;
    if (!base || !w1d || !row_ptr || !col || !values || n_points <= 0) return CDFTB_ERR_ARGUMENT;
    cdftb::lift_values_kernel<<<blocks_for(n_points * 32, 256), 256, 0, as_stream(stream)>>>(base, w1d, row_ptr, col,
                                                                                             n_points, ny, nz, values);
    return check_launch();
}

// ---------------------------------------------------------------------------------------------
// L^T for many fields with the CSR rows cut into segments of at most kLiftSegment entries. The rows
// are very uneven (thousands of entries next to a nucleus, none far away), so one warp per segment
// rather than per row keeps every SM busy; each segment leaves a 32-field partial and a second pass
// adds the partials of a row in segment order (deterministic).

namespace cdftb {
namespace {

__global__ void segment_counts_kernel(const long long* __restrict__ row_ptr, int64_t n_points, int* __restrict__ counts) {
    const int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    if (r < n_points) {
        const long long len = row_ptr[r + 1] - row_ptr[r];
        counts[r] = static_cast<int>((len + kLiftSegment - 1) / kLiftSegment);
    } else if (r == n_points) {
        counts[r] = 0;
    }
}

__global__ void segment_rows_kernel(const int* __restrict__ seg_ptr, int64_t n_points, int* __restrict__ seg_row) {
    const int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    if (r >= n_points) return;
    for (int sgi = seg_ptr[r]; sgi < seg_ptr[r + 1]; ++sgi) seg_row[sgi] = static_cast<int>(r);
}

__global__ void __launch_bounds__(256) lift_segments_kernel(const long long* __restrict__ row_ptr,
                                                            const int* __restrict__ col,
                                                            const double* __restrict__ values,
                                                            const int* __restrict__ seg_ptr,
                                                            const int* __restrict__ seg_row, int64_t n_points,
                                                            const double* __restrict__ rows,
                                                            double* __restrict__ partial) {
    const int64_t sgi = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (sgi >= seg_ptr[n_points]) return;
    const int r = seg_row[sgi];
    const long long eb0 = row_ptr[r] + (sgi - seg_ptr[r]) * int64_t(kLiftSegment);
    const long long ee = min(row_ptr[r + 1], eb0 + kLiftSegment);
    double acc[4] = {0.0, 0.0, 0.0, 0.0};  // four independent chains, added in a fixed order at the end
    for (long long eb = eb0; eb < ee; eb += 32) {
        int node_l = 0;
        double v_l = 0.0;
        if (eb + lane < ee) {
            node_l = col[eb + lane];
            v_l = values[eb + lane];
        }
        const int count = (ee - eb) < 32 ? static_cast<int>(ee - eb) : 32;
        int k = 0;
        for (; k + 8 <= count; k += 8) {
            double g[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) g[u] = rows[int64_t(__shfl_sync(0xffffffffu, node_l, k + u)) * MANY + lane];
#pragma unroll
            for (int u = 0; u < 8; ++u) acc[u & 3] = fma(g[u], __shfl_sync(0xffffffffu, v_l, k + u), acc[u & 3]);
        }
        for (; k < count; ++k)
            acc[0] = fma(rows[int64_t(__shfl_sync(0xffffffffu, node_l, k)) * MANY + lane],
                         __shfl_sync(0xffffffffu, v_l, k), acc[0]);
    }
    partial[sgi * MANY + lane] = (acc[0] + acc[1]) + (acc[2] + acc[3]);
}

__global__ void __launch_bounds__(256) lift_segments_sum_kernel(const int* __restrict__ seg_ptr, int64_t n_points,
                                                                const double* __restrict__ partial, int nf,
                                                                double* __restrict__ out, int64_t out_stride) {
    __shared__ double tile[MANY][MANY + 1];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int64_t j0 = int64_t(blockIdx.x) * MANY;
    for (int r = warp; r < MANY; r += 8) {
        const int64_t row = j0 + r;
        if (row >= n_points) break;
        double acc = 0.0;
        for (int sgi = seg_ptr[row]; sgi < seg_ptr[row + 1]; ++sgi) acc += partial[int64_t(sgi) * MANY + lane];
        tile[r][lane] = acc;
    }
    store_tile(tile, j0, n_points, nf, out, out_stride);
}

}  // namespace
}  // namespace cdftb

extern "C" int64_t cdftb_lift_segments_scratch_bytes(int64_t n_points) {
    if (n_points <= 0) return 0;
    size_t scan_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, static_cast<int*>(nullptr), static_cast<int*>(nullptr),
                                  static_cast<int>(n_points + 1));
    return static_cast<int64_t>(((n_points + 1) * 4 + 255) / 256 * 256 + scan_bytes);
}

extern "C" int cdftb_lift_plan_segments(const long long* row_ptr, int nx, int ny, int nz, int* seg_ptr, int* seg_row,
                                        int64_t capacity, void* scratch, int64_t scratch_bytes,
                                        cdftb_stream_t stream) {
    const int64_t n_points = int64_t(nx) * ny * nz;
    if (!row_ptr || !seg_ptr || !seg_row || !scratch || n_points <= 0 || n_points >= (1ll << 31) - 1)
        return CDFTB_ERR_ARGUMENT;
    if (scratch_bytes < cdftb_lift_segments_scratch_bytes(n_points)) return CDFTB_ERR_ARGUMENT;
    cudaStream_t s = as_stream(stream);
    int* counts = static_cast<int*>(scratch);
    char* temp = static_cast<char*>(scratch) + ((n_points + 1) * 4 + 255) / 256 * 256;
    size_t scan_bytes = static_cast<size_t>(scratch_bytes) - (temp - static_cast<char*>(scratch));
    cdftb::segment_counts_kernel<<<blocks_for(n_points + 1, 256), 256, 0, s>>>(row_ptr, n_points, counts);
    int st = check_launch();
    if (st != CDFTB_OK) return st;
    if ((st = check(cub::DeviceScan::ExclusiveSum(temp, scan_bytes, counts, seg_ptr, static_cast<int>(n_points + 1),
                                                  s))) != CDFTB_OK)
        return st;
    // capacity bounds the segment count by construction: sum ceil(len/S) <= nnz/S + rows
    (void)capacity;
    cdftb::segment_rows_kernel<<<blocks_for(n_points, 256), 256, 0, s>>>(seg_ptr, n_points, seg_row);
    return check_launch();
}

extern "C" int cdftb_quadrature_lift_many_f64(const long long* row_ptr, const int* col, const double* values,
                                              const int* seg_ptr, const int* seg_row, int64_t seg_capacity, int nx,
                                              int ny, int nz, int64_t m, const double* node_values, int nf,
                                              int64_t x_stride, double* out, int64_t out_stride, void* scratch,
                                              int64_t scratch_bytes, cdftb_stream_t stream) {
    const int64_t n_points = int64_t(nx) * ny * nz;
    if (m <= 0 || nf < 1 || n_points <= 0 || !row_ptr || !col || !values || !seg_ptr || !seg_row || !node_values ||
        !out || !scratch || seg_capacity < cdftb_lift_segments_capacity(m, n_points))
        return CDFTB_ERR_ARGUMENT;
    if (scratch_bytes < (m + seg_capacity) * cdftb::MANY * 8) return CDFTB_ERR_ARGUMENT;
    cudaStream_t s = as_stream(stream);
    double* rows = static_cast<double*>(scratch);
    double* partial = rows + m * cdftb::MANY;
    for (int f0 = 0; f0 < nf; f0 += cdftb::MANY) {
        const int count = nf - f0 < cdftb::MANY ? nf - f0 : cdftb::MANY;
        int st = cdftb::fields_to_rows(node_values + f0 * x_stride, count, x_stride, m, rows, s);
        if (st != CDFTB_OK) return st;
        cdftb::lift_segments_kernel<<<blocks_for(seg_capacity * 32, 256), 256, 0, s>>>(row_ptr, col, values, seg_ptr,
                                                                                       seg_row, n_points, rows, partial);
        if ((st = check_launch()) != CDFTB_OK) return st;
        cdftb::lift_segments_sum_kernel<<<static_cast<unsigned>(ceil_div(n_points, cdftb::MANY)), 256, 0, s>>>(
            seg_ptr, n_points, partial, count, out + f0 * out_stride, out_stride);
        if ((st = check_launch()) != CDFTB_OK) return st;
    }
    return CDFTB_OK;
}
