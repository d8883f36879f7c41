// (e2-e5) The small dense steps of Rayleigh--Ritz kept on the device, so an eigensolver iteration
// needs no host round trip: Cholesky of the m x m Gram matrix, the triangular solve L^{-1} B
// applied column by column (what torch.linalg.solve_triangular does for each grid point,
// src/cdft/eigen/rayleigh_ritz.py:51-72), the symmetric eigenproblem of the subspace matrix by
// cyclic Jacobi (rayleigh_ritz.py:97-99), the block rotation U^T Q (rayleigh_ritz.py:100), the
// residual H psi - eps psi (rayleigh_ritz.py:105-115) and the Lanczos vector updates
// (src/cdft/operators/hamiltonian.py:252-262). m is at most 32.

#include <math.h>

#include "common.cuh"

namespace cdftb {

namespace {

constexpr int MMAX = 32;

__global__ void cholesky_kernel(const double* __restrict__ gram, double* __restrict__ lower, int* __restrict__ info,
                                int m, int groups) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= groups) return;
    const double* s = gram + static_cast<int64_t>(g) * m * m;
    double* l = lower + static_cast<int64_t>(g) * m * m;
    int bad = 0;
    for (int i = 0; i < m * m; ++i) l[i] = 0.0;
    for (int j = 0; j < m && !bad; ++j) {
        double d = s[j * m + j];
        for (int k = 0; k < j; ++k) d -= l[j * m + k] * l[j * m + k];
        if (!(d > 0.0)) {
            bad = j + 1;
            break;
        }
        const double ljj = sqrt(d);
        l[j * m + j] = ljj;
        for (int i = j + 1; i < m; ++i) {
            double v = s[i * m + j];
            for (int k = 0; k < j; ++k) v -= l[i * m + k] * l[j * m + k];
            l[i * m + j] = v / ljj;
        }
    }
    info[g] = bad;
}

// Forward substitution x = L^{-1} b for every column p of a block (rows are orbitals).
__global__ void trsm_lower_kernel(const double* __restrict__ lower, const double* __restrict__ in, int64_t in_stride,
                                  void* out, int out_dtype, int64_t out_stride, int m, int64_t n, int groups) {
    __shared__ double l[MMAX * MMAX];
    const int g = blockIdx.y;
    for (int i = threadIdx.x; i < m * m; i += blockDim.x) l[i] = lower[static_cast<int64_t>(g) * m * m + i];
    __syncthreads();
    const double* src = in + g * in_stride;
    for (int64_t p = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; p < n;
         p += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        double x[MMAX];
#pragma unroll
        for (int i = 0; i < MMAX; ++i) {
            if (i >= m) break;
            double v = src[i * n + p];
            for (int k = 0; k < i; ++k) v -= l[i * m + k] * x[k];
            x[i] = v / l[i * m + i];
            store_as<double>(out, out_dtype, g * out_stride + i * n + p, x[i]);
        }
    }
}

__global__ void eigh_kernel(const double* __restrict__ matrix, double* __restrict__ evals, double* __restrict__ vectors,
                            int m, int groups) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= groups) return;
    double a[MMAX * MMAX];
    double v[MMAX * MMAX];
    const double* src = matrix + static_cast<int64_t>(g) * m * m;
    for (int i = 0; i < m; ++i)
        for (int j = 0; j < m; ++j) {
            a[i * m + j] = 0.5 * (src[i * m + j] + src[j * m + i]);
            v[i * m + j] = (i == j) ? 1.0 : 0.0;
        }
    for (int sweep = 0; sweep < 64; ++sweep) {
        double off = 0.0, diag = 0.0;
        for (int i = 0; i < m; ++i) {
            diag += a[i * m + i] * a[i * m + i];
            for (int j = i + 1; j < m; ++j) off += a[i * m + j] * a[i * m + j];
        }
        if (off <= 1e-36 * diag || off == 0.0) break;
        for (int p = 0; p < m - 1; ++p) {
            for (int q = p + 1; q < m; ++q) {
                const double apq = a[p * m + q];
                if (apq == 0.0) continue;
                const double app = a[p * m + p];
                const double aqq = a[q * m + q];
                const double theta = (aqq - app) / (2.0 * apq);
                const double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0);
                const double s = t * c;
                for (int k = 0; k < m; ++k) {
                    const double akp = a[k * m + p];
                    const double akq = a[k * m + q];
                    a[k * m + p] = c * akp - s * akq;
                    a[k * m + q] = s * akp + c * akq;
                }
                for (int k = 0; k < m; ++k) {
                    const double apk = a[p * m + k];
                    const double aqk = a[q * m + k];
                    a[p * m + k] = c * apk - s * aqk;
                    a[q * m + k] = s * apk + c * aqk;
                }
                a[p * m + q] = 0.0;
                a[q * m + p] = 0.0;
                for (int k = 0; k < m; ++k) {
                    const double vkp = v[k * m + p];
                    const double vkq = v[k * m + q];
                    v[k * m + p] = c * vkp - s * vkq;
                    v[k * m + q] = s * vkp + c * vkq;
                }
            }
        }
    }
    // Sort ascending (selection sort: m is small) and write eigenvectors as rows.
    int order[MMAX];
    for (int i = 0; i < m; ++i) order[i] = i;
    for (int i = 0; i < m; ++i) {
        int best = i;
        for (int j = i + 1; j < m; ++j)
            if (a[order[j] * m + order[j]] < a[order[best] * m + order[best]]) best = j;
        const int tmp = order[i];
        order[i] = order[best];
        order[best] = tmp;
    }
    double* ev = evals + static_cast<int64_t>(g) * m;
    double* vec = vectors + static_cast<int64_t>(g) * m * m;
    for (int k = 0; k < m; ++k) {
        const int col = order[k];
        ev[k] = a[col * m + col];
        for (int j = 0; j < m; ++j) vec[k * m + j] = v[j * m + col];
    }
}

// eigh_kernel for a width known at compile time (m <= 6): the same sweeps, rotations and sort in the
// same order, with the matrices in registers instead of local memory.
template <int M>
__global__ void eigh_fixed_kernel(const double* __restrict__ matrix, double* __restrict__ evals,
                                  double* __restrict__ vectors, int groups) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= groups) return;
    double a[M][M];
    double v[M][M];
    const double* src = matrix + static_cast<int64_t>(g) * M * M;
#pragma unroll
    for (int i = 0; i < M; ++i)
#pragma unroll
        for (int j = 0; j < M; ++j) {
            a[i][j] = 0.5 * (src[i * M + j] + src[j * M + i]);
            v[i][j] = (i == j) ? 1.0 : 0.0;
        }
    for (int sweep = 0; sweep < 64; ++sweep) {
        double off = 0.0, diag = 0.0;
#pragma unroll
        for (int i = 0; i < M; ++i) {
            diag += a[i][i] * a[i][i];
#pragma unroll
            for (int j = i + 1; j < M; ++j) off += a[i][j] * a[i][j];
        }
        if (off <= 1e-36 * diag || off == 0.0) break;
#pragma unroll
        for (int p = 0; p < M - 1; ++p) {
#pragma unroll
            for (int q = p + 1; q < M; ++q) {
                const double apq = a[p][q];
                if (apq == 0.0) continue;
                const double app = a[p][p];
                const double aqq = a[q][q];
                const double theta = (aqq - app) / (2.0 * apq);
                const double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0);
                const double s = t * c;
#pragma unroll
                for (int k = 0; k < M; ++k) {
                    const double akp = a[k][p];
                    const double akq = a[k][q];
                    a[k][p] = c * akp - s * akq;
                    a[k][q] = s * akp + c * akq;
                }
#pragma unroll
                for (int k = 0; k < M; ++k) {
                    const double apk = a[p][k];
                    const double aqk = a[q][k];
                    a[p][k] = c * apk - s * aqk;
                    a[q][k] = s * apk + c * aqk;
                }
                a[p][q] = 0.0;
                a[q][p] = 0.0;
#pragma unroll
                for (int k = 0; k < M; ++k) {
                    const double vkp = v[k][p];
                    const double vkq = v[k][q];
                    v[k][p] = c * vkp - s * vkq;
                    v[k][q] = s * vkp + c * vkq;
                }
            }
        }
    }
    // ascending order (the selection sort of eigh_kernel), eigenvectors written as rows
    double d[M];
    int order[M];
#pragma unroll
    for (int i = 0; i < M; ++i) {
        d[i] = a[i][i];
        order[i] = i;
    }
#pragma unroll
    for (int i = 0; i < M; ++i) {
        int best = i;
#pragma unroll
        for (int j = i + 1; j < M; ++j)
            if (d[j] < d[best]) best = j;
        // swap entries i and best of (d, order) with register-only selects
#pragma unroll
        for (int j = i + 1; j < M; ++j)
            if (j == best) {
                const double td = d[i];
                d[i] = d[j];
                d[j] = td;
                const int to = order[i];
                order[i] = order[j];
                order[j] = to;
            }
    }
    double* ev = evals + static_cast<int64_t>(g) * M;
    double* vec = vectors + static_cast<int64_t>(g) * M * M;
#pragma unroll
    for (int k = 0; k < M; ++k) {
        ev[k] = d[k];
#pragma unroll
        for (int col = 0; col < M; ++col)
            if (col == order[k]) {
#pragma unroll
                for (int j = 0; j < M; ++j) vec[k * M + j] = v[j][col];
            }
    }
}

__global__ void rotate_kernel(const double* __restrict__ r, const double* __restrict__ in, int64_t in_stride, void* out,
                              int out_dtype, int64_t out_stride, int m_out, int m_in, int64_t n) {
    __shared__ double rs[MMAX * MMAX];
    const int g = blockIdx.y;
    for (int i = threadIdx.x; i < m_out * m_in; i += blockDim.x) rs[i] = r[static_cast<int64_t>(g) * m_out * m_in + i];
    __syncthreads();
    const double* src = in + g * in_stride;
    for (int64_t p = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; p < n;
         p += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        double x[MMAX];
        for (int j = 0; j < m_in; ++j) x[j] = src[j * n + p];
        for (int i = 0; i < m_out; ++i) {
            double v = 0.0;
            for (int j = 0; j < m_in; ++j) v = fma(rs[i * m_in + j], x[j], v);
            store_as<double>(out, out_dtype, g * out_stride + i * n + p, v);
        }
    }
}

__global__ void residual_kernel(const double* __restrict__ a, const double* __restrict__ b,
                                const double* __restrict__ evals, double* __restrict__ out, int m, int64_t n,
                                int64_t group_stride) {
    const int g = blockIdx.y;
    for (int64_t p = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; p < n;
         p += static_cast<int64_t>(gridDim.x) * blockDim.x)
        for (int i = 0; i < m; ++i) {
            const int64_t k = g * group_stride + i * n + p;
            out[k] = a[k] - evals[g * m + i] * b[k];
        }
}

__global__ void lanczos_kernel(int mode, double* __restrict__ w, const double* __restrict__ v,
                               const double* __restrict__ v_prev, const double* __restrict__ s1,
                               const double* __restrict__ s2, int64_t n) {
    const int g = blockIdx.y;
    const double a1 = s1 ? s1[g] : 0.0;
    const double a2 = s2 ? s2[g] : 0.0;
    for (int64_t p = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; p < n;
         p += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t k = g * n + p;
        if (mode == 0 || mode == 1) {
            // w - a1 v - a2 v_prev, as (w - a1 v) - a2 v_prev (hamiltonian.py:255, 258)
            w[k] = (w[k] - a1 * v[k]) - a2 * v_prev[k];
        } else {
            // v_next = w / sqrt(a1) with a1 = <w, w> (hamiltonian.py:259-262)
            w[k] = w[k] / sqrt(a1 > 0.0 ? a1 : 0.0);
        }
    }
}

// The same two kernels for a block width known at compile time (the common m <= 8): the orbital
// values of a point stay in registers instead of a runtime-indexed array.
template <int M>
__global__ void trsm_lower_fixed_kernel(const double* __restrict__ lower, const double* __restrict__ in,
                                        int64_t in_stride, void* out, int out_dtype, int64_t out_stride, int64_t n) {
    __shared__ double l[M * M];
    const int g = blockIdx.y;
    for (int i = threadIdx.x; i < M * M; i += blockDim.x) l[i] = lower[static_cast<int64_t>(g) * M * M + i];
    __syncthreads();
    const double* src = in + g * in_stride;
    auto solve = [&](int64_t p, double* x) {
#pragma unroll
        for (int i = 0; i < M; ++i) {
            double v = x[i];
#pragma unroll
            for (int k = 0; k < i; ++k) v -= l[i * M + k] * x[k];
            x[i] = v / l[i * M + i];
            store_as<double>(out, out_dtype, g * out_stride + i * n + p, x[i]);
        }
    };
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    int64_t p = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    // two points per thread at a time: both points' loads are in flight before either is solved
    for (; p + stride < n; p += 2 * stride) {
        double x0[M], x1[M];
#pragma unroll
        for (int i = 0; i < M; ++i) {
            x0[i] = src[i * n + p];
            x1[i] = src[i * n + p + stride];
        }
        solve(p, x0);
        solve(p + stride, x1);
    }
    if (p < n) {
        double x0[M];
#pragma unroll
        for (int i = 0; i < M; ++i) x0[i] = src[i * n + p];
        solve(p, x0);
    }
}

template <int M>
__global__ void rotate_fixed_kernel(const double* __restrict__ r, const double* __restrict__ in, int64_t in_stride,
                                    void* out, int out_dtype, int64_t out_stride, int64_t n) {
    __shared__ double rs[M * M];
    const int g = blockIdx.y;
    for (int i = threadIdx.x; i < M * M; i += blockDim.x) rs[i] = r[static_cast<int64_t>(g) * M * M + i];
    __syncthreads();
    const double* src = in + g * in_stride;
    for (int64_t p = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; p < n;
         p += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        double x[M];
#pragma unroll
        for (int j = 0; j < M; ++j) x[j] = src[j * n + p];
#pragma unroll
        for (int i = 0; i < M; ++i) {
            double v = 0.0;
#pragma unroll
            for (int j = 0; j < M; ++j) v = fma(rs[i * M + j], x[j], v);
            store_as<double>(out, out_dtype, g * out_stride + i * n + p, v);
        }
    }
}

// The end of Rayleigh--Ritz in one pass over the block: v_i = sum_j R_ij basis_j and
// (A v)_i = sum_j R_ij applied_j (the FMA order of rotate_fixed_kernel), the residual
// rho_i = (A v)_i - lambda_i v_i (as residual_kernel), v written out and q rho_i^2 summed. A CTA
// takes a fixed chunk of points of one group, two points per thread at a time, and writes one
// partial per row; ritz_final_kernel adds the partials in chunk order (deterministic).
constexpr int RITZ_THREADS = 256;

template <int M>
__global__ void __launch_bounds__(RITZ_THREADS) ritz_fixed_kernel(const double* __restrict__ r,
                                                                 const double* __restrict__ basis,
                                                                 const double* __restrict__ applied,
                                                                 const double* __restrict__ evals,
                                                                 const double* __restrict__ q, int64_t q_stride,
                                                                 int64_t n, int64_t chunk,
                                                                 double* __restrict__ vectors,
                                                                 double* __restrict__ partial) {
    __shared__ double rs[M * M];
    __shared__ double lam[M];
    __shared__ double red[RITZ_THREADS / 32][M];
    const int g = blockIdx.y;
    const int c = blockIdx.x;
    for (int i = threadIdx.x; i < M * M; i += blockDim.x) rs[i] = r[static_cast<int64_t>(g) * M * M + i];
    if (threadIdx.x < M) lam[threadIdx.x] = evals[static_cast<int64_t>(g) * M + threadIdx.x];
    __syncthreads();
    const int64_t base = static_cast<int64_t>(g) * M * n;
    const double* qg = q + g * q_stride;
    const int64_t p0 = c * chunk;
    const int64_t p1 = (p0 + chunk < n) ? p0 + chunk : n;
    double acc[M];
#pragma unroll
    for (int i = 0; i < M; ++i) acc[i] = 0.0;
    auto point = [&](int64_t p, const double* x, const double* y, double w) {
#pragma unroll
        for (int i = 0; i < M; ++i) {
            double v = 0.0, av = 0.0;
#pragma unroll
            for (int j = 0; j < M; ++j) {
                v = fma(rs[i * M + j], x[j], v);
                av = fma(rs[i * M + j], y[j], av);
            }
            vectors[base + i * n + p] = v;
            const double res = av - lam[i] * v;
            acc[i] = fma(res * w, res, acc[i]);
        }
    };
    int64_t p = p0 + threadIdx.x;
    constexpr bool kPairs = M <= 5;  // two points in flight per thread where the registers allow it
    for (; kPairs && p + RITZ_THREADS < p1; p += 2 * RITZ_THREADS) {
        double x0[M], y0[M], x1[M], y1[M];
#pragma unroll
        for (int j = 0; j < M; ++j) {
            x0[j] = basis[base + j * n + p];
            y0[j] = applied[base + j * n + p];
            x1[j] = basis[base + j * n + p + RITZ_THREADS];
            y1[j] = applied[base + j * n + p + RITZ_THREADS];
        }
        const double w0 = qg[p], w1 = qg[p + RITZ_THREADS];
        point(p, x0, y0, w0);
        point(p + RITZ_THREADS, x1, y1, w1);
    }
    for (; p < p1; p += RITZ_THREADS) {
        double x0[M], y0[M];
#pragma unroll
        for (int j = 0; j < M; ++j) {
            x0[j] = basis[base + j * n + p];
            y0[j] = applied[base + j * n + p];
        }
        point(p, x0, y0, qg[p]);
    }
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < M; ++i) {
        double v = acc[i];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        if (lane == 0) red[warp][i] = v;
    }
    __syncthreads();
    if (threadIdx.x < M) {
        double v = 0.0;
        for (int w = 0; w < RITZ_THREADS / 32; ++w) v += red[w][threadIdx.x];
        partial[(static_cast<int64_t>(g) * gridDim.x + c) * M + threadIdx.x] = v;
    }
}

// One warp per (group, row): lanes take chunks lane, lane + 32, ... in order, then a fixed shuffle tree.
__global__ void ritz_final_kernel(const double* __restrict__ partial, int m, int chunks, int groups,
                                  double* __restrict__ out) {
    const int64_t idx = (blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (idx >= static_cast<int64_t>(groups) * m) return;
    const int64_t g = idx / m;
    const int i = static_cast<int>(idx - g * m);
    double v = 0.0;
    for (int c = lane; c < chunks; c += 32) v += partial[(g * chunks + c) * m + i];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if (lane == 0) out[idx] = v;
}

int ritz_chunks(int64_t n, int groups) {
    int64_t chunks = ceil_div(int64_t(8) * 148, groups);  // about 8 CTAs per SM over the whole launch
    const int64_t most = ceil_div(n, int64_t(2048));
    if (chunks > most) chunks = most;
    return static_cast<int>(chunks < 1 ? 1 : chunks);
}

// CTAs along the points of each group: about 8 per SM over the whole launch (all groups), so that
// with many groups every thread loops over several points instead of the launch running many
// short waves of one point per thread.
inline unsigned point_blocks(int64_t n, int groups) {
    const int64_t b = ceil_div(n, 256);
    int64_t cap = ceil_div(int64_t(148) * 8, groups > 0 ? groups : 1);
    if (cap < 1) cap = 1;
    return static_cast<unsigned>(b < cap ? b : cap);
}

}  // namespace

}  // namespace cdftb

using namespace cdftb;

extern "C" int cdftb_small_cholesky_f64(const double* gram, double* lower, int* info, int m, int groups,
                                        cdftb_stream_t stream) {
    if (!gram || !lower || !info || m <= 0 || m > MMAX || groups <= 0) return CDFTB_ERR_ARGUMENT;
    cholesky_kernel<<<static_cast<unsigned>(ceil_div(groups, 32)), 32, 0, as_stream(stream)>>>(gram, lower, info, m, groups);
    return check_launch();
}

extern "C" int cdftb_block_trsm_lower_f64(const double* lower, const double* in, int64_t in_group_stride, void* out,
                                          int out_dtype, int64_t out_group_stride, int m, int64_t n, int groups,
                                          cdftb_stream_t stream) {
    if (!lower || !in || !out || m <= 0 || m > MMAX || n <= 0 || groups <= 0 || groups > 65535) return CDFTB_ERR_ARGUMENT;
    dim3 grid(point_blocks(n, groups), groups);
    cudaStream_t s = as_stream(stream);
    switch (m) {
#define CDFTB_TRSM(M)                                                                                             \
    case M:                                                                                                       \
        trsm_lower_fixed_kernel<M><<<grid, 256, 0, s>>>(lower, in, in_group_stride, out, out_dtype, out_group_stride, \
                                                        n);                                                       \
        return check_launch();
        CDFTB_TRSM(1) CDFTB_TRSM(2) CDFTB_TRSM(3) CDFTB_TRSM(4) CDFTB_TRSM(5) CDFTB_TRSM(6) CDFTB_TRSM(7) CDFTB_TRSM(8)
#undef CDFTB_TRSM
        default: break;
    }
    trsm_lower_kernel<<<grid, 256, 0, s>>>(lower, in, in_group_stride, out, out_dtype, out_group_stride, m, n, groups);
    return check_launch();
}

extern "C" int cdftb_small_eigh_f64(const double* matrix, double* evals, double* vectors, int m, int groups,
                                    cdftb_stream_t stream) {
    if (!matrix || !evals || !vectors || m <= 0 || m > MMAX || groups <= 0) return CDFTB_ERR_ARGUMENT;
    const unsigned blocks = static_cast<unsigned>(ceil_div(groups, 32));
    cudaStream_t s = as_stream(stream);
    switch (m) {
#define CDFTB_EIGH(M)                                                                \
    case M:                                                                          \
        eigh_fixed_kernel<M><<<blocks, 32, 0, s>>>(matrix, evals, vectors, groups); \
        return check_launch();
        CDFTB_EIGH(1) CDFTB_EIGH(2) CDFTB_EIGH(3) CDFTB_EIGH(4) CDFTB_EIGH(5) CDFTB_EIGH(6)
#undef CDFTB_EIGH
        default: break;
    }
    eigh_kernel<<<blocks, 32, 0, s>>>(matrix, evals, vectors, m, groups);
    return check_launch();
}

extern "C" int cdftb_block_rotate_f64(const double* r, const double* in, int64_t in_group_stride, void* out,
                                      int out_dtype, int64_t out_group_stride, int m_out, int m_in, int64_t n,
                                      int groups, cdftb_stream_t stream) {
    if (!r || !in || !out || m_out <= 0 || m_in <= 0 || m_out > MMAX || m_in > MMAX || n <= 0 || groups <= 0 ||
        groups > 65535)
        return CDFTB_ERR_ARGUMENT;
    dim3 grid(point_blocks(n, groups), groups);
    cudaStream_t s = as_stream(stream);
    if (m_out == m_in) {
        switch (m_in) {
#define CDFTB_ROT(M)                                                                                                 \
    case M:                                                                                                          \
        rotate_fixed_kernel<M><<<grid, 256, 0, s>>>(r, in, in_group_stride, out, out_dtype, out_group_stride, n); \
        return check_launch();
            CDFTB_ROT(1) CDFTB_ROT(2) CDFTB_ROT(3) CDFTB_ROT(4) CDFTB_ROT(5) CDFTB_ROT(6) CDFTB_ROT(7) CDFTB_ROT(8)
#undef CDFTB_ROT
            default: break;
        }
    }
    rotate_kernel<<<grid, 256, 0, s>>>(r, in, in_group_stride, out, out_dtype, out_group_stride, m_out, m_in, n);
    return check_launch();
}

extern "C" int cdftb_block_residual_f64(const double* a, const double* b, const double* evals, double* out, int m,
                                        int64_t n, int groups, int64_t group_stride, cdftb_stream_t stream) {
    if (!a || !b || !evals || !out || m <= 0 || n <= 0 || groups <= 0 || groups > 65535) return CDFTB_ERR_ARGUMENT;
    dim3 grid(point_blocks(n, groups), groups);
    residual_kernel<<<grid, 256, 0, as_stream(stream)>>>(a, b, evals, out, m, n, group_stride);
    return check_launch();
}

extern "C" int cdftb_lanczos_update_f64(int mode, double* w, const double* v, const double* v_prev, const double* s1,
                                        const double* s2, int64_t n, int groups, cdftb_stream_t stream) {
    if (!w || mode < 0 || mode > 2 || n <= 0 || groups <= 0 || groups > 65535) return CDFTB_ERR_ARGUMENT;
    if (mode < 2 && (!v || !v_prev || !s1 || !s2)) return CDFTB_ERR_ARGUMENT;
    if (mode == 2 && !s1) return CDFTB_ERR_ARGUMENT;
    dim3 grid(point_blocks(n, groups), groups);
    lanczos_kernel<<<grid, 256, 0, as_stream(stream)>>>(mode, w, v, v_prev, s1, s2, n);
    return check_launch();
}

extern "C" int64_t cdftb_block_ritz_scratch_bytes(int m, int64_t n, int groups) {
    if (m <= 0 || n <= 0 || groups <= 0) return 0;
    return static_cast<int64_t>(groups) * ritz_chunks(n, groups) * m * 8;
}

extern "C" int cdftb_block_ritz_f64(const double* r, const double* basis, const double* applied, const double* evals,
                                    const double* q, int64_t q_group_stride, int m, int64_t n, int groups,
                                    double* vectors, double* norms_sq, void* scratch, int64_t scratch_bytes,
                                    cdftb_stream_t stream) {
    if (!r || !basis || !applied || !evals || !q || !vectors || !norms_sq || m <= 0 || m > 8 || n <= 0 ||
        groups <= 0 || groups > 65535 || q_group_stride < 0)
        return CDFTB_ERR_ARGUMENT;
    if (!scratch || scratch_bytes < cdftb_block_ritz_scratch_bytes(m, n, groups)) return CDFTB_ERR_ARGUMENT;
    const int chunks = ritz_chunks(n, groups);
    const int64_t chunk = ceil_div(n, static_cast<int64_t>(chunks));
    const int used = static_cast<int>(ceil_div(n, chunk));
    cudaStream_t s = as_stream(stream);
    double* partial = static_cast<double*>(scratch);
    dim3 grid(used, groups);
    switch (m) {
#define CDFTB_RITZ(M)                                                                                             \
    case M:                                                                                                       \
        ritz_fixed_kernel<M><<<grid, RITZ_THREADS, 0, s>>>(r, basis, applied, evals, q, q_group_stride, n, chunk, \
                                                           vectors, partial);                                     \
        break;
        CDFTB_RITZ(1) CDFTB_RITZ(2) CDFTB_RITZ(3) CDFTB_RITZ(4) CDFTB_RITZ(5) CDFTB_RITZ(6) CDFTB_RITZ(7) CDFTB_RITZ(8)
#undef CDFTB_RITZ
        default: return CDFTB_ERR_ARGUMENT;
    }
    int rc = check_launch();
    if (rc != CDFTB_OK) return rc;
    const int64_t warps = static_cast<int64_t>(groups) * m;
    ritz_final_kernel<<<static_cast<unsigned>(ceil_div(warps * 32, 256)), 256, 0, s>>>(partial, m, used, groups,
                                                                                       norms_sq);
    return check_launch();
}

