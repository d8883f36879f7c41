// (e1) Tall-skinny weighted products M_ij = sum_p q_p a_ip b_jp for blocks of a few rows and
// O(10^5-10^6) columns: the Gram, cross and inner products of the measure
// (src/cdft/eigen/measure.py:72-96). Two deterministic passes: every CTA reduces a fixed chunk of
// columns for a tile of (i, j) pairs into a partial, and a second kernel sums the partials of each
// pair in chunk order, so the result does not depend on scheduling.

#include <cuda.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "common.cuh"

namespace cdftb {

namespace {

constexpr int RT = 256;

struct CrossShape {
    int ti, tj, tiles_i, tiles_j, chunks;
    int64_t chunk;
};

CrossShape cross_shape(int ma, int mb, int64_t n, int groups) {
    CrossShape s{};
    if (ma == 1 && mb == 1) {
        s.ti = s.tj = 1;
    } else if (ma <= 6 && mb <= 6) {
        s.ti = s.tj = ma > mb ? ma : mb;  // one tile of exactly the block width (2 .. 6)
    } else {
        s.ti = s.tj = 4;
    }
    s.tiles_i = static_cast<int>(ceil_div(ma, s.ti));
    s.tiles_j = static_cast<int>(ceil_div(mb, s.tj));
    const int64_t blocks_per_chunkset = static_cast<int64_t>(s.tiles_i) * s.tiles_j * groups;
    int64_t chunks = ceil_div(8 * 148, blocks_per_chunkset);  // about 8 CTAs of 256 threads per SM
    const int64_t max_chunks = ceil_div(n, 2048);
    if (chunks > max_chunks) chunks = max_chunks;
    if (chunks < 1) chunks = 1;
    s.chunk = ceil_div(n, chunks);
    s.chunks = static_cast<int>(ceil_div(n, s.chunk));
    return s;
}

// SAME: a and b are the same rows (a Gram matrix), each row is loaded once. Each thread takes the
// columns p0 + t, p0 + t + RT, ... U at a time (independent loads in flight), always in the same
// order, so the partial of a chunk does not depend on scheduling (nor on U or the tile shape: an
// entry's sum runs over the same columns in the same order). Tiles of 16 entries or more take two
// points at a time, smaller ones four; tiles of up to 5 x 5 fit two CTAs per SM.
template <int TI, int TJ, bool SAME>
__global__ void __launch_bounds__(RT, (TI <= 5 && TJ <= 5) ? 2 : 1) cross_partial_kernel(const double* __restrict__ a, int ma, int64_t sa,
                                                            const double* __restrict__ b, int mb, int64_t sb,
                                                            const double* __restrict__ q, int64_t q_stride, int64_t n,
                                                            int tiles_j, int64_t chunk, int chunks,
                                                            double* __restrict__ partial) {
    constexpr int U = (TI * TJ >= 16) ? 2 : 4;
    const int c = blockIdx.x;
    const int tile = blockIdx.y;
    const int g = blockIdx.z;
    const int i0 = (tile / tiles_j) * TI;
    const int j0 = (tile % tiles_j) * TJ;
    const int64_t p0 = c * chunk;
    const int64_t p1 = (p0 + chunk < n) ? p0 + chunk : n;
    const double* ag = a + g * sa;
    const double* bg = b + g * sb;
    const double* qg = q ? q + g * q_stride : nullptr;
    double acc[TI][TJ];
#pragma unroll
    for (int i = 0; i < TI; ++i)
#pragma unroll
        for (int j = 0; j < TJ; ++j) acc[i][j] = 0.0;
    int64_t p = p0 + threadIdx.x;
    for (; p + (U - 1) * RT < p1; p += U * RT) {
        double w[U], av[U][TI], bv[U][TJ];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int64_t pu = p + u * RT;
            w[u] = qg ? qg[pu] : 1.0;
#pragma unroll
            for (int i = 0; i < TI; ++i) av[u][i] = (i0 + i < ma) ? ag[(i0 + i) * n + pu] : 0.0;
            if (!SAME) {
#pragma unroll
                for (int j = 0; j < TJ; ++j) bv[u][j] = (j0 + j < mb) ? bg[(j0 + j) * n + pu] : 0.0;
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
#pragma unroll
            for (int i = 0; i < TI; ++i) {
                const double wa = av[u][i] * w[u];
#pragma unroll
                for (int j = 0; j < TJ; ++j) acc[i][j] = fma(wa, SAME ? av[u][j] : bv[u][j], acc[i][j]);
            }
        }
    }
    for (; p < p1; p += RT) {
        const double w = qg ? qg[p] : 1.0;
        double av[TI], bv[TJ];
#pragma unroll
        for (int i = 0; i < TI; ++i) av[i] = (i0 + i < ma) ? ag[(i0 + i) * n + p] : 0.0;
#pragma unroll
        for (int j = 0; j < TJ; ++j) bv[j] = SAME ? av[j] : ((j0 + j < mb) ? bg[(j0 + j) * n + p] : 0.0);
#pragma unroll
        for (int i = 0; i < TI; ++i) {
            const double wa = av[i] * w;
#pragma unroll
            for (int j = 0; j < TJ; ++j) acc[i][j] = fma(wa, bv[j], acc[i][j]);
        }
    }
    __shared__ double red[RT / 32][TI * TJ];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < TI; ++i)
#pragma unroll
        for (int j = 0; j < TJ; ++j) {
            double v = acc[i][j];
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
            if (lane == 0) red[warp][i * TJ + j] = v;
        }
    __syncthreads();
    if (threadIdx.x < TI * TJ) {
        double v = 0.0;
        for (int w = 0; w < RT / 32; ++w) v += red[w][threadIdx.x];
        partial[((static_cast<int64_t>(g) * gridDim.y + tile) * chunks + c) * (TI * TJ) + threadIdx.x] = v;
    }
}

// One warp per output entry: lanes take chunks lane, lane + 32, ... in order, then a fixed shuffle
// tree combines the lanes -- the same order on every run.
__global__ void cross_final_kernel(const double* __restrict__ partial, int ma, int mb, int ti, int tj, int tiles_j,
                                   int tiles, int chunks, int groups, double* __restrict__ out) {
    const int64_t idx = (blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int64_t total = static_cast<int64_t>(groups) * ma * mb;
    if (idx >= total) return;
    const int g = static_cast<int>(idx / (static_cast<int64_t>(ma) * mb));
    const int rem = static_cast<int>(idx % (static_cast<int64_t>(ma) * mb));
    const int i = rem / mb;
    const int j = rem % mb;
    const int tile = (i / ti) * tiles_j + (j / tj);
    const int slot = (i % ti) * tj + (j % tj);
    const double* src = partial + (static_cast<int64_t>(g) * tiles + tile) * chunks * (ti * tj) + slot;
    double v = 0.0;
    for (int c = lane; c < chunks; c += 32) v += src[static_cast<int64_t>(c) * ti * tj];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if (lane == 0) out[idx] = v;
}

}  // namespace

}  // namespace cdftb

using namespace cdftb;

extern "C" int64_t cdftb_measure_cross_scratch_bytes(int ma, int mb, int64_t n, int groups) {
    if (ma <= 0 || mb <= 0 || n <= 0 || groups <= 0) return 0;
    CrossShape s = cross_shape(ma, mb, n, groups);
    return static_cast<int64_t>(groups) * s.tiles_i * s.tiles_j * s.chunks * s.ti * s.tj * 8;
}

namespace cdftb {
namespace {
int launch_cross(const double* a, int ma, int64_t group_stride_a, const double* b, int mb, int64_t group_stride_b,
                 const double* q, int64_t q_group_stride, int64_t n, int groups, double* out, void* scratch,
                 int64_t scratch_bytes, cudaStream_t st) {
    if (!a || !b || !out || ma <= 0 || mb <= 0 || n <= 0 || groups <= 0 || groups > 65535) return CDFTB_ERR_ARGUMENT;
    CrossShape s = cross_shape(ma, mb, n, groups);
    const int64_t need = cdftb_measure_cross_scratch_bytes(ma, mb, n, groups);
    if (!scratch || scratch_bytes < need) return CDFTB_ERR_ARGUMENT;
    double* partial = static_cast<double*>(scratch);
    const int tiles = s.tiles_i * s.tiles_j;
    dim3 grid(s.chunks, tiles, groups);
    // the same rows on both sides (a Gram matrix): one load per element
    const bool same = a == b && ma == mb && group_stride_a == group_stride_b && s.tiles_i == 1 && s.tiles_j == 1;
#define CDFTB_CROSS_LAUNCH(TI_, TJ_, SAME_)                                                                 \
    cross_partial_kernel<TI_, TJ_, SAME_><<<grid, RT, 0, st>>>(a, ma, group_stride_a, b, mb, group_stride_b, q, \
                                                               q_group_stride, n, s.tiles_j, s.chunk, s.chunks,  \
                                                               partial)
    if (s.tiles_i * s.tiles_j > 1) {
        CDFTB_CROSS_LAUNCH(4, 4, false);
    } else {
        switch (s.ti) {
#define CDFTB_CROSS_WIDTH(T_)                        \
    case T_:                                         \
        if (same) CDFTB_CROSS_LAUNCH(T_, T_, true);  \
        else CDFTB_CROSS_LAUNCH(T_, T_, false);      \
        break;
            CDFTB_CROSS_WIDTH(1) CDFTB_CROSS_WIDTH(2) CDFTB_CROSS_WIDTH(3) CDFTB_CROSS_WIDTH(4) CDFTB_CROSS_WIDTH(5)
            CDFTB_CROSS_WIDTH(6)
#undef CDFTB_CROSS_WIDTH
            default: return CDFTB_ERR_ARGUMENT;
        }
    }
#undef CDFTB_CROSS_LAUNCH
    int rc = check_launch();
    if (rc != CDFTB_OK) return rc;
    const int64_t total = static_cast<int64_t>(groups) * ma * mb;
    cross_final_kernel<<<static_cast<unsigned>(ceil_div(total * 32, 256)), 256, 0, st>>>(partial, ma, mb, s.ti, s.tj,
                                                                                         s.tiles_j, tiles, s.chunks,
                                                                                         groups, out);
    return check_launch();
}
}  // namespace
}  // namespace cdftb

extern "C" int cdftb_measure_cross_f64(const double* a, int ma, int64_t group_stride_a, const double* b, int mb,
                                       int64_t group_stride_b, const double* q, int64_t n, int groups, double* out,
                                       void* scratch, int64_t scratch_bytes, cdftb_stream_t stream) {
    return launch_cross(a, ma, group_stride_a, b, mb, group_stride_b, q, 0, n, groups, out, scratch, scratch_bytes,
                        as_stream(stream));
}

extern "C" int cdftb_measure_cross_grouped_f64(const double* a, int ma, int64_t group_stride_a, const double* b, int mb,
                                               int64_t group_stride_b, const double* q, int64_t q_group_stride,
                                               int64_t n, int groups, double* out, void* scratch,
                                               int64_t scratch_bytes, cdftb_stream_t stream) {
    if (!q || q_group_stride < 0) return CDFTB_ERR_ARGUMENT;
    return launch_cross(a, ma, group_stride_a, b, mb, group_stride_b, q, q_group_stride, n, groups, out, scratch,
                        scratch_bytes, as_stream(stream));
}

// ---------------------------------------------------------------------------------------------
// cdftb_measure_cross_static_f64: the same product with its partials in a fixed device array of
// this library instead of caller scratch, for callers that cannot allocate device memory. The
// array lives once per device (each device's copy of this module). Its address is looked up with
// cudaGetSymbolAddress on the first call in each CUDA context and kept with that context's ID: a
// device reset destroys the primary context, the module is loaded again (possibly elsewhere), and
// the next call, seeing a new context ID, looks the address up again. The first pass writes every
// partial that the second pass reads, so nothing in the array has to start at zero. Two calls whose
// work overlaps on the GPU (other streams, other host threads) share the array and race.

namespace cdftb {
namespace {

constexpr int64_t kStaticCrossScratchBytes = int64_t(4) << 20;
constexpr int kMaxDevices = 64;

__device__ __align__(256) static unsigned char g_static_cross_scratch[kStaticCrossScratchBytes];

struct StaticScratchEntry {
    unsigned long long context_id = 0;  // 0: not looked up yet (CUDA context IDs start at 1)
    void* address = nullptr;
};
StaticScratchEntry g_static_cross[kMaxDevices];
std::mutex g_static_cross_mutex;

// The ID of the calling thread's current CUDA context, through the driver entry points the runtime
// hands out (no link against the driver library); 0 when there is none yet or the lookup failed.
unsigned long long current_context_id() {
    static PFN_cuCtxGetCurrent_v4000 get_current = nullptr;
    static PFN_cuCtxGetId_v12000 get_id = nullptr;
    if (!get_current || !get_id) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &p, 4000, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return 0;
        get_current = reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(p);
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &p, 12000, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return 0;
        get_id = reinterpret_cast<PFN_cuCtxGetId_v12000>(p);
    }
    CUcontext ctx = nullptr;
    if (get_current(&ctx) != CUDA_SUCCESS || !ctx) return 0;
    unsigned long long id = 0;
    if (get_id(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}

int static_cross_scratch(void** out) {
    int dev = -1;
    int rc = check(cudaGetDevice(&dev));
    if (rc != CDFTB_OK) return rc;
    if (dev < 0 || dev >= kMaxDevices) return CDFTB_ERR_CAPACITY;
    std::lock_guard<std::mutex> lock(g_static_cross_mutex);
    StaticScratchEntry& entry = g_static_cross[dev];
    unsigned long long id = current_context_id();
    if (id != 0 && id == entry.context_id) {
        *out = entry.address;
        return CDFTB_OK;
    }
    void* p = nullptr;
    rc = check(cudaGetSymbolAddress(&p, g_static_cross_scratch));  // makes the runtime's context current
    if (rc != CDFTB_OK) return rc;
    if (id == 0) id = current_context_id();
    entry.context_id = id;  // still 0 if the driver gave no ID: then the next call looks it up again
    entry.address = p;
    *out = p;
    return CDFTB_OK;
}

}  // namespace
}  // namespace cdftb

extern "C" int64_t cdftb_measure_cross_static_capacity_bytes(void) { return kStaticCrossScratchBytes; }

extern "C" int cdftb_measure_cross_static_f64(const double* a, int ma, int64_t group_stride_a, const double* b,
                                              int mb, int64_t group_stride_b, const double* q, int64_t n, int groups,
                                              double* out, cdftb_stream_t stream) {
    if (!a || !b || !out || ma <= 0 || mb <= 0 || n <= 0 || groups <= 0 || groups > 65535) return CDFTB_ERR_ARGUMENT;
    const int64_t need = cdftb_measure_cross_scratch_bytes(ma, mb, n, groups);
    if (need > kStaticCrossScratchBytes) return CDFTB_ERR_CAPACITY;
    void* scratch = nullptr;
    const int rc = static_cross_scratch(&scratch);
    if (rc != CDFTB_OK) return rc;
    return cdftb_measure_cross_f64(a, ma, group_stride_a, b, mb, group_stride_b, q, n, groups, out, scratch,
                                   kStaticCrossScratchBytes, stream);
}
