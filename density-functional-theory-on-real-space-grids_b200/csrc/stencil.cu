// (a) The staggered divergence-form apply and (b) the fused Chebyshev filter.
//
// One kernel serves every mode. A CTA owns a TY x TZ tile of (y, z) columns (z contiguous, one
// warp per z row) and a chunk of x planes, and marches along x: each x plane of the input, with a
// (2p-1)-point halo in y and z, is staged once in shared memory; the y- and z-direction parts of
// sum_d D_d^T[w_d D_d phi] are formed from it (faces in shared memory), and the x-direction part is
// carried in per-thread register queues of the last 2p planes of phi, x faces and y+z terms, so
// that every plane is read from memory once per CTA. The epilogue applies the mode: the raw
// divergence, the kinetic term 0.5 (h^3/omega) div, the full apply + V phi, or one step of the
// scaled Chebyshev recurrence (A y - c y) a - b y_prev with (c, a, b) read from a device table.
//
// Reference arithmetic: src/cdft/operators/divergence.py:99-197 (taps, face order, transpose),
// src/cdft/operators/hamiltonian.py:303-318 (epilogue), src/cdft/eigen/chefsi.py:81-160 (recurrence).

#include "common.cuh"

namespace cdftb {

namespace {

constexpr int TZ = 32;
constexpr int TY = 8;
constexpr int THREADS = TZ * TY;

enum Mode { MODE_DIV = 0, MODE_KINETIC = 1, MODE_APPLY = 2, MODE_CHEB_FIRST = 3, MODE_CHEB = 4 };

struct StencilArgs {
    const void* in;
    int in_dtype;
    const void* prev;
    int prev_dtype;
    void* out;
    int out_dtype;
    int64_t batch;
    int nx, ny, nz;
    const void* w0;
    const void* w1;
    const void* w2;
    const void* inv_w;
    const void* pot;
    int geo_dtype;
    int64_t pot_stride;
    int orb_per_group;
    const double* coef;
    int degree;
    int step;
    int mode;
    int xchunk;
    int tiles_z;
    double taps[8];
};

template <typename T, int P>
__global__ void __launch_bounds__(THREADS) stencil_kernel(const StencilArgs a) {
    constexpr int H = 2 * P - 1;  // halo reach of the composite stencil
    constexpr int K = 2 * P;      // taps per staggered derivative
    constexpr int PW = TZ + 2 * H;
    constexpr int PH = TY + 2 * H;
    __shared__ T s_phi[PH][PW];
    __shared__ T s_fy[TY + K - 1][TZ];
    __shared__ T s_fz[TY][TZ + K - 1];

    const int tz = threadIdx.x;
    const int ty = threadIdx.y;
    const int tid = ty * TZ + tz;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const int64_t n_points = static_cast<int64_t>(nx) * ny * nz;
    const int tile = blockIdx.x;
    const int y0 = (tile / a.tiles_z) * TY;
    const int z0 = (tile % a.tiles_z) * TZ;
    const int xa = blockIdx.y * a.xchunk;
    const int xe = min(xa + a.xchunk, nx) - 1;
    const int64_t b = blockIdx.z;
    const int y = y0 + ty;
    const int z = z0 + tz;
    const bool valid = (y < ny) && (z < nz);
    const int64_t base = b * n_points;

    T taps[K];
#pragma unroll
    for (int k = 0; k < K; ++k) taps[k] = static_cast<T>(a.taps[k]);

    T phiq[K], fq[K], yzq[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        phiq[k] = T(0);
        fq[k] = T(0);
        yzq[k] = T(0);
    }

    T c_coef = T(0), a_coef = T(0), b_coef = T(0);
    int64_t pot_base = 0;
    if (a.mode >= MODE_APPLY) {
        const int64_t group = b / a.orb_per_group;
        pot_base = group * a.pot_stride;
        if (a.mode >= MODE_CHEB_FIRST) {
            const double* row = a.coef + (group * a.degree + a.step) * 3;
            c_coef = static_cast<T>(row[0]);
            a_coef = static_cast<T>(row[1]);
            b_coef = static_cast<T>(row[2]);
        }
    }

    for (int q = xa - H; q <= xe + H; ++q) {
        __syncthreads();
        const bool plane_in = (q >= 0) && (q < nx);
        for (int idx = tid; idx < PH * PW; idx += THREADS) {
            const int r = idx / PW;
            const int c = idx - r * PW;
            const int gy = y0 - H + r;
            const int gz = z0 - H + c;
            T v = T(0);
            if (plane_in && gy >= 0 && gy < ny && gz >= 0 && gz < nz)
                v = load_as<T>(a.in, a.in_dtype, base + (static_cast<int64_t>(q) * ny + gy) * nz + gz);
            s_phi[r][c] = v;
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < K - 1; ++k) phiq[k] = phiq[k + 1];
        phiq[K - 1] = s_phi[ty + H][tz + H];

        const bool out_plane = (q >= xa) && (q <= xe);
        if (out_plane) {
            // y faces g = y0 - P + r, r in [0, TY + K - 1): node g + 1 + (k - P) is smem row r + k.
            for (int idx = tid; idx < (TY + K - 1) * TZ; idx += THREADS) {
                const int r = idx / TZ;
                const int c = idx - r * TZ;
                const int g = y0 - P + r;
                const int gz = z0 + c;
                T f = T(0);
                if (gz < nz && g >= -P && g <= ny + P - 1) {
                    T s = T(0);
#pragma unroll
                    for (int k = 0; k < K; ++k) s += taps[k] * s_phi[r + k][c + H];
                    f = load_as<T>(a.w1, a.geo_dtype, (static_cast<int64_t>(q) * (ny + K) + g + P) * nz + gz) * s;
                }
                s_fy[r][c] = f;
            }
            // z faces g = z0 - P + c: node is smem column c + k.
            for (int idx = tid; idx < TY * (TZ + K - 1); idx += THREADS) {
                const int r = idx / (TZ + K - 1);
                const int c = idx - r * (TZ + K - 1);
                const int g = z0 - P + c;
                const int gy = y0 + r;
                T f = T(0);
                if (gy < ny && g >= -P && g <= nz + P - 1) {
                    T s = T(0);
#pragma unroll
                    for (int k = 0; k < K; ++k) s += taps[k] * s_phi[r + H][c + k];
                    f = load_as<T>(a.w2, a.geo_dtype, (static_cast<int64_t>(q) * ny + gy) * (nz + K) + g + P) * s;
                }
                s_fz[r][c] = f;
            }
        }
        __syncthreads();
        T yz = T(0);
        if (out_plane) {
            T yt = T(0), zt = T(0);
#pragma unroll
            for (int k = 0; k < K; ++k) {
                yt += taps[k] * s_fy[ty + K - 1 - k][tz];
                zt += taps[k] * s_fz[ty][tz + K - 1 - k];
            }
            yz = yt + zt;
        }
#pragma unroll
        for (int k = 0; k < K - 1; ++k) yzq[k] = yzq[k + 1];
        yzq[K - 1] = yz;

        // x face f = q - P reads planes q - H .. q = phiq[0 .. K-1].
        T fx = T(0);
        const int f = q - P;
        if (q >= xa && valid && f <= nx + P - 1) {
            T s = T(0);
#pragma unroll
            for (int k = 0; k < K; ++k) s += taps[k] * phiq[k];
            fx = load_as<T>(a.w0, a.geo_dtype, (static_cast<int64_t>(f + P) * ny + y) * nz + z) * s;
        }
#pragma unroll
        for (int k = 0; k < K - 1; ++k) fq[k] = fq[k + 1];
        fq[K - 1] = fx;

        const int i = q - H;
        if (valid && i >= xa && i <= xe) {
            T xt = T(0);
#pragma unroll
            for (int k = 0; k < K; ++k) xt += taps[k] * fq[K - 1 - k];
            const T div = xt + yzq[0];
            const int64_t point = (static_cast<int64_t>(i) * ny + y) * nz + z;
            T result;
            if (a.mode == MODE_DIV) {
                result = div;
            } else {
                const T kin = (div * T(0.5)) * load_as<T>(a.inv_w, a.geo_dtype, point);
                if (a.mode == MODE_KINETIC) {
                    result = kin;
                } else {
                    const T phi = phiq[0];
                    const T applied = kin + phi * load_as<T>(a.pot, a.geo_dtype, pot_base + point);
                    if (a.mode == MODE_APPLY) {
                        result = applied;
                    } else {
                        result = (applied - c_coef * phi) * a_coef;
                        if (a.mode == MODE_CHEB) result -= b_coef * load_as<T>(a.prev, a.prev_dtype, base + point);
                    }
                }
            }
            store_as<T>(a.out, a.out_dtype, base + point, result);
        }
    }
}

int choose_xchunk(int nx, int64_t ctas_per_plane_set) {
    // Enough CTAs for about four per SM on 148 SMs; every chunk re-reads 2(2p-1) halo planes, so
    // chunks are not made shorter than 12 planes.
    const int64_t target = 4 * 148;
    int64_t chunks = ceil_div(target, ctas_per_plane_set);
    const int64_t max_chunks = ceil_div(nx, 12);
    if (chunks > max_chunks) chunks = max_chunks;
    if (chunks < 1) chunks = 1;
    return static_cast<int>(ceil_div(nx, chunks));
}

template <typename T>
int launch_typed(StencilArgs& a, int accuracy, cudaStream_t stream) {
    const int tiles_y = static_cast<int>(ceil_div(a.ny, TY));
    a.tiles_z = static_cast<int>(ceil_div(a.nz, TZ));
    const int64_t tiles = static_cast<int64_t>(tiles_y) * a.tiles_z;
    if (a.xchunk <= 0) a.xchunk = choose_xchunk(a.nx, tiles * a.batch);
    const int chunks = static_cast<int>(ceil_div(a.nx, a.xchunk));
    dim3 block(TZ, TY);
    for (int64_t first = 0; first < a.batch; first += 65535) {
        StencilArgs part = a;
        const int64_t count = (a.batch - first) < 65535 ? (a.batch - first) : 65535;
        const int64_t n_points = static_cast<int64_t>(a.nx) * a.ny * a.nz;
        // Offset the batch by advancing the pointers (types differ, so by bytes).
        auto adv = [&](const void* p, int dtype) -> const void* {
            return p ? static_cast<const char*>(p) + first * n_points * (dtype == CDFTB_F64 ? 8 : 4) : p;
        };
        part.in = adv(a.in, a.in_dtype);
        part.prev = adv(a.prev, a.prev_dtype);
        part.out = const_cast<void*>(adv(a.out, a.out_dtype));
        part.batch = count;
        if (first > 0 && a.mode >= MODE_APPLY) {
            // Re-base the group index: only valid when the split falls on a group boundary.
            if (first % a.orb_per_group != 0) return CDFTB_ERR_CAPACITY;
            const int64_t g0 = first / a.orb_per_group;
            part.pot = static_cast<const char*>(a.pot) + g0 * a.pot_stride * (a.geo_dtype == CDFTB_F64 ? 8 : 4);
            if (a.coef) part.coef = a.coef + g0 * a.degree * 3;
        }
        dim3 grid(static_cast<unsigned>(tiles), static_cast<unsigned>(chunks), static_cast<unsigned>(count));
        switch (accuracy) {
            case 2: stencil_kernel<T, 1><<<grid, block, 0, stream>>>(part); break;
            case 4: stencil_kernel<T, 2><<<grid, block, 0, stream>>>(part); break;
            case 6: stencil_kernel<T, 3><<<grid, block, 0, stream>>>(part); break;
            case 8: stencil_kernel<T, 4><<<grid, block, 0, stream>>>(part); break;
            default: return CDFTB_ERR_ARGUMENT;
        }
        int st = check_launch();
        if (st != CDFTB_OK) return st;
    }
    return CDFTB_OK;
}

int launch(StencilArgs& a, int accuracy, double spacing, int compute_dtype, cudaStream_t stream) {
    if (a.nx <= 0 || a.ny <= 0 || a.nz <= 0 || a.batch < 0 || !(spacing > 0.0)) return CDFTB_ERR_ARGUMENT;
    if (a.batch == 0) return CDFTB_OK;
    if (!a.in || !a.out || !a.w0 || !a.w1 || !a.w2) return CDFTB_ERR_ARGUMENT;
    if (a.mode >= MODE_KINETIC && !a.inv_w) return CDFTB_ERR_ARGUMENT;
    if (a.mode >= MODE_APPLY && (!a.pot || a.orb_per_group <= 0)) return CDFTB_ERR_ARGUMENT;
    if (a.mode >= MODE_CHEB_FIRST && !a.coef) return CDFTB_ERR_ARGUMENT;
    if (a.mode == MODE_CHEB && !a.prev) return CDFTB_ERR_ARGUMENT;
    StaggeredTaps t = staggered_taps(accuracy);
    if (t.half == 0) return CDFTB_ERR_ARGUMENT;
    // The reference multiplies each slice by (c_k * (1/h)) (divergence.py:112, 121).
    const double scale = 1.0 / spacing;
    for (int k = 0; k < 8; ++k) a.taps[k] = k < accuracy ? t.c[k] * scale : 0.0;
    if (compute_dtype == CDFTB_F64) return launch_typed<double>(a, accuracy, stream);
    if (compute_dtype == CDFTB_F32) return launch_typed<float>(a, accuracy, stream);
    return CDFTB_ERR_ARGUMENT;
}

StencilArgs args_from_operator(const cdftb_operator* op) {
    StencilArgs a{};
    a.nx = op->nx;
    a.ny = op->ny;
    a.nz = op->nz;
    a.w0 = op->face_weights[0];
    a.w1 = op->face_weights[1];
    a.w2 = op->face_weights[2];
    a.inv_w = op->inverse_weight;
    a.pot = op->potential;
    a.geo_dtype = op->dtype;
    a.pot_stride = op->potential_stride;
    a.orb_per_group = op->orbitals_per_group;
    return a;
}

}  // namespace

}  // namespace cdftb

using namespace cdftb;

extern "C" int cdftb_weighted_divergence_f64(const double* box, double* out, int64_t batch, int nx, int ny, int nz,
                                             const double* w0, const double* w1, const double* w2, double spacing,
                                             int accuracy, cdftb_stream_t stream) {
    StencilArgs a{};
    a.in = box;
    a.in_dtype = CDFTB_F64;
    a.out = out;
    a.out_dtype = CDFTB_F64;
    a.batch = batch;
    a.nx = nx;
    a.ny = ny;
    a.nz = nz;
    a.w0 = w0;
    a.w1 = w1;
    a.w2 = w2;
    a.geo_dtype = CDFTB_F64;
    a.mode = MODE_DIV;
    a.orb_per_group = 1;
    return launch(a, accuracy, spacing, CDFTB_F64, as_stream(stream));
}

extern "C" int cdftb_cusp_apply(const cdftb_operator* op, const void* phi, int in_dtype, void* out, int out_dtype,
                                int64_t batch, int kinetic_only, cdftb_stream_t stream) {
    if (!op) return CDFTB_ERR_ARGUMENT;
    StencilArgs a = args_from_operator(op);
    a.in = phi;
    a.in_dtype = in_dtype;
    a.out = out;
    a.out_dtype = out_dtype;
    a.batch = batch;
    a.mode = kinetic_only ? MODE_KINETIC : MODE_APPLY;
    return launch(a, op->accuracy, op->spacing, op->dtype, as_stream(stream));
}

extern "C" int cdftb_chebyshev_filter(const cdftb_operator* op, const void* block, int in_dtype, void* out,
                                      int out_dtype, void* work, int64_t batch, const double* coefficients,
                                      int degree, cdftb_stream_t stream) {
    if (!op || !block || !out || !work || !coefficients || degree < 1) return CDFTB_ERR_ARGUMENT;
    const int64_t n_points = static_cast<int64_t>(op->nx) * op->ny * op->nz;
    const int esize = op->dtype == CDFTB_F64 ? 8 : 4;
    // Step k (1-based) writes buffer (degree - k) mod 3: buffer 0 is `out`, so the last step lands
    // there, and three consecutive steps never share a buffer.
    void* bufs[3] = {out, work, static_cast<char*>(work) + batch * n_points * esize};
    const int dts[3] = {out_dtype, op->dtype, op->dtype};
    const void* y = block;
    int y_dt = in_dtype;
    const void* prev = nullptr;
    int prev_dt = in_dtype;
    for (int k = 1; k <= degree; ++k) {
        const int target = (degree - k) % 3;
        StencilArgs a = args_from_operator(op);
        a.in = y;
        a.in_dtype = y_dt;
        a.prev = prev;
        a.prev_dtype = prev_dt;
        a.out = bufs[target];
        a.out_dtype = dts[target];
        a.batch = batch;
        a.coef = coefficients;
        a.degree = degree;
        a.step = k - 1;
        a.mode = (k == 1) ? MODE_CHEB_FIRST : MODE_CHEB;
        int st = launch(a, op->accuracy, op->spacing, op->dtype, as_stream(stream));
        if (st != CDFTB_OK) return st;
        prev = y;
        prev_dt = y_dt;
        y = bufs[target];
        y_dt = dts[target];
    }
    return CDFTB_OK;
}
