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

__device__ __forceinline__ void cp_async(void* smem_dst, const void* gmem_src, bool pred, int bytes) {
    const unsigned dst = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
    const int src_size = pred ? bytes : 0;  // src-size 0 zero-fills the destination
    if (bytes == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(dst), "l"(gmem_src), "r"(src_size));
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(dst), "l"(gmem_src), "r"(src_size));
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }

template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

template <typename T, int P, int TYV>
struct StencilLayout {
    static constexpr int H = 2 * P - 1;
    static constexpr int K = 2 * P;
    static constexpr int PW = TZ + 2 * H;
    static constexpr int PH = TYV + 2 * H;
    static constexpr int NPHI = PH * PW;
    static constexpr int NW1 = (TYV + K - 1) * TZ;
    static constexpr int NW2 = TYV * (TZ + K - 1);
    static constexpr int NT = TYV * TZ;
    // stage: phi | w1 | w2 | w0 | inv | pot | prev
    static constexpr int OFF_W1 = NPHI;
    static constexpr int OFF_W2 = OFF_W1 + NW1;
    static constexpr int OFF_W0 = OFF_W2 + NW2;
    static constexpr int OFF_INV = OFF_W0 + NT;
    static constexpr int OFF_POT = OFF_INV + NT;
    static constexpr int OFF_PREV = OFF_POT + NT;
    static constexpr int STAGE = OFF_PREV + NT;
    static constexpr int NS = 3;
    static constexpr int OFF_FY = NS * STAGE;
    static constexpr int OFF_FZ = OFF_FY + NW1;
    static constexpr int TOTAL = OFF_FZ + NW2;
    static constexpr size_t BYTES = sizeof(T) * TOTAL;
};

// Everything a thread copies or reads per x plane is at a fixed position relative to the plane
// (only the plane index changes as the CTA marches), so the in-plane offsets, their validity and
// the shared-memory positions are worked out once per thread; a plane then costs one multiply-add
// and one asynchronous copy per element. Out-of-range elements are zero-filled by the copy itself
// (the Dirichlet halo, and faces that do not exist).
template <typename T, int P, int TYV>
struct ThreadPlan {
    using L = StencilLayout<T, P, TYV>;
    static constexpr int THR = TZ * TYV;
    static constexpr int IT_PHI = (L::NPHI + THR - 1) / THR;
    static constexpr int IT_W1 = (L::NW1 + THR - 1) / THR;
    static constexpr int IT_W2 = (L::NW2 + THR - 1) / THR;
    int phi_off[IT_PHI];
    int w1_off[IT_W1];
    int w2_off[IT_W2];
    int own_off;          // y * nz + z of the thread's own column
    unsigned phi_ok;      // bit k: element k lies in the grid (y, z)
    unsigned w1_ok, w2_ok;
    bool own_ok;
    int fy_src[IT_W1];    // smem index of the first tap of each y face this thread forms
    int fz_src[IT_W2];
};

template <typename T, int P, int TYV>
__device__ __forceinline__ void make_plan(ThreadPlan<T, P, TYV>& pl, int y0, int z0, int ny, int nz, int tid, int ty,
                                          int tz) {
    using L = StencilLayout<T, P, TYV>;
    using PL = ThreadPlan<T, P, TYV>;
    constexpr int H = L::H, K = L::K, PW = L::PW, THR = PL::THR;
    pl.phi_ok = pl.w1_ok = pl.w2_ok = 0u;
#pragma unroll
    for (int k = 0; k < PL::IT_PHI; ++k) {
        const int idx = tid + k * THR;
        const int r = idx / PW;
        const int c = idx - r * PW;
        const int gy = y0 - H + r;
        const int gz = z0 - H + c;
        const bool ok = idx < L::NPHI && gy >= 0 && gy < ny && gz >= 0 && gz < nz;
        pl.phi_off[k] = ok ? gy * nz + gz : 0;
        if (ok) pl.phi_ok |= 1u << k;
    }
#pragma unroll
    for (int k = 0; k < PL::IT_W1; ++k) {
        const int idx = tid + k * THR;
        const int r = idx / TZ;
        const int c = idx - r * TZ;
        const int g = y0 - P + r;
        const int gz = z0 + c;
        const bool ok = idx < L::NW1 && gz < nz && g >= -P && g <= ny + P - 1;
        pl.w1_off[k] = ok ? (g + P) * nz + gz : 0;
        if (ok) pl.w1_ok |= 1u << k;
        pl.fy_src[k] = r * PW + c + H;
    }
#pragma unroll
    for (int k = 0; k < PL::IT_W2; ++k) {
        const int idx = tid + k * THR;
        const int r = idx / (TZ + K - 1);
        const int c = idx - r * (TZ + K - 1);
        const int g = z0 - P + c;
        const int gy = y0 + r;
        const bool ok = idx < L::NW2 && gy < ny && g >= -P && g <= nz + P - 1;
        pl.w2_off[k] = ok ? gy * (nz + K) + g + P : 0;
        if (ok) pl.w2_ok |= 1u << k;
        pl.fz_src[k] = (r + H) * PW + c;
    }
    const int y = y0 + ty, z = z0 + tz;
    pl.own_ok = y < ny && z < nz;
    pl.own_off = pl.own_ok ? y * nz + z : 0;
}

template <typename T, int P, int TYV>
__device__ __forceinline__ void stage_loads(const StencilArgs& a, const ThreadPlan<T, P, TYV>& pl, T* st, int q, int xa,
                                            int xe, int64_t base, int64_t pot_base, int tid) {
    using L = StencilLayout<T, P, TYV>;
    using PL = ThreadPlan<T, P, TYV>;
    constexpr int H = L::H, K = L::K, THR = PL::THR;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const int64_t plane = static_cast<int64_t>(ny) * nz;
    const T* in = static_cast<const T*>(a.in);
    const bool plane_in = (q >= 0) && (q < nx);
    const T* in_q = in + base + (plane_in ? q * plane : 0);
#pragma unroll
    for (int k = 0; k < PL::IT_PHI; ++k) {
        const int idx = tid + k * THR;
        if (k == PL::IT_PHI - 1 && idx >= L::NPHI) break;
        const bool ok = plane_in && ((pl.phi_ok >> k) & 1u);
        cp_async(st + idx, in_q + pl.phi_off[k], ok, sizeof(T));
    }
    if (q >= xa && q <= xe) {
        const T* w1q = static_cast<const T*>(a.w1) + q * static_cast<int64_t>(ny + K) * nz;
        const T* w2q = static_cast<const T*>(a.w2) + q * static_cast<int64_t>(ny) * (nz + K);
#pragma unroll
        for (int k = 0; k < PL::IT_W1; ++k) {
            const int idx = tid + k * THR;
            if (k == PL::IT_W1 - 1 && idx >= L::NW1) break;
            cp_async(st + L::OFF_W1 + idx, w1q + pl.w1_off[k], (pl.w1_ok >> k) & 1u, sizeof(T));
        }
#pragma unroll
        for (int k = 0; k < PL::IT_W2; ++k) {
            const int idx = tid + k * THR;
            if (k == PL::IT_W2 - 1 && idx >= L::NW2) break;
            cp_async(st + L::OFF_W2 + idx, w2q + pl.w2_off[k], (pl.w2_ok >> k) & 1u, sizeof(T));
        }
    }
    const int f = q - P;
    if (q >= xa && f <= nx + P - 1) {
        const T* w0 = static_cast<const T*>(a.w0) + static_cast<int64_t>(f + P) * plane;
        cp_async(st + L::OFF_W0 + tid, w0 + pl.own_off, pl.own_ok, sizeof(T));
    }
    const int i = q - H;
    if (i >= xa && i <= xe && a.mode >= MODE_KINETIC) {
        const int64_t point = i * plane + pl.own_off;
        cp_async(st + L::OFF_INV + tid, static_cast<const T*>(a.inv_w) + point, pl.own_ok, sizeof(T));
        if (a.mode >= MODE_APPLY)
            cp_async(st + L::OFF_POT + tid, static_cast<const T*>(a.pot) + pot_base + point, pl.own_ok, sizeof(T));
        if (a.mode == MODE_CHEB)
            cp_async(st + L::OFF_PREV + tid, static_cast<const T*>(a.prev) + base + point, pl.own_ok, sizeof(T));
    }
}

template <typename T, int P, int TYV>
__global__ void __launch_bounds__(TZ* TYV) stencil_kernel(const StencilArgs a) {
    using L = StencilLayout<T, P, TYV>;
    using PL = ThreadPlan<T, P, TYV>;
    constexpr int H = L::H;
    constexpr int K = L::K;
    constexpr int PW = L::PW;
    constexpr int NS = L::NS;
    constexpr int THR = TZ * TYV;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* smem = reinterpret_cast<T*>(smem_raw);
    T* s_fy = smem + L::OFF_FY;
    T* s_fz = smem + L::OFF_FZ;

    const int tz = threadIdx.x;
    const int ty = threadIdx.y;
    const int tid = ty * TZ + tz;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const int64_t n_points = static_cast<int64_t>(nx) * ny * nz;
    const int tile = blockIdx.x;
    const int y0 = (tile / a.tiles_z) * TYV;
    const int z0 = (tile % a.tiles_z) * TZ;
    const int xa = blockIdx.y * a.xchunk;
    const int xe = min(xa + a.xchunk, nx) - 1;
    const int64_t b = blockIdx.z;
    const int64_t base = b * n_points;

    ThreadPlan<T, P, TYV> pl;
    make_plan<T, P, TYV>(pl, y0, z0, ny, nz, tid, ty, tz);
    const bool valid = pl.own_ok;

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

    const int q_first = xa - H;
    const int q_last = xe + H;
#pragma unroll
    for (int s = 0; s < NS - 1; ++s) {
        const int q = q_first + s;
        if (q <= q_last) stage_loads<T, P, TYV>(a, pl, smem + s * L::STAGE, q, xa, xe, base, pot_base, tid);
        cp_async_commit();
    }

    int stage = 0;
    for (int q = q_first; q <= q_last; ++q) {
        {
            const int qn = q + NS - 1;
            int ns = stage + NS - 1;
            if (ns >= NS) ns -= NS;
            if (qn <= q_last) stage_loads<T, P, TYV>(a, pl, smem + ns * L::STAGE, qn, xa, xe, base, pot_base, tid);
            cp_async_commit();
        }
        cp_async_wait<NS - 1>();
        __syncthreads();
        const T* st = smem + stage * L::STAGE;
        const T* s_phi = st;

#pragma unroll
        for (int k = 0; k < K - 1; ++k) phiq[k] = phiq[k + 1];
        phiq[K - 1] = s_phi[(ty + H) * PW + tz + H];

        const int f = q - P;
        const int i = q - H;
        const bool out_plane = (q >= xa) && (q <= xe);
        const T w0v = st[L::OFF_W0 + tid];
        const T invv = st[L::OFF_INV + tid];
        const T potv = st[L::OFF_POT + tid];
        const T prevv = st[L::OFF_PREV + tid];
        if (out_plane) {
            const T* w1s = st + L::OFF_W1;
            const T* w2s = st + L::OFF_W2;
#pragma unroll
            for (int k = 0; k < PL::IT_W1; ++k) {
                const int idx = tid + k * THR;
                if (k == PL::IT_W1 - 1 && idx >= L::NW1) break;
                const T* src = s_phi + pl.fy_src[k];
                T sum = T(0);
#pragma unroll
                for (int t = 0; t < K; ++t) sum += taps[t] * src[t * PW];
                s_fy[idx] = w1s[idx] * sum;
            }
#pragma unroll
            for (int k = 0; k < PL::IT_W2; ++k) {
                const int idx = tid + k * THR;
                if (k == PL::IT_W2 - 1 && idx >= L::NW2) break;
                const T* src = s_phi + pl.fz_src[k];
                T sum = T(0);
#pragma unroll
                for (int t = 0; t < K; ++t) sum += taps[t] * src[t];
                s_fz[idx] = w2s[idx] * sum;
            }
        }
        __syncthreads();
        T yz = T(0);
        if (out_plane) {
            T yt = T(0), zt = T(0);
#pragma unroll
            for (int k = 0; k < K; ++k) {
                yt += taps[k] * s_fy[(ty + K - 1 - k) * TZ + tz];
                zt += taps[k] * s_fz[ty * (TZ + K - 1) + tz + K - 1 - k];
            }
            yz = yt + zt;
        }
#pragma unroll
        for (int k = 0; k < K - 1; ++k) yzq[k] = yzq[k + 1];
        yzq[K - 1] = yz;

        T fx = T(0);
        if (q >= xa && valid && f <= nx + P - 1) {
            T sum = T(0);
#pragma unroll
            for (int k = 0; k < K; ++k) sum += taps[k] * phiq[k];
            fx = w0v * sum;
        }
#pragma unroll
        for (int k = 0; k < K - 1; ++k) fq[k] = fq[k + 1];
        fq[K - 1] = fx;

        if (valid && i >= xa && i <= xe) {
            T xt = T(0);
#pragma unroll
            for (int k = 0; k < K; ++k) xt += taps[k] * fq[K - 1 - k];
            const T div = xt + yzq[0];
            const int64_t point = static_cast<int64_t>(i) * ny * nz + pl.own_off;
            T result;
            if (a.mode == MODE_DIV) {
                result = div;
            } else {
                const T kin = (div * T(0.5)) * invv;
                if (a.mode == MODE_KINETIC) {
                    result = kin;
                } else {
                    const T phi = phiq[0];
                    const T applied = kin + phi * potv;
                    if (a.mode == MODE_APPLY) {
                        result = applied;
                    } else {
                        result = (applied - c_coef * phi) * a_coef;
                        if (a.mode == MODE_CHEB) result -= b_coef * prevv;
                    }
                }
            }
            store_as<T>(a.out, a.out_dtype, base + point, result);
        }
        stage = (stage + 1 == NS) ? 0 : stage + 1;
    }
    cp_async_wait<0>();
}

// Slab tile shape, process-wide: TY rows of 32 z-columns per CTA, and the shortest x chunk. Set by
// cdftb_stencil_set_tile (the host autotuner); 8 and 12 until then.
int g_tile_ty = 8;
int g_min_chunk = 12;
int g_target_ctas_per_sm = 4;

int choose_xchunk(int nx, int64_t ctas_per_plane_set) {
    // Enough CTAs for a few per SM on 148 SMs; every chunk re-reads 2(2p-1) halo planes, so chunks
    // are not made shorter than g_min_chunk planes.
    const int64_t target = static_cast<int64_t>(g_target_ctas_per_sm) * 148;
    int64_t chunks = ceil_div(target, ctas_per_plane_set);
    const int64_t max_chunks = ceil_div(nx, g_min_chunk);
    if (chunks > max_chunks) chunks = max_chunks;
    if (chunks < 1) chunks = 1;
    return static_cast<int>(ceil_div(nx, chunks));
}

template <typename T, int P, int TYV>
int launch_one(const StencilArgs& part, dim3 grid, cudaStream_t stream) {
    using L = StencilLayout<T, P, TYV>;
    static bool configured = false;  // one attribute call per instantiation and process
    if (!configured) {
        int st = check(cudaFuncSetAttribute(stencil_kernel<T, P, TYV>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            static_cast<int>(L::BYTES)));
        if (st != CDFTB_OK) return st;
        configured = true;
    }
    stencil_kernel<T, P, TYV><<<grid, dim3(TZ, TYV), L::BYTES, stream>>>(part);
    return check_launch();
}

template <typename T, int TYV>
int launch_typed_ty(StencilArgs& a, int accuracy, cudaStream_t stream) {
    const int tiles_y = static_cast<int>(ceil_div(a.ny, TYV));
    a.tiles_z = static_cast<int>(ceil_div(a.nz, TZ));
    const int64_t tiles = static_cast<int64_t>(tiles_y) * a.tiles_z;
    if (a.xchunk <= 0) a.xchunk = choose_xchunk(a.nx, tiles * a.batch);
    const int chunks = static_cast<int>(ceil_div(a.nx, a.xchunk));
    const int64_t n_points = static_cast<int64_t>(a.nx) * a.ny * a.nz;
    for (int64_t first = 0; first < a.batch; first += 65535) {
        StencilArgs part = a;
        const int64_t count = (a.batch - first) < 65535 ? (a.batch - first) : 65535;
        auto adv = [&](const void* p, int dtype) -> const void* {
            return p ? static_cast<const char*>(p) + first * n_points * (dtype == CDFTB_F64 ? 8 : 4) : p;
        };
        part.in = adv(a.in, a.in_dtype);
        part.prev = adv(a.prev, a.prev_dtype);
        part.out = const_cast<void*>(adv(a.out, a.out_dtype));
        part.batch = count;
        if (first > 0 && a.mode >= MODE_APPLY) {
            if (first % a.orb_per_group != 0) return CDFTB_ERR_CAPACITY;
            const int64_t g0 = first / a.orb_per_group;
            part.pot = static_cast<const char*>(a.pot) + g0 * a.pot_stride * (a.geo_dtype == CDFTB_F64 ? 8 : 4);
            if (a.coef) part.coef = a.coef + g0 * a.degree * 3;
        }
        dim3 grid(static_cast<unsigned>(tiles), static_cast<unsigned>(chunks), static_cast<unsigned>(count));
        int st;
        switch (accuracy) {
            case 2: st = launch_one<T, 1, TYV>(part, grid, stream); break;
            case 4: st = launch_one<T, 2, TYV>(part, grid, stream); break;
            case 6: st = launch_one<T, 3, TYV>(part, grid, stream); break;
            case 8: st = launch_one<T, 4, TYV>(part, grid, stream); break;
            default: return CDFTB_ERR_ARGUMENT;
        }
        if (st != CDFTB_OK) return st;
    }
    return CDFTB_OK;
}

template <typename T>
int launch_typed(StencilArgs& a, int accuracy, cudaStream_t stream) {
    switch (g_tile_ty) {
        case 4: return launch_typed_ty<T, 4>(a, accuracy, stream);
        case 16: return launch_typed_ty<T, 16>(a, accuracy, stream);
        default: return launch_typed_ty<T, 8>(a, accuracy, stream);
    }
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
    // The staged copies move raw elements: inputs, the previous iterate and the geometry must be
    // in the arithmetic type; only the output may differ.
    if (a.in_dtype != compute_dtype || a.geo_dtype != compute_dtype) return CDFTB_ERR_ARGUMENT;
    if (a.mode == MODE_CHEB && a.prev_dtype != compute_dtype) return CDFTB_ERR_ARGUMENT;
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

extern "C" int cdftb_stencil_set_tile(int tile_y, int min_chunk, int ctas_per_sm) {
    if (tile_y != 4 && tile_y != 8 && tile_y != 16) return CDFTB_ERR_ARGUMENT;
    if (min_chunk < 1 || ctas_per_sm < 1) return CDFTB_ERR_ARGUMENT;
    g_tile_ty = tile_y;
    g_min_chunk = min_chunk;
    g_target_ctas_per_sm = ctas_per_sm;
    return CDFTB_OK;
}

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

// The apply for any order on the caller's layout: one stencil_kernel launch.
int cdftb::generic_cusp_apply(const cdftb_operator* op, const void* phi, int in_dtype, void* out, int out_dtype,
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

// The filter for any order on the caller's layout: each step one stencil_kernel launch. Used for
// the orders the slab filter (filter.cu) does not take; work holds 3 * batch * N elements.
int cdftb::generic_chebyshev_filter(const cdftb_operator* op, const void* block, int in_dtype, void* out,
                                    int out_dtype, void* work, int64_t batch, const double* coefficients, int degree,
                                    cdftb_stream_t stream) {
    const int64_t n_points = static_cast<int64_t>(op->nx) * op->ny * op->nz;
    const int esize = op->dtype == CDFTB_F64 ? 8 : 4;
    const int dt = op->dtype;
    char* w = static_cast<char*>(work);
    void* buf_a = w;
    void* buf_b = w + batch * n_points * esize;
    const void* x = block;
    if (in_dtype != dt) {
        // The float filter of the mixed form reads the double block once, as a cast copy.
        void* xc = w + 2 * batch * n_points * esize;
        int st = cdftb_cast(block, in_dtype, xc, dt, batch * n_points, stream);
        if (st != CDFTB_OK) return st;
        x = xc;
    }
    // Y_1 -> A, Y_2 -> B, then each Y_{k+1} overwrites Y_{k-1} in place (a point's previous value is
    // read only by the thread writing that point); the last step writes `out` in out_dtype.
    const void* y = x;
    const void* prev = nullptr;
    for (int k = 1; k <= degree; ++k) {
        void* target = (k == degree) ? out : ((k % 2 == 1) ? buf_a : buf_b);
        StencilArgs a = args_from_operator(op);
        a.in = y;
        a.in_dtype = dt;
        a.prev = prev;
        a.prev_dtype = dt;
        a.out = target;
        a.out_dtype = (k == degree) ? out_dtype : dt;
        a.batch = batch;
        a.coef = coefficients;
        a.degree = degree;
        a.step = k - 1;
        a.mode = (k == 1) ? MODE_CHEB_FIRST : MODE_CHEB;
        int st = launch(a, op->accuracy, op->spacing, dt, as_stream(stream));
        if (st != CDFTB_OK) return st;
        prev = y;
        y = target;
    }
    return CDFTB_OK;
}
