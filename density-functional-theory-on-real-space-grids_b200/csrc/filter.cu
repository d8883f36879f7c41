// (b) The fused Chebyshev filter on slabs: every step of the scaled three-term recurrence
// (src/cdft/eigen/chefsi.py:81-160) is one launch of slab_filter_kernel, which applies the
// order-8 staggered divergence-form operator (src/cdft/operators/divergence.py:99-197, epilogue of
// src/cdft/operators/hamiltonian.py:303-318) and the recurrence update in one pass.
//
// Layout in HBM. The filter keeps its iterates in an internal layout: "lanes", each lane
// (nx, ny, nzp) with nzp = nz rounded up to even and the padding column held at zero. This kernel
// takes 8-byte lane points: in float32 a lane interleaves two orbitals (a float2 per point, so that
// the packed f32x2 FMA of sm_100 does two orbitals per instruction); in float64 a lane is one
// orbital. slab_filter_wide_kernel (below) takes 16-byte points -- four float32 or two float64
// orbitals -- and serves every call with one shared geometry. The block is packed into
// this layout once per filter call and the last step writes the caller's layout. The geometry (face
// weights, h^3/omega, potentials) is copied once per call into rows padded to 16 bytes so that TMA
// can read it.
//
// Kernel. A CTA owns a tile of 8 rows (y) x TZ columns (z) of one lane and marches along x over a
// chunk of planes. Its warps have three roles, coupled by mbarrier rings in shared memory:
//   producer (1 warp)   per plane, TMA copies of: the plane of phi with a 7-point halo in y and z
//                       (zero outside the grid: the Dirichlet boundary), the previous iterate, and
//                       the plane's face weights, h^3/omega and potential(s), into one of R slots;
//   pass groups (2)     per plane (groups alternate), the y- and z-direction parts of
//                       sum_d D_d^T[w_d D_d phi]: one thread per line segment of 8 outputs, a
//                       column (22 nodes -> 15 y faces -> 8 outputs in registers) or a row segment
//                       (the same along z), all on one code path, into one of RY result slots;
//   march (8 or 9)      one thread per (y, z) column: queues of the last 8 planes of phi, x faces and
//                       y+z parts in registers (slot = plane mod 8: the loop is unrolled by 8, so
//                       no register moves), the output of node i formed at plane i + 7 with the
//                       recurrence epilogue, stored with coalesced 8-byte writes.
// Every mbarrier wait is bounded: after kWaitLimitNs (or when another CTA has given up) the warp
// records the failure in g_device_error (read by cdftb_device_status) and leaves the kernel.

#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>
#include <map>
#include <mutex>
#include <tuple>

#include "common.cuh"

namespace cdftb {

__device__ int g_device_error = 0;
// The launch (by its token) whose CTAs must give up: a CTA that timed out writes its launch's token,
// so the other CTAs of that launch stop waiting, while later launches are unaffected.
__device__ unsigned g_abort_token = 0;

namespace {

constexpr int TY = 8;
constexpr int HALO = 7;
constexpr int NROW = TY + 2 * HALO;
constexpr int R = 6;      // plane slots in flight
constexpr int RY = 4;     // y+z result slots (a power of 2)
static_assert((RY & (RY - 1)) == 0, "result slots are a power of 2");
constexpr int NG = 2;     // pass warp groups; planes alternate between them
constexpr unsigned long long kWaitLimitNs = 2000000000ull;  // 2 s
static_assert(R % NG == 0 && RY % NG == 0, "a slot is always served by the same pass group");
constexpr unsigned kNapNs = 256;        // longest sleep between tries of the wide kernel's producer and pass groups

constexpr size_t align128(size_t b) { return (b + 127) / 128 * 128; }

template <int TZ, int SB>  // SB: bytes of a geometry element (4 or 8)
struct Shape {
    static constexpr int MW = TY * TZ / 32;  // march warps
    // pass items of a plane: TZ columns (y) and TY rows x NZS segments of 8 (z); the last z segment
    // is moved left to end at TZ (it then stores only the outputs the previous one did not)
    static constexpr int NZS = (TZ + 7) / 8;
    static constexpr int ITEMS = TZ + TY * NZS;
    static constexpr int PWG = (ITEMS + 31) / 32;  // pass warps per group
    static constexpr int PW = NG * PWG;            // pass warps
    static constexpr int WARPS = MW + PW + 1;
    static constexpr int T = WARPS * 32;
    static constexpr int BW = TZ + 18;  // phi box width: z0-8 .. z0+TZ+9 (16-byte rows, bank-shifted)
    static constexpr int ZROW = TZ + 2;
    // bytes each TMA box delivers
    static constexpr unsigned TX_PHI = NROW * BW * 8;
    static constexpr unsigned TX_PREV = TY * TZ * 8;
    static constexpr unsigned TX_W0 = TY * TZ * SB;
    static constexpr unsigned TX_W1 = (TY + 7) * TZ * SB;
    static constexpr unsigned TX_W2 = TY * (TZ + 8) * SB;
    static constexpr unsigned TX_INV = TY * TZ * SB;
    static constexpr unsigned TX_POT = TY * TZ * SB;
    // slot layout, every region 128-byte aligned
    static constexpr size_t O_PHI = 0;
    static constexpr size_t O_PREV = O_PHI + align128(TX_PHI);
    static constexpr size_t O_W0 = O_PREV + align128(TX_PREV);
    static constexpr size_t O_W1 = O_W0 + align128(TX_W0);
    static constexpr size_t O_W2 = O_W1 + align128(TX_W1);
    static constexpr size_t O_INV = O_W2 + align128(TX_W2);
    static constexpr size_t O_POT0 = O_INV + align128(TX_INV);
    static constexpr size_t O_POT1 = O_POT0 + align128(TX_POT);
    static constexpr size_t SLOT = O_POT1 + align128(TX_POT);
    static constexpr size_t O_YZ = R * SLOT;
    static constexpr size_t YZ_Z = size_t(TY) * TZ * 8;  // Z part after the Y part
    static constexpr size_t YZ_SLOT = align128(YZ_Z + size_t(TY) * ZROW * 8);
    static constexpr size_t O_BAR = O_YZ + RY * YZ_SLOT;
    static constexpr size_t BYTES = O_BAR + (2 * R + 2 * RY) * 8;
    static_assert(TY * TZ % 32 == 0, "march warps cover the tile");
    static_assert(TZ >= 8 && TZ % 2 == 0, "z segments of 8 inside the tile");
    static_assert((TZ - 8) + 22 <= BW - 1, "the last z segment's nodes lie inside the phi box");
    static_assert(BYTES <= 232448, "fits the opt-in shared memory of one CTA");
};

// Element arithmetic: a float2 lane (two orbitals, packed f32x2 instructions) or a double lane.
struct LaneF2 {
    using E = float2;
    using S = float;
    static __device__ __forceinline__ E fma(E a, E b, E c) { return __ffma2_rn(a, b, c); }
    static __device__ __forceinline__ E mul(E a, E b) { return __fmul2_rn(a, b); }
    static __device__ __forceinline__ E add(E a, E b) { return __fadd2_rn(a, b); }
    static __device__ __forceinline__ E neg(E a) { return make_float2(-a.x, -a.y); }
    static __device__ __forceinline__ E splat(S s) { return make_float2(s, s); }
    static __device__ __forceinline__ E zero() { return make_float2(0.f, 0.f); }
    static constexpr int ORBITALS = 2;
    static constexpr bool WIDE = false;
    static constexpr CUtensorMapDataType GEO_TYPE = CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
};

struct LaneD {
    using E = double;
    using S = double;
    static __device__ __forceinline__ E fma(E a, E b, E c) { return ::fma(a, b, c); }
    static __device__ __forceinline__ E mul(E a, E b) { return a * b; }
    static __device__ __forceinline__ E add(E a, E b) { return a + b; }
    static __device__ __forceinline__ E neg(E a) { return -a; }
    static __device__ __forceinline__ E splat(S s) { return s; }
    static __device__ __forceinline__ E zero() { return 0.0; }
    static constexpr int ORBITALS = 1;
    static constexpr bool WIDE = false;
    static constexpr CUtensorMapDataType GEO_TYPE = CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
};

struct FilterArgs {
    int nx, ny, nz, nzp;
    int tiles_z;
    int xchunk;
    int has_prev;
    int final_out;
    void* out;
    int out_dtype;
    int64_t batch;
    int64_t lane_first;  // first lane of this launch (launches are split at 65535 lanes)
    int orb_per_group;
    int shared_potential;  // one potential for every orbital
    unsigned token;        // this launch's abort token (never 0)
    int apply_only;        // out = A phi (no recurrence; coef unused)
    int per_system_geometry;  // face weights and h^3/omega per orbital group (systems on their own grids)
    const int* system_shapes;  // with per_system_geometry: each group's own grid (nx, ny, nz), or null
    int lanes_per_group;      // > 0: lanes aligned to orbital groups (lane l holds group l / lanes_per_group)
    int kinetic_only;      // with apply_only: out = 0.5 (h^3/omega) div phi (no potential)
    int stop_after_planes;  // > 0 only in the timeout test: the producer issues this many planes' copies
                            // and no more, so the consumers' bounded waits run out with no copy in flight
    const double* coef;
    int degree;
    int step;
    double taps[8];
};

struct FilterMaps {
    CUtensorMap phi, prev, w0, w1, w2, inv, pot;
};

__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long globaltimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(unsigned bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned bar, unsigned parity) {
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    return done != 0;
}

__device__ __forceinline__ void record_failure(unsigned token) {
    atomicOr(&g_device_error, 1);
    atomicExch(&g_abort_token, token);
}

// Bounded wait for the phase of this parity. False after limit_ns, or as soon as another warp or
// CTA of the same launch has given up; a timeout itself is recorded. With nap_ns > 0 the warp sleeps
// between tries, 32 ns doubling up to nap_ns: a role that runs ahead of the one it waits for (the
// producer, the pass groups) then takes few issue slots from the warps doing the work, at the cost
// of waking up to nap_ns late.
__device__ __noinline__ bool mbar_wait_bounded(unsigned bar, unsigned parity, unsigned long long limit_ns,
                                               unsigned token, unsigned nap_ns) {
    const unsigned long long start = globaltimer();
    unsigned nap = 32;
    for (unsigned it = 0; it < (1u << 30); ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if (nap_ns > 0) {
            __nanosleep(nap);
            nap = nap * 2 < nap_ns ? nap * 2 : nap_ns;
        }
        if ((it & 7) == 7) {
            if (*reinterpret_cast<volatile unsigned*>(&g_abort_token) == token) return false;
            if (globaltimer() - start > limit_ns) {
                record_failure(token);
                return false;
            }
        }
    }
    record_failure(token);
    return false;
}

__device__ __forceinline__ bool wait_full(unsigned bar, unsigned parity, unsigned token, unsigned nap_ns = 0) {
    if (mbar_try_wait(bar, parity)) return true;
    return mbar_wait_bounded(bar, parity, kWaitLimitNs, token, nap_ns);
}

// The same wait by every lane of a warp, with one verdict for the whole warp (a lane that gave up
// makes the warp leave together, so no lane waits in __syncwarp for an exited one).
__device__ __forceinline__ bool warp_wait(unsigned bar, unsigned parity, unsigned token, unsigned nap_ns = 0) {
    return __all_sync(0xffffffffu, wait_full(bar, parity, token, nap_ns)) != 0;
}

// warp_wait with a warp-uniform fast path: one try and one vote when the phase is complete for
// every lane; otherwise the whole warp takes the bounded wait together. No branch around the wait
// depends on a lane's own value, so the caller's code needs no divergence handling for it.
__device__ __forceinline__ bool warp_wait_uniform(unsigned bar, unsigned parity, unsigned token,
                                                  unsigned nap_ns = 0) {
    if (__all_sync(0xffffffffu, mbar_try_wait(bar, parity))) return true;
    return __all_sync(0xffffffffu, mbar_wait_bounded(bar, parity, kWaitLimitNs, token, nap_ns)) != 0;
}

__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            unsigned bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<unsigned long long>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar)
        : "memory");
}

// The orbital held by half h of lane l, or -1 for an empty half. Lanes run over the orbitals in order
// (lane l: orbitals ORBITALS l + h) or, aligned to orbital groups, over each group separately, so that
// no lane mixes two groups (lane l: group l / lpg, orbitals ORBITALS (l mod lpg) + h of that group).
// Lane indices fit 32 bits (a lane is a whole grid of points), so the division is a 32-bit one, which
// the compiler inlines: no call interrupts the loops that form orbitals on the fly.
template <int ORBITALS>
__host__ __device__ __forceinline__ int64_t lane_orbital(int64_t l, int h, int64_t batch, int opg, int lpg) {
    int64_t o;
    if (lpg > 0) {
        const int li = static_cast<int>(l);
        const int g = li / lpg;
        const int j = ORBITALS * (li - g * lpg) + h;
        if (j >= opg) return -1;
        o = int64_t(g) * opg + j;
    } else {
        o = ORBITALS * l + h;
    }
    return o < batch ? o : -1;
}

template <typename Lane, int TZ>
__global__ void __launch_bounds__(Shape<TZ, sizeof(typename Lane::S)>::T, 1)
    slab_filter_kernel(const __grid_constant__ FilterMaps maps, const FilterArgs a) {
    using S = typename Lane::S;
    using E = typename Lane::E;
    using SH = Shape<TZ, sizeof(S)>;
    constexpr int BW = SH::BW;
    extern __shared__ __align__(1024) unsigned char smem[];
    const unsigned bar_full = smem_u32(smem + SH::O_BAR);
    const unsigned bar_empty = bar_full + 8 * R;
    const unsigned bar_yfull = bar_empty + 8 * R;
    const unsigned bar_yempty = bar_yfull + 8 * RY;

    const int t = threadIdx.x;
    const int warp = t >> 5;
    const int nx = a.nx, ny = a.ny, nz = a.nz, nzp = a.nzp;
    const int y0 = (blockIdx.x / a.tiles_z) * TY;
    const int z0 = (blockIdx.x % a.tiles_z) * TZ;
    const int xa = blockIdx.y * a.xchunk;
    const int xe = min(xa + a.xchunk, nx) - 1;
    const int lane = static_cast<int>(a.lane_first) + blockIdx.z;
    // Planes marched: nodes xa-7 .. xe+7. A chunk that starts at the grid's first plane skips the 7
    // planes before it: phi is zero there (the Dirichlet boundary), and nothing formed at those
    // planes reaches an output -- the x faces that outputs 0.. need are all formed from plane 0 on,
    // with the zeroed queues standing for the nodes outside.
    const int q0 = xa > 0 ? xa - HALO : 0;
    const int npl = xe + HALO + 1 - q0;
    const bool has_prev = a.has_prev != 0;

    // the lane's orbitals (an empty second half borrows the first's group for its lookups)
    const int64_t o0 = lane_orbital<Lane::ORBITALS>(lane, 0, a.batch, a.orb_per_group, a.lanes_per_group);
    const int64_t o1s = (Lane::ORBITALS == 2)
                            ? lane_orbital<Lane::ORBITALS>(lane, 1, a.batch, a.orb_per_group, a.lanes_per_group)
                            : -1;
    const int64_t o1 = o1s >= 0 ? o1s : o0;
    const int g0 = a.shared_potential ? 0 : static_cast<int>(o0 / a.orb_per_group);
    const int g1 = a.shared_potential ? 0 : static_cast<int>(o1 / a.orb_per_group);
    const int gg = a.per_system_geometry ? static_cast<int>(o0 / a.orb_per_group) : 0;

    // Systems on their own grids: a tile wholly beyond its lane's system (every point zero in every
    // iterate: zero face weights, h^3/omega and potential there) stores its zeros and computes
    // nothing; an empty lane stores zeros too. The whole CTA leaves before any barrier is used.
    if (a.system_shapes != nullptr) {
        const int* shape = a.system_shapes + 3 * (o0 >= 0 ? gg : 0);
        if (o0 < 0 || xa >= shape[0] || y0 >= shape[1] || z0 >= shape[2]) {
            const int64_t plane_n = int64_t(ny) * nz;
            for (int k = t; k < (xe - xa + 1) * TY * TZ; k += blockDim.x) {
                const int i = xa + k / (TY * TZ);
                const int r = k % (TY * TZ);
                const int y = y0 + r / TZ, z = z0 + r % TZ;
                if (y >= ny || z >= nzp) continue;
                if (a.final_out) {
                    if (z >= nz) continue;
                    const int64_t pt = int64_t(i) * plane_n + int64_t(y) * nz + z;
                    if constexpr (Lane::ORBITALS == 2) {
                        if (o0 >= 0) store_as<float>(a.out, a.out_dtype, o0 * (plane_n * nx) + pt, 0.0f);
                        if (o1s >= 0) store_as<float>(a.out, a.out_dtype, o1s * (plane_n * nx) + pt, 0.0f);
                    } else {
                        if (o0 >= 0) store_as<double>(a.out, a.out_dtype, o0 * (plane_n * nx) + pt, 0.0);
                    }
                } else {
                    static_cast<E*>(a.out)[(int64_t(lane) * nx + i) * (int64_t(ny) * nzp) + int64_t(y) * nzp + z] =
                        Lane::zero();
                }
            }
            return;
        }
    }

    if (t == 0) {
        for (int s = 0; s < R; ++s) {
            mbar_init(bar_full + 8 * s, 1);
            mbar_init(bar_empty + 8 * s, SH::MW + SH::PWG);
        }
        for (int s = 0; s < RY; ++s) {
            mbar_init(bar_yfull + 8 * s, SH::PWG);
            mbar_init(bar_yempty + 8 * s, SH::MW);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();

    E tap[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) tap[j] = Lane::splat(static_cast<S>(a.taps[j]));

    if (warp == SH::MW + SH::PW) {
        // ------------------------------------------------------------------ producer
        if ((t & 31) != 0) return;
        const unsigned tx = SH::TX_PHI + (has_prev ? SH::TX_PREV : 0) + SH::TX_W0 + SH::TX_W1 + SH::TX_W2 +
                            SH::TX_INV + 2 * SH::TX_POT;
        int issued = 0;
        int s = 0, ph = 1;  // slot; parity of its previous use (the first R fills wait for nothing)
        for (int n = 0; n < npl; ++n) {
            if (a.stop_after_planes > 0 && n >= a.stop_after_planes) break;
            if (n >= R && !wait_full(bar_empty + 8 * s, ph, a.token)) break;
            const unsigned full = bar_full + 8 * s;
            unsigned char* slot = smem + s * SH::SLOT;
            const int q = q0 + n;
            mbar_expect_tx(full, tx);
            tma_load_4d(slot + SH::O_PHI, &maps.phi, z0 - 8, y0 - HALO, q, lane, full);
            if (has_prev) tma_load_4d(slot + SH::O_PREV, &maps.prev, z0, y0, q - HALO, lane, full);
            tma_load_4d(slot + SH::O_W0, &maps.w0, z0, y0, q, gg, full);  // x face q-4 is stored at index q
            tma_load_4d(slot + SH::O_W1, &maps.w1, z0, y0, q, gg, full);  // y faces y0-4 .. y0+10
            tma_load_4d(slot + SH::O_W2, &maps.w2, z0, y0, q, gg, full);  // z faces z0-4 .. z0+TZ+3
            tma_load_4d(slot + SH::O_INV, &maps.inv, z0, y0, q - HALO, gg, full);
            tma_load_4d(slot + SH::O_POT0, &maps.pot, z0, y0, q - HALO, g0, full);
            tma_load_4d(slot + SH::O_POT1, &maps.pot, z0, y0, q - HALO, g1, full);
            issued = n + 1;
            if (++s == R) {
                s = 0;
                ph ^= 1;
            }
        }
        if (issued < npl) {
            // Leaving early: let the copies already issued land first (bounded).
            for (int n = max(0, issued - R); n < issued; ++n) {
                const unsigned long long start = globaltimer();
                for (unsigned it = 0; it < (1u << 24); ++it)
                    if (mbar_try_wait(bar_full + 8 * (n % R), (n / R) & 1) || globaltimer() - start > 100000000ull)
                        break;
            }
        }
        return;
    }

    if (warp >= SH::MW) {
        // ------------------------------------------------------------------ pass groups
        const int grp = (warp - SH::MW) / SH::PWG;
        const int it = t - (SH::MW + grp * SH::PWG) * 32;  // item of the plane this thread takes
        // The item's line segment: 22 nodes at stride ns from node offset nb, 15 face weights at
        // stride ws from weight offset wb (both relative to the slot), 8 outputs at stride os from
        // output offset ob (relative to the result slot), the first `first` of them not stored.
        bool active = false;
        int nb = 0, ns = 0, wb = 0, ws = 0, ob = 0, os = 0, first = 0;
        if (it < TZ) {
            // y: column zc, nodes y0-7 .. y0+14, faces y0-4 .. y0+10, outputs y0 .. y0+7
            const int zc = it;
            active = z0 + zc < nz;
            nb = zc + 8;
            ns = BW;
            wb = SH::O_W1 / sizeof(S) + zc;
            ws = TZ;
            ob = zc;
            os = TZ;
        } else if (it < SH::ITEMS) {
            // z: row ry, outputs zs .. zs+7 (tile-relative), nodes zs-7 .. zs+14, faces zs-4 .. zs+10
            const int zi = it - TZ;
            const int ry = zi % TY;
            const int seg = zi / TY;
            const int zs = min(seg * 8, TZ - 8);
            first = seg * 8 - zs;
            active = y0 + ry < ny && z0 + zs < nz;
            nb = (ry + HALO) * BW + zs + 1;
            ns = 1;
            wb = SH::O_W2 / sizeof(S) + ry * (TZ + 8) + zs;
            ws = 1;
            ob = int(SH::YZ_Z / sizeof(E)) + ry * SH::ZROW + zs;
            os = 1;
        }
        int s = grp, ph = 0;  // slot and phase parity of plane n
        for (int n = grp; n < npl; n += NG) {
            if (!warp_wait(bar_full + 8 * s, ph, a.token)) return;
            const int q = q0 + n;
            if (q >= xa && q <= xe) {
                const int m = q - xa;
                const int ys = m & (RY - 1);
                const unsigned uy = m / RY;
                if (uy >= 1 && !warp_wait(bar_yempty + 8 * ys, (uy - 1) & 1, a.token)) return;
                if (active) {
                    const unsigned char* slot = smem + s * SH::SLOT;
                    const E* nodes = reinterpret_cast<const E*>(slot) + nb;
                    const S* w = reinterpret_cast<const S*>(slot) + wb;
                    E* out = reinterpret_cast<E*>(smem + SH::O_YZ + ys * SH::YZ_SLOT) + ob;
                    E v[NROW];
#pragma unroll
                    for (int r = 0; r < NROW; ++r) v[r] = nodes[r * ns];
                    E f[TY + 7];
#pragma unroll
                    for (int rf = 0; rf < TY + 7; ++rf) {
                        E sum = Lane::zero();
#pragma unroll
                        for (int j = 0; j < 8; ++j) sum = Lane::fma(tap[j], v[rf + j], sum);
                        f[rf] = Lane::mul(Lane::splat(w[rf * ws]), sum);
                    }
#pragma unroll
                    for (int o = 0; o < TY; ++o) {
                        E acc = Lane::zero();
#pragma unroll
                        for (int j = 0; j < 8; ++j) acc = Lane::fma(tap[j], f[o + 7 - j], acc);
                        if (o >= first) out[o * os] = acc;
                    }
                }
                __syncwarp();
                if ((t & 31) == 0) mbar_arrive(bar_yfull + 8 * ys);
            } else {
                __syncwarp();
            }
            if ((t & 31) == 0) mbar_arrive(bar_empty + 8 * s);
            s += NG;
            if (s >= R) {
                s -= R;
                ph ^= 1;
            }
        }
        return;
    }

    // ---------------------------------------------------------------------- march
    const int ty = t / TZ;
    const int tz = t - ty * TZ;
    const int y = y0 + ty;
    const int z = z0 + tz;
    const bool own_in = y < ny && z < nz;
    const bool own_pad = y < ny && z < nzp;
    const int64_t plane_n = int64_t(ny) * nz;
    const int own = ty * TZ + tz;  // index in the (TY, TZ) boxes

    E cc = Lane::zero(), ca = Lane::zero(), cb = Lane::zero();
    if (!a.apply_only) {
        const int64_t c0 = o0 / a.orb_per_group;  // one coefficient table per orbital group
        const int64_t c1 = o1 / a.orb_per_group;
        const double* r0 = a.coef + (c0 * a.degree + a.step) * 3;
        const double* r1 = a.coef + (c1 * a.degree + a.step) * 3;
        if constexpr (Lane::ORBITALS == 2) {
            cc = make_float2(static_cast<float>(r0[0]), static_cast<float>(r1[0]));
            ca = make_float2(static_cast<float>(r0[1]), static_cast<float>(r1[1]));
            cb = make_float2(static_cast<float>(r0[2]), static_cast<float>(r1[2]));
        } else {
            cc = r0[0];
            ca = r0[1];
            cb = r0[2];
        }
    }

    E phq[8], fq[8], yzq[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        phq[j] = Lane::zero();
        fq[j] = Lane::zero();
        yzq[j] = Lane::zero();
    }

    int s = 0, sph = 0;  // slot and phase parity of plane n
    for (int n0 = 0; n0 < npl; n0 += 8) {
#pragma unroll
        for (int g = 0; g < 8; ++g) {
            const int n = n0 + g;
            if (n >= npl) break;
            if (!warp_wait(bar_full + 8 * s, sph, a.token)) return;
            const unsigned char* slot = smem + s * SH::SLOT;
            const int q = q0 + n;
            phq[g] = reinterpret_cast<const E*>(slot + SH::O_PHI)[(ty + HALO) * BW + tz + 8];
            {
                E sum = Lane::zero();
#pragma unroll
                for (int j = 0; j < 8; ++j) sum = Lane::fma(tap[j], phq[(g + 1 + j) & 7], sum);
                const S wx = own_in ? reinterpret_cast<const S*>(slot + SH::O_W0)[own] : S(0);
                fq[g] = Lane::mul(Lane::splat(wx), sum);  // x face q - 4
            }
            if (q >= xa && q <= xe) {
                const int m = q - xa;
                const int ys = m & (RY - 1);
                if (!warp_wait(bar_yfull + 8 * ys, (m / RY) & 1, a.token)) return;
                const unsigned char* yz = smem + SH::O_YZ + ys * SH::YZ_SLOT;
                yzq[g] = Lane::add(reinterpret_cast<const E*>(yz)[own],
                                   reinterpret_cast<const E*>(yz + SH::YZ_Z)[ty * SH::ZROW + tz]);
                __syncwarp();
                if ((t & 31) == 0) mbar_arrive(bar_yempty + 8 * ys);
            }
            const int i = q - HALO;
            if (i >= xa && own_pad) {
                E xt = Lane::zero();
#pragma unroll
                for (int j = 0; j < 8; ++j) xt = Lane::fma(tap[j], fq[(g - j) & 7], xt);
                const E div = Lane::add(xt, yzq[(g + 1) & 7]);
                const int64_t pt = int64_t(i) * plane_n + (own_in ? int64_t(y) * nz + z : 0);
                E res;
                if (own_in) {
                    const E phi = phq[(g + 1) & 7];
                    const S inv = reinterpret_cast<const S*>(slot + SH::O_INV)[own];
                    const E kin = Lane::mul(Lane::mul(div, Lane::splat(S(0.5))), Lane::splat(inv));
                    if (a.kinetic_only) {
                        res = kin;
                    } else {
                        E potv;
                        if constexpr (Lane::ORBITALS == 2)
                            potv = make_float2(reinterpret_cast<const S*>(slot + SH::O_POT0)[own],
                                               reinterpret_cast<const S*>(slot + SH::O_POT1)[own]);
                        else
                            potv = reinterpret_cast<const S*>(slot + SH::O_POT0)[own];
                        const E applied = Lane::fma(phi, potv, kin);
                        if (a.apply_only) {
                            res = applied;
                        } else {
                            res = Lane::mul(Lane::fma(Lane::neg(cc), phi, applied), ca);
                            if (has_prev)
                                res = Lane::fma(Lane::neg(cb), reinterpret_cast<const E*>(slot + SH::O_PREV)[own],
                                                res);
                        }
                    }
                } else {
                    res = Lane::zero();  // the padding column stays zero
                }
                if (a.final_out) {
                    if (own_in) {
                        if constexpr (Lane::ORBITALS == 2) {
                            if (o0 >= 0) store_as<float>(a.out, a.out_dtype, o0 * (plane_n * nx) + pt, res.x);
                            if (o1s >= 0) store_as<float>(a.out, a.out_dtype, o1s * (plane_n * nx) + pt, res.y);
                        } else {
                            store_as<double>(a.out, a.out_dtype, o0 * (plane_n * nx) + pt, res);
                        }
                    }
                } else {
                    E* out = static_cast<E*>(a.out);
                    out[(int64_t(lane) * nx + i) * (int64_t(ny) * nzp) + int64_t(y) * nzp + z] = res;
                }
            }
            __syncwarp();
            if ((t & 31) == 0) mbar_arrive(bar_empty + 8 * s);
            if (++s == R) {
                s = 0;
                sph ^= 1;
            }
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Wide lanes: 16 bytes per lane point -- four float32 orbitals (two packed f32x2 instructions per
// element operation) or two float64 orbitals. The instructions that do not scale with the orbitals
// (addressing, barrier waits, loads and stores of a point, the weights) are shared by twice as many
// orbitals as in slab_filter_kernel. The roles and rings are those of slab_filter_kernel; three parts
// are restructured so that a thread stays within its register share (one CTA per SM) and the roles
// wait on one another less:
//   tile        TY x TZ with TY = 8 or 13 (13 x 24 covers a 65-row grid in 5 tiles without padding);
//   pass item   streams its TY + 14 nodes through a window of 8, forming each face as soon as its 8
//               nodes are in and adding it at once to the TY outputs it reaches (TY accumulators);
//               the plane slot is released as soon as the outputs are in registers, before they are
//               stored to a result slot;
//   march       keeps the last 8 nodes and the 8 outputs still open: each new x face is added to all
//               of them, the newest output opens with its first face, and the oldest one is complete
//               after its last face, when its plane's y+z part joins it. The pass groups thus have
//               7 planes of lead on the march, and the result ring is 8 (or 6) slots deep.
// Lanes run over the orbitals in order (lane l: orbitals ORB l .. ORB l + ORB - 1); lanes aligned to
// orbital groups (per-system geometry) keep slab_filter_kernel.

struct WideF4 {  // four float32 orbitals
    using E = float4;
    using T = float2;  // a tap or weight, twice
    using S = float;
    static constexpr int ORB = 4;
    static constexpr bool WIDE = true;
    static constexpr CUtensorMapDataType GEO_TYPE = CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    static __device__ __forceinline__ float2 lo(E v) { return make_float2(v.x, v.y); }
    static __device__ __forceinline__ float2 hi(E v) { return make_float2(v.z, v.w); }
    static __device__ __forceinline__ E join(float2 a, float2 b) { return make_float4(a.x, a.y, b.x, b.y); }
    static __device__ __forceinline__ T splat(S s) { return make_float2(s, s); }
    // c - t v and -t v (the negation folded into the operand)
    static __device__ __forceinline__ E fmat_neg(T t, E v, E c) {
        const T n = make_float2(-t.x, -t.y);
        return join(__ffma2_rn(n, lo(v), lo(c)), __ffma2_rn(n, hi(v), hi(c)));
    }
    static __device__ __forceinline__ E mult_neg(T t, E v) {
        const T n = make_float2(-t.x, -t.y);
        return join(__fmul2_rn(n, lo(v)), __fmul2_rn(n, hi(v)));
    }
    // c + tap[k] v for the antisymmetric taps held as their lower four (k = 0..7, compile time)
    static __device__ __forceinline__ E fmat_k(const T* t4, int k, E v, E c) {
        return k < 4 ? fmat(t4[k], v, c) : fmat_neg(t4[7 - k], v, c);
    }
    static __device__ __forceinline__ E fmat(T t, E v, E c) {
        return join(__ffma2_rn(t, lo(v), lo(c)), __ffma2_rn(t, hi(v), hi(c)));
    }
    static __device__ __forceinline__ E mult(T t, E v) { return join(__fmul2_rn(t, lo(v)), __fmul2_rn(t, hi(v))); }
    static __device__ __forceinline__ E fma(E a, E b, E c) {
        return join(__ffma2_rn(lo(a), lo(b), lo(c)), __ffma2_rn(hi(a), hi(b), hi(c)));
    }
    static __device__ __forceinline__ E mul(E a, E b) { return join(__fmul2_rn(lo(a), lo(b)), __fmul2_rn(hi(a), hi(b))); }
    static __device__ __forceinline__ E add(E a, E b) { return join(__fadd2_rn(lo(a), lo(b)), __fadd2_rn(hi(a), hi(b))); }
    // a - b (the negation folded into the add's operand)
    static __device__ __forceinline__ E sub(E a, E b) {
        return join(__fadd2_rn(lo(a), make_float2(-b.x, -b.y)), __fadd2_rn(hi(a), make_float2(-b.z, -b.w)));
    }
    static __device__ __forceinline__ E neg(E a) { return make_float4(-a.x, -a.y, -a.z, -a.w); }
    static __device__ __forceinline__ E zero() { return make_float4(0.f, 0.f, 0.f, 0.f); }
    static __device__ __forceinline__ E make(const S* v) { return make_float4(v[0], v[1], v[2], v[3]); }
    static __device__ __forceinline__ void parts(E v, S* out) {
        out[0] = v.x;
        out[1] = v.y;
        out[2] = v.z;
        out[3] = v.w;
    }
};

struct WideD2 {  // two float64 orbitals
    using E = double2;
    using T = double;
    using S = double;
    static constexpr int ORB = 2;
    static constexpr bool WIDE = true;
    static constexpr CUtensorMapDataType GEO_TYPE = CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
    static __device__ __forceinline__ T splat(S s) { return s; }
    static __device__ __forceinline__ E fmat_neg(T t, E v, E c) {
        return make_double2(::fma(-t, v.x, c.x), ::fma(-t, v.y, c.y));
    }
    static __device__ __forceinline__ E mult_neg(T t, E v) { return make_double2(-t * v.x, -t * v.y); }
    static __device__ __forceinline__ E fmat_k(const T* t4, int k, E v, E c) {
        return k < 4 ? fmat(t4[k], v, c) : fmat_neg(t4[7 - k], v, c);
    }
    static __device__ __forceinline__ E fmat(T t, E v, E c) { return make_double2(::fma(t, v.x, c.x), ::fma(t, v.y, c.y)); }
    static __device__ __forceinline__ E mult(T t, E v) { return make_double2(t * v.x, t * v.y); }
    static __device__ __forceinline__ E fma(E a, E b, E c) {
        return make_double2(::fma(a.x, b.x, c.x), ::fma(a.y, b.y, c.y));
    }
    static __device__ __forceinline__ E mul(E a, E b) { return make_double2(a.x * b.x, a.y * b.y); }
    static __device__ __forceinline__ E add(E a, E b) { return make_double2(a.x + b.x, a.y + b.y); }
    static __device__ __forceinline__ E sub(E a, E b) { return make_double2(a.x - b.x, a.y - b.y); }
    static __device__ __forceinline__ E neg(E a) { return make_double2(-a.x, -a.y); }
    static __device__ __forceinline__ E zero() { return make_double2(0.0, 0.0); }
    static __device__ __forceinline__ E make(const S* v) { return make_double2(v[0], v[1]); }
    static __device__ __forceinline__ void parts(E v, S* out) {
        out[0] = v.x;
        out[1] = v.y;
    }
};

// Plane slots of the wide kernel (16-byte elements: a slot is 31-41 KB): as many as shared memory
// holds beside a result ring of at least 4, up to kWideMaxSlots. A deeper ring keeps more copies in
// flight per SM, which is what hides the copies' latency behind the march.
constexpr int kWideMaxSlots = 6;
constexpr size_t kWideSmem = 232448;  // the opt-in shared memory of one CTA

template <int TYW, int TZ, int SB, int ORB>  // TYW: tile rows; SB: bytes of a geometry element; ORB: potentials per lane
struct WideShape {
    static constexpr int NROWW = TYW + 2 * HALO;  // rows of the phi box
    static constexpr int EB = 16;
    // march warps: one thread per tile point (the last warp may have idle threads)
    static constexpr int MW = (TYW * TZ + 31) / 32;
    // pass items: TZ columns of TYW outputs (y) and TYW rows x NZS segments of TYW outputs (z); the
    // last z segment is moved left to end at TZ (it then stores only the outputs the previous one
    // did not): every item forms TYW outputs from TYW + 14 nodes
    static constexpr int NZS = (TZ + TYW - 1) / TYW;
    static constexpr int ITEMS = TZ + TYW * NZS;
    static constexpr int PWG = (ITEMS + 31) / 32;
    static constexpr int PW = NG * PWG;
    static constexpr int WARPS = MW + PW + 1;
    static constexpr int T = WARPS * 32;
    // odd row pitches (in 16-byte points): the 8 rows of a warp's z items then fall on 8 different
    // groups of 4 banks (an even pitch such as TZ + 18 puts them on 4)
    static constexpr int BW = TZ + 19;  // phi box: z0-8 .. z0+TZ+10
    static constexpr int ZROW = TZ + 3;
    static constexpr unsigned TX_PHI = NROWW * BW * EB;
    static constexpr unsigned TX_PREV = TYW * TZ * EB;
    static constexpr unsigned TX_W0 = TYW * TZ * SB;
    static constexpr unsigned TX_W1 = (TYW + 7) * TZ * SB;
    static constexpr unsigned TX_W2 = TYW * (TZ + 8) * SB;
    static constexpr unsigned TX_INV = TYW * TZ * SB;
    static constexpr unsigned TX_POT = TYW * TZ * SB;
    static constexpr size_t O_PHI = 0;
    static constexpr size_t O_PREV = O_PHI + align128(TX_PHI);
    static constexpr size_t O_W0 = O_PREV + align128(TX_PREV);
    static constexpr size_t O_W1 = O_W0 + align128(TX_W0);
    static constexpr size_t O_W2 = O_W1 + align128(TX_W1);
    static constexpr size_t O_INV = O_W2 + align128(TX_W2);
    static constexpr size_t O_POT = O_INV + align128(TX_INV);  // ORB potentials, POT_STEP apart
    static constexpr size_t POT_STEP = align128(TX_POT);
    static constexpr size_t SLOT = O_POT + ORB * POT_STEP;
    static constexpr size_t YZ_Z = size_t(TYW) * TZ * EB;
    static constexpr size_t YZ_SLOT = align128(YZ_Z + size_t(TYW) * ZROW * EB);
    static constexpr size_t need(int rw, int ry) { return rw * SLOT + ry * YZ_SLOT + (2 * rw + 2 * ry) * 8; }
    static constexpr int slots() {
        int rw = kWideMaxSlots;
        while (rw > 2 && need(rw, 4) > kWideSmem) --rw;
        return rw;
    }
    static constexpr int RWS = slots();
    // y+z result slots: the march adds a plane's y+z part when that output completes, 7 planes after
    // the pass formed it, so the result ring takes what is left, up to 8 (at least 4)
    static constexpr int result_slots() {
        int ry = 8;
        while (ry > 4 && need(RWS, ry) > kWideSmem) --ry;
        return ry;
    }
    static constexpr int RYW = result_slots();
    static constexpr size_t O_YZ = RWS * SLOT;
    static constexpr size_t O_BAR = O_YZ + RYW * YZ_SLOT;
    static constexpr size_t BYTES = O_BAR + (2 * RWS + 2 * RYW) * 8;
    static_assert(RWS >= NG && need(RWS, RYW) <= kWideSmem, "the rings fit one CTA's shared memory");
    static_assert(TZ >= TYW && TZ % 4 == 0, "z segments of TYW inside the tile; 16-byte float32 geometry rows");
    static_assert(BW % 2 == 1 && ZROW % 2 == 1, "odd row pitches");
    static_assert((TZ - TYW) + NROWW <= BW - 1, "the last z segment's nodes lie inside the phi box");
    // the idle march threads of the last warp read their tile's first point (see the kernel); the
    // per-point regions of a slot hold at least one warp's worth of points past the tile
    static_assert(TYW * TZ >= 32, "a tile of at least one warp");
    static_assert(BYTES <= 232448, "fits the opt-in shared memory of one CTA");
};

// One CTA per SM: the register budget per thread. The SM's 64 K registers are four files of 16 K,
// one per scheduler, and a CTA's warps are spread over the four, so the scheduler with the most
// warps (ceil(warps / 4)) bounds it: 128 registers for 13 to 16 warps, 170 for 9 to 12.
template <int T>
constexpr int wide_max_registers() {
    return (16384 / (((T / 32) + 3) / 4 * 32)) / 8 * 8 < 255 ? (16384 / (((T / 32) + 3) / 4 * 32)) / 8 * 8 : 255;
}

// GENERAL: the lane's orbitals, its geometry and the skip of tiles beyond its system's grid are
// looked up at run time, for lanes in orbital order or aligned to orbital groups (per-system
// geometry, a.lanes_per_group > 0). Otherwise the kernel takes lanes in orbital order over one
// shared geometry only, and carries none of those lookups.
template <typename W, int TYW, int TZ, bool GENERAL>
__global__ void __maxnreg__((wide_max_registers<WideShape<TYW, TZ, sizeof(typename W::S), W::ORB>::T>()))
    slab_filter_wide_kernel(const __grid_constant__ FilterMaps maps, const FilterArgs a) {
    using E = typename W::E;
    using S = typename W::S;
    constexpr int ORB = W::ORB;
    using SH = WideShape<TYW, TZ, sizeof(S), ORB>;
    constexpr int TY = TYW;              // this kernel's tile rows (the 8-byte-lane kernel keeps 8)
    constexpr int NROW = SH::NROWW;
    constexpr int BW = SH::BW;
    extern __shared__ __align__(1024) unsigned char smem[];
    const unsigned bar_full = smem_u32(smem + SH::O_BAR);
    constexpr int RW = SH::RWS;  // plane slots (planes n and n + RW share a slot)
    const unsigned bar_empty = bar_full + 8 * RW;
    const unsigned bar_yfull = bar_empty + 8 * RW;
    const unsigned bar_yempty = bar_yfull + 8 * SH::RYW;

    const int t = threadIdx.x;
    const int warp = t >> 5;
    const int nx = a.nx, ny = a.ny, nz = a.nz, nzp = a.nzp;
    const int y0 = (blockIdx.x / a.tiles_z) * TY;
    const int z0 = (blockIdx.x % a.tiles_z) * TZ;
    const int xa = blockIdx.y * a.xchunk;
    const int xe = min(xa + a.xchunk, nx) - 1;
    const int lane = static_cast<int>(a.lane_first) + blockIdx.z;
    const int q0 = xa > 0 ? xa - HALO : 0;
    const int npl = xe + HALO + 1 - q0;
    const bool has_prev = a.has_prev != 0;

    // The lane's orbitals: ORB lane + h in order, or, with lanes aligned to orbital groups (systems
    // on their own grids), orbitals ORB (l mod lpg) + h of group l / lpg; -1 for an empty slot, which
    // borrows the lane's first orbital for its lookups. Formed where they are used, so that no role
    // keeps them in registers through its loop.
    const int64_t orb0 = int64_t(ORB) * lane;
    auto orbital_at = [&](int h) -> int64_t {
        if constexpr (GENERAL) return lane_orbital<ORB>(lane, h, a.batch, a.orb_per_group, a.lanes_per_group);
        return orb0 + h < a.batch ? orb0 + h : -1;
    };
    auto orbital_of = [&](int h) -> int64_t {
        if constexpr (GENERAL) {
            const int64_t o = orbital_at(h), o0 = orbital_at(0);
            return o >= 0 ? o : (o0 >= 0 ? o0 : 0);
        }
        return orb0 + h < a.batch ? orb0 + h : orb0;
    };
    // the lane's geometry: its system's with per-system geometry, else the one shared copy
    const int geo = (GENERAL && a.per_system_geometry) ? static_cast<int>(orbital_of(0) / a.orb_per_group) : 0;

    // Systems on their own grids: a tile wholly beyond its lane's system (zero there in every
    // iterate) stores its zeros and computes nothing; so does an empty lane. The whole CTA leaves
    // before any barrier is used.
    if (GENERAL && a.system_shapes != nullptr) {
        const int* shape = a.system_shapes + 3 * geo;
        if (orbital_at(0) < 0 || xa >= shape[0] || y0 >= shape[1] || z0 >= shape[2]) {
            const int64_t plane_n = int64_t(ny) * nz;
            for (int k = t; k < (xe - xa + 1) * TY * TZ; k += blockDim.x) {
                const int i = xa + k / (TY * TZ);
                const int r = k % (TY * TZ);
                const int y = y0 + r / TZ, z = z0 + r % TZ;
                if (y >= ny || z >= nzp) continue;
                if (a.final_out) {
                    if (z >= nz) continue;
                    const int64_t pt = int64_t(i) * plane_n + int64_t(y) * nz + z;
#pragma unroll
                    for (int h = 0; h < ORB; ++h) {
                        const int64_t o = orbital_at(h);
                        if (o >= 0) store_as<S>(a.out, a.out_dtype, o * (plane_n * nx) + pt, S(0));
                    }
                } else {
                    static_cast<E*>(a.out)[(int64_t(lane) * nx + i) * (int64_t(ny) * nzp) + int64_t(y) * nzp + z] =
                        W::zero();
                }
            }
            return;
        }
    }

    if (t == 0) {
        for (int s = 0; s < RW; ++s) {
            mbar_init(bar_full + 8 * s, 1);
            mbar_init(bar_empty + 8 * s, SH::MW + SH::PWG);
        }
        for (int s = 0; s < SH::RYW; ++s) {
            mbar_init(bar_yfull + 8 * s, SH::PWG);
            mbar_init(bar_yempty + 8 * s, SH::MW);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();

    // the taps are antisymmetric (tap[7 - j] = -tap[j]): four registers serve all eight, the upper
    // four as negated operands (tapk below)
    typename W::T tap4[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) tap4[j] = W::splat(static_cast<S>(a.taps[j]));
#define tap(j) tap4[(j)]

    if (warp == SH::MW + SH::PW) {
        // ------------------------------------------------------------------ producer
        if ((t & 31) != 0) return;
        const unsigned tx = SH::TX_PHI + (has_prev ? SH::TX_PREV : 0) + SH::TX_W0 + SH::TX_W1 + SH::TX_W2 +
                            SH::TX_INV + ORB * SH::TX_POT;
        int grp[ORB];
#pragma unroll
        for (int h = 0; h < ORB; ++h)
            grp[h] = a.shared_potential ? 0 : static_cast<int>(orbital_of(h) / a.orb_per_group);
        int issued = 0;
        int s = 0, ph = 1;
        for (int n = 0; n < npl; ++n) {
            if (a.stop_after_planes > 0 && n >= a.stop_after_planes) break;
            if (n >= RW && !wait_full(bar_empty + 8 * s, ph, a.token, kNapNs)) break;
            const unsigned full = bar_full + 8 * s;
            unsigned char* slot = smem + s * SH::SLOT;
            const int q = q0 + n;
            mbar_expect_tx(full, tx);
            // lane buffers as 8-byte elements, two per point: x = 2 z
            tma_load_4d(slot + SH::O_PHI, &maps.phi, 2 * (z0 - 8), y0 - HALO, q, lane, full);
            if (has_prev) tma_load_4d(slot + SH::O_PREV, &maps.prev, 2 * z0, y0, q - HALO, lane, full);
            tma_load_4d(slot + SH::O_W0, &maps.w0, z0, y0, q, geo, full);
            tma_load_4d(slot + SH::O_W1, &maps.w1, z0, y0, q, geo, full);
            tma_load_4d(slot + SH::O_W2, &maps.w2, z0, y0, q, geo, full);
            tma_load_4d(slot + SH::O_INV, &maps.inv, z0, y0, q - HALO, geo, full);
#pragma unroll
            for (int h = 0; h < ORB; ++h)
                tma_load_4d(slot + SH::O_POT + h * SH::POT_STEP, &maps.pot, z0, y0, q - HALO, grp[h], full);
            issued = n + 1;
            if (++s == RW) {
                s = 0;
                ph ^= 1;
            }
        }
        if (issued < npl) {
            for (int n = max(0, issued - RW); n < issued; ++n) {
                const unsigned long long start = globaltimer();
                for (unsigned it = 0; it < (1u << 24); ++it)
                    if (mbar_try_wait(bar_full + 8 * (n % RW), (n / RW) & 1) || globaltimer() - start > 100000000ull)
                        break;
            }
        }
        return;
    }

    if (warp >= SH::MW) {
        // ------------------------------------------------------------------ pass groups
        const int pg = (warp - SH::MW) / SH::PWG;
        const int it = t - (SH::MW + pg * SH::PWG) * 32;
        bool active = false;
        int nb = 0, ns = 0, wb = 0, ws = 0, ob = 0, os = 0, first = 0;
        if (it < TZ) {
            const int zc = it;
            active = z0 + zc < nz;
            nb = zc + 8;
            ns = BW;
            wb = SH::O_W1 / sizeof(S) + zc;
            ws = TZ;
            ob = zc;
            os = TZ;
        } else if (it < SH::ITEMS) {
            const int zi = it - TZ;
            const int ry = zi % TY;
            const int seg = zi / TY;
            const int zs = min(seg * TY, TZ - TY);
            first = seg * TY - zs;
            active = y0 + ry < ny && z0 + zs < nz;
            nb = (ry + HALO) * BW + zs + 1;
            ns = 1;
            wb = SH::O_W2 / sizeof(S) + ry * (TZ + 8) + zs;
            ws = 1;
            ob = int(SH::YZ_Z / sizeof(E)) + ry * SH::ZROW + zs;
            os = 1;
        }
        int s = pg, ph = 0;
        for (int n = pg; n < npl; n += NG) {
            if (!warp_wait_uniform(bar_full + 8 * s, ph, a.token, kNapNs)) return;
            const int q = q0 + n;
            if (q >= xa && q <= xe) {
                E acc[TY];
                if (active) {
                    const unsigned char* slot = smem + s * SH::SLOT;
                    const E* nodes = reinterpret_cast<const E*>(slot) + nb;
                    const S* w = reinterpret_cast<const S*>(slot) + wb;
                    E win[8];
#pragma unroll
                    for (int r = 0; r < NROW; ++r) {
                        win[r & 7] = nodes[r * ns];
                        if (r >= 7) {
                            const int rf = r - 7;  // face rf from nodes rf .. rf + 7
                            // the taps are antisymmetric (tap[7 - j] = -tap[j]): four independent
                            // differences, then a chain of four (depth 5 instead of 8)
                            E sum = W::mult(tap(0), W::sub(win[rf & 7], win[(rf + 7) & 7]));
#pragma unroll
                            for (int j = 1; j < 4; ++j)
                                sum = W::fmat(tap(j), W::sub(win[(rf + j) & 7], win[(rf + 7 - j) & 7]), sum);
                            const E f = W::mult(W::splat(w[rf * ws]), sum);
                            // face rf reaches outputs o = rf - 7 .. rf with tap o + 7 - rf
#pragma unroll
                            for (int o = 0; o < TY; ++o) {
                                if (o < rf - 7 || o > rf) continue;
                                acc[o] = (o == rf) ? W::mult_neg(tap(0), f) : W::fmat_k(tap4, o + 7 - rf, f, acc[o]);
                            }
                        }
                    }
                }
                // the plane slot is free once the outputs are in registers; the result slot is
                // reused only after the march has taken its previous plane (7 planes behind)
                __syncwarp();
                if ((t & 31) == 0) mbar_arrive(bar_empty + 8 * s);
                const int m = q - xa;
                const int ys = m % SH::RYW;
                const unsigned uy = m / SH::RYW;
                if (uy >= 1 && !warp_wait_uniform(bar_yempty + 8 * ys, (uy - 1) & 1, a.token, kNapNs)) return;
                if (active) {
                    E* out = reinterpret_cast<E*>(smem + SH::O_YZ + ys * SH::YZ_SLOT) + ob;
#pragma unroll
                    for (int o = 0; o < TY; ++o)
                        if (o >= first) out[o * os] = acc[o];
                }
                __syncwarp();
                if ((t & 31) == 0) mbar_arrive(bar_yfull + 8 * ys);
            } else {
                __syncwarp();
                if ((t & 31) == 0) mbar_arrive(bar_empty + 8 * s);
            }
            s += NG;
            if (s >= RW) {
                s -= RW;
                ph ^= 1;
            }
        }
        return;
    }

    // ---------------------------------------------------------------------- march
    // Threads past the tile (when TY * TZ is not a multiple of 32) take part in every wait and
    // arrive, read their tile's first point and store nothing.
    const bool in_tile = t < TY * TZ;
    const int ty = in_tile ? t / TZ : 0;
    const int tz = in_tile ? t - ty * TZ : 0;
    const int y = y0 + ty;
    const int z = z0 + tz;
    const bool own_in = in_tile && y < ny && z < nz;
    const bool own_pad = in_tile && y < ny && z < nzp;
    const int64_t plane_n = int64_t(ny) * nz;
    const int own = ty * TZ + tz;

    E cc = W::zero(), ca = W::zero(), cb = W::zero();
    if (!a.apply_only) {
        S c3[3][ORB];
#pragma unroll
        for (int h = 0; h < ORB; ++h) {
            const int64_t o = orbital_of(h);
            const double* r = a.coef + ((o / a.orb_per_group) * a.degree + a.step) * 3;
#pragma unroll
            for (int k = 0; k < 3; ++k) c3[k][h] = static_cast<S>(r[k]);
        }
        cc = W::make(c3[0]);
        ca = W::make(c3[1]);
        cb = W::make(c3[2]);
    }

    E phq[8], acc[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        phq[j] = W::zero();
        acc[j] = W::zero();
    }

    const int own_off = y * nzp + z;  // this thread's point within a plane of the lane buffer
    int s = 0, sph = 0;   // plane slot and its phase parity
    int ys = 0, yph = 0;  // result slot of the next output completed, and its phase parity
    for (int n0 = 0; n0 < npl; n0 += 8) {
#pragma unroll
        for (int g = 0; g < 8; ++g) {
            const int n = n0 + g;
            if (n >= npl) break;
            if (!warp_wait_uniform(bar_full + 8 * s, sph, a.token)) return;
            const unsigned char* slot = smem + s * SH::SLOT;
            const int q = q0 + n;
            phq[g] = reinterpret_cast<const E*>(slot + SH::O_PHI)[(ty + HALO) * BW + tz + 8];
            E face;
            {
                // antisymmetric taps: sum_j<4 tap[j] (node q-7+j - node q-j)
                E sum = W::mult(tap(0), W::sub(phq[(g + 1) & 7], phq[g & 7]));
#pragma unroll
                for (int j = 1; j < 4; ++j)
                    sum = W::fmat(tap(j), W::sub(phq[(g + 1 + j) & 7], phq[(g + 8 - j) & 7]), sum);
                // outside the grid the weight is the copy's zero fill (an idle thread's face is
                // never stored)
                const S wx = reinterpret_cast<const S*>(slot + SH::O_W0)[own];
                face = W::mult(W::splat(wx), sum);  // x face q - 4
            }
            // the face reaches the open outputs q - 7 .. q (slot (g - d) & 7 holds output q - d, tap 7 - d)
#pragma unroll
            for (int d = 1; d < 8; ++d) acc[(g - d) & 7] = W::fmat_k(tap4, 7 - d, face, acc[(g - d) & 7]);
            const int i = q - HALO;  // output complete at this plane (slot (g + 1) & 7)
            if (i >= xa) {
                // the y+z part of output i, formed by a pass group 7 planes ago
                if (!warp_wait_uniform(bar_yfull + 8 * ys, yph, a.token)) return;
                const unsigned char* yzs = smem + SH::O_YZ + ys * SH::YZ_SLOT;
                const E yz = W::add(reinterpret_cast<const E*>(yzs)[own],
                                    reinterpret_cast<const E*>(yzs + SH::YZ_Z)[ty * SH::ZROW + tz]);
                __syncwarp();
                if ((t & 31) == 0) mbar_arrive(bar_yempty + 8 * ys);
                if (++ys == SH::RYW) {
                    ys = 0;
                    yph ^= 1;
                }
                // every thread forms a result (the idle ones from their tile's first point); only
                // the stores depend on the thread, so no branch here does
                const E div = W::add(acc[(g + 1) & 7], yz);
                const E phi = phq[(g + 1) & 7];
                const S inv = reinterpret_cast<const S*>(slot + SH::O_INV)[own];
                E res = W::mult(W::splat(S(0.5) * inv), div);
                if (!a.kinetic_only) {
                    S pv[ORB];
#pragma unroll
                    for (int h = 0; h < ORB; ++h)
                        pv[h] = reinterpret_cast<const S*>(slot + SH::O_POT + h * SH::POT_STEP)[own];
                    const E applied = W::fma(phi, W::make(pv), res);
                    if (a.apply_only) {
                        res = applied;
                    } else {
                        res = W::mul(W::fma(W::neg(cc), phi, applied), ca);
                        if (has_prev)
                            res = W::fma(W::neg(cb), reinterpret_cast<const E*>(slot + SH::O_PREV)[own], res);
                    }
                }
                res = own_in ? res : W::zero();  // the padding column stays zero
                if (a.final_out) {
                    if (own_in) {
                        const int64_t pt = int64_t(i) * plane_n + int64_t(y) * nz + z;
                        S rv[ORB];
                        W::parts(res, rv);
#pragma unroll
                        for (int h = 0; h < ORB; ++h) {
                            if constexpr (GENERAL) {
                                if (const int64_t o = orbital_at(h); o >= 0)
                                    store_as<S>(a.out, a.out_dtype, o * (plane_n * nx) + pt, rv[h]);
                            } else if (orb0 + h < a.batch) {
                                store_as<S>(a.out, a.out_dtype, (orb0 + h) * (plane_n * nx) + pt, rv[h]);
                            }
                        }
                    }
                } else if (own_pad) {
                    // the plane's offset is the same for the whole CTA (uniform arithmetic)
                    static_cast<E*>(a.out)[(int64_t(lane) * nx + i) * (int64_t(ny) * nzp) + own_off] = res;
                }
            }
            // the newest output, q, opens with its first face (its slot held output q - 8, completed
            // on the previous plane); its y+z part joins when it completes
            acc[g] = W::mult_neg(tap(0), face);
            __syncwarp();
            if ((t & 31) == 0) mbar_arrive(bar_empty + 8 * s);
            if (++s == RW) {
                s = 0;
                sph ^= 1;
            }
        }
    }
}

#undef tap

// Internal layout from a caller block: lanes of (nx, ny, nzp), padding and missing orbitals zero.
// blockIdx.y walks the lanes (the lane's orbitals are found once), and each thread writes two
// consecutive z points of a row (nzp is even) with one 16-byte store.
template <typename Lane>
__global__ void pack_lanes_kernel(const void* __restrict__ in, int in_dtype, int64_t batch, int nx, int ny, int nz,
                                  int nzp, int64_t lanes, int opg, int lpg, typename Lane::E* __restrict__ out) {
    using E = typename Lane::E;
    const int half = nzp / 2;
    const int64_t pairs = int64_t(nx) * ny * half;  // per lane
    const int64_t n_points = int64_t(nx) * ny * nz;
    const bool narrow = pairs <= 0xffffffffll;
    for (int64_t l = blockIdx.y; l < lanes; l += gridDim.y) {
        int64_t a0, a1;
        if constexpr (Lane::ORBITALS == 2) {
            a0 = lane_orbital<2>(l, 0, batch, opg, lpg);
            a1 = lane_orbital<2>(l, 1, batch, opg, lpg);
        } else {
            a0 = l;
            a1 = -1;
        }
        E* dst = out + l * (2 * pairs);
        for (int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; k < pairs;
             k += int64_t(gridDim.x) * blockDim.x) {
            int64_t xy;
            int zp;
            if (narrow) {
                const unsigned uk = static_cast<unsigned>(k), row = uk / static_cast<unsigned>(half);
                xy = row;
                zp = 2 * static_cast<int>(uk - row * static_cast<unsigned>(half));
            } else {
                xy = k / half;
                zp = 2 * static_cast<int>(k - xy * half);
            }
            const int64_t pt = xy * nz + zp;
            const bool in1 = zp + 1 < nz;  // zp < nz always (nzp - nz is 0 or 1)
            E v0, v1;
            if constexpr (Lane::ORBITALS == 2) {
                v0.x = a0 >= 0 ? load_as<float>(in, in_dtype, a0 * n_points + pt) : 0.f;
                v0.y = a1 >= 0 ? load_as<float>(in, in_dtype, a1 * n_points + pt) : 0.f;
                v1.x = (a0 >= 0 && in1) ? load_as<float>(in, in_dtype, a0 * n_points + pt + 1) : 0.f;
                v1.y = (a1 >= 0 && in1) ? load_as<float>(in, in_dtype, a1 * n_points + pt + 1) : 0.f;
                reinterpret_cast<float4*>(dst)[k] = make_float4(v0.x, v0.y, v1.x, v1.y);
            } else {
                v0 = load_as<double>(in, in_dtype, a0 * n_points + pt);
                v1 = in1 ? load_as<double>(in, in_dtype, a0 * n_points + pt + 1) : 0.0;
                reinterpret_cast<double2*>(dst)[k] = make_double2(v0, v1);
            }
        }
    }
}

// Wide lanes from a caller block: lane l holds orbitals ORB l .. ORB l + ORB - 1 as one 16-byte
// element per point, padding and missing orbitals zero. blockIdx.y walks the lanes; one point per
// thread.
template <typename W>
__global__ void pack_wide_kernel(const void* __restrict__ in, int in_dtype, int64_t batch, int nx, int ny, int nz,
                                 int nzp, int64_t lanes, int opg, int lpg, typename W::E* __restrict__ out) {
    using S = typename W::S;
    constexpr int ORB = W::ORB;
    const int64_t per_lane = int64_t(nx) * ny * nzp;
    const int64_t n_points = int64_t(nx) * ny * nz;
    const bool narrow = per_lane <= 0xffffffffll;
    for (int64_t l = blockIdx.y; l < lanes; l += gridDim.y) {
        typename W::E* dst = out + l * per_lane;
        int64_t orb[ORB];
#pragma unroll
        for (int h = 0; h < ORB; ++h) orb[h] = lane_orbital<ORB>(l, h, batch, opg, lpg);
        for (int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; k < per_lane;
             k += int64_t(gridDim.x) * blockDim.x) {
            int64_t xy;
            int zp;
            if (narrow) {
                const unsigned uk = static_cast<unsigned>(k), row = uk / static_cast<unsigned>(nzp);
                xy = row;
                zp = static_cast<int>(uk - row * static_cast<unsigned>(nzp));
            } else {
                xy = k / nzp;
                zp = static_cast<int>(k - xy * nzp);
            }
            S v[ORB];
#pragma unroll
            for (int h = 0; h < ORB; ++h) v[h] = S(0);
            if (zp < nz) {
                const int64_t pt = xy * nz + zp;
#pragma unroll
                for (int h = 0; h < ORB; ++h)
                    if (orb[h] >= 0) v[h] = load_as<S>(in, in_dtype, orb[h] * n_points + pt);
            }
            dst[k] = W::make(v);
        }
    }
}

// rows x cols -> rows x cols_pad (zeros in the padding), for the geometry copies TMA reads.
template <typename S>
__global__ void pad_rows_kernel(const S* __restrict__ src, int64_t rows, int cols, int cols_pad, int64_t src_stride,
                                S* __restrict__ dst) {
    const int64_t total = rows * cols_pad;
    for (int64_t idx = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; idx < total;
         idx += int64_t(gridDim.x) * blockDim.x) {
        const int64_t r = idx / cols_pad;
        const int c = static_cast<int>(idx - r * cols_pad);
        dst[idx] = c < cols ? src[r * src_stride + c] : S(0);
    }
}

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return nullptr;
        fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// A tiled map over a C-ordered array dims[rank-1] x ... x dims[0] (dims[0] contiguous).
int encode_map(CUtensorMap* map, CUtensorMapDataType type, int esize, int rank, void* base, const int64_t* dims,
               const unsigned* box) {
    auto enc = tensor_map_encoder();
    if (!enc) return CDFTB_ERR_LAUNCH;
    cuuint64_t gdim[5], gstride[4];
    cuuint32_t bdim[5], estr[5];
    int64_t stride = esize;
    for (int d = 0; d < rank; ++d) {
        gdim[d] = cuuint64_t(dims[d]);
        bdim[d] = box[d];
        estr[d] = 1;
        if (d >= 1) gstride[d - 1] = cuuint64_t(stride);
        stride *= dims[d];
    }
    const CUresult r = enc(map, type, rank, base, gdim, gstride, bdim, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                           CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? CDFTB_OK : CDFTB_ERR_ARGUMENT;
}

// Lanes per orbital group when lanes are aligned to groups (float32 lanes with per-system geometry), else 0.
int aligned_lanes_per_group(const cdftb_operator* op) {
    return (op->per_system_geometry && op->dtype == CDFTB_F32) ? (op->orbitals_per_group + 1) / 2 : 0;
}

int64_t lanes_of(const cdftb_operator* op, int64_t batch) {
    if (op->dtype != CDFTB_F32) return batch;
    const int lpg = aligned_lanes_per_group(op);
    return lpg > 0 ? ceil_div(batch, op->orbitals_per_group) * lpg : (batch + 1) / 2;
}

int padded_z(int nz) { return nz + (nz & 1); }

int64_t round_up(int64_t v, int64_t m) { return (v + m - 1) / m * m; }

int64_t systems_of(const cdftb_operator* op, int64_t batch) {
    return op->potential_stride == 0 ? 1 : ceil_div(batch, op->orbitals_per_group);
}

// Geometry copies: one, or one per orbital group.
int64_t geometry_systems(const cdftb_operator* op, int64_t batch) {
    return op->per_system_geometry ? ceil_div(batch, op->orbitals_per_group) : 1;
}

// Element counts of the padded geometry copies: w0, w1, w2, inv, potentials.
struct GeoPack {
    int nzg, nz8g;
    int64_t n_w0, n_w1, n_w2, n_inv, n_pot;
    int64_t total() const { return n_w0 + n_w1 + n_w2 + n_inv + n_pot; }
};

GeoPack geo_pack(const cdftb_operator* op, int64_t batch) {
    const int per16 = op->dtype == CDFTB_F32 ? 4 : 2;
    GeoPack g{};
    g.nzg = static_cast<int>(round_up(op->nz, per16));
    g.nz8g = static_cast<int>(round_up(op->nz + 8, per16));
    const int64_t nx = op->nx, ny = op->ny;
    const int64_t ng = geometry_systems(op, batch);
    g.n_w0 = round_up(ng * (nx + 8) * ny * g.nzg, per16);
    g.n_w1 = round_up(ng * nx * (ny + 8) * g.nzg, per16);
    g.n_w2 = round_up(ng * nx * ny * g.nz8g, per16);
    g.n_inv = round_up(ng * nx * ny * g.nzg, per16);
    g.n_pot = systems_of(op, batch) * nx * ny * g.nzg;
    return g;
}


// x chunks: one CTA per SM is resident and a CTA's time grows with the planes it marches (its
// chunk plus 14 halo planes), so pick the chunk count that minimises waves x planes.
int choose_chunk(int nx, int64_t ctas_per_chunkset, int sms) {
    int best = nx;
    int64_t best_cost = -1;
    for (int chunks = 1; chunks <= 16; ++chunks) {
        const int len = static_cast<int>(ceil_div(nx, chunks));
        if (chunks > 1 && len < 8) break;
        const int64_t waves = ceil_div(ctas_per_chunkset * ceil_div(nx, len), sms);
        const int64_t cost = waves * (len + 2 * HALO);
        if (best_cost < 0 || cost < best_cost) {
            best_cost = cost;
            best = len;
        }
    }
    return best;
}

int sm_count() {
    static int count = 0;
    if (count == 0) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || count <= 0)
            count = 148;
    }
    return count;
}

// Abort tokens: never 0, distinct between the two kernels (8-byte lanes 1 .. 2^30 - 1, wide lanes
// 2^30 .. 2^31 - 1), taken atomically so that launches from several host threads never share one.
std::atomic<unsigned> g_next_token{0};

unsigned next_launch_token(bool wide) {
    unsigned v = g_next_token.fetch_add(1u, std::memory_order_relaxed) & 0x3fffffffu;
    if (v == 0) v = g_next_token.fetch_add(1u, std::memory_order_relaxed) & 0x3fffffffu;
    return wide ? (0x40000000u | v) : v;
}

// The timeout test's one-shot setting (cdftb_filter_test_withhold): the next slab launch stops
// issuing copies after this many planes. 0: off.
std::atomic<int> g_test_stop_after{0};

int take_test_stop() { return g_test_stop_after.exchange(0, std::memory_order_relaxed); }

template <typename Lane, int TZ>
int launch_slab(const FilterMaps& maps, FilterArgs a, int64_t lanes, cudaStream_t stream, int xchunk = 0) {
    using SH = Shape<TZ, sizeof(typename Lane::S)>;
    static bool configured = false;
    if (!configured) {
        int st = check(cudaFuncSetAttribute(slab_filter_kernel<Lane, TZ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            static_cast<int>(SH::BYTES)));
        if (st != CDFTB_OK) return st;
        configured = true;
    }
    const int tiles_y = static_cast<int>(ceil_div(a.ny, TY));
    a.tiles_z = static_cast<int>(ceil_div(a.nzp, TZ));
    const int64_t tiles = int64_t(tiles_y) * a.tiles_z;
    a.xchunk = xchunk > 0 ? (xchunk < a.nx ? xchunk : a.nx) : choose_chunk(a.nx, tiles * lanes, sm_count());
    const int chunks = static_cast<int>(ceil_div(a.nx, a.xchunk));
    for (int64_t first = 0; first < lanes; first += 65535) {
        const int64_t count = (lanes - first) < 65535 ? (lanes - first) : 65535;
        a.lane_first = first;
        a.token = next_launch_token(false);
        a.stop_after_planes = take_test_stop();
        dim3 grid(static_cast<unsigned>(tiles), static_cast<unsigned>(chunks), static_cast<unsigned>(count));
        slab_filter_kernel<Lane, TZ><<<grid, SH::T, SH::BYTES, stream>>>(maps, a);
        int st = check_launch();
        if (st != CDFTB_OK) return st;
    }
    return CDFTB_OK;
}

template <typename S>
int pad_rows(const void* src, int64_t rows, int cols, int cols_pad, S* dst, cudaStream_t stream) {
    const int64_t total = rows * cols_pad;
    const unsigned blocks = static_cast<unsigned>(std::min<int64_t>(ceil_div(total, 256), 148 * 16));
    pad_rows_kernel<S><<<blocks, 256, 0, stream>>>(static_cast<const S*>(src), rows, cols, cols_pad, cols, dst);
    return check_launch();
}

// Copies the geometry into the padded rows TMA reads (at geo, element type S) and encodes the maps
// of the geometry; kinetic_only zeroes the potential rows instead of copying them.
template <typename Lane>
int prepare_geometry(const cdftb_operator* op, int64_t batch, void* geo_base, int ty, int tz, bool kinetic_only,
                     FilterMaps* maps, cudaStream_t stream) {
    using S = typename Lane::S;
    const int nx = op->nx, ny = op->ny, nz = op->nz;
    const GeoPack gp = geo_pack(op, batch);
    S* w0p = static_cast<S*>(geo_base);
    S* w1p = w0p + gp.n_w0;
    S* w2p = w1p + gp.n_w1;
    S* invp = w2p + gp.n_w2;
    S* potp = invp + gp.n_inv;
    const int64_t nsys = systems_of(op, batch);
    const int64_t ng = geometry_systems(op, batch);  // per-system arrays follow each other in memory
    int st;
    if ((st = pad_rows<S>(op->face_weights[0], ng * (nx + 8) * ny, nz, gp.nzg, w0p, stream)) != CDFTB_OK) return st;
    if ((st = pad_rows<S>(op->face_weights[1], ng * nx * (ny + 8), nz, gp.nzg, w1p, stream)) != CDFTB_OK) return st;
    if ((st = pad_rows<S>(op->face_weights[2], ng * nx * ny, nz + 8, gp.nz8g, w2p, stream)) != CDFTB_OK) return st;
    if ((st = pad_rows<S>(op->inverse_weight, ng * nx * ny, nz, gp.nzg, invp, stream)) != CDFTB_OK) return st;
    if (kinetic_only || !op->potential) {
        if ((st = check(cudaMemsetAsync(potp, 0, gp.n_pot * sizeof(S), stream))) != CDFTB_OK) return st;
    } else if (op->potential_stride == 0 || op->potential_stride == int64_t(nx) * ny * nz) {
        // every system's row block at once (rows of consecutive systems are consecutive)
        if ((st = pad_rows<S>(op->potential, nsys * nx * ny, nz, gp.nzg, potp, stream)) != CDFTB_OK) return st;
    } else {
        for (int64_t g = 0; g < nsys; ++g) {
            const void* src = static_cast<const S*>(op->potential) + g * op->potential_stride;
            if ((st = pad_rows<S>(src, int64_t(nx) * ny, nz, gp.nzg, potp + g * int64_t(nx) * ny * gp.nzg, stream)) !=
                CDFTB_OK)
                return st;
        }
    }
    const CUtensorMapDataType gt = Lane::GEO_TYPE;
    const int sb = sizeof(S);
    const unsigned tile_box[4] = {unsigned(tz), unsigned(ty), 1, 1};
    const int64_t d_w0[4] = {gp.nzg, ny, nx + 8, ng};
    const int64_t d_w1[4] = {gp.nzg, ny + 8, nx, ng};
    const unsigned b_w1[4] = {unsigned(tz), unsigned(ty + 7), 1, 1};
    const int64_t d_w2[4] = {gp.nz8g, ny, nx, ng};
    const unsigned b_w2[4] = {unsigned(tz + 8), unsigned(ty), 1, 1};
    const int64_t d_inv[4] = {gp.nzg, ny, nx, ng};
    const int64_t d_pot[4] = {gp.nzg, ny, nx, nsys};
    const unsigned b_pot[4] = {unsigned(tz), unsigned(ty), 1, 1};
    if ((st = encode_map(&maps->w0, gt, sb, 4, w0p, d_w0, tile_box)) != CDFTB_OK) return st;
    if ((st = encode_map(&maps->w1, gt, sb, 4, w1p, d_w1, b_w1)) != CDFTB_OK) return st;
    if ((st = encode_map(&maps->w2, gt, sb, 4, w2p, d_w2, b_w2)) != CDFTB_OK) return st;
    if ((st = encode_map(&maps->inv, gt, sb, 4, invp, d_inv, tile_box)) != CDFTB_OK) return st;
    return encode_map(&maps->pot, gt, sb, 4, potp, d_pot, b_pot);
}

template <typename Lane>
int pack_block(const cdftb_operator* op, const void* block, int in_dtype, int64_t batch, int nx, int ny, int nz,
               int nzp, int64_t lanes, void* dst, cudaStream_t stream) {
    // the lane buffers start 16-byte aligned (TMA needs it too) and a lane is an even number of points
    if ((reinterpret_cast<uintptr_t>(dst) & 15) != 0 || (nzp & 1) != 0) return CDFTB_ERR_ARGUMENT;
    const int64_t pairs = int64_t(nx) * ny * (nzp / 2);
    const unsigned ly = static_cast<unsigned>(std::min<int64_t>(lanes, 65535));
    const unsigned bx = static_cast<unsigned>(
        std::max<int64_t>(1, std::min<int64_t>(ceil_div(pairs, 256), ceil_div(int64_t(148) * 16, ly))));
    pack_lanes_kernel<Lane><<<dim3(bx, ly), 256, 0, stream>>>(block, in_dtype, batch, nx, ny, nz, nzp, lanes,
                                                        op->orbitals_per_group, aligned_lanes_per_group(op),
                                                        static_cast<typename Lane::E*>(dst));
    return check_launch();
}

int encode_lane_maps(void* buf, int nzp, int ny, int nx, int64_t lanes, int tz, CUtensorMap* phi, CUtensorMap* prev) {
    const int64_t lane_dims[4] = {nzp, ny, nx, lanes};
    const unsigned phi_box[4] = {unsigned(tz + 18), unsigned(NROW), 1, 1};
    const unsigned prev_box[4] = {unsigned(tz), unsigned(TY), 1, 1};
    int st = encode_map(phi, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, 4, buf, lane_dims, phi_box);
    if (st == CDFTB_OK) st = encode_map(prev, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, 4, buf, lane_dims, prev_box);
    return st;
}

FilterArgs base_args(const cdftb_operator* op, int64_t batch) {
    FilterArgs a{};
    a.nx = op->nx;
    a.ny = op->ny;
    a.nz = op->nz;
    a.nzp = padded_z(op->nz);
    a.batch = batch;
    a.orb_per_group = op->orbitals_per_group;
    a.shared_potential = op->potential_stride == 0;
    a.per_system_geometry = op->per_system_geometry != 0;
    a.system_shapes = op->per_system_geometry ? op->system_shapes : nullptr;
    a.lanes_per_group = aligned_lanes_per_group(op);
    const StaggeredTaps taps = staggered_taps(8);
    const double scale = 1.0 / op->spacing;  // taps c_k * (1/h), divergence.py:112, 121
    for (int j = 0; j < 8; ++j) a.taps[j] = taps.c[j] * scale;
    return a;
}

template <typename Lane>
int launch_any_tz(int tz, const FilterMaps& m, const FilterArgs& a, int64_t lanes, cudaStream_t stream,
                  int xchunk = 0) {
    return tz == 36 ? launch_slab<Lane, 36>(m, a, lanes, stream, xchunk)
                    : launch_slab<Lane, 32>(m, a, lanes, stream, xchunk);
}

// ---- wide lanes (slab_filter_wide_kernel): launch, lane maps, packing
bool g_wide = true;  // guarded by g_tune_mutex (declared below with the tuner)

template <typename W, int TYW, int TZ, bool GENERAL>
int launch_wide_as(const FilterMaps& maps, FilterArgs a, int64_t lanes, cudaStream_t stream, int xchunk) {
    using SH = WideShape<TYW, TZ, sizeof(typename W::S), W::ORB>;
    static bool configured = false;
    if (!configured) {
        int st = check(cudaFuncSetAttribute(slab_filter_wide_kernel<W, TYW, TZ, GENERAL>,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(SH::BYTES)));
        if (st != CDFTB_OK) return st;
        // a CTA this kernel's registers cannot hold is refused here, before any launch
        cudaFuncAttributes attr{};
        st = check(cudaFuncGetAttributes(&attr, slab_filter_wide_kernel<W, TYW, TZ, GENERAL>));
        if (st != CDFTB_OK) return st;
        if (attr.maxThreadsPerBlock < SH::T) return CDFTB_ERR_CAPACITY;
        configured = true;
    }
    const int tiles_y = static_cast<int>(ceil_div(a.ny, TYW));
    a.tiles_z = static_cast<int>(ceil_div(a.nzp, TZ));
    const int64_t tiles = int64_t(tiles_y) * a.tiles_z;
    a.xchunk = xchunk > 0 ? (xchunk < a.nx ? xchunk : a.nx) : choose_chunk(a.nx, tiles * lanes, sm_count());
    const int chunks = static_cast<int>(ceil_div(a.nx, a.xchunk));
    for (int64_t first = 0; first < lanes; first += 65535) {
        const int64_t count = (lanes - first) < 65535 ? (lanes - first) : 65535;
        a.lane_first = first;
        a.token = next_launch_token(true);
        a.stop_after_planes = take_test_stop();
        dim3 grid(static_cast<unsigned>(tiles), static_cast<unsigned>(chunks), static_cast<unsigned>(count));
        slab_filter_wide_kernel<W, TYW, TZ, GENERAL><<<grid, SH::T, SH::BYTES, stream>>>(maps, a);
        int st = check_launch();
        if (st != CDFTB_OK) return st;
    }
    return CDFTB_OK;
}

// Lanes aligned to orbital groups (per-system geometry) take the general instantiation, and so do
// the float64 lanes in 8-row tiles: there the general kernels keep every value in registers, where
// the in-order ones spill 4 bytes (16 He 65^3 systems, 8 x 36: 257.7 against 262.1 us per step).
// Elsewhere the in-order kernels are the faster ones (float32, 128 systems, 13 x 24: 1102 against
// 1124 us; float64, one system, 13 x 24: 33.3 against 34.1 us).
template <typename W, int TYW, int TZ>
int launch_wide(const FilterMaps& maps, const FilterArgs& a, int64_t lanes, cudaStream_t stream, int xchunk = 0) {
    if constexpr (W::ORB == 2 && TYW == 8) {
        return launch_wide_as<W, TYW, TZ, true>(maps, a, lanes, stream, xchunk);
    } else {
        return a.lanes_per_group > 0 ? launch_wide_as<W, TYW, TZ, true>(maps, a, lanes, stream, xchunk)
                                     : launch_wide_as<W, TYW, TZ, false>(maps, a, lanes, stream, xchunk);
    }
}

// Lane buffers of 16-byte points described as 8-byte elements, two per point.
int encode_wide_lane_maps(void* buf, int nzp, int ny, int nx, int64_t lanes, int ty, int tz, CUtensorMap* phi,
                          CUtensorMap* prev) {
    const int64_t lane_dims[4] = {2 * int64_t(nzp), ny, nx, lanes};
    const unsigned phi_box[4] = {unsigned(2 * (tz + 19)), unsigned(ty + 2 * HALO), 1, 1};  // WideShape::BW points
    const unsigned prev_box[4] = {unsigned(2 * tz), unsigned(ty), 1, 1};
    int st = encode_map(phi, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, 4, buf, lane_dims, phi_box);
    if (st == CDFTB_OK) st = encode_map(prev, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, 4, buf, lane_dims, prev_box);
    return st;
}

template <typename W>
int pack_wide(const void* block, int in_dtype, int64_t batch, int nx, int ny, int nz, int nzp, int64_t lanes,
              int opg, int lpg, void* dst, cudaStream_t stream) {
    if ((reinterpret_cast<uintptr_t>(dst) & 15) != 0) return CDFTB_ERR_ARGUMENT;
    const int64_t per_lane = int64_t(nx) * ny * nzp;
    const unsigned ly = static_cast<unsigned>(std::min<int64_t>(lanes, 65535));
    const unsigned bx = static_cast<unsigned>(
        std::max<int64_t>(1, std::min<int64_t>(ceil_div(per_lane, 256), ceil_div(int64_t(148) * 16, ly))));
    pack_wide_kernel<W><<<dim3(bx, ly), 256, 0, stream>>>(block, in_dtype, batch, nx, ny, nz, nzp, lanes, opg, lpg,
                                                          static_cast<typename W::E*>(dst));
    return check_launch();
}

// The same steps for both lane layouts: two-orbital (LaneF2) or one-orbital (LaneD) lane points of
// 8 bytes, or wide ones of 16 bytes (WideF4, WideD2).
// Wide lanes per orbital group when lanes are aligned to groups (per-system geometry), else 0.
int wide_lanes_per_group(const cdftb_operator* op, int orbitals) {
    return op->per_system_geometry ? static_cast<int>(ceil_div(op->orbitals_per_group, orbitals)) : 0;
}

template <typename L>
int64_t lane_count(const cdftb_operator* op, int64_t batch) {
    if constexpr (L::WIDE) {
        const int lpg = wide_lanes_per_group(op, L::ORB);
        return lpg > 0 ? ceil_div(batch, op->orbitals_per_group) * lpg : ceil_div(batch, L::ORB);
    } else {
        return lanes_of(op, batch);
    }
}

// The call's arguments for lane layout L (the wide layouts align their own lanes to groups).
template <typename L>
FilterArgs lane_args(const cdftb_operator* op, int64_t batch) {
    FilterArgs a = base_args(op, batch);
    if constexpr (L::WIDE) a.lanes_per_group = wide_lanes_per_group(op, L::ORB);
    return a;
}

template <typename L>
constexpr int64_t lane_point_bytes() {
    return L::WIDE ? 16 : 8;
}

template <typename L>
int encode_lanes(void* buf, int nzp, int ny, int nx, int64_t lanes, int ty, int tz, CUtensorMap* phi,
                 CUtensorMap* prev) {
    if constexpr (L::WIDE)
        return encode_wide_lane_maps(buf, nzp, ny, nx, lanes, ty, tz, phi, prev);
    else
        return encode_lane_maps(buf, nzp, ny, nx, lanes, tz, phi, prev);
}

template <typename L>
int pack_lanes(const cdftb_operator* op, const void* block, int in_dtype, int64_t batch, int nx, int ny, int nz,
               int nzp, int64_t lanes, void* dst, cudaStream_t stream) {
    if constexpr (L::WIDE)
        return pack_wide<L>(block, in_dtype, batch, nx, ny, nz, nzp, lanes, op->orbitals_per_group,
                            wide_lanes_per_group(op, L::ORB), dst, stream);
    else
        return pack_block<L>(op, block, in_dtype, batch, nx, ny, nz, nzp, lanes, dst, stream);
}

// The tilings (rows TY x columns TZ) each lane layout has: the 8-byte-lane kernel 8 x 32 and 8 x 36;
// the wide kernel also 13 x 24 (65 rows in five tiles, 66 columns in three: He at h = 0.25).
struct Tile {
    int ty, tz;
};
constexpr Tile kNarrowTiles[] = {{8, 32}, {8, 36}};
constexpr Tile kWideTiles[] = {{8, 32}, {8, 36}, {13, 24}};

template <typename L>
int launch_tz(int ty, int tz, const FilterMaps& m, const FilterArgs& a, int64_t lanes, cudaStream_t stream,
              int xchunk = 0) {
    if constexpr (L::WIDE) {
        if (ty == 13) return launch_wide<L, 13, 24>(m, a, lanes, stream, xchunk);
        return tz == 36 ? launch_wide<L, 8, 36>(m, a, lanes, stream, xchunk)
                        : launch_wide<L, 8, 32>(m, a, lanes, stream, xchunk);
    } else {
        return launch_any_tz<L>(tz, m, a, lanes, stream, xchunk);
    }
}

// The tiling that wastes the fewest padded points (ties: the earlier entry).
template <typename L>
Tile choose_tile(int ny, int nzp) {
    Tile best = L::WIDE ? kWideTiles[0] : kNarrowTiles[0];
    int64_t best_pts = -1;
    const Tile* list = L::WIDE ? kWideTiles : kNarrowTiles;
    const int count = L::WIDE ? 3 : 2;
    for (int i = 0; i < count; ++i) {
        const int64_t pts = ceil_div(ny, list[i].ty) * list[i].ty * ceil_div(nzp, list[i].tz) * list[i].tz;
        if (best_pts < 0 || pts < best_pts) {
            best_pts = pts;
            best = list[i];
        }
    }
    return best;
}

// ---- the tile autotuner
// The tile (8 x 32, 8 x 36, and for the wide kernel 13 x 24 rows x columns) and the x chunk of a slab
// launch decide the CTA count, the waves, the padding and the halo work; which wins depends on the
// grid, the lane count and the GPU. With the autotuner
// on, the first filter call for a (device, grid, precision, lanes) key times every candidate on the
// call's own buffers (the first Chebyshev step, which the real run then recomputes), keeps the
// fastest in a host table, and every later filter or apply launch for that key uses it. Every
// candidate gives bit-identical results: each output is formed by the same arithmetic in the same
// order whatever the tiling. Off, the heuristics choose_tile / choose_chunk decide.
struct TileChoice {
    int ty;
    int tz;
    int xchunk;  // 0: choose_chunk
};

// device, nx, ny, nz, precision (+ CDFTB_WIDE_LANES for the wide kernel), lanes
using TuneKey = std::tuple<int, int, int, int, int, int64_t>;
std::mutex g_tune_mutex;
std::map<TuneKey, TileChoice> g_tuned;
bool g_autotune = false;

TuneKey tune_key(const cdftb_operator* op, int64_t lanes, bool wide) {
    int dev = 0;
    cudaGetDevice(&dev);
    return TuneKey(dev, op->nx, op->ny, op->nz, op->dtype + (wide ? CDFTB_WIDE_LANES : 0), lanes);
}

bool tuned_choice(const TuneKey& key, TileChoice* out) {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    auto it = g_tuned.find(key);
    if (it == g_tuned.end()) return false;
    *out = it->second;
    return true;
}

// Times every candidate tiling: one untimed launch, then three timed ones each. With apply null,
// the launch is the first Chebyshev step (packed block in buf[2] -> buf[0]); otherwise it is the
// apply described by *apply (packed block in buf[2], written to the caller's output, which the
// real launch then rewrites). Synchronises the stream.
template <typename Lane>
int tune_slab(const cdftb_operator* op, int64_t batch, void* geo_base, void* buf[3], int64_t lanes,
              const double* coefficients, int degree, cudaStream_t stream, TileChoice* best,
              const FilterArgs* apply = nullptr) {
    const int nx = op->nx, ny = op->ny, nzp = padded_z(op->nz);
    cudaEvent_t e0, e1;
    int st = check(cudaEventCreate(&e0));
    if (st != CDFTB_OK) return st;
    if ((st = check(cudaEventCreate(&e1))) != CDFTB_OK) {
        cudaEventDestroy(e0);
        return st;
    }
    float best_ms = -1.0f;
    const Tile t0 = choose_tile<Lane>(ny, nzp);
    *best = TileChoice{t0.ty, t0.tz, 0};
    const Tile* list = Lane::WIDE ? kWideTiles : kNarrowTiles;
    const int count = Lane::WIDE ? 3 : 2;
    for (int ti = 0; ti < count; ++ti) {
        const int ty = list[ti].ty, tz = list[ti].tz;
        FilterMaps m{};
        const bool kinetic = apply != nullptr && apply->kinetic_only;
        if ((st = prepare_geometry<Lane>(op, batch, geo_base, ty, tz, kinetic, &m, stream)) != CDFTB_OK) break;
        if ((st = encode_lanes<Lane>(buf[2], nzp, ny, nx, lanes, ty, tz, &m.phi, &m.prev)) != CDFTB_OK) break;
        FilterArgs a = lane_args<Lane>(op, batch);
        if (apply) {
            a = *apply;
        } else {
            a.coef = coefficients;
            a.degree = degree;
            a.step = 0;
            a.has_prev = 0;
            a.final_out = 0;
            a.out = buf[0];
            a.out_dtype = 0;
        }
        const int64_t tiles = int64_t(ceil_div(ny, ty)) * ceil_div(nzp, tz);
        int chunks_list[5] = {1, 2, 3, 4, 0};
        chunks_list[4] = static_cast<int>(ceil_div(nx, choose_chunk(nx, tiles * lanes, sm_count())));
        for (int c = 0; c < 5 && st == CDFTB_OK; ++c) {
            const int chunks = chunks_list[c];
            if (chunks < 1 || (c == 4 && chunks <= 4)) continue;  // the heuristic's chunk, when not already tried
            const int xchunk = static_cast<int>(ceil_div(nx, chunks));
            if (chunks > 1 && (xchunk < 8 || ceil_div(nx, xchunk) != chunks)) continue;
            if ((st = launch_tz<Lane>(ty, tz, m, a, lanes, stream, xchunk)) != CDFTB_OK) break;
            if ((st = check(cudaEventRecord(e0, stream))) != CDFTB_OK) break;
            for (int r = 0; r < 3 && st == CDFTB_OK; ++r) st = launch_tz<Lane>(ty, tz, m, a, lanes, stream, xchunk);
            if (st != CDFTB_OK) break;
            if ((st = check(cudaEventRecord(e1, stream))) != CDFTB_OK) break;
            if ((st = check(cudaEventSynchronize(e1))) != CDFTB_OK) break;
            float ms = 0.0f;
            if ((st = check(cudaEventElapsedTime(&ms, e0, e1))) != CDFTB_OK) break;
            if (best_ms < 0.0f || ms < best_ms) {
                best_ms = ms;
                *best = TileChoice{ty, tz, xchunk};
            }
        }
        if (st != CDFTB_OK) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return st;
}

template <typename Lane>
int slab_filter(const cdftb_operator* op, const void* block, int in_dtype, void* out, int out_dtype, void* work,
                int64_t batch, const double* coefficients, int degree, cudaStream_t stream) {
    const int nx = op->nx, ny = op->ny, nz = op->nz;
    const int nzp = padded_z(nz);
    const int64_t lanes = lane_count<Lane>(op, batch);
    const int64_t lane_bytes = int64_t(nx) * ny * nzp * lane_point_bytes<Lane>();
    char* w = static_cast<char*>(work);
    void* buf[3] = {w, w + lanes * lane_bytes, w + 2 * lanes * lane_bytes};
    int st = pack_lanes<Lane>(op, block, in_dtype, batch, nx, ny, nz, nzp, lanes, buf[2], stream);
    if (st != CDFTB_OK) return st;
    const Tile t0 = choose_tile<Lane>(ny, nzp);
    TileChoice choice{t0.ty, t0.tz, 0};
    const TuneKey key = tune_key(op, lanes, Lane::WIDE);
    bool autotune;
    {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        autotune = g_autotune;
    }
    if (!tuned_choice(key, &choice) && autotune) {
        if ((st = tune_slab<Lane>(op, batch, w + 3 * lanes * lane_bytes, buf, lanes, coefficients, degree, stream,
                                  &choice)) != CDFTB_OK)
            return st;
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        g_tuned[key] = choice;
    }
    const int ty = choice.ty, tz = choice.tz;
    FilterMaps geo_maps{};
    if ((st = prepare_geometry<Lane>(op, batch, w + 3 * lanes * lane_bytes, ty, tz, false, &geo_maps, stream)) !=
        CDFTB_OK)
        return st;
    FilterMaps maps[3];
    for (int b = 0; b < 3; ++b)
        if ((st = encode_lanes<Lane>(buf[b], nzp, ny, nx, lanes, ty, tz, &maps[b].phi, &maps[b].prev)) != CDFTB_OK)
            return st;
    FilterArgs a = lane_args<Lane>(op, batch);
    a.coef = coefficients;
    a.degree = degree;
    // Y_1 -> buf0, Y_2 -> buf1, then Y_{k+1} overwrites Y_{k-1} in place (a point's previous value
    // is read only by the CTA that writes that point); the packed block is buf2.
    int y = 2, prev = -1;
    for (int k = 1; k <= degree; ++k) {
        const int dst = (k == 1) ? 0 : (k == 2 ? 1 : prev);
        a.has_prev = prev >= 0;
        a.step = k - 1;
        a.final_out = k == degree;
        a.out = a.final_out ? out : buf[dst];
        a.out_dtype = out_dtype;
        FilterMaps m = geo_maps;
        m.phi = maps[y].phi;
        m.prev = maps[prev >= 0 ? prev : y].prev;
        if ((st = launch_tz<Lane>(ty, tz, m, a, lanes, stream, choice.xchunk)) != CDFTB_OK) return st;
        prev = y;
        y = dst;
    }
    return CDFTB_OK;
}

template <typename Lane>
int slab_apply(const cdftb_operator* op, const void* phi, int in_dtype, void* out, int out_dtype, void* work,
               int64_t batch, int kinetic_only, cudaStream_t stream) {
    const int nx = op->nx, ny = op->ny, nz = op->nz;
    const int nzp = padded_z(nz);
    const int64_t lanes = lane_count<Lane>(op, batch);
    const int64_t lane_bytes = int64_t(nx) * ny * nzp * lane_point_bytes<Lane>();
    char* w = static_cast<char*>(work);
    const Tile t0 = choose_tile<Lane>(ny, nzp);
    TileChoice choice{t0.ty, t0.tz, 0};
    const TuneKey key = tune_key(op, lanes, Lane::WIDE);
    const bool known = tuned_choice(key, &choice);
    int st = pack_lanes<Lane>(op, phi, in_dtype, batch, nx, ny, nz, nzp, lanes, w, stream);
    if (st != CDFTB_OK) return st;
    bool autotune;
    {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        autotune = g_autotune;
    }
    if (!known && autotune) {
        FilterArgs t = lane_args<Lane>(op, batch);
        t.apply_only = 1;
        t.kinetic_only = kinetic_only != 0;
        t.degree = 1;
        t.final_out = 1;
        t.out = out;
        t.out_dtype = out_dtype;
        void* bufs[3] = {nullptr, nullptr, w};
        if ((st = tune_slab<Lane>(op, batch, w + lanes * lane_bytes, bufs, lanes, nullptr, 1, stream, &choice, &t)) !=
            CDFTB_OK)
            return st;
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        g_tuned[key] = choice;
    }
    const int ty = choice.ty, tz = choice.tz;
    FilterMaps m{};
    if ((st = prepare_geometry<Lane>(op, batch, w + lanes * lane_bytes, ty, tz, kinetic_only != 0, &m, stream)) !=
        CDFTB_OK)
        return st;
    if ((st = encode_lanes<Lane>(w, nzp, ny, nx, lanes, ty, tz, &m.phi, &m.prev)) != CDFTB_OK) return st;
    FilterArgs a = lane_args<Lane>(op, batch);
    a.apply_only = 1;
    a.kinetic_only = kinetic_only != 0;
    a.degree = 1;
    a.final_out = 1;
    a.out = out;
    a.out_dtype = out_dtype;
    return launch_tz<Lane>(ty, tz, m, a, lanes, stream, choice.xchunk);
}

// Wide lanes serve every filter and apply with one shared geometry (lanes need not follow orbital
// groups). Measured on He 65^3 they were faster at every batch tried, from one system of 5 orbitals
// (2 or 3 wide lanes) to 32 systems.
bool wide_applies(const cdftb_operator* op, int64_t batch) {
    bool on;
    {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        on = g_wide;
    }
    return on && batch > 0;
}

// Lane bytes of the larger layout a call may use (the wide one when it can apply).
int64_t lane_bytes_total(const cdftb_operator* op, int64_t batch) {
    const int64_t points = int64_t(op->nx) * op->ny * padded_z(op->nz);
    int64_t total = lanes_of(op, batch) * points * 8;
    const int64_t wide = op->dtype == CDFTB_F32 ? lane_count<WideF4>(op, batch) : lane_count<WideD2>(op, batch);
    return std::max<int64_t>(total, wide * points * 16);
}

}  // namespace

int64_t slab_filter_work_bytes(const cdftb_operator* op, int64_t batch) {
    const int64_t sb = op->dtype == CDFTB_F32 ? 4 : 8;
    return 3 * lane_bytes_total(op, batch) + geo_pack(op, batch).total() * sb;
}

bool slab_filter_applies(const cdftb_operator* op) {
    return op->accuracy == 8 && (op->dtype == CDFTB_F32 || op->dtype == CDFTB_F64) && op->nx > 0 && op->ny > 0 &&
           op->nz > 0;
}

int64_t slab_apply_work_bytes(const cdftb_operator* op, int64_t batch) {
    const int64_t sb = op->dtype == CDFTB_F32 ? 4 : 8;
    return lane_bytes_total(op, batch) + geo_pack(op, batch).total() * sb;
}

int slab_chebyshev_filter(const cdftb_operator* op, const void* block, int in_dtype, void* out, int out_dtype,
                          void* work, int64_t batch, const double* coefficients, int degree, cudaStream_t stream) {
    if (wide_applies(op, batch)) {
        if (op->dtype == CDFTB_F32)
            return slab_filter<WideF4>(op, block, in_dtype, out, out_dtype, work, batch, coefficients, degree, stream);
        return slab_filter<WideD2>(op, block, in_dtype, out, out_dtype, work, batch, coefficients, degree, stream);
    }
    if (op->dtype == CDFTB_F32)
        return slab_filter<LaneF2>(op, block, in_dtype, out, out_dtype, work, batch, coefficients, degree, stream);
    return slab_filter<LaneD>(op, block, in_dtype, out, out_dtype, work, batch, coefficients, degree, stream);
}

}  // namespace cdftb

extern "C" int cdftb_filter_autotune(int enable) {
    std::lock_guard<std::mutex> lock(cdftb::g_tune_mutex);
    cdftb::g_autotune = enable != 0;
    return CDFTB_OK;
}

extern "C" int cdftb_filter_wide(int enable) {
    std::lock_guard<std::mutex> lock(cdftb::g_tune_mutex);
    cdftb::g_wide = enable != 0;
    return CDFTB_OK;
}

extern "C" int cdftb_filter_tuned_tile(int nx, int ny, int nz, int dtype, int64_t lanes, int* tile_z, int* x_chunk) {
    if (!tile_z || !x_chunk || nx <= 0 || ny <= 0 || nz <= 0 || lanes <= 0) return CDFTB_ERR_ARGUMENT;
    int dev = 0;
    int st = cdftb::check(cudaGetDevice(&dev));
    if (st != CDFTB_OK) return st;
    cdftb::TileChoice c{};
    if (!cdftb::tuned_choice(cdftb::TuneKey(dev, nx, ny, nz, dtype, lanes), &c)) {
        *tile_z = 0;
        *x_chunk = 0;
        return CDFTB_OK;
    }
    *tile_z = c.tz;
    *x_chunk = c.xchunk;
    return CDFTB_OK;
}

extern "C" int cdftb_filter_tuned_tile_rows(int nx, int ny, int nz, int dtype, int64_t lanes, int* tile_y) {
    if (!tile_y || nx <= 0 || ny <= 0 || nz <= 0 || lanes <= 0) return CDFTB_ERR_ARGUMENT;
    int dev = 0;
    int st = cdftb::check(cudaGetDevice(&dev));
    if (st != CDFTB_OK) return st;
    cdftb::TileChoice c{};
    *tile_y = cdftb::tuned_choice(cdftb::TuneKey(dev, nx, ny, nz, dtype, lanes), &c) ? c.ty : 0;
    return CDFTB_OK;
}

extern "C" int cdftb_filter_test_withhold(int planes) {
    if (planes < 0) return CDFTB_ERR_ARGUMENT;
    cdftb::g_test_stop_after.store(planes, std::memory_order_relaxed);
    return CDFTB_OK;
}

extern "C" int cdftb_device_status(int* flags) {
    if (!flags) return CDFTB_ERR_ARGUMENT;
    int v = 0;
    int st = cdftb::check(cudaMemcpyFromSymbol(&v, cdftb::g_device_error, sizeof(int)));
    if (st != CDFTB_OK) return st;
    *flags = v;
    if (v) {
        const int zero = 0;
        st = cdftb::check(cudaMemcpyToSymbol(cdftb::g_device_error, &zero, sizeof(int)));
        if (st != CDFTB_OK) return st;
    }
    return v ? CDFTB_ERR_TIMEOUT : CDFTB_OK;
}

extern "C" int64_t cdftb_chebyshev_filter_work_bytes(const cdftb_operator* op, int64_t batch) {
    if (!op || batch <= 0 || op->nx <= 0 || op->ny <= 0 || op->nz <= 0) return 0;
    if (cdftb::slab_filter_applies(op)) return cdftb::slab_filter_work_bytes(op, batch);
    const int64_t esize = op->dtype == CDFTB_F64 ? 8 : 4;
    return 3 * batch * int64_t(op->nx) * op->ny * op->nz * esize;
}

extern "C" int cdftb_chebyshev_filter(const cdftb_operator* op, const void* block, int in_dtype, void* out,
                                      int out_dtype, void* work, int64_t work_bytes, int64_t batch,
                                      const double* coefficients, int degree, cdftb_stream_t stream) {
    if (!op || !block || !out || !work || !coefficients || degree < 1 || batch < 0) return CDFTB_ERR_ARGUMENT;
    if (batch == 0) return CDFTB_OK;
    if (op->nx <= 0 || op->ny <= 0 || op->nz <= 0 || !(op->spacing > 0.0)) return CDFTB_ERR_ARGUMENT;
    if (work_bytes < cdftb_chebyshev_filter_work_bytes(op, batch)) return CDFTB_ERR_ARGUMENT;
    if (op->dtype != CDFTB_F64 && op->dtype != CDFTB_F32) return CDFTB_ERR_ARGUMENT;
    if ((in_dtype != CDFTB_F64 && in_dtype != CDFTB_F32) || (out_dtype != CDFTB_F64 && out_dtype != CDFTB_F32))
        return CDFTB_ERR_ARGUMENT;
    if (!op->face_weights[0] || !op->face_weights[1] || !op->face_weights[2] || !op->inverse_weight ||
        !op->potential || op->orbitals_per_group <= 0)
        return CDFTB_ERR_ARGUMENT;
    if (reinterpret_cast<uintptr_t>(work) % 16 != 0) return CDFTB_ERR_ARGUMENT;
    if (cdftb::slab_filter_applies(op))
        return cdftb::slab_chebyshev_filter(op, block, in_dtype, out, out_dtype, work, batch, coefficients, degree,
                                            cdftb::as_stream(stream));
    if (op->per_system_geometry) return CDFTB_ERR_ARGUMENT;  // the generic stencil shares one geometry
    return cdftb::generic_chebyshev_filter(op, block, in_dtype, out, out_dtype, work, batch, coefficients, degree,
                                           stream);
}

extern "C" int64_t cdftb_cusp_apply_work_bytes(const cdftb_operator* op, int64_t batch) {
    if (!op || batch <= 0 || op->nx <= 0 || op->ny <= 0 || op->nz <= 0) return 0;
    return cdftb::slab_filter_applies(op) ? cdftb::slab_apply_work_bytes(op, batch) : 0;
}

extern "C" int cdftb_cusp_apply(const cdftb_operator* op, const void* phi, int in_dtype, void* out, int out_dtype,
                                int64_t batch, int kinetic_only, void* work, int64_t work_bytes,
                                cdftb_stream_t stream) {
    if (!op || !phi || !out || batch < 0) return CDFTB_ERR_ARGUMENT;
    if (batch == 0) return CDFTB_OK;
    const bool slab = work && cdftb::slab_filter_applies(op) && work_bytes >= cdftb_cusp_apply_work_bytes(op, batch) &&
                      reinterpret_cast<uintptr_t>(work) % 16 == 0 && op->spacing > 0.0 && op->face_weights[0] &&
                      op->face_weights[1] && op->face_weights[2] && op->inverse_weight &&
                      (kinetic_only || (op->potential && op->orbitals_per_group > 0)) &&
                      (in_dtype == CDFTB_F64 || in_dtype == CDFTB_F32) &&
                      (out_dtype == CDFTB_F64 || out_dtype == CDFTB_F32);
    if (!slab) {
        if (op->per_system_geometry) return CDFTB_ERR_ARGUMENT;  // the generic stencil shares one geometry
        return cdftb::generic_cusp_apply(op, phi, in_dtype, out, out_dtype, batch, kinetic_only, stream);
    }
    cudaStream_t s = cdftb::as_stream(stream);
    if (cdftb::wide_applies(op, batch)) {
        if (op->dtype == CDFTB_F32)
            return cdftb::slab_apply<cdftb::WideF4>(op, phi, in_dtype, out, out_dtype, work, batch, kinetic_only, s);
        return cdftb::slab_apply<cdftb::WideD2>(op, phi, in_dtype, out, out_dtype, work, batch, kinetic_only, s);
    }
    if (op->dtype == CDFTB_F32)
        return cdftb::slab_apply<cdftb::LaneF2>(op, phi, in_dtype, out, out_dtype, work, batch, kinetic_only, s);
    return cdftb::slab_apply<cdftb::LaneD>(op, phi, in_dtype, out, out_dtype, work, batch, kinetic_only, s);
}
