/*
 * cdftb: the B200 (sm_100a) kernels of the cdft hot path behind a plain C ABI.
 *
 * Every entry point takes raw device pointers, sizes and a CUDA stream, enqueues its work on that
 * stream and returns a status code (CDFTB_OK = 0). No entry point synchronises the device or
 * allocates memory unless its comment says so; scratch buffers are passed in by the caller, sized
 * by the matching *_scratch_bytes query. Arrays are C-ordered; a grid field is (nx, ny, nz) with z
 * contiguous; a block of orbitals is (batch, nx*ny*nz). Reference interfaces each entry point
 * replaces are cited as path:line inside the reference project (VaclavSvo/Density-functional-
 * theory-on-real-space-grids).
 */
#ifndef CDFTB_H
#define CDFTB_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* cdftb_stream_t; /* a cudaStream_t */

enum cdftb_status {
    CDFTB_OK = 0,
    CDFTB_ERR_ARGUMENT = 1,     /* bad shape, null pointer, unsupported order or dtype */
    CDFTB_ERR_LAUNCH = 2,       /* a CUDA launch or runtime call failed (cdftb_last_cuda_error) */
    CDFTB_ERR_NOT_POSITIVE = 3, /* a Gram matrix was not positive definite (Cholesky failed) */
    CDFTB_ERR_TIMEOUT = 4,      /* a bounded device-side wait gave up */
    CDFTB_ERR_CAPACITY = 5      /* a size exceeds a compiled limit */
};

enum cdftb_dtype { CDFTB_F64 = 0, CDFTB_F32 = 1 };

/* Added to a dtype in the tuned-tile query (cdftb_filter_tuned_tile) for the wide-lane kernels. */
enum { CDFTB_WIDE_LANES = 16 };

/* Library version (major*10000 + minor*100 + patch) and the status text. */
int cdftb_version(void);
const char* cdftb_status_string(int status);
/* The cudaError_t of the last failed CUDA call made by this library on this host thread. */
int cdftb_last_cuda_error(void);
/* Number of kernels this library has launched in this process (for launch accounting). */
unsigned long long cdftb_launch_count(void);

/*
 * The cusp-factorised operator A = (1/2 w) sum_d D_d^T [f^2_face,d D_d .] + V on one grid.
 * face_weights[d] has the grid shape extended by `accuracy` along d, indexed from face -accuracy/2
 * (src/cdft/operators/cusp.py:168-214); inverse_weight = h^3/omega (N); potential = V (N per
 * group, groups `potential_stride` elements apart; orbital b uses group b / orbitals_per_group).
 * `dtype` says whether the weight and potential arrays are double or float. The measure
 * `quadrature` (omega, N, always double) is used by the reductions.
 * per_system_geometry = 1: face_weights[d] and inverse_weight hold one array per orbital group,
 * back to back (systems on their own grids, embedded in a common box with zero weights, zero
 * h^3/omega and zero potential outside each system); only the order-8 slab paths take it.
 */
typedef struct cdftb_operator {
    int nx, ny, nz;
    int accuracy;          /* staggered order, 2..8, even */
    double spacing;
    int dtype;             /* enum cdftb_dtype of face_weights / inverse_weight / potential */
    const void* face_weights[3];
    const void* inverse_weight;
    const void* potential;
    int64_t potential_stride;
    int orbitals_per_group;
    const double* quadrature;
    int per_system_geometry;
    /* With per_system_geometry: each orbital group's own grid (nx, ny, nz), 3 ints per group in
     * device memory, or NULL. A system sits at the low corner of the operator's box and is zero
     * beyond its own grid; the slab kernel's CTAs whose tile lies wholly beyond it store zeros and
     * compute nothing. No reference counterpart: the reference solves one grid at a time. */
    const int* system_shapes;
} cdftb_operator;

/* (a1) out = sum_d D_d^T [w_d D_d box], f64, batched.
 * Replaces src/cdft/operators/divergence.py:153 weighted_divergence and the CUDA dispatch
 * src/cdft/operators/fused.py:353 device_weighted_divergence. */
int cdftb_weighted_divergence_f64(const double* box, double* out, int64_t batch, int nx, int ny, int nz,
                                  const double* w0, const double* w1, const double* w2, double spacing,
                                  int accuracy, cdftb_stream_t stream);

/* (a2) out = A phi for a batch of orbitals (src/cdft/operators/hamiltonian.py:251-318,
 * apply / apply_with_potential / kinetic_apply). out may be double or float (out_dtype).
 * kinetic_only = 1 drops the V phi term (hamiltonian.py:303). With device scratch of at least
 * cdftb_cusp_apply_work_bytes(op, batch) bytes (work, work_bytes; non-zero only for order 8) the
 * apply runs as one launch of the slab kernel (phi in either dtype); with work NULL it runs the
 * generic stencil on the caller's layout (phi must then be in the operator's dtype). */
int64_t cdftb_cusp_apply_work_bytes(const cdftb_operator* op, int64_t batch);
int cdftb_cusp_apply(const cdftb_operator* op, const void* phi, int in_dtype, void* out, int out_dtype,
                     int64_t batch, int kinetic_only, void* work, int64_t work_bytes, cdftb_stream_t stream);

/* Slab tile of the apply/filter kernels, process-wide: tile_y rows (4, 8 or 16) of 32 z columns per
 * CTA, x chunks no shorter than min_chunk planes, about ctas_per_sm CTAs per SM. Chosen by the
 * host autotuner; no reference counterpart (the reference has no kernels of its own). */
int cdftb_stencil_set_tile(int tile_y, int min_chunk, int ctas_per_sm);

/* (b) The scaled Chebyshev filter of degree `degree` (src/cdft/eigen/chefsi.py:81-160,
 * chebyshev_filter / chebyshev_recurrence, with fused.py:391 chebyshev_update fused into each apply).
 * coefficients: device table (groups, degree, 3) of rows (c, a_k, b_k) from chefsi.py:116
 * chebyshev_coefficients, one table per potential group. block and out are in_dtype/out_dtype
 * (a double block with a float operator is cast once); work is device scratch of at least
 * cdftb_chebyshev_filter_work_bytes(op, batch) bytes, given as work_bytes. The input block is never
 * written. Order 8 runs the slab filter (internal layout: lanes of 16-byte points holding four
 * float32 or two float64 orbitals, or with per-system geometry 8-byte points of two float32 or one
 * float64; z padded to even; TMA-staged tiles, bounded waits reported by cdftb_device_status); other
 * orders run one stencil launch per step on the caller's layout. */
int64_t cdftb_chebyshev_filter_work_bytes(const cdftb_operator* op, int64_t batch);
int cdftb_chebyshev_filter(const cdftb_operator* op, const void* block, int in_dtype, void* out, int out_dtype,
                           void* work, int64_t work_bytes, int64_t batch, const double* coefficients, int degree,
                           cdftb_stream_t stream);

/* No reference counterpart (the reference has no kernels of its own to tune): the tile autotuner of
 * the order-8 slab kernels. With it enabled, the first cdftb_chebyshev_filter or cdftb_cusp_apply
 * call for a (device, grid, precision, lane count) key times each candidate tiling -- z tiles of 32
 * or 36 columns, 1 to 4 x chunks and the heuristic's chunk -- on that call's own buffers, keeps the
 * fastest, and every later filter or apply launch for the key uses it. That first call synchronises
 * its stream (make it before any stream capture); results are bit-identical whatever the tiling. Disabled (the
 * default in the C library), heuristics choose the tiling. cdftb_filter_tuned_tile reports the
 * table's entry for a key (tile_z 32, 36 or 24, x_chunk in planes; both 0 when the key is not tuned)
 * and cdftb_filter_tuned_tile_rows its tile rows (8, or 13 for the wide kernel's 13 x 24 tile; 0 when
 * not tuned);
 * dtype is CDFTB_F32 or CDFTB_F64 and lanes is the launch's lane count (cdftb_operator orbitals in
 * pairs for float32, one each for float64); for the wide-lane kernels (cdftb_filter_wide) dtype is
 * CDFTB_F32 + CDFTB_WIDE_LANES or CDFTB_F64 + CDFTB_WIDE_LANES and lanes counts four float32 or two
 * float64 orbitals each. */
int cdftb_filter_autotune(int enable);
int cdftb_filter_tuned_tile(int nx, int ny, int nz, int dtype, int64_t lanes, int* tile_z, int* x_chunk);
int cdftb_filter_tuned_tile_rows(int nx, int ny, int nz, int dtype, int64_t lanes, int* tile_y);

/* No reference counterpart: wide lanes for cdftb_chebyshev_filter and cdftb_cusp_apply. Enabled
 * (the default), every order-8 call with one shared geometry (no per-system geometry) runs a
 * kernel that holds 16 bytes per lane point -- four float32 or two float64 orbitals -- instead of
 * 8: the same operator and recurrence, its sums in another order (results differ from the
 * 8-byte-lane kernel by rounding). Calls with per-system geometry, or all calls when disabled, use
 * the 8-byte lanes. The work-size queries cover both layouts. */
int cdftb_filter_wide(int enable);

/* No reference counterpart: the error flags the library's kernels set on the device (bit 0: a
 * bounded wait on a TMA barrier gave up). Synchronises the device, returns the flags in *flags and
 * clears them; status CDFTB_ERR_TIMEOUT when any flag was set. */
int cdftb_device_status(int* flags);

/* No reference counterpart: a test of the bounded waits above. The next slab-filter launch (filter
 * step or one-launch apply, order 8) issues the TMA copies of its first `planes` planes in x and no
 * more, so its consumers' waits run out (2 s) with no copy in flight; the launch then records the
 * timeout (cdftb_device_status returns CDFTB_ERR_TIMEOUT once) and its outputs are not written. One
 * launch only: the setting clears itself. 0 turns a pending setting off. */
int cdftb_filter_test_withhold(int planes);

/* (e1) out[g][i][j] = sum_p q[p] a[g][i][p] b[g][j][p] (src/cdft/eigen/measure.py:72-96,
 * Measure.inner/gram/cross), f64, deterministic two-pass reduction. a and b hold `groups`
 * blocks of ma and mb rows, group_stride_a/b elements apart. q may be NULL (plain sum). */
int64_t cdftb_measure_cross_scratch_bytes(int ma, int mb, int64_t n, int groups);
int cdftb_measure_cross_f64(const double* a, int ma, int64_t group_stride_a, const double* b, int mb,
                            int64_t group_stride_b, const double* q, int64_t n, int groups, double* out,
                            void* scratch, int64_t scratch_bytes, cdftb_stream_t stream);
/* The same with one measure per group (q + g * q_group_stride): systems on their own grids in one
 * call (src/cdft/eigen/measure.py:72-96 per system). */
int cdftb_measure_cross_grouped_f64(const double* a, int ma, int64_t group_stride_a, const double* b, int mb,
                                    int64_t group_stride_b, const double* q, int64_t q_group_stride, int64_t n,
                                    int groups, double* out, void* scratch, int64_t scratch_bytes,
                                    cdftb_stream_t stream);

/* No reference counterpart: cdftb_measure_cross_f64 for callers that cannot allocate device
 * memory. Same arguments and results (bit-identical), but the partials go to a fixed device array
 * of this library, cdftb_measure_cross_static_capacity_bytes() = 4 MiB per device, instead of
 * caller scratch. This call allocates nothing (no cudaMalloc, no cudaFree).
 * - Returns CDFTB_ERR_CAPACITY when cdftb_measure_cross_scratch_bytes(ma, mb, n, groups) exceeds
 *   that capacity.
 * - The first call in each CUDA context on a device looks up the array's address
 *   (cudaGetSymbolAddress, checked; CDFTB_ERR_LAUNCH on failure) and keeps it with the context's ID,
 *   so after a device reset (a new primary context) the next call looks it up again. That set-up
 *   call must come before any stream capture.
 * - Calls whose work overlaps on the GPU (several streams or host threads on one device) share the
 *   array and race; the caller orders them.
 * - Nothing in the array has to start at zero: the first pass writes every partial the second
 *   pass reads. */
int64_t cdftb_measure_cross_static_capacity_bytes(void);
int cdftb_measure_cross_static_f64(const double* a, int ma, int64_t group_stride_a, const double* b, int mb,
                                   int64_t group_stride_b, const double* q, int64_t n, int groups, double* out,
                                   cdftb_stream_t stream);

/* (e2) Per group: lower = chol(gram), info[g] = 0, or k+1 if the leading minor k is not positive
 * (src/cdft/eigen/rayleigh_ritz.py:62-63 torch.linalg.cholesky). */
int cdftb_small_cholesky_f64(const double* gram, double* lower, int* info, int m, int groups,
                             cdftb_stream_t stream);

/* (e2') out[g][:, p] = L[g]^{-1} in[g][:, p] by forward substitution for every column p
 * (src/cdft/eigen/rayleigh_ritz.py:72 solve_triangular_wide; src/cdft/precision.py:292-308). */
int cdftb_block_trsm_lower_f64(const double* lower, const double* in, int64_t in_group_stride, void* out,
                               int out_dtype, int64_t out_group_stride, int m, int64_t n, int groups,
                               cdftb_stream_t stream);

/* (e3) Per group: H = 0.5 (M + M^T) of the m x m matrix M, then eigenvalues ascending and
 * orthonormal eigenvectors by cyclic Jacobi (rayleigh_ritz.py:97-99). vectors[g] holds the
 * eigenvectors as ROWS (vectors[g][k][:] is the k-th eigenvector). */
int cdftb_small_eigh_f64(const double* matrix, double* evals, double* vectors, int m, int groups,
                         cdftb_stream_t stream);

/* (e4) out[g][i][p] = sum_j R[g][i][j] in[g][j][p]: the block rotation U^T Q of
 * rayleigh_ritz.py:100. f64 in, out_dtype out. */
int cdftb_block_rotate_f64(const double* r, const double* in, int64_t in_group_stride, void* out,
                           int out_dtype, int64_t out_group_stride, int m_out, int m_in, int64_t n,
                           int groups, cdftb_stream_t stream);

/* (e6) The end of Rayleigh--Ritz in one pass (rayleigh_ritz.py:100-115): per group g and point p,
 * v_i = sum_j R[g][i][j] basis[g][j][p] (written to vectors), (A v)_i = sum_j R[g][i][j] applied[g][j][p],
 * and the residual rho_i = (A v)_i - evals[g][i] v_i, whose measure norm
 * norms_sq[g][i] = sum_p q[g][p] rho_i(p)^2 is returned squared (q_group_stride 0: one q for every
 * group). Blocks are m consecutive rows of n; m <= 8. Deterministic: partials per fixed chunk of
 * points in scratch (>= cdftb_block_ritz_scratch_bytes), added in chunk order. The same values as
 * two cdftb_block_rotate_f64, cdftb_block_residual_f64 and a measure product, without the rotated
 * applied block and the residual block in memory. */
int64_t cdftb_block_ritz_scratch_bytes(int m, int64_t n, int groups);
int cdftb_block_ritz_f64(const double* r, const double* basis, const double* applied, const double* evals,
                         const double* q, int64_t q_group_stride, int m, int64_t n, int groups, double* vectors,
                         double* norms_sq, void* scratch, int64_t scratch_bytes, cdftb_stream_t stream);

/* (e5) out[g][i][p] = a[g][i][p] - evals[g][i] * b[g][i][p] (rayleigh_ritz.py:114 residual).
 * Each group's m rows are m consecutive rows of n elements, groups group_stride elements apart. */
int cdftb_block_residual_f64(const double* a, const double* b, const double* evals, double* out, int m,
                             int64_t n, int groups, int64_t group_stride, cdftb_stream_t stream);

/* Lanczos vector update (src/cdft/operators/hamiltonian.py:252-262): with device scalars
 * alpha = <v,w>, beta_prev:  w <- w - alpha v - beta_prev v_prev. Then, after the two
 * re-orthogonalisation products c1 = <w,v>, c2 = <w,v_prev>: w <- w - c1 v - c2 v_prev. mode 0
 * does the first update, mode 1 the second, mode 2 the normalisation v_next = w / beta. Each
 * scalar pointer indexes one value per group (groups vectors n elements apart). */
int cdftb_lanczos_update_f64(int mode, double* w, const double* v, const double* v_prev,
                             const double* s1, const double* s2, int64_t n, int groups,
                             cdftb_stream_t stream);

/* Cast between double and float blocks (the precision boundary of the mixed form). */
int cdftb_cast(const void* in, int in_dtype, void* out, int out_dtype, int64_t count, cdftb_stream_t stream);


/* ---- (c) Coulomb-cutoff Poisson (src/cdft/operators/poisson.py:21-107) ---- */

/* Plan for one grid: pads every axis to fft_friendly(ceil(pad_factor n)) (poisson.py:36-40), builds
 * the truncated kernel K(G) (poisson.py:43-64) and two transform buffers for up to max_batch
 * densities. Allocates device memory (the only allocating calls are *_create). Writes the padded
 * shape (3 ints) and the cutoff radius. */
int cdftb_poisson_plan_create(int nx, int ny, int nz, double spacing, double pad_factor, int max_batch,
                              void** plan, int* padded_shape, double* cutoff_radius);
int cdftb_poisson_plan_destroy(void* plan);
/* The device kernel table K (padded0, padded1, padded2/2+1) of a plan. */
int cdftb_poisson_kernel_table(void* plan, const double** table);
/* v = irfftn(rfftn(pad(rho)) K)[:n] for `batch` densities (batch x N each): CoulombCutoffPoisson.solve
 * (poisson.py:66-84). */
int cdftb_poisson_solve(void* plan, const double* density, double* potential, int batch, cdftb_stream_t stream);

/* ---- (d) exchange-correlation, spin-restricted (src/cdft/xc/base.py:115-189) ---- */

/* Slater + VWN5 (xc/lda.py:113-159, 201-217; dispatch name lda_vwn): e = e_xc per volume, v = de/dn. */
int cdftb_xc_lda_vwn_f64(const double* density, int64_t points, double* e, double* v, cdftb_stream_t stream);
/* PBE exchange + correlation (xc/gga.py:43-90; dispatch name pbe): e, v = de/dn, vs = de/dsigma. */
int cdftb_xc_pbe_f64(const double* density, const double* sigma, int64_t points, double* e, double* v, double* vs,
                     cdftb_stream_t stream);

/* ---- (d) every native functional, spin-restricted or spin-polarised (src/cdft/xc/base.py:45-189) ---- */

/* The functional names of src/cdft/xc/dispatch.py:26-44 (_builders). */
typedef enum cdftb_xc_id {
    CDFTB_XC_LDA_VWN = 0,      /* lda_vwn: Slater + VWN5 */
    CDFTB_XC_LDA_PW92 = 1,     /* lda_pw92: Slater + PW92 (original parameters) */
    CDFTB_XC_LDA_PW92_MOD = 2, /* lda_pw92_mod: Slater + PW92 (modified parameters, as inside PBE) */
    CDFTB_XC_LDA_PZ81 = 3,     /* lda_pz81: Slater + PZ81 */
    CDFTB_XC_PBE = 4,          /* pbe: PBE exchange + PBE correlation */
    CDFTB_XC_BLYP = 5,         /* blyp: B88 exchange + LYP correlation */
    CDFTB_XC_LDA_X = 6,        /* lda_x: Slater exchange alone */
    CDFTB_XC_LDA_C_VWN = 7,    /* lda_c_vwn */
    CDFTB_XC_LDA_C_PW = 8,     /* lda_c_pw */
    CDFTB_XC_LDA_C_PW_MOD = 9, /* lda_c_pw_mod */
    CDFTB_XC_LDA_C_PZ = 10,    /* lda_c_pz */
    CDFTB_XC_GGA_X_PBE = 11,   /* gga_x_pbe */
    CDFTB_XC_GGA_C_PBE = 12,   /* gga_c_pbe */
    CDFTB_XC_GGA_X_B88 = 13,   /* gga_x_b88 */
    CDFTB_XC_GGA_C_LYP = 14    /* gga_c_lyp */
} cdftb_xc_id;

/* 1 if `functional` (a cdftb_xc_id) needs sigma, 0 if not, -1 for an unknown id. */
int cdftb_xc_is_gga(int functional);

/* SemiLocalFunctional.evaluate (xc/base.py:115-156) for one functional on `points` points:
 * density (n_spin, points) with n_spin 1 (total density) or 2 (n_up, n_dn rows); for a GGA, sigma
 * (1, points) or (3, points) = (uu, ud, dd) rows. Writes e (points,) the energy per volume,
 * v (n_spin, points) = de/dn per channel and, for a GGA, v_sigma (1 or 3, points) = de/dsigma per
 * component. Spin split, thresholds, clamps and empty points as base.py:45-80, 171-189; the
 * derivatives are exact derivatives of the energy density (forward-mode dual numbers), as the
 * reference's autograd gives them. sigma and v_sigma may be NULL for an LDA. */
int cdftb_xc_eval_f64(int functional, int n_spin, const double* density, const double* sigma, int64_t points,
                      double* e, double* v, double* v_sigma, cdftb_stream_t stream);

/* ---- (s2) density mixing ---- */

/* The Kerker preconditioner (src/cdft/scf/mixing.py:35-56, KerkerPreconditioner.__call__): for each
 * of `channels` residual rows of the box (nx, ny, nz), out = irfftn(rfftn(F) q^2 / (q^2 + q0^2)),
 * q from 2 pi fftfreq(n, spacing) per axis, a periodic transform of the box (not zero-padded).
 * Any edge up to 1024 (direct axis sums, not FFTs). work: device scratch of at least
 * cdftb_kerker_work_bytes(nx, ny, nz, channels) bytes. residual and out may not overlap. */
int64_t cdftb_kerker_work_bytes(int nx, int ny, int nz, int channels);
int cdftb_kerker_precondition_f64(const double* residual, int channels, int nx, int ny, int nz, double spacing,
                                  double q0, double* out, void* work, int64_t work_bytes, cdftb_stream_t stream);

/* The same periodic box transform with a filter chosen by `kind`: 0 the Kerker filter above
 * (param = q0), 1 the Teter--Payne--Allan kinetic preconditioner of LOBPCG
 * (src/cdft/eigen/lobpcg.py:160-189, LOBPCG._apply_preconditioner): P(x) / (P(x) + 16 x^4),
 * P = 27 + 18 x + 12 x^2 + 8 x^3, x = (q^2 / 2) / E_ref with param = E_ref > 0. Same work size. */
int cdftb_reciprocal_filter_f64(const double* field, int channels, int nx, int ny, int nz, double spacing, int kind,
                                double param, double* out, void* work, int64_t work_bytes, cdftb_stream_t stream);

/* ---- (d4) cusp-aware quadrature interpolant (src/cdft/operators/quadrature.py:506-650) ---- */

/* Stencil corner (m x 3 ints) and the three 8-point Lagrange weight vectors (m x 24) of every point
 * (quadrature.py:56-93, 524-541); *bad_flag is set if a stencil leaves the grid. */
int cdftb_quadrature_stencils(const double* points, int64_t m, int nx, int ny, int nz, double ox, double oy,
                              double oz, double spacing, int* base, double* w1d, int* bad_flag,
                              cdftb_stream_t stream);
/* CSR of L^T (row_ptr: N+1 int64, col: 512 m node indices sorted by (grid point, node)), built by a
 * device radix sort in caller scratch (quadrature.py:580-608). */
int64_t cdftb_lift_plan_scratch_bytes(int64_t m, int64_t n_points);
int cdftb_lift_plan_build(const int* base, int64_t m, int nx, int ny, int nz, long long* row_ptr, int* col,
                          void* scratch, int64_t scratch_bytes, cdftb_stream_t stream);
/* out[f][node] = (L field_f)[node] for nf fields (quadrature.py:613-620 interpolate). */
int cdftb_quadrature_interpolate_f64(const int* base, const double* w1d, int64_t m, int nx, int ny, int nz,
                                     const double* fields, int nf, int64_t field_stride, double* out,
                                     int64_t out_stride, cdftb_stream_t stream);
/* values[e] = the weight of CSR entry e of L^T (row_ptr[nx*ny*nz] entries), for the lifts below. */
int cdftb_lift_plan_values_f64(const int* base, const double* w1d, const long long* row_ptr, const int* col, int nx,
                               int ny, int nz, double* values, cdftb_stream_t stream);
/* out[f] = L^T x_f for nf node vectors (quadrature.py:628-638 lift). values: the entry weights of
 * cdftb_lift_plan_values_f64, or NULL to form them from base and w1d on the fly. */
int cdftb_quadrature_lift_f64(const int* base, const double* w1d, const long long* row_ptr, const int* col,
                              const double* values, int nx, int ny, int nz, const double* node_values, int nf,
                              int64_t x_stride, double* out, int64_t out_stride, cdftb_stream_t stream);
/* The same two products for many fields (the systems of a batch): up to 32 fields per pass, one
 * lane per field, after copying the fields into point-major rows of 32 in caller scratch of
 * cdftb_quadrature_many_scratch_bytes(m, n_points) bytes. The lift walks the CSR rows in segments
 * of at most 256 entries (cdftb_lift_plan_segments: seg_ptr[n_points + 1], seg_row[capacity],
 * capacity = cdftb_lift_segments_capacity(m, n_points)) and needs the entry weights (values).
 * Results equal the one-field entry points up to the order of the sums (~1e-16 relative). */
int64_t cdftb_quadrature_many_scratch_bytes(int64_t m, int64_t n_points);
int64_t cdftb_lift_segments_capacity(int64_t m, int64_t n_points);
int64_t cdftb_lift_segments_scratch_bytes(int64_t n_points);
int cdftb_lift_plan_segments(const long long* row_ptr, int nx, int ny, int nz, int* seg_ptr, int* seg_row,
                             int64_t capacity, void* scratch, int64_t scratch_bytes, cdftb_stream_t stream);
int cdftb_quadrature_interpolate_many_f64(const int* base, const double* w1d, int64_t m, int nx, int ny, int nz,
                                          const double* fields, int nf, int64_t field_stride, double* out,
                                          int64_t out_stride, void* scratch, int64_t scratch_bytes,
                                          cdftb_stream_t stream);
/* The many-field interpolant with the nodes grouped by base cell: group_nodes (m node indices) and
 * group_ptr (groups + 1 offsets) cut the nodes into groups whose members share a base cell (the
 * host keeps groups to four nodes, so that a crowded cell does not hold up the launch). The nodes of
 * a group read the same 8 x 8 x 8 box, which one warp reads once for four of them. Results equal
 * cdftb_quadrature_interpolate_many_f64's bit for bit; the same scratch. No reference counterpart
 * (the reference multiplies by its CSR matrix L, quadrature.py:613-620). */
int cdftb_quadrature_interpolate_grouped_f64(const int* base, const double* w1d, int64_t m, int nx, int ny, int nz,
                                             const int* group_nodes, const int* group_ptr, int64_t groups,
                                             const double* fields, int nf, int64_t field_stride, double* out,
                                             int64_t out_stride, void* scratch, int64_t scratch_bytes,
                                             cdftb_stream_t stream);
int cdftb_quadrature_lift_many_f64(const long long* row_ptr, const int* col, const double* values, const int* seg_ptr,
                                   const int* seg_row, int64_t seg_capacity, int nx, int ny, int nz, int64_t m,
                                   const double* node_values, int nf, int64_t x_stride, double* out,
                                   int64_t out_stride, void* scratch, int64_t scratch_bytes, cdftb_stream_t stream);

/* ---- (c2, s1) the Kohn-Sham potentials (src/cdft/scf/step.py:224-313) ---- */

/* c = S^{-1} (nucleus_f2 * rho(R_a)) per system (step.py:240-242). */
int cdftb_cusp_coefficients_f64(const double* rho_at_nuclei, const double* nucleus_f2, const double* overlap,
                                int n_atoms, int batch, double* coefficients, cdftb_stream_t stream);
/* rho = n / f^2, n_smooth = n - sum_a c_a exp(-2 Z_a s_a) (step.py:235-244). */
int cdftb_hartree_split_f64(const double* density, const double* f2, const double* cusp_grid,
                            const double* coefficients, int n_atoms, int64_t n_points, int batch, double* rho,
                            double* n_smooth, cdftb_stream_t stream);
/* Node side, LDA: from rho_node (batch x m) then vsmooth_node (batch x m) -> lift inputs
 * [batch][w f2 vH, w f2 v_xc] and w e_xc (step.py:247-261 with the interpolant fused in by the caller). */
int cdftb_potentials_node_lda_f64(const double* fields, int64_t m, const double* weights, const double* f2_node,
                                  const double* v1s_node, const double* coefficients, int n_atoms, int batch,
                                  double* lift_inputs, double* xc_energy_density, cdftb_stream_t stream);
/* Grid side, LDA: effective = (hartree_w + xc_w)/omega, v_hartree, terms [3][N] = (hartree_w rho,
 * xc_w rho, far_w e_xc), v_xc (optional) (step.py:245-303). */
int cdftb_potentials_grid_lda_f64(const double* density, const double* rho, const double* f2,
                                  const double* far_weights, const double* mass_weights, const double* v_smooth,
                                  const double* v1s_grid, const double* coefficients, int n_atoms,
                                  const double* lifted, int64_t n_points, int batch, double* effective,
                                  double* v_hartree, double* terms, double* v_xc, cdftb_stream_t stream);
/* One SCF iteration's output density and density residual (src/cdft/scf/step.py:366-370,
 * src/cdft/scf/loop.py:298-301 and 375-376):
 * rho_out = sum_k occ_k v_k^2 over the k orbitals (batch, k, n_points) of each system, n_out =
 * rho_out f2, residual_terms = mass |n_out - n_in| / f2 (its row sums are the residual norms). */
int cdftb_density_residual_f64(const double* vectors, const double* occupations, int k, int64_t n_points, int batch,
                               const double* f2, const double* mass_weights, const double* n_in, double* rho_out,
                               double* n_out, double* residual_terms, cdftb_stream_t stream);
/* Grid half of the external energy parts (hamiltonian.py:360-378): out (batch, 2, n_points) =
 * (far_w weight (grad rho . grad u), far_w weight rho W); their row sums enter (1/2) Q[f^2 grad rho .
 * grad u] and Q[f^2 rho W]. grad is (batch, 3, n_points), grad_u (3, n_points). */
int cdftb_external_grid_terms_f64(const double* grad, const double* rho, const double* weight, const double* grad_u,
                                  const double* transformed_potential, const double* far_weights, int64_t n_points,
                                  int batch, double* out, cdftb_stream_t stream);
/* Deterministic row sums of a rows x len array (the energy integrals). */
int64_t cdftb_row_sums_scratch_bytes(int rows, int64_t len);
int cdftb_row_sums_f64(const double* a, int rows, int64_t len, double* out, void* scratch, int64_t scratch_bytes,
                       cdftb_stream_t stream);
/* out (+)= sign * d/d(axis) in, central weights `coefficients` (accuracy+1 taps), zero halo
 * (src/cdft/operators/laplacian.py:111-130, grid.py:745-758). */
int cdftb_fd_derivative_f64(const double* in, double* out, int nx, int ny, int nz, int axis, int accuracy,
                            const double* coefficients, double spacing, int64_t batch, int accumulate, double sign,
                            cdftb_stream_t stream);
/* The three partial derivatives of a batch of fields (src/cdft/grid.py:740-743 gradient): in is
 * (batch, N), out (batch, 3, N); each component is bit for bit cdftb_fd_derivative_f64's for its
 * axis (accumulate 0, sign 1), from one pass over the field. */
int cdftb_gradient_f64(const double* in, double* out, int nx, int ny, int nz, int accuracy, const double* coefficients,
                       double spacing, int64_t batch, cdftb_stream_t stream);

/* ---- geometry on the device (src/cdft/operators/cusp.py, quadrature.py, scf/step.py:129-165) ----
 * In these entry points `charges`, `positions` and `spheres` are HOST arrays (a few numbers per
 * nucleus, passed to the kernels by value); every other pointer is device memory. */

/* u, grad u (3 x N), f^2 and W = -|grad u|^2/2 with the 4^3 cell average within 2h (cusp.py:46-145).
 * gl4 = four Gauss-Legendre offsets (times h/2) then their weights (times 1/2). */
int cdftb_geometry_cusp_fields(int n_atoms, const double* charges, const double* positions, int nx, int ny, int nz,
                               double ox, double oy, double oz, double spacing, const double* gl4, double* u,
                               double* grad_u, double* f2, double* transformed_potential, int* n_averaged,
                               cdftb_stream_t stream);
/* f^2 at the staggered faces of each axis (cusp.py:168-214); *underflow set if u > 354. */
int cdftb_geometry_face_weights(int n_atoms, const double* charges, const double* positions, int nx, int ny, int nz,
                                double ox, double oy, double oz, double spacing, int accuracy, double* w0, double* w1,
                                double* w2, int* underflow, cdftb_stream_t stream);
/* Node partition P, weights = base P, f^2, grad u and W at the sphere nodes (quadrature.py:296-308,
 * 360-419). spheres: per nucleus (centre xyz, radius, taper centre, taper width). */
int cdftb_geometry_node_fields(int n_atoms, const double* charges, const double* positions, const double* spheres,
                               double cell_width, const double* node_points, const int* owner,
                               const double* base_weights, int64_t m, double* partition, double* weights,
                               double* f2, double* grad_u, double* transformed_potential, cdftb_stream_t stream);
/* far = prod_a (1 - p_a), far_w = h^3 far, plain_far = far_w f^2 on the grid (quadrature.py:312-319). */
int cdftb_geometry_grid_far(int n_atoms, const double* charges, const double* positions, const double* spheres, int nx,
                            int ny, int nz, double ox, double oy, double oz, double spacing, const double* f2,
                            double* far, double* far_weights, double* plain_far, cdftb_stream_t stream);
/* Lumped far mass weights of overlapping spheres on the refined lattice (quadrature.py:421-497). */
int cdftb_geometry_lumped_far(int n_atoms, const double* charges, const double* positions, const double* spheres,
                              int nx, int ny, int nz, double ox, double oy, double oz, double spacing, int refine,
                              const double* fine_x, const double* fine_y, const double* fine_z, const double* mx,
                              const int* lox, const int* hix, const double* my, const int* loy, const int* hiy,
                              const double* mz, const int* loz, const int* hiz, const double* plain_far, double margin,
                              double width, double* work, double* lumped_far, cdftb_stream_t stream);
/* omega, W~/omega, h^3/omega and the measure from lifted = [lift(w f2), lift(w W f2)]
 * (quadrature.py:327, 731-753); *nonpositive set if some omega <= 0. */
int cdftb_geometry_bare_terms(const double* lifted, const double* far_mass, const double* far_weights,
                              const double* transformed_potential, const double* f2, int64_t n_points, double spacing,
                              double* mass, double* potential, double* inverse_weight, double* quadrature,
                              int* nonpositive, cdftb_stream_t stream);
/* exp(-2 Z_a s) and the 1s potential on the grid and at the nodes (step.py:154-156). */
int cdftb_geometry_step_fields(int n_atoms, const double* charges, const double* positions, int nx, int ny, int nz,
                               double ox, double oy, double oz, double spacing, const double* node_points, int64_t m,
                               double* cusp_grid, double* v1s_grid, double* v1s_node, cdftb_stream_t stream);
/* Hydrogenic superposition and its charge terms omega * total / f^2 (src/cdft/scf/loop.py:173-193). */
int cdftb_geometry_initial_density(int n_atoms, const double* charges, const double* positions, int nx, int ny, int nz,
                                   double ox, double oy, double oz, double spacing, double zeta_scale, const double* f2,
                                   const double* mass, double* total, double* charge_terms, cdftb_stream_t stream);
/* a <- s a. */
int cdftb_scale_f64(double* a, int64_t n, double s, cdftb_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* CDFTB_H */
