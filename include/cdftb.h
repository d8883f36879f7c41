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

/* Library version (major*10000 + minor*100 + patch) and the status text. */
int cdftb_version(void);
const char* cdftb_status_string(int status);
/* The cudaError_t of the last failed CUDA call made by this library on this host thread. */
int cdftb_last_cuda_error(void);

/*
 * The cusp-factorised operator A = (1/2 w) sum_d D_d^T [f^2_face,d D_d .] + V on one grid.
 * face_weights[d] has the grid shape extended by `accuracy` along d, indexed from face -accuracy/2
 * (src/cdft/operators/cusp.py:168-214); inverse_weight = h^3/omega (N); potential = V (N per
 * group, groups `potential_stride` elements apart; orbital b uses group b / orbitals_per_group).
 * `dtype` says whether the weight and potential arrays are double or float. The measure
 * `quadrature` (omega, N, always double) is used by the reductions.
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
} cdftb_operator;

/* (a1) out = sum_d D_d^T [w_d D_d box], f64, batched.
 * Replaces src/cdft/operators/divergence.py:153 weighted_divergence and the CUDA dispatch
 * src/cdft/operators/fused.py:353 device_weighted_divergence. */
int cdftb_weighted_divergence_f64(const double* box, double* out, int64_t batch, int nx, int ny, int nz,
                                  const double* w0, const double* w1, const double* w2, double spacing,
                                  int accuracy, cdftb_stream_t stream);

/* (a2) out = A phi for a batch of orbitals (src/cdft/operators/hamiltonian.py:251-318,
 * apply / apply_with_potential / kinetic_apply). in_dtype/out_dtype select double or float
 * for phi/out; the arithmetic runs in the operator's dtype. kinetic_only = 1 drops the V phi term
 * (hamiltonian.py:303 kinetic_apply). */
int cdftb_cusp_apply(const cdftb_operator* op, const void* phi, int in_dtype, void* out, int out_dtype,
                     int64_t batch, int kinetic_only, cdftb_stream_t stream);

/* (b) The scaled Chebyshev filter of degree `degree` (src/cdft/eigen/chefsi.py:81-160,
 * chebyshev_filter / chebyshev_recurrence, with fused.py:391 chebyshev_update fused into each apply).
 * coefficients: device table (groups, degree, 3) of rows (c, a_k, b_k) from chefsi.py:116
 * chebyshev_coefficients, one table per potential group. block and out are in_dtype/out_dtype;
 * work holds two blocks of the operator's dtype (2 * batch * N elements). */
int cdftb_chebyshev_filter(const cdftb_operator* op, const void* block, int in_dtype, void* out, int out_dtype,
                           void* work, int64_t batch, const double* coefficients, int degree,
                           cdftb_stream_t stream);

/* (e1) out[g][i][j] = sum_p q[p] a[g][i][p] b[g][j][p] (src/cdft/eigen/measure.py:72-96,
 * Measure.inner/gram/cross), f64, deterministic two-pass reduction. a and b hold `groups`
 * blocks of ma and mb rows, group_stride_a/b elements apart. q may be NULL (plain sum). */
int64_t cdftb_measure_cross_scratch_bytes(int ma, int mb, int64_t n, int groups);
int cdftb_measure_cross_f64(const double* a, int ma, int64_t group_stride_a, const double* b, int mb,
                            int64_t group_stride_b, const double* q, int64_t n, int groups, double* out,
                            void* scratch, int64_t scratch_bytes, cdftb_stream_t stream);

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

#ifdef __cplusplus
}
#endif

#endif /* CDFTB_H */
