// (c2, d, s1) The Kohn--Sham potentials on the device (src/cdft/scf/step.py:224-313): the Hartree
// split n = sum_a c_a exp(-2 Z_a s_a) + n_s, the pointwise XC kernels, the node- and grid-side
// assembly of the lumped weights omega~ (quadrature.py:711-753) fused with the functional, and the
// deterministic row sums and finite-difference gradient the energies need.

#include "common.cuh"
#include "xc_device.cuh"

namespace cdftb {

namespace {

constexpr int MAX_ATOMS = 8;

inline unsigned blocks_for(int64_t n, int threads) {
    const int64_t b = ceil_div(n, threads);
    return static_cast<unsigned>(b < 148 * 32 ? b : 148 * 32);
}

#define GRID_STRIDE(i, n) \
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < (n); i += static_cast<int64_t>(gridDim.x) * blockDim.x)

// k -> (system g, point i) of a (batch, np) array; 32-bit division when the whole index fits.
__device__ __forceinline__ void split_index(int64_t k, int64_t np, bool narrow, int64_t& g, int64_t& i) {
    if (narrow) {
        const unsigned uk = static_cast<unsigned>(k), un = static_cast<unsigned>(np), ug = uk / un;
        g = ug;
        i = uk - ug * un;
    } else {
        g = k / np;
        i = k - g * np;
    }
}

__global__ void xc_lda_kernel(const double* __restrict__ n, int64_t p, double* __restrict__ e, double* __restrict__ v) {
    GRID_STRIDE(i, p) {
        double ei, vi;
        xc::lda_vwn(n[i], ei, vi);
        e[i] = ei;
        v[i] = vi;
    }
}

__global__ void xc_pbe_kernel(const double* __restrict__ n, const double* __restrict__ sigma, int64_t p,
                              double* __restrict__ e, double* __restrict__ v, double* __restrict__ vs) {
    GRID_STRIDE(i, p) {
        double ei, vi, vsi;
        xc::pbe(n[i], sigma[i], ei, vi, vsi);
        e[i] = ei;
        v[i] = vi;
        vs[i] = vsi;
    }
}

// c = S^{-1} (nucleus_f2 * rho(R_a)) by Gaussian elimination with partial pivoting, one system per
// thread (step.py:240-242; n_atoms <= MAX_ATOMS).
__global__ void cusp_coefficients_kernel(const double* __restrict__ rho_at_nuclei, const double* __restrict__ nucleus_f2,
                                         const double* __restrict__ overlap, int na, int batch,
                                         double* __restrict__ coef) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= batch) return;
    double a[MAX_ATOMS][MAX_ATOMS + 1];
    for (int i = 0; i < na; ++i) {
        for (int j = 0; j < na; ++j) a[i][j] = overlap[i * na + j];
        a[i][na] = nucleus_f2[i] * rho_at_nuclei[g * na + i];
    }
    for (int c = 0; c < na; ++c) {
        int piv = c;
        for (int r = c + 1; r < na; ++r)
            if (fabs(a[r][c]) > fabs(a[piv][c])) piv = r;
        if (piv != c)
            for (int k = 0; k <= na; ++k) {
                const double t = a[c][k];
                a[c][k] = a[piv][k];
                a[piv][k] = t;
            }
        for (int r = c + 1; r < na; ++r) {
            const double f = a[r][c] / a[c][c];
            for (int k = c; k <= na; ++k) a[r][k] -= f * a[c][k];
        }
    }
    for (int r = na - 1; r >= 0; --r) {
        double v = a[r][na];
        for (int k = r + 1; k < na; ++k) v -= a[r][k] * coef[g * na + k];
        coef[g * na + r] = v / a[r][r];
    }
}

// rho = n / f^2 and n_smooth = n - sum_a c_a exp(-2 Z_a s_a) (step.py:235-244).
__global__ void hartree_split_kernel(const double* __restrict__ n, const double* __restrict__ f2,
                                     const double* __restrict__ cusp_grid, const double* __restrict__ coef, int na,
                                     int64_t np, int batch, double* __restrict__ rho, double* __restrict__ n_smooth) {
    const bool narrow = np * batch <= 0xffffffffll;
    GRID_STRIDE(k, np * batch) {
        int64_t g, i;
        split_index(k, np, narrow, g, i);
        const double nv = n[k];
        rho[k] = nv / f2[i];
        double cusp = 0.0;
        for (int a = 0; a < na; ++a) {
            const double t = coef[g * na + a] * cusp_grid[a * np + i];
            cusp = (a == 0) ? t : cusp + t;
        }
        n_smooth[k] = nv - cusp;
    }
}

// Node side of potentials(), LDA: x_H = w f2 vH, x_xc = w f2 v_xc (the lift inputs of the lumped
// Hartree and XC weights) and e_w = w e_xc (the node part of the XC energy).
// fields: rho_node (batch x m) followed by vsmooth_node (batch x m); outputs x [batch][2][m],
// e_w [batch][m].
__global__ void node_lda_kernel(const double* __restrict__ fields, int64_t m, const double* __restrict__ weights,
                                const double* __restrict__ f2n, const double* __restrict__ v1s_node,
                                const double* __restrict__ coef, int na, int batch, double* __restrict__ x,
                                double* __restrict__ e_w) {
    const bool narrow = m * batch <= 0xffffffffll;
    GRID_STRIDE(k, m * batch) {
        int64_t g, i;
        split_index(k, m, narrow, g, i);
        const double rho_node = fields[g * m + i];
        double vh = 0.0;
        for (int a = 0; a < na; ++a) {
            const double t = coef[g * na + a] * v1s_node[a * m + i];
            vh = (a == 0) ? t : vh + t;
        }
        vh = vh + fields[(batch + g) * m + i];
        const double f2 = f2n[i];
        const double nn = f2 * rho_node;
        double e, v;
        xc::lda_vwn(nn, e, v);
        const double w = weights[i];
        x[g * 2 * m + i] = w * (f2 * vh);
        x[g * 2 * m + m + i] = w * (f2 * v);
        e_w[g * m + i] = w * e;
    }
}

// Grid side, LDA: hartree_w = L_H + far_w (f2 vH), xc_w = L_xc + far_w (f2 v_xc),
// effective = (hartree_w + xc_w) / omega (step.py:249-303); terms [3][np] = (hartree_w rho,
// xc_w rho, far_w e_xc) for the energy sums; v_hartree = sum_a c_a v1s_a + v_smooth.
__global__ void grid_lda_kernel(const double* __restrict__ n, const double* __restrict__ rho,
                                const double* __restrict__ f2, const double* __restrict__ far_w,
                                const double* __restrict__ mass, const double* __restrict__ v_smooth,
                                const double* __restrict__ v1s_grid, const double* __restrict__ coef, int na,
                                const double* __restrict__ lifted, int64_t np, int batch, double* __restrict__ effective,
                                double* __restrict__ v_hartree, double* __restrict__ terms, double* __restrict__ v_xc) {
    const bool narrow = np * batch <= 0xffffffffll;
    GRID_STRIDE(k, np * batch) {
        int64_t g, i;
        split_index(k, np, narrow, g, i);
        double vh = 0.0;
        for (int a = 0; a < na; ++a) {
            const double t = coef[g * na + a] * v1s_grid[a * np + i];
            vh = (a == 0) ? t : vh + t;
        }
        vh = vh + v_smooth[k];
        double e, v;
        xc::lda_vwn(n[k], e, v);
        const double fw = far_w[i];
        const double f = f2[i];
        const double hw = lifted[g * 2 * np + i] + fw * (f * vh);
        const double xw = lifted[g * 2 * np + np + i] + fw * (f * v);
        const double r = rho[k];
        effective[k] = (hw + xw) / mass[i];
        v_hartree[k] = vh;
        if (v_xc) v_xc[k] = v;
        terms[g * 3 * np + i] = hw * r;
        terms[g * 3 * np + np + i] = xw * r;
        terms[g * 3 * np + 2 * np + i] = fw * e;
    }
}

// Deterministic row sums: pass 1 sums fixed chunks, pass 2 sums the chunk partials in order.
constexpr int RS_THREADS = 256;

__global__ void row_partial_kernel(const double* __restrict__ a, int64_t len, int64_t chunk, int chunks,
                                   double* __restrict__ partial) {
    const int r = blockIdx.y;
    const int c = blockIdx.x;
    const int64_t p0 = static_cast<int64_t>(c) * chunk;
    const int64_t p1 = (p0 + chunk < len) ? p0 + chunk : len;
    double s = 0.0;
    for (int64_t p = p0 + threadIdx.x; p < p1; p += RS_THREADS) s += a[static_cast<int64_t>(r) * len + p];
    __shared__ double red[RS_THREADS / 32];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < RS_THREADS / 32; ++w) t += red[w];
        partial[static_cast<int64_t>(r) * chunks + c] = t;
    }
}

__global__ void row_final_kernel(const double* __restrict__ partial, int rows, int chunks, double* __restrict__ out) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    double t = 0.0;
    for (int c = 0; c < chunks; ++c) t += partial[static_cast<int64_t>(r) * chunks + c];
    out[r] = t;
}

void row_shape(int rows, int64_t len, int64_t& chunk, int& chunks) {
    int64_t want = ceil_div(2 * 148, rows);
    const int64_t max_chunks = ceil_div(len, 4096);
    if (want > max_chunks) want = max_chunks;
    if (want < 1) want = 1;
    chunk = ceil_div(len, want);
    chunks = static_cast<int>(ceil_div(len, chunk));
}

// Order-8 (or any even order <= 8) central first derivative along `axis`, zero halo
// (src/cdft/operators/laplacian.py:111-130; grid.py:745-758).
__global__ void fd_derivative_kernel(const double* __restrict__ in, double* __restrict__ out, int nx, int ny, int nz,
                                     int axis, int half, const double* __restrict__ coeffs_dev, double scale,
                                     int64_t batch, int accumulate, double sign) {
    const int64_t np = static_cast<int64_t>(nx) * ny * nz;
    const bool narrow = np * batch <= 0xffffffffll;  // 32-bit index arithmetic suffices
    GRID_STRIDE(k, np * batch) {
        int64_t g, i;
        int ix, iy, iz;
        if (narrow) {
            const unsigned uk = static_cast<unsigned>(k), unp = static_cast<unsigned>(np);
            const unsigned ug = uk / unp, ui = uk - ug * unp;
            const unsigned uyz = static_cast<unsigned>(ny) * static_cast<unsigned>(nz);
            const unsigned ux = ui / uyz, r = ui - ux * uyz;
            const unsigned uy = r / static_cast<unsigned>(nz);
            g = ug;
            i = ui;
            ix = static_cast<int>(ux);
            iy = static_cast<int>(uy);
            iz = static_cast<int>(r - uy * static_cast<unsigned>(nz));
        } else {
            g = k / np;
            i = k - g * np;
            ix = static_cast<int>(i / (static_cast<int64_t>(ny) * nz));
            iy = static_cast<int>((i / nz) % ny);
            iz = static_cast<int>(i % nz);
        }
        const int pos = axis == 0 ? ix : (axis == 1 ? iy : iz);
        const int ext = axis == 0 ? nx : (axis == 1 ? ny : nz);
        const int64_t stride = axis == 0 ? static_cast<int64_t>(ny) * nz : (axis == 1 ? nz : 1);
        double acc = 0.0;
        bool first = true;
        for (int t = 0; t <= 2 * half; ++t) {
            const double c = coeffs_dev[t];
            if (c == 0.0) continue;
            const int off = t - half;
            const int q = pos + off;
            const double val = (q >= 0 && q < ext) ? in[g * np + i + off * stride] : 0.0;
            const double term = val * (c * scale);
            acc = first ? term : acc + term;
            first = false;
        }
        if (accumulate)
            out[k] += sign * acc;
        else
            out[k] = sign * acc;
    }
}

// The three partial derivatives of a batch of fields at once, out[g][axis][i] (the (..., 3, N)
// gradient): per point the same sums, in the same order, as three fd_derivative_kernel calls, so the
// result is theirs bit for bit, with the field read once and no stacking copy.
__global__ void gradient_kernel(const double* __restrict__ in, double* __restrict__ out, int nx, int ny, int nz,
                                int half, const double* __restrict__ coeffs_dev, double scale, int64_t batch) {
    const int64_t np = static_cast<int64_t>(nx) * ny * nz;
    const int64_t plane = static_cast<int64_t>(ny) * nz;
    GRID_STRIDE(k, np * batch) {
        const int64_t g = k / np, i = k - g * np;
        const int ix = static_cast<int>(i / plane);
        const int iy = static_cast<int>((i / nz) % ny);
        const int iz = static_cast<int>(i % nz);
        const double* src = in + g * np + i;
#pragma unroll
        for (int axis = 0; axis < 3; ++axis) {
            const int pos = axis == 0 ? ix : (axis == 1 ? iy : iz);
            const int ext = axis == 0 ? nx : (axis == 1 ? ny : nz);
            const int64_t stride = axis == 0 ? plane : (axis == 1 ? nz : 1);
            double acc = 0.0;
            bool first = true;
            for (int t = 0; t <= 2 * half; ++t) {
                const double c = coeffs_dev[t];
                if (c == 0.0) continue;
                const int off = t - half;
                const int q = pos + off;
                const double val = (q >= 0 && q < ext) ? src[off * stride] : 0.0;
                const double term = val * (c * scale);
                acc = first ? term : acc + term;
                first = false;
            }
            out[(g * 3 + axis) * np + i] = 1.0 * acc;
        }
    }
}

// The output density and the density residual of one SCF iteration, per system g and point i
// (src/cdft/scf/step.py:366-370 output_density; src/cdft/scf/loop.py:298-301 and 375-376, the
// residual norm):
//   rho_out = sum_k occ_k v_k^2,  n_out = rho_out f^2,  res = mass |n_out - n_in| / f^2.
// Products and sums are rounded one at a time (no contraction), in the order of those lines.
__global__ void density_residual_kernel(const double* __restrict__ vectors, const double* __restrict__ occ, int k,
                                        int64_t np, int batch, const double* __restrict__ f2,
                                        const double* __restrict__ mass, const double* __restrict__ n_in,
                                        double* __restrict__ rho_out, double* __restrict__ n_out,
                                        double* __restrict__ res) {
    const bool narrow = np * batch <= 0xffffffffll;
    GRID_STRIDE(idx, np * batch) {
        int64_t g, i;
        split_index(idx, np, narrow, g, i);
        const double* v = vectors + g * k * np + i;
        double r = __dmul_rn(occ[0], __dmul_rn(v[0], v[0]));
        for (int j = 1; j < k; ++j) r = __dadd_rn(r, __dmul_rn(occ[j], __dmul_rn(v[j * np], v[j * np])));
        const double f = f2[i];
        const double n = __dmul_rn(r, f);
        rho_out[idx] = r;
        n_out[idx] = n;
        res[idx] = __dmul_rn(mass[i], __ddiv_rn(fabs(__dsub_rn(n, n_in[idx])), f));
    }
}

// Grid half of the external energy parts (hamiltonian.py:360-378), per system g and point i:
//   out[g][0][i] = far_w (weight ((g0 u0 + g1 u1) + g2 u2)),  out[g][1][i] = far_w ((weight rho) W),
// with grad (batch, 3, np) the density gradient, u the cusp exponent's gradient (3, np) and W the
// transformed potential; rounded one operation at a time in that order.
__global__ void external_grid_kernel(const double* __restrict__ grad, const double* __restrict__ rho,
                                     const double* __restrict__ weight, const double* __restrict__ grad_u,
                                     const double* __restrict__ tpot, const double* __restrict__ far_w, int64_t np,
                                     int batch, double* __restrict__ out) {
    const bool narrow = np * batch <= 0xffffffffll;
    GRID_STRIDE(idx, np * batch) {
        int64_t g, i;
        split_index(idx, np, narrow, g, i);
        const double* gr = grad + g * 3 * np + i;
        const double dot = __dadd_rn(__dadd_rn(__dmul_rn(gr[0], grad_u[i]), __dmul_rn(gr[np], grad_u[np + i])),
                                     __dmul_rn(gr[2 * np], grad_u[2 * np + i]));
        const double w = weight[i], fw = far_w[i];
        out[g * 2 * np + i] = __dmul_rn(fw, __dmul_rn(w, dot));
        out[g * 2 * np + np + i] = __dmul_rn(fw, __dmul_rn(__dmul_rn(w, rho[idx]), tpot[i]));
    }
}

}  // namespace

}  // namespace cdftb

using namespace cdftb;

extern "C" int cdftb_xc_lda_vwn_f64(const double* n, int64_t p, double* e, double* v, cdftb_stream_t stream) {
    if (p < 0 || (p > 0 && (!n || !e || !v))) return CDFTB_ERR_ARGUMENT;
    if (p == 0) return CDFTB_OK;
    xc_lda_kernel<<<blocks_for(p, 256), 256, 0, as_stream(stream)>>>(n, p, e, v);
    return check_launch();
}

extern "C" int cdftb_xc_pbe_f64(const double* n, const double* sigma, int64_t p, double* e, double* v, double* vs,
                                cdftb_stream_t stream) {
    if (p < 0 || (p > 0 && (!n || !sigma || !e || !v || !vs))) return CDFTB_ERR_ARGUMENT;
    if (p == 0) return CDFTB_OK;
    xc_pbe_kernel<<<blocks_for(p, 256), 256, 0, as_stream(stream)>>>(n, sigma, p, e, v, vs);
    return check_launch();
}

extern "C" int cdftb_cusp_coefficients_f64(const double* rho_at_nuclei, const double* nucleus_f2, const double* overlap,
                                           int n_atoms, int batch, double* coefficients, cdftb_stream_t stream) {
    if (n_atoms < 1 || n_atoms > MAX_ATOMS || batch < 1 || !rho_at_nuclei || !nucleus_f2 || !overlap || !coefficients)
        return CDFTB_ERR_ARGUMENT;
    cusp_coefficients_kernel<<<static_cast<unsigned>(ceil_div(batch, 64)), 64, 0, as_stream(stream)>>>(
        rho_at_nuclei, nucleus_f2, overlap, n_atoms, batch, coefficients);
    return check_launch();
}

extern "C" int cdftb_hartree_split_f64(const double* density, const double* f2, const double* cusp_grid,
                                       const double* coefficients, int n_atoms, int64_t n_points, int batch, double* rho,
                                       double* n_smooth, cdftb_stream_t stream) {
    if (n_atoms < 0 || n_atoms > MAX_ATOMS || n_points <= 0 || batch < 1 || !density || !f2 || !rho || !n_smooth ||
        (n_atoms > 0 && (!cusp_grid || !coefficients)))
        return CDFTB_ERR_ARGUMENT;
    hartree_split_kernel<<<blocks_for(n_points * batch, 256), 256, 0, as_stream(stream)>>>(
        density, f2, cusp_grid, coefficients, n_atoms, n_points, batch, rho, n_smooth);
    return check_launch();
}

extern "C" int cdftb_potentials_node_lda_f64(const double* fields, int64_t m, const double* weights, const double* f2_node,
                                             const double* v1s_node, const double* coefficients, int n_atoms, int batch,
                                             double* lift_inputs, double* xc_energy_density, cdftb_stream_t stream) {
    if (m < 0 || n_atoms < 0 || n_atoms > MAX_ATOMS || batch < 1) return CDFTB_ERR_ARGUMENT;
    if (m == 0) return CDFTB_OK;
    if (!fields || !weights || !f2_node || !lift_inputs || !xc_energy_density || (n_atoms > 0 && (!v1s_node || !coefficients)))
        return CDFTB_ERR_ARGUMENT;
    node_lda_kernel<<<blocks_for(m * batch, 256), 256, 0, as_stream(stream)>>>(fields, m, weights, f2_node, v1s_node,
                                                                                coefficients, n_atoms, batch, lift_inputs,
                                                                                xc_energy_density);
    return check_launch();
}

extern "C" int cdftb_potentials_grid_lda_f64(const double* density, const double* rho, const double* f2,
                                             const double* far_weights, const double* mass_weights,
                                             const double* v_smooth, const double* v1s_grid, const double* coefficients,
                                             int n_atoms, const double* lifted, int64_t n_points, int batch,
                                             double* effective, double* v_hartree, double* terms, double* v_xc,
                                             cdftb_stream_t stream) {
    if (n_points <= 0 || batch < 1 || n_atoms < 0 || n_atoms > MAX_ATOMS) return CDFTB_ERR_ARGUMENT;
    if (!density || !rho || !f2 || !far_weights || !mass_weights || !v_smooth || !lifted || !effective || !v_hartree ||
        !terms || (n_atoms > 0 && (!v1s_grid || !coefficients)))
        return CDFTB_ERR_ARGUMENT;
    grid_lda_kernel<<<blocks_for(n_points * batch, 256), 256, 0, as_stream(stream)>>>(
        density, rho, f2, far_weights, mass_weights, v_smooth, v1s_grid, coefficients, n_atoms, lifted, n_points, batch,
        effective, v_hartree, terms, v_xc);
    return check_launch();
}

extern "C" int64_t cdftb_row_sums_scratch_bytes(int rows, int64_t len) {
    if (rows <= 0 || len <= 0) return 0;
    int64_t chunk;
    int chunks;
    row_shape(rows, len, chunk, chunks);
    return static_cast<int64_t>(rows) * chunks * 8;
}

extern "C" int cdftb_density_residual_f64(const double* vectors, const double* occupations, int k, int64_t n_points,
                                          int batch, const double* f2, const double* mass_weights,
                                          const double* n_in, double* rho_out, double* n_out, double* residual_terms,
                                          cdftb_stream_t stream) {
    if (!vectors || !occupations || !f2 || !mass_weights || !n_in || !rho_out || !n_out || !residual_terms || k < 1 ||
        n_points <= 0 || batch < 1)
        return CDFTB_ERR_ARGUMENT;
    density_residual_kernel<<<blocks_for(n_points * batch, 256), 256, 0, as_stream(stream)>>>(
        vectors, occupations, k, n_points, batch, f2, mass_weights, n_in, rho_out, n_out, residual_terms);
    return check_launch();
}

extern "C" int cdftb_external_grid_terms_f64(const double* grad, const double* rho, const double* weight,
                                             const double* grad_u, const double* transformed_potential,
                                             const double* far_weights, int64_t n_points, int batch, double* out,
                                             cdftb_stream_t stream) {
    if (!grad || !rho || !weight || !grad_u || !transformed_potential || !far_weights || !out || n_points <= 0 ||
        batch < 1)
        return CDFTB_ERR_ARGUMENT;
    external_grid_kernel<<<blocks_for(n_points * batch, 256), 256, 0, as_stream(stream)>>>(
        grad, rho, weight, grad_u, transformed_potential, far_weights, n_points, batch, out);
    return check_launch();
}

extern "C" int cdftb_row_sums_f64(const double* a, int rows, int64_t len, double* out, void* scratch,
                                  int64_t scratch_bytes, cdftb_stream_t stream) {
    if (!a || !out || rows <= 0 || rows > 65535 || len <= 0) return CDFTB_ERR_ARGUMENT;
    if (!scratch || scratch_bytes < cdftb_row_sums_scratch_bytes(rows, len)) return CDFTB_ERR_ARGUMENT;
    int64_t chunk;
    int chunks;
    row_shape(rows, len, chunk, chunks);
    cudaStream_t s = as_stream(stream);
    double* partial = static_cast<double*>(scratch);
    row_partial_kernel<<<dim3(chunks, rows), RS_THREADS, 0, s>>>(a, len, chunk, chunks, partial);
    int st = check_launch();
    if (st != CDFTB_OK) return st;
    row_final_kernel<<<static_cast<unsigned>(ceil_div(rows, 64)), 64, 0, s>>>(partial, rows, chunks, out);
    return check_launch();
}

extern "C" int cdftb_gradient_f64(const double* in, double* out, int nx, int ny, int nz, int accuracy,
                                  const double* coefficients, double spacing, int64_t batch, cdftb_stream_t stream) {
    if (!in || !out || !coefficients || accuracy < 2 || accuracy > 8 || accuracy % 2 || !(spacing > 0.0) || batch < 1 ||
        nx <= 0 || ny <= 0 || nz <= 0)
        return CDFTB_ERR_ARGUMENT;
    const int64_t np = static_cast<int64_t>(nx) * ny * nz;
    gradient_kernel<<<blocks_for(np * batch, 256), 256, 0, as_stream(stream)>>>(in, out, nx, ny, nz, accuracy / 2,
                                                                              coefficients, 1.0 / spacing, batch);
    return check_launch();
}

extern "C" int cdftb_fd_derivative_f64(const double* in, double* out, int nx, int ny, int nz, int axis, int accuracy,
                                       const double* coefficients, double spacing, int64_t batch, int accumulate,
                                       double sign, cdftb_stream_t stream) {
    if (!in || !out || !coefficients || axis < 0 || axis > 2 || accuracy < 2 || accuracy > 8 || accuracy % 2 ||
        !(spacing > 0.0) || batch < 1)
        return CDFTB_ERR_ARGUMENT;
    const int64_t np = static_cast<int64_t>(nx) * ny * nz;
    fd_derivative_kernel<<<blocks_for(np * batch, 256), 256, 0, as_stream(stream)>>>(
        in, out, nx, ny, nz, axis, accuracy / 2, coefficients, 1.0 / spacing, batch, accumulate, sign);
    return check_launch();
}
