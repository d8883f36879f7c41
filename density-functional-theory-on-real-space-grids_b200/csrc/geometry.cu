// Geometry of the cusp-factorised operator and quadrature, built on the device: the Kato factor's
// fields on the grid (src/cdft/operators/cusp.py:46-145), the face weights f^2 at the staggered
// faces (cusp.py:168-214), the sphere nodes' partition weights and analytic fields
// (src/cdft/operators/quadrature.py:296-308, 360-419), the far factor on the grid (:499-504), the
// lumped far weights of overlapping spheres on the twice-refined lattice (:421-497), the bare
// operator terms (:731-753) and the Hartree-split tensors (src/cdft/scf/step.py:129-165).
// The node set itself (sphere-rule positions and radial x angular weights) is a small host-side
// plan; everything grid- or node-sized is computed here.

#include <math.h>

#include "common.cuh"

namespace cdftb {

namespace {

constexpr int MAX_ATOMS = 8;

struct Nuclei {
    int n;
    double z[MAX_ATOMS];
    double r[MAX_ATOMS][3];
    // sphere rule per nucleus
    double centre[MAX_ATOMS][3];
    double radius[MAX_ATOMS];
    double taper_centre[MAX_ATOMS];
    double taper_width[MAX_ATOMS];
    double cell_width;  // h sqrt(2) for the Becke cells
};

#define GRID_STRIDE(i, n) \
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < (n); i += static_cast<int64_t>(gridDim.x) * blockDim.x)

inline unsigned blocks_for(int64_t n, int threads) {
    const int64_t b = ceil_div(n, threads);
    return static_cast<unsigned>(b < 148 * 32 ? b : 148 * 32);
}

__device__ __forceinline__ double norm3(double x, double y, double z) { return sqrt(x * x + y * y + z * z); }

__device__ __forceinline__ void grid_point(int64_t i, int nx, int ny, int nz, double ox, double oy, double oz, double h,
                                           double* p) {
    const int ix = static_cast<int>(i / (static_cast<int64_t>(ny) * nz));
    const int iy = static_cast<int>((i / nz) % ny);
    const int iz = static_cast<int>(i % nz);
    p[0] = ox + static_cast<double>(ix) * h;
    p[1] = oy + static_cast<double>(iy) * h;
    p[2] = oz + static_cast<double>(iz) * h;
}

// u, grad u, f^2 and W = -|grad u|^2/2, with the 4^3 Gauss--Legendre cell average of |grad u|^2 and
// grad u within `reach` of a nucleus (cusp.py:74-145). gl: 4 offsets (already * h/2) and 4 weights.
__global__ void cusp_fields_kernel(Nuclei nuc, int nx, int ny, int nz, double ox, double oy, double oz, double h,
                                   double reach, const double* __restrict__ gl, double* __restrict__ u_out,
                                   double* __restrict__ grad_u, double* __restrict__ f2, double* __restrict__ w_out,
                                   int* __restrict__ n_averaged) {
    const int64_t np = static_cast<int64_t>(nx) * ny * nz;
    GRID_STRIDE(i, np) {
        double p[3];
        grid_point(i, nx, ny, nz, ox, oy, oz, h, p);
        double u = 0.0, g[3] = {0.0, 0.0, 0.0};
        bool near = false;
        for (int a = 0; a < nuc.n; ++a) {
            const double d[3] = {p[0] - nuc.r[a][0], p[1] - nuc.r[a][1], p[2] - nuc.r[a][2]};
            const double dist = norm3(d[0], d[1], d[2]);
            u += nuc.z[a] * dist;
            const double safe = fmax(dist, 1.0e-30);
            if (!(dist <= 1.0e-12))
                for (int k = 0; k < 3; ++k) g[k] += nuc.z[a] * (d[k] / safe);
            if (dist <= reach) near = true;
        }
        double w = -0.5 * (g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
        if (near) {
            double ms = 0.0, mv[3] = {0.0, 0.0, 0.0}, total = 0.0;
            for (int ix = 0; ix < 4; ++ix)
                for (int iy = 0; iy < 4; ++iy)
                    for (int iz = 0; iz < 4; ++iz) {
                        const double weight = gl[4 + ix] * gl[4 + iy] * gl[4 + iz];
                        total += weight;
                        const double q[3] = {p[0] + gl[ix], p[1] + gl[iy], p[2] + gl[iz]};
                        double gg[3] = {0.0, 0.0, 0.0};
                        for (int a = 0; a < nuc.n; ++a) {
                            const double d[3] = {q[0] - nuc.r[a][0], q[1] - nuc.r[a][1], q[2] - nuc.r[a][2]};
                            const double dist = fmax(norm3(d[0], d[1], d[2]), 1.0e-300);
                            for (int k = 0; k < 3; ++k) gg[k] = gg[k] + nuc.z[a] * d[k] / dist;
                        }
                        ms = ms + weight * (gg[0] * gg[0] + gg[1] * gg[1] + gg[2] * gg[2]);
                        for (int k = 0; k < 3; ++k) mv[k] = mv[k] + weight * gg[k];
                    }
            w = -0.5 * ms / total;
            for (int k = 0; k < 3; ++k) g[k] = mv[k] / total;
            atomicAdd(n_averaged, 1);
        }
        u_out[i] = u;
        for (int k = 0; k < 3; ++k) grad_u[k * np + i] = g[k];
        f2[i] = exp(-2.0 * u);
        w_out[i] = w;
    }
}

// f^2 at the faces of `axis`: the grid shape extended by `acc` along axis, face index from -acc/2.
__global__ void face_weights_kernel(Nuclei nuc, int nx, int ny, int nz, double ox, double oy, double oz, double h,
                                    int axis, int acc, double* __restrict__ out, int* __restrict__ underflow) {
    int s[3] = {nx, ny, nz};
    s[axis] += acc;
    const int half = acc / 2;
    const int64_t total = static_cast<int64_t>(s[0]) * s[1] * s[2];
    const double o[3] = {ox, oy, oz};
    GRID_STRIDE(i, total) {
        const int idx[3] = {static_cast<int>(i / (static_cast<int64_t>(s[1]) * s[2])), static_cast<int>((i / s[2]) % s[1]),
                            static_cast<int>(i % s[2])};
        double c[3];
        for (int d = 0; d < 3; ++d) {
            double index = static_cast<double>(idx[d]);
            if (d == axis) index = index - half + 0.5;
            c[d] = o[d] + index * h;
        }
        double u = 0.0;
        for (int a = 0; a < nuc.n; ++a) {
            double sq = 0.0;
            for (int d = 0; d < 3; ++d) {
                const double t = c[d] - nuc.r[a][d];
                sq = sq + t * t;
            }
            u = u + nuc.z[a] * sqrt(sq);
        }
        if (u > 354.0) atomicOr(underflow, 1);
        out[i] = exp(-2.0 * u);
    }
}

__device__ __forceinline__ double bump(const Nuclei& nuc, int a, const double* p) {
    const double s = norm3(p[0] - nuc.centre[a][0], p[1] - nuc.centre[a][1], p[2] - nuc.centre[a][2]);
    const double v = 0.5 * erfc((s - nuc.taper_centre[a]) / nuc.taper_width[a]);
    return s < nuc.radius[a] ? v : 0.0;
}

__device__ __forceinline__ double far_factor(const Nuclei& nuc, const double* p) {
    double far = 1.0;
    for (int a = 0; a < nuc.n; ++a) far = far * (1.0 - bump(nuc, a, p));
    return far;
}

// Node fields: partition P (quadrature.py:393-419), weights = base * P, u, grad u, f^2, W.
__global__ void node_fields_kernel(Nuclei nuc, const double* __restrict__ pts, const int* __restrict__ owner,
                                   const double* __restrict__ base_w, int64_t m, double* __restrict__ partition,
                                   double* __restrict__ weights, double* __restrict__ f2, double* __restrict__ grad_u,
                                   double* __restrict__ w_node) {
    GRID_STRIDE(i, m) {
        const double p[3] = {pts[i * 3], pts[i * 3 + 1], pts[i * 3 + 2]};
        const double near = 1.0 - far_factor(nuc, p);
        double cells[MAX_ATOMS];
        double dist[MAX_ATOMS];
        for (int a = 0; a < nuc.n; ++a)
            dist[a] = norm3(p[0] - nuc.centre[a][0], p[1] - nuc.centre[a][1], p[2] - nuc.centre[a][2]);
        if (nuc.n == 1) {
            cells[0] = 1.0;
        } else {
            double sum = 0.0;
            for (int a = 0; a < nuc.n; ++a) {
                double c = 1.0;
                for (int b = 0; b < nuc.n; ++b)
                    if (a != b) c = c * 0.5 * erfc((dist[a] - dist[b]) / nuc.cell_width);
                cells[a] = c;
            }
            for (int a = 0; a < nuc.n; ++a) sum += cells[a];
            sum = fmax(sum, 1.0e-300);
            for (int a = 0; a < nuc.n; ++a) cells[a] = cells[a] / sum;
        }
        const int own = owner[i];
        double share = cells[own];
        for (int b = 0; b < nuc.n; ++b)
            if (b != own) share = share + cells[b] * (dist[b] >= nuc.radius[b] ? 1.0 : 0.0);
        const double part = share * near;
        partition[i] = part;
        weights[i] = base_w[i] * part;
        double u = 0.0, g[3] = {0.0, 0.0, 0.0};
        for (int a = 0; a < nuc.n; ++a) {
            const double d[3] = {p[0] - nuc.r[a][0], p[1] - nuc.r[a][1], p[2] - nuc.r[a][2]};
            const double dd = fmax(norm3(d[0], d[1], d[2]), 1.0e-300);
            u = u + nuc.z[a] * dd;
            for (int k = 0; k < 3; ++k) g[k] = g[k] + nuc.z[a] * (d[k] / dd);
        }
        f2[i] = exp(-2.0 * u);
        for (int k = 0; k < 3; ++k) grad_u[k * m + i] = g[k];
        w_node[i] = -0.5 * (g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
    }
}

// far factor on the grid and its h^3 weights; plain far mass weights h^3 far f^2.
__global__ void grid_far_kernel(Nuclei nuc, int nx, int ny, int nz, double ox, double oy, double oz, double h,
                                const double* __restrict__ f2, double* __restrict__ far, double* __restrict__ far_w,
                                double* __restrict__ plain_far) {
    const int64_t np = static_cast<int64_t>(nx) * ny * nz;
    const double h3 = h * h * h;
    GRID_STRIDE(i, np) {
        double p[3];
        grid_point(i, nx, ny, nz, ox, oy, oz, h, p);
        const double f = far_factor(nuc, p);
        far[i] = f;
        far_w[i] = h3 * f;
        plain_far[i] = (h3 * f) * f2[i];
    }
}

// Lumped far weights, pass 1: collapsed[X][Y][c] = sum over fine z (ascending) of
// vol far f^2 (X, Y, z) * Mz[c][z] (quadrature.py:470-486). Mz is dense (nz x nzf); zlo/zhi give the
// fine-z range with a non-zero entry for each coarse c.
__global__ void lumped_collapse_kernel(Nuclei nuc, const double* __restrict__ fx, int nxf, const double* __restrict__ fy,
                                       int nyf, const double* __restrict__ fz, int nzf, const double* __restrict__ mz,
                                       const int* __restrict__ zlo, const int* __restrict__ zhi, int nz, double volume,
                                       double* __restrict__ collapsed) {
    const int64_t total = static_cast<int64_t>(nxf) * nyf * nz;
    GRID_STRIDE(k, total) {
        const int c = static_cast<int>(k % nz);
        const int64_t xy = k / nz;
        const int Y = static_cast<int>(xy % nyf);
        const int X = static_cast<int>(xy / nyf);
        double acc = 0.0;
        for (int z = zlo[c]; z < zhi[c]; ++z) {
            const double p[3] = {fx[X], fy[Y], fz[z]};
            double far = 1.0, u = 0.0;
            for (int a = 0; a < nuc.n; ++a) {
                const double s = norm3(p[0] - nuc.centre[a][0], p[1] - nuc.centre[a][1], p[2] - nuc.centre[a][2]);
                const double bmp = s < nuc.radius[a] ? 0.5 * erfc((s - nuc.taper_centre[a]) / nuc.taper_width[a]) : 0.0;
                far = far * (1.0 - bmp);
                u = u + nuc.z[a] * s;
            }
            const double value = volume * far * exp(-2.0 * u);
            acc = acc + value * mz[static_cast<int64_t>(c) * nzf + z];
        }
        collapsed[k] = acc;
    }
}

// out[a][Y][c] = sum_X m[a][X] in[X][Y][c] (banded m: X in [lo[a], hi[a])).
__global__ void band_contract_kernel(const double* __restrict__ m, const int* __restrict__ lo, const int* __restrict__ hi,
                                     int na, int nfine, const double* __restrict__ in, int64_t inner,
                                     double* __restrict__ out) {
    const int64_t total = static_cast<int64_t>(na) * inner;
    GRID_STRIDE(k, total) {
        const int a = static_cast<int>(k / inner);
        const int64_t r = k - a * inner;
        double acc = 0.0;
        for (int X = lo[a]; X < hi[a]; ++X) acc += m[static_cast<int64_t>(a) * nfine + X] * in[X * inner + r];
        out[k] = acc;
    }
}

// [a][b][c] from [a][Y][c] with the y band: out[a][b][c] = sum_Y my[b][Y] in[a][Y][c].
__global__ void band_contract_mid_kernel(const double* __restrict__ m, const int* __restrict__ lo,
                                         const int* __restrict__ hi, int nb, int nfine, const double* __restrict__ in,
                                         int na, int nc, double* __restrict__ out) {
    const int64_t total = static_cast<int64_t>(na) * nb * nc;
    GRID_STRIDE(k, total) {
        const int c = static_cast<int>(k % nc);
        const int b = static_cast<int>((k / nc) % nb);
        const int a = static_cast<int>(k / (static_cast<int64_t>(nc) * nb));
        double acc = 0.0;
        for (int Y = lo[b]; Y < hi[b]; ++Y)
            acc += m[static_cast<int64_t>(b) * nfine + Y] * in[(static_cast<int64_t>(a) * nfine + Y) * nc + c];
        out[k] = acc;
    }
}

// lumped_far = plain_far + interior (lumped - plain_far), interior = erfc((margin - face)/width)/2.
__global__ void lumped_blend_kernel(int nx, int ny, int nz, double ox, double oy, double oz, double h, double margin,
                                    double width, const double* __restrict__ lumped, const double* __restrict__ plain_far,
                                    double* __restrict__ out) {
    const int64_t np = static_cast<int64_t>(nx) * ny * nz;
    const double up[3] = {ox + (nx - 1) * h, oy + (ny - 1) * h, oz + (nz - 1) * h};
    GRID_STRIDE(i, np) {
        double p[3];
        grid_point(i, nx, ny, nz, ox, oy, oz, h, p);
        const double lo_face = fmin(fmin(p[0] - ox, p[1] - oy), p[2] - oz);
        const double hi_face = fmin(fmin(up[0] - p[0], up[1] - p[1]), up[2] - p[2]);
        const double face = fmin(lo_face, hi_face);
        const double interior = 0.5 * erfc((margin - face) / width);
        out[i] = plain_far[i] + interior * (lumped[i] - plain_far[i]);
    }
}

// omega = lift(w f^2) + far_mass; W~/omega = (lift(w W f^2) + far_w (W f^2)) / omega; h^3/omega and
// the measure q = (omega/h^3) h^3 (quadrature.py:327, 731-753). lifted = [lift(w f2), lift(w W f2)].
__global__ void bare_terms_kernel(const double* __restrict__ lifted, const double* __restrict__ far_mass,
                                  const double* __restrict__ far_w, const double* __restrict__ w_grid,
                                  const double* __restrict__ f2, int64_t np, double h3, double* __restrict__ mass,
                                  double* __restrict__ potential, double* __restrict__ inverse_weight,
                                  double* __restrict__ quadrature, int* __restrict__ nonpositive) {
    GRID_STRIDE(i, np) {
        const double om = lifted[i] + far_mass[i];
        if (!(om > 0.0)) atomicOr(nonpositive, 1);
        mass[i] = om;
        potential[i] = (lifted[np + i] + far_w[i] * (w_grid[i] * f2[i])) / om;
        inverse_weight[i] = h3 / om;
        quadrature[i] = (om / h3) * h3;
    }
}

__device__ __forceinline__ double hydrogenic_1s(double z, double s) {
    const double x = z * s;
    if (x < 1.0e-3)
        return (3.141592653589793 / (z * z)) *
               (1.0 - (2.0 / 3.0) * x * x + (2.0 / 3.0) * x * x * x - 0.4 * x * x * x * x + (8.0 / 45.0) * x * x * x * x * x);
    const double safe = fmax(s, 1.0e-300);
    return (3.141592653589793 / (z * z * z)) * (1.0 - exp(-2.0 * x) * (1.0 + x)) / safe;
}

// exp(-2 Z_a s_a) and the 1s potential on the grid, the 1s potential at the nodes (step.py:154-156).
__global__ void step_grid_kernel(Nuclei nuc, int nx, int ny, int nz, double ox, double oy, double oz, double h,
                                 double* __restrict__ cusp_grid, double* __restrict__ v1s_grid) {
    const int64_t np = static_cast<int64_t>(nx) * ny * nz;
    GRID_STRIDE(i, np) {
        double p[3];
        grid_point(i, nx, ny, nz, ox, oy, oz, h, p);
        for (int a = 0; a < nuc.n; ++a) {
            const double s = norm3(p[0] - nuc.r[a][0], p[1] - nuc.r[a][1], p[2] - nuc.r[a][2]);
            cusp_grid[a * np + i] = exp(-2.0 * nuc.z[a] * s);
            v1s_grid[a * np + i] = hydrogenic_1s(nuc.z[a], s);
        }
    }
}

__global__ void step_node_kernel(Nuclei nuc, const double* __restrict__ pts, int64_t m, double* __restrict__ v1s_node) {
    GRID_STRIDE(i, m) {
        for (int a = 0; a < nuc.n; ++a) {
            const double s = norm3(pts[i * 3] - nuc.r[a][0], pts[i * 3 + 1] - nuc.r[a][1], pts[i * 3 + 2] - nuc.r[a][2]);
            v1s_node[a * m + i] = hydrogenic_1s(nuc.z[a], s);
        }
    }
}

// Hydrogenic superposition sum_a (Z^3/pi) exp(-2 Z s_a) and rho = total / f^2 (loop.py:184-190).
__global__ void initial_density_kernel(Nuclei nuc, int nx, int ny, int nz, double ox, double oy, double oz, double h,
                                       double scale, const double* __restrict__ f2, const double* __restrict__ mass,
                                       double* __restrict__ total, double* __restrict__ charge_terms) {
    const int64_t np = static_cast<int64_t>(nx) * ny * nz;
    GRID_STRIDE(i, np) {
        double p[3];
        grid_point(i, nx, ny, nz, ox, oy, oz, h, p);
        double t = 0.0;
        for (int a = 0; a < nuc.n; ++a) {
            const double zeta = nuc.z[a] * scale;
            const double s = norm3(p[0] - nuc.r[a][0], p[1] - nuc.r[a][1], p[2] - nuc.r[a][2]);
            t = t + (zeta * zeta * zeta / 3.141592653589793) * exp(-2.0 * zeta * s);
        }
        total[i] = t;
        charge_terms[i] = mass[i] * (t / f2[i]);
    }
}

__global__ void scale_kernel(double* __restrict__ a, int64_t n, double s) {
    GRID_STRIDE(i, n) a[i] = a[i] * s;
}

Nuclei make_nuclei(int n, const double* charges, const double* positions, const double* sphere) {
    Nuclei nuc{};
    nuc.n = n;
    for (int a = 0; a < n; ++a) {
        nuc.z[a] = charges[a];
        for (int d = 0; d < 3; ++d) nuc.r[a][d] = positions[a * 3 + d];
        if (sphere) {
            // sphere rows: centre x, y, z, radius, taper centre, taper width
            for (int d = 0; d < 3; ++d) nuc.centre[a][d] = sphere[a * 6 + d];
            nuc.radius[a] = sphere[a * 6 + 3];
            nuc.taper_centre[a] = sphere[a * 6 + 4];
            nuc.taper_width[a] = sphere[a * 6 + 5];
        }
    }
    return nuc;
}

}  // namespace

}  // namespace cdftb

using namespace cdftb;

// Descriptor of the nuclei on the host: charges (n), positions (n x 3), and per-nucleus sphere rows
// (centre xyz, radius, taper centre, taper width) or NULL.
extern "C" int cdftb_geometry_cusp_fields(int n_atoms, const double* charges, const double* positions, int nx, int ny,
                                          int nz, double ox, double oy, double oz, double spacing, const double* gl4,
                                          double* u, double* grad_u, double* f2, double* transformed_potential,
                                          int* n_averaged, cdftb_stream_t stream) {
    if (n_atoms < 1 || n_atoms > MAX_ATOMS || !charges || !positions || !gl4 || !u || !grad_u || !f2 ||
        !transformed_potential || !n_averaged)
        return CDFTB_ERR_ARGUMENT;
    Nuclei nuc = make_nuclei(n_atoms, charges, positions, nullptr);
    const int64_t np = static_cast<int64_t>(nx) * ny * nz;
    cusp_fields_kernel<<<blocks_for(np, 128), 128, 0, as_stream(stream)>>>(nuc, nx, ny, nz, ox, oy, oz, spacing, 2.0 * spacing,
                                                                            gl4, u, grad_u, f2, transformed_potential,
                                                                            n_averaged);
    return check_launch();
}

extern "C" int cdftb_geometry_face_weights(int n_atoms, const double* charges, const double* positions, int nx, int ny,
                                           int nz, double ox, double oy, double oz, double spacing, int accuracy,
                                           double* w0, double* w1, double* w2, int* underflow, cdftb_stream_t stream) {
    if (n_atoms < 0 || n_atoms > MAX_ATOMS || !w0 || !w1 || !w2 || !underflow || accuracy < 2) return CDFTB_ERR_ARGUMENT;
    Nuclei nuc = make_nuclei(n_atoms, charges, positions, nullptr);
    double* outs[3] = {w0, w1, w2};
    for (int axis = 0; axis < 3; ++axis) {
        int s[3] = {nx, ny, nz};
        s[axis] += accuracy;
        const int64_t total = static_cast<int64_t>(s[0]) * s[1] * s[2];
        face_weights_kernel<<<blocks_for(total, 256), 256, 0, as_stream(stream)>>>(nuc, nx, ny, nz, ox, oy, oz, spacing, axis,
                                                                                    accuracy, outs[axis], underflow);
        int st = check_launch();
        if (st != CDFTB_OK) return st;
    }
    return CDFTB_OK;
}

extern "C" int cdftb_geometry_node_fields(int n_atoms, const double* charges, const double* positions,
                                          const double* spheres, double cell_width, const double* node_points,
                                          const int* owner, const double* base_weights, int64_t m, double* partition,
                                          double* weights, double* f2, double* grad_u, double* transformed_potential,
                                          cdftb_stream_t stream) {
    if (n_atoms < 1 || n_atoms > MAX_ATOMS || !spheres || m < 0) return CDFTB_ERR_ARGUMENT;
    if (m == 0) return CDFTB_OK;
    Nuclei nuc = make_nuclei(n_atoms, charges, positions, spheres);
    nuc.cell_width = cell_width;
    node_fields_kernel<<<blocks_for(m, 128), 128, 0, as_stream(stream)>>>(nuc, node_points, owner, base_weights, m, partition,
                                                                           weights, f2, grad_u, transformed_potential);
    return check_launch();
}

extern "C" int cdftb_geometry_grid_far(int n_atoms, const double* charges, const double* positions, const double* spheres,
                                       int nx, int ny, int nz, double ox, double oy, double oz, double spacing,
                                       const double* f2, double* far, double* far_weights, double* plain_far,
                                       cdftb_stream_t stream) {
    if (n_atoms < 0 || n_atoms > MAX_ATOMS || (n_atoms > 0 && !spheres) || !f2 || !far || !far_weights || !plain_far)
        return CDFTB_ERR_ARGUMENT;
    Nuclei nuc = make_nuclei(n_atoms, charges, positions, spheres);
    const int64_t np = static_cast<int64_t>(nx) * ny * nz;
    grid_far_kernel<<<blocks_for(np, 256), 256, 0, as_stream(stream)>>>(nuc, nx, ny, nz, ox, oy, oz, spacing, f2, far,
                                                                        far_weights, plain_far);
    return check_launch();
}

// The lumped far weights of overlapping spheres. fine_axes: the three fine coordinate arrays
// (lengths nf0, nf1, nf2); m_d: dense (n_d x nf_d) transposed interpolation matrices with band
// ranges lo_d/hi_d (per coarse index) -- the one-dimensional matrices of quadrature.py:449-467.
// work: nf0*nf1*nz + n0*nf1*nz doubles.
extern "C" int cdftb_geometry_lumped_far(int n_atoms, const double* charges, const double* positions,
                                         const double* spheres, int nx, int ny, int nz, double ox, double oy, double oz,
                                         double spacing, int refine, const double* fine_x, const double* fine_y,
                                         const double* fine_z, const double* mx, const int* lox, const int* hix,
                                         const double* my, const int* loy, const int* hiy, const double* mz,
                                         const int* loz, const int* hiz, const double* plain_far, double margin,
                                         double width, double* work, double* lumped_far, cdftb_stream_t stream) {
    if (n_atoms < 1 || n_atoms > MAX_ATOMS || !spheres || refine < 1 || !work || !lumped_far) return CDFTB_ERR_ARGUMENT;
    Nuclei nuc = make_nuclei(n_atoms, charges, positions, spheres);
    cudaStream_t s = as_stream(stream);
    const int nxf = nx * refine, nyf = ny * refine, nzf = nz * refine;
    const double volume = (spacing / refine) * (spacing / refine) * (spacing / refine);
    double* collapsed = work;                                             // [nxf][nyf][nz]
    double* tmp = work + static_cast<int64_t>(nxf) * nyf * nz;            // [nx][nyf][nz]
    const int64_t c_total = static_cast<int64_t>(nxf) * nyf * nz;
    lumped_collapse_kernel<<<blocks_for(c_total, 128), 128, 0, s>>>(nuc, fine_x, nxf, fine_y, nyf, fine_z, nzf, mz, loz, hiz,
                                                                     nz, volume, collapsed);
    int st = check_launch();
    if (st != CDFTB_OK) return st;
    band_contract_kernel<<<blocks_for(static_cast<int64_t>(nx) * nyf * nz, 256), 256, 0, s>>>(
        mx, lox, hix, nx, nxf, collapsed, static_cast<int64_t>(nyf) * nz, tmp);
    if ((st = check_launch()) != CDFTB_OK) return st;
    // reuse `collapsed` for [nx][ny][nz]
    band_contract_mid_kernel<<<blocks_for(static_cast<int64_t>(nx) * ny * nz, 256), 256, 0, s>>>(my, loy, hiy, ny, nyf, tmp,
                                                                                                 nx, nz, collapsed);
    if ((st = check_launch()) != CDFTB_OK) return st;
    lumped_blend_kernel<<<blocks_for(static_cast<int64_t>(nx) * ny * nz, 256), 256, 0, s>>>(
        nx, ny, nz, ox, oy, oz, spacing, margin, width, collapsed, plain_far, lumped_far);
    return check_launch();
}

extern "C" int cdftb_geometry_bare_terms(const double* lifted, const double* far_mass, const double* far_weights,
                                         const double* transformed_potential, const double* f2, int64_t n_points,
                                         double spacing, double* mass, double* potential, double* inverse_weight,
                                         double* quadrature, int* nonpositive, cdftb_stream_t stream) {
    if (!lifted || !far_mass || !far_weights || !transformed_potential || !f2 || !mass || !potential || !inverse_weight ||
        !quadrature || !nonpositive || n_points <= 0)
        return CDFTB_ERR_ARGUMENT;
    const double h3 = spacing * spacing * spacing;
    bare_terms_kernel<<<blocks_for(n_points, 256), 256, 0, as_stream(stream)>>>(lifted, far_mass, far_weights,
                                                                                transformed_potential, f2, n_points, h3, mass,
                                                                                potential, inverse_weight, quadrature,
                                                                                nonpositive);
    return check_launch();
}

extern "C" int cdftb_geometry_step_fields(int n_atoms, const double* charges, const double* positions, int nx, int ny,
                                          int nz, double ox, double oy, double oz, double spacing,
                                          const double* node_points, int64_t m, double* cusp_grid, double* v1s_grid,
                                          double* v1s_node, cdftb_stream_t stream) {
    if (n_atoms < 1 || n_atoms > MAX_ATOMS || !cusp_grid || !v1s_grid || (m > 0 && (!node_points || !v1s_node)))
        return CDFTB_ERR_ARGUMENT;
    Nuclei nuc = make_nuclei(n_atoms, charges, positions, nullptr);
    const int64_t np = static_cast<int64_t>(nx) * ny * nz;
    step_grid_kernel<<<blocks_for(np, 256), 256, 0, as_stream(stream)>>>(nuc, nx, ny, nz, ox, oy, oz, spacing, cusp_grid,
                                                                         v1s_grid);
    int st = check_launch();
    if (st != CDFTB_OK || m == 0) return st;
    step_node_kernel<<<blocks_for(m, 256), 256, 0, as_stream(stream)>>>(nuc, node_points, m, v1s_node);
    return check_launch();
}

extern "C" int cdftb_geometry_initial_density(int n_atoms, const double* charges, const double* positions, int nx, int ny,
                                              int nz, double ox, double oy, double oz, double spacing, double zeta_scale,
                                              const double* f2, const double* mass, double* total, double* charge_terms,
                                              cdftb_stream_t stream) {
    if (n_atoms < 1 || n_atoms > MAX_ATOMS || !f2 || !mass || !total || !charge_terms) return CDFTB_ERR_ARGUMENT;
    Nuclei nuc = make_nuclei(n_atoms, charges, positions, nullptr);
    const int64_t np = static_cast<int64_t>(nx) * ny * nz;
    initial_density_kernel<<<blocks_for(np, 256), 256, 0, as_stream(stream)>>>(nuc, nx, ny, nz, ox, oy, oz, spacing,
                                                                               zeta_scale, f2, mass, total, charge_terms);
    return check_launch();
}

extern "C" int cdftb_scale_f64(double* a, int64_t n, double s, cdftb_stream_t stream) {
    if (!a || n < 0) return CDFTB_ERR_ARGUMENT;
    if (n == 0) return CDFTB_OK;
    scale_kernel<<<blocks_for(n, 256), 256, 0, as_stream(stream)>>>(a, n, s);
    return check_launch();
}
