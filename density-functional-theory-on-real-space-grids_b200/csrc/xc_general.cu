// (d) Every native semi-local functional of the reference, spin-restricted or spin-polarised, with
// its first derivatives. The reference writes each functional once as an energy density of the
// per-spin ingredients (n_up, n_dn, sigma_uu, sigma_ud, sigma_dd) and differentiates it with
// autograd (src/cdft/xc/base.py:115-189); here the same energy densities are evaluated on
// forward-mode dual numbers that carry all five partial derivatives at once, so v_xc and v_sigma
// are exact derivatives of the energy density (to rounding), with no hand-derived formula.
//
// Conventions kept from base.py:45-80, 171-189:
//   - n_spin = 1: n_up = n_dn = n/2 and sigma_uu = sigma_ud = sigma_dd = sigma/4; n_spin = 2: the
//     rows as given, sigma ordered (uu, ud, dd);
//   - a point with n_up + n_dn < 1e-14 is empty: e = v = v_sigma = 0;
//   - each density channel is clamped at 0.5e-14 and sigma_uu, sigma_dd at 1e-40 (sigma_ud is not
//     clamped); a clamped input passes no derivative (torch's clamp_min rule), and neither does a
//     clamped spin polarisation (base.py:218-226).
// The spin-restricted derivatives follow the chain rule of that split: v = (dE/dn_up + dE/dn_dn)/2,
// v_sigma = (dE/dsigma_uu + dE/dsigma_ud + dE/dsigma_dd)/4.
//
// Functionals (the name table of src/cdft/xc/dispatch.py:26-44), by cdftb_xc_id in cdftb.h:
//   LDA: Slater (lda.py:37-46), VWN5 (lda.py:113-159), PW92 in the original and modified parameter
//   sets (lda.py:49-110), PZ81 (lda.py:162-195); GGA: PBE x (gga.py:43-59), PBE c (gga.py:62-90),
//   B88 x (gga.py:93-122), LYP c (gga.py:125-159); and the combinations lda_vwn, lda_pw92,
//   lda_pw92_mod, lda_pz81, pbe, blyp.

#include "common.cuh"

namespace cdftb {
namespace {

constexpr double kPiX = 3.141592653589793;

// ---- forward-mode dual numbers with N partials
template <int N>
struct Dual {
    double v;
    double d[N];
};

template <int N>
__device__ __forceinline__ Dual<N> constant(double x) {
    Dual<N> r;
    r.v = x;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = 0.0;
    return r;
}

template <int N>
__device__ __forceinline__ Dual<N> variable(double x, int k) {
    Dual<N> r = constant<N>(x);
    if (k < N) r.d[k] = 1.0;
    return r;
}

// x with every partial scaled by s (the chain rule of a unary function with derivative s)
template <int N>
__device__ __forceinline__ Dual<N> chain(double value, double s, const Dual<N>& x) {
    Dual<N> r;
    r.v = value;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = s * x.d[k];
    return r;
}

template <int N>
__device__ __forceinline__ Dual<N> operator+(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    r.v = a.v + b.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] + b.d[k];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator+(const Dual<N>& a, double b) {
    Dual<N> r = a;
    r.v = a.v + b;
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator+(double a, const Dual<N>& b) {
    Dual<N> r = b;
    r.v = a + b.v;
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a) {
    Dual<N> r;
    r.v = -a.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = -a.d[k];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    r.v = a.v - b.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] - b.d[k];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a, double b) {
    Dual<N> r = a;
    r.v = a.v - b;
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(double a, const Dual<N>& b) {
    Dual<N> r;
    r.v = a - b.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = -b.d[k];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    r.v = a.v * b.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(const Dual<N>& a, double b) {
    return chain(a.v * b, b, a);
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(double a, const Dual<N>& b) {
    return chain(a * b.v, a, b);
}
template <int N>
__device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    r.v = a.v / b.v;
    const double bb = b.v * b.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = (a.d[k] * b.v - a.v * b.d[k]) / bb;
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, double b) {
    Dual<N> r;
    r.v = a.v / b;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] / b;
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator/(double a, const Dual<N>& b) {
    return chain(a / b.v, -a / (b.v * b.v), b);
}

template <int N>
__device__ __forceinline__ Dual<N> dsqrt(const Dual<N>& x) {
    const double s = sqrt(x.v);
    return chain(s, 0.5 / s, x);
}
template <int N>
__device__ __forceinline__ Dual<N> dlog(const Dual<N>& x) {
    return chain(log(x.v), 1.0 / x.v, x);
}
template <int N>
__device__ __forceinline__ Dual<N> dlog1p(const Dual<N>& x) {
    return chain(log1p(x.v), 1.0 / (1.0 + x.v), x);
}
template <int N>
__device__ __forceinline__ Dual<N> dexp(const Dual<N>& x) {
    const double e = exp(x.v);
    return chain(e, e, x);
}
template <int N>
__device__ __forceinline__ Dual<N> datan(const Dual<N>& x) {
    return chain(atan(x.v), 1.0 / (1.0 + x.v * x.v), x);
}
template <int N>
__device__ __forceinline__ Dual<N> dasinh(const Dual<N>& x) {
    return chain(asinh(x.v), 1.0 / sqrt(1.0 + x.v * x.v), x);
}
// x^p with autograd's rule p x^(p-1)
template <int N>
__device__ __forceinline__ Dual<N> dpow(const Dual<N>& x, double p) {
    return chain(pow(x.v, p), p * pow(x.v, p - 1.0), x);
}
template <int N>
__device__ __forceinline__ Dual<N> clamp_min(const Dual<N>& x, double floor) {
    return x.v >= floor ? x : constant<N>(floor);
}
template <int N>
__device__ __forceinline__ Dual<N> clamp(const Dual<N>& x, double lo, double hi) {
    if (x.v < lo) return constant<N>(lo);
    if (x.v > hi) return constant<N>(hi);
    return x;
}

// ---- shared building blocks (base.py:196-235)
template <int N>
__device__ __forceinline__ Dual<N> wigner_seitz(const Dual<N>& n) {
    return dpow(3.0 / (4.0 * kPiX * n), 1.0 / 3.0);
}
template <int N>
__device__ __forceinline__ Dual<N> polarisation(const Dual<N>& up, const Dual<N>& dn) {
    return clamp((up - dn) / (up + dn), -1.0 + 1.0e-15, 1.0 - 1.0e-15);
}
template <int N>
__device__ __forceinline__ Dual<N> f_zeta(const Dual<N>& z) {
    return (dpow(1.0 + z, 4.0 / 3.0) + dpow(1.0 - z, 4.0 / 3.0) - 2.0) / (pow(2.0, 4.0 / 3.0) - 2.0);
}
__device__ __forceinline__ double fpp0_exact() { return 4.0 / (9.0 * (pow(2.0, 1.0 / 3.0) - 1.0)); }
__device__ __forceinline__ double slater_unpolarised() { return 0.75 * pow(3.0 / kPiX, 1.0 / 3.0); }
__device__ __forceinline__ double fermi_constant() { return pow(3.0 * kPiX * kPiX, 1.0 / 3.0); }

template <int N>
__device__ __forceinline__ Dual<N> slater(const Dual<N>& up, const Dual<N>& dn) {
    const double factor = pow(2.0, 1.0 / 3.0) * slater_unpolarised();
    return -factor * (dpow(up, 4.0 / 3.0) + dpow(dn, 4.0 / 3.0));
}

// ---- VWN5 (lda.py:113-159)
struct Vwn {
    double a, x0, b, c;
};
template <int N>
__device__ __forceinline__ Dual<N> vwn_aux(const Dual<N>& x, Vwn p) {
    const Dual<N> big_x = x * x + p.b * x + p.c;
    const double big_x0 = p.x0 * p.x0 + p.b * p.x0 + p.c;
    const double q = sqrt(4.0 * p.c - p.b * p.b);
    const Dual<N> at = datan(q / (2.0 * x + p.b));
    return p.a * (dlog(x * x / big_x) + (2.0 * p.b / q) * at -
                  (p.b * p.x0 / big_x0) * (dlog(dpow(x - p.x0, 2.0) / big_x) + (2.0 * (p.b + 2.0 * p.x0) / q) * at));
}
template <int N>
__device__ __forceinline__ Dual<N> vwn5(const Dual<N>& up, const Dual<N>& dn) {
    const Dual<N> n = up + dn;
    const Dual<N> x = dsqrt(wigner_seitz(n));
    const Dual<N> zeta = polarisation(up, dn);
    const Dual<N> para = vwn_aux(x, Vwn{0.0310907, -0.10498, 3.72744, 12.9352});
    const Dual<N> ferro = vwn_aux(x, Vwn{0.01554535, -0.32500, 7.06042, 18.0578});
    const Dual<N> alpha_c = vwn_aux(x, Vwn{-1.0 / (6.0 * kPiX * kPiX), -0.0047584, 1.13107, 13.0045});
    const Dual<N> fz = f_zeta(zeta);
    const Dual<N> z4 = dpow(zeta, 4.0);
    const Dual<N> eps = para + alpha_c * fz * (1.0 - z4) / fpp0_exact() + (ferro - para) * fz * z4;
    return n * eps;
}

// ---- PW92 (lda.py:49-110)
struct Pw {
    double a, a1, b1, b2, b3, b4;
};
template <int N>
__device__ __forceinline__ Dual<N> pw92_g(const Dual<N>& rs, Pw p) {
    const Dual<N> s = dsqrt(rs);
    const Dual<N> den = 2.0 * p.a * (p.b1 * s + p.b2 * rs + p.b3 * rs * s + p.b4 * rs * rs);
    return -2.0 * p.a * (1.0 + p.a1 * rs) * dlog1p(1.0 / den);
}
template <int N>
__device__ __forceinline__ Dual<N> pw92_epsilon(const Dual<N>& rs, const Dual<N>& zeta, bool modified) {
    const Pw para_p = modified ? Pw{0.0310907, 0.21370, 7.5957, 3.5876, 1.6382, 0.49294}
                               : Pw{0.031091, 0.21370, 7.5957, 3.5876, 1.6382, 0.49294};
    const Pw ferro_p = modified ? Pw{0.01554535, 0.20548, 14.1189, 6.1977, 3.3662, 0.62517}
                                : Pw{0.015545, 0.20548, 14.1189, 6.1977, 3.3662, 0.62517};
    const Pw stiff_p = modified ? Pw{0.0168869, 0.11125, 10.357, 3.6231, 0.88026, 0.49671}
                                : Pw{0.016887, 0.11125, 10.357, 3.6231, 0.88026, 0.49671};
    const double fpp0 = modified ? fpp0_exact() : 1.709921;
    const Dual<N> para = pw92_g(rs, para_p);
    const Dual<N> ferro = pw92_g(rs, ferro_p);
    const Dual<N> alpha_c = -pw92_g(rs, stiff_p);
    const Dual<N> fz = f_zeta(zeta);
    const Dual<N> z4 = dpow(zeta, 4.0);
    return para + alpha_c * fz * (1.0 - z4) / fpp0 + (ferro - para) * fz * z4;
}
template <int N>
__device__ __forceinline__ Dual<N> pw92(const Dual<N>& up, const Dual<N>& dn, bool modified) {
    const Dual<N> n = up + dn;
    return n * pw92_epsilon(wigner_seitz(n), polarisation(up, dn), modified);
}

// ---- PZ81 (lda.py:162-195)
struct Pz {
    double gamma, b1, b2, a, b, c, d;
};
template <int N>
__device__ __forceinline__ Dual<N> pz81_epsilon(const Dual<N>& rs, Pz p) {
    if (rs.v >= 1.0) return p.gamma / (1.0 + p.b1 * dsqrt(rs) + p.b2 * rs);
    const Dual<N> l = dlog(rs);
    return p.a * l + p.b + p.c * rs * l + p.d * rs;
}
template <int N>
__device__ __forceinline__ Dual<N> pz81(const Dual<N>& up, const Dual<N>& dn) {
    const Dual<N> n = up + dn;
    const Dual<N> rs = wigner_seitz(n);
    const Dual<N> zeta = polarisation(up, dn);
    const Dual<N> para = pz81_epsilon(rs, Pz{-0.1423, 1.0529, 0.3334, 0.0311, -0.048, 0.0020, -0.0116});
    const Dual<N> ferro = pz81_epsilon(rs, Pz{-0.0843, 1.3981, 0.2611, 0.01555, -0.0269, 0.0007, -0.0048});
    return n * (para + f_zeta(zeta) * (ferro - para));
}

// ---- PBE (gga.py:28-90)
template <int N>
__device__ __forceinline__ Dual<N> pbe_x(const Dual<N>& up, const Dual<N>& dn, const Dual<N>& suu,
                                         const Dual<N>& sdd) {
    const double kappa = 0.804, mu = 0.2195149727645171;
    const double kf = fermi_constant();
    Dual<N> total = constant<N>(0.0);
    const Dual<N>* ns[2] = {&up, &dn};
    const Dual<N>* ss[2] = {&suu, &sdd};
#pragma unroll
    for (int c = 0; c < 2; ++c) {
        const Dual<N> n2 = 2.0 * *ns[c];
        const Dual<N> s2 = (4.0 * *ss[c]) / (4.0 * (kf * kf) * dpow(n2, 8.0 / 3.0));
        const Dual<N> fx = 1.0 + kappa - kappa / (1.0 + mu * s2 / kappa);
        total = total + 0.5 * (-slater_unpolarised() * dpow(n2, 4.0 / 3.0)) * fx;
    }
    return total;
}
template <int N>
__device__ __forceinline__ Dual<N> pbe_c(const Dual<N>& up, const Dual<N>& dn, const Dual<N>& suu,
                                         const Dual<N>& sud, const Dual<N>& sdd) {
    const double beta = 0.06672455060314922;
    const double gamma = (1.0 - log(2.0)) / (kPiX * kPiX);
    const Dual<N> n = up + dn;
    const Dual<N> rs = wigner_seitz(n);
    const Dual<N> zeta = polarisation(up, dn);
    const Dual<N> eps = pw92_epsilon(rs, zeta, true);
    const Dual<N> phi = 0.5 * (dpow(1.0 + zeta, 2.0 / 3.0) + dpow(1.0 - zeta, 2.0 / 3.0));
    const Dual<N> sigma = suu + 2.0 * sud + sdd;
    const Dual<N> k_f = fermi_constant() * dpow(n, 1.0 / 3.0);
    const Dual<N> k_s_sq = 4.0 * k_f / kPiX;
    const Dual<N> t2 = sigma / (4.0 * phi * phi * k_s_sq * n * n);
    const Dual<N> phi3 = dpow(phi, 3.0);
    const Dual<N> a = (beta / gamma) / (dexp(-eps / (gamma * phi3)) - 1.0);
    const Dual<N> at2 = a * t2;
    const Dual<N> h = gamma * phi3 * dlog1p((beta / gamma) * t2 * (1.0 + at2) / (1.0 + at2 + at2 * at2));
    return n * (eps + h);
}

// ---- B88 (gga.py:93-122) and LYP (gga.py:125-159)
template <int N>
__device__ __forceinline__ Dual<N> b88_x(const Dual<N>& up, const Dual<N>& dn, const Dual<N>& suu,
                                         const Dual<N>& sdd) {
    const double beta = 0.0042;
    const double c_lda = 1.5 * pow(3.0 / (4.0 * kPiX), 1.0 / 3.0);
    Dual<N> total = constant<N>(0.0);
    const Dual<N>* ns[2] = {&up, &dn};
    const Dual<N>* ss[2] = {&suu, &sdd};
#pragma unroll
    for (int c = 0; c < 2; ++c) {
        const Dual<N> n43 = dpow(*ns[c], 4.0 / 3.0);
        const Dual<N> x2 = *ss[c] / (n43 * n43);
        const Dual<N> x = dsqrt(x2);
        total = total - c_lda * n43 - beta * n43 * x2 / (1.0 + 6.0 * beta * x * dasinh(x));
    }
    return total;
}
template <int N>
__device__ __forceinline__ Dual<N> lyp_c(const Dual<N>& up, const Dual<N>& dn, const Dual<N>& suu,
                                         const Dual<N>& sud, const Dual<N>& sdd) {
    const double a = 0.04918, b = 0.132, c = 0.2533, d = 0.349;
    const double c_f = 0.3 * pow(3.0 * kPiX * kPiX, 2.0 / 3.0);
    const Dual<N> n = up + dn;
    const Dual<N> n_m13 = dpow(n, -1.0 / 3.0);
    const Dual<N> denom = 1.0 + d * n_m13;
    const Dual<N> omega = dexp(-c * n_m13) / denom * dpow(n, -11.0 / 3.0);
    const Dual<N> delta = c * n_m13 + d * n_m13 / denom;
    const Dual<N> sigma = suu + 2.0 * sud + sdd;
    const Dual<N> nab = up * dn;
    const Dual<N> first = -a * 4.0 / denom * nab / n;
    const Dual<N> bracket =
        nab * (pow(2.0, 11.0 / 3.0) * c_f * (dpow(up, 8.0 / 3.0) + dpow(dn, 8.0 / 3.0)) +
               (47.0 / 18.0 - 7.0 * delta / 18.0) * sigma - (2.5 - delta / 18.0) * (suu + sdd) -
               (delta - 11.0) / 9.0 * (up / n * suu + dn / n * sdd)) -
        (2.0 / 3.0) * n * n * sigma + ((2.0 / 3.0) * n * n - up * up) * sdd + ((2.0 / 3.0) * n * n - dn * dn) * suu;
    return first - a * b * omega * bracket;
}

// cdftb_xc_id (include/cdftb.h)
enum : int {
    LDA_VWN = CDFTB_XC_LDA_VWN, LDA_PW92 = CDFTB_XC_LDA_PW92, LDA_PW92_MOD = CDFTB_XC_LDA_PW92_MOD,
    LDA_PZ81 = CDFTB_XC_LDA_PZ81, PBE = CDFTB_XC_PBE, BLYP = CDFTB_XC_BLYP, LDA_X = CDFTB_XC_LDA_X,
    LDA_C_VWN = CDFTB_XC_LDA_C_VWN, LDA_C_PW = CDFTB_XC_LDA_C_PW, LDA_C_PW_MOD = CDFTB_XC_LDA_C_PW_MOD,
    LDA_C_PZ = CDFTB_XC_LDA_C_PZ, GGA_X_PBE = CDFTB_XC_GGA_X_PBE, GGA_C_PBE = CDFTB_XC_GGA_C_PBE,
    GGA_X_B88 = CDFTB_XC_GGA_X_B88, GGA_C_LYP = CDFTB_XC_GGA_C_LYP, XC_COUNT = CDFTB_XC_GGA_C_LYP + 1
};

__host__ __device__ constexpr bool is_gga(int id) {
    return id == PBE || id == BLYP || id == GGA_X_PBE || id == GGA_C_PBE || id == GGA_X_B88 || id == GGA_C_LYP;
}

template <int ID, int N>
__device__ __forceinline__ Dual<N> energy(const Dual<N>& u, const Dual<N>& dn, const Dual<N>& suu,
                                          const Dual<N>& sud, const Dual<N>& sdd) {
    if constexpr (ID == LDA_X) return slater(u, dn);
    else if constexpr (ID == LDA_C_VWN) return vwn5(u, dn);
    else if constexpr (ID == LDA_C_PW) return pw92(u, dn, false);
    else if constexpr (ID == LDA_C_PW_MOD) return pw92(u, dn, true);
    else if constexpr (ID == LDA_C_PZ) return pz81(u, dn);
    else if constexpr (ID == LDA_VWN) return slater(u, dn) + vwn5(u, dn);
    else if constexpr (ID == LDA_PW92) return slater(u, dn) + pw92(u, dn, false);
    else if constexpr (ID == LDA_PW92_MOD) return slater(u, dn) + pw92(u, dn, true);
    else if constexpr (ID == LDA_PZ81) return slater(u, dn) + pz81(u, dn);
    else if constexpr (ID == GGA_X_PBE) return pbe_x(u, dn, suu, sdd);
    else if constexpr (ID == GGA_C_PBE) return pbe_c(u, dn, suu, sud, sdd);
    else if constexpr (ID == GGA_X_B88) return b88_x(u, dn, suu, sdd);
    else if constexpr (ID == GGA_C_LYP) return lyp_c(u, dn, suu, sud, sdd);
    else if constexpr (ID == PBE) return pbe_x(u, dn, suu, sdd) + pbe_c(u, dn, suu, sud, sdd);
    else return b88_x(u, dn, suu, sdd) + lyp_c(u, dn, suu, sud, sdd);  // BLYP
}

// One thread per point; rows of `p` points: density (n_spin, p), sigma (1 or 3, p), v (n_spin, p),
// vs (1 or 3, p). LDA carries the two density partials, GGA all five.
template <int ID, int NS>
__global__ void __launch_bounds__(128) xc_eval_kernel(const double* __restrict__ density,
                                                      const double* __restrict__ sigma, int64_t p,
                                                      double* __restrict__ e, double* __restrict__ v,
                                                      double* __restrict__ vs) {
    constexpr bool GGA = is_gga(ID);
    constexpr int N = GGA ? 5 : 2;
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < p; i += int64_t(gridDim.x) * blockDim.x) {
        double nu, nd, suu = 0.0, sud = 0.0, sdd = 0.0;
        if (NS == 1) {
            nu = nd = 0.5 * density[i];
            if (GGA) suu = sud = sdd = 0.25 * sigma[i];
        } else {
            nu = density[i];
            nd = density[p + i];
            if (GGA) {
                suu = sigma[i];
                sud = sigma[p + i];
                sdd = sigma[2 * p + i];
            }
        }
        if (!(nu + nd >= 1.0e-14)) {  // an empty point (base.py:176-189)
            e[i] = 0.0;
            v[i] = 0.0;
            if (NS == 2) v[p + i] = 0.0;
            if (GGA) {
                vs[i] = 0.0;
                if (NS == 2) {
                    vs[p + i] = 0.0;
                    vs[2 * p + i] = 0.0;
                }
            }
            continue;
        }
        const double floor = 0.5e-14;
        const Dual<N> u = clamp_min(variable<N>(nu, 0), floor);
        const Dual<N> dn = clamp_min(variable<N>(nd, 1), floor);
        const Dual<N> s_uu = clamp_min(variable<N>(suu, 2), 1.0e-40);
        const Dual<N> s_ud = variable<N>(sud, 3);
        const Dual<N> s_dd = clamp_min(variable<N>(sdd, 4), 1.0e-40);
        const Dual<N> out = energy<ID, N>(u, dn, s_uu, s_ud, s_dd);
        e[i] = out.v;
        if (NS == 1) {
            v[i] = 0.5 * (out.d[0] + out.d[1]);
            if constexpr (GGA) vs[i] = 0.25 * (out.d[2] + out.d[3] + out.d[4]);
        } else {
            v[i] = out.d[0];
            v[p + i] = out.d[1];
            if constexpr (GGA) {
                vs[i] = out.d[2];
                vs[p + i] = out.d[3];
                vs[2 * p + i] = out.d[4];
            }
        }
    }
}

template <int ID>
int launch_xc(int n_spin, const double* density, const double* sigma, int64_t p, double* e, double* v, double* vs,
              cudaStream_t st) {
    // a grid-stride loop: at most 64 CTAs of 128 threads per SM's worth (148 SMs), fewer for small p
    const unsigned blocks = static_cast<unsigned>(ceil_div(p, 128) < 148 * 16 ? ceil_div(p, 128) : 148 * 16);
    if (n_spin == 1)
        xc_eval_kernel<ID, 1><<<blocks, 128, 0, st>>>(density, sigma, p, e, v, vs);
    else
        xc_eval_kernel<ID, 2><<<blocks, 128, 0, st>>>(density, sigma, p, e, v, vs);
    return check_launch();
}

}  // namespace
}  // namespace cdftb

extern "C" int cdftb_xc_is_gga(int functional) {
    if (functional < 0 || functional >= cdftb::XC_COUNT) return -1;
    return cdftb::is_gga(functional) ? 1 : 0;
}

extern "C" int cdftb_xc_eval_f64(int functional, int n_spin, const double* density, const double* sigma, int64_t p,
                                 double* e, double* v, double* v_sigma, cdftb_stream_t stream) {
    using namespace cdftb;
    if (functional < 0 || functional >= XC_COUNT || (n_spin != 1 && n_spin != 2) || p < 0) return CDFTB_ERR_ARGUMENT;
    if (p == 0) return CDFTB_OK;
    if (!density || !e || !v || (is_gga(functional) && (!sigma || !v_sigma))) return CDFTB_ERR_ARGUMENT;
    cudaStream_t st = as_stream(stream);
    switch (functional) {
        case LDA_VWN: return launch_xc<LDA_VWN>(n_spin, density, sigma, p, e, v, v_sigma, st);
        case LDA_PW92: return launch_xc<LDA_PW92>(n_spin, density, sigma, p, e, v, v_sigma, st);
        case LDA_PW92_MOD: return launch_xc<LDA_PW92_MOD>(n_spin, density, sigma, p, e, v, v_sigma, st);
        case LDA_PZ81: return launch_xc<LDA_PZ81>(n_spin, density, sigma, p, e, v, v_sigma, st);
        case PBE: return launch_xc<PBE>(n_spin, density, sigma, p, e, v, v_sigma, st);
        case BLYP: return launch_xc<BLYP>(n_spin, density, sigma, p, e, v, v_sigma, st);
        case LDA_X: return launch_xc<LDA_X>(n_spin, density, sigma, p, e, v, v_sigma, st);
        case LDA_C_VWN: return launch_xc<LDA_C_VWN>(n_spin, density, sigma, p, e, v, v_sigma, st);
        case LDA_C_PW: return launch_xc<LDA_C_PW>(n_spin, density, sigma, p, e, v, v_sigma, st);
        case LDA_C_PW_MOD: return launch_xc<LDA_C_PW_MOD>(n_spin, density, sigma, p, e, v, v_sigma, st);
        case LDA_C_PZ: return launch_xc<LDA_C_PZ>(n_spin, density, sigma, p, e, v, v_sigma, st);
        case GGA_X_PBE: return launch_xc<GGA_X_PBE>(n_spin, density, sigma, p, e, v, v_sigma, st);
        case GGA_C_PBE: return launch_xc<GGA_C_PBE>(n_spin, density, sigma, p, e, v, v_sigma, st);
        case GGA_X_B88: return launch_xc<GGA_X_B88>(n_spin, density, sigma, p, e, v, v_sigma, st);
        default: return launch_xc<GGA_C_LYP>(n_spin, density, sigma, p, e, v, v_sigma, st);
    }
}
