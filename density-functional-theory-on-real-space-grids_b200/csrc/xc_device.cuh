// (d) Spin-restricted LDA (Slater + VWN5) and PBE energy densities with closed-form first
// derivatives, per point. The reference evaluates the same energy densities and differentiates
// them with autograd (src/cdft/xc/base.py:115-189, lda.py:113-159, 201-217, gga.py:28-90); here the
// derivatives are written out by hand. Conventions kept: the density is split n_up = n_dn = n/2
// and each channel clamped at 0.5e-14, a point with n < 1e-14 is empty (e = v = v_sigma = 0),
// sigma_uu = sigma_dd = max(sigma/4, 1e-40) with sigma_ud = sigma/4 unclamped (base.py:45-80,
// 171-189). At zeta = 0 every spin-interpolation term and its derivative vanish.
#pragma once

#include <math.h>

namespace cdftb {
namespace xc {

constexpr double kDensityThreshold = 1.0e-14;
constexpr double kSigmaThreshold = 1.0e-40;
constexpr double kPi = 3.141592653589793;

// (3/4)(3/pi)^(1/3) and (3 pi^2)^(1/3), as the reference computes them in double.
__device__ __forceinline__ double slater_constant() { return 0.75 * cbrt(3.0 / kPi); }
__device__ __forceinline__ double kf_constant() { return cbrt(3.0 * kPi * kPi); }

struct VWNParams {
    double a, x0, b, c;
};

// VWN eq. (4.4) fit and its x-derivative (lda.py:122-134).
__device__ __forceinline__ void vwn_aux(double x, VWNParams p, double& value, double& deriv) {
    const double big_x = x * x + p.b * x + p.c;
    const double big_x0 = p.x0 * p.x0 + p.b * p.x0 + p.c;
    const double q = sqrt(4.0 * p.c - p.b * p.b);
    const double at = atan(q / (2.0 * x + p.b));
    const double xm = x - p.x0;
    const double r = p.b * p.x0 / big_x0;
    value = p.a * (log(x * x / big_x) + (2.0 * p.b / q) * at - r * (log(xm * xm / big_x) + (2.0 * (p.b + 2.0 * p.x0) / q) * at));
    const double dx = 2.0 * x + p.b;
    deriv = p.a * (2.0 / x - dx / big_x - p.b / big_x - r * (2.0 / xm - dx / big_x - (p.b + 2.0 * p.x0) / big_x));
}

// Slater exchange + VWN5 correlation: e (per volume) and v = de/dn.
__device__ __forceinline__ void lda_vwn(double n, double& e, double& v) {
    if (!(n >= kDensityThreshold)) {
        e = 0.0;
        v = 0.0;
        return;
    }
    const double floor = 0.5 * kDensityThreshold;
    const double nu = fmax(0.5 * n, floor);
    const double factor = cbrt(2.0) * slater_constant();
    const double nu13 = cbrt(nu);
    const double ex = -factor * (2.0 * (nu * nu13));
    const double vx = -(4.0 / 3.0) * factor * nu13;
    const double nt = nu + nu;
    const double rs = cbrt(3.0 / (4.0 * kPi * nt));
    const double x = sqrt(rs);
    double eps, deps;
    vwn_aux(x, VWNParams{0.0310907, -0.10498, 3.72744, 12.9352}, eps, deps);
    e = ex + nt * eps;
    v = vx + eps - (x / 6.0) * deps;
}

struct PW92Params {
    double a, a1, b1, b2, b3, b4;
};

// PW92 G(rs) (lda.py:55-61) and dG/drs.
__device__ __forceinline__ void pw92_g(double rs, PW92Params p, double& g, double& dg) {
    const double s = sqrt(rs);
    const double den = 2.0 * p.a * (p.b1 * s + p.b2 * rs + p.b3 * rs * s + p.b4 * rs * rs);
    const double dden = 2.0 * p.a * (p.b1 / (2.0 * s) + p.b2 + 1.5 * p.b3 * s + 2.0 * p.b4 * rs);
    const double l = log1p(1.0 / den);
    const double dl = -dden / (den * (den + 1.0));
    g = -2.0 * p.a * (1.0 + p.a1 * rs) * l;
    dg = -2.0 * p.a * p.a1 * l - 2.0 * p.a * (1.0 + p.a1 * rs) * dl;
}

// PBE exchange + correlation (gga.py:28-90): e, v = de/dn, vs = de/dsigma.
__device__ __forceinline__ void pbe(double n, double sigma, double& e, double& v, double& vs) {
    if (!(n >= kDensityThreshold)) {
        e = 0.0;
        v = 0.0;
        vs = 0.0;
        return;
    }
    const double kappa = 0.804, mu = 0.2195149727645171;
    const double beta = 0.06672455060314922;
    const double gamma = (1.0 - log(2.0)) / (kPi * kPi);
    const double kf = kf_constant();
    const double cx = slater_constant();
    const double floor = 0.5 * kDensityThreshold;
    const double nu = fmax(0.5 * n, floor);
    const double s_quarter = 0.25 * sigma;
    const bool s_clamped = !(s_quarter >= kSigmaThreshold);
    const double s_c = s_clamped ? kSigmaThreshold : s_quarter;
    // exchange: two equal channels of (1/2) e_x^unif(2 n_s) F_x(s^2), n2 = 2 n_s
    const double n2 = 2.0 * nu;
    const double n2_13 = cbrt(n2);
    const double n2_43 = n2 * n2_13;
    const double n2_83 = n2_43 * n2_43;
    const double s2 = (4.0 * s_c) / (4.0 * kf * kf * n2_83);
    const double den = 1.0 + mu * s2 / kappa;
    const double fx = 1.0 + kappa - kappa / den;
    const double dfx = mu / (den * den);
    const double ex = -cx * n2_43 * fx;
    const double vx = cx * n2_13 * (-(4.0 / 3.0) * fx + (8.0 / 3.0) * dfx * s2);
    const double vsx = s_clamped ? 0.0 : -cx * n2_43 * dfx / (4.0 * kf * kf * n2_83);
    // correlation: PW92 (modified) at zeta = 0, phi = 1
    const double nt = nu + nu;
    const double rs = cbrt(3.0 / (4.0 * kPi * nt));
    double eps, deps_drs;
    pw92_g(rs, PW92Params{0.0310907, 0.21370, 7.5957, 3.5876, 1.6382, 0.49294}, eps, deps_drs);
    const double deps_dn = deps_drs * (-rs / (3.0 * nt));
    const double sig_tot = s_c + 2.0 * s_quarter + s_c;
    const double dsig_tot = (s_clamped ? 0.0 : 0.5) + 0.5;
    const double k_f = kf * cbrt(nt);
    const double k_s_sq = 4.0 * k_f / kPi;
    const double t2 = sig_tot / (4.0 * k_s_sq * nt * nt);
    const double bg = beta / gamma;
    const double ex_eps = exp(-eps / gamma);
    const double a = bg / (ex_eps - 1.0);
    const double da_deps = bg * ex_eps / (gamma * (ex_eps - 1.0) * (ex_eps - 1.0));
    const double at2 = a * t2;
    const double num = t2 * (1.0 + at2);
    const double dd = 1.0 + at2 + at2 * at2;
    const double ratio = num / dd;
    const double h = gamma * log1p(bg * ratio);
    const double common = gamma * bg / (1.0 + bg * ratio);
    const double dr_dy = ((1.0 + 2.0 * at2) * dd - num * (a + 2.0 * a * at2)) / (dd * dd);
    const double dr_da = (t2 * t2 * dd - num * (t2 + 2.0 * at2 * t2)) / (dd * dd);
    const double dh_dy = common * dr_dy;
    const double dh_da = common * dr_da;
    const double dy_dn = -(7.0 / 3.0) * t2 / nt;
    const double dy_ds = dsig_tot / (4.0 * k_s_sq * nt * nt);
    const double ec = nt * (eps + h);
    const double vc = eps + h + nt * (deps_dn + dh_da * da_deps * deps_dn + dh_dy * dy_dn);
    const double vsc = nt * dh_dy * dy_ds;
    e = ex + ec;
    v = vx + vc;
    vs = vsx + vsc;
}

}  // namespace xc
}  // namespace cdftb
