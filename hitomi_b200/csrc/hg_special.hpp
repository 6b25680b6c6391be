// hg_special.hpp -- host-side special functions the estimators need (FP64).
//
//  * Wigner 3j symbol (Racah's closed form) -- the coupling weights the reference takes
//    from gsl_sf_coupling_3j through its wigner_3j macro (common.hpp:29).
//  * Spherical Bessel j_l(x) -- series for x < 1, Miller downward recurrence for
//    1 <= x < l, upward recurrence from the closed forms j_0, j_1 for x >= l.
//  * The reference evaluates j_l through a natural cubic spline of 10^6 knots on
//    [0, 1e4] (bessel.hpp:10-37).  The spline, not exact j_l, is what its results
//    contain (interpolation error ~1e-10), so BesselSpline rebuilds that same spline:
//    knots x_i = i * dx, values j_l(x_i), second-derivative coefficients c_i from the
//    natural-boundary tridiagonal system, evaluated as y_i + t (b_i + t (c_i + t d_i)).
#pragma once

#include <cmath>
#include <cstdlib>
#include <vector>

namespace hg {
// one copy per translation unit: each .cu file names its own HG_TU_NS, so the kernels and
// helpers of this header never collide at link time
inline namespace HG_TU_NS {

inline double lnfact(int n) { return std::lgamma((double)n + 1.0); }

// (j1 j2 j3; m1 m2 m3) for integer arguments.
inline double wigner3j(int j1, int j2, int j3, int m1, int m2, int m3) {
    if (j1 < 0 || j2 < 0 || j3 < 0) return 0.0;
    if (m1 + m2 + m3 != 0) return 0.0;
    if (std::abs(m1) > j1 || std::abs(m2) > j2 || std::abs(m3) > j3) return 0.0;
    if (j3 > j1 + j2 || j3 < std::abs(j1 - j2)) return 0.0;
    int a1 = j1 + j2 - j3, a2 = j1 - j2 + j3, a3 = -j1 + j2 + j3, a4 = j1 + j2 + j3 + 1;
    double lndelta = 0.5 * (lnfact(a1) + lnfact(a2) + lnfact(a3) - lnfact(a4));
    double lnpre = 0.5 * (lnfact(j1 + m1) + lnfact(j1 - m1) + lnfact(j2 + m2) + lnfact(j2 - m2) + lnfact(j3 + m3) +
                          lnfact(j3 - m3));
    int t1 = j2 - j3 - m1, t2 = j1 - j3 + m2;
    int kmin = 0;
    if (t1 > kmin) kmin = t1;
    if (t2 > kmin) kmin = t2;
    int kmax = a1;
    if (j1 - m1 < kmax) kmax = j1 - m1;
    if (j2 + m2 < kmax) kmax = j2 + m2;
    double sum = 0.0;
    for (int k = kmin; k <= kmax; k++) {
        double ln = lnfact(k) + lnfact(a1 - k) + lnfact(j1 - m1 - k) + lnfact(j2 + m2 - k) + lnfact(k - t1) +
                    lnfact(k - t2);
        double term = std::exp(lndelta + lnpre - ln);
        sum += (k & 1) ? -term : term;
    }
    int ph = j1 - j2 - m3;
    return (ph & 1) ? -sum : sum;
}

inline double sph_bessel_series(int l, double x) {
    double pre = 1.0;
    for (int i = 1; i <= l; i++) pre *= x / (2.0 * i + 1.0);
    double y = -0.5 * x * x, term = 1.0, sum = 1.0;
    for (int k = 1; k < 200; k++) {
        term *= y / ((double)k * (2.0 * l + 2.0 * k + 1.0));
        sum += term;
        if (std::fabs(term) < 1e-18 * std::fabs(sum)) break;
    }
    return pre * sum;
}

inline double sph_bessel(int l, double x) {
    if (x == 0.0) return (l == 0) ? 1.0 : 0.0;
    if (x < 1.0) return sph_bessel_series(l, x);
    double s = std::sin(x), c = std::cos(x);
    double j0 = s / x;
    if (l == 0) return j0;
    double j1 = s / (x * x) - c / x;
    if (x >= (double)l) {
        double jm = j0, jc = j1;
        for (int k = 1; k < l; k++) {
            double jn = (2.0 * k + 1.0) / x * jc - jm;
            jm = jc;
            jc = jn;
        }
        return jc;
    }
    int start = l + 30 + (int)x;
    double jp = 0.0, jc = 1e-300, jl = 0.0, j1u = 0.0;
    for (int k = start; k >= 1; k--) {
        double jm = (2.0 * k + 1.0) / x * jc - jp;
        jp = jc;
        jc = jm;
        if (k - 1 == l) jl = jc;
        if (k - 1 == 1) j1u = jc;
        if (std::fabs(jc) > 1e250) {
            jc *= 1e-250;
            jp *= 1e-250;
            jl *= 1e-250;
            j1u *= 1e-250;
        }
    }
    if (std::fabs(j0) >= std::fabs(j1)) return jl * (j0 / jc);
    return jl * (j1 / j1u);
}

// Natural cubic spline of j_l on the reference's knot set (bessel.hpp:14-25).
struct BesselSpline {
    int l = -1;
    double xmin = 0.0, xmax = 10000.0, dx = 0.0;
    int n = 1000000;
    std::vector<double> x, y, c;  // knots, values, c_i = s''(x_i)/2

    void build(int ell) {
        l = ell;
        dx = (xmax - xmin) / double(n - 1);
        x.resize(n);
        y.resize(n);
        c.assign(n, 0.0);
        for (int i = 0; i < n; i++) {
            x[i] = xmin + dx * double(i);
            y[i] = sph_bessel(ell, x[i]);
        }
        int m = n - 2;
        std::vector<double> cp(m), dp(m);
        for (int i = 0; i < m; i++) {
            double h0 = x[i + 1] - x[i], h1 = x[i + 2] - x[i + 1];
            double diag = 2.0 * (h0 + h1);
            double rhs = 3.0 * ((y[i + 2] - y[i + 1]) / h1 - (y[i + 1] - y[i]) / h0);
            double offm = h0;  // coupling to the previous unknown
            if (i == 0) {
                cp[i] = h1 / diag;
                dp[i] = rhs / diag;
            } else {
                double den = diag - offm * cp[i - 1];
                cp[i] = h1 / den;
                dp[i] = (rhs - offm * dp[i - 1]) / den;
            }
        }
        c[m] = dp[m - 1];
        for (int i = m - 2; i >= 0; i--) c[i + 1] = dp[i] - cp[i] * c[i + 2];
        c[0] = 0.0;
        c[n - 1] = 0.0;
    }

    double eval(double xv) const {
        if (xv < x[0] || xv > x[n - 1]) return NAN;
        long i = (long)((xv - xmin) / dx);
        if (i > n - 2) i = n - 2;
        if (i < 0) i = 0;
        while (i > 0 && x[i] > xv) i--;
        while (i < n - 2 && x[i + 1] <= xv) i++;
        double h = x[i + 1] - x[i], t = xv - x[i];
        double b = (y[i + 1] - y[i]) / h - h * (c[i + 1] + 2.0 * c[i]) / 3.0;
        double d = (c[i + 1] - c[i]) / (3.0 * h);
        return y[i] + t * (b + t * (c[i] + t * d));
    }
};

}  // namespace HG_TU_NS
}  // namespace hg
