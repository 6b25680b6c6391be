/*
 * oracle/shim/gsl/hx_gsl_impl.h -- TEST INFRASTRUCTURE ONLY (the CPU oracle's build).
 *
 * GSL 2.7.1 (the version hitomi's install.sh:31 pins) is not installed in this
 * image.  The reference's headers call exactly these GSL routines:
 *   gsl_sf_legendre_sphPlm        tools.hpp:59
 *   gsl_sf_bessel_jl              bessel.hpp:20
 *   gsl_sf_coupling_3j            common.hpp:29 (wigner_3j macro)
 *   gsl_interp_accel_*, gsl_spline_* with gsl_interp_cspline   bessel.hpp:23-36
 * Each is restated here from its published mathematics (no GSL code):
 *   - sphPlm: sqrt((2l+1)/4pi) sqrt((l-m)!/(l+m)!) P_l^m(x) with the Condon-Shortley
 *     phase, via the standard three-term recurrence in l on normalised functions;
 *   - j_l(x): ascending series for x < 1, Miller downward recurrence normalised
 *     by j_0 = sin x / x for 1 <= x < l, upward recurrence from j_0, j_1 for x >= l;
 *   - 3j: Racah's closed-form sum;
 *   - natural cubic spline: c_i = s''(x_i)/2 from the symmetric tridiagonal system
 *     h_{i-1} c_{i-1} + 2 (h_{i-1}+h_i) c_i + h_i c_{i+1} = 3 (dy_i/h_i - dy_{i-1}/h_{i-1}),
 *     c_0 = c_{n-1} = 0, evaluated as y_i + dx (b_i + dx (c_i + dx d_i)).
 * tests/test_oracle_shims.py checks each against scipy.special, scipy.interpolate and
 * sympy's exact 3j symbols.
 */
#ifndef HITOMI_ORACLE_GSL_IMPL_H
#define HITOMI_ORACLE_GSL_IMPL_H

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

/* ---------------------------------------------------------------- Legendre */
static inline double gsl_sf_legendre_sphPlm(const int l, int m, const double x) {
    if (m < 0 || l < m || x < -1.0 || x > 1.0) {
        fprintf(stderr, "gsl_sf_legendre_sphPlm: domain error l=%d m=%d x=%g\n", l, m, x);
        abort();
    }
    /* normalised Y_m^m(x) = (-1)^m sqrt((2m+1)/(4pi) * (2m-1)!!/(2m)!!) (1-x^2)^{m/2} */
    double pmm = 1.0 / sqrt(4.0 * M_PI);
    double s2 = (1.0 - x) * (1.0 + x);
    for (int i = 1; i <= m; i++) pmm *= -sqrt((2.0 * i + 1.0) / (2.0 * i)) * sqrt(s2);
    /* pmm now = (-1)^m sqrt((2m+1)/4pi prod...) ; fix the (2m+1) factor: above used
       product over i of sqrt((2i+1)/(2i)), which equals sqrt((2m+1)!!/(2m)!!) */
    if (l == m) return pmm;
    double pmmp1 = x * sqrt(2.0 * m + 3.0) * pmm;
    if (l == m + 1) return pmmp1;
    double pll = 0.0;
    for (int ll = m + 2; ll <= l; ll++) {
        double a = sqrt((4.0 * ll * ll - 1.0) / ((double)ll * ll - (double)m * m));
        double b = sqrt((((double)(ll - 1) * (ll - 1)) - (double)m * m) / (4.0 * (ll - 1) * (ll - 1) - 1.0));
        pll = a * (x * pmmp1 - b * pmm);
        pmm = pmmp1;
        pmmp1 = pll;
    }
    return pll;
}

/* ---------------------------------------------------------- spherical Bessel */
static inline double hx_jl_series(int l, double x) {
    /* j_l(x) = x^l/(2l+1)!! * sum_k (-x^2/2)^k / (k! (2l+3)(2l+5)...(2l+2k+1)) */
    double pre = 1.0;
    for (int i = 1; i <= l; i++) pre *= x / (2.0 * i + 1.0);
    double y = -0.5 * x * x;
    double term = 1.0, sum = 1.0;
    for (int k = 1; k < 200; k++) {
        term *= y / ((double)k * (2.0 * l + 2.0 * k + 1.0));
        sum += term;
        if (fabs(term) < 1e-18 * fabs(sum)) break;
    }
    return pre * sum;
}

static inline double gsl_sf_bessel_jl(const int l, const double x) {
    if (l < 0 || x < 0.0) {
        fprintf(stderr, "gsl_sf_bessel_jl: domain error l=%d x=%g\n", l, x);
        abort();
    }
    if (x == 0.0) return (l == 0) ? 1.0 : 0.0;
    if (x < 1.0) return hx_jl_series(l, x);
    double j0 = sin(x) / x;
    if (l == 0) return j0;
    if (x >= (double)l) {
        double jm = j0;
        double jc = sin(x) / (x * x) - cos(x) / x;
        for (int k = 1; k < l; k++) {
            double jn = (2.0 * k + 1.0) / x * jc - jm;
            jm = jc;
            jc = jn;
        }
        return jc;
    }
    /* 1 <= x < l : Miller downward recurrence from well above l, normalised by
     * whichever of the closed forms j_0, j_1 is larger at this x (never near a zero). */
    int start = l + 30 + (int)x;
    double jp = 0.0, jc = 1e-300, jl_val = 0.0, j1_u = 0.0, jm;
    for (int k = start; k >= 1; k--) {
        jm = (2.0 * k + 1.0) / x * jc - jp;
        jp = jc;
        jc = jm;
        if (k - 1 == l) jl_val = jc;
        if (k - 1 == 1) j1_u = jc;
        if (fabs(jc) > 1e250) {
            jc *= 1e-250;
            jp *= 1e-250;
            jl_val *= 1e-250;
            j1_u *= 1e-250;
        }
    }
    /* jc is now proportional to j_0, j1_u to j_1 */
    double j1 = sin(x) / (x * x) - cos(x) / x;
    if (fabs(j0) >= fabs(j1)) return jl_val * (j0 / jc);
    return jl_val * (j1 / j1_u);
}

/* ----------------------------------------------------------- Wigner 3j (Racah) */
static inline double hx_lnfact(int n) { return lgamma((double)n + 1.0); }

static inline double gsl_sf_coupling_3j(int two_ja, int two_jb, int two_jc, int two_ma, int two_mb, int two_mc) {
    if (two_ja < 0 || two_jb < 0 || two_jc < 0) {
        fprintf(stderr, "gsl_sf_coupling_3j: domain error\n");
        abort();
    }
    if (two_ma + two_mb + two_mc != 0) return 0.0;
    if (abs(two_ma) > two_ja || abs(two_mb) > two_jb || abs(two_mc) > two_jc) return 0.0;
    if ((two_ja + two_ma) % 2 || (two_jb + two_mb) % 2 || (two_jc + two_mc) % 2) return 0.0;
    if (two_jc > two_ja + two_jb || two_jc < abs(two_ja - two_jb)) return 0.0;
    if ((two_ja + two_jb + two_jc) % 2) return 0.0;
    int ja = two_ja, jb = two_jb, jc = two_jc, ma = two_ma, mb = two_mb, mc = two_mc;
    /* all quantities below are integers because of the parity checks above */
    int a1 = (ja + jb - jc) / 2, a2 = (ja - jb + jc) / 2, a3 = (-ja + jb + jc) / 2;
    int a4 = (ja + jb + jc) / 2 + 1;
    double lndelta = 0.5 * (hx_lnfact(a1) + hx_lnfact(a2) + hx_lnfact(a3) - hx_lnfact(a4));
    double lnpre = 0.5 * (hx_lnfact((ja + ma) / 2) + hx_lnfact((ja - ma) / 2) + hx_lnfact((jb + mb) / 2) +
                          hx_lnfact((jb - mb) / 2) + hx_lnfact((jc + mc) / 2) + hx_lnfact((jc - mc) / 2));
    int kmin = 0;
    int t1 = (jb - jc - ma) / 2;  /* k >= t1 */
    int t2 = (ja - jc + mb) / 2;  /* k >= t2 */
    if (t1 > kmin) kmin = t1;
    if (t2 > kmin) kmin = t2;
    int kmax = a1;
    if ((ja - ma) / 2 < kmax) kmax = (ja - ma) / 2;
    if ((jb + mb) / 2 < kmax) kmax = (jb + mb) / 2;
    double sum = 0.0;
    for (int k = kmin; k <= kmax; k++) {
        double ln = hx_lnfact(k) + hx_lnfact(a1 - k) + hx_lnfact((ja - ma) / 2 - k) + hx_lnfact((jb + mb) / 2 - k) +
                    hx_lnfact(k - t1) + hx_lnfact(k - t2);
        double term = exp(lndelta + lnpre - ln);
        sum += (k % 2) ? -term : term;
    }
    int ph = (ja - jb - mc) / 2;
    return (ph % 2) ? -sum : sum;
}

/* ------------------------------------------------------ natural cubic spline */
typedef struct {
    size_t cache;
} gsl_interp_accel;

typedef struct {
    int kind;
} gsl_interp_type;

static const gsl_interp_type hx_cspline_type = {1};
static const gsl_interp_type *gsl_interp_cspline = &hx_cspline_type;

typedef struct {
    size_t n;
    std::vector<double> *x, *y, *c;
} gsl_spline;

static inline gsl_interp_accel *gsl_interp_accel_alloc(void) {
    gsl_interp_accel *a = (gsl_interp_accel *)malloc(sizeof(gsl_interp_accel));
    a->cache = 0;
    return a;
}
static inline void gsl_interp_accel_free(gsl_interp_accel *a) { free(a); }

static inline gsl_spline *gsl_spline_alloc(const gsl_interp_type *T, size_t n) {
    (void)T;
    gsl_spline *s = (gsl_spline *)malloc(sizeof(gsl_spline));
    s->n = n;
    s->x = new std::vector<double>(n);
    s->y = new std::vector<double>(n);
    s->c = new std::vector<double>(n, 0.0);
    return s;
}

static inline void gsl_spline_free(gsl_spline *s) {
    if (!s) return;
    delete s->x;
    delete s->y;
    delete s->c;
    free(s);
}

static inline int gsl_spline_init(gsl_spline *s, const double *xa, const double *ya, size_t n) {
    std::vector<double> &x = *s->x, &y = *s->y, &c = *s->c;
    for (size_t i = 0; i < n; i++) {
        x[i] = xa[i];
        y[i] = ya[i];
        c[i] = 0.0;
    }
    if (n < 3) return 0;
    size_t m = n - 2; /* unknowns c_1..c_{n-2} */
    std::vector<double> diag(m), off(m), rhs(m);
    for (size_t i = 0; i < m; i++) {
        double h0 = x[i + 1] - x[i];
        double h1 = x[i + 2] - x[i + 1];
        diag[i] = 2.0 * (h0 + h1);
        off[i] = h1;
        rhs[i] = 3.0 * ((y[i + 2] - y[i + 1]) / h1 - (y[i + 1] - y[i]) / h0);
    }
    /* symmetric tridiagonal solve (Thomas) */
    std::vector<double> cp(m), dp(m);
    cp[0] = off[0] / diag[0];
    dp[0] = rhs[0] / diag[0];
    for (size_t i = 1; i < m; i++) {
        double den = diag[i] - off[i - 1] * cp[i - 1];
        cp[i] = off[i] / den;
        dp[i] = (rhs[i] - off[i - 1] * dp[i - 1]) / den;
    }
    c[m] = dp[m - 1];
    for (size_t i = m - 1; i-- > 0;) c[i + 1] = dp[i] - cp[i] * c[i + 2];
    c[0] = 0.0;
    c[n - 1] = 0.0;
    return 0;
}

static inline double gsl_spline_eval(const gsl_spline *s, double xv, gsl_interp_accel *a) {
    const std::vector<double> &x = *s->x, &y = *s->y, &c = *s->c;
    size_t n = s->n;
    if (xv < x[0] || xv > x[n - 1]) {
        fprintf(stderr, "gsl_spline_eval: interpolation error x=%g outside [%g,%g]\n", xv, x[0], x[n - 1]);
        abort();
    }
    size_t lo = 0, hi = n - 1;
    if (a && a->cache < n - 1 && x[a->cache] <= xv && xv < x[a->cache + 1]) {
        lo = a->cache;
    } else {
        while (hi - lo > 1) {
            size_t mid = (lo + hi) / 2;
            if (x[mid] > xv) hi = mid;
            else lo = mid;
        }
        if (a) a->cache = lo;
    }
    if (lo >= n - 1) lo = n - 2;
    double h = x[lo + 1] - x[lo];
    double dx = xv - x[lo];
    double b = (y[lo + 1] - y[lo]) / h - h * (c[lo + 1] + 2.0 * c[lo]) / 3.0;
    double d = (c[lo + 1] - c[lo]) / (3.0 * h);
    return y[lo] + dx * (b + dx * (c[lo] + dx * d));
}

#endif
