// hg_common.cuh -- shared device/host helpers for the hitomi B200 estimator library.
//
// Every formula that decides a bin, a shell, a window or a harmonic is evaluated
// here in FP64 with the same expression order as the reference
// (src/hitomi_measurement/field.hpp, tools.hpp), using non-contracting intrinsics
// where the reference's rounding decides an integer (bin index, shell membership).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cmath>

#ifndef HG_PI
#define HG_PI 3.14159265358979323846
#endif

#ifndef HG_TU_NS
#error "define HG_TU_NS (a namespace name unique to this translation unit) before including"
#endif

namespace hg {
// one copy per translation unit: each .cu file names its own HG_TU_NS, so the kernels and
// helpers of this header never collide at link time
inline namespace HG_TU_NS {

template <typename T>
struct cplx {
    T x, y;
};

template <typename T>
__host__ __device__ __forceinline__ cplx<T> mk(T a, T b) {
    cplx<T> c;
    c.x = a;
    c.y = b;
    return c;
}
template <typename T>
__host__ __device__ __forceinline__ cplx<T> operator+(cplx<T> a, cplx<T> b) { return mk<T>(a.x + b.x, a.y + b.y); }
template <typename T>
__host__ __device__ __forceinline__ cplx<T> operator-(cplx<T> a, cplx<T> b) { return mk<T>(a.x - b.x, a.y - b.y); }
template <typename T>
__host__ __device__ __forceinline__ cplx<T> operator*(cplx<T> a, cplx<T> b) {
    return mk<T>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename T>
__host__ __device__ __forceinline__ cplx<T> operator*(cplx<T> a, T s) { return mk<T>(a.x * s, a.y * s); }
template <typename T>
__host__ __device__ __forceinline__ cplx<T> conjg(cplx<T> a) { return mk<T>(a.x, -a.y); }
// a conj(b) with every product and sum rounded separately, as std::complex<double> evaluates
// it on the host: the imaginary part of a conj(a) is then exactly zero (a fused multiply-add
// would leave the rounding error of one product in it)
__device__ __forceinline__ cplx<double> mul_conj_rn(cplx<double> a, cplx<double> b) {
    return mk<double>(__dadd_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)),
                      __dsub_rn(__dmul_rn(a.y, b.x), __dmul_rn(a.x, b.y)));
}

typedef cplx<double> zd;
typedef cplx<float> zf;

// Device-side bounds checks of the check build (-DHG_CHECK, libhitomi_b200_check.so): a
// failed check counts itself in hg_check_word[0], the first one also records its site code
// and the offending index, and the guarded access is skipped, so nothing faults; the engine
// reads the word at the end of every API call and fails the call with that record.  Without
// HG_CHECK every check is the constant true and compiles to nothing.
#ifdef HG_CHECK
__device__ unsigned long long hg_check_word[3];  // failures, site code, index
__device__ __forceinline__ bool hg_check(bool ok, int site, long long index) {
    if (ok) return true;
    if (atomicAdd(&hg_check_word[0], 1ull) == 0ull) {
        hg_check_word[1] = (unsigned long long)site;
        hg_check_word[2] = (unsigned long long)index;
    }
    return false;
}
#define HG_IN_BOUNDS(cond, site, index) hg_check((cond), (site), (long long)(index))
#else
#define HG_IN_BOUNDS(cond, site, index) true
#endif
// check sites (the code a failed check reports)
enum HgCheckSite {
    HG_SITE_RECORD = 1,       // a particle record outside its tile's range (k_bin_scatter)
    HG_SITE_TILE_CELL = 2,    // a stencil point outside the CTA's tile (k_tile_accum*)
    HG_SITE_MESH_CELL = 3,    // a mesh cell outside the mesh (tile write-out)
    HG_SITE_CROWD = 4,        // a staging slot outside the staging buffer
    HG_SITE_BIN = 5,          // a coarse bin outside the binning arrays (k_pk_bin)
    HG_SITE_CHAIN_ROW = 6,    // a chain row outside the kept cube (k_chain_x*)
    HG_SITE_MIXED = 7,        // a mixed-radix line index outside the line (k_fft_pass_mixed)
};

// Wrapped integer mode / offset of array index i on an axis of n cells, the rule
// of field.hpp:363-365: index i < n/2 is i, otherwise i - n.
__host__ __device__ __forceinline__ int wrap_index(int i, int n) { return (i < n / 2) ? i : i - n; }

// (a, b, c) with idx = (a * nb + b) * nc + c, in 32-bit unsigned arithmetic (every linear
// index of a supported mesh is below 2^31; 64-bit division costs several times more)
__device__ __forceinline__ void split3(unsigned idx, unsigned nb, unsigned nc, int &a, int &b, int &c) {
    const unsigned q = idx / nc;
    c = (int)(idx - q * nc);
    const unsigned r = q / nb;
    b = (int)(q - r * nb);
    a = (int)r;
}

// (n - i) mod n for 0 <= i < n: the index of -k
__host__ __device__ __forceinline__ int neg_index(int i, int n) { return i ? n - i : 0; }

// Axis constants shared by the k-space kernels (all FP64).
struct Grid {
    int n[3];          // mesh cells per axis
    double L[3];       // box size per axis
    double dk[3];      // 2 pi / L  (field.hpp:357-359)
    double dr[3];      // L / n     (field.hpp:940-942)
    double volume;     // L0 L1 L2
    long long ntot;    // n0 n1 n2
};

// kvec component for wrapped mode index n on an axis: (double) n * dk
// (field.hpp:363: `(double) i * dk[0]` or `(double) (i - n) * dk[0]`).
__host__ __device__ __forceinline__ double kcomp(int nwrap, double dk) { return (double)nwrap * dk; }

// |k| = sqrt(kx*kx + ky*ky + kz*kz), left-to-right, no FMA contraction (field.hpp:366).
__device__ __forceinline__ double kmag_exact(double kx, double ky, double kz) {
    double s = __dadd_rn(__dadd_rn(__dmul_rn(kx, kx), __dmul_rn(ky, ky)), __dmul_rn(kz, kz));
    return __dsqrt_rn(s);
}
static inline double kmag_exact_host(double kx, double ky, double kz) {
    volatile double a = kx * kx;
    volatile double b = ky * ky;
    volatile double c = kz * kz;
    volatile double s = a + b;
    s = s + c;
    return std::sqrt((double)s);
}

// Integer the reference derives from a kvec component inside the window and shot-noise
// functions: (int)(kvec / dk + 1e-5)  (field.hpp:667-669, 1264-1266).  For negative
// modes this is n + 1, not n -- reproduced, not corrected.
__device__ __forceinline__ int window_index(double kv, double dk) {
    return (int)__dadd_rn(__ddiv_rn(kv, dk), 1.0e-5);
}

// sin(x)/x factor per axis with the reference's zero test (field.hpp:670-675).
__device__ __forceinline__ double sinc_axis(int i, int n) {
    if (i == 0) return 1.0;
    double x = HG_PI * (double)i / (double)n;
    return sin(x) / x;
}

// Assignment-function window W(k) = (prod sinc)^p, p = 1,2,3 for NGP/CIC/TSC
// (field.hpp:641-717) and p = 4 for PCS (project extension).
__device__ __forceinline__ double window_fn(const double kv[3], const Grid &g, int p) {
    int i = window_index(kv[0], g.dk[0]);
    int j = window_index(kv[1], g.dk[1]);
    int k = window_index(kv[2], g.dk[2]);
    double ret = sinc_axis(i, g.n[0]) * sinc_axis(j, g.n[1]) * sinc_axis(k, g.n[2]);
    double w = ret;
    for (int q = 1; q < p; q++) w *= ret;
    return w;
}

// Aliasing shot-noise function C(k) of Jing (2005) eq. 20 (field.hpp:1252-1310);
// PCS (project extension) uses prod(1 - 4/3 s^2 + 2/5 s^4 - 4/315 s^6).
__device__ __forceinline__ double shotnoise_fn(const double kv[3], const Grid &g, int assign) {
    if (assign == 0) return 1.0;
    int id[3] = {window_index(kv[0], g.dk[0]), window_index(kv[1], g.dk[1]), window_index(kv[2], g.dk[2])};
    double ret = 1.0;
    for (int a = 0; a < 3; a++) {
        double s = (id[a] != 0) ? sin(HG_PI * (double)id[a] / (double)g.n[a]) : 0.0;
        double s2 = s * s;
        double f;
        if (assign == 1) f = 1.0 - (2.0 / 3.0) * s2;
        else if (assign == 2) f = 1.0 - s2 + 2.0 * (s2 * s2) / 15.0;
        else f = 1.0 - (4.0 / 3.0) * s2 + (2.0 / 5.0) * s2 * s2 - (4.0 / 315.0) * s2 * s2 * s2;
        ret *= f;
    }
    return ret;
}

// Reduced spherical harmonic  Yhat_lm(v) = conj(Y_lm(v_hat)) sqrt(4 pi / (2l+1))
// (tools.hpp:12-68), Condon-Shortley phase included, Y_l^{-m} = (-1)^m conj(Y_l^m).
// Evaluated with the normalised associated-Legendre recurrence on P_l^|m| / sin^|m|
// and the azimuthal factor (sin theta e^{+-i phi})^|m| = ((x +- i y)/r)^|m|, which is
// algebraically the reference's acos/exp form without its loss of accuracy near the axes.
__host__ __device__ inline zd ylm_reduced(int l, int m, double x, double y, double z) {
    if (l == 0 && m == 0) return mk<double>(1.0, 0.0);
    double r = sqrt(x * x + y * y + z * z);
    if (fabs(r) < 1.0e-15) return mk<double>(0.0, 0.0);
    double mu = z / r;
    int am = m < 0 ? -m : m;
    double pmm = 1.0 / sqrt(4.0 * HG_PI);
    for (int i = 1; i <= am; i++) pmm *= -sqrt((2.0 * i + 1.0) / (2.0 * i));
    double plm;
    if (l == am) {
        plm = pmm;
    } else {
        double p1 = mu * sqrt(2.0 * am + 3.0) * pmm;
        if (l == am + 1) {
            plm = p1;
        } else {
            double p0 = pmm, pl = 0.0;
            for (int ll = am + 2; ll <= l; ll++) {
                double a = sqrt((4.0 * ll * ll - 1.0) / ((double)ll * ll - (double)am * am));
                double b = sqrt((((double)(ll - 1) * (ll - 1)) - (double)am * am) / (4.0 * (ll - 1) * (ll - 1) - 1.0));
                pl = a * (mu * p1 - b * p0);
                p0 = p1;
                p1 = pl;
            }
            plm = pl;
        }
    }
    // (sin theta e^{i sgn(m) phi})^|m|
    double ex = 1.0, ey = 0.0;
    double ux = x / r, uy = (m < 0 ? -y : y) / r;
    for (int i = 0; i < am; i++) {
        double tx = ex * ux - ey * uy;
        double ty = ex * uy + ey * ux;
        ex = tx;
        ey = ty;
    }
    double sgn = (m < 0 && (am & 1)) ? -1.0 : 1.0;  // (-1)^((M-|M|)/2)
    double norm = sqrt(4.0 * HG_PI / (2.0 * l + 1.0));
    // conj(sgn * plm * e) * norm
    return mk<double>(sgn * plm * ex * norm, -sgn * plm * ey * norm);
}

}  // namespace HG_TU_NS
}  // namespace hg
