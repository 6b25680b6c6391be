/*
 * oracle/shim/fftw3.h -- TEST INFRASTRUCTURE ONLY (the CPU oracle's build).
 *
 * FFTW 3.3.10 (the version hitomi's install.sh:30 pins) is not installed in this
 * image, so the reference's headers cannot be compiled as shipped.  This header
 * provides exactly the FFTW subset those headers call (src/hitomi_measurement/
 * field.hpp:321-323,339-341,391-393,440-442,902-904,1024-1026,1154-1156 and
 * particle_reconstruction.hpp:107-115), backed by a project-written double
 * precision mixed-radix FFT.  The transform is FFTW's unnormalised convention:
 *   FFTW_FORWARD  (-1):  X[k] = sum_j x[j] exp(-2 pi i j k / n)
 *   FFTW_BACKWARD (+1):  X[k] = sum_j x[j] exp(+2 pi i j k / n)
 * applied along each of the three axes of a row-major n0 x n1 x n2 array.
 *
 * Algorithm: power-of-two lengths use an iterative Stockham autosort FFT (radix 4,
 * one radix-2 stage when log2 n is odd); other lengths a recursive Cooley-Tukey over
 * their prime factors with direct DFTs of the odd primes.  Twiddles come from sincos
 * of an exactly reduced angle.  Nothing here is FFTW's code.  tests/test_oracle_shims.py
 * checks it against numpy.fft (pocketfft) for power-of-two, mixed and prime lengths, both
 * signs: <= 6e-16 of the largest output.  FFTW itself is not in this image, so the distance
 * to FFTW's own rounding is not measured; two correctly rounded double FFTs differ at the
 * same ~1e-16 level, far inside the oracle's 1e-10 budget.
 */
#ifndef HITOMI_ORACLE_FFTW3_SHIM_H
#define HITOMI_ORACLE_FFTW3_SHIM_H

#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <vector>

typedef double fftw_complex[2];

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_ESTIMATE (1U << 6)

struct hx_fftw_plan_s {
    int n[3];
    fftw_complex *in;
    fftw_complex *out;
    int sign;
};
typedef hx_fftw_plan_s *fftw_plan;

/* Zero-filled, unlike FFTW's allocator: the reference's reconstruction skips the k = 0
 * element of its displacement arrays without writing it (particle_reconstruction.hpp:64-71)
 * and then transforms it, so with an uninitialised block its result depends on what the heap
 * held (a uniform shift of one coordinate).  Zero is what a fresh page gives and what the
 * method intends (no displacement from the mean density). */
static inline fftw_complex *fftw_alloc_complex(size_t n) {
    void *p = nullptr;
    const size_t bytes = (n ? n : 1) * sizeof(fftw_complex);
    if (posix_memalign(&p, 64, bytes) != 0) return nullptr;
    memset(p, 0, bytes);
    return (fftw_complex *)p;
}
static inline void fftw_free(void *p) { free(p); }

namespace hx_fft {

typedef std::complex<double> cd;

/* exp(sign * 2 pi i * k / n), with k reduced to [0, n) and the angle folded into
 * the first octant so every twiddle is computed from a small exact argument. */
static inline cd twiddle(long long k, long long n, int sign) {
    k %= n;
    if (k < 0) k += n;
    /* angle = 2 pi k / n ; use symmetry around multiples of n/8 when exact */
    long long k8 = 8 * k;
    double c, s;
    if (k8 % n == 0) {
        static const double q[8][2] = {{1, 0}, {M_SQRT1_2, M_SQRT1_2}, {0, 1}, {-M_SQRT1_2, M_SQRT1_2},
                                       {-1, 0}, {-M_SQRT1_2, -M_SQRT1_2}, {0, -1}, {M_SQRT1_2, -M_SQRT1_2}};
        int o = (int)(k8 / n);
        c = q[o][0];
        s = q[o][1];
    } else {
        double a = 2.0 * M_PI * (double)k / (double)n;
        if (2 * k > n) a = -2.0 * M_PI * (double)(n - k) / (double)n;
        c = cos(a);
        s = sin(a);
    }
    return cd(c, sign * s);
}

struct Plan1D {
    int n;
    int sign;
    bool pow2;
    std::vector<int> factors;      /* radix sequence (general sizes) */
    std::vector<cd> tw;            /* tw[k] = exp(sign 2 pi i k / n), k in [0,n) */
    mutable std::vector<cd> work;
    /* power-of-two sizes: iterative Stockham, radix 4 then one radix 2 if needed,
       per-stage twiddles stored contiguously */
    std::vector<int> radix;
    std::vector<std::vector<cd>> stw;
    Plan1D(int n_, int sign_) : n(n_), sign(sign_) {
        pow2 = (n & (n - 1)) == 0;
        int m = n;
        while (m % 4 == 0) { factors.push_back(4); m /= 4; }
        while (m % 2 == 0) { factors.push_back(2); m /= 2; }
        for (int p = 3; (long long)p * p <= m; p += 2)
            while (m % p == 0) { factors.push_back(p); m /= p; }
        if (m > 1) factors.push_back(m);
        tw.resize(n);
        for (int k = 0; k < n; k++) tw[k] = twiddle(k, n, sign);
        work.resize(n);
        if (pow2) {
            int Ns = 1;
            while (Ns < n) {
                int R = (n / Ns >= 4) ? 4 : 2;
                radix.push_back(R);
                /* twiddles w_{Ns R}^{r k}, k in [0,Ns), r in [1,R) */
                std::vector<cd> t((size_t)Ns * (R - 1));
                for (int k = 0; k < Ns; k++)
                    for (int r = 1; r < R; r++) t[(size_t)k * (R - 1) + (r - 1)] = tw[(size_t)((long long)r * k * (n / (Ns * R)))];
                stw.push_back(t);
                Ns *= R;
            }
        }
    }
    /* out[k*os] = sum_j in[j*is] w^(jk), length len = product of factors[f..] */
    void rec(const cd *in, long long is, cd *out, int len, size_t f) const {
        if (len == 1) { out[0] = in[0]; return; }
        int p = factors[f];
        int m = len / p;
        for (int r = 0; r < p; r++) rec(in + r * is, is * p, out + (long long)r * m, m, f + 1);
        long long tstride = (long long)n / len;
        cd tmp[64];
        std::vector<cd> big;
        cd *t = tmp;
        if (p > 64) { big.resize(p); t = big.data(); }
        for (int k = 0; k < m; k++) {
            for (int r = 0; r < p; r++) t[r] = out[(long long)r * m + k] * tw[(size_t)((long long)r * k * tstride % n)];
            long long ps = (long long)n / p;
            for (int q = 0; q < p; q++) {
                cd acc = 0.0;
                for (int r = 0; r < p; r++) acc += t[r] * tw[(size_t)(((long long)r * q % p) * ps)];
                work[q] = acc;
            }
            for (int q = 0; q < p; q++) out[k + (long long)q * m] = work[q];
        }
    }
    /* Stockham autosort: X = DFT(x), ping-pong between a and b, result returned */
    cd *stockham(cd *a, cd *b) const {
        int Ns = 1;
        const double sg = (double)sign;
        for (size_t s = 0; s < radix.size(); s++) {
            int R = radix[s];
            int LR = n / R;
            const cd *t = stw[s].data();
            if (R == 4) {
                for (int j = 0; j < LR; j++) {
                    int k = j % Ns;
                    cd v0 = a[j], v1 = a[j + LR] * t[3 * k], v2 = a[j + 2 * LR] * t[3 * k + 1], v3 = a[j + 3 * LR] * t[3 * k + 2];
                    cd a0 = v0 + v2, a1 = v0 - v2, b0 = v1 + v3, b1 = v1 - v3;
                    cd jb1(-sg * b1.imag(), sg * b1.real());
                    int d = (j / Ns) * Ns * 4 + k;
                    b[d] = a0 + b0;
                    b[d + Ns] = a1 + jb1;
                    b[d + 2 * Ns] = a0 - b0;
                    b[d + 3 * Ns] = a1 - jb1;
                }
            } else {
                for (int j = 0; j < LR; j++) {
                    int k = j % Ns;
                    cd v0 = a[j], v1 = a[j + LR] * t[k];
                    int d = (j / Ns) * Ns * 2 + k;
                    b[d] = v0 + v1;
                    b[d + Ns] = v0 - v1;
                }
            }
            std::swap(a, b);
            Ns *= R;
        }
        return a;
    }
    void exec(cd *data, cd *scratch) const {
        if (pow2) {
            cd *r = stockham(data, scratch);
            if (r != data) memcpy((void *)data, (const void *)r, sizeof(cd) * n);
            return;
        }
        rec(data, 1, scratch, n, 0);
        memcpy((void *)data, (const void *)scratch, sizeof(cd) * n);
    }
};

/* Transform all lines of a row-major (n0,n1,n2) array along one axis.  Lines are
 * gathered in blocks of adjacent inner indices so strided axes stay cache friendly. */
static inline void transform_axis(cd *a, const int *nn, int axis, int sign) {
    long long n0 = nn[0], n1 = nn[1], n2 = nn[2];
    long long L = nn[axis];
    long long inner = (axis == 0) ? n1 * n2 : (axis == 1) ? n2 : 1;
    long long outer = (axis == 0) ? 1 : (axis == 1) ? n0 : n0 * n1;
    Plan1D plan((int)L, sign);
    const long long B = (inner >= 16) ? 16 : inner;
    std::vector<cd> line((size_t)L * B), scratch((size_t)L);
    for (long long o = 0; o < outer; o++) {
        cd *base = a + o * L * inner;
        for (long long i0 = 0; i0 < inner; i0 += B) {
            long long nb = (inner - i0 < B) ? inner - i0 : B;
            for (long long j = 0; j < L; j++)
                for (long long b = 0; b < nb; b++) line[(size_t)(b * L + j)] = base[j * inner + i0 + b];
            for (long long b = 0; b < nb; b++) plan.exec(&line[(size_t)(b * L)], scratch.data());
            for (long long j = 0; j < L; j++)
                for (long long b = 0; b < nb; b++) base[j * inner + i0 + b] = line[(size_t)(b * L + j)];
        }
    }
}

}  // namespace hx_fft

static inline fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex *in, fftw_complex *out, int sign,
                                         unsigned flags) {
    (void)flags;
    fftw_plan p = new hx_fftw_plan_s;
    p->n[0] = n0;
    p->n[1] = n1;
    p->n[2] = n2;
    p->in = in;
    p->out = out;
    p->sign = sign;
    return p;
}

static inline void fftw_execute(const fftw_plan p) {
    long long tot = (long long)p->n[0] * p->n[1] * p->n[2];
    if (p->out != p->in) memcpy(p->out, p->in, sizeof(fftw_complex) * tot);
    hx_fft::cd *a = reinterpret_cast<hx_fft::cd *>(p->out);
    for (int ax = 2; ax >= 0; ax--) hx_fft::transform_axis(a, p->n, ax, p->sign);
}

static inline void fftw_destroy_plan(fftw_plan p) { delete p; }

#endif
