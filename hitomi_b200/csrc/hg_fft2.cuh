// hg_fft2.cuh -- register-resident two-level line FFTs for lengths L = R1 * R2 <= 1024.
//
// A line of L points is handled by R2 threads that each hold R1 values (R1 = Q R2, Q = 1, 2
// or 3; L = 192 is 24 x 8 with a prime-factor 24-point register DFT):
//   step A  thread t loads x[R2 n1 + t], n1 < R1, does a DFT of size R1 in registers and
//           multiplies by the twiddle w_L^(t k1);
//   one exchange through shared memory (conflict-free layouts below);
//   step B  thread t takes k1 in {t + d R2, d < Q}, does a DFT of size R2
//           over n2 and ends up holding X[k1 + R1 k2].
// The positions a thread holds after step B are {t + R2 m, m < R1}: exactly its step-A
// input set.  So an inverse transform can be followed by a pointwise product and a
// forward transform without any data movement in between (k_chain_x_reg).
//
// Global <-> register traffic is direct and coalesced: for a tile of B columns of a
// strided axis ("COLS") thread = t B + b, so a warp reads 32 consecutive columns of one
// row; for B contiguous lines ("ROWS") thread = b R2 + t, so a warp reads R2-element runs.
// Shared memory is touched twice per element per transform (vs twice per radix pass).
#pragma once

#include "hg_common.cuh"
#include "hg_fft.cuh"
#include "hg_chain.cuh"

namespace hg {
// one copy per translation unit: each .cu file names its own HG_TU_NS, so the kernels and
// helpers of this header never collide at link time
inline namespace HG_TU_NS {

// exp(-2 pi i k / 32), k = 0..31 (correctly rounded doubles), as compile-time constants
__host__ __device__ constexpr double tw32_re(int k) {
    switch (k) {
        case 0: return 1.0;
        case 1: return 0.9807852804032304;
        case 2: return 0.9238795325112867;
        case 3: return 0.8314696123025452;
        case 4: return 0.7071067811865476;
        case 5: return 0.5555702330196022;
        case 6: return 0.3826834323650898;
        case 7: return 0.19509032201612828;
        case 8: return 0.0;
        case 9: return -0.19509032201612828;
        case 10: return -0.3826834323650898;
        case 11: return -0.5555702330196022;
        case 12: return -0.7071067811865476;
        case 13: return -0.8314696123025452;
        case 14: return -0.9238795325112867;
        case 15: return -0.9807852804032304;
        case 16: return -1.0;
        case 17: return -0.9807852804032304;
        case 18: return -0.9238795325112867;
        case 19: return -0.8314696123025452;
        case 20: return -0.7071067811865476;
        case 21: return -0.5555702330196022;
        case 22: return -0.3826834323650898;
        case 23: return -0.19509032201612828;
        case 24: return 0.0;
        case 25: return 0.19509032201612828;
        case 26: return 0.3826834323650898;
        case 27: return 0.5555702330196022;
        case 28: return 0.7071067811865476;
        case 29: return 0.8314696123025452;
        case 30: return 0.9238795325112867;
        case 31: return 0.9807852804032304;
        default: return 0.0;
    }
}
__host__ __device__ constexpr double tw32_im(int k) {
    switch (k) {
        case 0: return 0.0;
        case 1: return -0.19509032201612828;
        case 2: return -0.3826834323650898;
        case 3: return -0.5555702330196022;
        case 4: return -0.7071067811865476;
        case 5: return -0.8314696123025452;
        case 6: return -0.9238795325112867;
        case 7: return -0.9807852804032304;
        case 8: return -1.0;
        case 9: return -0.9807852804032304;
        case 10: return -0.9238795325112867;
        case 11: return -0.8314696123025452;
        case 12: return -0.7071067811865476;
        case 13: return -0.5555702330196022;
        case 14: return -0.3826834323650898;
        case 15: return -0.19509032201612828;
        case 16: return 0.0;
        case 17: return 0.19509032201612828;
        case 18: return 0.3826834323650898;
        case 19: return 0.5555702330196022;
        case 20: return 0.7071067811865476;
        case 21: return 0.8314696123025452;
        case 22: return 0.9238795325112867;
        case 23: return 0.9807852804032304;
        case 24: return 1.0;
        case 25: return 0.9807852804032304;
        case 26: return 0.9238795325112867;
        case 27: return 0.8314696123025452;
        case 28: return 0.7071067811865476;
        case 29: return 0.5555702330196022;
        case 30: return 0.3826834323650898;
        case 31: return 0.19509032201612828;
        default: return 0.0;
    }
}

__host__ __device__ constexpr int ilog2c(int v) { return v <= 1 ? 0 : 1 + ilog2c(v >> 1); }
__host__ __device__ constexpr int brevc(int i, int bits) { return bits == 0 ? 0 : ((i & 1) << (bits - 1)) | brevc(i >> 1, bits - 1); }

// v * exp(DIR 2 pi i K / 32)
template <typename T, int DIR, int K>
__device__ __forceinline__ cplx<T> tw32_mul(cplx<T> v) {
    constexpr T c = (T)tw32_re(K), s = (T)tw32_im(K);  // exp(-2 pi i K/32)
    if constexpr (DIR < 0) return mk<T>(v.x * c - v.y * s, v.x * s + v.y * c);
    else return mk<T>(v.x * c + v.y * s, v.y * c - v.x * s);
}

template <typename T, int R, int I>
__device__ __forceinline__ void brev_swaps(cplx<T> *v) {
    if constexpr (I < R) {
        constexpr int J = brevc(I, ilog2c(R));
        if constexpr (J > I) {
            cplx<T> t = v[I];
            v[I] = v[J];
            v[J] = t;
        }
        brev_swaps<T, R, I + 1>(v);
    }
}

template <typename T, int R, int DIR, int LEN, int J>
__device__ __forceinline__ void bfly_stage(cplx<T> *v) {
    if constexpr (J < LEN / 2) {
        constexpr int K = J * (32 / LEN);  // w_LEN^J = w_32^K
#pragma unroll
        for (int i = 0; i < R; i += LEN) {
            cplx<T> u = v[i + J];
            cplx<T> t = v[i + J + LEN / 2];
            if constexpr (K == 8) t = mul_i<T, DIR>(t);
            else if constexpr (K != 0) t = tw32_mul<T, DIR, K>(t);
            v[i + J] = u + t;
            v[i + J + LEN / 2] = u - t;
        }
        bfly_stage<T, R, DIR, LEN, J + 1>(v);
    }
}

template <typename T, int R, int DIR, int LEN>
__device__ __forceinline__ void bfly_stages(cplx<T> *v) {
    if constexpr (LEN <= R) {
        bfly_stage<T, R, DIR, LEN, 0>(v);
        bfly_stages<T, R, DIR, LEN * 2>(v);
    }
}

// 3-point DFT in place, X[q] = sum_r v[r] exp(DIR 2 pi i r q / 3):
// X0 = a + b + c, X1,2 = a - (b + c)/2 +- DIR i (sqrt(3)/2) (b - c).
template <typename T, int DIR>
__device__ __forceinline__ void dft3(cplx<T> &a, cplx<T> &b, cplx<T> &c) {
    constexpr T h = (T)0.8660254037844386;  // sqrt(3) / 2
    const cplx<T> sum = b + c, dif = b - c;
    const cplx<T> m = mk<T>(a.x - (T)0.5 * sum.x, a.y - (T)0.5 * sum.y);
    const cplx<T> u = (DIR > 0) ? mk<T>(-h * dif.y, h * dif.x) : mk<T>(h * dif.y, -h * dif.x);
    a = a + sum;
    b = m + u;
    c = m - u;
}

template <typename T, int R, int DIR>
__device__ __forceinline__ void dft_reg(cplx<T> *v);

// 24-point DFT as 8 x 3 with the prime-factor (Good-Thomas) maps: input n = (3 n1 + 8 n2)
// mod 24, output k = (9 k1 + 16 k2) mod 24, so that W24^(n k) = W8^(n1 k1) W3^(n2 k2) and
// no twiddles sit between the 3-point and the 8-point transforms.
template <typename T, int DIR>
__device__ __forceinline__ void dft24(cplx<T> *v) {
    cplx<T> a[3][8];
#pragma unroll
    for (int n1 = 0; n1 < 8; n1++)
#pragma unroll
        for (int n2 = 0; n2 < 3; n2++) a[n2][n1] = v[(3 * n1 + 8 * n2) % 24];
#pragma unroll
    for (int n1 = 0; n1 < 8; n1++) dft3<T, DIR>(a[0][n1], a[1][n1], a[2][n1]);
#pragma unroll
    for (int k2 = 0; k2 < 3; k2++) dft_reg<T, 8, DIR>(a[k2]);
#pragma unroll
    for (int k1 = 0; k1 < 8; k1++)
#pragma unroll
        for (int k2 = 0; k2 < 3; k2++) v[(9 * k1 + 16 * k2) % 24] = a[k2][k1];
}

// In-register DFT of size R, natural-order output, X[q] = sum_r v[r] exp(DIR 2 pi i r q / R):
// for a power of two <= 32, bit-reversal permutation then radix-2 decimation-in-time
// stages; R = 24 by the prime-factor form.  Every index and twiddle is a compile-time constant.
template <typename T, int R, int DIR>
__device__ __forceinline__ void dft_reg(cplx<T> *v) {
    if constexpr (R == 24) {
        dft24<T, DIR>(v);
    } else {
        brev_swaps<T, R, 0>(v);
        bfly_stages<T, R, DIR, 2>(v);
    }
}

template <int L>
struct Split;
template <> struct Split<8> { static constexpr int R1 = 4, R2 = 2; };
template <> struct Split<16> { static constexpr int R1 = 4, R2 = 4; };
template <> struct Split<32> { static constexpr int R1 = 8, R2 = 4; };
template <> struct Split<64> { static constexpr int R1 = 8, R2 = 8; };
template <> struct Split<128> { static constexpr int R1 = 16, R2 = 8; };
template <> struct Split<192> { static constexpr int R1 = 24, R2 = 8; };
template <> struct Split<256> { static constexpr int R1 = 16, R2 = 16; };
template <> struct Split<512> { static constexpr int R1 = 32, R2 = 16; };
template <> struct Split<1024> { static constexpr int R1 = 32, R2 = 32; };

// Shared-memory exchange buffers for B lines.  COLS: S[(k1 R2 + t) B + b].
// ROWS: S[b LP + k1 (R2 + 1) + t] with LP = R1 (R2 + 1).
template <int L, bool COLS, int B>
struct XchgLayout {
    static constexpr int R1 = Split<L>::R1, R2 = Split<L>::R2;
    static constexpr int LP = R1 * (R2 + 1);
    static constexpr int ELEMS = COLS ? L * B : LP * B;
    __device__ static __forceinline__ int at(int b, int k1, int t) {
        return COLS ? (k1 * R2 + t) * B + b : b * LP + k1 * (R2 + 1) + t;
    }
};

// One full line transform on values already in registers (v[n1] = x[R2 n1 + t]).
// On return v holds X at positions t + R2 m in the order of `pos_of_reg`.
template <typename T, int L, int DIR, bool COLS, int B>
__device__ __forceinline__ void line_fft2(cplx<T> *v, cplx<T> *S, int t, int b, const cplx<T> *__restrict__ tw) {
    using X = XchgLayout<L, COLS, B>;
    constexpr int R1 = X::R1, R2 = X::R2;
    dft_reg<T, R1, DIR>(v);
#pragma unroll
    for (int k1 = 1; k1 < R1; k1++) v[k1] = mul_tw<T, DIR>(v[k1], tw[t * k1]);  // t k1 < R1 R2 = L
#pragma unroll
    for (int k1 = 0; k1 < R1; k1++) S[X::at(b, k1, t)] = v[k1];
    __syncthreads();
#pragma unroll
    for (int d = 0; d < R1 / R2; d++) {
        const int k1 = t + d * R2;
#pragma unroll
        for (int n2 = 0; n2 < R2; n2++) v[d * R2 + n2] = S[X::at(b, k1, n2)];
    }
    __syncthreads();
#pragma unroll
    for (int d = 0; d < R1 / R2; d++) dft_reg<T, R2, DIR>(&v[d * R2]);
}

// line_fft2 (column layout) with the exchange in rounds of RS values of k1 through a buffer
// of RS R2 B elements (RS = R2: a third of L B at 192 = 24 x 8; RS = R2 / 2: a sixth).  The
// k1 of step B's block d are [d R2, (d+1) R2), which thread t reads at k1 = t + d R2; a block
// moves in R2 / RS rounds, each thread keeping what it reads in u until the block's last
// round has written its values out.  Same values, same order of operations.
template <typename T, int L, int DIR, int B, int RS>
__device__ __forceinline__ void line_fft2_q(cplx<T> *v, cplx<T> *S, int t, int b, const cplx<T> *__restrict__ tw) {
    constexpr int R1 = Split<L>::R1, R2 = Split<L>::R2;
    static_assert(R2 % RS == 0, "rounds of a whole number per block");
    dft_reg<T, R1, DIR>(v);
#pragma unroll
    for (int k1 = 1; k1 < R1; k1++) v[k1] = mul_tw<T, DIR>(v[k1], tw[t * k1]);  // t k1 < R1 R2 = L
    if constexpr (RS == R2) {  // one round per block: its reads land in registers already written out
#pragma unroll
        for (int d = 0; d < R1 / R2; d++) {
#pragma unroll
            for (int q = 0; q < R2; q++) S[(q * R2 + t) * B + b] = v[d * R2 + q];
            __syncthreads();
#pragma unroll
            for (int n2 = 0; n2 < R2; n2++) v[d * R2 + n2] = S[(t * R2 + n2) * B + b];
            __syncthreads();
        }
#pragma unroll
        for (int d = 0; d < R1 / R2; d++) dft_reg<T, R2, DIR>(&v[d * R2]);
        return;
    }
#pragma unroll
    for (int d = 0; d < R1 / R2; d++) {
        cplx<T> u[R2];
#pragma unroll
        for (int h = 0; h < R2 / RS; h++) {
#pragma unroll
            for (int q = 0; q < RS; q++) S[(q * R2 + t) * B + b] = v[d * R2 + h * RS + q];
            __syncthreads();
            if (t >= h * RS && t < (h + 1) * RS) {
#pragma unroll
                for (int n2 = 0; n2 < R2; n2++) u[n2] = S[((t - h * RS) * R2 + n2) * B + b];
            }
            __syncthreads();
        }
#pragma unroll
        for (int n2 = 0; n2 < R2; n2++) v[d * R2 + n2] = u[n2];
    }
#pragma unroll
    for (int d = 0; d < R1 / R2; d++) dft_reg<T, R2, DIR>(&v[d * R2]);
}

// Register slot r = d R2 + k2 holds position k1 + R1 k2 with k1 = t + d R2.
template <int L>
__device__ __forceinline__ int pos_of_reg(int t, int r) {
    constexpr int R1 = Split<L>::R1, R2 = Split<L>::R2;
    const int d = r / R2, k2 = r % R2;
    return t + d * R2 + R1 * k2;
}
// Step-A register n1 holds position R2 n1 + t.  The register holding a given step-A index
// n1 after a step B: n1 = d + (R1/R2) k2 -> r = d R2 + k2.
template <int L>
__device__ __forceinline__ int reg_of_n1(int n1) {
    constexpr int R1 = Split<L>::R1, R2 = Split<L>::R2;
    constexpr int Q = R1 / R2;
    const int d = n1 % Q, k2 = n1 / Q;
    return d * R2 + k2;
}

template <typename T, int L, bool COLS>
struct Fft2Cfg {
    static constexpr int R2 = Split<L>::R2;
    // lines per CTA: columns (strided axes) or whole lines (contiguous axis); lengths
    // >= 512 hold 32 values per thread, so their CTAs are capped at 256 threads.  FP64 rows
    // shorter than 512 take half as many lines (128 threads): a 192-point FP64 row tile of 32
    // lines needs 114 KB of shared memory, so one CTA (8 warps) filled an SM; 16 lines fit
    // three (chain z passes 1.01 -> 0.85 ms per mock).  At 512 points, halved row tiles
    // together with 4-column pipelined tiles made the density transform slower (1.85 ->
    // 2.27 ms), so those keep 256 threads.
    static constexpr int RB = (sizeof(T) == 8 && L < 512 ? 128 : 256) / R2;
    static constexpr int B = COLS ? ((L >= 512) ? 256 / R2 : ((sizeof(T) == 4) ? 32 : 16))
                                  : (RB > 64 ? 64 : (RB < 1 ? 1 : RB));
    static constexpr int NT = R2 * B;
};

// Generic pass: same tile geometry and loader/storer functors as k_fft_pass.
template <typename T, int L, int DIR, bool COLS, class LD, class ST>
__global__ void __launch_bounds__(Fft2Cfg<T, L, COLS>::NT)
    k_fft2_pass(LD ld, ST st, PassGeom g, const cplx<T> *__restrict__ tw) {
    using CF = Fft2Cfg<T, L, COLS>;
    using X = XchgLayout<L, COLS, CF::B>;
    constexpr int R1 = X::R1, R2 = X::R2, B = CF::B;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx<T> *S = reinterpret_cast<cplx<T> *>(smem_raw);
    int t, b;
    if (COLS) {
        t = threadIdx.x / B;
        b = threadIdx.x % B;
    } else {
        b = threadIdx.x / R2;
        t = threadIdx.x % R2;
    }
    long long o, i;
    bool ok;
    if (COLS) {
        long long tiles_per_outer = (g.n_inner + B - 1) / B;
        o = (long long)blockIdx.x / tiles_per_outer;
        i = ((long long)blockIdx.x - o * tiles_per_outer) * B + b;
        ok = i < g.n_inner;
    } else {
        o = (long long)blockIdx.x * B + b;
        i = 0;
        ok = o < g.n_outer;
    }
    cplx<T> *Tw = S + X::ELEMS;  // twiddles, staged for the whole CTA (barrier below)
    for (int e = threadIdx.x; e < L; e += CF::NT) Tw[e] = tw[e];
    cplx<T> v[R1];
#pragma unroll
    for (int n1 = 0; n1 < R1; n1++) v[n1] = ok ? ld(o, R2 * n1 + t, i) : mk<T>(0, 0);
    __syncthreads();
    line_fft2<T, L, DIR, COLS, B>(v, S, t, b, Tw);
    if (ok) {
#pragma unroll
        for (int r = 0; r < R1; r++) st(o, pos_of_reg<L>(t, r), i, v[r]);
    }
}

template <typename T, int L, bool COLS>
inline size_t fft2_smem() {
    using CF = Fft2Cfg<T, L, COLS>;
    return ((size_t)XchgLayout<L, COLS, CF::B>::ELEMS + L) * sizeof(cplx<T>);  // exchange buffer, twiddles
}

// Strided passes over arrays of rows (PipeArr, PipeRowsCompactL), software-pipelined: a persistent CTA walks its
// tiles (L rows x PB columns) and, while it transforms one tile, the next one streams into the
// other half of a double buffer with cp.async (no registers held, no wait until the data is
// needed).  The tile's buffer then serves as the transform's exchange buffer.  Without this
// the pass is latency-bound: a CTA's loads are all issued at its start and nothing is in
// flight while it computes and stores.
template <typename T, int L>
struct PipeCfg {
    static constexpr int R2 = Split<L>::R2;
    // columns per tile: the double buffer of FP64 1024-point tiles takes 4 columns to stay
    // within the 227 KB a CTA may hold (at 512 points 4 columns, three CTAs per SM instead of
    // one, measured slower: the FP64 density transform 1.83 -> 2.45 ms)
    // FP32 lines of 256 and 512 points take 16 columns (128-byte row segments; the FP32
    // correlation-field passes at 512 points 0.34 -> 0.25 ms each against 8 columns).  (A
    // 192-point FP64 variant with 16 threads and 12 values per thread per line, twice the
    // warps per SM, was slower on the chain's y passes: 2.26 -> 2.34 ms per mock.)
    static constexpr int B = (L >= 1024 && sizeof(T) == 8) ? 4
                           : (L >= 256 && sizeof(T) == 8) ? 8
                           : (L >= 1024) ? 8 : 16;
    static constexpr int NT = R2 * B;
    // double buffer, then the L twiddles (staged once per persistent CTA)
    static constexpr size_t smem() { return (2 * (size_t)L * B + L) * sizeof(cplx<T>); }
};

// Row sources of the pipelined pass: line(o) once per tile, then row(line, l) = the start of
// row l of that line (inner elements contiguous), or nullptr for a row that is zero.
template <typename T>
struct PipeArr {  // [o][L][inner] (LdArr)
    const cplx<T> *p;
    long long L, inner;
    using Line = const cplx<T> *;
    __device__ __forceinline__ Line line(long long o) const { return p + o * L * inner; }
    __device__ __forceinline__ const cplx<T> *row(Line b, int l) const { return b + (long long)l * inner; }
};
template <typename T>
struct PipeRowsCompactL {  // LdRowsCompactL: compact rows c in cyr[o] of the line o = lines[q]
    const cplx<T> *p;
    int K, M, s;
    long long inner;
    const int *lines;
    const int2 *cyr;
    struct Line {
        const cplx<T> *b;
        int lo, hi;
    };
    __device__ __forceinline__ Line line(long long q) const {
        const int o = lines[q];
        const int2 r = cyr[o];
        return Line{p + (long long)o * K * inner, r.x, r.y};
    }
    __device__ __forceinline__ const cplx<T> *row(const Line &ln, int l) const {
        const int n = (l < M / 2) ? l : l - M;
        const int c = n + s;
        return (c >= ln.lo && c <= ln.hi) ? ln.b + (long long)c * inner : nullptr;
    }
};

__device__ __forceinline__ void cp_async_elem(void *sdst, const void *gsrc, int bytes, bool ok) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
    if (bytes == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gsrc), "r"(ok ? 8 : 0));
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gsrc), "r"(ok ? 16 : 0));
}

template <typename T, int L, int DIR, class SRC, class ST>
__global__ void __launch_bounds__(PipeCfg<T, L>::NT)
    k_fft2_pass_pipe(SRC src, ST st, PassGeom g, const cplx<T> *__restrict__ tw) {
    using PC = PipeCfg<T, L>;
    using X = XchgLayout<L, true, PC::B>;
    constexpr int R1 = X::R1, R2 = X::R2, B = PC::B, NT = PC::NT;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx<T> *buf = reinterpret_cast<cplx<T> *>(smem_raw);  // [2][L][B]
    cplx<T> *Tw = buf + 2 * L * B;                          // [L]
    for (int e = threadIdx.x; e < L; e += NT) Tw[e] = tw[e];  // first read after the loop's first barrier
    const int t = threadIdx.x / B, b = threadIdx.x % B;
    const long long tpo = (g.n_inner + B - 1) / B;
    const long long ntiles = g.n_outer * tpo;
    // element e of a tile (row e / B, column e % B), NT at a time
    // rows the source does not hold (pruned rows) are zero-filled: cp.async with no source bytes
    auto prefetch = [&](long long tile, cplx<T> *dst) {
        const long long o = tile / tpo, i0 = (tile - o * tpo) * B;
        const typename SRC::Line ln = src.line(o);
#pragma unroll 4
        for (int e = threadIdx.x; e < L * B; e += NT) {
            const int l = e / B, c = e - l * B;
            const cplx<T> *row = src.row(ln, l);
            const bool ok = (i0 + c) < g.n_inner && row != nullptr;
            cp_async_elem(dst + e, ok ? row + i0 + c : src.p, (int)sizeof(cplx<T>), ok);
        }
        asm volatile("cp.async.commit_group;\n" ::);
    };
    int cur = 0;
    long long tile = blockIdx.x;
    if (tile < ntiles) prefetch(tile, buf);
    for (; tile < ntiles; tile += gridDim.x) {
        const long long next = tile + gridDim.x;
        if (next < ntiles) prefetch(next, buf + (size_t)(cur ^ 1) * L * B);
        else asm volatile("cp.async.commit_group;\n" ::);  // keep one group per iteration
        asm volatile("cp.async.wait_group 1;\n" ::);
        __syncthreads();
        cplx<T> *S = buf + (size_t)cur * L * B;
        cplx<T> v[R1];
#pragma unroll
        for (int n1 = 0; n1 < R1; n1++) v[n1] = S[(R2 * n1 + t) * B + b];
        __syncthreads();  // every value is in registers: S becomes the exchange buffer
        line_fft2<T, L, DIR, true, B>(v, S, t, b, Tw);
        const long long o = tile / tpo, i = (tile - o * tpo) * B + b;
        if (i < g.n_inner) {
#pragma unroll
            for (int r = 0; r < R1; r++) st(o, pos_of_reg<L>(t, r), i, v[r]);
        }
        __syncthreads();  // S is the target of the prefetch two tiles on
        cur ^= 1;
    }
    asm volatile("cp.async.wait_group 0;\n" ::);
}

template <typename T, int L, int DIR, class SRC, class ST>
inline cudaError_t launch_fft2_pipe(SRC src, ST st, PassGeom g, const cplx<T> *tw, cudaStream_t stream) {
    using PC = PipeCfg<T, L>;
    auto kern = k_fft2_pass_pipe<T, L, DIR, SRC, ST>;
    const size_t smem = PC::smem();
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, PC::NT, smem);
    if (e != cudaSuccess) return e;
    const long long ntiles = g.n_outer * ((g.n_inner + PC::B - 1) / PC::B);
    const long long grid = std::min<long long>(ntiles, 148LL * std::max(per_sm, 1));
    if (grid <= 0) return cudaSuccess;
    kern<<<(unsigned)grid, PC::NT, smem, stream>>>(src, st, g, tw);
    return cudaGetLastError();
}

// Real rows -> half spectra, two rows per complex transform: line b carries rows 2o (real
// part) and 2o + 1 (imaginary part) of (mesh - sub) scl; after the transform
// A(k) = (Z(k) + conj Z(-k)) / 2 and B(k) = (Z(k) - conj Z(-k)) / (2 i) are the two rows'
// spectra, of which k = 0 .. hz - 1 are stored ([row][hz]).  Half the transform work of a
// complex pass over real input.
template <typename T, int L, int DIR>
__global__ void __launch_bounds__(Fft2Cfg<T, L, false>::NT)
    k_fft2_r2c_pair(const T *__restrict__ mesh, T sub, T scl, cplx<T> *__restrict__ H, long long npair, int hz,
                    const cplx<T> *__restrict__ tw) {
    using CF = Fft2Cfg<T, L, false>;
    using X = XchgLayout<L, false, CF::B>;
    constexpr int R1 = X::R1, R2 = X::R2, B = CF::B, LP = L + 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx<T> *S = reinterpret_cast<cplx<T> *>(smem_raw);
    const int b = threadIdx.x / R2, t = threadIdx.x % R2;
    const long long o = (long long)blockIdx.x * B + b;
    const bool ok = o < npair;
    const T *ra = mesh + 2 * o * L, *rb = ra + L;
    constexpr int ELEMS = (X::ELEMS > B * LP) ? X::ELEMS : B * LP;
    cplx<T> *Tw = S + ELEMS;  // twiddles, staged for the whole CTA (barrier below)
    for (int e = threadIdx.x; e < L; e += CF::NT) Tw[e] = tw[e];
    cplx<T> v[R1];
#pragma unroll
    for (int n1 = 0; n1 < R1; n1++) {
        const int p = R2 * n1 + t;
        v[n1] = ok ? mk<T>((ra[p] - sub) * scl, (rb[p] - sub) * scl) : mk<T>(0, 0);
    }
    __syncthreads();
    line_fft2<T, L, DIR, false, B>(v, S, t, b, Tw);  // ends with S free
#pragma unroll
    for (int r = 0; r < R1; r++) S[b * LP + pos_of_reg<L>(t, r)] = v[r];
    __syncthreads();
    if (ok) {
        cplx<T> *ha = H + 2 * o * hz, *hb = ha + hz;
        for (int k = t; k < hz; k += R2) {
            const cplx<T> z = S[b * LP + k], zm = S[b * LP + ((L - k) & (L - 1))];
            ha[k] = mk<T>((T)0.5 * (z.x + zm.x), (T)0.5 * (z.y - zm.y));
            hb[k] = mk<T>((T)0.5 * (z.y + zm.y), (T)0.5 * (zm.x - z.x));
        }
    }
}

template <typename T, int L, int DIR>
inline cudaError_t launch_r2c_pair_L(const T *mesh, T sub, T scl, cplx<T> *H, long long nrows, int hz,
                                     const cplx<T> *tw, cudaStream_t stream) {
    using CF = Fft2Cfg<T, L, false>;
    using X = XchgLayout<L, false, CF::B>;
    const size_t elems = std::max<size_t>((size_t)X::ELEMS, (size_t)CF::B * (L + 1));
    const size_t smem = (elems + L) * sizeof(cplx<T>);  // exchange / row buffer, twiddles
    auto kern = k_fft2_r2c_pair<T, L, DIR>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const long long npair = nrows / 2;
    const long long blocks = (npair + CF::B - 1) / CF::B;
    if (blocks <= 0) return cudaSuccess;
    kern<<<(unsigned)blocks, CF::NT, smem, stream>>>(mesh, sub, scl, H, npair, hz, tw);
    return cudaGetLastError();
}

// false when the length has no paired kernel (the caller then runs the plain pass)
template <typename T, int DIR>
inline bool launch_r2c_pair(int L, const T *mesh, T sub, T scl, cplx<T> *H, long long nrows, int hz,
                            const cplx<T> *tw, cudaStream_t stream, cudaError_t &err) {
    if (nrows % 2) return false;
    switch (L) {
        case 8: err = launch_r2c_pair_L<T, 8, DIR>(mesh, sub, scl, H, nrows, hz, tw, stream); return true;
        case 16: err = launch_r2c_pair_L<T, 16, DIR>(mesh, sub, scl, H, nrows, hz, tw, stream); return true;
        case 32: err = launch_r2c_pair_L<T, 32, DIR>(mesh, sub, scl, H, nrows, hz, tw, stream); return true;
        case 64: err = launch_r2c_pair_L<T, 64, DIR>(mesh, sub, scl, H, nrows, hz, tw, stream); return true;
        case 128: err = launch_r2c_pair_L<T, 128, DIR>(mesh, sub, scl, H, nrows, hz, tw, stream); return true;
        case 256: err = launch_r2c_pair_L<T, 256, DIR>(mesh, sub, scl, H, nrows, hz, tw, stream); return true;
        case 512: err = launch_r2c_pair_L<T, 512, DIR>(mesh, sub, scl, H, nrows, hz, tw, stream); return true;
        case 1024: err = launch_r2c_pair_L<T, 1024, DIR>(mesh, sub, scl, H, nrows, hz, tw, stream); return true;
        default: return false;
    }
}

template <class LD>
struct IsLdArr : std::false_type {};
template <typename U>
struct IsLdArr<LdArr<U>> : std::true_type {};

template <typename T, int L, int DIR, class LD, class ST>
inline cudaError_t launch_fft2_L(LD ld, ST st, PassGeom g, const cplx<T> *tw, cudaStream_t stream) {
    if constexpr (IsLdArr<LD>::value) {
        // plain strided source: the pipelined pass (LdArr's inner stride is the pass's own)
        if (g.n_inner > 1 && ld.inner == g.n_inner && ld.L == L)
            return launch_fft2_pipe<T, L, DIR>(PipeArr<T>{ld.p, ld.L, ld.inner}, st, g, tw, stream);
    }
    if constexpr (std::is_same<LD, LdRowsCompactL<T>>::value) {
        // the chain's pruned inverse y pass: compact rows, zero outside the shell's extent
        if (g.n_inner > 1 && ld.inner == g.n_inner && ld.M == L)
            return launch_fft2_pipe<T, L, DIR>(PipeRowsCompactL<T>{ld.p, ld.K, ld.M, ld.s, ld.inner, ld.lines, ld.cyr},
                                               st, g, tw, stream);
    }
    if (g.n_inner == 1) {
        using CF = Fft2Cfg<T, L, false>;
        size_t smem = fft2_smem<T, L, false>();
        auto kern = k_fft2_pass<T, L, DIR, false, LD, ST>;
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        long long tiles = (g.n_outer + CF::B - 1) / CF::B;
        if (tiles <= 0) return cudaSuccess;
        kern<<<(unsigned)tiles, CF::NT, smem, stream>>>(ld, st, g, tw);
    } else {
        using CF = Fft2Cfg<T, L, true>;
        size_t smem = fft2_smem<T, L, true>();
        auto kern = k_fft2_pass<T, L, DIR, true, LD, ST>;
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        long long tiles = g.n_outer * ((g.n_inner + CF::B - 1) / CF::B);
        if (tiles <= 0) return cudaSuccess;
        kern<<<(unsigned)tiles, CF::NT, smem, stream>>>(ld, st, g, tw);
    }
    return cudaGetLastError();
}

// Any supported length: the two-level register FFT for its lengths, the Stockham pass for
// other powers of two, the mixed-radix pass for the rest.
template <typename T, int DIR, class LD, class ST>
inline cudaError_t launch_pass_any(int L, LD ld, ST st, PassGeom g, const cplx<T> *tw, cudaStream_t stream) {
    switch (L) {
        case 8: return launch_fft2_L<T, 8, DIR>(ld, st, g, tw, stream);
        case 16: return launch_fft2_L<T, 16, DIR>(ld, st, g, tw, stream);
        case 32: return launch_fft2_L<T, 32, DIR>(ld, st, g, tw, stream);
        case 64: return launch_fft2_L<T, 64, DIR>(ld, st, g, tw, stream);
        case 128: return launch_fft2_L<T, 128, DIR>(ld, st, g, tw, stream);
        case 192: return launch_fft2_L<T, 192, DIR>(ld, st, g, tw, stream);
        case 256: return launch_fft2_L<T, 256, DIR>(ld, st, g, tw, stream);
        case 512: return launch_fft2_L<T, 512, DIR>(ld, st, g, tw, stream);
        case 1024: return launch_fft2_L<T, 1024, DIR>(ld, st, g, tw, stream);
        default:
            if (fft_supported_length(L)) return launch_fft_pass<T, DIR>(L, ld, st, g, tw, stream);
            return launch_fft_mixed<T, DIR>(L, ld, st, g, tw, stream);
    }
}

// The chain kernel's launch shape (a tunable variant): B columns per CTA; GS: the CTA's G
// tile (L x B) staged once in shared memory for all shells, else each thread reads its G
// values from global memory (L2-resident) per shell; PF: the next shell's input rows stream
// into shared memory by cp.async while the current one is transformed, else each shell's
// rows are loaded into registers when it starts.  Less shared memory per CTA means more
// CTAs per SM; which is faster depends on the precision and the line length, so the engine
// times the variants once per geometry and keeps the fastest.
// MINB: CTAs per SM the compiler must fit (the register cap: 65536 / (MINB x threads);
// 0 keeps the default, 2 CTAs for FP32 and 1 for FP64).  The FP64 transform holds 24 complex
// values per thread and is latency-bound at the two CTAs of 128 threads its 255 registers
// allow; the capped variants trade spills for more warps in flight.
// v12: the 192-point kernel with 12 values per thread (k_chain_x_192); xr: the exchange in
// rounds (line_fft2_q), which lets a fourth (xr 1) or, with registers capped for five CTAs,
// a fifth (xr 2) staged FP64 CTA fit on an SM.
struct ChainVariant {
    int B;
    bool gs, pf;
    int minb;
    bool v12;
    int xr;  // the exchange in rounds (line_fft2_q): 1 a third of the exchange buffer at 192,
             // 2 a sixth
};
constexpr ChainVariant kChainVariants[] = {
    {16, true, true, 0, false},  {16, false, true, 0, false},  {16, false, false, 0, false},
    {8, true, true, 0, false},   {8, false, false, 0, false},  {16, false, false, 3, false},
    {16, false, false, 4, false}, {8, false, false, 8, false}, {8, false, false, 4, true},
    {16, false, false, 2, true},  {8, true, false, 4, true},   {8, false, false, 3, true},
    {8, false, true, 0, false},   {8, true, true, 0, false, 1}, {8, true, true, 5, false, 2}};
constexpr int kNumChainVariants = 15;

template <typename T, int L, int B, bool GS, bool PF, int XR = 0>
struct ChainCfg {
    static constexpr int R2 = Split<L>::R2;
    static constexpr int NT = R2 * B;
    // exchange buffer (XR: one round's RS R2 B, RS = R2 / XR), G tile (GS), the next shell's
    // K kept rows (PF), the L twiddles
    static constexpr int RS = XR ? R2 / XR : R2;
    static constexpr int XE = XR ? RS * R2 * B : XchgLayout<L, true, B>::ELEMS;
    static size_t smem(int K) {
        return sizeof(cplx<T>) * ((size_t)XE + (GS ? (size_t)L * B : 0) + (PF ? (size_t)K * B : 0) + (size_t)L);
    }
};

// Fused chain x-pass with the register FFT: T2 layout [j][cx][y][z] (rows of `plane`
// columns), G [x][y][z].  Per shell j: load the K kept rows, inverse FFT, * G, forward FFT,
// store the K kept rows.  The product happens in the positions a thread holds after the
// inverse transform, which are its step-A positions of the forward transform.  The twiddle
// table is staged in shared memory once per CTA (the transforms read it on every shell; from
// shared memory those reads wait less than L1 hits do), and the prefetch buffer holds only
// the K kept rows, so that three FP64 CTAs of the staged variants fit on an SM.
template <typename T, int L, int B, bool GS, bool PF, int MINB, int XR = 0>
__global__ void __launch_bounds__(ChainCfg<T, L, B, GS, PF, XR>::NT, MINB ? MINB : ((sizeof(T) == 4) ? 2 : 1))
    k_chain_x_reg(cplx<T> *t2, const cplx<T> *__restrict__ G, int ns, int K, int s, long long plane,
                  const cplx<T> *__restrict__ tw, const int *__restrict__ ext) {
    using CF = ChainCfg<T, L, B, GS, PF, XR>;
    using X = XchgLayout<L, true, B>;
    constexpr int R1 = X::R1, R2 = X::R2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx<T> *S = reinterpret_cast<cplx<T> *>(smem_raw);
    cplx<T> *Gs = S + CF::XE;                // [x][b] (GS)
    cplx<T> *Pb = Gs + (GS ? L * B : 0);     // next shell's K kept rows, [c][b] (PF)
    cplx<T> *Tw = Pb + (PF ? K * B : 0);     // twiddles [L]
    const int t = threadIdx.x / B, b = threadIdx.x % B;
    const long long i = (long long)blockIdx.x * B + b;
    const bool ok = i < plane;
    for (int e = threadIdx.x; e < L; e += CF::NT) Tw[e] = tw[e];
    if constexpr (GS) {
        for (int e = threadIdx.x; e < L * B; e += CF::NT) {
            const int x = e / B, bb = e % B;
            const long long ii = (long long)blockIdx.x * B + bb;
            Gs[e] = (ii < plane) ? G[(long long)x * plane + ii] : mk<T>(0, 0);
        }
    }
    __syncthreads();
    // shell j's input rows |n| <= e_j (the rows the pruned y pass wrote; ext null: all K)
    auto ext_of = [&](int j) {
        const int e = ext ? ext[j] : s;
        return HG_IN_BOUNDS(e <= s, HG_SITE_CHAIN_ROW, e) ? e : s;
    };
    // those rows of shell j into Pb (row c = n + s; columns past the plane zero-filled)
    auto prefetch = [&](int j) {
        const cplx<T> *tj = t2 + (long long)j * K * plane;
        const int e0 = s - ext_of(j), nr = 2 * ext_of(j) + 1;
        for (int e = threadIdx.x; e < nr * B; e += CF::NT) {
            const int c = e0 + e / B, bb = e % B;
            const long long ii = (long long)blockIdx.x * B + bb;
            const bool in = ii < plane;
            cp_async_elem(Pb + c * B + bb, tj + (long long)c * plane + (in ? ii : 0), (int)sizeof(cplx<T>), in);
        }
        asm volatile("cp.async.commit_group;\n" ::);
    };
    auto g_at = [&](int pos) -> cplx<T> {
        if constexpr (GS) return Gs[pos * B + b];
        else return ok ? G[(long long)pos * plane + i] : mk<T>(0, 0);
    };
    if constexpr (PF) {
        if (ns > 0) prefetch(0);
    }
    for (int j = 0; j < ns; j++) {
        cplx<T> *tj = t2 + (long long)j * K * plane;
        const int ej = ext_of(j);
        cplx<T> v[R1];
        if constexpr (PF) {
            asm volatile("cp.async.wait_group 0;\n" ::);
            __syncthreads();
#pragma unroll
            for (int n1 = 0; n1 < R1; n1++) {
                const int x = R2 * n1 + t;
                const int n = (x < L / 2) ? x : x - L;
                v[n1] = (n >= -ej && n <= ej) ? Pb[(n + s) * B + b] : mk<T>(0, 0);
            }
            __syncthreads();  // Pb is read: the next shell streams in while this one is transformed
            if (j + 1 < ns) prefetch(j + 1);
        } else {
#pragma unroll
            for (int n1 = 0; n1 < R1; n1++) {
                const int x = R2 * n1 + t;
                const int n = (x < L / 2) ? x : x - L;
                v[n1] = (ok && n >= -ej && n <= ej) ? tj[(long long)(n + s) * plane + i] : mk<T>(0, 0);
            }
        }
        if constexpr (XR != 0) line_fft2_q<T, L, +1, B, CF::RS>(v, S, t, b, Tw);
        else line_fft2<T, L, +1, true, B>(v, S, t, b, Tw);
        if constexpr (R1 == R2) {
#pragma unroll
            for (int r = 0; r < R1; r++) v[r] = v[r] * g_at(pos_of_reg<L>(t, r));
        } else {
            cplx<T> u[R1];
#pragma unroll
            for (int n1 = 0; n1 < R1; n1++) {
                const int r = reg_of_n1<L>(n1);
                u[n1] = v[r] * g_at(pos_of_reg<L>(t, r));
            }
#pragma unroll
            for (int n1 = 0; n1 < R1; n1++) v[n1] = u[n1];
        }
        if constexpr (XR != 0) line_fft2_q<T, L, -1, B, CF::RS>(v, S, t, b, Tw);
        else line_fft2<T, L, -1, true, B>(v, S, t, b, Tw);
        if (ok) {
#pragma unroll
            for (int r = 0; r < R1; r++) {
                const int p = pos_of_reg<L>(t, r);
                const int n = (p < L / 2) ? p : p - L;
                if (n >= -s && n <= s) tj[(long long)(n + s) * plane + i] = v[r];
            }
        }
    }
}

// ---- 192-point lines with 12 values per thread (16 threads per line): 192 = 12 x 4 x 4.
// The two-level transform above holds 24 complex values per thread for this length; in FP64
// that needs 255 registers and leaves two CTAs of 128 threads per SM, too few warps to hide
// the memory latency.  Here: stage A, thread t takes x[16 n1 + t] (n1 < 12), their 12-point
// DFT (prime-factor 3 x 4: input index (4 na + 3 nb) mod 12, output (4 ka + 9 kb) mod 12,
// no twiddles inside) and multiplies output k1 by W_192^(t k1).  One 16-point DFT over t per
// k1 remains, done as 4 x 4 (t = a + 4 c, k2 = q + 4 r): stage B, per item (k1, a), the
// 4-point DFT over c of S[k1][a + 4c] times W_16^(a q); stage C, per item (k1, q), the
// 4-point DFT over a, giving X[k1 + 12 (q + 4 r)].  Items are 0..47; thread t takes t,
// t + 16 and t + 32 in stages B and C.

template <typename T, int DIR>
__device__ __forceinline__ void dft12(cplx<T> *v) {
    cplx<T> a[3][4];
#pragma unroll
    for (int nb = 0; nb < 4; nb++)
#pragma unroll
        for (int na = 0; na < 3; na++) a[na][nb] = v[(4 * na + 3 * nb) % 12];
#pragma unroll
    for (int nb = 0; nb < 4; nb++) dft3<T, DIR>(a[0][nb], a[1][nb], a[2][nb]);
#pragma unroll
    for (int ka = 0; ka < 3; ka++) dft4<T, DIR>(a[ka][0], a[ka][1], a[ka][2], a[ka][3]);
#pragma unroll
    for (int ka = 0; ka < 3; ka++)
#pragma unroll
        for (int kb = 0; kb < 4; kb++) v[(4 * ka + 9 * kb) % 12] = a[ka][kb];
}

// line position held in register 4 j + r after line_fft192_12
__device__ __forceinline__ int l192_pos(int t, int j, int r) { return ((t >> 2) + 4 * j) + 12 * ((t & 3) + 4 * r); }

// One 192-point transform of B lines; S: [192][B] exchange buffer (column layout).  On entry
// v[n1] = x[16 n1 + t]; on return v[4 j + r] = X[l192_pos(t, j, r)], S free for reuse.
template <typename T, int DIR, int B>
__device__ __forceinline__ void line_fft192_12(cplx<T> *v, cplx<T> *S, int t, int b, const cplx<T> *__restrict__ tw) {
    dft12<T, DIR>(v);
#pragma unroll
    for (int k1 = 1; k1 < 12; k1++) v[k1] = mul_tw<T, DIR>(v[k1], tw[t * k1]);  // W_192^(t k1)
#pragma unroll
    for (int k1 = 0; k1 < 12; k1++) S[(k1 * 16 + t) * B + b] = v[k1];
    __syncthreads();
    const int a = t & 3;
#pragma unroll
    for (int j = 0; j < 3; j++) {  // stage B: item (k1, a)
        const int k1 = (t >> 2) + 4 * j;
        cplx<T> u0 = S[(k1 * 16 + a) * B + b], u1 = S[(k1 * 16 + a + 4) * B + b];
        cplx<T> u2 = S[(k1 * 16 + a + 8) * B + b], u3 = S[(k1 * 16 + a + 12) * B + b];
        dft4<T, DIR>(u0, u1, u2, u3);
        v[4 * j] = u0;
        v[4 * j + 1] = mul_tw<T, DIR>(u1, tw[12 * a]);  // W_16^(a q) = W_192^(12 a q)
        v[4 * j + 2] = mul_tw<T, DIR>(u2, tw[24 * a]);
        v[4 * j + 3] = mul_tw<T, DIR>(u3, tw[36 * a]);
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < 3; j++) {
        const int k1 = (t >> 2) + 4 * j;
#pragma unroll
        for (int q = 0; q < 4; q++) S[(k1 * 16 + q * 4 + a) * B + b] = v[4 * j + q];
    }
    __syncthreads();
    const int q = t & 3;
#pragma unroll
    for (int j = 0; j < 3; j++) {  // stage C: item (k1, q)
        const int k1 = (t >> 2) + 4 * j;
        cplx<T> w0 = S[(k1 * 16 + q * 4) * B + b], w1 = S[(k1 * 16 + q * 4 + 1) * B + b];
        cplx<T> w2 = S[(k1 * 16 + q * 4 + 2) * B + b], w3 = S[(k1 * 16 + q * 4 + 3) * B + b];
        dft4<T, DIR>(w0, w1, w2, w3);
        v[4 * j] = w0;
        v[4 * j + 1] = w1;
        v[4 * j + 2] = w2;
        v[4 * j + 3] = w3;
    }
    __syncthreads();
}

// The fused chain x-pass (as k_chain_x_reg) on 192-point lines with line_fft192_12.  The
// inverse transform leaves the positions l192_pos, which are not the forward transform's
// step-A positions, so the product with G goes through the exchange buffer.  MINB CTAs per SM
// set the register cap (4 x 128 threads: 128 registers).
template <typename T, int B, bool GS, int MINB>
__global__ void __launch_bounds__(16 * B, MINB)
    k_chain_x_192(cplx<T> *t2, const cplx<T> *__restrict__ G, int ns, int K, int s, long long plane,
                  const cplx<T> *__restrict__ tw, const int *__restrict__ ext) {
    constexpr int L = 192;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx<T> *S = reinterpret_cast<cplx<T> *>(smem_raw);  // [192][B]
    cplx<T> *Gs = S + L * B;                               // [192][B] (GS)
    cplx<T> *Tw = Gs + (GS ? L * B : 0);                   // twiddles [192]
    const int t = threadIdx.x / B, b = threadIdx.x % B;
    const long long i = (long long)blockIdx.x * B + b;
    const bool ok = i < plane;
    for (int e = threadIdx.x; e < L; e += 16 * B) Tw[e] = tw[e];
    if constexpr (GS) {
        for (int e = threadIdx.x; e < L * B; e += 16 * B) {
            const int x = e / B, bb = e % B;
            const long long ii = (long long)blockIdx.x * B + bb;
            Gs[e] = (ii < plane) ? G[(long long)x * plane + ii] : mk<T>(0, 0);
        }
    }
    __syncthreads();
    for (int j = 0; j < ns; j++) {
        cplx<T> *tj = t2 + (long long)j * K * plane;
        int ej = ext ? ext[j] : s;  // shell j's input rows |n| <= e_j
        if (!HG_IN_BOUNDS(ej <= s, HG_SITE_CHAIN_ROW, ej)) ej = s;
        cplx<T> v[12];
#pragma unroll
        for (int n1 = 0; n1 < 12; n1++) {
            const int x = 16 * n1 + t;
            const int n = (x < L / 2) ? x : x - L;
            v[n1] = (ok && n >= -ej && n <= ej) ? tj[(long long)(n + s) * plane + i] : mk<T>(0, 0);
        }
        line_fft192_12<T, +1, B>(v, S, t, b, Tw);
#pragma unroll
        for (int jj = 0; jj < 3; jj++)
#pragma unroll
            for (int r = 0; r < 4; r++) {
                const int p = l192_pos(t, jj, r);
                cplx<T> gv;
                if constexpr (GS) gv = Gs[p * B + b];
                else gv = ok ? G[(long long)p * plane + i] : mk<T>(0, 0);
                S[p * B + b] = v[4 * jj + r] * gv;
            }
        __syncthreads();
#pragma unroll
        for (int n1 = 0; n1 < 12; n1++) v[n1] = S[(16 * n1 + t) * B + b];
        __syncthreads();
        line_fft192_12<T, -1, B>(v, S, t, b, Tw);
        if (ok) {
#pragma unroll
            for (int jj = 0; jj < 3; jj++)
#pragma unroll
                for (int r = 0; r < 4; r++) {
                    const int p = l192_pos(t, jj, r);
                    const int n = (p < L / 2) ? p : p - L;
                    if (n >= -s && n <= s) tj[(long long)(n + s) * plane + i] = v[4 * jj + r];
                }
        }
    }
}

template <typename T, int B, bool GS, int MINB>
inline cudaError_t launch_chain_x_192(cplx<T> *t2, const cplx<T> *G, int ns, int K, int s, long long plane,
                                      const cplx<T> *tw, const int *ext, cudaStream_t st) {
    const size_t smem = sizeof(cplx<T>) * (192 * B * (GS ? 2 : 1) + 192);
    cudaError_t e = cudaFuncSetAttribute(k_chain_x_192<T, B, GS, MINB>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const unsigned tiles = (unsigned)((plane + B - 1) / B);
    k_chain_x_192<T, B, GS, MINB><<<tiles, 16 * B, smem, st>>>(t2, G, ns, K, s, plane, tw, ext);
    return cudaGetLastError();
}

template <typename T, int L, int B, bool GS, bool PF, int MINB = 0, int XR = 0>
inline cudaError_t launch_chain_x_v(cplx<T> *t2, const cplx<T> *G, int ns, int K, int s, long long plane,
                                    const cplx<T> *tw, const int *ext, cudaStream_t st) {
    using CF = ChainCfg<T, L, B, GS, PF, XR>;
    const size_t smem = CF::smem(K);
    cudaError_t e = cudaFuncSetAttribute(k_chain_x_reg<T, L, B, GS, PF, MINB, XR>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const unsigned tiles = (unsigned)((plane + B - 1) / B);
    k_chain_x_reg<T, L, B, GS, PF, MINB, XR><<<tiles, CF::NT, smem, st>>>(t2, G, ns, K, s, plane, tw, ext);
    return cudaGetLastError();
}

// variant v of kChainVariants
template <typename T, int L>
inline cudaError_t launch_chain_x_reg_L(int v, cplx<T> *t2, const cplx<T> *G, int ns, int K, int s, long long plane,
                                        const cplx<T> *tw, const int *ext, cudaStream_t st) {
    switch (v) {
        case 1: return launch_chain_x_v<T, L, 16, false, true>(t2, G, ns, K, s, plane, tw, ext, st);
        case 2: return launch_chain_x_v<T, L, 16, false, false>(t2, G, ns, K, s, plane, tw, ext, st);
        case 3: return launch_chain_x_v<T, L, 8, true, true>(t2, G, ns, K, s, plane, tw, ext, st);
        case 4: return launch_chain_x_v<T, L, 8, false, false>(t2, G, ns, K, s, plane, tw, ext, st);
        case 5: return launch_chain_x_v<T, L, 16, false, false, 3>(t2, G, ns, K, s, plane, tw, ext, st);
        case 6: return launch_chain_x_v<T, L, 16, false, false, 4>(t2, G, ns, K, s, plane, tw, ext, st);
        case 7: return launch_chain_x_v<T, L, 8, false, false, 8>(t2, G, ns, K, s, plane, tw, ext, st);
        case 8:
            if constexpr (L == 192) return launch_chain_x_192<T, 8, false, 4>(t2, G, ns, K, s, plane, tw, ext, st);
            return cudaErrorInvalidValue;
        case 9:
            if constexpr (L == 192) return launch_chain_x_192<T, 16, false, 2>(t2, G, ns, K, s, plane, tw, ext, st);
            return cudaErrorInvalidValue;
        case 10:
            if constexpr (L == 192) return launch_chain_x_192<T, 8, true, 4>(t2, G, ns, K, s, plane, tw, ext, st);
            return cudaErrorInvalidValue;
        case 11:
            if constexpr (L == 192) return launch_chain_x_192<T, 8, false, 3>(t2, G, ns, K, s, plane, tw, ext, st);
            return cudaErrorInvalidValue;
        case 12: return launch_chain_x_v<T, L, 8, false, true>(t2, G, ns, K, s, plane, tw, ext, st);
        case 13: return launch_chain_x_v<T, L, 8, true, true, 0, 1>(t2, G, ns, K, s, plane, tw, ext, st);
        case 14:
            if constexpr (Split<L>::R2 % 2 == 0) return launch_chain_x_v<T, L, 8, true, true, 5, 2>(t2, G, ns, K, s, plane, tw, ext, st);
            return cudaErrorInvalidValue;
        default: return launch_chain_x_v<T, L, 16, true, true>(t2, G, ns, K, s, plane, tw, ext, st);
    }
}

// whether variant v exists for line length L (8 .. 11: the 12-values-per-thread 192 kernel)
inline bool chain_variant_exists(int L, int v) { return v < 8 || v > 11 || L == 192; }

}  // namespace HG_TU_NS
}  // namespace hg
