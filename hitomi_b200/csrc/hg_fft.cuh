// hg_fft.cuh -- batched 1-D FFT passes over the axes of a 3-D mesh (sm_100a).
//
// A 3-D transform is three passes, one per axis.  Each CTA stages a tile of B lines
// x L points in shared memory, runs a Stockham autosort FFT on them (radix-8 passes,
// one radix-4 or radix-2 pass for the remainder; every thread holds exactly 8 complex
// values per pass), and writes the tile back.  Lines along the contiguous axis are
// loaded whole; lines along a strided axis are loaded as B adjacent columns so each
// row of the tile is one coalesced segment.
//
// What is loaded and what is stored is delegated to loader / storer functors, so a
// pass can fuse its neighbours: a loader can synthesise the input from k-space
// formulas (shell filter, Y_lm, 1/W) or multiply by another field, and a storer can
// prune the output to the modes a later stage needs.  Pruned inputs are not read.
//
// Sign convention (FFTW's, which the reference uses): dir = -1 forward
// X[k] = sum_j x[j] e^{-2 pi i jk/L}; dir = +1 backward with e^{+2 pi i jk/L}; no scaling.
#pragma once

#include "hg_common.cuh"

#include <algorithm>

namespace hg {
// one copy per translation unit: each .cu file names its own HG_TU_NS, so the kernels and
// helpers of this header never collide at link time
inline namespace HG_TU_NS {

template <typename T>
struct TwTable {
    const cplx<T> *tw;  // tw[m] = exp(-2 pi i m / L), m in [0, L)
};

template <typename T, int DIR>
__device__ __forceinline__ cplx<T> mul_tw(cplx<T> v, cplx<T> w) {
    // multiply by w (DIR = -1) or conj(w) (DIR = +1)
    if (DIR < 0) return mk<T>(v.x * w.x - v.y * w.y, v.x * w.y + v.y * w.x);
    return mk<T>(v.x * w.x + v.y * w.y, v.y * w.x - v.x * w.y);
}

// multiply by exp(DIR * i pi / 2) = DIR * i
template <typename T, int DIR>
__device__ __forceinline__ cplx<T> mul_i(cplx<T> v) {
    if (DIR < 0) return mk<T>(v.y, -v.x);
    return mk<T>(-v.y, v.x);
}

template <typename T, int DIR>
__device__ __forceinline__ void dft2(cplx<T> &a, cplx<T> &b) {
    cplx<T> t = a;
    a = t + b;
    b = t - b;
}

// in-place 4-point DFT, natural order output: X[q] = sum_r v[r] w4^{rq}, w4 = e^{DIR 2 pi i/4}
template <typename T, int DIR>
__device__ __forceinline__ void dft4(cplx<T> &v0, cplx<T> &v1, cplx<T> &v2, cplx<T> &v3) {
    cplx<T> t0 = v0 + v2, t1 = v0 - v2;
    cplx<T> t2 = v1 + v3, t3 = mul_i<T, DIR>(v1 - v3);
    v0 = t0 + t2;
    v2 = t0 - t2;
    v1 = t1 + t3;
    v3 = t1 - t3;
}

// in-place 8-point DFT, natural order output
template <typename T, int DIR>
__device__ __forceinline__ void dft8(cplx<T> *v) {
    const T h = (T)0.70710678118654752440084436210485;
    // layer 1: pairs (r, r+4)
    cplx<T> a0 = v[0] + v[4], b0 = v[0] - v[4];
    cplx<T> a1 = v[1] + v[5], b1 = v[1] - v[5];
    cplx<T> a2 = v[2] + v[6], b2 = v[2] - v[6];
    cplx<T> a3 = v[3] + v[7], b3 = v[3] - v[7];
    // b_r *= w8^r, w8 = e^{DIR i pi/4}
    b1 = mk<T>(h * (b1.x - DIR * b1.y), h * (b1.y + DIR * b1.x));
    b2 = mul_i<T, DIR>(b2);
    b3 = mk<T>(h * (-b3.x - DIR * b3.y), h * (-b3.y + DIR * b3.x));
    dft4<T, DIR>(a0, a1, a2, a3);  // even outputs X[0],X[2],X[4],X[6]
    dft4<T, DIR>(b0, b1, b2, b3);  // odd outputs  X[1],X[3],X[5],X[7]
    v[0] = a0; v[2] = a1; v[4] = a2; v[6] = a3;
    v[1] = b0; v[3] = b1; v[5] = b2; v[7] = b3;
}

// One Stockham pass of radix R over B lines of length L resident in shared memory.
// Every thread owns 8 / R items (8 complex values in registers).
template <typename T, int L, int R, int DIR, int NT>
__device__ __forceinline__ void stockham_pass(cplx<T> *s, int LP, int B, int Ns, const cplx<T> *__restrict__ tw) {
    constexpr int IT = 8 / R;      // items per thread
    constexpr int LR = L / R;      // butterflies per line
    cplx<T> v[8];
    const int nitems = B * LR;
#pragma unroll
    for (int q = 0; q < IT; q++) {
        int it = threadIdx.x + q * NT;
        if (it < nitems) {
            int b = it / LR, j = it - b * LR;
            const cplx<T> *line = s + (size_t)b * LP;
#pragma unroll
            for (int r = 0; r < R; r++) v[q * R + r] = line[j + r * LR];
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < IT; q++) {
        int it = threadIdx.x + q * NT;
        if (it < nitems) {
            int b = it / LR, j = it - b * LR;
            int k = j % Ns;
            int tstep = L / (Ns * R);  // twiddle w_{Ns R}^{r k} = tw[r k tstep]
#pragma unroll
            for (int r = 1; r < R; r++) v[q * R + r] = mul_tw<T, DIR>(v[q * R + r], tw[(r * k * tstep) & (L - 1)]);
            if (R == 8) dft8<T, DIR>(&v[q * R]);
            else if (R == 4) dft4<T, DIR>(v[q * R], v[q * R + 1], v[q * R + 2], v[q * R + 3]);
            else dft2<T, DIR>(v[q * R], v[q * R + 1]);
            int idxD = (j / Ns) * Ns * R + k;
            cplx<T> *line = s + (size_t)b * LP;
#pragma unroll
            for (int r = 0; r < R; r++) line[idxD + r * Ns] = v[q * R + r];
        }
    }
    __syncthreads();
}

template <typename T, int L, int DIR, int NT>
__device__ __forceinline__ void smem_fft(cplx<T> *s, int LP, int B, const cplx<T> *__restrict__ tw) {
    int Ns = 1;
#pragma unroll 1
    for (; Ns * 8 <= L; Ns *= 8) stockham_pass<T, L, 8, DIR, NT>(s, LP, B, Ns, tw);
    if (Ns * 4 == L) stockham_pass<T, L, 4, DIR, NT>(s, LP, B, Ns, tw);
    else if (Ns * 2 == L) stockham_pass<T, L, 2, DIR, NT>(s, LP, B, Ns, tw);
}

// Tile geometry of one pass.  A 3-D array viewed as [outer][L][inner]; lines are
// (outer, *, inner).  inner == 1: a tile is B consecutive outer lines; otherwise a
// tile is B consecutive inner columns of one outer slab.
struct PassGeom {
    long long n_outer;
    long long n_inner;
};

template <typename T, int L, int DIR, int NT, int ELEMS, class LD, class ST>
__global__ void __launch_bounds__(NT) k_fft_pass(LD ld, ST st, PassGeom g, const cplx<T> *__restrict__ tw) {
    constexpr int B = ELEMS / L;
    constexpr int LP = L + ((sizeof(T) == 4) ? 1 : 1);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx<T> *s = reinterpret_cast<cplx<T> *>(smem_raw);
    const bool contig = (g.n_inner == 1);
    long long o0, i0;
    if (contig) {
        o0 = (long long)blockIdx.x * B;
        i0 = 0;
    } else {
        long long tiles_per_outer = (g.n_inner + B - 1) / B;
        o0 = (long long)blockIdx.x / tiles_per_outer;
        i0 = ((long long)blockIdx.x - o0 * tiles_per_outer) * B;
    }
    // ---- load
    for (int e = threadIdx.x; e < B * L; e += NT) {
        int b, l;
        long long o, i;
        if (contig) {
            b = e / L;
            l = e - b * L;
            o = o0 + b;
            i = 0;
        } else {
            l = e / B;
            b = e - l * B;
            o = o0;
            i = i0 + b;
        }
        bool ok = contig ? (o < g.n_outer) : (i < g.n_inner);
        s[(size_t)b * LP + l] = ok ? ld(o, l, i) : mk<T>(0, 0);
    }
    __syncthreads();
    smem_fft<T, L, DIR, NT>(s, LP, B, tw);
    // ---- store
    for (int e = threadIdx.x; e < B * L; e += NT) {
        int b, l;
        long long o, i;
        if (contig) {
            b = e / L;
            l = e - b * L;
            o = o0 + b;
            i = 0;
        } else {
            l = e / B;
            b = e - l * B;
            o = o0;
            i = i0 + b;
        }
        bool ok = contig ? (o < g.n_outer) : (i < g.n_inner);
        if (ok) st(o, l, i, s[(size_t)b * LP + l]);
    }
}

// ---------------------------------------------------------------- plain functors
// Load/store a complex array laid out as [outer][L][inner].
template <typename T>
struct LdArr {
    const cplx<T> *p;
    long long L, inner;
    __device__ __forceinline__ cplx<T> operator()(long long o, int l, long long i) const {
        return p[(o * L + l) * inner + i];
    }
};
template <typename T>
struct StArr {
    cplx<T> *p;
    long long L, inner;
    __device__ __forceinline__ void operator()(long long o, int l, long long i, cplx<T> v) const {
        p[(o * L + l) * inner + i] = v;
    }
};

// Tile parameters per precision: ELEMS complex values per CTA (64 KB of shared memory),
// NT = ELEMS / 8 threads.
template <typename T>
struct FFTTile;
template <>
struct FFTTile<float> {
    static constexpr int ELEMS = 8192;
    static constexpr int NT = 1024;
};
template <>
struct FFTTile<double> {
    static constexpr int ELEMS = 4096;
    static constexpr int NT = 512;
};

template <typename T, int L>
inline size_t fft_smem_bytes() {
    constexpr int B = FFTTile<T>::ELEMS / L;
    return (size_t)B * (L + 1) * sizeof(cplx<T>);
}

template <typename T, int L>
inline long long fft_num_tiles(PassGeom g) {
    constexpr int B = FFTTile<T>::ELEMS / L;
    if (g.n_inner == 1) return (g.n_outer + B - 1) / B;
    return g.n_outer * ((g.n_inner + B - 1) / B);
}

template <typename T, int L, int DIR, class LD, class ST>
inline cudaError_t launch_fft_pass_L(LD ld, ST st, PassGeom g, const cplx<T> *tw, cudaStream_t stream) {
    constexpr int NT = FFTTile<T>::NT;
    constexpr int ELEMS = FFTTile<T>::ELEMS;
    size_t smem = fft_smem_bytes<T, L>();
    auto kern = k_fft_pass<T, L, DIR, NT, ELEMS, LD, ST>;
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr_set = true;
    }
    long long tiles = fft_num_tiles<T, L>(g);
    if (tiles <= 0) return cudaSuccess;
    kern<<<(unsigned)tiles, NT, smem, stream>>>(ld, st, g, tw);
    return cudaGetLastError();
}

// Runtime dispatch over the supported power-of-two line lengths 8..1024.
template <typename T, int DIR, class LD, class ST>
inline cudaError_t launch_fft_pass(int L, LD ld, ST st, PassGeom g, const cplx<T> *tw, cudaStream_t stream) {
    switch (L) {
        case 8: return launch_fft_pass_L<T, 8, DIR>(ld, st, g, tw, stream);
        case 16: return launch_fft_pass_L<T, 16, DIR>(ld, st, g, tw, stream);
        case 32: return launch_fft_pass_L<T, 32, DIR>(ld, st, g, tw, stream);
        case 64: return launch_fft_pass_L<T, 64, DIR>(ld, st, g, tw, stream);
        case 128: return launch_fft_pass_L<T, 128, DIR>(ld, st, g, tw, stream);
        case 256: return launch_fft_pass_L<T, 256, DIR>(ld, st, g, tw, stream);
        case 512: return launch_fft_pass_L<T, 512, DIR>(ld, st, g, tw, stream);
        case 1024: return launch_fft_pass_L<T, 1024, DIR>(ld, st, g, tw, stream);
        default: return cudaErrorInvalidValue;
    }
}

inline bool fft_supported_length(int L) {
    return L >= 8 && L <= 1024 && (L & (L - 1)) == 0;
}

// ---------------------------------------------------------------- mixed-radix lengths
// Lines whose length is not a power of two (the reference transforms any n_mesh with
// FFTW, e.g. its survey meshes 250 x 460 x 260): a Stockham autosort transform over the
// factors of L (4s, then 2, then odd primes up to HG_MAX_RADIX), computed output by output
// between two shared-memory buffers.  Pass s with radix R after Ns = R_0 ... R_{s-1}: output
// o = (j / Ns) Ns R + k + q Ns (k = j mod Ns, q < R) is
//   sum_r in[j + r L / R] exp(DIR 2 pi i r (k + q Ns) / (Ns R)),
// the twiddle and the R-point DFT in one sum (every exponent is a multiple of 1 / L, read
// from the context's L-point table).  A pass costs L R complex products per line; the
// supported meshes' lines keep R <= 23.
#define HG_MAX_RADIX 31
#define HG_MAX_STAGES 16
struct MixedPlan {
    int L, nst;
    int R[HG_MAX_STAGES];
};

inline bool mixed_plan(int L, MixedPlan &p) {
    if (L < 2 || L > 2048) return false;
    p.L = L;
    p.nst = 0;
    int n = L;
    auto push = [&](int r) {
        if (p.nst >= HG_MAX_STAGES) return false;
        p.R[p.nst++] = r;
        n /= r;
        return true;
    };
    while (n % 4 == 0)
        if (!push(4)) return false;
    while (n % 2 == 0)
        if (!push(2)) return false;
    for (int f = 3; n > 1 && f <= HG_MAX_RADIX; f += 2)
        while (n % f == 0)
            if (!push(f)) return false;
    return n == 1;
}

template <typename T, int DIR, class LD, class ST>
__global__ void __launch_bounds__(256) k_fft_pass_mixed(LD ld, ST st, PassGeom g, MixedPlan pl, int B,
                                                        const cplx<T> *__restrict__ tw) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int L = pl.L;
    cplx<T> *s0 = reinterpret_cast<cplx<T> *>(smem_raw);
    cplx<T> *s1 = s0 + (size_t)B * L;
    cplx<T> *tws = s1 + (size_t)B * L;
    for (int e = threadIdx.x; e < L; e += blockDim.x) tws[e] = tw[e];
    const bool contig = (g.n_inner == 1);
    long long o0, i0;
    if (contig) {
        o0 = (long long)blockIdx.x * B;
        i0 = 0;
    } else {
        const long long tiles_per_outer = (g.n_inner + B - 1) / B;
        o0 = (long long)blockIdx.x / tiles_per_outer;
        i0 = ((long long)blockIdx.x - o0 * tiles_per_outer) * B;
    }
    // element e of the tile: line b, position l (contiguous axis: whole lines; strided axis:
    // B adjacent columns, so consecutive threads read consecutive addresses)
    auto at = [&](int e, int &b, int &l, long long &o, long long &i) {
        if (contig) {
            b = e / L;
            l = e - b * L;
            o = o0 + b;
            i = 0;
        } else {
            l = e / B;
            b = e - l * B;
            o = o0;
            i = i0 + b;
        }
        return contig ? (o < g.n_outer) : (i < g.n_inner);
    };
    for (int e = threadIdx.x; e < B * L; e += blockDim.x) {
        int b, l;
        long long o, i;
        const bool ok = at(e, b, l, o, i);
        s0[(size_t)b * L + l] = ok ? ld(o, l, i) : mk<T>(0, 0);
    }
    __syncthreads();
    cplx<T> *cur = s0, *nxt = s1;
    int Ns = 1;
    for (int sidx = 0; sidx < pl.nst; sidx++) {
        const int R = pl.R[sidx], LR = L / R, NsR = Ns * R, step = L / NsR;
        for (int e = threadIdx.x; e < B * L; e += blockDim.x) {
            const int b = e / L, o = e - b * L;
            const int blk = o / NsR, rem = o - blk * NsR, q = rem / Ns, k = rem - q * Ns;
            const int j = blk * Ns + k, m = (k + q * Ns) * step;
            if (!HG_IN_BOUNDS(j + (R - 1) * LR < L, HG_SITE_MIXED, j)) continue;
            const cplx<T> *line = cur + (size_t)b * L;
            cplx<T> acc = line[j];
            int ex = 0;
            for (int r = 1; r < R; r++) {
                ex += m;
                if (ex >= L) ex -= L;
                acc = acc + mul_tw<T, DIR>(line[j + r * LR], tws[ex]);
            }
            nxt[(size_t)b * L + o] = acc;
        }
        __syncthreads();
        cplx<T> *t = cur;
        cur = nxt;
        nxt = t;
        Ns = NsR;
    }
    for (int e = threadIdx.x; e < B * L; e += blockDim.x) {
        int b, l;
        long long o, i;
        if (at(e, b, l, o, i)) st(o, l, i, cur[(size_t)b * L + l]);
    }
}

template <typename T, int DIR, class LD, class ST>
inline cudaError_t launch_fft_mixed(int L, LD ld, ST st, PassGeom g, const cplx<T> *tw, cudaStream_t stream) {
    MixedPlan pl;
    if (!mixed_plan(L, pl)) return cudaErrorInvalidValue;
    // B lines per CTA: two line buffers and the twiddles within 96 KB
    const int per = (int)((96 * 1024) / sizeof(cplx<T>));
    const int B = std::max(1, std::min(64, (per - L) / (2 * L)));
    const size_t smem = ((size_t)2 * B * L + L) * sizeof(cplx<T>);
    auto kern = k_fft_pass_mixed<T, DIR, LD, ST>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const long long tiles = (g.n_inner == 1) ? (g.n_outer + B - 1) / B : g.n_outer * ((g.n_inner + B - 1) / B);
    if (tiles <= 0) return cudaSuccess;
    kern<<<(unsigned)tiles, 256, smem, stream>>>(ld, st, g, pl, B, tw);
    return cudaGetLastError();
}

// Every length a pass accepts: the power-of-two register and Stockham kernels, and the
// mixed-radix kernel for lengths whose prime factors are at most HG_MAX_RADIX.
inline bool fft_any_length(int L) {
    MixedPlan pl;
    return fft_supported_length(L) || (L >= 8 && mixed_plan(L, pl));
}

}  // namespace HG_TU_NS
}  // namespace hg
