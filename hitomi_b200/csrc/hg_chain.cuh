// hg_chain.cuh -- pruned shell-field transforms on the reduced M^3 grid.
//
// A chain takes the compact k-space cube A_j(n), |n_a| <= s (K = 2s+1 per axis, one cube
// per shell j), to Qhat_j(n) = FFT[ IFFT[A_j] * G ](n) on the same cube.  Only the last
// spatial axis ever holds all M points of every line:
//
//   B1  z   A  [j][cx][cy][cz]  -> T1 [j][cx][cy][z]     (K^2 lines, K -> M)
//   B2  y   T1 [j][cx][cy][z]   -> T2 [j][cx][y][z]      (K M lines, K -> M)
//   X   x   T2 [j][cx][y][z]    -> T2                    (M^2 lines per j: K -> M, * G, M -> K)
//   F2  y   T2 [j][cx][y][z]    -> T1 [j][cx][cy][z]     (K M lines, M -> K)
//   F3  z   T1 [j][cx][cy][z]   -> Q  [j][cx][cy][cz]    (K^2 lines, M -> K)
//
// B1, B2, F2, F3 are the generic pass kernel with pruning functors.  X is one kernel that
// stages a tile of G (M x B columns) in shared memory once and runs every shell j through
// it: inverse FFT along x, multiply by G, forward FFT along x, keep the K modes.  The M^3
// field F_j G never touches HBM.
#pragma once

#include "hg_common.cuh"
#include "hg_fft.cuh"

namespace hg {
// one copy per translation unit: each .cu file names its own HG_TU_NS, so the kernels and
// helpers of this header never collide at link time
inline namespace HG_TU_NS {

// wrapped mode n of line position p on an axis of M points; compact index c = n + s
__device__ __forceinline__ int pos_to_c(int p, int M, int s) {
    int n = (p < M / 2) ? p : p - M;
    return (n >= -s && n <= s) ? n + s : -1;
}

// B1: compact cube line (K contiguous) -> positions of an M-point line (contig mode)
template <typename T>
struct LdCube {
    const cplx<T> *p;
    int K, M, s;
    __device__ __forceinline__ cplx<T> operator()(long long o, int l, long long i) const {
        int c = pos_to_c(l, M, s);
        return (c >= 0) ? p[o * K + c] : mk<T>(0, 0);
    }
};
// F3: keep the K kept positions of a contiguous M-point line into a compact line
template <typename T>
struct StCube {
    cplx<T> *p;
    int K, M, s;
    __device__ __forceinline__ void operator()(long long o, int l, long long i, cplx<T> v) const {
        int c = pos_to_c(l, M, s);
        if (c >= 0) p[o * K + c] = v;
    }
};
// B2 / F2 (strided, along the middle axis): arrays [o][Lc][inner] with Lc = K (compact)
// or M (full) rows.  Loader reads compact rows, storer writes full rows, or the reverse.
template <typename T>
struct LdRowsCompact {  // input [o][K][inner], position l -> compact row
    const cplx<T> *p;
    int K, M, s;
    long long inner;
    __device__ __forceinline__ cplx<T> operator()(long long o, int l, long long i) const {
        int c = pos_to_c(l, M, s);
        return (c >= 0) ? p[(o * K + c) * inner + i] : mk<T>(0, 0);
    }
};
template <typename T>
struct StRowsCompact {  // output [o][K][inner], keep compact rows only
    cplx<T> *p;
    int K, M, s;
    long long inner;
    __device__ __forceinline__ void operator()(long long o, int l, long long i, cplx<T> v) const {
        int c = pos_to_c(l, M, s);
        if (c >= 0) p[(o * K + c) * inner + i] = v;
    }
};

// Column pruning of the forward passes F2 and F3: the pair sums read Qhat only at shell
// modes, so a z line (cx, cy) that no shell mode has is not transformed by F3, and F2 stores
// per cx only the range of cy that holds such columns.
template <typename T>
struct StRowsCompactD {  // StRowsCompact that keeps, per cx, the rows cy in [cyr.x, cyr.y] only
    cplx<T> *p;
    int K, M, s;
    long long inner;
    int kx;             // lines (j, cx) per shell: o = j kx + cx
    const int2 *cyr;    // [kx]: the smallest and largest cy of the needed columns (cx, cy)
    __device__ __forceinline__ void operator()(long long o, int l, long long i, cplx<T> v) const {
        const int c = pos_to_c(l, M, s);
        const int2 r = cyr[(int)o % kx];  // the same for the whole line
        if (c >= r.x && c <= r.y) p[(o * K + c) * inner + i] = v;
    }
};
template <typename T>
struct LdArrL {  // [o][L][inner] at line lines[q]
    const cplx<T> *p;
    long long L, inner;
    const int *lines;
    __device__ __forceinline__ cplx<T> operator()(long long q, int l, long long i) const {
        return p[((long long)lines[q] * L + l) * inner + i];
    }
};
template <typename T>
struct StCubeL {  // StCube at line lines[q]
    cplx<T> *p;
    int K, M, s;
    const int *lines;
    __device__ __forceinline__ void operator()(long long q, int l, long long i, cplx<T> v) const {
        const int c = pos_to_c(l, M, s);
        if (c >= 0) p[(long long)lines[q] * K + c] = v;
    }
};

// Shell-extent pruning of B1 and B2.  Shell j's modes reach |n_a| <= e_j,a only (e_j grows
// with k_j; the cube side K = 2s+1 is set by the largest shell), so B2 transforms only the
// lines (j, cx) with |cx - s_x| <= e_j,x, and B1 only the lines (j, cx, cy) whose cy lies in
// the range of shell j's modes at that cx (a disc's row, narrower than |cy - s_y| <= e_j,y
// away from cx = s_x): pass line q is line lines[q] of the full layout.  T1 and T2 lines
// outside those sets are never written, and their readers (B2's rows, X's rows) treat them
// as zero by the same ranges.
template <typename T>
struct LdCubeL {  // B1: compact cube line lines[q], kept modes |n_z| <= e_j,z
    const cplx<T> *p;
    int K, M, s;
    const int *lines;
    const int4 *ext;  // per shell (e_x, e_y, e_z, -)
    int kxky;         // Kx Ky: lines per shell
    __device__ __forceinline__ cplx<T> operator()(long long q, int l, long long i) const {
        const int o = lines[q];
        const int e = ext[o / kxky].z;
        const int n = (l < M / 2) ? l : l - M;
        return (n >= -e && n <= e) ? p[(long long)o * K + n + s] : mk<T>(0, 0);
    }
};
template <typename T>
struct LdRowsCompactL {  // B2: [o][K][inner] at line lines[q], compact rows c in cyr[o]
    const cplx<T> *p;
    int K, M, s;
    long long inner;
    const int *lines;
    const int2 *cyr;  // per line (j, cx): the compact rows B1 wrote (shell j's modes' cy range)
    __device__ __forceinline__ cplx<T> operator()(long long q, int l, long long i) const {
        const int o = lines[q];
        const int2 r = cyr[o];
        const int n = (l < M / 2) ? l : l - M;
        const int c = n + s;
        return (c >= r.x && c <= r.y) ? p[((long long)o * K + c) * inner + i] : mk<T>(0, 0);
    }
};
template <typename T>
struct StArrL {  // [o][L][inner] at line lines[q]
    cplx<T> *p;
    long long L, inner;
    const int *lines;
    __device__ __forceinline__ void operator()(long long q, int l, long long i, cplx<T> v) const {
        p[((long long)lines[q] * L + l) * inner + i] = v;
    }
};

// X: fused  inverse FFT (x) -> * G -> forward FFT (x)  over all shells of a family.
// T2 layout [j][cx][y][z] (K rows of M*M); G layout [x][y][z].  One CTA per tile of
// B consecutive (y,z) columns; shells processed in a loop.  Shared memory: the G tile
// (B lines x M) and the work tile (B lines x M).
template <typename T, int L>
struct XTile {
    static constexpr int ELEMS = FFTTile<T>::ELEMS;
    static constexpr int NT = FFTTile<T>::NT;
    static constexpr int B = ELEMS / L;
    static constexpr int LP = L + 1;
};

template <typename T, int L>
__global__ void __launch_bounds__(XTile<T, L>::NT)
    k_chain_x(cplx<T> *t2, const cplx<T> *__restrict__ G, int ns, int K, int s, long long plane,
              const cplx<T> *__restrict__ tw, const int *__restrict__ ext_x) {
    using X = XTile<T, L>;
    constexpr int B = X::B, LP = X::LP, NT = X::NT;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx<T> *g = reinterpret_cast<cplx<T> *>(smem_raw);
    cplx<T> *w = g + B * LP;
    const long long i0 = (long long)blockIdx.x * B;  // first (y,z) column of the tile
    // G tile: rows x in [0, L), columns i0..i0+B
    for (int e = threadIdx.x; e < B * L; e += NT) {
        int x = e / B, b = e - x * B;
        long long i = i0 + b;
        g[b * LP + x] = (i < plane) ? G[(long long)x * plane + i] : mk<T>(0, 0);
    }
    for (int j = 0; j < ns; j++) {
        cplx<T> *tj = t2 + (long long)j * K * plane;
        const int ej = ext_x ? ext_x[j] : s;  // rows of shell j that B2 wrote
        __syncthreads();
        for (int e = threadIdx.x; e < B * L; e += NT) {
            int x = e / B, b = e - x * B;
            long long i = i0 + b;
            const int n = (x < L / 2) ? x : x - L;
            w[b * LP + x] = (n >= -ej && n <= ej && i < plane) ? tj[(long long)(n + s) * plane + i] : mk<T>(0, 0);
        }
        __syncthreads();
        smem_fft<T, L, +1, NT>(w, LP, B, tw);
        for (int e = threadIdx.x; e < B * L; e += NT) {
            int b = e / L, x = e - b * L;
            w[b * LP + x] = w[b * LP + x] * g[b * LP + x];
        }
        __syncthreads();
        smem_fft<T, L, -1, NT>(w, LP, B, tw);
        for (int e = threadIdx.x; e < B * L; e += NT) {
            int x = e / B, b = e - x * B;
            long long i = i0 + b;
            int c = pos_to_c(x, L, s);
            if (c >= 0 && i < plane) tj[(long long)c * plane + i] = w[b * LP + x];
        }
    }
}

template <typename T, int L>
inline size_t chain_x_smem() {
    using X = XTile<T, L>;
    return (size_t)2 * X::B * X::LP * sizeof(cplx<T>);
}

template <typename T, int L>
inline cudaError_t launch_chain_x_L(cplx<T> *t2, const cplx<T> *G, int ns, int K, int s, long long plane,
                                    const cplx<T> *tw, const int *ext, cudaStream_t st) {
    using X = XTile<T, L>;
    size_t smem = chain_x_smem<T, L>();
    cudaFuncSetAttribute(k_chain_x<T, L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    unsigned tiles = (unsigned)((plane + X::B - 1) / X::B);
    k_chain_x<T, L><<<tiles, X::NT, smem, st>>>(t2, G, ns, K, s, plane, tw, ext);
    return cudaGetLastError();
}

template <typename T>
inline cudaError_t launch_chain_x(int L, cplx<T> *t2, const cplx<T> *G, int ns, int K, int s, long long plane,
                                  const cplx<T> *tw, const int *ext, cudaStream_t st) {
    switch (L) {
        case 8: return launch_chain_x_L<T, 8>(t2, G, ns, K, s, plane, tw, ext, st);
        case 16: return launch_chain_x_L<T, 16>(t2, G, ns, K, s, plane, tw, ext, st);
        case 32: return launch_chain_x_L<T, 32>(t2, G, ns, K, s, plane, tw, ext, st);
        case 64: return launch_chain_x_L<T, 64>(t2, G, ns, K, s, plane, tw, ext, st);
        case 128: return launch_chain_x_L<T, 128>(t2, G, ns, K, s, plane, tw, ext, st);
        case 256: return launch_chain_x_L<T, 256>(t2, G, ns, K, s, plane, tw, ext, st);
        case 512: return launch_chain_x_L<T, 512>(t2, G, ns, K, s, plane, tw, ext, st);
        case 1024: return launch_chain_x_L<T, 1024>(t2, G, ns, K, s, plane, tw, ext, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace HG_TU_NS
}  // namespace hg
