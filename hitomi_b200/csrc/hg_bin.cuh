// hg_bin.cuh -- power-spectrum binning over a transformed field.
//
//   AxisTabs        per-axis sinc / sine tables with the reference's window index quirk
//   Spec<T>         read access to a half or full spectrum
//   k_pk_bin_list   binned  (f1 conj f2 - S C(k)) / W^2 * Yhat_lm(k)  (field.hpp:765-852)
//                   over the in-bin modes (k_pk_modes_*, once per context)
//   k_pk_bin        the same over the whole mode cube (the allocation-free entry point)
#pragma once

#include "hg_common.cuh"

namespace hg {
// one copy per translation unit: each .cu file names its own HG_TU_NS, so the kernels and
// helpers of this header never collide at link time
inline namespace HG_TU_NS {

// Per-axis tables indexed by array index i (mode n = wrap(i)):
//   tw[i] = sinc(pi w / n)   with w = (int)(n dk / dk + 1e-5)   (window, field.hpp:664-675)
//   ts[i] = sin(pi w / n)    (0 when w == 0)                   (shot noise, field.hpp:1261-1272)
struct AxisTabs {
    const double *tw[3];
    const double *ts[3];
    const double *tc[3];  // cos(pi w / n); needed only when interlace != 0
    int interlace;
};

// Per-axis factors of the separable weights of the shot-noise correlation field:
//   cf[i]  = the axis factor of C(k) for the assignment scheme (shot_tab's per-axis f),
//   df[i]  = the axis factor of the alternating image sum (interlacing only),
//   iw2[i] = 1 / (tw[i]^p)^2, so that 1 / W(k)^2 = iw2[x] iw2[y] iw2[z].
struct XiTabs {
    const double *cf[3];
    const double *df[3];
    const double *iw2[3];
    int interlace;
};

// Per-axis aliasing sums of W^2 over the images k + 2 k_N n (s = sin, c = cos of pi k / 2 k_N):
//   C_p = sum_n W_p^2        (Jing 2005 eq. 20; PCS from the same sum):
//         1, 1 - 2/3 s^2, 1 - s^2 + 2/15 s^4, 1 - 4/3 s^2 + 2/5 s^4 - 4/315 s^6
//   D_p = sum_n (-1)^n W_p^2 (closed form of the alternating sum of sinc^2p):
//         c, c (c^2 + 5) / 6, c (c^4 + 58 c^2 + 61) / 120, c (c^6 + 543 c^4 + 3111 c^2 + 1385) / 5040
// Interlacing two fields offset by half a cell keeps only the images with even n_x+n_y+n_z,
// so its shot-noise function is C_int = (prod_a C_a + prod_a D_a) / 2.
__host__ __device__ __forceinline__ double alias_c(int assign, double sn) {
    double s2 = sn * sn;
    if (assign == 0) return 1.0;
    if (assign == 1) return 1.0 - (2.0 / 3.0) * s2;
    if (assign == 2) return 1.0 - s2 + 2.0 * (s2 * s2) / 15.0;
    return 1.0 - (4.0 / 3.0) * s2 + (2.0 / 5.0) * s2 * s2 - (4.0 / 315.0) * s2 * s2 * s2;
}
__host__ __device__ __forceinline__ double alias_d(int assign, double c) {
    double c2 = c * c;
    if (assign == 0) return c;
    if (assign == 1) return c * (c2 + 5.0) / 6.0;
    if (assign == 2) return c * (c2 * c2 + 58.0 * c2 + 61.0) / 120.0;
    return c * (c2 * c2 * c2 + 543.0 * c2 * c2 + 3111.0 * c2 + 1385.0) / 5040.0;
}


__device__ __forceinline__ double window_tab(const AxisTabs &t, int ix, int iy, int iz, int p) {
    double ret = t.tw[0][ix] * t.tw[1][iy] * t.tw[2][iz];
    double w = ret;
    for (int q = 1; q < p; q++) w *= ret;
    return w;
}

__device__ __forceinline__ double shot_tab(const AxisTabs &t, int ix, int iy, int iz, int assign) {
    if (t.interlace)
        return 0.5 * (alias_c(assign, t.ts[0][ix]) * alias_c(assign, t.ts[1][iy]) * alias_c(assign, t.ts[2][iz]) +
                      alias_d(assign, t.tc[0][ix]) * alias_d(assign, t.tc[1][iy]) * alias_d(assign, t.tc[2][iz]));
    if (assign == 0) return 1.0;
    const double s[3] = {t.ts[0][ix], t.ts[1][iy], t.ts[2][iz]};
    double ret = 1.0;
    for (int a = 0; a < 3; a++) {
        double s2 = s[a] * s[a];
        double f;
        if (assign == 1) f = 1.0 - (2.0 / 3.0) * s2;
        else if (assign == 2) f = 1.0 - s2 + 2.0 * (s2 * s2) / 15.0;
        else f = 1.0 - (4.0 / 3.0) * s2 + (2.0 / 5.0) * s2 * s2 - (4.0 / 315.0) * s2 * s2 * s2;
        ret *= f;
    }
    return ret;
}

// Read access to a transformed field, either a half spectrum [n0][n1][n2/2+1] of a real
// input (negative kz by Hermitian symmetry) or a full [n0][n1][n2] spectrum.
template <typename T>
struct Spec {
    const cplx<T> *p;
    int n0, n1, n2;
    int half;
    __device__ __forceinline__ zd at(int ix, int iy, int iz) const {
        if (!half) {
            cplx<T> v = p[((long long)ix * n1 + iy) * n2 + iz];
            return mk<double>((double)v.x, (double)v.y);
        }
        int hz = n2 / 2 + 1;
        if (iz < hz) {
            cplx<T> v = p[((long long)ix * n1 + iy) * hz + iz];
            return mk<double>((double)v.x, (double)v.y);
        }
        int jx = neg_index(ix, n0), jy = neg_index(iy, n1), jz = n2 - iz;
        cplx<T> v = p[((long long)jx * n1 + jy) * hz + jz];
        return mk<double>((double)v.x, -(double)v.y);
    }
};

// sgn * conj(F(-k)): the transform of the conjugated weights, e.g.
// F_{l,-m}(k) = (-1)^m conj(F_{l,m}(-k)) since Yhat_{l,-m} = (-1)^m conj(Yhat_{l,m}).
template <typename T>
struct SpecMirror {
    Spec<T> s;
    double sgn;
    __device__ __forceinline__ zd at(int ix, int iy, int iz) const {
        zd v = s.at(neg_index(ix, s.n0), neg_index(iy, s.n1), neg_index(iz, s.n2));
        return mk<double>(sgn * v.x, -sgn * v.y);
    }
};

struct LM {
    int l, m;
};

#define HG_MAX_LM 16

struct LMList {
    int n;
    LM lm[HG_MAX_LM];
};

// P-binning over the mode cube [lo, lo+cnt) (wrapped modes).  acc: [nbin][nlm] complex,
// nmode: [nbin].  lut maps the fine index int(|k|/1e-4 + 0.5) to up to two coarse bins.
// Sum of v over the lanes of `grp` (a match_any group), valid in every member; all members
// call it together.
__device__ __forceinline__ double group_sum(double v, unsigned grp) {
    double s = 0.0;
    for (unsigned m = grp; m; m &= m - 1) s += __shfl_sync(grp, v, __ffs(m) - 1);
    return s;
}

// P binning (as k_pk_bin_list below) over the whole mode cube [lo, lo + cnt), without a mode
// list: the allocation-free entry point's (hg_static.cu), which has no room to keep one.
// Whole warps walk the mode cube together (every lane runs every iteration, so full-warp
// intrinsics are safe); lanes whose modes fall in the same bin pool their values through
// shuffles and one of them adds the pooled value to the block's shared-memory bins, which
// keeps the number of (serialising) FP64 shared-memory atomics near one per bin per warp
// step instead of one per mode.
template <typename T, class F1, class F2>
__global__ void k_pk_bin(F1 f1, F2 f2, Grid g, AxisTabs tabs, int3 lo, int3 cnt, const int2 *lut, int lutn,
                         int nbin, LMList lms, double S_re, double S_im, int assign, int wpow, double *acc,
                         unsigned long long *nmode, int k0_special, double k0_re, double k0_im) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *sacc = reinterpret_cast<double *>(smem_raw);
    unsigned long long *scnt = reinterpret_cast<unsigned long long *>(sacc + 2 * nbin * lms.n);
    for (int q = threadIdx.x; q < 2 * nbin * lms.n; q += blockDim.x) sacc[q] = 0.0;
    for (int q = threadIdx.x; q < nbin; q += blockDim.x) scnt[q] = 0ull;
    __syncthreads();
    const long long total = (long long)cnt.x * cnt.y * cnt.z;
    const int lane = threadIdx.x & 31;
    const long long wstride = (long long)gridDim.x * blockDim.x;
    for (long long wbase = (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31); wbase < total; wbase += wstride) {
        const long long idx = wbase + lane;
        int2 b = make_int2(-1, -1);
        zd pk2 = mk<double>(0.0, 0.0);
        double kv[3] = {0.0, 0.0, 0.0};
        if (idx < total) {
            int nx, ny, nz;
            split3((unsigned)idx, (unsigned)cnt.y, (unsigned)cnt.z, nx, ny, nz);
            nx += lo.x;
            ny += lo.y;
            nz += lo.z;
            const int ix = nx < 0 ? nx + g.n[0] : nx, iy = ny < 0 ? ny + g.n[1] : ny, iz = nz < 0 ? nz + g.n[2] : nz;
            kv[0] = kcomp(wrap_index(ix, g.n[0]), g.dk[0]);
            kv[1] = kcomp(wrap_index(iy, g.n[1]), g.dk[1]);
            kv[2] = kcomp(wrap_index(iz, g.n[2]), g.dk[2]);
            double kmag = kmag_exact(kv[0], kv[1], kv[2]);
            int kindex = (int)__dadd_rn(__ddiv_rn(kmag, 0.0001), 0.5);
            if (kindex < lutn) b = lut[kindex];
            if (b.x >= 0) {
                zd d1 = f1.at(ix, iy, iz), d2 = f2.at(ix, iy, iz);
                if (k0_special && ix == 0 && iy == 0 && iz == 0) {
                    pk2 = mk<double>(k0_re, k0_im);
                } else {
                    pk2 = mul_conj_rn(d1, d2);
                }
                double C = shot_tab(tabs, ix, iy, iz, assign);
                pk2 = pk2 - mk<double>(S_re * C, S_im * C);
                double wf = window_tab(tabs, ix, iy, iz, wpow);
                double w2 = wf * wf;
                pk2 = mk<double>(pk2.x / w2, pk2.y / w2);
            }
        }
        if (__all_sync(0xffffffffu, b.x < 0)) continue;
        const unsigned gx = __match_any_sync(0xffffffffu, b.x);
        const unsigned gy = __match_any_sync(0xffffffffu, b.y);
        const bool lx = (lane == __ffs(gx) - 1), ly = (lane == __ffs(gy) - 1);
        for (int q = 0; q < lms.n; q++) {
            zd v = mk<double>(0.0, 0.0);
            if (b.x >= 0) v = pk2 * ylm_reduced(lms.lm[q].l, lms.lm[q].m, kv[0], kv[1], kv[2]);
            const double sxr = group_sum(v.x, gx), sxi = group_sum(v.y, gx);
            if (b.x >= 0 && lx && HG_IN_BOUNDS(b.x < nbin, HG_SITE_BIN, b.x)) {
                atomicAdd(&sacc[2 * (b.x * lms.n + q)], sxr);
                atomicAdd(&sacc[2 * (b.x * lms.n + q) + 1], sxi);
            }
            const double syr = group_sum(v.x, gy), syi = group_sum(v.y, gy);
            if (b.y >= 0 && ly && HG_IN_BOUNDS(b.y < nbin, HG_SITE_BIN, b.y)) {
                atomicAdd(&sacc[2 * (b.y * lms.n + q)], syr);
                atomicAdd(&sacc[2 * (b.y * lms.n + q) + 1], syi);
            }
        }
        if (b.x >= 0 && lx) atomicAdd(&scnt[b.x], (unsigned long long)__popc(gx));
        if (b.y >= 0 && ly) atomicAdd(&scnt[b.y], (unsigned long long)__popc(gy));
    }
    __syncthreads();
    for (int q = threadIdx.x; q < 2 * nbin * lms.n; q += blockDim.x)
        if (sacc[q] != 0.0) atomicAdd(&acc[q], sacc[q]);
    for (int q = threadIdx.x; q < nbin; q += blockDim.x)
        if (scnt[q]) atomicAdd(&nmode[q], scnt[q]);
}

// The P-binning cube's modes that fall in some bin, with what the binning needs of each that
// does not depend on the field (its array indices, bins, C(k), W(k), k), built once per
// context: each binning then reads the spectrum at those modes only (k_pk_bin_list).
struct PkMode {
    int ix, iy, iz;
    int2 b;
    double C, wf;
    double kv[3];
    zd y[3];  // Yhat_l0(k) for l = 0, 2, 4 (the box multipoles), as ylm_reduced gives them
};

// Yhat_lm(k) of a listed mode: the stored value for (l, 0), l = 0, 2, 4, else evaluated
__device__ __forceinline__ zd pk_mode_ylm(const PkMode &m, int l, int mm) {
    if (mm == 0 && (l == 0 || l == 2 || l == 4)) return m.y[l >> 1];
    return ylm_reduced(l, mm, m.kv[0], m.kv[1], m.kv[2]);
}

// Mode idx of the cube [lo, lo + cnt) of wrapped modes: array indices, k (the reference's FP64
// expressions, kmag_exact) and the bins of the fine index int(|k| / 1e-4 + 0.5) through lut.
__device__ __forceinline__ int2 pk_mode_at(const Grid &g, int3 lo, int3 cnt, const int2 *lut, int lutn, long long idx,
                                           int &ix, int &iy, int &iz, double kv[3]) {
    int nx, ny, nz;
    split3((unsigned)idx, (unsigned)cnt.y, (unsigned)cnt.z, nx, ny, nz);
    nx += lo.x;
    ny += lo.y;
    nz += lo.z;
    ix = nx < 0 ? nx + g.n[0] : nx;
    iy = ny < 0 ? ny + g.n[1] : ny;
    iz = nz < 0 ? nz + g.n[2] : nz;
    kv[0] = kcomp(wrap_index(ix, g.n[0]), g.dk[0]);
    kv[1] = kcomp(wrap_index(iy, g.n[1]), g.dk[1]);
    kv[2] = kcomp(wrap_index(iz, g.n[2]), g.dk[2]);
    const double kmag = kmag_exact(kv[0], kv[1], kv[2]);
    const int kindex = (int)__dadd_rn(__ddiv_rn(kmag, 0.0001), 0.5);
    return (kindex < lutn) ? lut[kindex] : make_int2(-1, -1);
}

// flag[idx] = 1 when mode idx falls in a bin
__global__ void k_pk_modes_flag(Grid g, int3 lo, int3 cnt, const int2 *lut, int lutn, unsigned *flag) {
    const long long total = (long long)cnt.x * cnt.y * cnt.z;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        int ix, iy, iz;
        double kv[3];
        flag[idx] = pk_mode_at(g, lo, cnt, lut, lutn, idx, ix, iy, iz, kv).x >= 0 ? 1u : 0u;
    }
}

// the flagged modes at their exclusive-scan positions (cube order)
__global__ void k_pk_modes_fill(Grid g, AxisTabs tabs, int3 lo, int3 cnt, const int2 *lut, int lutn, int assign,
                                int wpow, const unsigned *pos, PkMode *out) {
    const long long total = (long long)cnt.x * cnt.y * cnt.z;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        PkMode m;
        m.b = pk_mode_at(g, lo, cnt, lut, lutn, idx, m.ix, m.iy, m.iz, m.kv);
        if (m.b.x < 0) continue;
        m.C = shot_tab(tabs, m.ix, m.iy, m.iz, assign);
        m.wf = window_tab(tabs, m.ix, m.iy, m.iz, wpow);
        for (int q = 0; q < 3; q++) m.y[q] = ylm_reduced(2 * q, 0, m.kv[0], m.kv[1], m.kv[2]);
        out[pos[idx]] = m;
    }
}

// Binned (f1 conj f2 - S C(k)) / W^2 * Yhat_lm(k) over the mode list (field.hpp:765-852);
// acc: [nbin][nlm] complex, nmode: [nbin].  Whole warps walk the list together (every lane
// runs every iteration, so full-warp intrinsics are safe); lanes whose modes fall in the same
// bin pool their values through shuffles and one of them adds the pooled value to the
// block's shared-memory bins, which keeps the number of (serialising) FP64 shared-memory
// atomics near one per bin per warp step instead of one per mode.
template <class F1, class F2>
__global__ void k_pk_bin_list(F1 f1, F2 f2, const PkMode *modes, long long nmodes, int nbin, LMList lms, double S_re,
                              double S_im, double *acc, unsigned long long *nmode, int k0_special, double k0_re,
                              double k0_im) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *sacc = reinterpret_cast<double *>(smem_raw);
    unsigned long long *scnt = reinterpret_cast<unsigned long long *>(sacc + 2 * nbin * lms.n);
    for (int q = threadIdx.x; q < 2 * nbin * lms.n; q += blockDim.x) sacc[q] = 0.0;
    for (int q = threadIdx.x; q < nbin; q += blockDim.x) scnt[q] = 0ull;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const long long wstride = (long long)gridDim.x * blockDim.x;
    for (long long wbase = (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31); wbase < nmodes; wbase += wstride) {
        const long long e = wbase + lane;
        int2 b = make_int2(-1, -1);
        zd pk2 = mk<double>(0.0, 0.0);
        const PkMode *mp = modes + (e < nmodes ? e : 0);
        if (e < nmodes) {
            const PkMode &m = *mp;
            b = m.b;
            const zd d1 = f1.at(m.ix, m.iy, m.iz), d2 = f2.at(m.ix, m.iy, m.iz);
            if (k0_special && m.ix == 0 && m.iy == 0 && m.iz == 0) {
                pk2 = mk<double>(k0_re, k0_im);
            } else {
                pk2 = mul_conj_rn(d1, d2);
            }
            pk2 = pk2 - mk<double>(S_re * m.C, S_im * m.C);
            const double w2 = m.wf * m.wf;
            pk2 = mk<double>(pk2.x / w2, pk2.y / w2);
        }
        // the list runs in cube order, so a warp's modes share one or two bins: per distinct
        // bin, a butterfly sum over the warp (log 32 shuffles, not one per member)
        const int nq = lms.n > 0 ? lms.n : 1;  // (the mode counts are added in pass q = 0)
        for (int q = 0; q < nq; q++) {
            zd v = mk<double>(0.0, 0.0);
            if (q < lms.n && b.x >= 0) v = pk2 * pk_mode_ylm(*mp, lms.lm[q].l, lms.lm[q].m);
            for (int side = 0; side < 2; side++) {
                const int mine = side ? b.y : b.x;
                unsigned rem = __ballot_sync(0xffffffffu, mine >= 0);
                while (rem) {
                    const int u = __shfl_sync(0xffffffffu, mine, __ffs(rem) - 1);
                    const bool in = (mine == u);
                    const unsigned grp = __ballot_sync(0xffffffffu, in);
                    double sr = in ? v.x : 0.0, si = in ? v.y : 0.0;
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) {
                        sr += __shfl_xor_sync(0xffffffffu, sr, o);
                        si += __shfl_xor_sync(0xffffffffu, si, o);
                    }
                    if (lane == 0 && HG_IN_BOUNDS(u < nbin, HG_SITE_BIN, u)) {
                        if (q < lms.n) {
                            atomicAdd(&sacc[2 * (u * lms.n + q)], sr);
                            atomicAdd(&sacc[2 * (u * lms.n + q) + 1], si);
                        }
                        if (q == 0) atomicAdd(&scnt[u], (unsigned long long)__popc(grp));
                    }
                    rem &= ~grp;
                }
            }
        }
    }
    __syncthreads();
    for (int q = threadIdx.x; q < 2 * nbin * lms.n; q += blockDim.x)
        if (sacc[q] != 0.0) atomicAdd(&acc[q], sacc[q]);
    for (int q = threadIdx.x; q < nbin; q += blockDim.x)
        if (scnt[q]) atomicAdd(&nmode[q], scnt[q]);
}

// Several spectra binned against one in a single pass (the survey P_l: every M of one l):
// per mode, sum_q w_q ((F_q conj F2 - S_q C(k)) / W^2) Yhat_{l_q m_q}(k), binned like k_pk_bin
// (the bin average is linear, so this equals the weighted sum of the per-term averages of
// powerspec.hpp:36-77 with the same mode counts).  F_q is a stored spectrum, or the mirror
// sg conj F(-k) of one.
#define HG_MAX_PK_TERMS 9
template <typename T>
struct PkTerm {
    Spec<T> f;
    int mirror;
    double sg;
    double S_re, S_im;
    int l, m;
    double w;
};
template <typename T>
struct PkTerms {
    int n;
    PkTerm<T> t[HG_MAX_PK_TERMS];
};

template <typename T, class F2>
__global__ void k_pk_bin_terms(PkTerms<T> terms, F2 f2, Grid g, AxisTabs tabs, int3 lo, int3 cnt, const int2 *lut,
                               int lutn, int nbin, int assign, int wpow, double *acc, unsigned long long *nmode) {
    __shared__ double sacc[2 * 256];
    __shared__ unsigned long long scnt[256];
    for (int q = threadIdx.x; q < 2 * nbin; q += blockDim.x) sacc[q] = 0.0;
    for (int q = threadIdx.x; q < nbin; q += blockDim.x) scnt[q] = 0ull;
    __syncthreads();
    const long long total = (long long)cnt.x * cnt.y * cnt.z;
    const int lane = threadIdx.x & 31;
    const long long wstride = (long long)gridDim.x * blockDim.x;
    for (long long wbase = (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31); wbase < total; wbase += wstride) {
        const long long idx = wbase + lane;
        int2 b = make_int2(-1, -1);
        zd v = mk<double>(0.0, 0.0);
        if (idx < total) {
            int nx, ny, nz;
            split3((unsigned)idx, (unsigned)cnt.y, (unsigned)cnt.z, nx, ny, nz);
            nx += lo.x;
            ny += lo.y;
            nz += lo.z;
            const int ix = nx < 0 ? nx + g.n[0] : nx, iy = ny < 0 ? ny + g.n[1] : ny, iz = nz < 0 ? nz + g.n[2] : nz;
            double kv[3];
            kv[0] = kcomp(wrap_index(ix, g.n[0]), g.dk[0]);
            kv[1] = kcomp(wrap_index(iy, g.n[1]), g.dk[1]);
            kv[2] = kcomp(wrap_index(iz, g.n[2]), g.dk[2]);
            const double kmag = kmag_exact(kv[0], kv[1], kv[2]);
            const int kindex = (int)__dadd_rn(__ddiv_rn(kmag, 0.0001), 0.5);
            if (kindex < lutn) b = lut[kindex];
            if (b.x >= 0) {
                const zd d2 = f2.at(ix, iy, iz);
                const double C = shot_tab(tabs, ix, iy, iz, assign);
                const double wf = window_tab(tabs, ix, iy, iz, wpow);
                const double w2 = wf * wf;
                const int jx = neg_index(ix, g.n[0]), jy = neg_index(iy, g.n[1]), jz = neg_index(iz, g.n[2]);
                for (int q = 0; q < terms.n; q++) {
                    const PkTerm<T> &tq = terms.t[q];
                    zd d1;
                    if (tq.mirror) {
                        const zd u = tq.f.at(jx, jy, jz);
                        d1 = mk<double>(tq.sg * u.x, -tq.sg * u.y);
                    } else {
                        d1 = tq.f.at(ix, iy, iz);
                    }
                    zd pk2 = d1 * conjg(d2) - mk<double>(tq.S_re * C, tq.S_im * C);
                    pk2 = mk<double>(pk2.x / w2, pk2.y / w2);
                    const zd y = ylm_reduced(tq.l, tq.m, kv[0], kv[1], kv[2]);
                    v = v + (pk2 * y) * tq.w;
                }
            }
        }
        if (__all_sync(0xffffffffu, b.x < 0)) continue;
        const unsigned gx = __match_any_sync(0xffffffffu, b.x);
        const unsigned gy = __match_any_sync(0xffffffffu, b.y);
        const bool lx = (lane == __ffs(gx) - 1), ly = (lane == __ffs(gy) - 1);
        const double sxr = group_sum(v.x, gx), sxi = group_sum(v.y, gx);
        if (b.x >= 0 && lx && HG_IN_BOUNDS(b.x < nbin, HG_SITE_BIN, b.x)) {
            atomicAdd(&sacc[2 * b.x], sxr);
            atomicAdd(&sacc[2 * b.x + 1], sxi);
            atomicAdd(&scnt[b.x], (unsigned long long)__popc(gx));
        }
        const double syr = group_sum(v.x, gy), syi = group_sum(v.y, gy);
        if (b.y >= 0 && ly && HG_IN_BOUNDS(b.y < nbin, HG_SITE_BIN, b.y)) {
            atomicAdd(&sacc[2 * b.y], syr);
            atomicAdd(&sacc[2 * b.y + 1], syi);
            atomicAdd(&scnt[b.y], (unsigned long long)__popc(gy));
        }
    }
    __syncthreads();
    for (int q = threadIdx.x; q < 2 * nbin; q += blockDim.x)
        if (sacc[q] != 0.0) atomicAdd(&acc[q], sacc[q]);
    for (int q = threadIdx.x; q < nbin; q += blockDim.x)
        if (scnt[q]) atomicAdd(&nmode[q], scnt[q]);
}

}  // namespace HG_TU_NS
}  // namespace hg
