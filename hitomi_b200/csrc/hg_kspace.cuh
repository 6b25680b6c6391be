// hg_kspace.cuh -- k-space and configuration-space kernels of the estimators.
//
//   k_axis_tables   per-axis sinc / sine tables with the reference's window index quirk
//   (P binning: k_pk_bin_list, hg_bin.cuh)
//   k_shell_D       delta(k)/W(k) for every (shell, mode) entry      (field.hpp:346-401)
//   k_family_A      A_f,i(k) = Yhat_f(k) delta/W / n_i
//   k_scatter_*     place k-space inputs on the compact shell / G cubes
//   k_pair_dot_items sum over a shell of A_a(k) Qhat_b(-k)
//   k_xi_orbit_hist last inverse-FFT pass of the shot-noise correlation field fused with
//                   its radial histogram over integer n^2 = |x/dr|^2
//   k_bessel_table, k_sn_matrix   spline-evaluated j_l products summed over n^2
#pragma once

#include <algorithm>
#include <type_traits>

#include "hg_common.cuh"
#include "hg_fft.cuh"
#include "hg_bin.cuh"
#include "hg_fft2.cuh"

namespace hg {
// one copy per translation unit: each .cu file names its own HG_TU_NS, so the kernels and
// helpers of this header never collide at link time
inline namespace HG_TU_NS {

__global__ void k_xi_tables(int n, const double *tw, const double *ts, const double *tc, int assign, int wpow,
                            double *cf, double *df, double *iw2) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    cf[i] = alias_c(assign, ts[i]);
    df[i] = alias_d(assign, tc[i]);
    double w = tw[i];
    for (int q = 1; q < wpow; q++) w *= tw[i];
    iw2[i] = 1.0 / (w * w);
}

// Per-axis window / shot-noise tables.  exact = 0: the reference's window index (n + 1 for
// negative modes, field.hpp:667-669); exact = 1: the mode index itself, used by the schemes
// the reference does not have (PCS, interlacing).
__global__ void k_axis_tables(Grid g, int axis, int exact, double *tw, double *ts, double *tc) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int n = g.n[axis];
    if (i >= n) return;
    double kv = kcomp(wrap_index(i, n), g.dk[axis]);
    int w = exact ? wrap_index(i, n) : window_index(kv, g.dk[axis]);
    tw[i] = sinc_axis(w, n);
    ts[i] = (w != 0) ? sin(HG_PI * (double)w / (double)n) : 0.0;
    tc[i] = (w != 0) ? cos(HG_PI * (double)w / (double)n) : 1.0;
}

// Interlacing (half-cell shifted second assignment): F = (F_0 + e^{i pi (nx/Nx + ny/Ny + nz/Nz)} F_s) / 2
// over a half spectrum (nz = iz) or a full one (nz wrapped).  The shifted catalogue sits at
// x + dr/2, so its transform carries e^{-i k dr/2}; the phase undoes it.
template <typename T>
__global__ void k_interlace(cplx<T> *F, const cplx<T> *Fs, int n0, int n1, int n2, int nzs, int half) {
    const long long total = (long long)n0 * n1 * nzs;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        int ix, iy, iz;
        split3((unsigned)idx, (unsigned)n1, (unsigned)nzs, ix, iy, iz);
        int nz = half ? iz : wrap_index(iz, n2);
        double q = (double)wrap_index(ix, n0) / n0 + (double)wrap_index(iy, n1) / n1 + (double)nz / n2;
        double sn, cs;
        sincospi(q, &sn, &cs);
        cplx<T> a = F[idx], b = Fs[idx];
        double br = (double)b.x, bi = (double)b.y;
        double re = 0.5 * ((double)a.x + (cs * br - sn * bi));
        double im = 0.5 * ((double)a.y + (cs * bi + sn * br));
        F[idx] = mk<T>((T)re, (T)im);
    }
}

// out[k] = sgn conj(in[-k]) over a full spectrum: the transform of the conjugated weights
// (F_{l,-m} = (-1)^m conj F_{l,m}(-k) since Yhat_{l,-m} = (-1)^m conj Yhat_{l,m}).
template <typename T>
__global__ void k_mirror(const cplx<T> *in, cplx<T> *out, int n0, int n1, int n2, T sgn) {
    const long long total = (long long)n0 * n1 * n2;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        int ix, iy, iz;
        split3((unsigned)idx, (unsigned)n1, (unsigned)n2, ix, iy, iz);
        cplx<T> v = in[((long long)neg_index(ix, n0) * n1 + neg_index(iy, n1)) * n2 + neg_index(iz, n2)];
        out[idx] = mk<T>(sgn * v.x, -sgn * v.y);
    }
}

// Shell entries: wrapped mode (nx, ny, nz) and shell index.
struct ShellEnt {
    int nx, ny, nz, shell;
};

__device__ __forceinline__ int mod_idx(int n, int N) { return ((n % N) + N) % N; }

template <typename T>
__global__ void k_shell_D(const ShellEnt *ent, long long ne, Spec<T> f, Grid g, AxisTabs tabs, int wpow, double2 *D) {
    long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    ShellEnt s = ent[e];
    int ix = mod_idx(s.nx, g.n[0]), iy = mod_idx(s.ny, g.n[1]), iz = mod_idx(s.nz, g.n[2]);
    zd d = f.at(ix, iy, iz);
    double wf = window_tab(tabs, ix, iy, iz, wpow);
    D[e] = make_double2(d.x / wf, d.y / wf);
}

// A[e] = (Yhat_lm(k) * D[e]) * scale_shell[shell(e)]   (scale = 1/n_mode or a Bessel weight)
__global__ void k_family_A(const ShellEnt *ent, long long ne, Grid g, int l, int m, const double2 *D,
                           const double *shell_scale, double2 *A) {
    long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    ShellEnt s = ent[e];
    zd y = ylm_reduced(l, m, kcomp(s.nx, g.dk[0]), kcomp(s.ny, g.dk[1]), kcomp(s.nz, g.dk[2]));
    zd v = y * mk<double>(D[e].x, D[e].y);
    double sc = shell_scale[s.shell];
    A[e] = make_double2(v.x * sc, v.y * sc);
}

// BAO reconstruction (particle_reconstruction.hpp:39-94): the full complex spectrum of the
// a-th displacement component, Psi_a(k) = -i (W_G(k) / b1) (k_a / k^2) D(k) / W(k) / V with
// W_G = exp(-(k R_G)^2 / 2), zero at k = 0 (|k| < 1e-10); D from the half spectrum.
template <typename T>
__global__ void k_recon_psi(Spec<T> f, Grid g, AxisTabs tabs, int wpow, int axis, double RG, double b1,
                            cplx<T> *out) {
    const long long total = g.ntot;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int iz = (int)(idx % g.n[2]);
        const int iy = (int)((idx / g.n[2]) % g.n[1]);
        const int ix = (int)(idx / ((long long)g.n[2] * g.n[1]));
        const double kv[3] = {kcomp(wrap_index(ix, g.n[0]), g.dk[0]), kcomp(wrap_index(iy, g.n[1]), g.dk[1]),
                              kcomp(wrap_index(iz, g.n[2]), g.dk[2])};
        const double kmag = sqrt(kv[0] * kv[0] + kv[1] * kv[1] + kv[2] * kv[2]);
        cplx<T> r = mk<T>(0, 0);
        if (!(kmag < 1.0e-10)) {
            const double kr = kmag * RG;
            const double wg = exp(-(kr * kr) / 2.0);
            const double c = (wg / b1) * (kv[axis] / (kmag * kmag));
            const zd d = f.at(ix, iy, iz);
            const double wf = window_tab(tabs, ix, iy, iz, wpow);
            // -i c (d / W) / V
            const double dr = (d.x / wf) / g.volume, di = (d.y / wf) / g.volume;
            r = mk<T>((T)(c * di), (T)(-c * dr));
        }
        out[idx] = r;
    }
}

// psi[i] = Re(field[i]) * norm (the displacement in position units)
template <typename T>
__global__ void k_real_scaled(const cplx<T> *in, long long n, double norm, T *out) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = (T)((double)in[i].x * norm);
}

// Shift each particle by the TSC-interpolated displacement (particle_reconstruction.hpp:152-205):
// anchor int(x n / L + 0.5), the reference's flat-index rule (only 0 <= flat < N is used),
// the 27 terms added to the position in the reference's order.  out: [n][3] doubles.
template <typename T>
__global__ void k_recon_shift(PartSrc src, Grid g, const T *__restrict__ p0, const T *__restrict__ p1,
                              const T *__restrict__ p2, double *out) {
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < src.n;
         p += (long long)gridDim.x * blockDim.x) {
        const double *rec = reinterpret_cast<const double *>(src.base + p * src.stride) + src.pos_off;
        double pos[3] = {rec[0], rec[1], rec[2]};
        double w[3][3];
        long long iw[3][3];
        for (int a = 0; a < 3; a++) {
            const double xp = pos[a] * double(g.n[a]) / g.L[a];
            const int i1 = (int)(xp + 0.5);
            const double dx = xp - double(i1);
            w[0][a] = __dmul_rn(__dmul_rn(0.5, __dsub_rn(0.5, dx)), __dsub_rn(0.5, dx));
            w[1][a] = __dsub_rn(0.75, __dmul_rn(dx, dx));
            w[2][a] = __dmul_rn(__dmul_rn(0.5, __dadd_rn(0.5, dx)), __dadd_rn(0.5, dx));
            iw[0][a] = i1 - 1;
            iw[1][a] = i1;
            iw[2][a] = i1 + 1;
        }
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++)
                for (int k = 0; k < 3; k++) {
                    const long long coord = (iw[i][0] * g.n[1] + iw[j][1]) * g.n[2] + iw[k][2];
                    if (coord < 0 || coord >= g.ntot) continue;
                    const double ww = __dmul_rn(__dmul_rn(w[i][0], w[j][1]), w[k][2]);
                    pos[0] = __dadd_rn(pos[0], __dmul_rn(ww, (double)p0[coord]));
                    pos[1] = __dadd_rn(pos[1], __dmul_rn(ww, (double)p1[coord]));
                    pos[2] = __dadd_rn(pos[2], __dmul_rn(ww, (double)p2[coord]));
                }
        out[3 * p + 0] = pos[0];
        out[3 * p + 1] = pos[1];
        out[3 * p + 2] = pos[2];
    }
}

// Scatter A[e] into the compact cube of its shell: buf[shell][nx+s][ny+s][nz+s].
template <typename T>
__global__ void k_scatter_cube(const ShellEnt *ent, long long ne, const double2 *A, int3 K, int3 s, cplx<T> *buf) {
    long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    ShellEnt q = ent[e];
    long long vol = (long long)K.x * K.y * K.z;
    long long idx = (long long)q.shell * vol + ((long long)(q.nx + s.x) * K.y + (q.ny + s.y)) * K.z + (q.nz + s.z);
    buf[idx] = mk<T>((T)A[e].x, (T)A[e].y);
}

// G input on the compact cube [lo, lo+cnt): g(k) = (delta(k)/W(k)) / V  (field.hpp:636-637,
// 332-335), with the k = 0 mode from the FP64 field integral.
template <typename T>
__global__ void k_scatter_G(Spec<T> f, Grid g, AxisTabs tabs, int wpow, int3 lo, int3 cnt, double k0_re, double k0_im,
                            cplx<T> *buf) {
    long long total = (long long)cnt.x * cnt.y * cnt.z;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        int nx, ny, nz;
        split3((unsigned)idx, (unsigned)cnt.y, (unsigned)cnt.z, nx, ny, nz);
        nx += lo.x;
        ny += lo.y;
        nz += lo.z;
        int ix = mod_idx(nx, g.n[0]), iy = mod_idx(ny, g.n[1]), iz = mod_idx(nz, g.n[2]);
        zd d = (ix == 0 && iy == 0 && iz == 0) ? mk<double>(k0_re, k0_im) : f.at(ix, iy, iz);
        double wf = window_tab(tabs, ix, iy, iz, wpow);
        double re = d.x / wf / g.volume, im = d.y / wf / g.volume;
        buf[idx] = mk<T>((T)re, (T)im);
    }
}

__device__ __forceinline__ int neg_c(int n, int M, int s) {
    int m = -n;
    if (m >= M / 2) m -= M;  // a whole (unreduced) axis: -(-M/2) is the same mode as -M/2
    return m + s;
}

// out[i][j] = sum_{e in shell i} A[e] * Q[j](-n_e), Q the compact cubes of a chain family.
// The sums are cut into work items: a warp takes up to 32 PD_LANE entries of one shell and
// gathers Q[j](-n_e) for every j (groups of PD_JG accumulators), so each lane keeps PD_JG
// independent loads in flight instead of one; warp sums go to part[item][j], and
// k_pair_sum_items adds a shell's items in a fixed order (deterministic).
#define PD_LANE 4
#define PD_JG 8
struct PairItem {
    int i, e0, e1;
};
template <typename T>
__global__ void k_pair_dot_items(const PairItem *items, int nitems, const ShellEnt *ent, const double2 *A,
                                 const cplx<T> *Q, int3 K, int3 M, int3 s, int ns_j, double2 *part) {
    const int wid = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (wid >= nitems) return;  // whole warps
    const PairItem it = items[wid];
    const long long vol = (long long)K.x * K.y * K.z;
    for (int j0 = 0; j0 < ns_j; j0 += PD_JG) {
        double ar[PD_JG], ai[PD_JG];
#pragma unroll
        for (int q = 0; q < PD_JG; q++) ar[q] = ai[q] = 0.0;
        for (int e = it.e0 + lane; e < it.e1; e += 32) {
            const ShellEnt q = ent[e];
            const long long idx =
                ((long long)neg_c(q.nx, M.x, s.x) * K.y + neg_c(q.ny, M.y, s.y)) * K.z + neg_c(q.nz, M.z, s.z);
            const double2 a = A[e];
            cplx<T> v[PD_JG];
#pragma unroll
            for (int jj = 0; jj < PD_JG; jj++) v[jj] = (j0 + jj < ns_j) ? Q[(long long)(j0 + jj) * vol + idx] : mk<T>(0, 0);
#pragma unroll
            for (int jj = 0; jj < PD_JG; jj++) {
                const double qx = (double)v[jj].x, qy = (double)v[jj].y;
                ar[jj] += a.x * qx - a.y * qy;
                ai[jj] += a.x * qy + a.y * qx;
            }
        }
#pragma unroll
        for (int jj = 0; jj < PD_JG; jj++) {
            double r = ar[jj], im = ai[jj];
            for (int o = 16; o > 0; o >>= 1) {
                r += __shfl_xor_sync(0xffffffffu, r, o);
                im += __shfl_xor_sync(0xffffffffu, im, o);
            }
            if (lane == 0 && j0 + jj < ns_j) part[(long long)wid * ns_j + j0 + jj] = make_double2(r, im);
        }
    }
}

// out[i][j] = sum over shell i's items (contiguous from istart[i]) of part[item][j]: one
// warp per output, lane l adds items l, l + 32, ... in order, then a fixed shuffle tree
__global__ void k_pair_sum_items(const int *istart, const double2 *part, int ns_i, int ns_j, double2 *out) {
    const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= (long long)ns_i * ns_j) return;  // whole warps
    const int q = (int)w, i = q / ns_j, j = q - i * ns_j;
    double r = 0.0, im = 0.0;
    for (int it = istart[i] + lane; it < istart[i + 1]; it += 32) {
        const double2 v = part[(long long)it * ns_j + j];
        r += v.x;
        im += v.y;
    }
    for (int d = 16; d > 0; d >>= 1) {
        r += __shfl_xor_sync(0xffffffffu, r, d);
        im += __shfl_xor_sync(0xffffffffu, im, d);
    }
    if (lane == 0) out[q] = make_double2(r, im);
}

// ---------------------------------------------------------------- shot-noise field
// Loader for the first inverse pass (along x) of
//   xi(x) = (1/V) sum_k (f1 conj f2 - S C(k)) / W(k)^2 e^{ikx}   (field.hpp:1116-1160)
// synthesising the k-space input from the half spectrum on the fly.
// SE: the spectrum's element type (an FP32 field may read the FP64 density directly).
template <typename T, typename SE = T>
struct LdXiHat {  // (|delta|^2 - S C(k)) / W(k)^2 / V  (field.hpp:1000-1020), separable tables
    Spec<SE> f;
    int n2;
    XiTabs xt;
    double S;
    double k0;  // (f1 conj f2)(k = 0) from the FP64 field integrals
    double invV;
    __device__ __forceinline__ T value(int ix, int iy, int iz) const {
        double p2;
        if (ix == 0 && iy == 0 && iz == 0) {
            p2 = k0;
        } else {
            zd d = f.at(ix, iy, iz);
            p2 = d.x * d.x + d.y * d.y;
        }
        return value_p2(ix, iy, iz, p2);
    }
    // the (x, y) factors of C, the interlaced image sum and 1 / W^2 (products formed in the same
    // order as value_p2, so value_xyz gives identical values)
    struct XY {
        double c, d, iw;
    };
    __device__ __forceinline__ XY xy(int ix, int iy) const {
        return XY{xt.cf[0][ix] * xt.cf[1][iy], xt.interlace ? xt.df[0][ix] * xt.df[1][iy] : 0.0,
                  xt.iw2[0][ix] * xt.iw2[1][iy]};
    }
    __device__ __forceinline__ T value_xyz(const XY &a, bool k0mode, int iz, cplx<SE> e) const {
        const double dx = (double)e.x, dy = (double)e.y;
        const double p2 = k0mode ? k0 : dx * dx + dy * dy;
        double C = a.c * xt.cf[2][iz];
        if (xt.interlace) C = 0.5 * (C + a.d * xt.df[2][iz]);
        const double iw = a.iw * xt.iw2[2][iz];
        return (T)(invV * ((p2 - S * C) * iw));
    }
    __device__ __forceinline__ T value_p2(int ix, int iy, int iz, double p2) const {
        double C = xt.cf[0][ix] * xt.cf[1][iy] * xt.cf[2][iz];
        if (xt.interlace) C = 0.5 * (C + xt.df[0][ix] * xt.df[1][iy] * xt.df[2][iz]);
        double iw = xt.iw2[0][ix] * xt.iw2[1][iy] * xt.iw2[2][iz];
        return (T)(invV * ((p2 - S * C) * iw));
    }
};

// The same spectrum as a complex field on the full grid (for k_synth: x = l, (y, z) = i), on
// meshes whose correlation field is transformed whole (k_xi_fold)
template <typename T, typename SE = T>
struct LdXiHatFull {
    LdXiHat<T, SE> h;
    __device__ __forceinline__ cplx<T> operator()(long long, int l, long long i) const {
        const unsigned ui = (unsigned)i;
        const int iy = (int)(ui / (unsigned)h.n2), iz = (int)(ui - (unsigned)iy * (unsigned)h.n2);
        return mk<T>(h.value(l, iy, iz), (T)0);
    }
};

// The real correlation-field spectrum P of the box, two kz columns per complex value:
// out[ix][iy][j] = P(ix, iy, 2j) + i P(ix, iy, 2j + 1)  ([n0][n1][n2/2]).  A complex
// transform of these lines along x and y gives both planes' transforms at once; the
// histogram kernel separates them.  By mirror pairs of rows: the kz >= n2/2 + 1 half of row (x, y) is the
// conjugate of the other row's (-x, -y) lower half, so a CTA that writes both rows of a pair
// reads every spectrum element from HBM once (the pair's second read of it comes from the
// cache) instead of twice.  Grid (n1, n0/2 + 1): CTA (y, x) takes row (x, y) and its mirror;
// on the planes x = 0 and x = n0/2, which are their own mirrors, only y <= n1/2.  A thread's
// four spectrum elements are addressed first and loaded together.
template <typename T, typename SE>
__global__ void k_synth_pairs_rows(LdXiHat<T, SE> ld, int n0, int n1, int nh, cplx<T> *out) {
    const int ix = blockIdx.y, iy = blockIdx.x;
    if ((ix == 0 || 2 * ix == n0) && 2 * iy > n1) return;  // counted as the mirror of y' < n1/2
    const int mx = (n0 - ix) % n0, my = (n1 - iy) % n1;
    const long long r = (long long)ix * n1 + iy, m = (long long)mx * n1 + my;
    const int n2 = 2 * nh, hz = nh + 1;
    const cplx<SE> *Hr = ld.f.p + r * hz, *Hm = ld.f.p + m * hz;
    const typename LdXiHat<T, SE>::XY ar = ld.xy(ix, iy), am = ld.xy(mx, my);
    const bool r0 = (ix == 0 && iy == 0), m0 = (mx == 0 && my == 0);
    for (int j = threadIdx.x; j < nh; j += blockDim.x) {
        const int k0 = 2 * j, k1 = 2 * j + 1;
        // kz < hz from the row itself, else (conjugated) from the mirror row at n2 - kz
        const cplx<SE> *pa0 = (k0 < hz) ? Hr + k0 : Hm + (n2 - k0);
        const cplx<SE> *pa1 = (k1 < hz) ? Hr + k1 : Hm + (n2 - k1);
        const cplx<SE> *pb0 = (k0 < hz) ? Hm + k0 : Hr + (n2 - k0);
        const cplx<SE> *pb1 = (k1 < hz) ? Hm + k1 : Hr + (n2 - k1);
        const cplx<SE> a0 = *pa0, a1 = *pa1, b0 = *pb0, b1 = *pb1;
        out[r * nh + j] = mk<T>(ld.value_xyz(ar, r0 && k0 == 0, k0, a0), ld.value_xyz(ar, false, k1, a1));
        if (m != r) out[m * nh + j] = mk<T>(ld.value_xyz(am, m0 && k0 == 0, k0, b0), ld.value_xyz(am, false, k1, b1));
    }
}


// Cross-spectrum version for the survey (field.hpp:1116-1160): (f1 conj f2 - S C(k)) / W^2 / V
// with complex S, f1 = the Yhat_LM-weighted D - alpha R field, f2 = the w^2 D + alpha^2 R field.
template <typename T>
struct LdXiCross {
    Spec<T> f1, f2;
    int n2;
    XiTabs xt;
    double S_re, S_im;
    double k0_re, k0_im;  // (f1 conj f2)(k = 0) from the FP64 field integrals
    double invV;
    __device__ __forceinline__ cplx<T> operator()(long long o, int l, long long i) const {
        int ix = l;
        const unsigned ui = (unsigned)i;
        const int iy = (int)(ui / (unsigned)n2);
        const int iz = (int)(ui - (unsigned)iy * (unsigned)n2);
        zd p2;
        if (ix == 0 && iy == 0 && iz == 0) {
            p2 = mk<double>(k0_re, k0_im);
        } else {
            p2 = f1.at(ix, iy, iz) * conjg(f2.at(ix, iy, iz));
        }
        double C = xt.cf[0][ix] * xt.cf[1][iy] * xt.cf[2][iz];
        if (xt.interlace) C = 0.5 * (C + xt.df[0][ix] * xt.df[1][iy] * xt.df[2][iz]);
        double iw = xt.iw2[0][ix] * xt.iw2[1][iy] * xt.iw2[2][iz];
        return mk<T>((T)(invV * ((p2.x - S_re * C) * iw)), (T)(invV * ((p2.y - S_im * C) * iw)));
    }
};

// out[ix][i] = ld(0, ix, i) over the full grid (i = iy * nz + iz): the correlation-field
// spectrum materialised by a grid-stride elementwise pass, so that the transform passes
// that follow are plain loads.
template <typename T, class LD>
__global__ void k_synth(LD ld, int n0, long long yz, cplx<T> *out) {
    const long long total = (long long)n0 * yz;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const unsigned u = (unsigned)idx, q = u / (unsigned)yz;
        out[idx] = ld(0, (int)q, (long long)(u - q * (unsigned)yz));
    }
}

// One product of reduced harmonics with its Wigner weight: w Yhat_l1m1 Yhat_l2m2.
struct YTerm {
    int l1, m1, l2, m2;
    double w;
};
#define HG_MAX_TERMS 24
#define HG_MAX_HIST 8
#define HG_CHEB 17
struct HistSpec {
    int nh;                      // number of histograms
    int nterm[HG_MAX_HIST];      // terms per histogram
    int parity[HG_MAX_HIST];     // (-1)^(l1+l2) of the histogram's terms
    YTerm term[HG_MAX_HIST][12];
    // m1 + m2 = 0: f_h is a real polynomial in mu = cos(theta) of degree l1 + l2, kept as
    // Chebyshev coefficients (exact interpolation at l1 + l2 + 1 Chebyshev nodes); f0 is
    // its value at r = 0, where Yhat_lm = 0 unless l = m = 0 (tools.hpp:12-68)
    int deg[HG_MAX_HIST];
    double cheb[HG_MAX_HIST][HG_CHEB];
    double f0[HG_MAX_HIST];
};

// sum_j c_j T_j(mu), Clenshaw recurrence
__device__ __forceinline__ double cheb_eval(const double *c, int deg, double mu) {
    double b1 = 0.0, b2 = 0.0;
    for (int j = deg; j >= 1; j--) {
        const double b0 = 2.0 * mu * b1 - b2 + c[j];
        b2 = b1;
        b1 = b0;
    }
    return mu * b1 - b2 + c[0];
}

// Last inverse pass (along z) over one symmetry orbit of (x, y) lines, fused with
//   T_h(n^2) += sum over the orbit and z <-> -z of xi(x) f_h(theta)
// where f_h = sum_terms w Yhat_l1m1 Yhat_l2m2 depends only on the polar angle (m1+m2 = 0),
// and n^2 = wx^2 + wy^2 + wz^2 in cell units (cubic cells).  The 8 lines are transformed
// with the register two-level FFT (R2 threads per line), then laid out in shared memory
// for the histogram.
template <typename T, int L>
struct OrbitCfg {
    static constexpr int B = 8;
    static constexpr int NT = Split<L>::R2 * B;
    static constexpr int LP = L + 1;
    static constexpr size_t smem() {
        return sizeof(cplx<T>) * ((size_t)B * LP > (size_t)XchgLayout<L, false, B>::ELEMS
                                      ? (size_t)B * LP
                                      : (size_t)XchgLayout<L, false, B>::ELEMS);
    }
};

template <typename T, int L>
__global__ void __launch_bounds__(OrbitCfg<T, L>::NT)
    k_xi_orbit_hist(const cplx<T> *xi, const int2 *orbit_reps, const int *orbit_n2xy, int n_orbits,
                    const cplx<T> *tw, HistSpec hs, long long n2dim, double *hist) {
    const int cta = blockIdx.x;  // orbits 2 cta and 2 cta + 1
    using OC = OrbitCfg<T, L>;
    constexpr int B = OC::B, LP = OC::LP, NT = OC::NT;
    constexpr int R1 = Split<L>::R1, R2 = Split<L>::R2;
    static_assert(B == 8, "two orbits of four representative lines per CTA");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx<T> *s = reinterpret_cast<cplx<T> *>(smem_raw);
    // the CTA's two orbits: their representative lines (with mirrors) and n_x^2 + n_y^2,
    // read once (the histogram phase consults them for every cell)
    __shared__ int2 reps[8];
    __shared__ int n2o[2];
    if (threadIdx.x < 8) {
        const int orb = 2 * cta + (threadIdx.x >> 2);
        reps[threadIdx.x] = (orb < n_orbits) ? orbit_reps[4 * orb + (threadIdx.x & 3)] : make_int2(-1, -1);
        if ((threadIdx.x & 3) == 0) n2o[threadIdx.x >> 2] = (orb < n_orbits) ? orbit_n2xy[orb] : 0;
    }
    __syncthreads();
    const int b = threadIdx.x / R2, t = threadIdx.x % R2;
    // xi holds Z = A + i B ([n0][n1][L/2]) after the x and y passes, A and B the transforms
    // of the even and odd kz planes of the real spectrum: A(x) = (Z(x) + conj Z(-x)) / 2,
    // B(x) = (Z(x) - conj Z(-x)) / (2 i), with -x the mirror line (-x, -y)
    constexpr int NH = L / 2;
    // (staging the 8 lines and their mirrors through shared memory with contiguous loads was
    // measured slower: 0.59 -> 0.74 ms per 512^3 mock)
    const int2 rep = reps[b];
    const int line = rep.x, mirror = rep.y;
    cplx<T> v[R1];
#pragma unroll
    for (int n1_ = 0; n1_ < R1; n1_++) {
        v[n1_] = mk<T>(0, 0);
        if (line >= 0) {
            const int kz = R2 * n1_ + t, j = kz >> 1;
            const cplx<T> zp = xi[(long long)line * NH + j], zm = xi[(long long)mirror * NH + j];
            v[n1_] = (kz & 1) ? mk<T>((T)0.5 * (zp.y + zm.y), (T)0.5 * (zm.x - zp.x))
                              : mk<T>((T)0.5 * (zp.x + zm.x), (T)0.5 * (zp.y - zm.y));
        }
    }
    line_fft2<T, L, +1, false, B>(v, s, t, b, tw);
#pragma unroll
    for (int r = 0; r < R1; r++) s[b * LP + pos_of_reg<L>(t, r)] = v[r];
    __syncthreads();
    // The mirror line carries conj xi(x, y, -z): with the pair folded over +-z, its even
    // part is the conjugate of the representative's and its odd part minus the conjugate,
    // so a representative with a distinct mirror adds 2 Re of its even part and 2i Im of its
    // odd part; a line that is its own mirror adds both parts as they are.  The planes z = 0
    // and z = L/2 (the reference's coordinate -L/2, field.hpp:1050) hold one cell per line,
    // weighted by f(mu) with mu of that sign, for either parity.
    for (int q = threadIdx.x; q < 2 * (L / 2 + 1); q += NT) {
        const int o = q / (L / 2 + 1), iz = q - o * (L / 2 + 1);
        const int orb = 2 * cta + o;
        if (orb >= n_orbits) continue;
        const int iz2 = (L - iz) % L;
        double er = 0, ei = 0, orr = 0, oi = 0;
        for (int bb = 4 * o; bb < 4 * o + 4; bb++) {
            const int2 rb = reps[bb];
            if (rb.x < 0) continue;
            const cplx<T> a = s[bb * LP + iz];
            const cplx<T> c = (iz2 == iz) ? mk<T>(0, 0) : s[bb * LP + iz2];
            if (rb.y == rb.x) {
                er += (double)a.x + (double)c.x;
                ei += (double)a.y + (double)c.y;
                orr += (double)a.x - (double)c.x;
                oi += (double)a.y - (double)c.y;
            } else {
                er += 2.0 * ((double)a.x + (double)c.x);
                oi += 2.0 * ((double)a.y - (double)c.y);
            }
        }
        if (iz2 == iz) {  // z = 0 or the Nyquist plane (z = -L/2): the cell counts once, either parity
            orr = er;
            oi = ei;
        }
        const int n2xy = n2o[o];
        int wz = wrap_index(iz, L);
        long long n2 = (long long)n2xy + (long long)wz * wz;
        const double r = sqrt((double)n2);
        const double mu = (n2 > 0) ? (double)wz / r : 0.0;
        for (int h = 0; h < hs.nh; h++) {
            const double f = (n2 > 0) ? cheb_eval(hs.cheb[h], hs.deg[h], mu) : hs.f0[h];
            zd src = (hs.parity[h] > 0) ? mk<double>(er, ei) : mk<double>(orr, oi);
            zd val = mk<double>(f * src.x, f * src.y);
            if (val.x != 0.0) atomicAdd(&hist[2 * ((long long)h * n2dim + n2)], val.x);
            if (val.y != 0.0) atomicAdd(&hist[2 * ((long long)h * n2dim + n2) + 1], val.y);
        }
    }
}

// The same histogram for weights that also depend on the azimuth (the survey's M != 0
// terms, m1 + m2 = -M): every (x, y) line on its own, B lines per CTA; the z <-> -z pair of
// a line shares n^2 and is added once.  f_h = sum_terms w Yhat_l1m1 Yhat_l2m2 at the cell.
template <typename T, int L>
__global__ void __launch_bounds__(OrbitCfg<T, L>::NT)
    k_xi_line_hist(const cplx<T> *xi, int n0, int n1, const cplx<T> *tw, HistSpec hs, long long n2dim, double *hist) {
    using OC = OrbitCfg<T, L>;
    constexpr int B = OC::B, LP = OC::LP, NT = OC::NT;
    constexpr int R1 = Split<L>::R1, R2 = Split<L>::R2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx<T> *s = reinterpret_cast<cplx<T> *>(smem_raw);
    const long long nlines = (long long)n0 * n1;
    const int b = threadIdx.x / R2, t = threadIdx.x % R2;
    const long long line = (long long)blockIdx.x * B + b;
    cplx<T> v[R1];
#pragma unroll
    for (int n1_ = 0; n1_ < R1; n1_++) v[n1_] = (line < nlines) ? xi[line * L + R2 * n1_ + t] : mk<T>(0, 0);
    line_fft2<T, L, +1, false, B>(v, s, t, b, tw);
#pragma unroll
    for (int r = 0; r < R1; r++) s[b * LP + pos_of_reg<L>(t, r)] = v[r];
    __syncthreads();
    for (int q = threadIdx.x; q < B * (L / 2 + 1); q += NT) {
        const int bb = q / (L / 2 + 1), iz = q % (L / 2 + 1);
        const long long ln = (long long)blockIdx.x * B + bb;
        if (ln >= nlines) continue;
        const int wx = wrap_index((int)(ln / n1), n0), wy = wrap_index((int)(ln % n1), n1);
        const int iz2 = (L - iz) % L;
        const int wz = wrap_index(iz, L);
        const cplx<T> a = s[bb * LP + iz], c = s[bb * LP + iz2];
        const long long n2 = (long long)wx * wx + (long long)wy * wy + (long long)wz * wz;
        for (int h = 0; h < hs.nh; h++) {
            zd fp = mk<double>(0.0, 0.0), fm = mk<double>(0.0, 0.0);
            for (int k = 0; k < hs.nterm[h]; k++) {
                const YTerm &yt = hs.term[h][k];
                fp = fp + (ylm_reduced(yt.l1, yt.m1, (double)wx, (double)wy, (double)wz) *
                           ylm_reduced(yt.l2, yt.m2, (double)wx, (double)wy, (double)wz)) * yt.w;
                if (iz2 != iz)
                    fm = fm + (ylm_reduced(yt.l1, yt.m1, (double)wx, (double)wy, (double)(-wz)) *
                               ylm_reduced(yt.l2, yt.m2, (double)wx, (double)wy, (double)(-wz))) * yt.w;
            }
            zd val = fp * mk<double>((double)a.x, (double)a.y);
            if (iz2 != iz) val = val + fm * mk<double>((double)c.x, (double)c.y);
            if (val.x != 0.0) atomicAdd(&hist[2 * ((long long)h * n2dim + n2)], val.x);
            if (val.y != 0.0) atomicAdd(&hist[2 * ((long long)h * n2dim + n2) + 1], val.y);
        }
    }
}

// The correlation-field histogram on any mesh (unequal cells, z lines of any length), from
// the transformed field xi [n0][n1][n2] in memory: key q is an octant cell (a, b, c),
// 0 <= a <= n0/2 ..., the cells (+-a, +-b, +-c) share the reference's |r| (rvec per axis
// (i < n/2 ? i : i - n) dr_axis, field.hpp:1040-1050), and
//   hist[h][q] = sum over those cells of xi(x) f_h(x),  f_h = sum_terms w Yhat_l1m1 Yhat_l2m2
// at the cell's physical direction (POLY: m1 + m2 = 0, f_h as the Chebyshev polynomial in
// mu = r_z / r, f0 at r = 0).  One thread per key gathers its mirror cells: no atomics.
template <typename T, bool POLY>
__global__ void k_xi_fold(const cplx<T> *__restrict__ xi, int n0, int n1, int n2, double dr0, double dr1, double dr2,
                          HistSpec hs, long long nkey, double *hist) {
    const int h1 = n1 / 2 + 1, h2 = n2 / 2 + 1;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < nkey;
         q += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(q % h2), b = (int)((q / h2) % h1), a = (int)(q / ((long long)h1 * h2));
        const int xs[2] = {a, n0 - a}, ys[2] = {b, n1 - b}, zs[2] = {c, n2 - c};
        const int nxm = (a == 0 || 2 * a == n0) ? 1 : 2, nym = (b == 0 || 2 * b == n1) ? 1 : 2,
                  nzm = (c == 0 || 2 * c == n2) ? 1 : 2;
        zd acc[HG_MAX_HIST];
        for (int h = 0; h < HG_MAX_HIST; h++) acc[h] = mk<double>(0.0, 0.0);
        for (int u = 0; u < nxm; u++)
            for (int v = 0; v < nym; v++)
                for (int w = 0; w < nzm; w++) {
                    const int ix = xs[u], iy = ys[v], iz = zs[w];
                    const double rx = (double)(ix < n0 / 2 ? ix : ix - n0) * dr0;
                    const double ry = (double)(iy < n1 / 2 ? iy : iy - n1) * dr1;
                    const double rz = (double)(iz < n2 / 2 ? iz : iz - n2) * dr2;
                    const cplx<T> x = xi[((long long)ix * n1 + iy) * n2 + iz];
                    const zd val = mk<double>((double)x.x, (double)x.y);
                    for (int h = 0; h < hs.nh; h++) {
                        zd f;
                        if (POLY) {
                            const double r = sqrt(rx * rx + ry * ry + rz * rz);
                            f = mk<double>((r > 0.0) ? cheb_eval(hs.cheb[h], hs.deg[h], rz / r) : hs.f0[h], 0.0);
                        } else {
                            f = mk<double>(0.0, 0.0);
                            for (int k = 0; k < hs.nterm[h]; k++) {
                                const YTerm &yt = hs.term[h][k];
                                f = f + (ylm_reduced(yt.l1, yt.m1, rx, ry, rz) * ylm_reduced(yt.l2, yt.m2, rx, ry, rz)) *
                                            yt.w;
                            }
                        }
                        acc[h] = acc[h] + f * val;
                    }
                }
        for (int h = 0; h < hs.nh; h++) {
            hist[2 * ((long long)h * nkey + q)] = acc[h].x;
            hist[2 * ((long long)h * nkey + q) + 1] = acc[h].y;
        }
    }
}

// J[i][q] = j_l(k_i r_q) at the keys' radii (the octant keys of k_xi_fold)
__global__ void k_bessel_table_r(const double *sy, const double *sc, int sn, double xmin, double dx, const double *kv,
                                 int nk, const double *rk, long long nkey, double *J);

// y += x (n doubles)
__global__ void k_axpy(double *y, const double *x, long long n) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] += x[i];
}

// Natural-spline evaluation of j_l at x (knots xmin + dx i, bessel.hpp:14-25).
__device__ __forceinline__ double spline_eval(const double *y, const double *c, int n, double xmin, double dx, double xv) {
    long i = (long)((xv - xmin) / dx);
    if (i > n - 2) i = n - 2;
    if (i < 0) i = 0;
    while (i > 0 && xmin + dx * double(i) > xv) i--;
    while (i < n - 2 && xmin + dx * double(i + 1) <= xv) i++;
    double xi = xmin + dx * double(i), xi1 = xmin + dx * double(i + 1);
    double h = xi1 - xi, t = xv - xi;
    double b = (y[i + 1] - y[i]) / h - h * (c[i + 1] + 2.0 * c[i]) / 3.0;
    double d = (c[i + 1] - c[i]) / (3.0 * h);
    return y[i] + t * (b + t * (c[i] + t * d));
}

// J[i][n2] = j_l(k_i * r(n2)),  r(n2) = dr sqrt(n2)
__global__ void k_bessel_table(const double *sy, const double *sc, int sn, double xmin, double dx, const double *kv,
                               int nk, double dr, long long n2dim, double *J) {
    long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (long long)nk * n2dim) return;
    int i = (int)(q / n2dim);
    long long n2 = q - (long long)i * n2dim;
    double r = dr * sqrt((double)n2);
    double x = kv[i] * r;
    double xmax = xmin + dx * double(sn - 1);
    J[q] = (x <= xmax) ? spline_eval(sy, sc, sn, xmin, dx, x) : 0.0;
}

__global__ void k_bessel_table_r(const double *sy, const double *sc, int sn, double xmin, double dx, const double *kv,
                                 int nk, const double *rk, long long nkey, double *J) {
    long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (long long)nk * nkey) return;
    const int i = (int)(q / nkey);
    const double x = kv[i] * rk[q - (long long)i * nkey];
    const double xmax = xmin + dx * double(sn - 1);
    J[q] = (x <= xmax) ? spline_eval(sy, sc, sn, xmin, dx, x) : 0.0;
}

// out[i1][i2] = sum_n2 J1[i1][n2] J2[i2][n2] hist[n2], as a skinny product J1 diag(h) J2^T.
// Persistent blocks walk chunks of HG_SN_CHUNK values of n2; each chunk's J1 rows, J2 rows and
// hist values stream into shared memory by cp.async (two stages: the next chunk loads while
// the current one is summed); a thread owns a 4 x 4 register tile of (i1, i2) and one residue
// class of the chunk; residue groups are summed in shared memory and each block writes its
// na x nb partial sums; k_sum_parts adds the partials in a fixed order (deterministic).
#define HG_SN_CHUNK 64
#define HG_SN_THREADS 256
// doubles of one stage: J1 and J2 rows (row r at r CHP + r / 4: one extra slot per tile of
// four rows puts the rows that a warp's tiles read at the same c on different banks), hist
__host__ __device__ inline int sn_off_b(int na4) { return 4 * na4 * (HG_SN_CHUNK + 1) + na4; }
__host__ __device__ inline int sn_off_h(int na4, int nb4) {  // even: the hist values are read as double2
    return (sn_off_b(na4) + 4 * nb4 * (HG_SN_CHUNK + 1) + nb4 + 1) & ~1;
}
__host__ __device__ inline int sn_stage_doubles(int na4, int nb4) { return sn_off_h(na4, nb4) + 2 * HG_SN_CHUNK; }
__global__ void __launch_bounds__(HG_SN_THREADS)
    k_sn_partial(const double *__restrict__ J1, int na, const double *__restrict__ J2, int nb,
                 const double *__restrict__ hist, long long n2dim, double *part) {
    constexpr int CH = HG_SN_CHUNK, CHP = HG_SN_CHUNK + 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int na4 = (na + 3) / 4, nb4 = (nb + 3) / 4;
    const int ntile = na4 * nb4;
    const int ngroup = max(1, HG_SN_THREADS / ntile);
    const int SD = sn_stage_doubles(na4, nb4);
    double *stage0 = reinterpret_cast<double *>(smem_raw);
    const int t = threadIdx.x;
    // padding rows (na <= r < 4 na4) feed only the tiles' unused accumulators: zero them once
    for (int e = t; e < 2 * SD; e += blockDim.x) stage0[e] = 0.0;
    __syncthreads();
    const int tile = t % ntile, grp = t / ntile;
    const bool active = (t < ntile * ngroup);
    const int ta = tile / nb4, tb = tile % nb4;
    const int offb = sn_off_b(na4), offh = sn_off_h(na4, nb4);
    double acc[4][4][2];
#pragma unroll
    for (int u = 0; u < 4; u++)
#pragma unroll
        for (int v = 0; v < 4; v++) acc[u][v][0] = acc[u][v][1] = 0.0;
    const long long nchunk = (n2dim + CH - 1) / CH;
    // chunk ch into stage buf: values past n2dim are zero-filled (no source bytes)
    auto prefetch = [&](long long ch, double *buf) {
        const long long n0 = ch * CH;
        for (int e = t; e < na * CH; e += blockDim.x) {
            const int r = e / CH, c = e - r * CH;
            const bool ok = n0 + c < n2dim;
            cp_async_elem(buf + r * CHP + (r >> 2) + c, J1 + (ok ? (long long)r * n2dim + n0 + c : 0), 8, ok);
        }
        for (int e = t; e < nb * CH; e += blockDim.x) {
            const int r = e / CH, c = e - r * CH;
            const bool ok = n0 + c < n2dim;
            cp_async_elem(buf + offb + r * CHP + (r >> 2) + c, J2 + (ok ? (long long)r * n2dim + n0 + c : 0), 8, ok);
        }
        for (int e = t; e < 2 * CH; e += blockDim.x) {
            const bool ok = n0 + (e >> 1) < n2dim;
            cp_async_elem(buf + offh + e, hist + (ok ? 2 * n0 + e : 0), 8, ok);
        }
        asm volatile("cp.async.commit_group;\n" ::);
    };
    int cur = 0;
    long long ch = blockIdx.x;
    if (ch < nchunk) prefetch(ch, stage0);
    for (; ch < nchunk; ch += gridDim.x) {
        const long long nx = ch + gridDim.x;
        if (nx < nchunk) prefetch(nx, stage0 + (size_t)(cur ^ 1) * SD);
        else asm volatile("cp.async.commit_group;\n" ::);  // one group per iteration
        asm volatile("cp.async.wait_group 1;\n" ::);
        __syncthreads();
        const double *sa = stage0 + (size_t)cur * SD;
        const double *sj = sa + offb;
        const double2 *sh = reinterpret_cast<const double2 *>(sa + offh);
        if (active) {
            for (int c = grp; c < CH; c += ngroup) {
                double av[4];
                double2 bv[4];
                const double2 h = sh[c];
#pragma unroll
                for (int u = 0; u < 4; u++) av[u] = sa[(4 * ta + u) * CHP + ta + c];
#pragma unroll
                for (int v = 0; v < 4; v++) {
                    const double j = sj[(4 * tb + v) * CHP + tb + c];
                    bv[v] = make_double2(j * h.x, j * h.y);
                }
#pragma unroll
                for (int u = 0; u < 4; u++)
#pragma unroll
                    for (int v = 0; v < 4; v++) {
                        acc[u][v][0] += av[u] * bv[v].x;
                        acc[u][v][1] += av[u] * bv[v].y;
                    }
            }
        }
        __syncthreads();  // this stage is the target of the prefetch two chunks on
        cur ^= 1;
    }
    asm volatile("cp.async.wait_group 0;\n" ::);
    __syncthreads();
    double2 *red = reinterpret_cast<double2 *>(smem_raw);
    for (int e = t; e < ntile * 16; e += blockDim.x) red[e] = make_double2(0.0, 0.0);
    __syncthreads();
    for (int g = 0; g < ngroup; g++) {
        if (active && grp == g) {
#pragma unroll
            for (int u = 0; u < 4; u++)
#pragma unroll
                for (int v = 0; v < 4; v++) {
                    double2 &r = red[tile * 16 + u * 4 + v];
                    r.x += acc[u][v][0];
                    r.y += acc[u][v][1];
                }
        }
        __syncthreads();
    }
    for (int e = t; e < na * nb; e += blockDim.x) {
        int i1 = e / nb, i2 = e % nb;
        double2 r = red[((i1 / 4) * nb4 + (i2 / 4)) * 16 + (i1 % 4) * 4 + (i2 % 4)];
        part[2 * ((long long)blockIdx.x * na * nb + e)] = r.x;
        part[2 * ((long long)blockIdx.x * na * nb + e) + 1] = r.y;
    }
}


#define HG_SN_MAXROWS 64  // rows per operand and launch (4 x 4 tiles, at most 256 of them)
inline size_t sn_partial_smem(int na, int nb) {
    const int na4 = (na + 3) / 4, nb4 = (nb + 3) / 4;
    size_t stages = sizeof(double) * 2 * (size_t)sn_stage_doubles(na4, nb4);
    size_t red = sizeof(double2) * 16 * (size_t)na4 * nb4;
    return stages > red ? stages : red;
}
inline int sn_partial_blocks(long long n2dim) {
    long long nchunk = (n2dim + HG_SN_CHUNK - 1) / HG_SN_CHUNK;
    return (int)std::min<long long>(nchunk, 2 * 148);
}

// ---------------------------------------------------------------- 3PCF (zeta)
// Per-mode factor of the 3PCF filtered fields (field.hpp:403-445) without the Bessel weight:
//   U(k) = Yhat_lm(k) delta(k) / W(k) / V        over the full grid, delta(0) = k0_re.
template <typename T>
__global__ void k_zeta_U(Spec<T> f, Grid g, AxisTabs tabs, int wpow, int l, int m, double k0_re, double k0_im,
                         cplx<T> *U) {
    const long long total = (long long)g.n[0] * g.n[1] * g.n[2];
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        int ix, iy, iz;
        split3((unsigned)idx, (unsigned)g.n[1], (unsigned)g.n[2], ix, iy, iz);
        zd d = (ix == 0 && iy == 0 && iz == 0) ? mk<double>(k0_re, k0_im) : f.at(ix, iy, iz);
        double wf = window_tab(tabs, ix, iy, iz, wpow);
        zd y = ylm_reduced(l, m, kcomp(wrap_index(ix, g.n[0]), g.dk[0]), kcomp(wrap_index(iy, g.n[1]), g.dk[1]),
                           kcomp(wrap_index(iz, g.n[2]), g.dk[2]));
        zd v = y * mk<double>(d.x / wf, d.y / wf);
        U[idx] = mk<T>((T)(v.x / g.volume), (T)(v.y / g.volume));
    }
}

// Loader of the first inverse pass (along x) of the fields F_r = IFFT[j_l(|k| r) U(k)]
// for a block of radii: o = radius within the block, l = ix, i = iy * nz + iz.
// J[r][n2] = j_l(dk r sqrt(n2)) with n2 = |n|^2 of the wrapped mode (cubic box).
// Other meshes (octant = 1): J[r][q] at the k-space octant key q = (|wx| h1 + |wy|) h2 + |wz|,
// h_a = n_a / 2 + 1, whose |k| is the reference's sqrt(kx^2 + ky^2 + kz^2).
template <typename T>
struct LdZetaField {
    const cplx<T> *U;
    const double *J;  // rows of the block's radii
    long long n2dim;  // keys per row
    int n0, n1, n2;
    int octant;
    __device__ __forceinline__ cplx<T> operator()(long long o, int l, long long i) const {
        const unsigned ui = (unsigned)i;
        const int iy = (int)(ui / (unsigned)n2);
        const int iz = (int)(ui - (unsigned)iy * (unsigned)n2);
        int wx = wrap_index(l, n0), wy = wrap_index(iy, n1), wz = wrap_index(iz, n2);
        long long q = octant ? ((long long)abs(wx) * (n1 / 2 + 1) + abs(wy)) * (n2 / 2 + 1) + abs(wz)
                             : (long long)wx * wx + (long long)wy * wy + (long long)wz * wz;
        double j = J[o * n2dim + q];
        cplx<T> u = U[(long long)l * n1 * n2 + i];
        return mk<T>((T)(j * (double)u.x), (T)(j * (double)u.y));
    }
};

// part[block][i1][i2] = sum over this block's cells x of Fa[i1](x) Fb[i2](x) G(x)
// (complex, FP64 accumulation).  Per chunk of HG_ZR_CHUNK cells the fields are staged in
// shared memory (as FP64, Fb premultiplied by G); a thread owns a 4 x 4 tile of (i1, i2)
// and one residue class of the chunk's cells; the residue groups are summed at the end.
#define HG_ZR_CHUNK 64
#define HG_ZR_THREADS 256
template <typename T>
__global__ void __launch_bounds__(HG_ZR_THREADS)
    k_zeta_pairsum(const cplx<T> *__restrict__ Fa, int na, const cplx<T> *__restrict__ Fb, int nb,
                   const cplx<T> *__restrict__ G, long long ntot, double *part) {
    constexpr int CH = HG_ZR_CHUNK, CHP = HG_ZR_CHUNK + 1;  // padded rows: distinct rows, distinct banks
    // operands staged in FP64 in both forms (FP32 staging and FP32 products were measured
    // slower: 19.1 against 18.1 ms per config-5 mock)
    using A = double;
    using A2 = double2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int na4 = (na + 3) / 4, nb4 = (nb + 3) / 4;
    const int ntile = na4 * nb4;
    const int ngroup = max(1, HG_ZR_THREADS / ntile);
    // row r of a staged operand starts at r CHP + r / 4 (one extra slot per tile of four
    // rows: the 16-byte rows a warp's tiles read at the same c fall on different banks;
    // measured 21.3 -> 18.1 ms per config-5 mock)
    constexpr int SH = 1;
    A2 *sa = reinterpret_cast<A2 *>(smem_raw);       // [4 na4][CHP] (+ na4)
    A2 *sb = sa + (size_t)4 * na4 * CHP + SH * na4;  // [4 nb4][CHP] (+ nb4)
    const int t = threadIdx.x;
    const int tile = t % ntile, grp = t / ntile;
    const bool active = (t < ntile * ngroup);
    const int ta = tile / nb4, tb = tile % nb4;
    double acc[4][4][2];
#pragma unroll
    for (int u = 0; u < 4; u++)
#pragma unroll
        for (int v = 0; v < 4; v++) acc[u][v][0] = acc[u][v][1] = 0.0;
    const long long nchunk = (ntot + CH - 1) / CH;
    for (long long ch = blockIdx.x; ch < nchunk; ch += gridDim.x) {
        const long long x0 = ch * CH;
        __syncthreads();
        for (int e = t; e < 4 * na4 * CH; e += blockDim.x) {
            int r = e / CH, c = e % CH;
            A2 v;
            v.x = v.y = (A)0;
            if (r < na && x0 + c < ntot) {
                cplx<T> a = Fa[(long long)r * ntot + x0 + c];
                v.x = (A)a.x;
                v.y = (A)a.y;
            }
            sa[r * CHP + SH * (r >> 2) + c] = v;
        }
        for (int e = t; e < 4 * nb4 * CH; e += blockDim.x) {
            int r = e / CH, c = e % CH;
            A2 v;
            v.x = v.y = (A)0;
            if (r < nb && x0 + c < ntot) {
                cplx<T> b = Fb[(long long)r * ntot + x0 + c];
                cplx<T> gg = G[x0 + c];
                const A br = (A)b.x, bi = (A)b.y, gr = (A)gg.x, gi = (A)gg.y;
                v.x = br * gr - bi * gi;
                v.y = br * gi + bi * gr;
            }
            sb[r * CHP + SH * (r >> 2) + c] = v;
        }
        __syncthreads();
        if (active) {
            for (int c = grp; c < CH; c += ngroup) {
                A2 av[4], bv[4];
#pragma unroll
                for (int u = 0; u < 4; u++) av[u] = sa[(4 * ta + u) * CHP + SH * ta + c];
#pragma unroll
                for (int v = 0; v < 4; v++) bv[v] = sb[(4 * tb + v) * CHP + SH * tb + c];
#pragma unroll
                for (int u = 0; u < 4; u++)
#pragma unroll
                    for (int v = 0; v < 4; v++) {
                        acc[u][v][0] += av[u].x * bv[v].x - av[u].y * bv[v].y;
                        acc[u][v][1] += av[u].x * bv[v].y + av[u].y * bv[v].x;
                    }
            }
        }
    }
    // sum the residue groups through shared memory: red[tile][u][v] (complex)
    __syncthreads();
    double2 *red = reinterpret_cast<double2 *>(smem_raw);
    const int nred = ntile * 16;
    for (int e = t; e < nred; e += blockDim.x) red[e] = make_double2(0.0, 0.0);
    __syncthreads();
    for (int g = 0; g < ngroup; g++) {
        if (active && grp == g) {
#pragma unroll
            for (int u = 0; u < 4; u++)
#pragma unroll
                for (int v = 0; v < 4; v++) {
                    double2 &r = red[tile * 16 + u * 4 + v];
                    r.x += acc[u][v][0];
                    r.y += acc[u][v][1];
                }
        }
        __syncthreads();
    }
    for (int e = t; e < na * nb; e += blockDim.x) {
        int i1 = e / nb, i2 = e % nb;
        int tl = (i1 / 4) * nb4 + (i2 / 4);
        double2 r = red[tl * 16 + (i1 % 4) * 4 + (i2 % 4)];
        part[2 * ((long long)blockIdx.x * na * nb + e)] = r.x;
        part[2 * ((long long)blockIdx.x * na * nb + e) + 1] = r.y;
    }
}

inline size_t zeta_pairsum_smem(int na, int nb) {
    size_t stage = sizeof(double2) * (size_t)((na + 3) / 4 + (nb + 3) / 4) * (4 * (HG_ZR_CHUNK + 1) + 1);
    size_t red = sizeof(double2) * 16 * (size_t)((na + 3) / 4) * ((nb + 3) / 4);
    return stage > red ? stage : red;
}

// out[o] = sum_b part[b][o], complex: one warp per output, lane l adds b = l, l + 32, ...
// in order, then a fixed shuffle tree (deterministic; the block partials' loads overlap).
__global__ void k_sum_parts(const double *part, int nblk, int nout, double2 *out) {
    const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= nout) return;  // whole warps
    const int o = (int)w;
    double re = 0.0, im = 0.0;
    for (int b = lane; b < nblk; b += 32) {
        const double2 v = reinterpret_cast<const double2 *>(part)[(long long)b * nout + o];
        re += v.x;
        im += v.y;
    }
    for (int d = 16; d > 0; d >>= 1) {
        re += __shfl_xor_sync(0xffffffffu, re, d);
        im += __shfl_xor_sync(0xffffffffu, im, d);
    }
    if (lane == 0) out[o] = make_double2(re, im);
}
// threads for k_sum_parts over nout outputs
inline long long sum_parts_threads(long long nout) { return nout * 32; }

// Functors used by the transform passes.
template <typename T>
struct LdMeshDelta {  // real density rho -> (rho - nbar) dV  (field.hpp:520-523, 313-318)
    const T *mesh;
    long long L;
    T nbar, dV;
    __device__ __forceinline__ cplx<T> operator()(long long o, int l, long long i) const {
        return mk<T>((mesh[o * L + l] - nbar) * dV, (T)0);
    }
};
template <typename T>
struct LdPlanar {  // complex mesh held as separate re / im arrays (rows of L along the last axis)
    const T *re, *im;
    long long L;
    __device__ __forceinline__ cplx<T> operator()(long long o, int l, long long i) const {
        return mk<T>(re[o * L + l], im[o * L + l]);
    }
};
template <typename T>
struct StHalf {  // keep the non-negative half of the last axis
    cplx<T> *H;
    int L, hz;
    __device__ __forceinline__ void operator()(long long o, int l, long long i, cplx<T> v) const {
        if (l < hz) H[o * hz + l] = v;
    }
};


}  // namespace HG_TU_NS
}  // namespace hg
