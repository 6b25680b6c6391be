// hg_kspace.cuh -- k-space and configuration-space kernels of the estimators.
//
//   k_axis_tables   per-axis sinc / sine tables with the reference's window index quirk
//   k_pk_bin        binned  (f1 conj f2 - S C(k)) / W^2 * Yhat_lm(k)  (field.hpp:765-852)
//   k_shell_D       delta(k)/W(k) for every (shell, mode) entry      (field.hpp:346-401)
//   k_family_A      A_f,i(k) = Yhat_f(k) delta/W / n_i
//   k_scatter_*     place k-space inputs on the compact shell / G cubes
//   k_pair_dot_cube sum over a shell of A_a(k) Qhat_b(-k)
//   k_xi_orbit_hist last inverse-FFT pass of the shot-noise correlation field fused with
//                   its radial histogram over integer n^2 = |x/dr|^2
//   k_bessel_table, k_sn_matrix   spline-evaluated j_l products summed over n^2
#pragma once

#include "hg_common.cuh"
#include "hg_fft.cuh"
#include "hg_bin.cuh"

namespace hg {

__global__ void k_axis_tables(Grid g, int axis, double *tw, double *ts) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int n = g.n[axis];
    if (i >= n) return;
    double kv = kcomp(wrap_index(i, n), g.dk[axis]);
    int w = window_index(kv, g.dk[axis]);
    tw[i] = sinc_axis(w, n);
    ts[i] = (w != 0) ? sin(HG_PI * (double)w / (double)n) : 0.0;
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
        int nz = lo.z + (int)(idx % cnt.z);
        int ny = lo.y + (int)((idx / cnt.z) % cnt.y);
        int nx = lo.x + (int)(idx / ((long long)cnt.z * cnt.y));
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

// out[i][j] = sum_{e in shell i} A[e] * Q[j](-n_e), Q the compact cubes of a chain family;
// one block per (i, j); deterministic.
template <typename T>
__global__ void k_pair_dot_cube(const int *start, const ShellEnt *ent, const double2 *A, const cplx<T> *Q, int3 K,
                                int3 M, int3 s, int ns_j, double2 *out) {
    int i = blockIdx.x, j = blockIdx.y;
    __shared__ double red[2][32];
    const long long vol = (long long)K.x * K.y * K.z;
    const cplx<T> *Qj = Q + (long long)j * vol;
    double sr = 0.0, si = 0.0;
    for (int e = start[i] + threadIdx.x; e < start[i + 1]; e += blockDim.x) {
        ShellEnt q = ent[e];
        long long idx = ((long long)neg_c(q.nx, M.x, s.x) * K.y + neg_c(q.ny, M.y, s.y)) * K.z + neg_c(q.nz, M.z, s.z);
        cplx<T> v = Qj[idx];
        double2 a = A[e];
        double qx = (double)v.x, qy = (double)v.y;
        sr += a.x * qx - a.y * qy;
        si += a.x * qy + a.y * qx;
    }
    for (int o = 16; o > 0; o >>= 1) {
        sr += __shfl_down_sync(0xffffffffu, sr, o);
        si += __shfl_down_sync(0xffffffffu, si, o);
    }
    int w = threadIdx.x >> 5, ln = threadIdx.x & 31;
    if (ln == 0) {
        red[0][w] = sr;
        red[1][w] = si;
    }
    __syncthreads();
    if (w == 0) {
        int nw = blockDim.x >> 5;
        sr = (ln < nw) ? red[0][ln] : 0.0;
        si = (ln < nw) ? red[1][ln] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            sr += __shfl_down_sync(0xffffffffu, sr, o);
            si += __shfl_down_sync(0xffffffffu, si, o);
        }
        if (ln == 0) out[(long long)i * ns_j + j] = make_double2(sr, si);
    }
}

// ---------------------------------------------------------------- shot-noise field
// Loader for the first inverse pass (along x) of
//   xi(x) = (1/V) sum_k (f1 conj f2 - S C(k)) / W(k)^2 e^{ikx}   (field.hpp:1116-1160)
// synthesising the k-space input from the half spectrum on the fly.
template <typename T>
struct LdXiHat {
    Spec<T> f;
    Grid g;
    AxisTabs tabs;
    int assign, wpow;
    double S_re, S_im;
    double k0_re, k0_im;  // (f1 conj f2)(k = 0) from the FP64 field integrals
    double invV;
    __device__ __forceinline__ cplx<T> operator()(long long o, int l, long long i) const {
        int ix = l;
        int iy = (int)(i / g.n[2]);
        int iz = (int)(i - (long long)iy * g.n[2]);
        zd pk2;
        if (ix == 0 && iy == 0 && iz == 0) {
            pk2 = mk<double>(k0_re, k0_im);
        } else {
            zd d = f.at(ix, iy, iz);
            pk2 = d * conjg(d);
        }
        double C = shot_tab(tabs, ix, iy, iz, assign);
        pk2 = pk2 - mk<double>(S_re * C, S_im * C);
        double wf = window_tab(tabs, ix, iy, iz, wpow);
        double w2 = wf * wf;
        return mk<T>((T)(invV * (pk2.x / w2)), (T)(invV * (pk2.y / w2)));
    }
};

// One product of reduced harmonics with its Wigner weight: w Yhat_l1m1 Yhat_l2m2.
struct YTerm {
    int l1, m1, l2, m2;
    double w;
};
#define HG_MAX_TERMS 24
#define HG_MAX_HIST 8
struct HistSpec {
    int nh;                      // number of histograms
    int nterm[HG_MAX_HIST];      // terms per histogram
    int parity[HG_MAX_HIST];     // (-1)^(l1+l2) of the histogram's terms
    YTerm term[HG_MAX_HIST][12];
};

// Last inverse pass (along z) over one symmetry orbit of (x, y) lines, fused with
//   T_h(n^2) += sum over the orbit and z <-> -z of xi(x) f_h(theta)
// where f_h = sum_terms w Yhat_l1m1 Yhat_l2m2 depends only on the polar angle (m1+m2 = 0),
// and n^2 = wx^2 + wy^2 + wz^2 in cell units (cubic cells).
template <typename T, int L>
__global__ void __launch_bounds__(L) k_xi_orbit_hist(const cplx<T> *xi, const int *orbit_lines, const int *orbit_n2xy,
                                                    int n_orbits, const cplx<T> *tw, HistSpec hs, long long n2dim,
                                                    double *hist) {
    constexpr int B = 8;
    constexpr int LP = L + 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx<T> *s = reinterpret_cast<cplx<T> *>(smem_raw);
    const int orb = blockIdx.x;
    const int *lines = orbit_lines + 8 * orb;
    for (int e = threadIdx.x; e < B * L; e += L) {
        int b = e / L, z = e - b * L;
        int line = lines[b];
        s[b * LP + z] = (line >= 0) ? xi[(long long)line * L + z] : mk<T>(0, 0);
    }
    __syncthreads();
    smem_fft<T, L, +1, L>(s, LP, B, tw);
    const int n2xy = orbit_n2xy[orb];
    const double rho = sqrt((double)n2xy);
    for (int iz = threadIdx.x; iz <= L / 2; iz += L) {
        int iz2 = (L - iz) % L;
        double er = 0, ei = 0, orr = 0, oi = 0;
        for (int b = 0; b < B; b++) {
            if (lines[b] < 0) continue;
            cplx<T> a = s[b * LP + iz];
            if (iz2 == iz) {
                er += (double)a.x;
                ei += (double)a.y;
            } else {
                cplx<T> c = s[b * LP + iz2];
                er += (double)a.x + (double)c.x;
                ei += (double)a.y + (double)c.y;
                orr += (double)a.x - (double)c.x;
                oi += (double)a.y - (double)c.y;
            }
        }
        int wz = wrap_index(iz, L);
        long long n2 = (long long)n2xy + (long long)wz * wz;
        for (int h = 0; h < hs.nh; h++) {
            zd f = mk<double>(0.0, 0.0);
            for (int t = 0; t < hs.nterm[h]; t++) {
                const YTerm &yt = hs.term[h][t];
                zd y1 = ylm_reduced(yt.l1, yt.m1, rho, 0.0, (double)wz);
                zd y2 = ylm_reduced(yt.l2, yt.m2, rho, 0.0, (double)wz);
                f = f + (y1 * y2) * yt.w;
            }
            zd src = (hs.parity[h] > 0) ? mk<double>(er, ei) : mk<double>(orr, oi);
            zd v = f * src;
            if (v.x != 0.0) atomicAdd(&hist[2 * ((long long)h * n2dim + n2)], v.x);
            if (v.y != 0.0) atomicAdd(&hist[2 * ((long long)h * n2dim + n2) + 1], v.y);
        }
    }
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

// out[i1][i2] = sum_n2 J1[i1][n2] J2[i2][n2] hist[n2]; one block per (i1, i2).
__global__ void k_sn_matrix(const double *J1, const double *J2, const double *hist, long long n2dim, int nk,
                            double2 *out) {
    int i1 = blockIdx.x, i2 = blockIdx.y;
    __shared__ double red[2][32];
    double sr = 0.0, si = 0.0;
    const double *a = J1 + (long long)i1 * n2dim, *b = J2 + (long long)i2 * n2dim;
    for (long long n2 = threadIdx.x; n2 < n2dim; n2 += blockDim.x) {
        double hr = hist[2 * n2], hi = hist[2 * n2 + 1];
        if (hr == 0.0 && hi == 0.0) continue;
        double jj = a[n2] * b[n2];
        sr += jj * hr;
        si += jj * hi;
    }
    for (int o = 16; o > 0; o >>= 1) {
        sr += __shfl_down_sync(0xffffffffu, sr, o);
        si += __shfl_down_sync(0xffffffffu, si, o);
    }
    int w = threadIdx.x >> 5, ln = threadIdx.x & 31;
    if (ln == 0) {
        red[0][w] = sr;
        red[1][w] = si;
    }
    __syncthreads();
    if (w == 0) {
        int nw = blockDim.x >> 5;
        sr = (ln < nw) ? red[0][ln] : 0.0;
        si = (ln < nw) ? red[1][ln] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            sr += __shfl_down_sync(0xffffffffu, sr, o);
            si += __shfl_down_sync(0xffffffffu, si, o);
        }
        if (ln == 0) out[(long long)i1 * nk + i2] = make_double2(sr, si);
    }
}

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
struct StHalf {  // keep the non-negative half of the last axis
    cplx<T> *H;
    int L, hz;
    __device__ __forceinline__ void operator()(long long o, int l, long long i, cplx<T> v) const {
        if (l < hz) H[o * hz + l] = v;
    }
};


}  // namespace hg
