// hg_engine.cu -- the estimator engine behind the C ABI in include/hitomi_gpu.h.
//
// One Engine<T> per context; T = double for the plain FP64 form, float for the chosen
// FP32 form (FP32 mesh / FFT / fields; FP64 bin sums, shell sums, scalars, shot noise).
//
// Periodic-box pipeline for one catalogue (cached until the particles change):
//   assignment (hg_assign.cuh) -> rho(x) -> r2c forward FFT (z, y, x passes) -> delta(k)
// as a half spectrum; the k = 0 mode is rebuilt from the FP64 field integral.
//
// Bispectrum signal.  The reference forms, for each k1 row and each k2, full-mesh fields
//   F_i(x) = IFFT[S_i(k) Yhat(k) delta/W] / n_i,  G(x) = IFFT[delta/W] / V
// and sums dV sum_x F1 F2 G (bispec.hpp:1097-1168).  Here the same number is computed as
//   sum_x F_a,i F_b,j G = sum_{k in shell i} A_a,i(k) Qhat_b,j(-k),
//   Qhat_b,j = FFT[F_b,j G],
// on a reduced M^3 grid: the shells only hold modes with |n_a| <= s, so F F G needs
// G only up to |n_a| <= 2s and is sampled without aliasing on any grid with M >= 4s+1.
// One chain (inverse FFT, multiply by G, forward FFT) per (family b, shell j) then gives
// the whole k1 x k2 matrix for every family a paired with b.
//
// Bispectrum shot noise.  xi(x) = IFFT[(|delta|^2 - N C)/W^2]/V is transformed on the full
// mesh; its last pass is fused with a histogram over integer n^2 = |x/dr|^2 (cubic cells),
// which turns sum_x j_l1(k1 r) j_l2(k2 r) xi Yhat1 Yhat2 into a sum over distinct radii.
#include "hitomi_gpu.h"
#include "hg_common.cuh"
#include "hg_fft.cuh"
#include "hg_assign.cuh"
#include "hg_kspace.cuh"
#include "hg_special.hpp"

#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <set>
#include <string>
#include <vector>

using namespace hg;

namespace {

struct DBuf {
    void *p = nullptr;
    size_t n = 0;
    DBuf() = default;
    DBuf(const DBuf &) = delete;
    DBuf &operator=(const DBuf &) = delete;
    ~DBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    cudaError_t ensure(size_t bytes) {
        if (bytes <= n && p) return cudaSuccess;
        release();
        cudaError_t e = cudaMalloc(&p, bytes ? bytes : 16);
        if (e == cudaSuccess) n = bytes;
        else p = nullptr;
        return e;
    }
};

template <class X>
inline X *dp(const DBuf &b) {
    return reinterpret_cast<X *>(b.p);
}

struct HgError {
    std::string msg;
};

#define HG_CK(x)                                                                                    \
    do {                                                                                            \
        cudaError_t e_ = (x);                                                                       \
        if (e_ != cudaSuccess)                                                                      \
            throw HgError{std::string(#x) + ": " + cudaGetErrorString(e_) + " (" + __FILE__ + ":" + \
                          std::to_string(__LINE__) + ")"};                                          \
    } while (0)

#define HG_REQUIRE(cond, text)                  \
    do {                                        \
        if (!(cond)) throw HgError{std::string(text)}; \
    } while (0)

inline unsigned grid1(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

int next_pow2(int v) {
    int p = 1;
    while (p < v) p <<= 1;
    return p;
}

// A family of shell fields: Yhat_lm weighting.
struct Fam {
    int l, m;
    bool operator<(const Fam &o) const { return l != o.l ? l < o.l : m < o.m; }
    bool operator==(const Fam &o) const { return l == o.l && m == o.m; }
};

}  // namespace

struct hg_ctx {
    hg_config cfg;
    std::string err;
    double last_ms = 0.0;
    long long last_launches = 0;
    virtual ~hg_ctx() {}
    virtual void set_particles(int slot, const double *base, long long n, long long stride, int pos_off, int los_off,
                               int w_off, bool on_device) = 0;
    virtual void set_profiling(bool on) = 0;
    virtual std::string kernel_stats() = 0;
    virtual void pk_box(int ell, double *pk_save, int *n_mode, double *norm) = 0;
    virtual void bk_box(int l1, int l2, int L, int ith, double *bk_save, double *sn_save, double *norm) = 0;
    virtual void zeta_box(int l1, int l2, int L, int ith, double *zeta_save, double *sn_save, double *norm) = 0;
    virtual void survey_scalars(double *alpha, double *vs, double *nbar, double *wd, double *wr) = 0;
    virtual void pk_survey(int ell, double alpha, double vs, double *pk_save, int *n_mode, double *norm) = 0;
};

namespace {

template <typename T>
struct Engine : public hg_ctx {
    using C = cplx<T>;
    Grid g;
    cudaStream_t st = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::vector<double> kbin, rbin;
    int wpow;  // window power p: NGP 1, CIC 2, TSC 3, PCS 4

    // catalogues
    struct Slot {
        DBuf raw;
        long long n = 0, stride = 0;
        int pos_off = 0, los_off = -1, w_off = -1;
        std::vector<double> host_w;  // weights (survey), for FP64 host sums
        const void *ext = nullptr;   // caller-owned device array (hg_set_particles_device)
        bool set = false;
        const unsigned char *base() const {
            return reinterpret_cast<const unsigned char *>(ext ? ext : raw.p);
        }
    } slot[2];

    // tables
    std::map<int, std::unique_ptr<DBuf>> tw;  // per line length
    DBuf tab_w[3], tab_s[3];
    AxisTabs tabs;
    DBuf lut;
    int lutn = 0;

    // assignment scratch
    DBuf cnt, off, cursor, rec, cubtmp, mass;
    // fields
    DBuf mesh;        // real density rho (box)
    DBuf H;           // half spectrum of dV (rho - nbar)
    bool dens_valid = false;
    double dens_mass = 0.0;   // sum_cells rho  (FP64)
    double delta0 = 0.0, N0 = 0.0;

    // bispectrum state
    struct ShellSet {
        bool built = false;
        int ns = 0;
        std::vector<int> start;       // [ns+1]
        std::vector<int> nmode;       // [ns]
        std::vector<ShellEnt> ent;    // sorted by shell
        int s[3] = {0, 0, 0};         // max |n_a| of any shell mode
        int M[3] = {0, 0, 0};         // reduced transform grid
        int gext[3] = {0, 0, 0};      // G cube half extent (or -1: whole axis)
        DBuf d_ent, d_start, d_scale;
    } shells;
    DBuf shD;                                   // delta/W per entry
    std::map<Fam, std::unique_ptr<DBuf>> famA;  // A_f per entry
    std::map<Fam, std::unique_ptr<DBuf>> famQ;  // QE_f [ns][ne]
    DBuf Gbuf, chain;
    bool G_valid = false;
    std::map<std::pair<Fam, Fam>, std::vector<double>> pairs;  // [ns][ns] complex, key (a, b): sum A_a,i Q_b,j

    // shot-noise state
    DBuf xi;
    std::vector<int> orbit_lines, orbit_n2xy;
    DBuf d_orbit_lines, d_orbit_n2xy;
    long long n2dim = 0;
    std::map<int, std::unique_ptr<BesselSpline>> splines;
    std::map<int, std::pair<std::unique_ptr<DBuf>, std::unique_ptr<DBuf>>> d_splines;
    DBuf hist, Jtab1, Jtab2, snmat, d_kv;

    long long launches = 0;

    // per-kernel device timing (CUDA events on the context stream) and modelled bytes
    bool profiling = false;
    struct PRecd {
        const char *name;
        cudaEvent_t a, b;
        double bytes;
    };
    std::vector<PRecd> pend;
    std::vector<cudaEvent_t> ev_pool;
    struct KAgg {
        long long launches = 0;
        double ms = 0.0, bytes = 0.0;
    };
    std::map<std::string, KAgg> kagg;
    cudaEvent_t take_ev() {
        if (!ev_pool.empty()) {
            cudaEvent_t e = ev_pool.back();
            ev_pool.pop_back();
            return e;
        }
        cudaEvent_t e;
        HG_CK(cudaEventCreate(&e));
        return e;
    }
    void kb(const char *name, double bytes) {
        launches++;
        if (!profiling) return;
        PRecd r{name, take_ev(), nullptr, bytes};
        HG_CK(cudaEventRecord(r.a, st));
        pend.push_back(r);
    }
    void ke() {
        HG_CK(cudaGetLastError());
        if (!profiling || pend.empty() || pend.back().b) return;
        pend.back().b = take_ev();
        HG_CK(cudaEventRecord(pend.back().b, st));
    }
    void prof_flush() {
        if (pend.empty()) return;
        HG_CK(cudaStreamSynchronize(st));
        for (auto &r : pend) {
            float ms = 0.f;
            if (r.b) HG_CK(cudaEventElapsedTime(&ms, r.a, r.b));
            KAgg &k = kagg[r.name];
            k.launches++;
            k.ms += ms;
            k.bytes += r.bytes;
            ev_pool.push_back(r.a);
            if (r.b) ev_pool.push_back(r.b);
        }
        pend.clear();
    }

    explicit Engine(const hg_config &c) {
        cfg = c;
        for (int a = 0; a < 3; a++) {
            HG_REQUIRE(fft_supported_length(c.n_mesh[a]), "n_mesh must be a power of two in [8, 1024] on every axis");
            HG_REQUIRE(c.boxsize[a] > 0.0, "boxsize must be > 0");
            g.n[a] = c.n_mesh[a];
            g.L[a] = c.boxsize[a];
            g.dk[a] = 2.0 * HG_PI / c.boxsize[a];
            g.dr[a] = c.boxsize[a] / double(c.n_mesh[a]);
        }
        HG_REQUIRE(c.assign >= 0 && c.assign <= 3, "assignment must be NGP, CIC, TSC or PCS");
        HG_REQUIRE(c.n_kbin >= 2 && c.kmax > c.kmin && c.kmin > 0.0, "need n_kbin >= 2 and 0 < kmin < kmax");
        HG_REQUIRE(c.n_rbin >= 2 && c.rmax > c.rmin && c.rmin > 0.0, "need n_rbin >= 2 and 0 < rmin < rmax");
        HG_REQUIRE(c.interlace == 0, "interlacing is not available in this build");
        g.volume = c.boxsize[0] * c.boxsize[1] * c.boxsize[2];
        g.ntot = (long long)c.n_mesh[0] * c.n_mesh[1] * c.n_mesh[2];
        wpow = c.assign + 1;
        // tools.hpp:118-134
        double dk = (c.kmax - c.kmin) / double(c.n_kbin - 1);
        for (int i = 0; i < c.n_kbin; i++) kbin.push_back(c.kmin + dk * double(i));
        double dr = (c.rmax - c.rmin) / double(c.n_rbin - 1);
        for (int i = 0; i < c.n_rbin; i++) rbin.push_back(c.rmin + dr * double(i));
        HG_CK(cudaSetDevice(c.device));
        HG_CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        HG_CK(cudaEventCreate(&ev0));
        HG_CK(cudaEventCreate(&ev1));
        for (int a = 0; a < 3; a++) {
            HG_CK(tab_w[a].ensure(sizeof(double) * g.n[a]));
            HG_CK(tab_s[a].ensure(sizeof(double) * g.n[a]));
            k_axis_tables<<<grid1(g.n[a], 128), 128, 0, st>>>(g, a, dp<double>(tab_w[a]), dp<double>(tab_s[a]));
            HG_CK(cudaGetLastError());
            tabs.tw[a] = dp<double>(tab_w[a]);
            tabs.ts[a] = dp<double>(tab_s[a]);
        }
        build_lut();
        HG_CK(cudaStreamSynchronize(st));
    }

    ~Engine() override {
        if (st) cudaStreamSynchronize(st);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (st) cudaStreamDestroy(st);
    }

    void set_profiling(bool on) override {
        profiling = on;
        if (on) kagg.clear();
    }
    std::string kernel_stats() override {
        std::string out;
        char line[256];
        for (auto &kv : kagg) {
            snprintf(line, sizeof(line), "%s\t%lld\t%.6f\t%.6e\n", kv.first.c_str(), kv.second.launches, kv.second.ms,
                     kv.second.bytes);
            out += line;
        }
        return out;
    }

    // ------------------------------------------------------------------ tables
    const C *twiddles(int L) {
        auto it = tw.find(L);
        if (it != tw.end()) return dp<C>(*it->second);
        std::vector<C> h(L);
        for (int m = 0; m < L; m++) {
            // exp(-2 pi i m / L) from an exactly reduced angle
            long long k = m;
            double c, s;
            if ((8LL * k) % L == 0) {
                static const double q[8][2] = {{1, 0}, {M_SQRT1_2, M_SQRT1_2}, {0, 1}, {-M_SQRT1_2, M_SQRT1_2},
                                               {-1, 0}, {-M_SQRT1_2, -M_SQRT1_2}, {0, -1}, {M_SQRT1_2, -M_SQRT1_2}};
                int o = (int)(8LL * k / L);
                c = q[o][0];
                s = q[o][1];
            } else {
                double a = 2.0 * HG_PI * (double)k / (double)L;
                if (2 * k > L) a = -2.0 * HG_PI * (double)(L - k) / (double)L;
                c = std::cos(a);
                s = std::sin(a);
            }
            h[m].x = (T)c;
            h[m].y = (T)(-s);
        }
        auto b = std::make_unique<DBuf>();
        HG_CK(b->ensure(sizeof(C) * L));
        HG_CK(cudaMemcpy(b->p, h.data(), sizeof(C) * L, cudaMemcpyHostToDevice));
        const C *p = dp<C>(*b);
        tw[L] = std::move(b);
        return p;
    }

    // field.hpp:775-837: fine bins of width 1e-4, coarse bin j takes fine i iff
    // lower_j < i 1e-4 <= upper_j.  lut[i] = up to two coarse bins.
    void build_lut() {
        const int n_temp = 100000;
        const double dk_temp = 0.0001;
        double dk_bin = kbin[1] - kbin[0];
        std::vector<int2> h(n_temp, make_int2(-1, -1));
        int last = -1;
        for (int i = 0; i < n_temp; i++) {
            double kt = double(i) * dk_temp;
            int nb = 0;
            for (int j = 0; j < cfg.n_kbin; j++) {
                double lower = (kbin[j] > dk_bin * 0.5) ? (kbin[j] - dk_bin * 0.5) : 0.0;
                double upper = kbin[j] + dk_bin * 0.5;
                if ((kt > lower) && (kt <= upper)) {
                    HG_REQUIRE(nb < 2, "a fine k bin belongs to more than two coarse bins");
                    if (nb == 0) h[i].x = j;
                    else h[i].y = j;
                    nb++;
                    last = i;
                }
            }
        }
        lutn = last + 1;
        HG_CK(lut.ensure(sizeof(int2) * std::max(lutn, 1)));
        if (lutn > 0) HG_CK(cudaMemcpy(lut.p, h.data(), sizeof(int2) * lutn, cudaMemcpyHostToDevice));
    }

    // ------------------------------------------------------------------ particles
    void set_particles(int s, const double *base, long long n, long long stride, int pos_off, int los_off,
                       int w_off, bool on_device) override {
        HG_REQUIRE(s == 0 || s == 1, "slot must be 0 (data) or 1 (randoms)");
        HG_REQUIRE(n > 0, "The number of particles should be > 0");
        HG_REQUIRE(base != nullptr, "null particle array");
        HG_REQUIRE(stride >= 24 && stride % 8 == 0, "stride_bytes must be a multiple of 8 and >= 24");
        HG_REQUIRE(pos_off >= 0 && (pos_off + 3) * 8 <= stride, "pos_off outside the record");
        HG_REQUIRE(w_off < 0 || (w_off + 1) * 8 <= stride, "w_off outside the record");
        HG_REQUIRE(los_off < 0 || (los_off + 3) * 8 <= stride, "los_off outside the record");
        Slot &S = slot[s];
        if (on_device) {
            S.ext = base;
        } else {
            S.ext = nullptr;
            HG_CK(S.raw.ensure((size_t)(n * stride)));
            HG_CK(cudaMemcpyAsync(S.raw.p, base, (size_t)(n * stride), cudaMemcpyHostToDevice, st));
        }
        S.n = n;
        S.stride = stride;
        S.pos_off = pos_off;
        S.los_off = los_off;
        S.w_off = w_off;
        S.set = true;
        HG_CK(cudaStreamSynchronize(st));
        invalidate();
    }

    void invalidate() {
        dens_valid = false;
        G_valid = false;
        famA.clear();
        famQ.clear();
        pairs.clear();
    }

    // ------------------------------------------------------------------ assignment
    AssignGeom make_geom(double shift) const {
        AssignGeom a;
        for (int q = 0; q < 3; q++) {
            a.n[q] = g.n[q];
            a.L[q] = g.L[q];
        }
        a.ntot = g.ntot;
        a.scheme = cfg.assign;
        a.periodic = (cfg.periodic || cfg.assign == HG_PCS) ? 1 : 0;
        a.shift = shift;
        const int tdef[3] = {8, 16, 32};
        for (int q = 0; q < 3; q++) {
            a.t[q] = std::min(tdef[q], g.n[q]);
            a.nt[q] = g.n[q] / a.t[q];
        }
        a.factor = 1.0 / (g.volume / double(g.ntot));
        return a;
    }

    // Assign one catalogue into the real mesh (rho); returns the FP64 in-bounds sum of rho.
    double assign_real(const PartSrc &src, const AssignGeom &ag, T *out) {
        const int ntiles = ag.nt[0] * ag.nt[1] * ag.nt[2];
        HG_CK(cnt.ensure(sizeof(unsigned) * (ntiles + 1)));
        HG_CK(off.ensure(sizeof(unsigned) * (ntiles + 1)));
        HG_CK(cursor.ensure(sizeof(unsigned) * (ntiles + 1)));
        HG_CK(mass.ensure(sizeof(double) * 2));
        HG_CK(cudaMemsetAsync(cnt.p, 0, sizeof(unsigned) * (ntiles + 1), st));
        HG_CK(cudaMemsetAsync(cursor.p, 0, sizeof(unsigned) * (ntiles + 1), st));
        HG_CK(cudaMemsetAsync(mass.p, 0, sizeof(double) * 2, st));
        kb("assign_bin_count", double(src.n) * 24.0);
        k_bin_count<<<grid1(src.n, 256), 256, 0, st>>>(src, ag, dp<unsigned>(cnt), dp<double>(mass));
        ke();
        size_t tb = 0;
        HG_CK(cub::DeviceScan::ExclusiveSum(nullptr, tb, dp<unsigned>(cnt), dp<unsigned>(off), ntiles + 1, st));
        HG_CK(cubtmp.ensure(tb));
        kb("assign_scan", double(ntiles + 1) * 8.0);
        HG_CK(cub::DeviceScan::ExclusiveSum(cubtmp.p, tb, dp<unsigned>(cnt), dp<unsigned>(off), ntiles + 1, st));
        ke();
        unsigned total = 0;
        double hm[2];
        HG_CK(cudaMemcpyAsync(&total, dp<unsigned>(off) + ntiles, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
        HG_CK(cudaMemcpyAsync(hm, mass.p, sizeof(double) * 2, cudaMemcpyDeviceToHost, st));
        HG_CK(cudaStreamSynchronize(st));
        HG_CK(rec.ensure(sizeof(PRec<T>) * std::max<size_t>(total, 1)));
        kb("assign_bin_scatter", double(src.n) * 24.0 + double(total) * sizeof(PRec<T>));
        k_bin_scatter<T><<<grid1(src.n, 256), 256, 0, st>>>(src, ag, dp<unsigned>(off), dp<unsigned>(cursor),
                                                            dp<PRec<T>>(rec));
        ke();
        size_t smem = sizeof(T) * ag.t[0] * ag.t[1] * ag.t[2];
        HG_CK(cudaFuncSetAttribute(k_tile_accum<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kb("assign_tile_accum", double(total) * sizeof(PRec<T>) + double(g.ntot) * sizeof(T));
        k_tile_accum<T, false><<<ntiles, 256, smem, st>>>(dp<PRec<T>>(rec), dp<unsigned>(off), ag, out, nullptr);
        ke();
        return hm[0];
    }

    template <int DIR, class LD, class ST>
    void pass(int L, LD ld, ST stt, long long outer, long long inner, const char *name = "fft_pass",
              double bytes = -1.0) {
        PassGeom pg{outer, inner};
        if (bytes < 0) bytes = 2.0 * double(outer) * L * inner * sizeof(C);
        const C *twp = twiddles(L);
        kb(name, bytes);
        HG_CK((launch_fft_pass<T, DIR>(L, ld, stt, pg, twp, st)));
        ke();
    }

    // In-place 3-D c2c transform of a batch of nb arrays [nb][M0][M1][M2].
    template <int DIR>
    void fft3(C *p, long long nb, const int *M, const char *name) {
        pass<DIR>(M[2], LdArr<T>{p, M[2], 1}, StArr<T>{p, M[2], 1}, nb * M[0] * M[1], 1, name);
        pass<DIR>(M[1], LdArr<T>{p, M[1], M[2]}, StArr<T>{p, M[1], M[2]}, nb * M[0], M[2], name);
        pass<DIR>(M[0], LdArr<T>{p, M[0], (long long)M[1] * M[2]}, StArr<T>{p, M[0], (long long)M[1] * M[2]}, nb,
                  (long long)M[1] * M[2], name);
    }

    // Box density contrast, forward transformed: H = FFT[dV (rho - N/V)] (half spectrum).
    void box_density() {
        if (dens_valid) return;
        Slot &S = slot[0];
        HG_REQUIRE(S.set, "no particles: call hg_set_particles(ctx, 0, ...) first");
        AssignGeom ag = make_geom(0.0);
        PartSrc src{S.base(), S.n, S.stride, S.pos_off, -1, nullptr, 1.0};
        HG_CK(mesh.ensure(sizeof(T) * g.ntot));
        dens_mass = assign_real(src, ag, dp<T>(mesh));
        const int hz = g.n[2] / 2 + 1;
        HG_CK(H.ensure(sizeof(C) * (size_t)g.n[0] * g.n[1] * hz));
        const double dV = g.volume / double(g.ntot);
        const double nbar = double(S.n) / g.volume;  // field.hpp:521
        pass<-1>(g.n[2], LdMeshDelta<T>{dp<T>(mesh), g.n[2], (T)nbar, (T)dV}, StHalf<T>{dp<C>(H), g.n[2], hz},
                 (long long)g.n[0] * g.n[1], 1, "fft_density_r2c_z",
                 double(g.ntot) * sizeof(T) + double(g.n[0]) * g.n[1] * hz * sizeof(C));
        pass<-1>(g.n[1], LdArr<T>{dp<C>(H), g.n[1], hz}, StArr<T>{dp<C>(H), g.n[1], hz}, g.n[0], hz, "fft_density_yx");
        pass<-1>(g.n[0], LdArr<T>{dp<C>(H), g.n[0], (long long)g.n[1] * hz},
                 StArr<T>{dp<C>(H), g.n[0], (long long)g.n[1] * hz}, 1, (long long)g.n[1] * hz, "fft_density_yx");
        // k = 0 from the FP64 integral: sum_c (rho_c - nbar) dV
        delta0 = (dens_mass - nbar * double(g.ntot)) * dV;
        N0 = dens_mass * dV;
        C z0;
        z0.x = (T)delta0;
        z0.y = (T)0;
        HG_CK(cudaMemcpyAsync(H.p, &z0, sizeof(C), cudaMemcpyHostToDevice, st));
        HG_CK(cudaStreamSynchronize(st));
        dens_valid = true;
    }

    Spec<T> half_spec() const { return Spec<T>{dp<C>(H), g.n[0], g.n[1], g.n[2], 1}; }

    // ------------------------------------------------------------------ P binning
    // Averages over each k bin of  (f conj f - S C(k)) / W^2 * Yhat_lm(k)  for a list of (l, m)
    // (TwoPointStatisticsClass::calcPowerSpectrum, field.hpp:765-852).  avg: [nbin][nlm] complex.
    void pk_bin(const std::vector<LM> &lm, double S_re, double S_im, std::vector<double> &avg,
                std::vector<unsigned long long> &nm) {
        const int nbin = cfg.n_kbin;
        HG_REQUIRE((int)lm.size() <= HG_MAX_LM, "too many multipoles in one binning call");
        LMList L;
        L.n = (int)lm.size();
        for (int q = 0; q < L.n; q++) L.lm[q] = lm[q];
        int3 lo, cn;
        int c[3];
        for (int a = 0; a < 3; a++) {
            double kedge = double(lutn) * 0.0001;
            c[a] = (int)std::floor(kedge / g.dk[a]) + 1;
        }
        auto rng = [&](int a, int &l0, int &cnt_) {
            int lo_ = std::max(-c[a], -g.n[a] / 2);
            int hi_ = std::min(c[a], g.n[a] / 2 - 1);
            l0 = lo_;
            cnt_ = hi_ - lo_ + 1;
        };
        rng(0, lo.x, cn.x);
        rng(1, lo.y, cn.y);
        rng(2, lo.z, cn.z);
        DBuf acc, cnt_d;
        HG_CK(acc.ensure(sizeof(double) * 2 * nbin * L.n));
        HG_CK(cnt_d.ensure(sizeof(unsigned long long) * nbin));
        HG_CK(cudaMemsetAsync(acc.p, 0, sizeof(double) * 2 * nbin * L.n, st));
        HG_CK(cudaMemsetAsync(cnt_d.p, 0, sizeof(unsigned long long) * nbin, st));
        size_t smem = sizeof(double) * 2 * nbin * L.n + sizeof(unsigned long long) * nbin;
        HG_CK(cudaFuncSetAttribute(k_pk_bin<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        long long total = (long long)cn.x * cn.y * cn.z;
        unsigned blocks = (unsigned)std::min<long long>(grid1(total, 256), 148 * 8);
        kb("pk_bin", double(total) * sizeof(C));
        k_pk_bin<T><<<blocks, 256, smem, st>>>(half_spec(), half_spec(), g, tabs, lo, cn, dp<int2>(lut), lutn, nbin, L,
                                               S_re, S_im, cfg.assign, wpow, dp<double>(acc),
                                               dp<unsigned long long>(cnt_d), 0, 0.0, 0.0);
        ke();
        std::vector<double> a(2 * nbin * L.n);
        nm.assign(nbin, 0);
        HG_CK(cudaMemcpyAsync(a.data(), acc.p, sizeof(double) * a.size(), cudaMemcpyDeviceToHost, st));
        HG_CK(cudaMemcpyAsync(nm.data(), cnt_d.p, sizeof(unsigned long long) * nbin, cudaMemcpyDeviceToHost, st));
        HG_CK(cudaStreamSynchronize(st));
        avg.assign(2 * nbin * L.n, 0.0);
        for (int j = 0; j < nbin; j++)
            for (int q = 0; q < L.n; q++) {
                if (nm[j] != 0) {
                    avg[2 * (j * L.n + q)] = a[2 * (j * L.n + q)] / double(nm[j]);
                    avg[2 * (j * L.n + q) + 1] = a[2 * (j * L.n + q) + 1] / double(nm[j]);
                }
            }
    }

    void begin() {
        launches = 0;
        HG_CK(cudaEventRecord(ev0, st));
    }
    void end() {
        prof_flush();
        HG_CK(cudaEventRecord(ev1, st));
        HG_CK(cudaEventSynchronize(ev1));
        float ms = 0.f;
        HG_CK(cudaEventElapsedTime(&ms, ev0, ev1));
        last_ms = ms;
        last_launches = launches;
    }

    // powerspec.hpp:273-332
    void pk_box(int ell, double *pk_save, int *n_mode, double *norm) override {
        HG_REQUIRE(ell >= 0, "ell must be >= 0");
        begin();
        box_density();
        std::vector<double> avg;
        std::vector<unsigned long long> nm;
        pk_bin({LM{ell, 0}}, double(slot[0].n), 0.0, avg, nm);
        for (int i = 0; i < cfg.n_kbin; i++) {
            pk_save[2 * i] = double(2 * ell + 1) * avg[2 * i];
            pk_save[2 * i + 1] = double(2 * ell + 1) * avg[2 * i + 1];
            if (n_mode) n_mode[i] = (int)nm[i];
        }
        if (norm) *norm = g.volume / double(slot[0].n) / double(slot[0].n);
        end();
    }

    // ------------------------------------------------------------------ shells
    void build_shells() {
        if (shells.built) return;
        ShellSet &S = shells;
        S.ns = cfg.n_kbin;
        double dk_in = kbin[1] - kbin[0];  // bispec.hpp:1144
        double upper_max = kbin[S.ns - 1] + dk_in * 0.5;
        for (int a = 0; a < 3; a++) S.s[a] = std::min((int)std::floor(upper_max / g.dk[a]) + 1, g.n[a] / 2);
        std::vector<std::vector<ShellEnt>> per(S.ns);
        for (int nx = -S.s[0]; nx <= S.s[0]; nx++) {
            if (nx >= g.n[0] / 2) continue;
            for (int ny = -S.s[1]; ny <= S.s[1]; ny++) {
                if (ny >= g.n[1] / 2) continue;
                for (int nz = -S.s[2]; nz <= S.s[2]; nz++) {
                    if (nz >= g.n[2] / 2) continue;
                    double kmag = kmag_exact_host(kcomp(nx, g.dk[0]), kcomp(ny, g.dk[1]), kcomp(nz, g.dk[2]));
                    for (int i = 0; i < S.ns; i++) {
                        // field.hpp:368-373
                        double lower = (kbin[i] > dk_in * 0.5) ? (kbin[i] - dk_in * 0.5) : 0.0;
                        double upper = kbin[i] + dk_in * 0.5;
                        if ((kmag > lower) && (kmag <= upper)) per[i].push_back(ShellEnt{nx, ny, nz, i});
                    }
                }
            }
        }
        S.start.assign(S.ns + 1, 0);
        S.nmode.assign(S.ns, 0);
        S.ent.clear();
        int smax[3] = {0, 0, 0};
        for (int i = 0; i < S.ns; i++) {
            S.start[i] = (int)S.ent.size();
            S.nmode[i] = (int)per[i].size();
            for (auto &e : per[i]) {
                S.ent.push_back(e);
                smax[0] = std::max(smax[0], std::abs(e.nx));
                smax[1] = std::max(smax[1], std::abs(e.ny));
                smax[2] = std::max(smax[2], std::abs(e.nz));
            }
        }
        S.start[S.ns] = (int)S.ent.size();
        for (int a = 0; a < 3; a++) {
            S.s[a] = smax[a];
            int need = 4 * smax[a] + 1;
            int m = std::max(8, next_pow2(need));
            if (m >= g.n[a]) {
                S.M[a] = g.n[a];
                S.gext[a] = -1;
            } else {
                S.M[a] = m;
                S.gext[a] = 2 * smax[a];
            }
        }
        HG_CK(S.d_ent.ensure(sizeof(ShellEnt) * std::max<size_t>(S.ent.size(), 1)));
        if (!S.ent.empty())
            HG_CK(cudaMemcpy(S.d_ent.p, S.ent.data(), sizeof(ShellEnt) * S.ent.size(), cudaMemcpyHostToDevice));
        HG_CK(S.d_start.ensure(sizeof(int) * (S.ns + 1)));
        HG_CK(cudaMemcpy(S.d_start.p, S.start.data(), sizeof(int) * (S.ns + 1), cudaMemcpyHostToDevice));
        std::vector<double> inv(S.ns);
        for (int i = 0; i < S.ns; i++) inv[i] = S.nmode[i] ? 1.0 / double(S.nmode[i]) : 0.0;
        HG_CK(S.d_scale.ensure(sizeof(double) * S.ns));
        HG_CK(cudaMemcpy(S.d_scale.p, inv.data(), sizeof(double) * S.ns, cudaMemcpyHostToDevice));
        S.built = true;
    }

    long long n_ent() const { return (long long)shells.ent.size(); }

    const double2 *family_A(const Fam &f) {
        auto it = famA.find(f);
        if (it != famA.end()) return dp<double2>(*it->second);
        auto b = std::make_unique<DBuf>();
        HG_CK(b->ensure(sizeof(double2) * std::max<long long>(n_ent(), 1)));
        if (n_ent() > 0) {
            kb("shell_family_A", double(n_ent()) * 48.0);
            k_family_A<<<grid1(n_ent(), 256), 256, 0, st>>>(dp<ShellEnt>(shells.d_ent), n_ent(), g, f.l, f.m,
                                                            dp<double2>(shD), dp<double>(shells.d_scale),
                                                            dp<double2>(*b));
            ke();
        }
        const double2 *p = dp<double2>(*b);
        famA[f] = std::move(b);
        return p;
    }

    void ensure_G() {
        if (G_valid) return;
        const ShellSet &S = shells;
        long long vol = (long long)S.M[0] * S.M[1] * S.M[2];
        HG_CK(Gbuf.ensure(sizeof(C) * vol));
        HG_CK(cudaMemsetAsync(Gbuf.p, 0, sizeof(C) * vol, st));
        int3 lo, cn;
        int *lop[3] = {&lo.x, &lo.y, &lo.z};
        int *cnp[3] = {&cn.x, &cn.y, &cn.z};
        for (int a = 0; a < 3; a++) {
            if (S.gext[a] < 0) {
                *lop[a] = -g.n[a] / 2;
                *cnp[a] = g.n[a];
            } else {
                *lop[a] = -S.gext[a];
                *cnp[a] = 2 * S.gext[a] + 1;
            }
        }
        long long total = (long long)cn.x * cn.y * cn.z;
        unsigned blocks = (unsigned)std::min<long long>(grid1(total, 256), 148 * 16);
        kb("scatter_G", double(total) * (sizeof(C) * 2));
        k_scatter_G<T><<<blocks, 256, 0, st>>>(half_spec(), g, tabs, wpow, lo, cn,
                                               make_int3(S.M[0], S.M[1], S.M[2]), delta0, 0.0, dp<C>(Gbuf));
        ke();
        fft3<+1>(dp<C>(Gbuf), 1, S.M, "fft_G_inv");
        G_valid = true;
    }

    // QE_b[j][e] = Qhat_b,j(-n_e),  Qhat_b,j = FFT[IFFT[A_b,j] * G] on the reduced grid.
    const double2 *family_Q(const Fam &b) {
        auto it = famQ.find(b);
        if (it != famQ.end()) return dp<double2>(*it->second);
        const ShellSet &S = shells;
        ensure_G();
        const double2 *A = family_A(b);
        long long vol = (long long)S.M[0] * S.M[1] * S.M[2];
        HG_CK(chain.ensure(sizeof(C) * vol * S.ns));
        HG_CK(cudaMemsetAsync(chain.p, 0, sizeof(C) * vol * S.ns, st));
        int3 M3 = make_int3(S.M[0], S.M[1], S.M[2]);
        kb("scatter_entries", double(n_ent()) * (16.0 + sizeof(C)));
        k_scatter_entries<T><<<grid1(n_ent(), 256), 256, 0, st>>>(dp<ShellEnt>(shells.d_ent), n_ent(), A, M3,
                                                                  dp<C>(chain));
        ke();
        fft3<+1>(dp<C>(chain), S.ns, S.M, "fft_chain_inv");
        // forward: first pass multiplies by G
        C *p = dp<C>(chain);
        pass<-1>(S.M[2], LdMulG<T>{p, dp<C>(Gbuf), S.M[2], (long long)S.M[0] * S.M[1]}, StArr<T>{p, S.M[2], 1},
                 (long long)S.ns * S.M[0] * S.M[1], 1, "fft_chain_fwd_mulG");
        pass<-1>(S.M[1], LdArr<T>{p, S.M[1], S.M[2]}, StArr<T>{p, S.M[1], S.M[2]}, (long long)S.ns * S.M[0], S.M[2],
                 "fft_chain_fwd");
        pass<-1>(S.M[0], LdArr<T>{p, S.M[0], (long long)S.M[1] * S.M[2]},
                 StArr<T>{p, S.M[0], (long long)S.M[1] * S.M[2]}, S.ns, (long long)S.M[1] * S.M[2], "fft_chain_fwd");
        auto q = std::make_unique<DBuf>();
        HG_CK(q->ensure(sizeof(double2) * std::max<long long>(n_ent(), 1) * S.ns));
        dim3 gr(grid1(n_ent(), 256), S.ns);
        kb("extract_neg", double(n_ent()) * S.ns * (16.0 + sizeof(C)));
        k_extract_neg<T><<<gr, 256, 0, st>>>(dp<ShellEnt>(shells.d_ent), n_ent(), S.ns, M3, p, dp<double2>(*q));
        ke();
        const double2 *r = dp<double2>(*q);
        famQ[b] = std::move(q);
        return r;
    }

    // pair matrix P[i][j] = sum_{e in shell i} A_a[e] QE_b[j][e]  (complex, [ns][ns])
    const std::vector<double> &pair_matrix(const Fam &a, const Fam &b) {
        auto key = std::make_pair(a, b);
        auto it = pairs.find(key);
        if (it != pairs.end()) return it->second;
        const ShellSet &S = shells;
        const double2 *A = family_A(a);
        const double2 *Q = family_Q(b);
        DBuf out;
        HG_CK(out.ensure(sizeof(double2) * S.ns * S.ns));
        dim3 gr(S.ns, S.ns);
        kb("pair_dot", double(n_ent()) * (S.ns + 1) * 16.0);
        k_pair_dot<<<gr, 256, 0, st>>>(dp<int>(shells.d_start), S.ns, A, Q, n_ent(), S.ns, dp<double2>(out));
        ke();
        std::vector<double> h(2 * S.ns * S.ns);
        HG_CK(cudaMemcpyAsync(h.data(), out.p, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, st));
        HG_CK(cudaStreamSynchronize(st));
        pairs[key] = h;
        return pairs[key];
    }

    // sum_x F_a,i F_b,j G  (without dV) for all (i, j): uses a chain on b, or on a transposed.
    std::vector<double> triple_sum(const Fam &a, const Fam &b) {
        const int ns = shells.ns;
        std::vector<double> r(2 * ns * ns);
        bool use_b = famQ.count(b) || !famQ.count(a);
        if (use_b) {
            const auto &P = pair_matrix(a, b);
            r = P;
        } else {
            const auto &P = pair_matrix(b, a);
            for (int i = 0; i < ns; i++)
                for (int j = 0; j < ns; j++) {
                    r[2 * (i * ns + j)] = P[2 * (j * ns + i)];
                    r[2 * (i * ns + j) + 1] = P[2 * (j * ns + i) + 1];
                }
        }
        return r;
    }

    void prepare_shells() {
        box_density();
        build_shells();
        HG_REQUIRE(n_ent() > 0, "no Fourier modes fall inside the k shells");
        if (!shD.p || shD.n < sizeof(double2) * n_ent() || famA.empty()) {
            HG_CK(shD.ensure(sizeof(double2) * n_ent()));
            kb("shell_D", double(n_ent()) * (16.0 + sizeof(C)));
            k_shell_D<T><<<grid1(n_ent(), 256), 256, 0, st>>>(dp<ShellEnt>(shells.d_ent), n_ent(), half_spec(), g,
                                                              tabs, wpow, dp<double2>(shD));
            ke();
        }
    }

    // ------------------------------------------------------------------ shot noise (xi)
    void build_orbits() {
        if (!orbit_lines.empty()) return;
        const int nx = g.n[0], ny = g.n[1];
        const bool swap = (nx == ny);
        for (int wx = 0; wx <= nx / 2; wx++)
            for (int wy = 0; wy <= ny / 2; wy++) {
                if (swap && wy > wx) continue;
                std::set<int> ls;
                int cand[8][2] = {{wx, wy}, {-wx, wy}, {wx, -wy}, {-wx, -wy}, {wy, wx}, {-wy, wx}, {wy, -wx}, {-wy, -wx}};
                int nc = swap ? 8 : 4;
                for (int q = 0; q < nc; q++) {
                    int ix = ((cand[q][0] % nx) + nx) % nx, iy = ((cand[q][1] % ny) + ny) % ny;
                    ls.insert(ix * ny + iy);
                }
                int k = 0;
                for (int l : ls) {
                    orbit_lines.push_back(l);
                    k++;
                }
                for (; k < 8; k++) orbit_lines.push_back(-1);
                orbit_n2xy.push_back(wx * wx + wy * wy);
            }
        HG_CK(d_orbit_lines.ensure(sizeof(int) * orbit_lines.size()));
        HG_CK(cudaMemcpy(d_orbit_lines.p, orbit_lines.data(), sizeof(int) * orbit_lines.size(), cudaMemcpyHostToDevice));
        HG_CK(d_orbit_n2xy.ensure(sizeof(int) * orbit_n2xy.size()));
        HG_CK(cudaMemcpy(d_orbit_n2xy.p, orbit_n2xy.data(), sizeof(int) * orbit_n2xy.size(), cudaMemcpyHostToDevice));
        n2dim = 0;
        for (int a = 0; a < 3; a++) n2dim += (long long)(g.n[a] / 2) * (g.n[a] / 2);
        n2dim += 1;
    }

    // hist[h][n2] = sum over cells with |x/dr|^2 = n2 of xi(x) f_h(x_hat)
    void xi_histograms(const HistSpec &hs, double S) {
        HG_REQUIRE(std::fabs(g.dr[0] - g.dr[1]) <= 1e-12 * g.dr[0] && std::fabs(g.dr[0] - g.dr[2]) <= 1e-12 * g.dr[0],
                   "bispectrum / 3PCF shot noise needs equal cell sizes on all axes");
        build_orbits();
        HG_CK(xi.ensure(sizeof(C) * g.ntot));
        const double invV = 1.0 / g.volume;  // field.hpp:1122
        LdXiHat<T> ld{half_spec(), g, tabs, cfg.assign, wpow, S, 0.0, delta0 * N0, 0.0, invV};
        long long yz = (long long)g.n[1] * g.n[2];
        pass<+1>(g.n[0], ld, StArr<T>{dp<C>(xi), g.n[0], yz}, 1, yz, "fft_xi_x_synth",
                 double(g.ntot) * sizeof(C) * 1.5);
        pass<+1>(g.n[1], LdArr<T>{dp<C>(xi), g.n[1], g.n[2]}, StArr<T>{dp<C>(xi), g.n[1], g.n[2]}, g.n[0], g.n[2],
                 "fft_xi_y");
        HG_CK(hist.ensure(sizeof(double) * 2 * n2dim * hs.nh));
        HG_CK(cudaMemsetAsync(hist.p, 0, sizeof(double) * 2 * n2dim * hs.nh, st));
        int n_orb = (int)orbit_n2xy.size();
        launch_orbit(g.n[2], hs, n_orb);
    }

    template <int L>
    void launch_orbit_L(const HistSpec &hs, int n_orb) {
        size_t smem = sizeof(C) * 8 * (L + 1);
        HG_CK(cudaFuncSetAttribute(k_xi_orbit_hist<T, L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kb("xi_orbit_hist", double(g.ntot) * sizeof(C));
        k_xi_orbit_hist<T, L><<<n_orb, L, smem, st>>>(dp<C>(xi), dp<int>(d_orbit_lines), dp<int>(d_orbit_n2xy),
                                                     n_orb, twiddles(L), hs, n2dim, dp<double>(hist));
        ke();
    }
    void launch_orbit(int L, const HistSpec &hs, int n_orb) {
        switch (L) {
            case 8: launch_orbit_L<8>(hs, n_orb); break;
            case 16: launch_orbit_L<16>(hs, n_orb); break;
            case 32: launch_orbit_L<32>(hs, n_orb); break;
            case 64: launch_orbit_L<64>(hs, n_orb); break;
            case 128: launch_orbit_L<128>(hs, n_orb); break;
            case 256: launch_orbit_L<256>(hs, n_orb); break;
            case 512: launch_orbit_L<512>(hs, n_orb); break;
            case 1024: launch_orbit_L<1024>(hs, n_orb); break;
            default: throw HgError{"unsupported n_mesh_z"};
        }
    }

    const BesselSpline &spline(int l) {
        auto it = splines.find(l);
        if (it != splines.end()) return *it->second;
        auto s = std::make_unique<BesselSpline>();
        s->build(l);
        auto dy = std::make_unique<DBuf>(), dc = std::make_unique<DBuf>();
        HG_CK(dy->ensure(sizeof(double) * s->n));
        HG_CK(dc->ensure(sizeof(double) * s->n));
        HG_CK(cudaMemcpy(dy->p, s->y.data(), sizeof(double) * s->n, cudaMemcpyHostToDevice));
        HG_CK(cudaMemcpy(dc->p, s->c.data(), sizeof(double) * s->n, cudaMemcpyHostToDevice));
        d_splines[l] = std::make_pair(std::move(dy), std::move(dc));
        const BesselSpline &r = *s;
        splines[l] = std::move(s);
        return r;
    }

    // J[i][n2] = j_l(kv[i] * dr sqrt(n2))
    void bessel_table(int l, const std::vector<double> &kv, DBuf &J) {
        const BesselSpline &s = spline(l);
        auto &sp = d_splines[l];
        HG_CK(d_kv.ensure(sizeof(double) * kv.size()));
        HG_CK(cudaMemcpyAsync(d_kv.p, kv.data(), sizeof(double) * kv.size(), cudaMemcpyHostToDevice, st));
        HG_CK(J.ensure(sizeof(double) * kv.size() * n2dim));
        long long tot = (long long)kv.size() * n2dim;
        kb("bessel_table", double(tot) * 8.0);
        k_bessel_table<<<grid1(tot, 256), 256, 0, st>>>(dp<double>(*sp.first), dp<double>(*sp.second),
                                                        s.n, s.xmin, s.dx, dp<double>(d_kv), (int)kv.size(), g.dr[0],
                                                        n2dim, dp<double>(J));
        ke();
        HG_CK(cudaStreamSynchronize(st));
    }

    // ------------------------------------------------------------------ bispectrum (box)
    // bispec.hpp:877-1203 for all k1 rows at once.
    void bk_box(int l1, int l2, int L, int ith, double *bk_save, double *sn_save, double *norm) override {
        HG_REQUIRE(l1 >= 0 && l2 >= 0 && L >= 0, "ell1, ell2, ELL must be >= 0");
        double w000 = wigner3j(l1, l2, L, 0, 0, 0);
        HG_REQUIRE(std::fabs(w000) >= 1.0e-10, "This multipole combination is not allowed: wigner_3j(ell1, ell2, ELL, 0,0,0) == 0");
        HG_REQUIRE(ith >= -1 && ith < cfg.n_kbin, "ith_kbin out of range");
        begin();
        prepare_shells();
        const int ns = shells.ns;
        const double Np = double(slot[0].n);
        const double dV = g.volume / double(g.ntot);
        const double red = double(g.ntot) / (double(shells.M[0]) * shells.M[1] * shells.M[2]);
        // (m1, m2) combinations with M = 0 (bispec.hpp:1123-1133)
        struct Combo {
            int m1, m2;
            double w;
        };
        std::vector<Combo> combos;
        for (int m1 = -l1; m1 <= l1; m1++)
            for (int m2 = -l2; m2 <= l2; m2++) {
                double w = w000 * wigner3j(l1, l2, L, m1, m2, 0);
                w *= double(2 * L + 1) * double(2 * l1 + 1) * double(2 * l2 + 1);
                if (std::fabs(w) < 1.0e-10) continue;
                combos.push_back({m1, m2, w});
            }
        std::vector<double> B(2 * ns * ns, 0.0), SN(2 * ns * ns, 0.0);
        for (const auto &c : combos) {
            std::vector<double> t = triple_sum(Fam{l1, c.m1}, Fam{l2, c.m2});
            for (int q = 0; q < 2 * ns * ns; q++) B[q] += c.w * (dV * red * t[q]);
        }
        // shot noise, bispec.hpp:909-1078
        std::vector<LM> lms;
        for (const auto &c : combos) {
            if (l2 == 0) lms.push_back(LM{l1, c.m1});
            if (l1 == 0) lms.push_back(LM{l2, c.m2});
        }
        std::vector<double> avg;
        std::vector<unsigned long long> nm;
        if (!lms.empty()) pk_bin(lms, Np, 0.0, avg, nm);
        int q = 0;
        for (const auto &c : combos) {
            for (int i1 = 0; i1 < ns; i1++)
                for (int i2 = 0; i2 < ns; i2++) {
                    double sr = 0.0, si = 0.0;
                    if (l1 == 0 && l2 == 0) sr += c.w * Np;
                    int qq = q;
                    if (l2 == 0) {
                        sr += c.w * avg[2 * (i1 * (int)lms.size() + qq)];
                        si += c.w * avg[2 * (i1 * (int)lms.size() + qq) + 1];
                        qq++;
                    }
                    if (l1 == 0) {
                        sr += c.w * avg[2 * (i2 * (int)lms.size() + qq)];
                        si += c.w * avg[2 * (i2 * (int)lms.size() + qq) + 1];
                    }
                    SN[2 * (i1 * ns + i2)] += sr;
                    SN[2 * (i1 * ns + i2) + 1] += si;
                }
            q += (l2 == 0) + (l1 == 0);
        }
        // xi term: hist of xi * sum_combos w Yhat_l1m1 Yhat_l2m2, then j_l1 j_l2 sums
        HistSpec hs;
        memset(&hs, 0, sizeof(hs));
        hs.nh = 1;
        hs.parity[0] = ((l1 + l2) % 2 == 0) ? 1 : -1;
        HG_REQUIRE(combos.size() <= 12, "too many (m1, m2) terms");
        for (const auto &c : combos) hs.term[0][hs.nterm[0]++] = YTerm{l1, c.m1, l2, c.m2, c.w};
        xi_histograms(hs, Np);
        bessel_table(l1, kbin, Jtab1);
        bessel_table(l2, kbin, Jtab2);
        HG_CK(snmat.ensure(sizeof(double2) * ns * ns));
        kb("sn_matrix", double(ns) * ns * n2dim * 24.0);
        k_sn_matrix<<<dim3(ns, ns), 256, 0, st>>>(dp<double>(Jtab1), dp<double>(Jtab2), dp<double>(hist), n2dim, ns,
                                                 dp<double2>(snmat));
        ke();
        std::vector<double> sd(2 * ns * ns);
        HG_CK(cudaMemcpyAsync(sd.data(), snmat.p, sizeof(double) * sd.size(), cudaMemcpyDeviceToHost, st));
        HG_CK(cudaStreamSynchronize(st));
        // * i^(l1+l2) * dV   (bispec.hpp:1053-1055)
        int p4 = (l1 + l2) % 4;
        for (int e = 0; e < ns * ns; e++) {
            double re = sd[2 * e] * dV, im = sd[2 * e + 1] * dV;
            double rr, ii;
            if (p4 == 0) { rr = re; ii = im; }
            else if (p4 == 1) { rr = -im; ii = re; }
            else if (p4 == 2) { rr = -re; ii = -im; }
            else { rr = im; ii = -re; }
            SN[2 * e] += rr;
            SN[2 * e + 1] += ii;
        }
        int r0 = (ith < 0) ? 0 : ith, r1 = (ith < 0) ? ns : ith + 1;
        for (int i1 = r0; i1 < r1; i1++)
            for (int i2 = 0; i2 < ns; i2++) {
                int o = (i1 - r0) * ns + i2;
                bk_save[2 * o] = B[2 * (i1 * ns + i2)];
                bk_save[2 * o + 1] = B[2 * (i1 * ns + i2) + 1];
                sn_save[2 * o] = SN[2 * (i1 * ns + i2)];
                sn_save[2 * o + 1] = SN[2 * (i1 * ns + i2) + 1];
            }
        if (norm) {
            double nv = g.volume / Np / Np;
            nv *= (g.volume / Np);
            *norm = nv;
        }
        end();
    }

    void zeta_box(int, int, int, int, double *, double *, double *) override {
        throw HgError{"hg_zeta_box is not available in this build"};
    }
    void survey_scalars(double *, double *, double *, double *, double *) override {
        throw HgError{"hg_survey_scalars is not available in this build"};
    }
    void pk_survey(int, double, double, double *, int *, double *) override {
        throw HgError{"hg_pk_survey is not available in this build"};
    }
};

thread_local std::string g_create_error;

}  // namespace

extern "C" {

int hg_create(hg_ctx **out, const hg_config *cfg) {
    if (!out || !cfg) return -1;
    *out = nullptr;
    try {
        if (cfg->precision == HG_FP64) *out = new Engine<double>(*cfg);
        else if (cfg->precision == HG_FP32) *out = new Engine<float>(*cfg);
        else throw HgError{"precision must be HG_FP64 or HG_FP32"};
        return 0;
    } catch (const HgError &e) {
        g_create_error = e.msg;
        return -1;
    } catch (const std::exception &e) {
        g_create_error = e.what();
        return -1;
    }
}

int hg_destroy(hg_ctx *ctx) {
    if (!ctx) return -1;
    delete ctx;
    return 0;
}

const char *hg_last_error(const hg_ctx *ctx) {
    if (!ctx) return g_create_error.c_str();
    return ctx->err.c_str();
}

#define HG_GUARD(ctx, body)                  \
    do {                                     \
        if (!(ctx)) return -1;               \
        try {                                \
            body;                            \
            (ctx)->err.clear();              \
            return 0;                        \
        } catch (const HgError &e) {         \
            (ctx)->err = e.msg;              \
            return -1;                       \
        } catch (const std::exception &e) {  \
            (ctx)->err = e.what();           \
            return -1;                       \
        }                                    \
    } while (0)

int hg_set_particles(hg_ctx *ctx, int slot, const double *base, long long n, long long stride_bytes, int pos_off,
                     int los_off, int w_off) {
    HG_GUARD(ctx, ctx->set_particles(slot, base, n, stride_bytes, pos_off, los_off, w_off, false));
}

int hg_set_particles_device(hg_ctx *ctx, int slot, const double *dev_base, long long n, long long stride_bytes,
                            int pos_off, int los_off, int w_off) {
    HG_GUARD(ctx, ctx->set_particles(slot, dev_base, n, stride_bytes, pos_off, los_off, w_off, true));
}

int hg_set_profiling(hg_ctx *ctx, int on) { HG_GUARD(ctx, ctx->set_profiling(on != 0)); }

int hg_kernel_stats(hg_ctx *ctx, char *buf, long long buflen) {
    if (!ctx || !buf || buflen <= 0) return -1;
    std::string s;
    try {
        s = ctx->kernel_stats();
    } catch (const HgError &e) {
        ctx->err = e.msg;
        return -1;
    }
    long long n = std::min<long long>((long long)s.size(), buflen - 1);
    memcpy(buf, s.data(), (size_t)n);
    buf[n] = 0;
    return 0;
}

int hg_pk_box(hg_ctx *ctx, int ell, double *pk_save, int *n_mode, double *norm) {
    if (!pk_save) return -1;
    HG_GUARD(ctx, ctx->pk_box(ell, pk_save, n_mode, norm));
}

int hg_bk_box(hg_ctx *ctx, int ell1, int ell2, int ELL, int ith_kbin, double *bk_save, double *sn_save, double *norm) {
    if (!bk_save || !sn_save) return -1;
    HG_GUARD(ctx, ctx->bk_box(ell1, ell2, ELL, ith_kbin, bk_save, sn_save, norm));
}

int hg_zeta_box(hg_ctx *ctx, int ell1, int ell2, int ELL, int ith_rbin, double *zeta_save, double *sn_save,
                double *norm) {
    if (!zeta_save || !sn_save) return -1;
    HG_GUARD(ctx, ctx->zeta_box(ell1, ell2, ELL, ith_rbin, zeta_save, sn_save, norm));
}

int hg_survey_scalars(hg_ctx *ctx, double *alpha, double *vsurvey, double *nbar, double *wsum_data,
                      double *wsum_rand) {
    HG_GUARD(ctx, ctx->survey_scalars(alpha, vsurvey, nbar, wsum_data, wsum_rand));
}

int hg_pk_survey(hg_ctx *ctx, int ell, double alpha, double vsurvey, double *pk_save, int *n_mode, double *norm) {
    if (!pk_save) return -1;
    HG_GUARD(ctx, ctx->pk_survey(ell, alpha, vsurvey, pk_save, n_mode, norm));
}

int hg_last_timing(const hg_ctx *ctx, double *device_ms, long long *kernel_launches) {
    if (!ctx) return -1;
    if (device_ms) *device_ms = ctx->last_ms;
    if (kernel_launches) *kernel_launches = ctx->last_launches;
    return 0;
}

}  // extern "C"
