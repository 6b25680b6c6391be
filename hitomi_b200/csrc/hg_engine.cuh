// hg_engine.cuh -- the estimator engine behind the C ABI in include/hitomi_gpu.h.
//
// One Engine<T> per context; T = double for the plain FP64 form, float for the chosen
// FP32 form (FP32 mesh / FFT / fields; FP64 assignment accumulators, bin sums, shell
// sums, scalars and shot-noise histograms).  Each precision is instantiated in its own
// translation unit (hg_engine_fp32.cu, hg_engine_fp64.cu); they meet only through the
// hg_ctx interface (hg_ctx.hpp).  An FP32 context whose hg_config.fp64_stages is non-zero
// owns an FP64 engine on the same stream and hands it the stages named there.
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
// One chain (hg_chain.cuh: pruned inverse FFT, multiply by G, pruned forward FFT) per
// (family b, shell j) then gives the whole k1 x k2 matrix for every family a paired with b.
//
// Bispectrum shot noise.  xi(x) = IFFT[(|delta|^2 - N C)/W^2]/V is transformed on the full
// mesh; its last pass is fused with a histogram over integer n^2 = |x/dr|^2 (equal cells,
// power-of-two z), or, on other meshes, the whole field is folded into octant cells with
// their exact |r|; either turns sum_x j_l1(k1 r) j_l2(k2 r) xi Yhat1 Yhat2 into a sum over
// distinct radii.
#include "hitomi_gpu.h"
#include "hg_ctx.hpp"
#include "hg_common.cuh"
#include "hg_fft.cuh"
#include "hg_assign.cuh"
#include "hg_kspace.cuh"
#include "hg_chain.cuh"
#include "hg_fft2.cuh"
#include "hg_special.hpp"

#include <cub/cub.cuh>

#include <exception>
#include <thread>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <set>
#include <string>
#include <tuple>
#include <vector>

using namespace hg;

namespace {

struct DBuf {
    void *p = nullptr;
    size_t n = 0;
    MemBudget *owner = nullptr;  // the context charged for this buffer
    DBuf() = default;
    DBuf(const DBuf &) = delete;
    DBuf &operator=(const DBuf &) = delete;
    ~DBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        if (p && owner) {
            std::lock_guard<std::mutex> lk(owner->m);
            owner->used -= n;
        }
        p = nullptr;
        n = 0;
        owner = nullptr;
    }
    // grows only; contents are not preserved across a growth
    cudaError_t ensure(size_t bytes) {
        if (bytes <= n && p) return cudaSuccess;
        release();
        const size_t want = bytes ? bytes : 16;
        MemBudget *b = current_budget();
        if (b) {  // reserve first, so two threads of one context cannot both pass the limit
            std::lock_guard<std::mutex> lk(b->m);
            if (b->limit && b->used + want > b->limit) {
                b->hit = true;
                return cudaErrorMemoryAllocation;
            }
            b->used += want;
        }
        cudaError_t e = cudaMalloc(&p, want);
        if (e != cudaSuccess) {
            p = nullptr;
            if (b) {
                std::lock_guard<std::mutex> lk(b->m);
                b->used -= want;
            }
            return e;
        }
        n = want;
        owner = b;
        return e;
    }
};

template <class X>
inline X *dp(const DBuf &b) {
    return reinterpret_cast<X *>(b.p);
}

#define HG_CK(x)                                                                                    \
    do {                                                                                            \
        cudaError_t e_ = (x);                                                                       \
        if (e_ != cudaSuccess)                                                                      \
            throw HgError{std::string(#x) + ": " + cudaGetErrorString(e_) + " (" + __FILE__ + ":" + \
                          std::to_string(__LINE__) + ")"};                                          \
    } while (0)

#define HG_REQUIRE(cond, text)                         \
    do {                                               \
        if (!(cond)) throw HgError{std::string(text)}; \
    } while (0)

inline unsigned grid1(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

// CTAs of `kern` (bs threads, no dynamic shared memory) that are resident on the GPU at once:
// the grid of a grid-stride kernel that runs as one wave (a grid of several waves leaves the
// last one partly empty).  Queried once per kernel.
template <class K>
inline unsigned resident_grid(K kern, int bs) {
    // one per kernel instantiation, initialised once even when contexts on several host
    // threads get here together (a function-local static)
    static const int per_sm = [&] {
        int v = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, kern, bs, 0) != cudaSuccess || v < 1) v = 1;
        return v;
    }();
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return (unsigned)(sms * per_sm);
}

int next_pow2(int v) {
    int p = 1;
    while (p < v) p <<= 1;
    return p;
}

// A family of shell fields: Yhat_lm weighting.
struct Fam {
    int l, m;
    bool operator<(const Fam &o) const { return l != o.l ? l < o.l : m < o.m; }
};

}  // namespace


namespace {

// p[0] = (re, im): a field's k = 0 value set on the stream, without a host copy and wait
template <typename T>
__global__ void k_set_k0(cplx<T> *p, T re, T im) {
    p[0] = mk<T>(re, im);
}

// element-wise precision change of a complex array (the density spectrum between the
// FP32 engine and its FP64 stages)
template <typename S, typename D>
__global__ void k_convert_spec(const cplx<S> *__restrict__ in, cplx<D> *__restrict__ out, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const cplx<S> v = in[i];
        cplx<D> w;
        w.x = (D)v.x;
        w.y = (D)v.y;
        out[i] = w;
    }
}

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
        const void *ext = nullptr;  // caller-owned device array (hg_set_particles_device)
        bool set = false;
        const unsigned char *base() const { return reinterpret_cast<const unsigned char *>(ext ? ext : raw.p); }
    } slot[2];

    // tables
    std::map<int, std::unique_ptr<DBuf>> tw;  // per line length
    DBuf tab_w[3], tab_s[3], tab_c[3];
    AxisTabs tabs;
    XiTabs xtabs;
    DBuf tab_cf[3], tab_df[3], tab_iw2[3];
    DBuf lut;
    int lutn = 0;

    // assignment scratch
    DBuf cnt, off, cursor, rec, cubtmp, mass, nch, choff, chunks;
    DBuf deflist, defcnt, cursor_back;  // particles whose stencil straddles a non-periodic edge
    static constexpr unsigned CHUNK = 2048;  // records per accumulation CTA
    // fields
    DBuf mesh;  // real density rho (box)
    DBuf H;     // half spectrum of dV (rho - nbar)
    DBuf H2;    // half spectrum of the half-cell shifted assignment (interlacing)
    bool dens_valid = false;
    // FP32 engine whose density the FP64 engine computed: that FP64 half spectrum (valid while
    // this density is), and whether H still waits for its narrowed copy.  The shot-noise
    // correlation field reads the FP64 spectrum directly; H is narrowed only when a stage of
    // this engine needs the spectrum itself (shell fields, G, the 3PCF, P binning).
    const cplx<double> *H_wide = nullptr;
    bool narrow_pending = false;
    struct PkBins {
        std::vector<double> avg;  // [nbin] complex bin averages before the (2l+1) factor
        std::vector<unsigned long long> nm;
    };
    std::map<int, PkBins> pk_cache;  // box P_l bins of the current density, by l
    double dens_mass = 0.0;  // sum_cells rho  (FP64)
    double delta0 = 0.0, N0 = 0.0;

    // binning scratch
    DBuf bin_acc, bin_cnt;
    DBuf pk_modes;             // the binning cube's in-bin modes (PkMode), built on first use
    long long n_pk_modes = -1;

    // bispectrum state (geometry: built once per context)
    struct ShellSet {
        bool built = false;
        int ns = 0;
        std::vector<int> start, nmode;
        std::vector<ShellEnt> ent;  // sorted by shell
        int s[3] = {0, 0, 0};       // max |n_a| of any shell mode; compact side K = 2s+1
        int K[3] = {0, 0, 0};
        int M[3] = {0, 0, 0};       // reduced transform grid
        int gs[3] = {0, 0, 0};      // G cube half extent (2s, or n/2 when the axis is not reduced)
        int KG[3] = {0, 0, 0};
        DBuf d_ent, d_start, d_scale;
        int nitems = 0;            // pair-sum work items (k_pair_dot_items)
        DBuf d_items, d_istart;
        // shell-extent pruning of the chains' inverse passes: per shell j, e_j,a = max |n_a|
        // of its modes (-1 for an empty shell); the B1 lines (j, cx, cy) and B2 lines (j, cx)
        // inside those extents, as indices into the full layouts
        std::vector<int> ext;       // [ns][3]
        DBuf d_ext4, d_extx;        // int4 per shell (e_x, e_y, e_z, 0); e_x per shell
        DBuf d_lines1, d_lines2;
        long long nl1 = 0, nl2 = 0;
        DBuf d_cyr1;  // [ns][Kx]: per (shell j, cx) the compact cy range of shell j's modes (B1 lines)
        // forward-pass column pruning: per cx the range of cy of the columns (cx, cy) that some
        // shell mode has (F2 rows), and the F3 lines (j, cx, cy) of those columns
        DBuf d_cyr, d_lines3;
        long long nl3 = 0;
        double disc_frac = 1.0;
    } shells;
    // The catalogue the bispectrum and 3PCF read: the box density (kind 0) or the survey's
    // D - alpha R field (kind 1).  G fields are keyed by GK = (L, M): the Yhat_LM-weighted
    // field of the survey drivers (bispec.hpp:268-283), (0, 0) for the box.
    struct SpecK {
        Spec<T> s;
        double k0r, k0i;  // FP64 value of the k = 0 mode
    };
    using GK = std::pair<int, int>;
    using FQ = std::tuple<int, int, int, int>;  // chain family (l, m) with its G key (L, M)
    // 0 box density; 1 survey D - alpha R; 2 randoms alone (window functions); 3 the
    // reconstructed box, D - alpha R of two box catalogues with the line of sight along z
    // (bispec.hpp:1426-1753): every particle's Yhat_LM(z) is 1 for M = 0 and 0 otherwise, so
    // only M = 0 terms remain and every (L, 0) field is the (0, 0) one
    int src_kind = -1;
    double src_alpha = 0.0;
    SpecK dsrc{};
    // per-catalogue bispectrum state
    DBuf shD;                                   // delta/W per entry
    std::map<Fam, std::unique_ptr<DBuf>> famA;  // A_f per entry (memory kept across catalogues)
    std::set<Fam> famA_ok;
    std::map<FQ, std::unique_ptr<DBuf>> famQ;  // Q cube per chain family and G
    std::set<FQ> famQ_ok;
    std::map<GK, std::unique_ptr<DBuf>> Gm;    // G on the reduced grid per G key
    std::set<GK> Gm_ok;
    DBuf Gc, Ac, T1, T2, pair_out;
    DBuf pair_part;  // per work item partial pair sums
    bool shD_valid = false;
    std::map<std::tuple<int, int, int, int, int, int>, std::vector<double>> pairs;  // (a, b, L, M)

    // shot-noise state
    DBuf xi;
    bool xi_valid = false;
    double xi_k0 = 0.0;  // the k = 0 product the cached box correlation field was made with
    std::vector<int> orbit_lines, orbit_n2xy;  // per orbit: 4 (line, mirror) pairs; n_x^2 + n_y^2
    DBuf d_orbit_lines, d_orbit_n2xy;
    long long n2dim = 0;  // 3 (n/2)^2 + 1 style count of integer n^2 (k space; r space on equal cells)
    // correlation-field histogram keys: integer n^2 = |x/dr|^2 on equal cells with a
    // power-of-two z axis (the orbit / line kernels), else octant cells (k_xi_fold); per key
    // the reference's |r| and the number of cells
    bool xi_general = false;
    long long nkey = 0;
    std::vector<double> key_r, key_cells;
    DBuf d_keyr;
    std::map<int, std::unique_ptr<BesselSpline>> splines;
    std::map<int, std::pair<std::unique_ptr<DBuf>, std::unique_ptr<DBuf>>> d_splines;
    std::map<int, std::unique_ptr<DBuf>> jtab_k;  // J_l[i][n2] at the k bins (geometry only)
    std::map<std::array<int, 3>, std::unique_ptr<DBuf>> hist_mp;  // per multipole (catalogue)
    std::set<std::array<int, 3>> hist_ok;
    DBuf hist_tmp, snmat, snblk, sn_part, d_kv;

    // survey state (per pair of catalogues): transformed Yhat_lm-weighted fields of two kinds,
    // SF_DELTA = n_D - alpha n_R with weights Yhat w (field.hpp:186-228) and SF_SN = n_D +
    // alpha^2 n_R with weights conj(Yhat) w^2 (field.hpp:249-284); m = 0 half spectra, m != 0
    // full ones (m < 0 as mirrors of m > 0); keyed (kind, l, m), valid for sf_alpha.
    // SF_WIN / SF_WIN_SN: the same fields of the randoms alone, n_R with weights Yhat w
    // (calcYlmWeightedDensity field.hpp:230-247) and conj(Yhat) w^2
    // (calcYlmWeightedDensityForThreePointWindowFunctionShotnoise field.hpp:286-306)
    enum { SF_DELTA = 0, SF_SN = 1, SF_WIN = 2, SF_WIN_SN = 3 };
    DBuf smesh_re, smesh_im, dmesh, psum_part, sfield_tmp;
    // both catalogues binned once per assignment offset (0, and 1/2 cell for interlacing);
    // every weighting reuses them
    struct SurveyBins {
        DBuf rec, chunks;
        unsigned total = 0, nchunks = 0;
        bool ok = false;
        bool neg = false;  // some particle has a negative coordinate (stencil_weight_bound)
    } sbins[2];
    std::map<std::array<int, 3>, std::unique_ptr<DBuf>> sfbuf;
    std::map<std::array<int, 3>, std::array<double, 2>> sfk0;
    std::set<std::array<int, 3>> sf_ok;
    double sf_alpha = 0.0;

    // 3PCF state: geometry tables (per context) and filtered fields (per catalogue)
    std::map<int, std::unique_ptr<DBuf>> jtab_r;  // J_l[j][n2] = j_l(dk r_j sqrt(n2))
    DBuf d_rv, Uz, zpart, zout;
    std::map<GK, std::unique_ptr<DBuf>> Gz;  // G on the full grid per G key
    std::set<GK> Gz_ok;
    // survey shot-noise histograms per multipole: sum_M sum_(m1,m2) w sum_{|x|^2 = n2} xi_LM Yhat1 Yhat2
    std::map<std::array<int, 3>, std::unique_ptr<DBuf>> hist_sv;
    std::set<std::array<int, 3>> hist_sv_ok;
    std::vector<int> zfine;                  // fine r index of each n2 (field.hpp:1044-1050), -1 if >= 10^4
    std::vector<std::vector<int>> zcoarse;   // coarse r bins of each fine index (field.hpp:1064-1085)
    std::vector<double> zcount;              // cells per coarse r bin
    struct ZKey {
        int l, m, r0, nr;
        bool operator<(const ZKey &o) const {
            return std::tie(l, m, r0, nr) < std::tie(o.l, o.m, o.r0, o.nr);
        }
    };
    std::map<ZKey, std::unique_ptr<DBuf>> zf;  // F_lm[r0 .. r0+nr) on the full grid
    size_t zfree0 = 0;                         // device memory available to the field cache
    std::set<ZKey> zf_ok;
    std::map<std::tuple<int, int, int, int, int, int, int>, std::vector<double>> zpairs;  // (a, b, row, L, M)

    long long launches = 0;

    // FP64 engine of the stages named in cfg.fp64_stages (FP32 form only), on this stream
    std::unique_ptr<hg_ctx> hi;
    int fp64_stages = 0;
    bool own_stream = true;

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

    explicit Engine(const hg_config &c) {
        cfg = c;
        for (int a = 0; a < 3; a++) {
            HG_REQUIRE(fft_any_length(c.n_mesh[a]) && c.n_mesh[a] % 2 == 0,
                       "n_mesh must be even, in [8, 2048] and a product of primes <= 31 on every axis");
            HG_REQUIRE(c.boxsize[a] > 0.0, "boxsize must be > 0");
            g.n[a] = c.n_mesh[a];
            g.L[a] = c.boxsize[a];
            g.dk[a] = 2.0 * HG_PI / c.boxsize[a];
            g.dr[a] = c.boxsize[a] / double(c.n_mesh[a]);
        }
        HG_REQUIRE(c.assign >= 0 && c.assign <= 3, "assignment must be NGP, CIC, TSC or PCS");
        HG_REQUIRE(c.n_kbin >= 2 && c.kmax > c.kmin && c.kmin > 0.0, "need n_kbin >= 2 and 0 < kmin < kmax");
        HG_REQUIRE(c.n_rbin >= 2 && c.rmax > c.rmin && c.rmin > 0.0, "need n_rbin >= 2 and 0 < rmin < rmax");
        g.volume = c.boxsize[0] * c.boxsize[1] * c.boxsize[2];
        g.ntot = (long long)c.n_mesh[0] * c.n_mesh[1] * c.n_mesh[2];
        HG_REQUIRE(g.ntot <= (1LL << 31), "n_mesh: at most 2^31 cells in all");
        choose_tiles();
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
        // the schemes the reference does not have use the exact window index and periodic wrap
        const int exact = (c.interlace || c.assign == HG_PCS) ? 1 : 0;
        tabs.interlace = c.interlace ? 1 : 0;
        xtabs.interlace = tabs.interlace;
        for (int a = 0; a < 3; a++) {
            HG_CK(tab_w[a].ensure(sizeof(double) * g.n[a]));
            HG_CK(tab_s[a].ensure(sizeof(double) * g.n[a]));
            HG_CK(tab_c[a].ensure(sizeof(double) * g.n[a]));
            k_axis_tables<<<grid1(g.n[a], 128), 128, 0, st>>>(g, a, exact, dp<double>(tab_w[a]), dp<double>(tab_s[a]),
                                                              dp<double>(tab_c[a]));
            HG_CK(cudaGetLastError());
            tabs.tw[a] = dp<double>(tab_w[a]);
            tabs.ts[a] = dp<double>(tab_s[a]);
            tabs.tc[a] = dp<double>(tab_c[a]);
            HG_CK(tab_cf[a].ensure(sizeof(double) * g.n[a]));
            HG_CK(tab_df[a].ensure(sizeof(double) * g.n[a]));
            HG_CK(tab_iw2[a].ensure(sizeof(double) * g.n[a]));
            k_xi_tables<<<grid1(g.n[a], 128), 128, 0, st>>>(g.n[a], tabs.tw[a], tabs.ts[a], tabs.tc[a], c.assign, wpow,
                                                            dp<double>(tab_cf[a]), dp<double>(tab_df[a]),
                                                            dp<double>(tab_iw2[a]));
            HG_CK(cudaGetLastError());
            xtabs.cf[a] = dp<double>(tab_cf[a]);
            xtabs.df[a] = dp<double>(tab_df[a]);
            xtabs.iw2[a] = dp<double>(tab_iw2[a]);
        }
        build_lut();
        HG_CK(cudaStreamSynchronize(st));
        if (sizeof(T) == 4 && c.fp64_stages != 0) {
            HG_REQUIRE((c.fp64_stages & ~(HG_STAGE_DENSITY | HG_STAGE_BK_SIGNAL | HG_STAGE_BK_SHOT)) == 0,
                       "fp64_stages holds unknown HG_STAGE_* bits");
            hg_config hc = c;
            hc.precision = HG_FP64;
            hc.fp64_stages = 0;
            hi.reset(make_engine_fp64(hc));
            hi->stage_adopt_stream(st);
            fp64_stages = c.fp64_stages;
        }
    }

    ~Engine() override {
        hi.reset();  // it runs on this engine's stream
        batch_release();
        if (st) cudaStreamSynchronize(st);
        for (auto e : ev_pool) cudaEventDestroy(e);
        for (auto &r : pend) {
            cudaEventDestroy(r.a);
            if (r.b) cudaEventDestroy(r.b);
        }
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (st && own_stream) cudaStreamDestroy(st);
    }

    // ------------------------------------------------------------------ profiling
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
    void set_profiling(bool on) override {
        profiling = on;
        if (on) kagg.clear();
        if (hi) hi->set_profiling(on);
    }
    std::string kernel_stats() override {
        prof_flush();
        std::string out;
        char line[256];
        for (auto &kv : kagg) {
            snprintf(line, sizeof(line), "%s\t%lld\t%.6f\t%.6e\n", kv.first.c_str(), kv.second.launches, kv.second.ms,
                     kv.second.bytes);
            out += line;
        }
        if (hi) {  // the FP64 stages, under their own names
            std::string h = hi->kernel_stats();
            size_t p0 = 0;
            while (p0 < h.size()) {
                size_t p1 = h.find('\n', p0);
                if (p1 == std::string::npos) p1 = h.size();
                if (p1 > p0) out += "fp64:" + h.substr(p0, p1 - p0) + "\n";
                p0 = p1 + 1;
            }
        }
        return out;
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
        check_word();
    }
    // check build: fail the call if a device-side bounds check failed (and clear the record)
    void check_word() {
#ifdef HG_CHECK
        unsigned long long w[3] = {0, 0, 0};
        HG_CK(cudaMemcpyFromSymbol(w, hg_check_word, sizeof(w)));
        if (w[0]) {
            const unsigned long long z[3] = {0, 0, 0};
            HG_CK(cudaMemcpyToSymbol(hg_check_word, z, sizeof(z)));
            throw HgError{"device bounds check failed " + std::to_string(w[0]) + " time(s); first at site " +
                          std::to_string(w[1]) + ", index " + std::to_string((long long)w[2])};
        }
#endif
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
    void set_particles(int s, const double *base, long long n, long long stride, int pos_off, int los_off, int w_off,
                       bool on_device) override {
        HG_REQUIRE(s == 0 || s == 1, "slot must be 0 (data) or 1 (randoms)");
        HG_REQUIRE(n > 0, "The number of particles should be > 0");
        HG_REQUIRE(n < (1LL << 31), "more than 2^31 - 1 particles in one catalogue");
        HG_REQUIRE(base != nullptr, "null particle array");
        HG_REQUIRE(stride >= 24 && stride % 8 == 0, "stride_bytes must be a multiple of 8 and >= 24");
        HG_REQUIRE(pos_off >= 0 && (pos_off + 3) * 8 <= stride, "pos_off outside the record");
        HG_REQUIRE(w_off < 0 || (w_off + 1) * 8 <= stride, "w_off outside the record");
        HG_REQUIRE(los_off < 0 || (los_off + 3) * 8 <= stride, "los_off outside the record");
        Slot &S = slot[s];
        wmax_cache[s] = -1.0;
        if (on_device) {
            cudaPointerAttributes at;
            HG_CK(cudaPointerGetAttributes(&at, base));
            HG_REQUIRE(at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged,
                       "hg_set_particles_device needs a device pointer");
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
        // the FP64 stages read the same device copy in place
        if (hi) hi->set_particles(s, reinterpret_cast<const double *>(S.base()), n, stride, pos_off, los_off, w_off, true);
    }

    // statistics state derived from the current source (the catalogue itself is unchanged)
    void invalidate_stats() {
        sn_xi_cache.clear();
        Gm_ok.clear();
        shD_valid = false;
        xi_valid = false;
        famA_ok.clear();
        famQ_ok.clear();
        hist_ok.clear();
        pairs.clear();
        Gz_ok.clear();
        zf_ok.clear();
        zpairs.clear();
        hist_sv_ok.clear();
    }

    // select the box (kind 0) or the survey with a given alpha (kind 1) as the source
    void set_source(int kind, double alpha) {
        if (kind != src_kind || (kind != 0 && alpha != src_alpha)) {
            invalidate_stats();
            src_kind = kind;
            src_alpha = alpha;
        }
        if (kind == 0) {
            box_density();
            dsrc = SpecK{half_spec_unnarrowed(), delta0, 0.0};  // its readers narrow first
        } else {
            dsrc = sfield(delta_kind(), 0, 0, alpha);
        }
    }
    // the Yhat-weighted field the current survey source is made of: D - alpha R, or the
    // randoms alone for the window functions (source kind 2)
    int delta_kind() const { return src_kind == 2 ? SF_WIN : SF_DELTA; }
    int sn_kind() const { return src_kind == 2 ? SF_WIN_SN : SF_SN; }

    // the spectrum whose IFFT / W / V is G for a G key
    SpecK g_source(const GK &gk) {
        if (src_kind == 0) return SpecK{half_spec(), delta0, 0.0};
        return sfield(delta_kind(), gk.first, gk.second, src_alpha);
    }

    void invalidate() {
        src_kind = -1;
        dens_valid = false;
        H_wide = nullptr;
        narrow_pending = false;
        pk_cache.clear();
        sn_xi_cache.clear();
        Gm_ok.clear();
        shD_valid = false;
        xi_valid = false;
        famA_ok.clear();
        famQ_ok.clear();
        hist_ok.clear();
        pairs.clear();
        Gz_ok.clear();
        zf_ok.clear();
        zpairs.clear();
        sf_ok.clear();
        hist_sv_ok.clear();
        sbins[0].ok = sbins[1].ok = false;
    }

    // ------------------------------------------------------------------ assignment
    // Assignment tile extents: 8 x 16 x 32 cells (or the whole axis when shorter) where those
    // divide the mesh; otherwise, per axis, divisors of n between 4 (the widest stencil)
    // and 32, the combination with the most cells up to 4096 (the shared-memory tile).
    int tile_t[3] = {8, 16, 32};
    void choose_tiles() {
        const int tdef[3] = {8, 16, 32};
        bool plain = true;
        for (int a = 0; a < 3; a++) plain = plain && g.n[a] % std::min(tdef[a], g.n[a]) == 0;
        if (plain) {
            for (int a = 0; a < 3; a++) tile_t[a] = std::min(tdef[a], g.n[a]);
            return;
        }
        std::vector<int> dv[3];
        for (int a = 0; a < 3; a++) {
            for (int d = 4; d <= 32; d++)
                if (g.n[a] % d == 0) dv[a].push_back(d);
            HG_REQUIRE(!dv[a].empty(), "n_mesh: every axis needs a divisor between 4 and 32 (the assignment tiles)");
        }
        long long best = -1;
        for (int x : dv[0])
            for (int y : dv[1])
                for (int z : dv[2]) {
                    const long long v = (long long)x * y * z;
                    // most cells, then the longest rows (z), then y
                    const long long key = v * 4096 + z * 64 + y;
                    if (v <= 4096 && key > best) {
                        best = key;
                        tile_t[0] = x;
                        tile_t[1] = y;
                        tile_t[2] = z;
                    }
                }
        HG_REQUIRE(best >= 0, "n_mesh: no assignment tile of at most 4096 cells");
    }
    AssignGeom make_geom(double shift) const {
        AssignGeom a;
        for (int q = 0; q < 3; q++) {
            a.n[q] = g.n[q];
            a.L[q] = g.L[q];
        }
        a.ntot = g.ntot;
        a.scheme = cfg.assign;
        a.periodic = (cfg.periodic || cfg.assign == HG_PCS || cfg.interlace) ? 1 : 0;
        a.shift = shift;
        for (int q = 0; q < 3; q++) {
            a.t[q] = tile_t[q];
            a.tsh[q] = -1;
            for (int b = 0; b < 31; b++)
                if ((1 << b) == a.t[q]) a.tsh[q] = b;
            a.nt[q] = g.n[q] / a.t[q];
            a.far[q] = 0x1p30 * g.L[q] / double(g.n[q]);
        }
        a.factor = 1.0 / (g.volume / double(g.ntot));
        // FP64 form: the reference's density rho = sum w (1/dV) prod(w_axis).  FP32 form: the
        // mass per cell (rho dV), which removes the float rounding of 1/dV and dV from every
        // cell; the FFT input (rho - N/V) dV is then mass - N/Ncells (same quantity).
        a.acc_factor = (sizeof(T) == 8) ? a.factor : 1.0;
        a.fix_bound = 0.0f;
        return a;
    }

    // Tile counts of several sources (pass 1).  Each source's edge-straddling particles go to
    // its own slice of the deferred list (at the running offset of the sources' sizes) and
    // are counted by a second launch; the scatter reads the same slices.
    // mass_part (when not null): room for ns x MASS_BLOCKS x 2 doubles; source q's blocks write
    // theirs at q MASS_BLOCKS 2 (see k_bin_count), mass_blocks[q] of them
    static constexpr int MASS_BLOCKS = 148 * 8;
    int mass_blocks[2] = {0, 0};
    void bin_count_sources(const PartSrc *srcs, int ns, const AssignGeom &ag, double *mass_part) {
        long long cap = 0;
        for (int q = 0; q < ns; q++) cap += srcs[q].n;
        HG_CK(deflist.ensure(sizeof(int) * std::max<long long>(cap, 1)));
        // + the non-finite particle count and the negative-coordinate flag
        HG_CK(defcnt.ensure(sizeof(unsigned) * (ns + 2)));
        HG_CK(cudaMemsetAsync(defcnt.p, 0, sizeof(unsigned) * (ns + 2), st));
        long long o = 0;
        for (int q = 0; q < ns; q++) {
            if (q < 2) mass_blocks[q] = 0;
            if (srcs[q].n == 0) continue;  // an empty catalogue (no data for a window function)
            Defer df{dp<int>(deflist) + o, dp<unsigned>(defcnt) + q, 0, dp<unsigned>(defcnt) + ns,
                     dp<unsigned>(defcnt) + ns + 1};
            const unsigned nb = (unsigned)std::min<long long>(
                grid1(srcs[q].n, 256), std::min<long long>(MASS_BLOCKS, resident_grid(k_bin_count, 256)));
            if (q < 2) mass_blocks[q] = (int)nb;
            kb("assign_bin_count", double(srcs[q].n) * 24.0);
            k_bin_count<<<nb, 256, 0, st>>>(srcs[q], ag, df, dp<unsigned>(cnt),
                                            mass_part ? mass_part + (size_t)q * MASS_BLOCKS * 2 : nullptr);
            ke();
            df.pass = 1;
            kb("assign_edge_count", 0.0);
            k_bin_count<<<148 * 8, 256, 0, st>>>(srcs[q], ag, df, dp<unsigned>(cnt), nullptr);
            ke();
            o += srcs[q].n;
        }
    }

    // After bin_count_sources(ns sources): queue the read-back of its non-finite particle
    // count and negative-coordinate flag into flags[0..1] (checked by check_finite once the
    // stream has been synchronised).
    void read_bad_count(int ns, unsigned *flags) {
        HG_CK(cudaMemcpyAsync(flags, dp<unsigned>(defcnt) + ns, 2 * sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    }
    static void check_finite(const unsigned *flags) {
        HG_REQUIRE(flags[0] == 0, "the catalogue holds " + std::to_string(flags[0]) +
                                      " particle(s) with a non-finite position, weight or line of sight");
    }
    // the largest product of the three axis weights of one stencil point: 1 for coordinates
    // >= 0 (and for NGP and PCS), 8 for CIC and TSC when a coordinate is negative
    float stencil_weight_bound(bool neg) const {
        return (neg && (cfg.assign == HG_CIC || cfg.assign == HG_TSC)) ? 8.0f : 1.0f;
    }

    // Records of several sources (pass 3), from the front of each tile's range, then the
    // deferred particles from the back.
    template <class MK>
    void bin_scatter_sources(const PartSrc *srcs, const MK *mks, int ns, const AssignGeom &ag, int ntiles,
                             typename MK::R *recp, double rec_bytes) {
        HG_CK(cursor_back.ensure(sizeof(unsigned) * (ntiles + 1)));
        HG_CK(cudaMemsetAsync(cursor_back.p, 0, sizeof(unsigned) * (ntiles + 1), st));
        long long o = 0, nsum = 0;
        for (int q = 0; q < ns; q++) nsum += srcs[q].n;
        for (int q = 0; q < ns; q++) {
            if (srcs[q].n == 0) continue;
            Defer df{dp<int>(deflist) + o, dp<unsigned>(defcnt) + q, 0, dp<unsigned>(defcnt) + ns,
                     dp<unsigned>(defcnt) + ns + 1};
            kb("assign_bin_scatter", double(srcs[q].n) * 24.0 + rec_bytes * double(srcs[q].n) / double(nsum));
            // (several waves: one resident wave was measured slower here, 0.83 -> 0.96 ms per
            // 1e7 particles, unlike the count pass)
            k_bin_scatter<MK><<<(unsigned)std::min<long long>(grid1(srcs[q].n, 256), 148 * 16), 256, 0, st>>>(
                srcs[q], ag, mks[q], df, dp<unsigned>(off), dp<unsigned>(cursor), dp<unsigned>(cursor_back), recp);
            ke();
            df.pass = 1;
            kb("assign_edge_scatter", 0.0);
            k_bin_scatter<MK><<<148 * 8, 256, 0, st>>>(srcs[q], ag, mks[q], df, dp<unsigned>(off),
                                                      dp<unsigned>(cursor), dp<unsigned>(cursor_back), recp);
            ke();
            o += srcs[q].n;
        }
    }

    // Assign one or more particle sources into one mesh of type U (real, or complex as
    // planar re/im arrays): tile binning of every source, scan, chunking, scatter of
    // compact records, tile accumulation.  Returns the FP64 in-bounds mass (real part)
    // when want_mass.
    template <typename U, bool CPLX>
    double assign_mesh(const std::vector<PartSrc> &srcs, const AssignGeom &ag, U *out_re, U *out_im, bool want_mass,
                       double *mass_im = nullptr) {
        const int ntiles = ag.nt[0] * ag.nt[1] * ag.nt[2];
        HG_CK(cnt.ensure(sizeof(unsigned) * (ntiles + 1)));
        HG_CK(off.ensure(sizeof(unsigned) * (ntiles + 1)));
        HG_CK(cursor.ensure(sizeof(unsigned) * (ntiles + 1)));
        HG_CK(nch.ensure(sizeof(unsigned) * (ntiles + 1)));
        HG_CK(choff.ensure(sizeof(unsigned) * (ntiles + 1)));
        HG_REQUIRE(srcs.size() <= 2, "at most two sources per assignment");
        HG_CK(mass.ensure(sizeof(double) * 2 * MASS_BLOCKS * 2));
        HG_CK(cudaMemsetAsync(cnt.p, 0, sizeof(unsigned) * (ntiles + 1), st));
        HG_CK(cudaMemsetAsync(cursor.p, 0, sizeof(unsigned) * (ntiles + 1), st));
        bin_count_sources(srcs.data(), (int)srcs.size(), ag, want_mass ? dp<double>(mass) : nullptr);
        size_t tb = 0, tb2 = 0;
        HG_CK(cub::DeviceScan::ExclusiveSum(nullptr, tb, dp<unsigned>(cnt), dp<unsigned>(off), ntiles + 1, st));
        HG_CK(cub::DeviceScan::ExclusiveSum(nullptr, tb2, dp<unsigned>(nch), dp<unsigned>(choff), ntiles + 1, st));
        HG_CK(cubtmp.ensure(std::max(tb, tb2)));
        kb("assign_scan", double(ntiles + 1) * 8.0);
        HG_CK(cub::DeviceScan::ExclusiveSum(cubtmp.p, tb, dp<unsigned>(cnt), dp<unsigned>(off), ntiles + 1, st));
        ke();
        kb("assign_chunks", double(ntiles + 1) * 16.0);
        k_chunk_count<<<grid1(ntiles + 1, 256), 256, 0, st>>>(dp<unsigned>(cnt), ntiles, CHUNK, dp<unsigned>(nch));
        ke();
        kb("assign_scan", double(ntiles + 1) * 8.0);
        HG_CK(cub::DeviceScan::ExclusiveSum(cubtmp.p, tb2, dp<unsigned>(nch), dp<unsigned>(choff), ntiles + 1, st));
        ke();
        unsigned tot[2] = {0, 0};
        double hm[2] = {0.0, 0.0};
        std::vector<double> mp(want_mass ? 2 * MASS_BLOCKS * 2 : 0);
        HG_CK(cudaMemcpyAsync(&tot[0], dp<unsigned>(off) + ntiles, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
        HG_CK(cudaMemcpyAsync(&tot[1], dp<unsigned>(choff) + ntiles, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
        if (want_mass)
            HG_CK(cudaMemcpyAsync(mp.data(), mass.p, sizeof(double) * mp.size(), cudaMemcpyDeviceToHost, st));
        unsigned flags[2] = {0, 0};
        read_bad_count((int)srcs.size(), flags);
        HG_CK(cudaStreamSynchronize(st));
        check_finite(flags);
        if (want_mass)  // block partials in a fixed order
            for (size_t q = 0; q < srcs.size(); q++)
                for (int b = 0; b < mass_blocks[q]; b++) {
                    hm[0] += mp[(q * MASS_BLOCKS + b) * 2];
                    hm[1] += mp[(q * MASS_BLOCKS + b) * 2 + 1];
                }
        const unsigned total = tot[0], nchunks = tot[1];
        // 25 % headroom: catalogues of varying size reuse the buffers without reallocating
        if (rec.n < sizeof(PRec<U>) * std::max<size_t>(total, 1))
            HG_CK(rec.ensure(sizeof(PRec<U>) * (std::max<size_t>(total, 1) * 5 / 4)));
        if (chunks.n < sizeof(Chunk) * std::max<size_t>(nchunks, 1))
            HG_CK(chunks.ensure(sizeof(Chunk) * (std::max<size_t>(nchunks, 1) * 5 / 4)));
        // exact fixed-point accumulation for real meshes of unweighted sources, whose
        // per-record weight |scale| acc_factor is known here (the stencil weights sum to one),
        // on meshes with at least W cells per axis (one add per record and cell)
        static_assert(CHUNK <= 2048, "the fixed-point lo word holds at most 2048 adds of < 2^20");
        bool fix = false;
        AssignGeom agx = ag;
        if constexpr (!CPLX) {  // FP32: two 32-bit words per cell; FP64: three
            fix = true;
            double wmax = 0.0;
            for (const auto &src : srcs) {
                fix = fix && src.cw == nullptr && !src.ylm_on && src.w_off < 0;
                wmax = std::max(wmax, std::fabs(src.scale));
            }
            for (int a = 0; a < 3; a++) fix = fix && ag.n[a] >= stencil_width(ag.scheme);
            agx.fix_bound = (float)(wmax * std::fabs(ag.acc_factor)) * stencil_weight_bound(flags[1] != 0);
            fix = fix && agx.fix_bound >= 0x1p-60f;
        }
        // split tiles of a fixed-point accumulation add their chunks' exact partial sums as
        // 64-bit integers in a staging slot (at most nchunks - ntiles split tiles), written
        // out once: the mesh does not depend on the order the chunks finish in
        const int cwords = sizeof(U) == 8 ? 2 : 1;
        const size_t tcells = (size_t)ag.t[0] * ag.t[1] * ag.t[2];
        const size_t nsplit_max = nchunks > (unsigned)ntiles ? nchunks - (unsigned)ntiles : 0;
        unsigned long long *crowd_p = nullptr;
        if (fix && nsplit_max > 0) {
            HG_CK(crowd.ensure(sizeof(unsigned long long) * cwords * tcells * nsplit_max));
            crowd_p = dp<unsigned long long>(crowd);
        }
        HG_CK(nslots.ensure(sizeof(unsigned)));
        HG_CK(cudaMemsetAsync(nslots.p, 0, sizeof(unsigned), st));
        kb("assign_chunks", double(ntiles) * 16.0);
        k_chunk_fill<<<grid1(ntiles, 256), 256, 0, st>>>(dp<unsigned>(off), dp<unsigned>(choff), ntiles, CHUNK,
                                                        dp<Chunk>(chunks), dp<unsigned>(nslots));
        ke();
        {
            std::vector<RecWeight<U>> mk(srcs.size());
            bin_scatter_sources(srcs.data(), mk.data(), (int)srcs.size(), ag, ntiles, dp<PRec<U>>(rec),
                                double(total) * sizeof(PRec<U>));
        }
        kb("assign_zero_split", 0.0);
        k_zero_split_tiles<U, CPLX><<<nchunks, 256, 0, st>>>(dp<Chunk>(chunks), ag, out_re, out_im, crowd_p, cwords);
        ke();
        const size_t tbytes = sizeof(U) * tcells;
        kb("assign_tile_accum", double(total) * sizeof(PRec<U>) + double(g.ntot) * sizeof(U) * (CPLX ? 2 : 1));
        switch (ag.scheme) {
            case HG_NGP: launch_tile_accum<U, CPLX, HG_NGP>(fix, tbytes, nchunks, agx, out_re, out_im, crowd_p); break;
            case HG_CIC: launch_tile_accum<U, CPLX, HG_CIC>(fix, tbytes, nchunks, agx, out_re, out_im, crowd_p); break;
            case HG_TSC: launch_tile_accum<U, CPLX, HG_TSC>(fix, tbytes, nchunks, agx, out_re, out_im, crowd_p); break;
            default: launch_tile_accum<U, CPLX, HG_PCS>(fix, tbytes, nchunks, agx, out_re, out_im, crowd_p); break;
        }
        ke();
        if constexpr (!CPLX) {
            if (crowd_p) {
                kb("assign_split_writeout", 0.0);
                k_crowd_writeout<U><<<nchunks, 256, 0, st>>>(dp<Chunk>(chunks), agx, crowd_p, out_re);
                ke();
            }
        }
        if (mass_im) *mass_im = hm[1];
        return hm[0];
    }
    DBuf crowd, nslots;  // split-tile staging of the fixed-point accumulation

    template <typename U, bool CPLX, int SCHEME>
    void launch_tile_accum(bool fix, size_t tbytes, unsigned nchunks, const AssignGeom &ag, U *out_re, U *out_im,
                           unsigned long long *crowd_p) {
        if constexpr (!CPLX) {
            if (fix) {  // FP32: two words of 4 bytes per cell; FP64: three
                const size_t sm = (sizeof(U) == 4) ? 2 * tbytes : (3 * tbytes) / 2;
                auto kern = k_tile_accum<U, false, true, SCHEME>;
                HG_CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
                kern<<<nchunks, 256, sm, st>>>(dp<PRec<U>>(rec), dp<Chunk>(chunks), ag, out_re, out_im, crowd_p);
                return;
            }
        }
        const size_t smem = tbytes * (CPLX ? 2 : 1);
        auto kern = k_tile_accum<U, CPLX, false, SCHEME>;
        HG_CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kern<<<nchunks, 256, smem, st>>>(dp<PRec<U>>(rec), dp<Chunk>(chunks), ag, out_re, out_im, nullptr);
    }

    double assign_real(const PartSrc &src, const AssignGeom &ag, T *out) {
        return assign_mesh<T, false>({src}, ag, out, nullptr, true);
    }

    template <int DIR, class LD, class ST>
    void pass(int L, LD ld, ST stt, long long outer, long long inner, const char *name = "fft_pass",
              double bytes = -1.0) {
        PassGeom pg{outer, inner};
        if (bytes < 0) bytes = 2.0 * double(outer) * L * inner * sizeof(C);
        const C *twp = twiddles(L);
        kb(name, bytes);
        HG_CK((launch_pass_any<T, DIR>(L, ld, stt, pg, twp, st)));
        ke();
    }

    // Box density contrast, forward transformed: H = FFT[dV (rho - N/V)] (half spectrum).
    // r2c transform of a real mesh into the half spectrum Hd: FFT[(mesh - sub) scl]
    void forward_real(const T *m, C *Hd, T sub, T scl, const char *name) {
        const int hz = g.n[2] / 2 + 1;
        // z: two real rows per complex transform (k_fft2_r2c_pair), the plain pass otherwise
        kb(name, double(g.ntot) * sizeof(T) + double(g.n[0]) * g.n[1] * hz * sizeof(C));
        cudaError_t pe = cudaSuccess;
        const bool paired =
            launch_r2c_pair<T, -1>(g.n[2], m, sub, scl, Hd, (long long)g.n[0] * g.n[1], hz, twiddles(g.n[2]), st, pe);
        HG_CK(pe);
        ke();
        if (!paired)
            pass<-1>(g.n[2], LdMeshDelta<T>{m, g.n[2], sub, scl}, StHalf<T>{Hd, g.n[2], hz}, (long long)g.n[0] * g.n[1],
                     1, name, double(g.ntot) * sizeof(T) + double(g.n[0]) * g.n[1] * hz * sizeof(C));
        pass<-1>(g.n[1], LdArr<T>{Hd, g.n[1], hz}, StArr<T>{Hd, g.n[1], hz}, g.n[0], hz, name);
        pass<-1>(g.n[0], LdArr<T>{Hd, g.n[0], (long long)g.n[1] * hz}, StArr<T>{Hd, g.n[0], (long long)g.n[1] * hz}, 1,
                 (long long)g.n[1] * hz, name);
    }

    // F = (F + phase * Fs) / 2 over a half (half = 1) or full spectrum
    void interlace_combine(C *F, const C *Fs, bool half) {
        const int nzs = half ? g.n[2] / 2 + 1 : g.n[2];
        const long long tot = (long long)g.n[0] * g.n[1] * nzs;
        unsigned blocks = (unsigned)std::min<long long>(grid1(tot, 256), 148 * 16);
        kb("interlace_combine", double(tot) * sizeof(C) * 3.0);
        k_interlace<T><<<blocks, 256, 0, st>>>(F, Fs, g.n[0], g.n[1], g.n[2], nzs, half ? 1 : 0);
        ke();
    }

    void box_density() {
        if (dens_valid) return;
        if (hi && (fp64_stages & HG_STAGE_DENSITY)) {  // computed by the FP64 engine, narrowed
            double d0, n0, m0;
            const void *Hh = hi->stage_density(&d0, &n0, &m0);
            launches += hi->stage_take_launches();
            stage_import_density(Hh, true, d0, n0, m0);
            return;
        }
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
        const bool mass_mesh = (sizeof(T) == 4);
        const T sub = mass_mesh ? (T)(double(S.n) / double(g.ntot)) : (T)nbar;
        const T scl = mass_mesh ? (T)1 : (T)dV;
        forward_real(dp<T>(mesh), dp<C>(H), sub, scl, "fft_density");
        if (cfg.interlace) {  // second assignment half a cell along every axis, combined in k space
            const double m1 = assign_real(src, make_geom(0.5), dp<T>(mesh));
            HG_CK(H2.ensure(sizeof(C) * (size_t)g.n[0] * g.n[1] * hz));
            forward_real(dp<T>(mesh), dp<C>(H2), sub, scl, "fft_density");
            interlace_combine(dp<C>(H), dp<C>(H2), true);
            dens_mass = 0.5 * (dens_mass + m1);
        }
        // k = 0 from the FP64 integral: sum_c (rho_c - nbar) dV
        delta0 = (dens_mass - nbar * double(g.ntot)) * dV;
        N0 = dens_mass * dV;
        kb("set_k0", double(sizeof(C)));
        k_set_k0<T><<<1, 1, 0, st>>>(dp<C>(H), (T)delta0, (T)0);
        ke();
        dens_valid = true;
    }

    // the density half spectrum in this engine's precision (narrowed first if it came from the
    // FP64 engine and was not yet needed)
    Spec<T> half_spec() {
        narrow_density();
        return half_spec_unnarrowed();
    }
    Spec<T> half_spec_unnarrowed() const { return Spec<T>{dp<C>(H), g.n[0], g.n[1], g.n[2], 1}; }
    void narrow_density() {
        if (!narrow_pending) return;
        narrow_pending = false;
        convert_spectrum(H_wide, true);
    }
    void convert_spectrum(const void *src, bool src_fp64) {
        const long long n = (long long)g.n[0] * g.n[1] * (g.n[2] / 2 + 1);
        const unsigned blocks = (unsigned)std::min<long long>(grid1(n, 256), 148 * 16);
        kb("stage_convert", double(n) * (sizeof(C) + (src_fp64 ? 16.0 : 8.0)));
        if (src_fp64)
            k_convert_spec<double, T><<<blocks, 256, 0, st>>>(reinterpret_cast<const cplx<double> *>(src), dp<C>(H), n);
        else
            k_convert_spec<float, T><<<blocks, 256, 0, st>>>(reinterpret_cast<const cplx<float> *>(src), dp<C>(H), n);
        ke();
    }

    // ------------------------------------------------------------------ P binning
    // Averages over each k bin of  (f conj f - S C(k)) / W^2 * Yhat_lm(k)  for a list of (l, m)
    // (TwoPointStatisticsClass::calcPowerSpectrum, field.hpp:765-852).  avg: [nbin][nlm] complex.
    void pk_bin(const std::vector<LM> &lm, double S_re, double S_im, std::vector<double> &avg,
                std::vector<unsigned long long> &nm) {
        pk_bin2(half_spec(), half_spec(), lm, S_re, S_im, avg, nm);
    }
    template <class F1>
    void pk_bin2(const F1 &f1, const Spec<T> &f2, const std::vector<LM> &lm, double S_re, double S_im,
                 std::vector<double> &avg, std::vector<unsigned long long> &nm) {
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
        HG_CK(bin_acc.ensure(sizeof(double) * 2 * nbin * L.n));
        HG_CK(bin_cnt.ensure(sizeof(unsigned long long) * nbin));
        HG_CK(cudaMemsetAsync(bin_acc.p, 0, sizeof(double) * 2 * nbin * L.n, st));
        HG_CK(cudaMemsetAsync(bin_cnt.p, 0, sizeof(unsigned long long) * nbin, st));
        size_t smem = sizeof(double) * 2 * nbin * L.n + sizeof(unsigned long long) * nbin;
        if (n_pk_modes < 0) build_pk_modes(lo, cn);
        HG_CK(cudaFuncSetAttribute(k_pk_bin_list<F1, Spec<T>>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        // one resident wave (a partial second wave was a third of the kernel's time)
        int per_sm = 1, sms = 148;
        HG_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pk_bin_list<F1, Spec<T>>, 256, smem));
        HG_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, cfg.device));
        const unsigned blocks =
            (unsigned)std::max<long long>(1, std::min<long long>(grid1(n_pk_modes, 256), (long long)sms * std::max(per_sm, 1)));
        kb("pk_bin", double(n_pk_modes) * (sizeof(PkMode) + 2.0 * sizeof(C)));
        k_pk_bin_list<F1, Spec<T>><<<blocks, 256, smem, st>>>(f1, f2, dp<PkMode>(pk_modes), n_pk_modes, nbin, L, S_re,
                                                              S_im, dp<double>(bin_acc), dp<unsigned long long>(bin_cnt),
                                                              0, 0.0, 0.0);
        ke();
        std::vector<double> a(2 * nbin * L.n);
        nm.assign(nbin, 0);
        HG_CK(cudaMemcpyAsync(a.data(), bin_acc.p, sizeof(double) * a.size(), cudaMemcpyDeviceToHost, st));
        HG_CK(cudaMemcpyAsync(nm.data(), bin_cnt.p, sizeof(unsigned long long) * nbin, cudaMemcpyDeviceToHost, st));
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

    // The binning cube's modes that fall in a bin (k_pk_modes_*), in cube order, once per context.
    void build_pk_modes(int3 lo, int3 cn) {
        const long long total = (long long)cn.x * cn.y * cn.z;
        DBuf flag, pos;
        HG_CK(flag.ensure(sizeof(unsigned) * (total + 1)));
        HG_CK(pos.ensure(sizeof(unsigned) * (total + 1)));
        HG_CK(cudaMemsetAsync(flag.p, 0, sizeof(unsigned) * (total + 1), st));
        const unsigned blocks = (unsigned)std::min<long long>(grid1(total, 256), 148 * 8);
        k_pk_modes_flag<<<blocks, 256, 0, st>>>(g, lo, cn, dp<int2>(lut), lutn, dp<unsigned>(flag));
        HG_CK(cudaGetLastError());
        size_t tb = 0;
        HG_CK(cub::DeviceScan::ExclusiveSum(nullptr, tb, dp<unsigned>(flag), dp<unsigned>(pos), total + 1, st));
        HG_CK(cubtmp.ensure(tb));
        HG_CK(cub::DeviceScan::ExclusiveSum(cubtmp.p, tb, dp<unsigned>(flag), dp<unsigned>(pos), total + 1, st));
        unsigned nm = 0;
        HG_CK(cudaMemcpyAsync(&nm, dp<unsigned>(pos) + total, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
        HG_CK(cudaStreamSynchronize(st));
        HG_CK(pk_modes.ensure(sizeof(PkMode) * std::max<unsigned>(nm, 1)));
        k_pk_modes_fill<<<blocks, 256, 0, st>>>(g, tabs, lo, cn, dp<int2>(lut), lutn, cfg.assign, wpow,
                                                dp<unsigned>(pos), dp<PkMode>(pk_modes));
        HG_CK(cudaGetLastError());
        HG_CK(cudaStreamSynchronize(st));  // flag and pos are released on return
        n_pk_modes = nm;
    }

    // averages over each k bin of sum_q w_q (F_q conj f2 - S_q C) / W^2 Yhat_{l_q m_q}
    void pk_bin_terms(const PkTerms<T> &terms, const Spec<T> &f2, std::vector<double> &avg,
                      std::vector<unsigned long long> &nm) {
        const int nbin = cfg.n_kbin;
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
        HG_CK(bin_acc.ensure(sizeof(double) * 2 * nbin));
        HG_CK(bin_cnt.ensure(sizeof(unsigned long long) * nbin));
        HG_CK(cudaMemsetAsync(bin_acc.p, 0, sizeof(double) * 2 * nbin, st));
        HG_CK(cudaMemsetAsync(bin_cnt.p, 0, sizeof(unsigned long long) * nbin, st));
        long long total = (long long)cn.x * cn.y * cn.z;
        unsigned blocks = (unsigned)std::min<long long>(grid1(total, 256), 148 * 8);
        kb("pk_bin", double(total) * sizeof(C) * (terms.n + 1));
        k_pk_bin_terms<T, Spec<T>><<<blocks, 256, 0, st>>>(terms, f2, g, tabs, lo, cn, dp<int2>(lut), lutn, nbin,
                                                           cfg.assign, wpow, dp<double>(bin_acc),
                                                           dp<unsigned long long>(bin_cnt));
        ke();
        std::vector<double> a(2 * nbin);
        nm.assign(nbin, 0);
        HG_CK(cudaMemcpyAsync(a.data(), bin_acc.p, sizeof(double) * a.size(), cudaMemcpyDeviceToHost, st));
        HG_CK(cudaMemcpyAsync(nm.data(), bin_cnt.p, sizeof(unsigned long long) * nbin, cudaMemcpyDeviceToHost, st));
        HG_CK(cudaStreamSynchronize(st));
        avg.assign(2 * nbin, 0.0);
        for (int j = 0; j < nbin; j++)
            if (nm[j] != 0) {
                avg[2 * j] = a[2 * j] / double(nm[j]);
                avg[2 * j + 1] = a[2 * j + 1] / double(nm[j]);
            }
    }

    // the box P_l bins of the current density (box_density() done), binned on first use
    const PkBins &box_pk_bins(int ell) {
        if (!pk_cache.count(ell)) {
            // one pass over the modes bins the requested multipole together with the
            // others of the usual set (0, 2, 4) not yet binned for this density: the pass
            // is latency-bound, so the extra multipoles cost next to nothing
            std::vector<LM> lm{LM{ell, 0}};
            for (int e : {0, 2, 4})
                if (e != ell && !pk_cache.count(e)) lm.push_back(LM{e, 0});
            std::vector<double> avg;
            std::vector<unsigned long long> nm;
            pk_bin(lm, double(slot[0].n), 0.0, avg, nm);
            const int nl = (int)lm.size();
            for (int q = 0; q < nl; q++) {
                PkBins &pb = pk_cache[lm[q].l];
                pb.avg.resize(2 * cfg.n_kbin);
                for (int i = 0; i < cfg.n_kbin; i++) {
                    pb.avg[2 * i] = avg[2 * (i * nl + q)];
                    pb.avg[2 * i + 1] = avg[2 * (i * nl + q) + 1];
                }
                pb.nm = nm;
            }
        }
        return pk_cache[ell];
    }

    // powerspec.hpp:273-332
    void pk_box(int ell, double *pk_save, int *n_mode, double *norm) override {
        HG_REQUIRE(ell >= 0, "ell must be >= 0");
        if (hi && (fp64_stages & HG_STAGE_DENSITY)) {  // binned from the FP64 spectrum
            begin();
            hi->pk_box(ell, pk_save, n_mode, norm);
            launches += hi->stage_take_launches();
            end();
            return;
        }
        begin();
        box_density();
        const PkBins &pb = box_pk_bins(ell);
        for (int i = 0; i < cfg.n_kbin; i++) {
            pk_save[2 * i] = double(2 * ell + 1) * pb.avg[2 * i];
            pk_save[2 * i + 1] = double(2 * ell + 1) * pb.avg[2 * i + 1];
            if (n_mode) n_mode[i] = (int)pb.nm[i];
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
        int sx[3];
        for (int a = 0; a < 3; a++) sx[a] = std::min((int)std::floor(upper_max / g.dk[a]) + 1, g.n[a] / 2);
        std::vector<std::vector<ShellEnt>> per(S.ns);
        for (int nx = -sx[0]; nx <= sx[0]; nx++) {
            if (nx >= g.n[0] / 2) continue;
            for (int ny = -sx[1]; ny <= sx[1]; ny++) {
                if (ny >= g.n[1] / 2) continue;
                for (int nz = -sx[2]; nz <= sx[2]; nz++) {
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
            S.K[a] = 2 * smax[a] + 1;
            int need = 4 * smax[a] + 1;
            int m = std::max(8, next_pow2(need));
            if (need > 128 && need <= 192) m = 192;  // 3 x 64: the register FFT's 24 x 8 split
            if (m >= g.n[a]) {
                // the y and z chain passes take any length; the fused x pass a power of two
                HG_REQUIRE(a != 0 || fft_supported_length(g.n[a]),
                           "the bispectrum's shells reach the whole of n_mesh_x, which is not a power of two");
                S.M[a] = g.n[a];
                S.gs[a] = g.n[a] / 2;  // whole axis
            } else {
                S.M[a] = m;
                S.gs[a] = 2 * smax[a];
            }
            S.KG[a] = 2 * S.gs[a] + 1;
        }
        HG_CK(S.d_ent.ensure(sizeof(ShellEnt) * std::max<size_t>(S.ent.size(), 1)));
        if (!S.ent.empty())
            HG_CK(cudaMemcpy(S.d_ent.p, S.ent.data(), sizeof(ShellEnt) * S.ent.size(), cudaMemcpyHostToDevice));
        HG_CK(S.d_start.ensure(sizeof(int) * (S.ns + 1)));
        HG_CK(cudaMemcpy(S.d_start.p, S.start.data(), sizeof(int) * (S.ns + 1), cudaMemcpyHostToDevice));
        {  // pair-sum work items: each shell cut into runs of at most 32 PD_LANE entries
            std::vector<PairItem> items;
            std::vector<int> istart(S.ns + 1, 0);
            for (int i = 0; i < S.ns; i++) {
                istart[i] = (int)items.size();
                for (int e = S.start[i]; e < S.start[i + 1]; e += 32 * PD_LANE)
                    items.push_back(PairItem{i, e, std::min(S.start[i + 1], e + 32 * PD_LANE)});
            }
            istart[S.ns] = (int)items.size();
            S.nitems = (int)items.size();
            HG_CK(S.d_items.ensure(sizeof(PairItem) * std::max(1, S.nitems)));
            if (S.nitems)
                HG_CK(cudaMemcpy(S.d_items.p, items.data(), sizeof(PairItem) * S.nitems, cudaMemcpyHostToDevice));
            HG_CK(S.d_istart.ensure(sizeof(int) * (S.ns + 1)));
            HG_CK(cudaMemcpy(S.d_istart.p, istart.data(), sizeof(int) * (S.ns + 1), cudaMemcpyHostToDevice));
        }
        {  // shell extents and the pruned line lists
            S.ext.assign(3 * S.ns, -1);
            for (int i = 0; i < S.ns; i++)
                for (int e = S.start[i]; e < S.start[i + 1]; e++) {
                    const ShellEnt &q = S.ent[e];
                    S.ext[3 * i] = std::max(S.ext[3 * i], std::abs(q.nx));
                    S.ext[3 * i + 1] = std::max(S.ext[3 * i + 1], std::abs(q.ny));
                    S.ext[3 * i + 2] = std::max(S.ext[3 * i + 2], std::abs(q.nz));
                }
            std::vector<int4> e4(S.ns);
            std::vector<int> ex(S.ns), l1, l2;
            // per (shell i, cx) the range of cy of shell i's modes: a z line (i, cx, cy) outside
            // it holds no mode, so B1 skips it and B2 reads it as zero
            std::vector<int2> cyr1((size_t)S.ns * S.K[0], make_int2(1, 0));
            for (int i = 0; i < S.ns; i++)
                for (int e = S.start[i]; e < S.start[i + 1]; e++) {
                    const ShellEnt &q = S.ent[e];
                    int2 &r = cyr1[(size_t)i * S.K[0] + q.nx + S.s[0]];
                    const int cy = q.ny + S.s[1];
                    if (r.x > r.y) r = make_int2(cy, cy);
                    r.x = std::min(r.x, cy);
                    r.y = std::max(r.y, cy);
                }
            for (int i = 0; i < S.ns; i++) {
                e4[i] = make_int4(S.ext[3 * i], S.ext[3 * i + 1], S.ext[3 * i + 2], 0);
                ex[i] = S.ext[3 * i];
                for (int cx = S.s[0] - ex[i]; cx <= S.s[0] + ex[i]; cx++) {
                    l2.push_back(i * S.K[0] + cx);
                    const int2 r = cyr1[(size_t)i * S.K[0] + cx];
                    for (int cy = r.x; cy <= r.y; cy++) l1.push_back((i * S.K[0] + cx) * S.K[1] + cy);
                }
            }
            HG_CK(S.d_cyr1.ensure(sizeof(int2) * cyr1.size()));
            HG_CK(cudaMemcpy(S.d_cyr1.p, cyr1.data(), sizeof(int2) * cyr1.size(), cudaMemcpyHostToDevice));
            HG_REQUIRE((long long)S.ns * S.K[0] * S.K[1] < (1LL << 31), "too many chain lines");
            S.nl1 = (long long)l1.size();
            S.nl2 = (long long)l2.size();
            HG_CK(S.d_ext4.ensure(sizeof(int4) * S.ns));
            HG_CK(cudaMemcpy(S.d_ext4.p, e4.data(), sizeof(int4) * S.ns, cudaMemcpyHostToDevice));
            HG_CK(S.d_extx.ensure(sizeof(int) * S.ns));
            HG_CK(cudaMemcpy(S.d_extx.p, ex.data(), sizeof(int) * S.ns, cudaMemcpyHostToDevice));
            HG_CK(S.d_lines1.ensure(sizeof(int) * std::max<size_t>(l1.size(), 1)));
            if (!l1.empty()) HG_CK(cudaMemcpy(S.d_lines1.p, l1.data(), sizeof(int) * l1.size(), cudaMemcpyHostToDevice));
            HG_CK(S.d_lines2.ensure(sizeof(int) * std::max<size_t>(l2.size(), 1)));
            if (!l2.empty()) HG_CK(cudaMemcpy(S.d_lines2.p, l2.data(), sizeof(int) * l2.size(), cudaMemcpyHostToDevice));
            std::vector<unsigned char> disc((size_t)S.K[0] * S.K[1], 0);
            for (const ShellEnt &q : S.ent) {  // Qhat is read at -k of the shell modes k: both signs
                disc[(size_t)(q.nx + S.s[0]) * S.K[1] + (q.ny + S.s[1])] = 1;
                disc[(size_t)(S.s[0] - q.nx) * S.K[1] + (S.s[1] - q.ny)] = 1;
            }
            std::vector<int> l3;
            for (int i = 0; i < S.ns; i++)
                for (int c = 0; c < S.K[0] * S.K[1]; c++)
                    if (disc[c]) l3.push_back(i * S.K[0] * S.K[1] + c);
            S.nl3 = (long long)l3.size();
            std::vector<int2> cyr(S.K[0], make_int2(1, 0));  // empty ranges by default
            long long nr = 0;
            for (int cx = 0; cx < S.K[0]; cx++) {
                for (int cy = 0; cy < S.K[1]; cy++)
                    if (disc[(size_t)cx * S.K[1] + cy]) {
                        if (cyr[cx].x > cyr[cx].y) cyr[cx] = make_int2(cy, cy);
                        cyr[cx].y = cy;
                    }
                if (cyr[cx].y >= cyr[cx].x) nr += cyr[cx].y - cyr[cx].x + 1;
            }
            S.disc_frac = disc.empty() ? 1.0 : double(nr) / double(disc.size());
            HG_CK(S.d_cyr.ensure(sizeof(int2) * S.K[0]));
            HG_CK(cudaMemcpy(S.d_cyr.p, cyr.data(), sizeof(int2) * S.K[0], cudaMemcpyHostToDevice));
            HG_CK(S.d_lines3.ensure(sizeof(int) * std::max<size_t>(l3.size(), 1)));
            if (!l3.empty()) HG_CK(cudaMemcpy(S.d_lines3.p, l3.data(), sizeof(int) * l3.size(), cudaMemcpyHostToDevice));
        }
        std::vector<double> inv(S.ns);
        for (int i = 0; i < S.ns; i++) inv[i] = S.nmode[i] ? 1.0 / double(S.nmode[i]) : 0.0;
        HG_CK(S.d_scale.ensure(sizeof(double) * S.ns));
        HG_CK(cudaMemcpy(S.d_scale.p, inv.data(), sizeof(double) * S.ns, cudaMemcpyHostToDevice));
        S.built = true;
    }

    long long n_ent() const { return (long long)shells.ent.size(); }
    long long cube_vol() const { return (long long)shells.K[0] * shells.K[1] * shells.K[2]; }

    DBuf &map_buf(std::map<Fam, std::unique_ptr<DBuf>> &m, const Fam &f) {
        auto &p = m[f];
        if (!p) p = std::make_unique<DBuf>();
        return *p;
    }

    const double2 *family_A(const Fam &f) {
        DBuf &b = map_buf(famA, f);
        if (famA_ok.count(f)) return dp<double2>(b);
        HG_CK(b.ensure(sizeof(double2) * std::max<long long>(n_ent(), 1)));
        kb("shell_family_A", double(n_ent()) * 48.0);
        k_family_A<<<grid1(n_ent(), 256), 256, 0, st>>>(dp<ShellEnt>(shells.d_ent), n_ent(), g, f.l, f.m,
                                                        dp<double2>(shD), dp<double>(shells.d_scale), dp<double2>(b));
        ke();
        famA_ok.insert(f);
        return dp<double2>(b);
    }

    void ensure_chain_tmp(long long t1, long long t2) {
        HG_CK(T1.ensure(sizeof(C) * std::max<long long>(t1, 1)));
        HG_CK(T2.ensure(sizeof(C) * std::max<long long>(t2, 1)));
    }

    // Transform-grid geometry of a set of chains: kept modes |n_a| <= s_a (compact side
    // K = 2s+1), transform grid M, and the cube |n_a| <= gs_a of G's input.
    struct ChainGeo {
        int ns;
        int s[3], K[3], M[3], gs[3], KG[3];
    };
    ChainGeo bk_geo() const {
        ChainGeo q;
        q.ns = shells.ns;
        for (int a = 0; a < 3; a++) {
            q.s[a] = shells.s[a];
            q.K[a] = shells.K[a];
            q.M[a] = shells.M[a];
            q.gs[a] = shells.gs[a];
            q.KG[a] = shells.KG[a];
        }
        return q;
    }

    // G(x) = IFFT[delta/W]/V on the geometry's grid, from the cube |n_a| <= gs_a (pruned passes)
    void build_G(const ChainGeo &S, DBuf &Gout, const SpecK &src) {
        const long long vol = (long long)S.M[0] * S.M[1] * S.M[2];
        const long long kg = (long long)S.KG[0] * S.KG[1] * S.KG[2];
        HG_CK(Gc.ensure(sizeof(C) * kg));
        HG_CK(Gout.ensure(sizeof(C) * vol));
        ensure_chain_tmp((long long)S.KG[0] * S.KG[1] * S.M[2], (long long)S.KG[0] * S.M[1] * S.M[2]);
        int3 lo = make_int3(-S.gs[0], -S.gs[1], -S.gs[2]);
        int3 cn = make_int3(S.KG[0], S.KG[1], S.KG[2]);
        unsigned blocks = (unsigned)std::min<long long>(grid1(kg, 256), 148 * 16);
        kb("scatter_G", double(kg) * (sizeof(C) * 2));
        k_scatter_G<T><<<blocks, 256, 0, st>>>(src.s, g, tabs, wpow, lo, cn, src.k0r, src.k0i, dp<C>(Gc));
        ke();
        const int M0 = S.M[0], M1 = S.M[1], M2 = S.M[2];
        pass<+1>(M2, LdCube<T>{dp<C>(Gc), S.KG[2], M2, S.gs[2]}, StArr<T>{dp<C>(T1), M2, 1},
                 (long long)S.KG[0] * S.KG[1], 1, "fft_G_inv",
                 double(kg + (long long)S.KG[0] * S.KG[1] * M2) * sizeof(C));
        pass<+1>(M1, LdRowsCompact<T>{dp<C>(T1), S.KG[1], M1, S.gs[1], M2}, StArr<T>{dp<C>(T2), M1, M2}, S.KG[0], M2,
                 "fft_G_inv", double((long long)S.KG[0] * S.KG[1] * M2 + (long long)S.KG[0] * M1 * M2) * sizeof(C));
        pass<+1>(M0, LdRowsCompact<T>{dp<C>(T2), S.KG[0], M0, S.gs[0], (long long)M1 * M2},
                 StArr<T>{dp<C>(Gout), M0, (long long)M1 * M2}, 1, (long long)M1 * M2, "fft_G_inv",
                 double((long long)S.KG[0] * M1 * M2 + vol) * sizeof(C));
    }

    const DBuf &ensure_G(const GK &gk) {
        auto &p = Gm[gk];
        if (!p) p = std::make_unique<DBuf>();
        if (!Gm_ok.count(gk)) {
            build_G(bk_geo(), *p, g_source(gk));
            Gm_ok.insert(gk);
        }
        return *p;
    }

    // Q[j] = FFT[IFFT[Ac[j]] * G] on the geometry's compact cube (hg_chain.cuh); Ac is filled.
    void run_chain(const ChainGeo &S, const DBuf &Gsrc, C *Q) {
        const int ns = S.ns;
        const int Kx = S.K[0], Ky = S.K[1], Kz = S.K[2];
        const int Mx = S.M[0], My = S.M[1], Mz = S.M[2];
        ensure_chain_tmp((long long)ns * Kx * Ky * Mz, (long long)ns * Kx * My * Mz);
        const long long o2 = (long long)ns * Kx;
        // inverse z and y passes over the lines inside each shell's extents only
        const ShellSet &SH = shells;
        const int *lines1 = dp<int>(SH.d_lines1), *lines2 = dp<int>(SH.d_lines2);
        const int4 *ext4 = dp<int4>(SH.d_ext4);
        double in_rows_x = 0.0;  // input rows of the fused x pass, summed over shells
        for (int j = 0; j < ns; j++) in_rows_x += double(2 * SH.ext[3 * j] + 1);
        pass<+1>(Mz, LdCubeL<T>{dp<C>(Ac), Kz, Mz, S.s[2], lines1, ext4, Kx * Ky}, StArrL<T>{dp<C>(T1), Mz, 1, lines1},
                 SH.nl1, 1, "chain_z", double(SH.nl1) * (Kz + Mz) * sizeof(C));
        pass<+1>(My, LdRowsCompactL<T>{dp<C>(T1), Ky, My, S.s[1], Mz, lines2, dp<int2>(SH.d_cyr1)},
                 StArrL<T>{dp<C>(T2), My, Mz, lines2}, SH.nl2, Mz, "chain_y",
                 double(SH.nl2) * (Ky + My) * Mz * sizeof(C));
        const C *Gp = dp<C>(Gsrc);
        const long long plane = (long long)My * Mz;
        const int *extx = dp<int>(SH.d_extx);
        const int var = chain_variant(Mx, Kx, S.s[0], ns, plane, Gp, extx);  // before the timed launch
        kb("chain_x_fused", (in_rows_x + double(ns) * Kx) * My * Mz * sizeof(C) + double(Mx) * My * Mz * sizeof(C));
        HG_CK(launch_chain_x_any(Mx, var, dp<C>(T2), Gp, ns, Kx, S.s[0], plane, extx));
        ke();
        // forward passes over the columns some shell mode has (the pair sums read nothing else)
        pass<-1>(My, LdArr<T>{dp<C>(T2), My, Mz},
                 StRowsCompactD<T>{dp<C>(T1), Ky, My, S.s[1], Mz, Kx, dp<int2>(SH.d_cyr)}, o2, Mz, "chain_y",
                 double(o2) * (SH.disc_frac * Ky + My) * Mz * sizeof(C));
        pass<-1>(Mz, LdArrL<T>{dp<C>(T1), Mz, 1, dp<int>(SH.d_lines3)}, StCubeL<T>{Q, Kz, Mz, S.s[2], dp<int>(SH.d_lines3)},
                 SH.nl3, 1, "chain_z", double(SH.nl3) * (Kz + Mz) * sizeof(C));
    }

    cudaError_t launch_chain_x_any(int Mx, int var, C *t2, const C *Gp, int ns, int Kx, int s0, long long plane,
                                   const int *extx) {
        switch (Mx) {
            case 256: return launch_chain_x_reg_L<T, 256>(var, t2, Gp, ns, Kx, s0, plane, twiddles(Mx), extx, st);
            case 192: return launch_chain_x_reg_L<T, 192>(var, t2, Gp, ns, Kx, s0, plane, twiddles(Mx), extx, st);
            case 128: return launch_chain_x_reg_L<T, 128>(var, t2, Gp, ns, Kx, s0, plane, twiddles(Mx), extx, st);
            case 64: return launch_chain_x_reg_L<T, 64>(var, t2, Gp, ns, Kx, s0, plane, twiddles(Mx), extx, st);
            case 32: return launch_chain_x_reg_L<T, 32>(var, t2, Gp, ns, Kx, s0, plane, twiddles(Mx), extx, st);
            default: return launch_chain_x<T>(Mx, t2, Gp, ns, Kx, s0, plane, twiddles(Mx), extx, st);
        }
    }

    // Launch-shape autotuning of the fused chain pass: the first time a chain runs on a given
    // grid, every variant (kChainVariants) transforms a copy of the chain's shells (all of
    // them, up to 2 GB: staging G once per CTA pays off over many shells, so fewer would
    // favour the variants that do not stage it) twice, and the variant with the fastest
    // second run is kept for the context.  The copy is restored before each run, so every
    // variant sees the same data; the real shells are untouched.
    struct Tuned {
        int variant;
        std::vector<float> ms;
    };
    std::map<int, Tuned> chain_tuned;  // by transform length
    DBuf tune_buf, tune_src;
    int chain_variant(int Mx, int Kx, int s0, int ns, long long plane, const C *Gp, const int *extx) {
        if (Mx != 32 && Mx != 64 && Mx != 128 && Mx != 192 && Mx != 256) return 0;
        auto it = chain_tuned.find(Mx);
        if (it != chain_tuned.end()) return it->second.variant;
        // HG_CHAIN_VARIANT=v: use variant v untimed (the tests run every variant this way)
        if (const char *fv = std::getenv("HG_CHAIN_VARIANT")) {
            const int v = std::atoi(fv);
            HG_REQUIRE(v >= 0 && v < kNumChainVariants && chain_variant_exists(Mx, v),
                       "HG_CHAIN_VARIANT names no chain variant for this transform length");
            chain_tuned[Mx] = Tuned{v, std::vector<float>(kNumChainVariants, 0.f)};
            return v;
        }
        const size_t per_shell = sizeof(C) * (size_t)Kx * plane;
        const int nsh = (int)std::max<size_t>(1, std::min<size_t>((size_t)ns, (2ull << 30) / per_shell));
        const size_t bytes = per_shell * nsh;
        HG_CK(tune_src.ensure(bytes));
        HG_CK(tune_buf.ensure(bytes));
        HG_CK(cudaMemcpyAsync(tune_src.p, T2.p, bytes, cudaMemcpyDeviceToDevice, st));
        Tuned tu{0, std::vector<float>(kNumChainVariants, 0.f)};
        float best = 1e30f;
        for (int v = 0; v < kNumChainVariants; v++) {
            if (!chain_variant_exists(Mx, v)) {
                tu.ms[v] = 0.f;
                continue;
            }
            for (int rep = 0; rep < 2; rep++) {
                HG_CK(cudaMemcpyAsync(tune_buf.p, tune_src.p, bytes, cudaMemcpyDeviceToDevice, st));
                HG_CK(cudaEventRecord(ev0, st));
                HG_CK(launch_chain_x_any(Mx, v, dp<C>(tune_buf), Gp, nsh, Kx, s0, plane, extx));
                HG_CK(cudaEventRecord(ev1, st));
            }
            HG_CK(cudaEventSynchronize(ev1));
            float ms = 0.f;
            HG_CK(cudaEventElapsedTime(&ms, ev0, ev1));
            tu.ms[v] = ms;
            if (ms < best) {
                best = ms;
                tu.variant = v;
            }
        }
        HG_CK(cudaEventRecord(ev0, st));  // begin()'s event, reused above: statistics time from here
        tune_buf.release();
        tune_src.release();
        chain_tuned[Mx] = tu;
        return tu.variant;
    }
    std::string tuning() override {
        std::string out;
        char line[256];
        for (const auto &kv : chain_tuned) {
            const ChainVariant &cv = kChainVariants[kv.second.variant];
            snprintf(line, sizeof(line), "chain_x L=%d %s: variant %d (%s, B=%d, G %s, %s, %s)", kv.first,
                     sizeof(T) == 8 ? "fp64" : "fp32", kv.second.variant,
                     cv.v12 ? "12 values per thread"
                            : (cv.xr == 1   ? "two-level register transform, exchange in rounds"
                               : cv.xr == 2 ? "two-level register transform, exchange in half rounds"
                                            : "two-level register transform"),
                     cv.B,
                     cv.gs ? "staged in shared memory" : "read from L2", cv.pf ? "cp.async prefetch" : "no prefetch",
                     cv.minb ? ("register cap for " + std::to_string(cv.minb) + " CTAs per SM").c_str()
                             : "default register budget");
            out += line;
            for (size_t v = 0; v < kv.second.ms.size(); v++) {
                snprintf(line, sizeof(line), "%s%.4f", v ? " " : "; ms per variant: ", kv.second.ms[v]);
                out += line;
            }
            out += "\n";
        }
        if (hi) out += hi->tuning();
        return out;
    }

    // Q_b[j] for the bispectrum shells with the G of key gk
    const C *family_Q(const Fam &b, const GK &gk) {
        const FQ key{b.l, b.m, gk.first, gk.second};
        auto &qp = famQ[key];
        if (!qp) qp = std::make_unique<DBuf>();
        DBuf &Q = *qp;
        if (famQ_ok.count(key)) return dp<C>(Q);
        const ChainGeo S = bk_geo();
        const DBuf &Gsrc = ensure_G(gk);
        const double2 *A = family_A(b);
        const long long cv = cube_vol();
        HG_CK(Ac.ensure(sizeof(C) * cv * S.ns));
        HG_CK(Q.ensure(sizeof(C) * cv * S.ns));
        HG_CK(cudaMemsetAsync(Ac.p, 0, sizeof(C) * cv * S.ns, st));
        kb("scatter_entries", double(n_ent()) * (16.0 + sizeof(C)));
        k_scatter_cube<T><<<grid1(n_ent(), 256), 256, 0, st>>>(dp<ShellEnt>(shells.d_ent), n_ent(), A,
                                                               make_int3(S.K[0], S.K[1], S.K[2]),
                                                               make_int3(S.s[0], S.s[1], S.s[2]), dp<C>(Ac));
        ke();
        run_chain(S, Gsrc, dp<C>(Q));
        famQ_ok.insert(key);
        return dp<C>(Q);
    }

    // pair matrix P[i][j] = sum_{e in shell i} A_a[e] Q_b,j(-n_e)  (complex, [ns][ns])
    const std::vector<double> &pair_matrix(const Fam &a, const Fam &b, const GK &gk) {
        auto key = std::make_tuple(a.l, a.m, b.l, b.m, gk.first, gk.second);
        auto it = pairs.find(key);
        if (it != pairs.end()) return it->second;
        const ShellSet &S = shells;
        const double2 *A = family_A(a);
        const C *Q = family_Q(b, gk);
        HG_CK(pair_out.ensure(sizeof(double2) * S.ns * S.ns));
        HG_CK(pair_part.ensure(sizeof(double2) * (size_t)std::max(1, S.nitems) * S.ns));
        kb("pair_dot", double(n_ent()) * (S.ns * sizeof(C) + 32.0));
        if (S.nitems)
            k_pair_dot_items<T><<<(unsigned)((S.nitems + 7) / 8), 256, 0, st>>>(
                dp<PairItem>(S.d_items), S.nitems, dp<ShellEnt>(shells.d_ent), A, Q, make_int3(S.K[0], S.K[1], S.K[2]),
                make_int3(S.M[0], S.M[1], S.M[2]), make_int3(S.s[0], S.s[1], S.s[2]), S.ns, dp<double2>(pair_part));
        k_pair_sum_items<<<grid1(32LL * S.ns * S.ns, 256), 256, 0, st>>>(dp<int>(S.d_istart), dp<double2>(pair_part),
                                                                           S.ns, S.ns, dp<double2>(pair_out));
        ke();
        std::vector<double> h(2 * S.ns * S.ns);
        HG_CK(cudaMemcpyAsync(h.data(), pair_out.p, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, st));
        HG_CK(cudaStreamSynchronize(st));
        pairs[key] = h;
        return pairs[key];
    }

    // sum_x F_a,i F_b,j G (without dV) for all (i, j): chain on b, or on a transposed.
    std::vector<double> triple_sum(const Fam &a, const Fam &b, const GK &gk, const std::set<FQ> &chains) {
        const int ns = shells.ns;
        if (chains.count(FQ{b.l, b.m, gk.first, gk.second})) return pair_matrix(a, b, gk);
        const auto &P = pair_matrix(b, a, gk);
        std::vector<double> r(2 * ns * ns);
        for (int i = 0; i < ns; i++)
            for (int j = 0; j < ns; j++) {
                r[2 * (i * ns + j)] = P[2 * (j * ns + i)];
                r[2 * (i * ns + j) + 1] = P[2 * (j * ns + i) + 1];
            }
        return r;
    }

    void prepare_shells() {
        build_shells();
        HG_REQUIRE(n_ent() > 0, "no Fourier modes fall inside the k shells");
        if (!shD_valid) {
            if (src_kind == 0) narrow_density();  // dsrc is the box density
            HG_CK(shD.ensure(sizeof(double2) * n_ent()));
            kb("shell_D", double(n_ent()) * (16.0 + sizeof(C)));
            k_shell_D<T><<<grid1(n_ent(), 256), 256, 0, st>>>(dp<ShellEnt>(shells.d_ent), n_ent(), dsrc.s, g, tabs,
                                                              wpow, dp<double2>(shD));
            ke();
            shD_valid = true;
        }
    }

    // ------------------------------------------------------------------ shot noise (xi)
    bool equal_cells() const {
        return std::fabs(g.dr[0] - g.dr[1]) <= 1e-12 * g.dr[0] && std::fabs(g.dr[0] - g.dr[2]) <= 1e-12 * g.dr[0];
    }
    void build_orbits() {
        if (nkey > 0) return;
        n2dim = 0;
        for (int a = 0; a < 3; a++) n2dim += (long long)(g.n[a] / 2) * (g.n[a] / 2);
        n2dim += 1;
        xi_general = !(equal_cells() && fft_supported_length(g.n[2]));
        if (xi_general) {
            build_octant_keys();
            return;
        }
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
                // representatives: one line of each mirror pair (x, y) <-> (-x, -y) (the set
                // is closed under the mirror), with its mirror
                int k = 0;
                for (int l : ls) {
                    const int ix = l / ny, iy = l % ny;
                    const int m = ((nx - ix) % nx) * ny + (ny - iy) % ny;
                    HG_REQUIRE(ls.count(m), "orbit not closed under the mirror");
                    if (l > m) continue;
                    HG_REQUIRE(k < 4, "more than four representative lines in an orbit");
                    orbit_lines.push_back(l);
                    orbit_lines.push_back(m);
                    k++;
                }
                for (; k < 4; k++) {
                    orbit_lines.push_back(-1);
                    orbit_lines.push_back(-1);
                }
                orbit_n2xy.push_back(wx * wx + wy * wy);
            }
        HG_CK(d_orbit_lines.ensure(sizeof(int) * orbit_lines.size()));
        HG_CK(cudaMemcpy(d_orbit_lines.p, orbit_lines.data(), sizeof(int) * orbit_lines.size(), cudaMemcpyHostToDevice));
        HG_CK(d_orbit_n2xy.ensure(sizeof(int) * orbit_n2xy.size()));
        HG_CK(cudaMemcpy(d_orbit_n2xy.p, orbit_n2xy.data(), sizeof(int) * orbit_n2xy.size(), cudaMemcpyHostToDevice));
        // keys n2: |r| = sqrt(n2 dr^2), cells per n2 from the per-axis counts of w^2
        nkey = n2dim;
        key_r.assign(nkey, 0.0);
        const double dr = g.dr[0];
        for (long long q = 0; q < nkey; q++) key_r[q] = std::sqrt(double(q) * (dr * dr));
        std::vector<std::vector<double>> c1(3);
        for (int a = 0; a < 3; a++) {
            const int h = g.n[a] / 2;
            c1[a].assign((size_t)h * h + 1, 0.0);
            for (int i = 0; i < g.n[a]; i++) {
                const int w = wrap_index(i, g.n[a]);
                c1[a][(size_t)w * w] += 1.0;
            }
        }
        key_cells.assign(nkey, 0.0);
        for (size_t a = 0; a < c1[0].size(); a++) {
            if (c1[0][a] == 0.0) continue;
            for (size_t b = 0; b < c1[1].size(); b++) {
                if (c1[1][b] == 0.0) continue;
                for (size_t c = 0; c < c1[2].size(); c++)
                    if (c1[2][c] != 0.0) key_cells[a + b + c] += c1[0][a] * c1[1][b] * c1[2][c];
            }
        }
    }
    // octant keys (a, b, c), 0 <= a <= n0/2 ...: |r| as the reference forms it per cell,
    // sqrt(rx^2 + ry^2 + rz^2) with r_axis = (i < n/2 ? i : i - n) dr_axis (field.hpp:1040-1050)
    void build_octant_keys() {
        const int h0 = g.n[0] / 2 + 1, h1 = g.n[1] / 2 + 1, h2 = g.n[2] / 2 + 1;
        nkey = (long long)h0 * h1 * h2;
        key_r.assign(nkey, 0.0);
        key_cells.assign(nkey, 0.0);
        auto comp = [&](int a, int i) {  // the component of the octant's representative cell
            const int n = g.n[a];
            return double(i < n / 2 ? i : i - n) * g.dr[a];
        };
        auto mult = [&](int a, int i) { return (i == 0 || 2 * i == g.n[a]) ? 1.0 : 2.0; };
        for (int a = 0; a < h0; a++)
            for (int b = 0; b < h1; b++)
                for (int c = 0; c < h2; c++) {
                    const long long q = ((long long)a * h1 + b) * h2 + c;
                    const double rx = comp(0, a), ry = comp(1, b), rz = comp(2, c);
                    key_r[q] = std::sqrt(rx * rx + ry * ry + rz * rz);
                    key_cells[q] = mult(0, a) * mult(1, b) * mult(2, c);
                }
        HG_CK(d_keyr.ensure(sizeof(double) * nkey));
        HG_CK(cudaMemcpy(d_keyr.p, key_r.data(), sizeof(double) * nkey, cudaMemcpyHostToDevice));
    }
    // hist[h][key] of the transformed correlation field in xi (a full [n0][n1][n2] array)
    void fold_hist(const HistSpec &hs, bool poly, double *hist) {
        const unsigned blocks = (unsigned)std::min<long long>(grid1(nkey, 128), 148 * 16);
        kb("xi_fold", double(g.ntot) * sizeof(C));
        if (poly)
            k_xi_fold<T, true><<<blocks, 128, 0, st>>>(dp<C>(xi), g.n[0], g.n[1], g.n[2], g.dr[0], g.dr[1], g.dr[2], hs,
                                                       nkey, hist);
        else
            k_xi_fold<T, false><<<blocks, 128, 0, st>>>(dp<C>(xi), g.n[0], g.n[1], g.n[2], g.dr[0], g.dr[1], g.dr[2],
                                                        hs, nkey, hist);
        ke();
    }

    // a survey correlation-field spectrum (complex) synthesised into xi, then its x pass in place
    template <class LD>
    void xi_x_pass(const LD &ld) {
        const long long yz = (long long)g.n[1] * g.n[2];
        unsigned blocks = (unsigned)std::min<long long>(grid1(g.ntot, 256), 148 * 16);
        kb("xi_synth", double(g.ntot) * sizeof(C) * 1.5);
        k_synth<T, LD><<<blocks, 256, 0, st>>>(ld, g.n[0], yz, dp<C>(xi));
        ke();
        pass<+1>(g.n[0], LdArr<T>{dp<C>(xi), g.n[0], yz}, StArr<T>{dp<C>(xi), g.n[0], yz}, 1, yz, "fft_xi_x");
    }

    // Box correlation field after its x and y inverse passes (cached per catalogue).  Its
    // spectrum P is real, so the even and odd kz planes travel as the real and imaginary
    // parts of one complex field (k_synth_pairs_rows: [n0][n1][n2/2] in xi): half the data
    // through the x and y passes; the histogram kernel separates them before its z pass.
    // k0prod: (f1 conj f2)(k = 0), delta0 N0 for the bispectrum shot noise (dn against the
    // density N, bispec.hpp:913-921), delta0^2 for the 2PCF (dn against itself)
    void ensure_xi() { ensure_xi(delta0 * N0); }
    void ensure_xi(double k0prod) {
        build_orbits();
        if (xi_valid && xi_k0 == k0prod) return;
        if (H_wide)  // the FP64 engine's density: |delta|^2 formed from it, not from a narrowed copy
            build_box_xi(Spec<double>{H_wide, g.n[0], g.n[1], g.n[2], 1}, double(slot[0].n), k0prod);
        else
            build_box_xi(half_spec(), double(slot[0].n), k0prod);
        xi_k0 = k0prod;
        xi_valid = true;
    }

    // The box correlation field of a real field's half spectrum f, (|f|^2 - S C) / W^2 / V,
    // after its x and y inverse passes, into xi (even and odd kz planes as one complex field)
    template <typename SE>
    void build_box_xi(const Spec<SE> &f, double S, double k0prod) {
        const int n0 = g.n[0], n1 = g.n[1], n2 = g.n[2], nh = n2 / 2;
        HG_CK(xi.ensure(sizeof(C) * g.ntot));
        const double invV = 1.0 / g.volume;  // field.hpp:1122
        LdXiHat<T, SE> ld{f, n2, xtabs, S, k0prod, invV};
        if (xi_general) {  // the whole complex field, all three inverse passes (fold_hist reads it)
            xi_x_pass(LdXiHatFull<T, SE>{ld});
            pass<+1>(n1, LdArr<T>{dp<C>(xi), n1, n2}, StArr<T>{dp<C>(xi), n1, n2}, n0, n2, "fft_xi_y");
            pass<+1>(n2, LdArr<T>{dp<C>(xi), n2, 1}, StArr<T>{dp<C>(xi), n2, 1}, (long long)n0 * n1, 1, "fft_xi_z",
                     double(g.ntot) * sizeof(C) * 2.0);
            return;
        }
        const long long yz = (long long)n1 * nh, tot = (long long)n0 * yz;
        const int bs = (int)std::min<long long>(256, (nh + 31) / 32 * 32);
        kb("xi_synth", double(tot) * (sizeof(C) + sizeof(cplx<SE>)));
        HG_REQUIRE(f.half, "the box correlation field is synthesised from a half spectrum");
        k_synth_pairs_rows<T, SE><<<dim3(n1, n0 / 2 + 1), bs, 0, st>>>(ld, n0, n1, nh, dp<C>(xi));
        ke();
        pass<+1>(n0, LdArr<T>{dp<C>(xi), n0, yz}, StArr<T>{dp<C>(xi), n0, yz}, 1, yz, "fft_xi_x");
        pass<+1>(n1, LdArr<T>{dp<C>(xi), n1, nh}, StArr<T>{dp<C>(xi), n1, nh}, n0, nh, "fft_xi_y");
    }

    // the box histograms of the current correlation field (hs.nh of them, [h][key], written
    // whole): the orbit kernel on its equal-cell power-of-two meshes, the fold otherwise
    void box_hist(const HistSpec &hs, double *hist) {
        if (xi_general) {
            fold_hist(hs, true, hist);
            return;
        }
        HG_CK(cudaMemsetAsync(hist, 0, sizeof(double) * 2 * nkey * hs.nh, st));
        launch_orbit(g.n[2], hs, (int)orbit_n2xy.size(), hist);
    }

    template <int L>
    void launch_orbit_L(const HistSpec &hs, int n_orb, double *hist) {
        size_t smem = OrbitCfg<T, L>::smem();
        HG_CK(cudaFuncSetAttribute(k_xi_orbit_hist<T, L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        const C *twp = twiddles(L);
        kb("xi_orbit_hist", double(g.ntot / 2) * sizeof(C));
        const int nblk = (n_orb + 1) / 2;
        k_xi_orbit_hist<T, L><<<nblk, OrbitCfg<T, L>::NT, smem, st>>>(
            dp<C>(xi), dp<int2>(d_orbit_lines), dp<int>(d_orbit_n2xy), n_orb, twp, hs, n2dim, hist);
        ke();
    }
    void launch_orbit(int L, const HistSpec &hs, int n_orb, double *hist) {
        switch (L) {
            case 8: launch_orbit_L<8>(hs, n_orb, hist); break;
            case 16: launch_orbit_L<16>(hs, n_orb, hist); break;
            case 32: launch_orbit_L<32>(hs, n_orb, hist); break;
            case 64: launch_orbit_L<64>(hs, n_orb, hist); break;
            case 128: launch_orbit_L<128>(hs, n_orb, hist); break;
            case 256: launch_orbit_L<256>(hs, n_orb, hist); break;
            case 512: launch_orbit_L<512>(hs, n_orb, hist); break;
            case 1024: launch_orbit_L<1024>(hs, n_orb, hist); break;
            default: throw HgError{"unsupported n_mesh_z"};
        }
    }

    // (m1, m2) combinations with M = 0 and |w| >= 1e-10 (bispec.hpp:923-931)
    struct Combo {
        int m1, m2;
        double w;
    };
    static std::vector<Combo> combos_of(const MP &mp) {
        std::vector<Combo> out;
        double w000 = wigner3j(mp.l1, mp.l2, mp.L, 0, 0, 0);
        for (int m1 = -mp.l1; m1 <= mp.l1; m1++)
            for (int m2 = -mp.l2; m2 <= mp.l2; m2++) {
                double w = w000 * wigner3j(mp.l1, mp.l2, mp.L, m1, m2, 0);
                w *= double(2 * mp.L + 1) * double(2 * mp.l1 + 1) * double(2 * mp.l2 + 1);
                if (std::fabs(w) < 1.0e-10) continue;
                out.push_back({m1, m2, w});
            }
        return out;
    }

    // Chebyshev coefficients of f_h(mu) = sum_terms w Yhat_l1m1 Yhat_l2m2 at (sqrt(1 - mu^2), 0, mu)
    // (real for m1 + m2 = 0, a polynomial of degree l1 + l2): interpolation at deg + 1 nodes
    static void orbit_weight_poly(HistSpec &hs, int h) {
        int D = 0;
        double f0 = 0.0;
        for (int q = 0; q < hs.nterm[h]; q++) {
            D = std::max(D, hs.term[h][q].l1 + hs.term[h][q].l2);
            if (hs.term[h][q].l1 == 0 && hs.term[h][q].l2 == 0) f0 += hs.term[h][q].w;
        }
        HG_REQUIRE(D < HG_CHEB, "multipole degree too large for the shot-noise weight polynomial");
        std::vector<double> fk(D + 1);
        for (int k = 0; k <= D; k++) {
            const double mu = std::cos(HG_PI * (k + 0.5) / double(D + 1));
            const double sx = std::sqrt(std::max(0.0, 1.0 - mu * mu));
            double f = 0.0;
            for (int q = 0; q < hs.nterm[h]; q++) {
                const YTerm &yt = hs.term[h][q];
                zd y1 = ylm_reduced(yt.l1, yt.m1, sx, 0.0, mu), y2 = ylm_reduced(yt.l2, yt.m2, sx, 0.0, mu);
                f += yt.w * (y1.x * y2.x - y1.y * y2.y);
            }
            fk[k] = f;
        }
        for (int j = 0; j <= D; j++) {
            double c = 0.0;
            for (int k = 0; k <= D; k++) c += fk[k] * std::cos(HG_PI * j * (k + 0.5) / double(D + 1));
            hs.cheb[h][j] = c * 2.0 / double(D + 1) * (j == 0 ? 0.5 : 1.0);
        }
        hs.deg[h] = D;
        hs.f0[h] = f0;
    }

    // hist_mp[mp][n2] = sum over cells with |x/dr|^2 = n2 of xi(x) sum_combos w Yhat1 Yhat2
    void ensure_histograms(const std::vector<MP> &mps) {
        ensure_xi();
        std::vector<MP> todo;
        for (const auto &mp : mps) {
            std::array<int, 3> key{mp.l1, mp.l2, mp.L};
            bool queued = false;
            for (const auto &q : todo) queued |= (q.l1 == mp.l1 && q.l2 == mp.l2 && q.L == mp.L);
            if (!hist_ok.count(key) && !queued) todo.push_back(mp);
        }
        for (size_t t0 = 0; t0 < todo.size(); t0 += HG_MAX_HIST) {
            HistSpec hs;
            memset(&hs, 0, sizeof(hs));
            hs.nh = (int)std::min<size_t>(HG_MAX_HIST, todo.size() - t0);
            for (int h = 0; h < hs.nh; h++) {
                const MP &mp = todo[t0 + h];
                hs.parity[h] = ((mp.l1 + mp.l2) % 2 == 0) ? 1 : -1;
                auto cs = combos_of(mp);
                HG_REQUIRE(cs.size() <= 12, "too many (m1, m2) terms in one multipole");
                for (const auto &c : cs) hs.term[h][hs.nterm[h]++] = YTerm{mp.l1, c.m1, mp.l2, c.m2, c.w};
                orbit_weight_poly(hs, h);
            }
            HG_CK(hist_tmp.ensure(sizeof(double) * 2 * nkey * hs.nh));
            box_hist(hs, dp<double>(hist_tmp));
            for (int h = 0; h < hs.nh; h++) {
                const MP &mp = todo[t0 + h];
                std::array<int, 3> key{mp.l1, mp.l2, mp.L};
                auto &p = hist_mp[key];
                if (!p) p = std::make_unique<DBuf>();
                HG_CK(p->ensure(sizeof(double) * 2 * nkey));
                HG_CK(cudaMemcpyAsync(p->p, dp<double>(hist_tmp) + 2 * nkey * h, sizeof(double) * 2 * nkey,
                                      cudaMemcpyDeviceToDevice, st));
                hist_ok.insert(key);
            }
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

    // J_l[i][n2] = j_l(kbin[i] * dr sqrt(n2)) (geometry only: cached for the context)
    const double *jtab(int l) {
        auto it = jtab_k.find(l);
        if (it != jtab_k.end()) return dp<double>(*it->second);
        const BesselSpline &s = spline(l);
        auto &sp = d_splines[l];
        HG_CK(d_kv.ensure(sizeof(double) * kbin.size()));
        HG_CK(cudaMemcpyAsync(d_kv.p, kbin.data(), sizeof(double) * kbin.size(), cudaMemcpyHostToDevice, st));
        auto J = std::make_unique<DBuf>();
        HG_CK(J->ensure(sizeof(double) * kbin.size() * nkey));
        long long tot = (long long)kbin.size() * nkey;
        kb("bessel_table", double(tot) * 8.0);
        if (xi_general)  // the octant keys' radii
            k_bessel_table_r<<<grid1(tot, 256), 256, 0, st>>>(dp<double>(*sp.first), dp<double>(*sp.second), s.n,
                                                              s.xmin, s.dx, dp<double>(d_kv), (int)kbin.size(),
                                                              dp<double>(d_keyr), nkey, dp<double>(*J));
        else
            k_bessel_table<<<grid1(tot, 256), 256, 0, st>>>(dp<double>(*sp.first), dp<double>(*sp.second), s.n,
                                                            s.xmin, s.dx, dp<double>(d_kv), (int)kbin.size(), g.dr[0],
                                                            n2dim, dp<double>(*J));
        ke();
        HG_CK(cudaStreamSynchronize(st));
        const double *p = dp<double>(*J);
        jtab_k[l] = std::move(J);
        return p;
    }

    // ------------------------------------------------------------------ bispectrum (box)
    // bispec.hpp:877-1203 for all k1 rows of several multipoles at once.
    // (m1, m2, M) combinations with |w| >= 1e-10, w = (2L+1)(2l1+1)(2l2+1) w3j(l1 l2 L; 0 0 0)
    // w3j(l1 l2 L; m1 m2 M): M = 0 only for the box (bispec.hpp:1129-1136), every M for the
    // survey (bispec.hpp:255-270).
    struct Combo3 {
        int m1, m2, M;
        double w;
    };
    static std::vector<Combo3> combos3(const MP &mp, bool all_M) {
        std::vector<Combo3> out;
        const double w000 = wigner3j(mp.l1, mp.l2, mp.L, 0, 0, 0);
        for (int m1 = -mp.l1; m1 <= mp.l1; m1++)
            for (int m2 = -mp.l2; m2 <= mp.l2; m2++)
                for (int M = all_M ? -mp.L : 0; M <= (all_M ? mp.L : 0); M++) {
                    double w = w000 * wigner3j(mp.l1, mp.l2, mp.L, m1, m2, M);
                    w *= double(2 * mp.L + 1) * double(2 * mp.l1 + 1) * double(2 * mp.l2 + 1);
                    if (std::fabs(w) < 1.0e-10) continue;
                    out.push_back({m1, m2, M, w});
                }
        return out;
    }

    // (m1, m2, M) terms over every M for the survey sources, M = 0 for the box ones (the
    // reconstructed box included: its particles' Yhat_LM(z) vanish for M != 0)
    bool all_M() const { return src_kind == 1 || src_kind == 2; }
    // the G field of an (L, M) term: G_LM for the survey sources, the one G of the box
    // (and of the reconstructed box, whose (L, 0) fields are all the (0, 0) one)
    GK g_key(int L, int M) const { return all_M() ? GK{L, M} : GK{0, 0}; }

    static void check_multipoles(const std::vector<MP> &mps) {
        HG_REQUIRE(!mps.empty(), "no multipoles requested");
        for (const auto &mp : mps) {
            HG_REQUIRE(mp.l1 >= 0 && mp.l2 >= 0 && mp.L >= 0, "ell1, ell2, ELL must be >= 0");
            HG_REQUIRE(std::fabs(wigner3j(mp.l1, mp.l2, mp.L, 0, 0, 0)) >= 1.0e-10,
                       "This multipole combination is not allowed: wigner_3j(ell1, ell2, ELL, 0,0,0) == 0");
        }
    }

    // B_raw[q] for every (k1, k2): sum over (m1, m2, M) of w dV sum_x F1 F2 G_LM
    // (bispec.hpp:1118-1170 box, 255-320 survey), [q][ns][ns] complex.  Chain families:
    // every self-paired family per G key, then a greedy cover of the remaining pairs.
    std::vector<std::vector<double>> bk_main(const std::vector<MP> &mps) {
        prepare_shells();
        const int ns = shells.ns;
        const double dV = g.volume / double(g.ntot);
        const double red = double(g.ntot) / (double(shells.M[0]) * shells.M[1] * shells.M[2]);
        std::vector<std::vector<Combo3>> cmb;
        std::map<GK, std::set<std::pair<Fam, Fam>>> upairs;
        for (const auto &mp : mps) {
            cmb.push_back(combos3(mp, all_M()));
            for (const auto &c : cmb.back()) {
                Fam a{mp.l1, c.m1}, b{mp.l2, c.m2};
                GK gk = g_key(mp.L, c.M);
                upairs[gk].insert(b < a ? std::make_pair(b, a) : std::make_pair(a, b));
            }
        }
        std::set<FQ> chains(famQ_ok.begin(), famQ_ok.end());
        for (const auto &kv : upairs) {
            const GK &gk = kv.first;
            auto has = [&](const Fam &f) { return chains.count(FQ{f.l, f.m, gk.first, gk.second}) > 0; };
            for (const auto &p : kv.second)
                if (!(p.first < p.second) && !(p.second < p.first))
                    chains.insert(FQ{p.first.l, p.first.m, gk.first, gk.second});
            while (true) {
                std::map<Fam, int> score;
                for (const auto &p : kv.second) {
                    if (has(p.first) || has(p.second)) continue;
                    score[p.first]++;
                    score[p.second]++;
                }
                if (score.empty()) break;
                Fam best = score.begin()->first;
                int bs = -1;
                for (const auto &sc : score)
                    if (sc.second > bs) {
                        bs = sc.second;
                        best = sc.first;
                    }
                chains.insert(FQ{best.l, best.m, gk.first, gk.second});
            }
        }
        std::vector<std::vector<double>> B(mps.size(), std::vector<double>(2 * ns * ns, 0.0));
        for (size_t q = 0; q < mps.size(); q++)
            for (const auto &c : cmb[q]) {
                GK gk = g_key(mps[q].L, c.M);
                std::vector<double> t = triple_sum(Fam{mps[q].l1, c.m1}, Fam{mps[q].l2, c.m2}, gk, chains);
                for (int e = 0; e < 2 * ns * ns; e++) B[q][e] += c.w * (dV * red * t[e]);
            }
        return B;
    }

    // SN += i^(l1+l2) dV sum_n2 J_l1(k1 r) J_l2(k2 r) hist(n2)  (bispec.hpp:1036-1060): the
    // skinny product J1 diag(hist) J2^T in row blocks, [ns][ns] complex
    void bk_sn_xi(const MP &mp, const double *hq, std::vector<double> &SNq) {
        // (l2, l1, L) has the same shot-noise weights as (l1, l2, L) (the 3j symbols change by
        // (-1)^(l1 + l2 + L) = 1), hence the same histogram, and its matrix is the transpose
        const int ns = cfg.n_kbin;
        auto sw = sn_xi_cache.find({mp.l2, mp.l1, mp.L});
        if (src_kind == 0 && mp.l1 != mp.l2 && sw != sn_xi_cache.end() && sw->second.first == src_kind) {
            const std::vector<double> &Tr = sw->second.second;
            for (int i1 = 0; i1 < ns; i1++)
                for (int i2 = 0; i2 < ns; i2++) {
                    SNq[2 * (i1 * ns + i2)] += Tr[2 * (i2 * ns + i1)];
                    SNq[2 * (i1 * ns + i2) + 1] += Tr[2 * (i2 * ns + i1) + 1];
                }
            return;
        }
        std::vector<double> add(2 * ns * ns, 0.0);
        bk_sn_xi_compute(mp, hq, add);
        for (size_t e = 0; e < add.size(); e++) SNq[e] += add[e];
        sn_xi_cache[{mp.l1, mp.l2, mp.L}] = {src_kind, std::move(add)};
    }
    // xi-term matrices of this catalogue by (l1, l2, L), with the source kind they came from
    std::map<std::array<int, 3>, std::pair<int, std::vector<double>>> sn_xi_cache;

    void bk_sn_xi_compute(const MP &mp, const double *hq, std::vector<double> &SNq) {
        const int ns = cfg.n_kbin;
        const double dV = g.volume / double(g.ntot);
        HG_CK(snmat.ensure(sizeof(double2) * ns * ns));
        const double *J1 = jtab(mp.l1);
        const double *J2 = jtab(mp.l2);
        const int nblk = sn_partial_blocks(nkey);
        const int rb = std::min(ns, HG_SN_MAXROWS);
        HG_CK(sn_part.ensure(sizeof(double) * 2 * (size_t)nblk * rb * rb));
        HG_CK(snblk.ensure(sizeof(double2) * (size_t)rb * rb));
        for (int a0 = 0; a0 < ns; a0 += rb)
            for (int b0 = 0; b0 < ns; b0 += rb) {
                const int na = std::min(rb, ns - a0), nb = std::min(rb, ns - b0);
                const size_t smem = sn_partial_smem(na, nb);
                HG_CK(cudaFuncSetAttribute(k_sn_partial, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
                kb("sn_matrix", double(na + 2 * nb + 2) * nkey * 8.0);
                k_sn_partial<<<nblk, HG_SN_THREADS, smem, st>>>(J1 + (size_t)a0 * nkey, na, J2 + (size_t)b0 * nkey,
                                                                nb, hq, nkey, dp<double>(sn_part));
                ke();
                kb("sn_matrix", double(nblk) * na * nb * 16.0);
                k_sum_parts<<<grid1(sum_parts_threads((long long)na * nb), 256), 256, 0, st>>>(dp<double>(sn_part), nblk, na * nb,
                                                                              dp<double2>(snblk));
                ke();
                // place the (a0, b0) block into the ns x ns matrix
                HG_CK(cudaMemcpy2DAsync(dp<double2>(snmat) + (size_t)a0 * ns + b0, sizeof(double2) * ns, snblk.p,
                                        sizeof(double2) * nb, sizeof(double2) * nb, na, cudaMemcpyDeviceToDevice, st));
            }
        std::vector<double> sd(2 * ns * ns);
        HG_CK(cudaMemcpyAsync(sd.data(), snmat.p, sizeof(double) * sd.size(), cudaMemcpyDeviceToHost, st));
        HG_CK(cudaStreamSynchronize(st));
        const int p4 = (mp.l1 + mp.l2) % 4;
        for (int e = 0; e < ns * ns; e++) {
            double re = sd[2 * e] * dV, im = sd[2 * e + 1] * dV;
            double rr = p4 == 0 ? re : p4 == 1 ? -im : p4 == 2 ? -re : im;
            double ii = p4 == 0 ? im : p4 == 1 ? re : p4 == 2 ? -im : -re;
            SNq[2 * e] += rr;
            SNq[2 * e + 1] += ii;
        }
    }

    void bk_box_multi(const std::vector<MP> &mps, int ith, double *bk_save, double *sn_save, double *norm) override {
        check_multipoles(mps);
        HG_REQUIRE(ith >= -1 && ith < cfg.n_kbin, "ith_kbin out of range");
        begin();
        set_source(0, 0.0);
        const int ns = cfg.n_kbin;
        const double Np = double(slot[0].n);
        std::vector<std::vector<double>> B, SN;
        if (hi && (fp64_stages & HG_STAGE_BK_SIGNAL)) {
            hi_density();
            B = hi->stage_bk_signal(mps);
        } else {
            B = bk_main(mps);
        }
        if (hi && (fp64_stages & HG_STAGE_BK_SHOT)) {
            hi_density();
            SN = hi->stage_bk_shot(mps);
        } else {
            SN = bk_shot(mps);
        }
        if (hi) launches += hi->stage_take_launches();
        const int r0 = (ith < 0) ? 0 : ith, r1 = (ith < 0) ? ns : ith + 1;
        const int rows = r1 - r0;
        for (size_t q = 0; q < mps.size(); q++)
            for (int i1 = r0; i1 < r1; i1++)
                for (int i2 = 0; i2 < ns; i2++) {
                    long long o = ((long long)q * rows + (i1 - r0)) * ns + i2;
                    bk_save[2 * o] = B[q][2 * (i1 * ns + i2)];
                    bk_save[2 * o + 1] = B[q][2 * (i1 * ns + i2) + 1];
                    sn_save[2 * o] = SN[q][2 * (i1 * ns + i2)];
                    sn_save[2 * o + 1] = SN[q][2 * (i1 * ns + i2) + 1];
                }
        if (norm) {
            double nv = g.volume / Np / Np;
            nv *= (g.volume / Np);
            *norm = nv;
        }
        end();
    }

    // box P_l bin averages [nbin][ells] complex (before the 2l + 1 factor) of the current
    // density, from the engine that computed it
    std::vector<double> pk_terms(const std::vector<int> &ells) {
        if (hi && (fp64_stages & HG_STAGE_DENSITY)) return hi->stage_pk_terms(ells);
        return stage_pk_terms(ells);
    }

    // the current box density on the FP64 engine: its own (HG_STAGE_DENSITY) or this one's
    // spectrum widened
    void hi_density() {
        if (!hi->stage_density_ready()) hi->stage_import_density(H.p, sizeof(T) == 8, delta0, N0, dens_mass);
    }

    // Box bispectrum shot noise (bispec.hpp:909-1078) of the current source: constant and P
    // terms, then the correlation-field term; [q][ns][ns] complex, all rows.
    std::vector<std::vector<double>> bk_shot(const std::vector<MP> &mps) {
        const int ns = cfg.n_kbin;
        const double Np = double(slot[0].n);
        std::vector<std::vector<Combo>> cmb;
        for (const auto &mp : mps) cmb.push_back(combos_of(mp));
        // shot noise (bispec.hpp:909-1078): P terms, constant term, xi term
        std::vector<LM> lms;
        std::vector<std::vector<int>> lm_idx(mps.size());
        for (size_t q = 0; q < mps.size(); q++)
            for (const auto &c : cmb[q]) {
                if (mps[q].l2 == 0) {
                    lm_idx[q].push_back((int)lms.size());
                    lms.push_back(LM{mps[q].l1, c.m1});
                }
                if (mps[q].l1 == 0) {
                    lm_idx[q].push_back((int)lms.size());
                    lms.push_back(LM{mps[q].l2, c.m2});
                }
            }
        const int nl = (int)lms.size();
        std::vector<double> avg(2 * ns * std::max(nl, 1), 0.0);
        std::vector<unsigned long long> nm;
        bool m0 = true;
        for (const LM &x : lms) m0 = m0 && x.m == 0;
        if (m0 && nl > 0) {
            // every term is a box P_l bin (m = 0, S = N): the P cache of this density, on the
            // FP64 engine when it computed the density
            std::vector<int> ells;
            for (const LM &x : lms)
                if (std::find(ells.begin(), ells.end(), x.l) == ells.end()) ells.push_back(x.l);
            const std::vector<double> a = pk_terms(ells);
            const int ne = (int)ells.size();
            for (int u = 0; u < nl; u++) {
                const int e = (int)(std::find(ells.begin(), ells.end(), lms[u].l) - ells.begin());
                for (int j = 0; j < ns; j++) {
                    avg[2 * (j * nl + u)] = a[2 * (j * ne + e)];
                    avg[2 * (j * nl + u) + 1] = a[2 * (j * ne + e) + 1];
                }
            }
        }
        for (int b0 = 0; b0 < nl && !m0; b0 += HG_MAX_LM) {
            int b1 = std::min(nl, b0 + HG_MAX_LM);
            std::vector<LM> part(lms.begin() + b0, lms.begin() + b1);
            std::vector<double> a;
            pk_bin(part, Np, 0.0, a, nm);
            const int np_ = b1 - b0;
            for (int j = 0; j < ns; j++)
                for (int u = 0; u < np_; u++) {
                    avg[2 * (j * nl + b0 + u)] = a[2 * (j * np_ + u)];
                    avg[2 * (j * nl + b0 + u) + 1] = a[2 * (j * np_ + u) + 1];
                }
        }
        std::vector<std::vector<double>> SN(mps.size(), std::vector<double>(2 * ns * ns, 0.0));
        for (size_t q = 0; q < mps.size(); q++) {
            const MP &mp = mps[q];
            int u = 0;
            for (const auto &c : cmb[q]) {
                int iu1 = -1, iu2 = -1;
                if (mp.l2 == 0) iu1 = lm_idx[q][u++];
                if (mp.l1 == 0) iu2 = lm_idx[q][u++];
                for (int i1 = 0; i1 < ns; i1++)
                    for (int i2 = 0; i2 < ns; i2++) {
                        double sr = 0.0, si = 0.0;
                        if (mp.l1 == 0 && mp.l2 == 0) sr += c.w * Np;
                        if (iu1 >= 0) {
                            sr += c.w * avg[2 * (i1 * nl + iu1)];
                            si += c.w * avg[2 * (i1 * nl + iu1) + 1];
                        }
                        if (iu2 >= 0) {
                            sr += c.w * avg[2 * (i2 * nl + iu2)];
                            si += c.w * avg[2 * (i2 * nl + iu2) + 1];
                        }
                        SN[q][2 * (i1 * ns + i2)] += sr;
                        SN[q][2 * (i1 * ns + i2) + 1] += si;
                    }
            }
        }
        ensure_histograms(mps);
        for (size_t q = 0; q < mps.size(); q++)
            bk_sn_xi(mps[q], dp<double>(*hist_mp[{mps[q].l1, mps[q].l2, mps[q].L}]), SN[q]);
        return SN;
    }

    // ------------------------------------------------------------------ batch (hg_batch_run)
    // Two device catalogue buffers: mock i is measured from one while a host thread stages
    // mock i + 1 through two pinned chunks into the other on the copy stream.
    DBuf bcat[2];
    cudaStream_t cst = nullptr;
    cudaEvent_t cev[2] = {nullptr, nullptr};
    void *pinned[2] = {nullptr, nullptr};
    static constexpr size_t PIN_CHUNK = 64u << 20;

    void batch_release() {
        if (cst) cudaStreamSynchronize(cst);
        for (int k = 0; k < 2; k++) {
            if (pinned[k]) cudaFreeHost(pinned[k]);
            if (cev[k]) cudaEventDestroy(cev[k]);
            pinned[k] = nullptr;
            cev[k] = nullptr;
        }
        if (cst) cudaStreamDestroy(cst);
        cst = nullptr;
    }

    // copy one catalogue into a device buffer (host thread: set_device first).  Page-locked
    // host memory is copied directly; pageable memory through the two pinned chunks, each
    // filled by several host threads.
    void batch_upload(const hg_mock &m, void *dst) {
        HG_CK(cudaSetDevice(cfg.device));
        const size_t bytes = (size_t)m.n * (size_t)m.stride_bytes;
        const unsigned char *src = reinterpret_cast<const unsigned char *>(m.base);
        cudaPointerAttributes at;
        if (cudaPointerGetAttributes(&at, src) == cudaSuccess && at.type == cudaMemoryTypeHost) {
            HG_CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, cst));
            HG_CK(cudaStreamSynchronize(cst));
            return;
        }
        cudaGetLastError();  // a pageable pointer may leave an error behind on older runtimes
        const unsigned nthr = std::max(1u, std::min(8u, std::thread::hardware_concurrency()));
        int k = 0;
        for (size_t o = 0; o < bytes; o += PIN_CHUNK, k ^= 1) {
            const size_t sz = std::min(PIN_CHUNK, bytes - o);
            HG_CK(cudaEventSynchronize(cev[k]));  // this chunk's previous copy is done
            {
                std::vector<std::thread> th;
                const size_t part = (sz + nthr - 1) / nthr;
                for (unsigned t = 0; t < nthr; t++) {
                    const size_t a = std::min(sz, t * part), b = std::min(sz, a + part);
                    if (b > a)
                        th.emplace_back([=] { memcpy(static_cast<unsigned char *>(pinned[k]) + a, src + o + a, b - a); });
                }
                for (auto &x : th) x.join();
            }
            HG_CK(cudaMemcpyAsync(reinterpret_cast<unsigned char *>(dst) + o, pinned[k], sz, cudaMemcpyHostToDevice,
                                  cst));
            HG_CK(cudaEventRecord(cev[k], cst));
        }
        HG_CK(cudaStreamSynchronize(cst));
    }

    void batch_run(const hg_mock *m, int n, const std::vector<int> &pk_ells, const std::vector<MP> &bk,
                   const std::vector<MP> &zeta, double *out) override {
        for (int e : pk_ells) HG_REQUIRE(e >= 0, "ell must be >= 0");
        if (!bk.empty()) check_multipoles(bk);
        if (!zeta.empty()) check_multipoles(zeta);
        size_t maxb = 0;
        for (int i = 0; i < n; i++) {
            HG_REQUIRE(m[i].base != nullptr && m[i].n > 0, "a mock has no particles");
            HG_REQUIRE(m[i].stride_bytes >= 24 && m[i].stride_bytes % 8 == 0 && m[i].pos_off >= 0 &&
                           (m[i].pos_off + 3) * 8 <= m[i].stride_bytes,
                       "a mock's stride_bytes / pos_off do not describe {x, y, z} doubles");
            maxb = std::max(maxb, (size_t)m[i].n * (size_t)m[i].stride_bytes);
        }
        // every allocation before the pipeline starts (no cudaMalloc beside running work)
        HG_CK(bcat[0].ensure(maxb));
        if (n > 1) HG_CK(bcat[1].ensure(maxb));
        if (!cst) {
            HG_CK(cudaStreamCreateWithFlags(&cst, cudaStreamNonBlocking));
            for (int k = 0; k < 2; k++) {
                HG_CK(cudaEventCreateWithFlags(&cev[k], cudaEventDisableTiming));
                HG_CK(cudaHostAlloc(&pinned[k], PIN_CHUNK, cudaHostAllocDefault));
            }
        }
        const long long blk = batch_block_len(cfg, (int)pk_ells.size(), (int)bk.size(), (int)zeta.size());
        const int nk = cfg.n_kbin, nr = cfg.n_rbin;
        std::exception_ptr up_err;
        auto upload = [&](int i) {
            try {
                batch_upload(m[i], bcat[i & 1].p);
            } catch (...) {
                up_err = std::current_exception();
            }
        };
        batch_done = 0;
        auto mock_error = [](int i, const std::string &m) { return HgError{"mock " + std::to_string(i) + ": " + m}; };
        upload(0);
        if (up_err) {
            try {
                std::rethrow_exception(up_err);
            } catch (const HgError &e) {
                throw mock_error(0, e.msg);
            }
        }
        double total_ms = 0.0;
        long long total_launches = 0;
        for (int i = 0; i < n; i++) {
            std::thread next;
            if (i + 1 < n) next = std::thread(upload, i + 1);
            try {
                set_particles(0, reinterpret_cast<const double *>(bcat[i & 1].p), m[i].n, m[i].stride_bytes,
                              m[i].pos_off, -1, -1, true);
                double *o = out + (long long)i * blk;
                for (size_t q = 0; q < pk_ells.size(); q++) {
                    pk_box(pk_ells[q], o + 2LL * q * nk, nullptr, o + 2LL * pk_ells.size() * nk + q);
                    total_ms += last_ms;
                    total_launches += last_launches;
                }
                o += 2LL * pk_ells.size() * nk + pk_ells.size();
                if (!bk.empty()) {
                    const long long sz = 2LL * bk.size() * nk * nk;
                    bk_box_multi(bk, -1, o, o + sz, o + 2 * sz);
                    total_ms += last_ms;
                    total_launches += last_launches;
                    o += 2 * sz + 1;
                }
                if (!zeta.empty()) {
                    const long long sz = 2LL * zeta.size() * nr * nr;
                    zeta_box_multi(zeta, -1, o, o + sz, o + 2 * sz);
                    total_ms += last_ms;
                    total_launches += last_launches;
                }
            } catch (const HgError &e) {
                if (next.joinable()) next.join();
                throw mock_error(i, e.msg);
            } catch (...) {
                if (next.joinable()) next.join();
                throw;
            }
            if (next.joinable()) next.join();
            batch_done = i + 1;
            if (up_err) {
                try {
                    std::rethrow_exception(up_err);
                } catch (const HgError &e) {
                    throw mock_error(i + 1, e.msg);
                }
            }
        }
        last_ms = total_ms;
        last_launches = total_launches;
    }

    // ------------------------------------------------------------------ stages (hg_ctx.hpp)
    void stage_adopt_stream(void *stream) override {
        if (st && own_stream) {
            HG_CK(cudaStreamSynchronize(st));
            HG_CK(cudaStreamDestroy(st));
        }
        st = reinterpret_cast<cudaStream_t>(stream);
        own_stream = false;
    }
    const void *stage_density(double *d0, double *n0, double *m0) override {
        box_density();
        *d0 = delta0;
        *n0 = N0;
        *m0 = dens_mass;
        return H.p;
    }
    bool stage_density_ready() const override { return dens_valid; }
    void stage_import_density(const void *src, bool src_fp64, double d0, double n0, double m0) override {
        const long long n = (long long)g.n[0] * g.n[1] * (g.n[2] / 2 + 1);
        HG_CK(H.ensure(sizeof(C) * n));
        if (sizeof(T) == 4 && src_fp64) {  // narrowed when first needed (narrow_density)
            H_wide = reinterpret_cast<const cplx<double> *>(src);
            narrow_pending = true;
        } else {
            H_wide = nullptr;
            narrow_pending = false;
            convert_spectrum(src, src_fp64);
        }
        delta0 = d0;
        N0 = n0;
        dens_mass = m0;
        dens_valid = true;  // statistics of the previous density were dropped by set_particles
        pk_cache.clear();
    }
    std::vector<std::vector<double>> stage_bk_signal(const std::vector<MP> &mps) override {
        set_source(0, 0.0);
        return bk_main(mps);
    }
    std::vector<std::vector<double>> stage_bk_shot(const std::vector<MP> &mps) override {
        set_source(0, 0.0);
        return bk_shot(mps);
    }
    std::vector<double> stage_pk_terms(const std::vector<int> &ells) override {
        box_density();
        const int ns = cfg.n_kbin, ne = (int)ells.size();
        std::vector<double> a(2 * ns * ne);
        for (int e = 0; e < ne; e++) {
            const PkBins &pb = box_pk_bins(ells[e]);
            for (int j = 0; j < ns; j++) {
                a[2 * (j * ne + e)] = pb.avg[2 * j];
                a[2 * (j * ne + e) + 1] = pb.avg[2 * j + 1];
            }
        }
        return a;
    }
    long long stage_take_launches() override {
        const long long l = launches;
        launches = 0;
        return l;
    }

    // ------------------------------------------------------------------ 3PCF (box)
    // k-space keys of the 3PCF fields' j_l(|k| r): integer |n|^2 on a cubic box and mesh,
    // octant modes (|wx|, |wy|, |wz|) with the reference's |k| otherwise
    bool zk_octant = false;
    long long nkk = 0;
    DBuf d_kkr;
    void zeta_geometry() {
        build_orbits();
        if (!zfine.empty()) return;
        zk_octant = !(g.n[0] == g.n[1] && g.n[0] == g.n[2] && cfg.boxsize[0] == cfg.boxsize[1] &&
                      cfg.boxsize[0] == cfg.boxsize[2]);
        if (zk_octant) {
            const int h0 = g.n[0] / 2 + 1, h1 = g.n[1] / 2 + 1, h2 = g.n[2] / 2 + 1;
            nkk = (long long)h0 * h1 * h2;
            std::vector<double> kr(nkk);
            auto comp = [&](int a, int i) {
                const int n = g.n[a];
                return double(i < n / 2 ? i : i - n) * g.dk[a];
            };
            for (int a = 0; a < h0; a++)
                for (int b = 0; b < h1; b++)
                    for (int c = 0; c < h2; c++) {
                        const double kx = comp(0, a), ky = comp(1, b), kz = comp(2, c);
                        kr[((long long)a * h1 + b) * h2 + c] = std::sqrt(kx * kx + ky * ky + kz * kz);
                    }
            HG_CK(d_kkr.ensure(sizeof(double) * nkk));
            HG_CK(cudaMemcpy(d_kkr.p, kr.data(), sizeof(double) * nkk, cudaMemcpyHostToDevice));
        } else {
            nkk = n2dim;
        }
        // rindex = int(|r| / 0.5 + 0.5), kept if < 10000 (field.hpp:1030-1053), per histogram key
        // (on equal cells |r|^2 = n2 dr^2, the reference's sum of (i dr)^2 exactly when those
        // squares are exact, e.g. an integer box over a power-of-two mesh)
        zfine.assign(nkey, -1);
        for (long long q = 0; q < nkey; q++) {
            const int ri = (int)(key_r[q] / 0.5 + 0.5);
            if (ri < 10000) zfine[q] = ri;
        }
        // coarse bins from neighbouring half widths (field.hpp:1058-1085)
        const int nr = cfg.n_rbin;
        std::vector<double> drb(nr - 1);
        for (int j = 0; j < nr - 1; j++) drb[j] = rbin[j + 1] - rbin[j];
        zcoarse.assign(10000, {});
        for (int j = 0; j < nr; j++) {
            double lower = (j == 0) ? ((rbin[j] > drb[j] * 0.5) ? (rbin[j] - drb[j] * 0.5) : 0.0)
                                    : rbin[j] - drb[j - 1] * 0.5;
            double upper = (j == nr - 1) ? (rbin[j] + drb[j - 1] * 0.5) : (rbin[j] + drb[j] * 0.5);
            for (int i = 0; i < 10000; i++) {
                double rt = double(i) * 0.5;
                if (rt > lower && rt <= upper) zcoarse[i].push_back(j);
            }
        }
        zcount.assign(nr, 0.0);
        for (long long q = 0; q < nkey; q++)
            if (zfine[q] >= 0)
                for (int j : zcoarse[zfine[q]]) zcount[j] += key_cells[q];
    }

    // J_l[j][key] = j_l(r_j |k|_key) at the r bins (keys: zeta_geometry; geometry only: cached)
    const double *jtab_rbins(int l) {
        auto it = jtab_r.find(l);
        if (it != jtab_r.end()) return dp<double>(*it->second);
        const BesselSpline &s = spline(l);
        auto &sp = d_splines[l];
        HG_CK(d_rv.ensure(sizeof(double) * rbin.size()));
        HG_CK(cudaMemcpyAsync(d_rv.p, rbin.data(), sizeof(double) * rbin.size(), cudaMemcpyHostToDevice, st));
        auto J = std::make_unique<DBuf>();
        HG_CK(J->ensure(sizeof(double) * rbin.size() * nkk));
        long long tot = (long long)rbin.size() * nkk;
        kb("bessel_table", double(tot) * 8.0);
        if (zk_octant)
            k_bessel_table_r<<<grid1(tot, 256), 256, 0, st>>>(dp<double>(*sp.first), dp<double>(*sp.second), s.n,
                                                              s.xmin, s.dx, dp<double>(d_rv), (int)rbin.size(),
                                                              dp<double>(d_kkr), nkk, dp<double>(*J));
        else
            k_bessel_table<<<grid1(tot, 256), 256, 0, st>>>(dp<double>(*sp.first), dp<double>(*sp.second), s.n,
                                                            s.xmin, s.dx, dp<double>(d_rv), (int)rbin.size(), g.dk[0],
                                                            n2dim, dp<double>(*J));
        ke();
        HG_CK(cudaStreamSynchronize(st));
        const double *p = dp<double>(*J);
        jtab_r[l] = std::move(J);
        return p;
    }

    // U = Yhat_lm F / W / V on the full grid, F the given spectrum (the density by default)
    void zeta_U(int l, int m) { zeta_U_of(dsrc, l, m); }
    void zeta_U_of(const SpecK &src, int l, int m) {
        if (src.s.p == dp<C>(H)) narrow_density();  // the box density
        HG_CK(Uz.ensure(sizeof(C) * g.ntot));
        unsigned blocks = (unsigned)std::min<long long>(grid1(g.ntot, 256), 148 * 16);
        kb("zeta_U", double(g.ntot) * (sizeof(C) * 1.5));
        k_zeta_U<T><<<blocks, 256, 0, st>>>(src.s, g, tabs, wpow, l, m, src.k0r, src.k0i, dp<C>(Uz));
        ke();
    }

    // inverse transform of nr fields on the full grid; the x pass reads through `ld`
    template <class LD>
    void full_inverse(LD ld, C *out, int nr, const char *name) {
        const int n0 = g.n[0], n1 = g.n[1], n2 = g.n[2];
        const long long yz = (long long)n1 * n2;
        const double fb = double(g.ntot) * sizeof(C) * nr;
        pass<+1>(n0, ld, StArr<T>{out, n0, yz}, nr, yz, name, fb * 1.5);
        pass<+1>(n1, LdArr<T>{out, n1, n2}, StArr<T>{out, n1, n2}, (long long)nr * n0, n2, name, fb * 2.0);
        pass<+1>(n2, LdArr<T>{out, n2, 1}, StArr<T>{out, n2, 1}, (long long)nr * n0 * n1, 1, name, fb * 2.0);
    }

    // G(x) = IFFT[delta / W] / V on the full grid (field.hpp:326-344 after the window correction)
    const C *ensure_Gz(const GK &gk) {
        auto &p = Gz[gk];
        if (!p) p = std::make_unique<DBuf>();
        if (Gz_ok.count(gk)) return dp<C>(*p);
        zeta_U_of(g_source(gk), 0, 0);
        HG_CK(p->ensure(sizeof(C) * g.ntot));
        full_inverse(LdArr<T>{dp<C>(Uz), g.n[0], (long long)g.n[1] * g.n[2]}, dp<C>(*p), 1, "zeta_G");
        Gz_ok.insert(gk);
        return dp<C>(*p);
    }

    size_t zf_bytes() const {
        size_t b = 0;
        for (const auto &kv : zf) b += kv.second->n;
        return b;
    }

    // F_lm[r] = IFFT[j_l(|k| r) U_lm] for r in [r0, r0+nr) (field.hpp:403-445), cached per catalogue
    const C *zeta_fields(const Fam &f, int r0, int nr, const ZKey *keep) {
        ZKey key{f.l, f.m, r0, nr};
        auto it = zf.find(key);
        if (it != zf.end() && zf_ok.count(key)) return dp<C>(*it->second);
        const size_t need = sizeof(C) * (size_t)g.ntot * nr;
        auto &p = zf[key];
        if (!p) p = std::make_unique<DBuf>();
        if (p->ensure(need) != cudaSuccess) {  // out of memory: release cached fields other than `keep`, retry
            cudaGetLastError();
            for (auto i = zf.begin(); i != zf.end();) {
                if ((keep && !(i->first < *keep) && !(*keep < i->first)) || !(i->first < key || key < i->first)) {
                    ++i;
                    continue;
                }
                zf_ok.erase(i->first);
                i = zf.erase(i);
            }
            HG_CK(zf[key]->ensure(need));
        }
        zeta_U(f.l, f.m);
        const double *J = jtab_rbins(f.l) + (size_t)r0 * nkk;
        LdZetaField<T> ld{dp<C>(Uz), J, nkk, g.n[0], g.n[1], g.n[2], zk_octant ? 1 : 0};
        full_inverse(ld, dp<C>(*p), nr, "zeta_fields");
        zf_ok.insert(key);
        return dp<C>(*p);
    }

    // P[i1][i2] = sum_x Fa[i1](x) Fb[i2](x) G(x), complex [na][nb]
    std::vector<double> zeta_pairsum(const C *Fa, int na, const C *Fb, int nb, const C *G) {
        const int nblk = 2 * 148;
        const size_t smem = zeta_pairsum_smem(na, nb);
        HG_CK(zpart.ensure(sizeof(double) * 2 * (size_t)nblk * na * nb));
        HG_CK(zout.ensure(sizeof(double2) * (size_t)na * nb));
        HG_CK(cudaFuncSetAttribute(k_zeta_pairsum<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kb("zeta_pairsum", double(g.ntot) * sizeof(C) * double(na + (Fa == Fb ? 0 : nb) + 1));
        k_zeta_pairsum<T><<<nblk, HG_ZR_THREADS, smem, st>>>(Fa, na, Fb, nb, G, g.ntot, dp<double>(zpart));
        ke();
        kb("zeta_pairsum", double(nblk) * na * nb * 16.0);
        k_sum_parts<<<grid1(sum_parts_threads((long long)na * nb), 256), 256, 0, st>>>(dp<double>(zpart), nblk, na * nb,
                                                                      dp<double2>(zout));
        ke();
        std::vector<double> h(2 * (size_t)na * nb);
        HG_CK(cudaMemcpyAsync(h.data(), zout.p, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, st));
        HG_CK(cudaStreamSynchronize(st));
        return h;
    }

    // sum_x F_a[i1] F_b[i2] G for the requested rows i1 (all, or `row`) and every i2:
    // [rows][ns] complex.  All rows come from the unordered pair (transposed when needed).
    std::vector<double> zeta_pair(const Fam &a, const Fam &b, int row, const GK &gk) {
        const int ns = cfg.n_rbin;
        const bool all = (row < 0);
        Fam p = a, q = b;
        bool swap = false;
        if (all && b < a) {
            std::swap(p, q);
            swap = true;
        }
        auto key = std::make_tuple(p.l, p.m, q.l, q.m, row, gk.first, gk.second);
        auto it = zpairs.find(key);
        if (it == zpairs.end()) {
            const int rows = all ? ns : 1;
            std::vector<double> out(2 * (size_t)rows * ns, 0.0);
            // radius tiles that fit next to the cached fields (one tile when memory allows);
            // the free memory is read once per context, then tracked by what the cache holds
            const double fb = double(sizeof(C)) * double(g.ntot);
            if (zfree0 == 0) {
                size_t fr = 0, tot = 0;
                HG_CK(cudaMemGetInfo(&fr, &tot));
                zfree0 = fr + zf_bytes();
            }
            double avail = double(zfree0) - double(size_t(4) << 30);
            int tile = (int)std::min<double>(64.0, std::floor(avail / (2.0 * fb)));
            HG_REQUIRE(tile >= 1, "not enough device memory for two 3PCF fields");
            tile = std::min(tile, ns);
            const int pr0 = all ? 0 : row, prn = all ? ns : 1;
            for (int a0 = pr0; a0 < pr0 + prn; a0 += tile) {
                const int an = std::min(tile, pr0 + prn - a0);
                for (int b0 = 0; b0 < ns; b0 += tile) {
                    const int bn = std::min(tile, ns - b0);
                    ZKey ka{p.l, p.m, a0, an};
                    const C *Fa = zeta_fields(p, a0, an, nullptr);
                    const C *Fb = (p.l == q.l && p.m == q.m && a0 == b0 && an == bn) ? Fa
                                                                                       : zeta_fields(q, b0, bn, &ka);
                    std::vector<double> t = zeta_pairsum(Fa, an, Fb, bn, ensure_Gz(gk));
                    for (int i1 = 0; i1 < an; i1++)
                        for (int i2 = 0; i2 < bn; i2++) {
                            size_t o = (size_t)(a0 - pr0 + i1) * ns + (b0 + i2);
                            out[2 * o] = t[2 * ((size_t)i1 * bn + i2)];
                            out[2 * o + 1] = t[2 * ((size_t)i1 * bn + i2) + 1];
                        }
                }
            }
            it = zpairs.emplace(key, std::move(out)).first;
        }
        if (!swap) return it->second;
        const auto &P = it->second;
        std::vector<double> r(2 * (size_t)ns * ns);
        for (int i = 0; i < ns; i++)
            for (int j = 0; j < ns; j++) {
                r[2 * ((size_t)i * ns + j)] = P[2 * ((size_t)j * ns + i)];
                r[2 * ((size_t)i * ns + j) + 1] = P[2 * ((size_t)j * ns + i) + 1];
            }
        return r;
    }

    // bispec.hpp:1205-1424 for all r1 rows (ith = -1) or one, for several multipoles.
    // zeta_raw = sum_(m1,m2,M) w i^(l1+l2) dV sum_x F1 F2 G_LM  (bispec.hpp:1354-1378 box,
    // 545-575 survey): [q][rows][ns] complex
    std::vector<std::vector<double>> zeta_main(const std::vector<MP> &mps, int ith) {
        const int ns = cfg.n_rbin;
        const double dV = g.volume / double(g.ntot);
        const int rows = (ith < 0) ? ns : 1;
        std::vector<std::vector<double>> Z(mps.size(), std::vector<double>(2 * (size_t)rows * ns, 0.0));
        for (size_t q = 0; q < mps.size(); q++) {
            const MP &mp = mps[q];
            const int p4 = (mp.l1 + mp.l2) % 4;
            for (const auto &c : combos3(mp, all_M())) {
                GK gk = g_key(mp.L, c.M);
                std::vector<double> t = zeta_pair(Fam{mp.l1, c.m1}, Fam{mp.l2, c.m2}, ith, gk);
                for (size_t e = 0; e < (size_t)rows * ns; e++) {
                    double re = c.w * (dV * t[2 * e]), im = c.w * (dV * t[2 * e + 1]);
                    double rr = p4 == 0 ? re : p4 == 1 ? -im : p4 == 2 ? -re : im;
                    double ii = p4 == 0 ? im : p4 == 1 ? re : p4 == 2 ? -im : -re;
                    Z[q][2 * e] += rr;
                    Z[q][2 * e + 1] += ii;
                }
            }
        }
        return Z;
    }

    // shot noise on the diagonal from a multipole's n^2 histogram (field.hpp:1030-1105,
    // bispec.hpp:1279-1285), written with the results
    void zeta_finish(const std::vector<MP> &mps, int ith, const std::vector<std::vector<double>> &Z,
                     const std::vector<const double *> &hists, double *zeta_save, double *sn_save) {
        const int ns = cfg.n_rbin;
        const double dV = g.volume / double(g.ntot);
        const int r0 = (ith < 0) ? 0 : ith, rows = (ith < 0) ? ns : 1;
        std::fill(sn_save, sn_save + 2 * mps.size() * (size_t)rows * ns, 0.0);
        std::vector<double> hist(2 * nkey);
        for (size_t q = 0; q < mps.size(); q++) {
            const MP &mp = mps[q];
            HG_CK(cudaMemcpyAsync(hist.data(), hists[q], sizeof(double) * hist.size(), cudaMemcpyDeviceToHost, st));
            HG_CK(cudaStreamSynchronize(st));
            std::vector<double> xr(ns, 0.0), xim(ns, 0.0);
            for (long long n2 = 0; n2 < nkey; n2++) {
                if (zfine[n2] < 0) continue;
                for (int j : zcoarse[zfine[n2]]) {
                    xr[j] += hist[2 * n2];
                    xim[j] += hist[2 * n2 + 1];
                }
            }
            const double sg = ((mp.l1 + mp.l2) % 2 == 0) ? 1.0 : -1.0;
            for (int i = r0; i < r0 + rows; i++) {
                double sc = zcount[i] != 0.0 ? sg / zcount[i] / zcount[i] / dV : 0.0;
                size_t o = (size_t)q * rows * ns + (size_t)(i - r0) * ns + i;
                sn_save[2 * o] = xr[i] * sc;
                sn_save[2 * o + 1] = xim[i] * sc;
            }
        }
        for (size_t q = 0; q < mps.size(); q++)
            for (size_t e = 0; e < (size_t)rows * ns; e++) {
                size_t o = q * (size_t)rows * ns + e;
                zeta_save[2 * o] = Z[q][2 * e];
                zeta_save[2 * o + 1] = Z[q][2 * e + 1];
            }
    }

    // bispec.hpp:1205-1424 for all r1 rows (ith = -1) or one, for several multipoles.
    void zeta_box_multi(const std::vector<MP> &mps, int ith, double *zeta_save, double *sn_save,
                        double *norm) override {
        check_multipoles(mps);
        HG_REQUIRE(ith >= -1 && ith < cfg.n_rbin, "ith_rbin out of range");
        begin();
        zeta_geometry();
        set_source(0, 0.0);
        std::vector<std::vector<double>> Z = zeta_main(mps, ith);
        ensure_histograms(mps);
        std::vector<const double *> hs;
        for (const auto &mp : mps) hs.push_back(dp<double>(*hist_mp[{mp.l1, mp.l2, mp.L}]));
        zeta_finish(mps, ith, Z, hs, zeta_save, sn_save);
        if (norm) {
            const double Np = double(slot[0].n);
            double nv = g.volume / Np / Np;
            nv *= (g.volume / Np);
            *norm = nv;
        }
        end();
    }

    // ------------------------------------------------------------------ survey geometry
    PartSrc survey_src(int s, bool ylm, int l, int m, double scale, int wp = 1, bool conj = false) const {
        const Slot &S = slot[s];
        PartSrc p{};
        p.base = S.base();
        p.n = S.n;
        p.stride = S.stride;
        p.pos_off = S.pos_off;
        p.w_off = S.w_off;
        p.cw = nullptr;
        p.scale = scale;
        p.ylm_on = ylm ? 1 : 0;
        p.ylm_l = l;
        p.ylm_m = m;
        p.los_off = S.los_off;
        p.wpow = wp;
        p.ylm_conj = conj ? 1 : 0;
        return p;
    }

    void require_survey(bool need_los) const {
        HG_REQUIRE(slot[0].set && slot[1].set,
                   "survey statistics need data (slot 0) and randoms (slot 1): call hg_set_particles for both");
        if (need_los)
            HG_REQUIRE(slot[0].los_off >= 0 && slot[1].los_off >= 0,
                       "survey multipoles need line-of-sight vectors: pass los_off for both catalogues");
    }

    // FP64 particle sums (block partials added on the host in block order)
    std::vector<double> particle_sums(int s, const PSumSpec &q) {
        const PartSrc src = survey_src(s, false, 0, 0, 1.0);
        if (src.n == 0) return std::vector<double>(2 * q.n, 0.0);
        const int nb = (int)std::min<long long>(grid1(src.n, 256), 148 * 8);
        HG_CK(psum_part.ensure(sizeof(double) * 2 * HG_PSUM_MAX * nb));
        kb("particle_sums", double(src.n) * 32.0);
        k_particle_sums<<<nb, 256, 0, st>>>(src, q, dp<double>(psum_part));
        ke();
        std::vector<double> h(2 * HG_PSUM_MAX * (size_t)nb);
        HG_CK(cudaMemcpyAsync(h.data(), psum_part.p, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, st));
        HG_CK(cudaStreamSynchronize(st));
        std::vector<double> out(2 * q.n, 0.0);
        for (int b = 0; b < nb; b++)
            for (int j = 0; j < 2 * q.n; j++) out[j] += h[(size_t)b * 2 * HG_PSUM_MAX + j];
        return out;
    }

    // alpha = sum w_D / sum w_R (particle.hpp:268-282); V_survey = (sum w_R)^2 / sum_c rho_R^2 dV
    // on an FP64 mesh in both forms (field.hpp:449-503); nbar = (sum w_D)^2 / V / sum w_D^2
    // (particle.hpp:284-300).
    void survey_scalars(double *alpha, double *vs, double *nbar, double *wd, double *wr) override {
        require_survey(false);
        begin();
        PSumSpec q{};
        q.n = 2;
        q.pw[0] = 1;
        q.l[0] = -1;
        q.pw[1] = 2;
        q.l[1] = -1;
        std::vector<double> sd = particle_sums(0, q);
        q.n = 1;
        std::vector<double> sr = particle_sums(1, q);
        const double wD = sd[0], w2D = sd[2], wR = sr[0];
        HG_REQUIRE(std::isfinite(wD) && std::isfinite(w2D) && std::isfinite(wR),
                   "the catalogue holds particle(s) with a non-finite weight");
        HG_REQUIRE(wD != 0.0 && wR != 0.0, "the summed weights of data and randoms must be non-zero");
        const double a = wD / wR;
        AssignGeom ag = make_geom(0.0);
        ag.acc_factor = ag.factor;  // rho = sum w (1/dV) prod(w_axis), FP64
        HG_CK(dmesh.ensure(sizeof(double) * g.ntot));
        assign_mesh<double, false>({survey_src(1, false, 0, 0, 1.0)}, ag, dp<double>(dmesh), nullptr, false);
        const int nb = 148 * 8;
        HG_CK(psum_part.ensure(sizeof(double) * nb));
        kb("survey_volume", double(g.ntot) * 8.0);
        k_sum_squares<<<nb, 256, 0, st>>>(dp<double>(dmesh), g.ntot, dp<double>(psum_part));
        ke();
        std::vector<double> h(nb);
        HG_CK(cudaMemcpyAsync(h.data(), psum_part.p, sizeof(double) * nb, cudaMemcpyDeviceToHost, st));
        HG_CK(cudaStreamSynchronize(st));
        double s2 = 0.0;
        for (int b = 0; b < nb; b++) s2 += h[b];
        const double dV = g.volume / double(g.ntot);
        const double V = wR * wR / (s2 * dV);
        dmesh.release();
        if (alpha) *alpha = a;
        if (vs) *vs = V;
        if (nbar) *nbar = wD * wD / V / w2D;
        if (wd) *wd = wD;
        if (wr) *wr = wR;
        end();
    }

    // FFT[dV (n_D - alpha n_R)] of the Yhat_lm(los)-weighted fields, m >= 0
    // (calcYlmWeightedDensityFluctuation field.hpp:186-228, then field.hpp:310-325).  m = 0 is
    // a real field (half spectrum); m > 0 is complex (full spectrum).
    // tile binning of data and randoms (positions only) for one assignment offset
    SurveyBins &survey_bins(int k) {
        SurveyBins &B = sbins[k];
        if (B.ok) return B;
        const AssignGeom ag = make_geom(k ? 0.5 : 0.0);
        const int ntiles = ag.nt[0] * ag.nt[1] * ag.nt[2];
        HG_CK(cnt.ensure(sizeof(unsigned) * (ntiles + 1)));
        HG_CK(off.ensure(sizeof(unsigned) * (ntiles + 1)));
        HG_CK(cursor.ensure(sizeof(unsigned) * (ntiles + 1)));
        HG_CK(nch.ensure(sizeof(unsigned) * (ntiles + 1)));
        HG_CK(choff.ensure(sizeof(unsigned) * (ntiles + 1)));
        HG_CK(cudaMemsetAsync(cnt.p, 0, sizeof(unsigned) * (ntiles + 1), st));
        HG_CK(cudaMemsetAsync(cursor.p, 0, sizeof(unsigned) * (ntiles + 1), st));
        const PartSrc src[2] = {survey_src(0, false, 0, 0, 1.0), survey_src(1, false, 0, 0, 1.0)};
        bin_count_sources(src, 2, ag, nullptr);
        size_t tb = 0, tb2 = 0;
        HG_CK(cub::DeviceScan::ExclusiveSum(nullptr, tb, dp<unsigned>(cnt), dp<unsigned>(off), ntiles + 1, st));
        HG_CK(cub::DeviceScan::ExclusiveSum(nullptr, tb2, dp<unsigned>(nch), dp<unsigned>(choff), ntiles + 1, st));
        HG_CK(cubtmp.ensure(std::max(tb, tb2)));
        HG_CK(cub::DeviceScan::ExclusiveSum(cubtmp.p, tb, dp<unsigned>(cnt), dp<unsigned>(off), ntiles + 1, st));
        k_chunk_count<<<grid1(ntiles + 1, 256), 256, 0, st>>>(dp<unsigned>(cnt), ntiles, CHUNK, dp<unsigned>(nch));
        HG_CK(cub::DeviceScan::ExclusiveSum(cubtmp.p, tb2, dp<unsigned>(nch), dp<unsigned>(choff), ntiles + 1, st));
        unsigned tot[2] = {0, 0};
        HG_CK(cudaMemcpyAsync(&tot[0], dp<unsigned>(off) + ntiles, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
        HG_CK(cudaMemcpyAsync(&tot[1], dp<unsigned>(choff) + ntiles, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
        unsigned flags[2] = {0, 0};
        read_bad_count(2, flags);
        HG_CK(cudaStreamSynchronize(st));
        check_finite(flags);
        B.neg = flags[1] != 0;
        B.total = tot[0];
        B.nchunks = tot[1];
        HG_CK(B.rec.ensure(sizeof(PRecS<T>) * std::max<size_t>(B.total, 1)));
        HG_CK(B.chunks.ensure(sizeof(Chunk) * std::max<size_t>(B.nchunks, 1)));
        k_chunk_fill<<<grid1(ntiles, 256), 256, 0, st>>>(dp<unsigned>(off), dp<unsigned>(choff), ntiles, CHUNK,
                                                        dp<Chunk>(B.chunks));
        {
            const RecIndex<T> mk[2] = {RecIndex<T>{0}, RecIndex<T>{1}};
            bin_scatter_sources(src, mk, 2, ag, ntiles, dp<PRecS<T>>(B.rec), double(B.total) * sizeof(PRecS<T>));
        }
        HG_CK(cudaGetLastError());
        B.ok = true;
        return B;
    }

    DBuf cwbuf[2];  // per-particle complex weights of the field being accumulated
    // max |w| of catalogue s (cached until the catalogue changes)
    double wmax_cache[2] = {-1.0, -1.0};
    double max_weight(int s) {
        if (wmax_cache[s] >= 0.0) return wmax_cache[s];
        const PartSrc src = survey_src(s, false, 0, 0, 1.0);
        if (src.n == 0) return wmax_cache[s] = 0.0;
        const int nb = (int)std::min<long long>(grid1(src.n, 256), 148 * 8);
        HG_CK(psum_part.ensure(sizeof(double) * nb));
        kb("particle_sums", double(src.n) * 8.0);
        k_max_weight<<<nb, 256, 0, st>>>(src, dp<double>(psum_part));
        ke();
        std::vector<double> h(nb);
        HG_CK(cudaMemcpyAsync(h.data(), psum_part.p, sizeof(double) * nb, cudaMemcpyDeviceToHost, st));
        HG_CK(cudaStreamSynchronize(st));
        double m = 0.0;
        for (double v : h) m = std::max(m, v);
        wmax_cache[s] = m;
        return m;
    }

    // accumulate one weighting of the binned catalogues; returns the FP64 in-bounds mass
    template <bool CPLX>
    std::array<double, 2> survey_accumulate(int k, const PartSrc srcs[2], T *re, T *im) {
        SurveyBins &B = survey_bins(k);
        AssignGeom ag = make_geom(k ? 0.5 : 0.0);
        ag.acc_factor = 1.0;
        FieldW fw;
        fw.s[0] = srcs[0];
        fw.s[1] = srcs[1];
        for (int q = 0; q < 2; q++) {  // harmonic-weighted sources: weights precomputed in order
            if (!srcs[q].ylm_on || srcs[q].cw || srcs[q].n == 0) continue;
            HG_CK(cwbuf[q].ensure(sizeof(double2) * std::max<long long>(srcs[q].n, 1)));
            const unsigned nb = (unsigned)std::min<long long>(grid1(srcs[q].n, 256), 148 * 16);
            kb("particle_sums", double(srcs[q].n) * (16.0 + 32.0));
            k_make_cw<<<nb, 256, 0, st>>>(srcs[q], dp<double2>(cwbuf[q]));
            ke();
            fw.s[q].cw = dp<double2>(cwbuf[q]);
        }
        HG_CK(mass.ensure(sizeof(double) * 2));
        HG_CK(cudaMemsetAsync(mass.p, 0, sizeof(double) * 2, st));
        kb("assign_zero_split", 0.0);
        k_zero_split_tiles<T, CPLX><<<B.nchunks, 256, 0, st>>>(dp<Chunk>(B.chunks), ag, re, im);
        ke();
        // exact fixed-point sums for FP32 fields whose per-record weight bound is known:
        // |Yhat_lm w^wpow scale| <= max|w|^wpow |scale| (|Yhat_lm| <= 1), one add per record
        // and cell (every axis at least W cells)
        bool fix = (sizeof(T) == 4);
        double wb = 0.0;
        for (int q = 0; q < 2; q++) {
            fix = fix && srcs[q].cw == nullptr;
            if (!fix) break;
            const double mw = max_weight(q);
            wb = std::max(wb, std::pow(mw, std::max(1, srcs[q].wpow)) * std::fabs(srcs[q].scale));
        }
        for (int a = 0; a < 3; a++) fix = fix && ag.n[a] >= stencil_width(ag.scheme);
        ag.fix_bound = (float)(wb * std::fabs(ag.acc_factor) * (1.0 + 1e-6)) * stencil_weight_bound(B.neg);
        fix = fix && ag.fix_bound >= 0x1p-60f && std::isfinite(ag.fix_bound);
        const size_t smem = sizeof(T) * ag.t[0] * ag.t[1] * ag.t[2] * (CPLX ? 2 : 1) * (fix ? 2 : 1);
        kb("assign_tile_accum", double(B.total) * sizeof(PRecS<T>) + double(g.ntot) * sizeof(T) * (CPLX ? 2 : 1));
        auto launch = [&](auto kern) {
            HG_CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            kern<<<B.nchunks, 256, smem, st>>>(dp<PRecS<T>>(B.rec), dp<Chunk>(B.chunks), ag, fw, re, im,
                                               dp<double>(mass));
        };
        auto by_scheme = [&](auto fixtag) {
            constexpr bool F = decltype(fixtag)::value;
            switch (ag.scheme) {
                case HG_NGP: launch(k_tile_accum_src<T, CPLX, HG_NGP, F>); break;
                case HG_CIC: launch(k_tile_accum_src<T, CPLX, HG_CIC, F>); break;
                case HG_TSC: launch(k_tile_accum_src<T, CPLX, HG_TSC, F>); break;
                default: launch(k_tile_accum_src<T, CPLX, HG_PCS, F>); break;
            }
        };
        if constexpr (sizeof(T) == 4) {
            if (fix) by_scheme(std::true_type{});
            else by_scheme(std::false_type{});
        } else {
            by_scheme(std::false_type{});
        }
        ke();
        double hm[2];
        HG_CK(cudaMemcpyAsync(hm, mass.p, sizeof(double) * 2, cudaMemcpyDeviceToHost, st));
        HG_CK(cudaStreamSynchronize(st));
        return {hm[0], hm[1]};
    }

    SpecK sfield(int kind, int l, int m, double alpha) {
        if (src_kind == 3) {  // line of sight z: Yhat_{l,0} = 1 per particle (see src_kind)
            HG_REQUIRE(m == 0, "the reconstructed box has M = 0 fields only");
            l = 0;
        }
        if (alpha != sf_alpha) {
            sf_ok.clear();
            sf_alpha = alpha;
        }
        const int hz = g.n[2] / 2 + 1;
        const bool real = (m == 0);
        const std::array<int, 3> key{kind, l, m};
        auto &pb = sfbuf[key];
        if (!pb) pb = std::make_unique<DBuf>();
        if (sf_ok.count(key)) {
            const auto &k0 = sfk0[key];
            return SpecK{Spec<T>{dp<C>(*pb), g.n[0], g.n[1], g.n[2], real ? 1 : 0}, k0[0], k0[1]};
        }
        const long long fsz = real ? (long long)g.n[0] * g.n[1] * hz : g.ntot;
        if (m < 0) {  // sgn conj(F_{l,|m|}(-k)), sgn = (-1)^m
            SpecK pos = sfield(kind, l, -m, alpha);
            const double sg = ((-m) % 2) ? -1.0 : 1.0;
            HG_CK(pb->ensure(sizeof(C) * fsz));
            unsigned blocks = (unsigned)std::min<long long>(grid1(g.ntot, 256), 148 * 16);
            kb("survey_mirror", double(g.ntot) * sizeof(C) * 2.0);
            k_mirror<T><<<blocks, 256, 0, st>>>(pos.s.p, dp<C>(*pb), g.n[0], g.n[1], g.n[2], (T)sg);
            ke();
            sfk0[key] = {sg * pos.k0r, -sg * pos.k0i};
            sf_ok.insert(key);
            return SpecK{Spec<T>{dp<C>(*pb), g.n[0], g.n[1], g.n[2], 0}, sg * pos.k0r, -sg * pos.k0i};
        }
        HG_CK(pb->ensure(sizeof(C) * fsz));
        const bool ylm = !(l == 0 && m == 0);
        std::vector<PartSrc> srcs;
        if (kind == SF_DELTA)
            srcs = {survey_src(0, ylm, l, m, 1.0), survey_src(1, ylm, l, m, -alpha)};
        else if (kind == SF_SN)
            srcs = {survey_src(0, ylm, l, m, 1.0, 2, true), survey_src(1, ylm, l, m, alpha * alpha, 2, true)};
        else if (kind == SF_WIN)  // the data (if any were binned with the randoms) weigh nothing
            srcs = {survey_src(0, ylm, l, m, 0.0), survey_src(1, ylm, l, m, 1.0)};
        else
            srcs = {survey_src(0, ylm, l, m, 0.0, 2, true), survey_src(1, ylm, l, m, 1.0, 2, true)};
        HG_CK(smesh_re.ensure(sizeof(T) * g.ntot));
        if (!real) HG_CK(smesh_im.ensure(sizeof(T) * g.ntot));
        const double dV = g.volume / double(g.ntot);
        // assign (mass units: dV rho, the transform's input) with a shift, transform into F;
        // returns the FP64 in-bounds mass, the transform's exact k = 0 value
        auto build = [&](double shift, C *F) {
            const int kb_ = shift != 0.0 ? 1 : 0;
            double mi = 0.0, mr;
            if (real) {
                const std::array<double, 2> mm = survey_accumulate<false>(kb_, srcs.data(), dp<T>(smesh_re), nullptr);
                mr = mm[0];
                mi = mm[1];
                forward_real(dp<T>(smesh_re), F, (T)0, (T)1, "fft_survey");
            } else {
                const std::array<double, 2> mm =
                    survey_accumulate<true>(kb_, srcs.data(), dp<T>(smesh_re), dp<T>(smesh_im));
                mr = mm[0];
                mi = mm[1];
                const long long yz = (long long)g.n[1] * g.n[2];
                pass<-1>(g.n[2], LdPlanar<T>{dp<T>(smesh_re), dp<T>(smesh_im), g.n[2]}, StArr<T>{F, g.n[2], 1},
                         (long long)g.n[0] * g.n[1], 1, "fft_survey", double(g.ntot) * (2 * sizeof(T) + sizeof(C)));
                pass<-1>(g.n[1], LdArr<T>{F, g.n[1], g.n[2]}, StArr<T>{F, g.n[1], g.n[2]}, g.n[0], g.n[2], "fft_survey");
                pass<-1>(g.n[0], LdArr<T>{F, g.n[0], yz}, StArr<T>{F, g.n[0], yz}, 1, yz, "fft_survey");
            }
            return std::array<double, 2>{mr * dV, real ? 0.0 : mi * dV};
        };
        std::array<double, 2> k0 = build(0.0, dp<C>(*pb));
        if (cfg.interlace) {
            HG_CK(sfield_tmp.ensure(sizeof(C) * fsz));
            std::array<double, 2> k1 = build(0.5, dp<C>(sfield_tmp));
            interlace_combine(dp<C>(*pb), dp<C>(sfield_tmp), real);
            k0 = {0.5 * (k0[0] + k1[0]), 0.5 * (k0[1] + k1[1])};
        }
        kb("set_k0", double(sizeof(C)));
        k_set_k0<T><<<1, 1, 0, st>>>(dp<C>(*pb), (T)k0[0], (T)k0[1]);
        ke();
        sfk0[key] = k0;
        sf_ok.insert(key);
        return SpecK{Spec<T>{dp<C>(*pb), g.n[0], g.n[1], g.n[2], real ? 1 : 0}, k0[0], k0[1]};
    }

    // S3_LM = sum_D w^3 Yhat_LM - alpha^3 sum_R w^3 Yhat_LM for M = -L..L (field.hpp:1212-1232);
    // M < 0 from Yhat_{L,-M} = (-1)^M conj Yhat_{L,M}
    std::map<int, std::vector<double>> s3_cache;  // per L: [M + L] complex, for s3_alpha
    double s3_alpha = 0.0;
    std::array<double, 2> survey_s3(int L, int M, double alpha) {
        if (src_kind == 3) {  // N_D - alpha^3 N_R (field.hpp:1242-1250): unit weights, Yhat_L0(z) = 1
            HG_REQUIRE(M == 0, "the reconstructed box has M = 0 terms only");
            return {double(slot[0].n) - alpha * alpha * alpha * double(slot[1].n), 0.0};
        }
        if (alpha != s3_alpha) {
            s3_cache.clear();
            s3_alpha = alpha;
        }
        auto it = s3_cache.find(L);
        if (it == s3_cache.end()) {
            PSumSpec q{};
            q.n = L + 1;
            HG_REQUIRE(q.n <= HG_PSUM_MAX, "ELL too large");
            for (int m = 0; m <= L; m++) {
                q.pw[m] = 3;
                q.l[m] = L;
                q.m[m] = m;
            }
            std::vector<double> sD = particle_sums(0, q), sR = particle_sums(1, q);
            const double a3 = alpha * alpha * alpha;
            std::vector<double> v(2 * (2 * L + 1));
            for (int m = 0; m <= L; m++) {
                const double re = sD[2 * m] - a3 * sR[2 * m], im = sD[2 * m + 1] - a3 * sR[2 * m + 1];
                const double sg = (m % 2) ? -1.0 : 1.0;
                v[2 * (L + m)] = re;
                v[2 * (L + m) + 1] = im;
                v[2 * (L - m)] = sg * re;
                v[2 * (L - m) + 1] = -sg * im;
            }
            it = s3_cache.emplace(L, std::move(v)).first;
        }
        return {it->second[2 * (L + M)], it->second[2 * (L + M) + 1]};
    }

    // S_LM = sum_D w^2 Yhat_LM + alpha^2 sum_R w^2 Yhat_LM (calcShotNoiseForPowerspectrum,
    // field.hpp:1164-1185), or sum_R w^2 Yhat_LM alone (rand_only:
    // calcShotNoiseForTwoPointWindowCorrelationFunction, field.hpp:1202-1217); any M
    std::array<double, 2> survey_s2(int L, int M, double alpha, bool rand_only) {
        const int am = M < 0 ? -M : M;
        PSumSpec q{};
        q.n = 1;
        q.pw[0] = 2;
        q.l[0] = L;
        q.m[0] = am;
        const std::vector<double> sR = particle_sums(1, q);
        double re = (rand_only ? 1.0 : alpha * alpha) * sR[0], im = (rand_only ? 1.0 : alpha * alpha) * sR[1];
        if (!rand_only) {
            const std::vector<double> sD = particle_sums(0, q);
            re += sD[0];
            im += sD[1];
        }
        if (M < 0) {  // Yhat_{L,-M} = (-1)^M conj Yhat_{L,M}
            const double sg = (am % 2) ? -1.0 : 1.0;
            re = sg * re;
            im = -sg * im;
        }
        return {re, im};
    }

    template <int LZ>
    void launch_line_L(const HistSpec &hs, double *hist) {
        size_t smem = OrbitCfg<T, LZ>::smem();
        HG_CK(cudaFuncSetAttribute(k_xi_line_hist<T, LZ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        const long long nl = (long long)g.n[0] * g.n[1];
        const unsigned blocks = (unsigned)((nl + OrbitCfg<T, LZ>::B - 1) / OrbitCfg<T, LZ>::B);
        kb("xi_line_hist", double(g.ntot) * sizeof(C));
        k_xi_line_hist<T, LZ><<<blocks, OrbitCfg<T, LZ>::NT, smem, st>>>(dp<C>(xi), g.n[0], g.n[1], twiddles(LZ), hs,
                                                                         n2dim, hist);
        ke();
    }
    void launch_line(const HistSpec &hs, double *hist) {
        switch (g.n[2]) {
            case 8: launch_line_L<8>(hs, hist); break;
            case 16: launch_line_L<16>(hs, hist); break;
            case 32: launch_line_L<32>(hs, hist); break;
            case 64: launch_line_L<64>(hs, hist); break;
            case 128: launch_line_L<128>(hs, hist); break;
            case 256: launch_line_L<256>(hs, hist); break;
            case 512: launch_line_L<512>(hs, hist); break;
            case 1024: launch_line_L<1024>(hs, hist); break;
            default: throw HgError{"unsupported n_mesh_z"};
        }
    }

    // hist_sv[mp][n2] = sum over M and the (m1, m2) of that M of w sum_{|x|^2 = n2} xi_LM(x)
    // Yhat_l1m1(x) Yhat_l2m2(x), with xi_LM = FFT_+[(dn_LM conj N_00 - S3_LM C) / W^2 / V]
    // (calcShotNoiseForBispectrum_ijk field.hpp:1116-1160; bispec.hpp:124-196, 400-460)
    void survey_histograms(const std::vector<MP> &mps) {
        build_orbits();
        std::vector<MP> todo;
        for (const auto &mp : mps) {
            std::array<int, 3> key{mp.l1, mp.l2, mp.L};
            bool queued = false;
            for (const auto &q : todo) queued |= (q.l1 == mp.l1 && q.l2 == mp.l2 && q.L == mp.L);
            if (!hist_sv_ok.count(key) && !queued) todo.push_back(mp);
        }
        if (todo.empty()) return;
        for (const auto &mp : todo) {
            auto &p = hist_sv[{mp.l1, mp.l2, mp.L}];
            if (!p) p = std::make_unique<DBuf>();
            HG_CK(p->ensure(sizeof(double) * 2 * nkey));
            HG_CK(cudaMemsetAsync(p->p, 0, sizeof(double) * 2 * nkey, st));
        }
        const double alpha = src_alpha;
        const SpecK n00 = sfield(sn_kind(), 0, 0, alpha);
        std::set<int> Ls;
        for (const auto &mp : todo) Ls.insert(mp.L);
        HG_CK(xi.ensure(sizeof(C) * g.ntot));
        xi_valid = false;  // the box correlation field is overwritten
        for (int L : Ls)
            for (int M = -L; M <= L; M++) {
                std::vector<std::pair<MP, std::vector<Combo3>>> hm;
                for (const auto &mp : todo) {
                    if (mp.L != L) continue;
                    std::vector<Combo3> cs;
                    for (const auto &c : combos3(mp, all_M()))
                        if (c.M == M) cs.push_back(c);
                    if (!cs.empty()) hm.push_back({mp, cs});
                }
                if (hm.empty()) continue;
                const SpecK f1 = sfield(delta_kind(), L, M, alpha);
                // the window 3PCF subtracts sum_R w^2 Yhat_LM (bispec.hpp:700), the survey
                // S3_LM (bispec.hpp:446)
                const std::array<double, 2> S3 = (src_kind == 2) ? survey_s2(L, M, 0.0, true) : survey_s3(L, M, alpha);
                // (f1 conj f2)(0) from the exact k = 0 values
                const double k0r = f1.k0r * n00.k0r + f1.k0i * n00.k0i, k0i = f1.k0i * n00.k0r - f1.k0r * n00.k0i;
                LdXiCross<T> ld{f1.s, n00.s, g.n[2], xtabs, S3[0], S3[1], k0r, k0i, 1.0 / g.volume};
                xi_x_pass(ld);
                pass<+1>(g.n[1], LdArr<T>{dp<C>(xi), g.n[1], g.n[2]}, StArr<T>{dp<C>(xi), g.n[1], g.n[2]}, g.n[0],
                         g.n[2], "fft_xi_y");
                if (xi_general) xi_z_pass();
                for (size_t h0 = 0; h0 < hm.size(); h0 += HG_MAX_HIST) {
                    HistSpec hs;
                    memset(&hs, 0, sizeof(hs));
                    hs.nh = (int)std::min<size_t>(HG_MAX_HIST, hm.size() - h0);
                    for (int h = 0; h < hs.nh; h++) {
                        const auto &e = hm[h0 + h];
                        HG_REQUIRE(e.second.size() <= 12, "too many (m1, m2) terms in one multipole");
                        hs.parity[h] = 1;
                        for (const auto &c : e.second)
                            hs.term[h][hs.nterm[h]++] = YTerm{e.first.l1, c.m1, e.first.l2, c.m2, c.w};
                    }
                    HG_CK(hist_tmp.ensure(sizeof(double) * 2 * nkey * hs.nh));
                    line_hist(hs, dp<double>(hist_tmp));
                    for (int h = 0; h < hs.nh; h++) {
                        const MP &mp = hm[h0 + h].first;
                        double *dst = dp<double>(*hist_sv[{mp.l1, mp.l2, mp.L}]);
                        k_axpy<<<grid1(2 * nkey, 256), 256, 0, st>>>(dst, dp<double>(hist_tmp) + 2 * nkey * h,
                                                                      2 * nkey);
                        HG_CK(cudaGetLastError());
                    }
                }
            }
        for (const auto &mp : todo) hist_sv_ok.insert({mp.l1, mp.l2, mp.L});
    }

    // the z inverse pass of a correlation field whose x and y passes are done, in place (the
    // meshes that fold_hist serves)
    void xi_z_pass() {
        pass<+1>(g.n[2], LdArr<T>{dp<C>(xi), g.n[2], 1}, StArr<T>{dp<C>(xi), g.n[2], 1}, (long long)g.n[0] * g.n[1], 1,
                 "fft_xi_z", double(g.ntot) * sizeof(C) * 2.0);
    }
    // histograms with azimuth-dependent weights ([h][key], written whole): the line kernel
    // (z pass fused) on its meshes, the fold of the fully transformed field otherwise
    void line_hist(const HistSpec &hs, double *hist) {
        if (xi_general) {
            fold_hist(hs, false, hist);
            return;
        }
        HG_CK(cudaMemsetAsync(hist, 0, sizeof(double) * 2 * nkey * hs.nh, st));
        launch_line(hs, hist);
    }

    static bool needs_los(const std::vector<MP> &mps) {
        for (const auto &mp : mps)
            if (mp.l1 || mp.l2 || mp.L) return true;
        return false;
    }

    // calcNormalizationForBiSpectrum (particle.hpp:319-332): V_s^2 / (sum w_D)^3
    double survey_bk_norm(double vs) {
        PSumSpec q{};
        q.n = 1;
        q.pw[0] = 1;
        q.l[0] = -1;
        const double wD = particle_sums(0, q)[0];
        HG_REQUIRE(wD != 0.0, "the summed data weights must be non-zero");
        double nv = vs / wD / wD;
        nv *= (vs / wD);
        return nv;
    }

    // calcBiSpectrum (bispec.hpp:4-352) for all k1 rows (ith = -1) or one, several multipoles
    void bk_survey_multi(const std::vector<MP> &mps, int ith, double alpha, double vs, double *bk_save,
                         double *sn_save, double *norm) override {
        check_multipoles(mps);
        HG_REQUIRE(ith >= -1 && ith < cfg.n_kbin, "ith_kbin out of range");
        require_survey(needs_los(mps));
        begin();
        set_source(1, alpha);
        bk_two_catalogues(mps, ith, alpha, bk_save, sn_save);
        if (norm) *norm = survey_bk_norm(vs);
        end();
    }

    // calcBiSpectrumForBOXForReconstruction (bispec.hpp:1426-1753): the survey estimator's
    // structure on the reconstructed box catalogues (source kind 3); norm V^2 / N_D^3
    void bk_box_recon_multi(const std::vector<MP> &mps, int ith, double alpha, double *bk_save, double *sn_save,
                            double *norm) override {
        check_multipoles(mps);
        HG_REQUIRE(ith >= -1 && ith < cfg.n_kbin, "ith_kbin out of range");
        require_box_recon();
        begin();
        set_source(3, alpha);
        bk_two_catalogues(mps, ith, alpha, bk_save, sn_save);
        if (norm) *norm = box_recon_norm();
        end();
    }
    void require_box_recon() const {
        HG_REQUIRE(slot[0].set && slot[1].set,
                   "the reconstructed box needs data (slot 0) and randoms (slot 1): call hg_set_particles for both");
    }
    double box_recon_norm() const {
        const double nd = double(slot[0].n);
        return g.volume / nd / nd * (g.volume / nd);
    }

    // B and its shot noise of a two-catalogue source (survey, reconstructed box): S3 term,
    // P terms, xi term (bispec.hpp:20-214, 1443-1616)
    void bk_two_catalogues(const std::vector<MP> &mps, int ith, double alpha, double *bk_save, double *sn_save) {
        const int ns = cfg.n_kbin;
        std::vector<std::vector<double>> B = bk_main(mps);
        // shot noise (bispec.hpp:20-214): S3 term, P terms, xi term
        const SpecK dn00 = sfield(SF_DELTA, 0, 0, alpha);
        std::vector<std::vector<double>> SN(mps.size(), std::vector<double>(2 * ns * ns, 0.0));
        std::vector<unsigned long long> nm;
        for (size_t q = 0; q < mps.size(); q++) {
            const MP &mp = mps[q];
            for (const auto &c : combos3(mp, all_M())) {
                const std::array<double, 2> S3 = survey_s3(mp.L, c.M, alpha);
                if (mp.l1 == 0 && mp.l2 == 0)
                    for (int e = 0; e < ns * ns; e++) {
                        SN[q][2 * e] += c.w * S3[0];
                        SN[q][2 * e + 1] += c.w * S3[1];
                    }
                if (mp.l2 == 0 || mp.l1 == 0) {
                    const SpecK nlm = sfield(SF_SN, mp.L, c.M, alpha);
                    if (mp.l2 == 0) {  // the k1 row's value on every k2
                        std::vector<double> avg;
                        pk_bin2(dn00.s, nlm.s, {LM{mp.l1, c.m1}}, S3[0], S3[1], avg, nm);
                        for (int i1 = 0; i1 < ns; i1++)
                            for (int i2 = 0; i2 < ns; i2++) {
                                SN[q][2 * (i1 * ns + i2)] += c.w * avg[2 * i1];
                                SN[q][2 * (i1 * ns + i2) + 1] += c.w * avg[2 * i1 + 1];
                            }
                    }
                    if (mp.l1 == 0) {
                        std::vector<double> avg;
                        pk_bin2(dn00.s, nlm.s, {LM{mp.l2, c.m2}}, S3[0], S3[1], avg, nm);
                        for (int i1 = 0; i1 < ns; i1++)
                            for (int i2 = 0; i2 < ns; i2++) {
                                SN[q][2 * (i1 * ns + i2)] += c.w * avg[2 * i2];
                                SN[q][2 * (i1 * ns + i2) + 1] += c.w * avg[2 * i2 + 1];
                            }
                    }
                }
            }
        }
        survey_histograms(mps);
        for (size_t q = 0; q < mps.size(); q++)
            bk_sn_xi(mps[q], dp<double>(*hist_sv[{mps[q].l1, mps[q].l2, mps[q].L}]), SN[q]);
        const int r0 = (ith < 0) ? 0 : ith, r1 = (ith < 0) ? ns : ith + 1;
        const int rows = r1 - r0;
        for (size_t q = 0; q < mps.size(); q++)
            for (int i1 = r0; i1 < r1; i1++)
                for (int i2 = 0; i2 < ns; i2++) {
                    long long o = ((long long)q * rows + (i1 - r0)) * ns + i2;
                    bk_save[2 * o] = B[q][2 * (i1 * ns + i2)];
                    bk_save[2 * o + 1] = B[q][2 * (i1 * ns + i2) + 1];
                    sn_save[2 * o] = SN[q][2 * (i1 * ns + i2)];
                    sn_save[2 * o + 1] = SN[q][2 * (i1 * ns + i2) + 1];
                }
    }

    // calcThreePointCorrelationFunctionForBOXForReconstruction (bispec.hpp:1755-1990): as
    // the survey 3PCF on the reconstructed box catalogues (source kind 3); norm V^2 / N_D^3
    void zeta_box_recon_multi(const std::vector<MP> &mps, int ith, double alpha, double *zeta_save,
                              double *sn_save, double *norm) override {
        check_multipoles(mps);
        HG_REQUIRE(ith >= -1 && ith < cfg.n_rbin, "ith_rbin out of range");
        require_box_recon();
        begin();
        zeta_geometry();
        set_source(3, alpha);
        std::vector<std::vector<double>> Z = zeta_main(mps, ith);
        survey_histograms(mps);
        std::vector<const double *> hs;
        for (const auto &mp : mps) hs.push_back(dp<double>(*hist_sv[{mp.l1, mp.l2, mp.L}]));
        zeta_finish(mps, ith, Z, hs, zeta_save, sn_save);
        if (norm) *norm = box_recon_norm();
        end();
    }

    // calcThreePointCorrelationFunction (bispec.hpp:355-614), all r1 rows or one
    void zeta_survey_multi(const std::vector<MP> &mps, int ith, double alpha, double vs, double *zeta_save,
                           double *sn_save, double *norm) override {
        check_multipoles(mps);
        HG_REQUIRE(ith >= -1 && ith < cfg.n_rbin, "ith_rbin out of range");
        require_survey(needs_los(mps));
        begin();
        zeta_geometry();
        set_source(1, alpha);
        std::vector<std::vector<double>> Z = zeta_main(mps, ith);
        survey_histograms(mps);
        std::vector<const double *> hs;
        for (const auto &mp : mps) hs.push_back(dp<double>(*hist_sv[{mp.l1, mp.l2, mp.L}]));
        zeta_finish(mps, ith, Z, hs, zeta_save, sn_save);
        if (norm) *norm = survey_bk_norm(vs);
        end();
    }

    // calcThreePointWindowCorrelationFunction (bispec.hpp:617-874): the survey 3PCF of the
    // randoms alone (Yhat w fields of n_R), its shot noise from conj(Yhat) w^2 fields of n_R
    // with sum_R w^2 Yhat_LM subtracted; *norm = V_survey^2 / (sum w_R)^3
    void zeta_window_multi(const std::vector<MP> &mps, int ith, double vs, double *zeta_save, double *sn_save,
                           double *norm) override {
        check_multipoles(mps);
        HG_REQUIRE(ith >= -1 && ith < cfg.n_rbin, "ith_rbin out of range");
        require_randoms(needs_los(mps));
        begin();
        zeta_geometry();
        set_source(2, 0.0);
        std::vector<std::vector<double>> Z = zeta_main(mps, ith);
        survey_histograms(mps);
        std::vector<const double *> hs;
        for (const auto &mp : mps) hs.push_back(dp<double>(*hist_sv[{mp.l1, mp.l2, mp.L}]));
        zeta_finish(mps, ith, Z, hs, zeta_save, sn_save);
        if (norm) {
            const double wR = weight_sum(1);
            HG_REQUIRE(wR != 0.0, "the summed random weights must be non-zero");
            double nv = vs / wR / wR;
            nv *= (vs / wR);
            *norm = nv;
        }
        end();
    }

    void require_randoms(bool need_los) const {
        HG_REQUIRE(slot[1].set, "window functions need the randoms (slot 1): call hg_set_particles(ctx, 1, ...)");
        if (need_los)
            HG_REQUIRE(slot[1].los_off >= 0, "window multipoles need line-of-sight vectors: pass los_off for the randoms");
    }

    double weight_sum(int s) {
        PSumSpec q{};
        q.n = 1;
        q.pw[0] = 1;
        q.l[0] = -1;
        return particle_sums(s, q)[0];
    }

    // ------------------------------------------------------------------ BAO reconstruction
    // calcReconstructionParticles (particle_reconstruction.hpp:12-208; box: :210-402) on this
    // context's mesh (the reference's n_mesh_recon): the D - alpha R field with the
    // context's scheme, its transform divided by W, three displacement components
    // Psi_a = FFT_+[-i (W_G / b1) (k_a / k^2) D / W / V] scaled by V_survey / sum w_D
    // (box: V / N_D, alpha = double(N_D / N_R) with the reference's integer division),
    // and every particle of both catalogues shifted by their TSC interpolation.
    DBuf psi_f[3], psi_tmp, shift_out;
    void reconstruct(int box, double b1, double RG, double alpha, double vs, double *posD, double *posR) override {
        HG_REQUIRE(slot[0].set && slot[1].set, "reconstruction needs data (slot 0) and randoms (slot 1)");
        HG_REQUIRE(b1 != 0.0, "b1_fid must be non-zero");
        begin();
        double a = alpha, norm;
        if (box) {
            a = double(slot[0].n / slot[1].n);  // particle_reconstruction.hpp:221 (integer division)
            norm = g.volume / double(slot[0].n);
        } else {
            const double wD = weight_sum(0);
            HG_REQUIRE(wD != 0.0, "the summed data weights must be non-zero");
            norm = vs / wD;
        }
        invalidate_stats();
        src_kind = -1;
        const SpecK D = sfield(SF_DELTA, 0, 0, a);
        HG_CK(psi_tmp.ensure(sizeof(C) * g.ntot));
        const long long yz = (long long)g.n[1] * g.n[2];
        const unsigned blocks = (unsigned)std::min<long long>(grid1(g.ntot, 256), 148 * 16);
        for (int ax = 0; ax < 3; ax++) {
            kb("recon_psi", double(g.ntot) * (sizeof(C) + 0.5 * sizeof(C)));
            k_recon_psi<T><<<blocks, 256, 0, st>>>(D.s, g, tabs, wpow, ax, RG, b1, dp<C>(psi_tmp));
            ke();
            pass<+1>(g.n[2], LdArr<T>{dp<C>(psi_tmp), g.n[2], 1}, StArr<T>{dp<C>(psi_tmp), g.n[2], 1},
                     (long long)g.n[0] * g.n[1], 1, "fft_recon");
            pass<+1>(g.n[1], LdArr<T>{dp<C>(psi_tmp), g.n[1], g.n[2]}, StArr<T>{dp<C>(psi_tmp), g.n[1], g.n[2]}, g.n[0],
                     g.n[2], "fft_recon");
            pass<+1>(g.n[0], LdArr<T>{dp<C>(psi_tmp), g.n[0], yz}, StArr<T>{dp<C>(psi_tmp), g.n[0], yz}, 1, yz,
                     "fft_recon");
            HG_CK(psi_f[ax].ensure(sizeof(T) * g.ntot));
            kb("recon_psi", double(g.ntot) * (sizeof(C) + sizeof(T)));
            k_real_scaled<T><<<blocks, 256, 0, st>>>(dp<C>(psi_tmp), g.ntot, norm, dp<T>(psi_f[ax]));
            ke();
        }
        psi_tmp.release();
        for (int s = 0; s < 2; s++) {
            double *dst = s == 0 ? posD : posR;
            if (!dst) continue;
            const PartSrc src = survey_src(s, false, 0, 0, 1.0);
            HG_CK(shift_out.ensure(sizeof(double) * 3 * src.n));
            kb("recon_shift", double(src.n) * (24.0 + 24.0));
            k_recon_shift<T><<<(unsigned)std::min<long long>(grid1(src.n, 256), 148 * 16), 256, 0, st>>>(
                src, g, dp<T>(psi_f[0]), dp<T>(psi_f[1]), dp<T>(psi_f[2]), dp<double>(shift_out));
            ke();
            HG_CK(cudaMemcpyAsync(dst, shift_out.p, sizeof(double) * 3 * src.n, cudaMemcpyDeviceToHost, st));
            HG_CK(cudaStreamSynchronize(st));
        }
        for (int ax = 0; ax < 3; ax++) psi_f[ax].release();
        shift_out.release();
        end();
    }

    // calcPowerSpectrumForBOXForReconstruction (powerspec.hpp:396-457): the box estimator on
    // dn = n_D - alpha n_R (weights 1) with shot noise N_D + alpha^2 N_R (field.hpp:1190-1196)
    void pk_box_recon(int ell, double alpha, double *pk_save, int *n_mode, double *norm) override {
        HG_REQUIRE(ell >= 0, "ell must be >= 0");
        HG_REQUIRE(slot[0].set && slot[1].set, "the reconstructed P needs data (slot 0) and randoms (slot 1)");
        begin();
        invalidate_stats();
        src_kind = -1;
        const SpecK f = sfield(SF_DELTA, 0, 0, alpha);
        const double S = double(slot[0].n) + alpha * alpha * double(slot[1].n);
        std::vector<double> avg;
        std::vector<unsigned long long> nm;
        pk_bin2(f.s, f.s, {LM{ell, 0}}, S, 0.0, avg, nm);
        for (int i = 0; i < cfg.n_kbin; i++) {
            pk_save[2 * i] = double(2 * ell + 1) * avg[2 * i];
            pk_save[2 * i + 1] = double(2 * ell + 1) * avg[2 * i + 1];
            if (n_mode) n_mode[i] = (int)nm[i];
        }
        if (norm) *norm = g.volume / double(slot[0].n) / double(slot[0].n);
        end();
    }

    // ------------------------------------------------------------------ 2PCF
    // The 2PCF's r binning (calcCorrelationFunction, field.hpp:854-977): fine index
    // int(|r| / 0.5 + 0.5) kept below 20000, coarse bin j takes fine i iff lower_j < 0.5 i <=
    // upper_j with the uniform width rbin[1] - rbin[0], averages by cell count.  Per n2 =
    // |x / dr|^2 (equal cell sizes; |r|^2 = n2 dr^2 is the reference's sum of (i dr)^2 exactly
    // when those squares are exact, e.g. dyadic dr): the fine index and the cells.
    struct Xi2Geo {
        bool built = false;
        std::vector<int> fine;                 // per n2; -1 past the fine table
        std::vector<std::vector<int>> coarse;  // per fine index
        std::vector<double> cells;             // per n2
    } x2;
    void xi2_geometry() {
        build_orbits();
        if (x2.built) return;
        x2.cells = key_cells;
        const int n_temp = 20000;
        const double dr_temp = 0.5;
        x2.fine.assign(nkey, -1);
        for (long long q = 0; q < nkey; q++) {
            const int ri = (int)(key_r[q] / dr_temp + 0.5);
            if (ri < n_temp) x2.fine[q] = ri;
        }
        const double dr_bin = rbin[1] - rbin[0];
        x2.coarse.assign(n_temp, {});
        for (int j = 0; j < cfg.n_rbin; j++) {
            const double lower = (rbin[j] > dr_bin * 0.5) ? (rbin[j] - dr_bin * 0.5) : 0.0;
            const double upper = rbin[j] + dr_bin * 0.5;
            for (int i = 0; i < n_temp; i++) {
                const double rt = double(i) * dr_temp;
                if ((rt > lower) && (rt <= upper)) x2.coarse[i].push_back(j);
            }
        }
        x2.built = true;
    }

    // xi_save[j] = scale * (sum of hist over the n2 of bin j) / (cells of bin j)
    void xi2_bin(const double *d_hist, double scale, double *xi_save, int *n_mode) {
        std::vector<double> h(2 * nkey);
        HG_CK(cudaMemcpyAsync(h.data(), d_hist, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, st));
        HG_CK(cudaStreamSynchronize(st));
        const int nr = cfg.n_rbin;
        std::vector<double> xr(nr, 0.0), xim(nr, 0.0), nm(nr, 0.0);
        for (long long q = 0; q < nkey; q++) {
            const int f = x2.fine[q];
            if (f < 0) continue;
            for (int j : x2.coarse[f]) {
                xr[j] += h[2 * q];
                xim[j] += h[2 * q + 1];
                nm[j] += x2.cells[q];
            }
        }
        for (int j = 0; j < nr; j++) {
            xi_save[2 * j] = nm[j] != 0.0 ? scale * (xr[j] / nm[j]) : 0.0;
            xi_save[2 * j + 1] = nm[j] != 0.0 ? scale * (xim[j] / nm[j]) : 0.0;
            if (n_mode) n_mode[j] = (int)nm[j];
        }
    }

    // calcTwoPointFunctionForBOXForReconstruction (powerspec.hpp:459-520): the box 2PCF of
    // dn = n_D - alpha n_R (weights 1), shot noise N_D + alpha^2 N_R, norm V / N_D^2
    void xi_box_recon(int ell, double alpha, double *xi_save, int *n_mode, double *norm) override {
        HG_REQUIRE(ell >= 0, "ell must be >= 0");
        HG_REQUIRE(slot[0].set && slot[1].set, "the reconstructed 2PCF needs data (slot 0) and randoms (slot 1)");
        begin();
        invalidate_stats();
        src_kind = -1;
        xi2_geometry();
        const SpecK f = sfield(SF_DELTA, 0, 0, alpha);
        build_box_xi(f.s, double(slot[0].n) + alpha * alpha * double(slot[1].n), f.k0r * f.k0r + f.k0i * f.k0i);
        xi_valid = false;  // not the box density's correlation field
        HistSpec hs;
        memset(&hs, 0, sizeof(hs));
        hs.nh = 1;
        hs.parity[0] = (ell % 2 == 0) ? 1 : -1;
        hs.term[0][hs.nterm[0]++] = YTerm{ell, 0, 0, 0, 1.0};
        orbit_weight_poly(hs, 0);
        HG_CK(hist_tmp.ensure(sizeof(double) * 2 * nkey));
        box_hist(hs, dp<double>(hist_tmp));
        xi2_bin(dp<double>(hist_tmp), double(2 * ell + 1), xi_save, n_mode);
        if (norm) *norm = g.volume / double(slot[0].n) / double(slot[0].n);
        end();
    }

    // calcTwoPointCorrelationFunctionForBOX (powerspec.hpp:334-393): xi = FFT_+[(|dn|^2 - N C)
    // / W^2] / V, r-binned with the Legendre weight L_l(mu); xi_save = (2l+1) xi, norm V / N^2
    void xi_box(int ell, double *xi_save, int *n_mode, double *norm) override {
        HG_REQUIRE(ell >= 0, "ell must be >= 0");
        begin();
        set_source(0, 0.0);
        xi2_geometry();
        ensure_xi(delta0 * delta0);
        HistSpec hs;
        memset(&hs, 0, sizeof(hs));
        hs.nh = 1;
        hs.parity[0] = (ell % 2 == 0) ? 1 : -1;
        hs.term[0][hs.nterm[0]++] = YTerm{ell, 0, 0, 0, 1.0};
        orbit_weight_poly(hs, 0);
        HG_CK(hist_tmp.ensure(sizeof(double) * 2 * nkey));
        box_hist(hs, dp<double>(hist_tmp));
        xi2_bin(dp<double>(hist_tmp), double(2 * ell + 1), xi_save, n_mode);
        if (norm) *norm = g.volume / double(slot[0].n) / double(slot[0].n);
        end();
    }

    // calcTwoPointCorrelationFunction (powerspec.hpp:93-180; window: false) and
    // calcTwoPointWindowCorrelationFunction (powerspec.hpp:182-270; window: true): sum over
    // M and m1 of w3j-weighted r-binned xi_LM Yhat_{l m1}(r), xi_LM = FFT_+[(dn_LM conj dn_00 -
    // S_LM C) / W^2] / V; norm V_survey / (sum w)^2 of the data (randoms for the window)
    void xi_survey(int ell, bool window, double alpha, double vs, double *xi_save, int *n_mode,
                   double *norm) override {
        HG_REQUIRE(ell >= 0, "ell must be >= 0");
        if (window) require_randoms(ell > 0);
        else require_survey(ell > 0);
        begin();
        set_source(window ? 2 : 1, window ? 0.0 : alpha);
        xi2_geometry();
        const SpecK f00 = sfield(delta_kind(), 0, 0, src_alpha);
        HG_CK(xi.ensure(sizeof(C) * g.ntot));
        xi_valid = false;  // the box correlation field is overwritten
        HG_CK(xi2acc.ensure(sizeof(double) * 2 * nkey));
        HG_CK(cudaMemsetAsync(xi2acc.p, 0, sizeof(double) * 2 * nkey, st));
        HG_CK(hist_tmp.ensure(sizeof(double) * 2 * nkey));
        for (int M = -ell; M <= ell; M++) {
            HistSpec hs;
            memset(&hs, 0, sizeof(hs));
            hs.nh = 1;
            hs.parity[0] = 1;
            for (int m1 = -ell; m1 <= ell; m1++) {
                double w = wigner3j(ell, 0, ell, 0, 0, 0) * wigner3j(ell, 0, ell, m1, 0, M);
                w *= double(2 * ell + 1) * double(2 * ell + 1);
                if (std::fabs(w) < 1.0e-10) continue;
                HG_REQUIRE(hs.nterm[0] < 12, "too many (m1) terms in one 2PCF multipole");
                hs.term[0][hs.nterm[0]++] = YTerm{ell, m1, 0, 0, w};
            }
            if (hs.nterm[0] == 0) continue;
            const SpecK f1 = sfield(delta_kind(), ell, M, src_alpha);
            const std::array<double, 2> S = survey_s2(ell, M, src_alpha, window);
            const double k0r = f1.k0r * f00.k0r + f1.k0i * f00.k0i, k0i = f1.k0i * f00.k0r - f1.k0r * f00.k0i;
            LdXiCross<T> ld{f1.s, f00.s, g.n[2], xtabs, S[0], S[1], k0r, k0i, 1.0 / g.volume};
            xi_x_pass(ld);
            pass<+1>(g.n[1], LdArr<T>{dp<C>(xi), g.n[1], g.n[2]}, StArr<T>{dp<C>(xi), g.n[1], g.n[2]}, g.n[0], g.n[2],
                     "fft_xi_y");
            if (xi_general) xi_z_pass();
            line_hist(hs, dp<double>(hist_tmp));
            k_axpy<<<grid1(2 * nkey, 256), 256, 0, st>>>(dp<double>(xi2acc), dp<double>(hist_tmp), 2 * nkey);
            HG_CK(cudaGetLastError());
        }
        xi2_bin(dp<double>(xi2acc), 1.0, xi_save, n_mode);
        if (norm) {
            const double ws = weight_sum(window ? 1 : 0);
            HG_REQUIRE(ws != 0.0, "the summed weights must be non-zero");
            *norm = vs / ws / ws;
        }
        end();
    }
    DBuf xi2acc;

    // calcPowerSpectrum (powerspec.hpp:4-91): sum over M of w3j-weighted binned
    // (dn_LM conj dn_00 - S_LM C) / W^2 Yhat_{l m1}(k), S_LM = sum_D w^2 Yhat_LM + alpha^2 sum_R
    // w^2 Yhat_LM (field.hpp:1164-1185).  Fields for M < 0 are mirrors of M > 0.
    void pk_survey(int ell, double alpha, double vs, double *pk_save, int *n_mode, double *norm) override {
        HG_REQUIRE(ell >= 0, "ell must be >= 0");
        require_survey(ell > 0);
        begin();
        const int nb = cfg.n_kbin;
        PSumSpec q{};
        q.n = ell + 1;
        HG_REQUIRE(q.n <= HG_PSUM_MAX, "ell too large");
        for (int M = 0; M <= ell; M++) {
            q.pw[M] = 2;
            q.l[M] = ell;
            q.m[M] = M;
        }
        std::vector<double> sD = particle_sums(0, q), sR = particle_sums(1, q);
        q.n = 1;
        q.pw[0] = 1;
        q.l[0] = -1;
        const double wD = particle_sums(0, q)[0];
        HG_REQUIRE(wD != 0.0, "the summed data weights must be non-zero");
        const Spec<T> f00 = sfield(SF_DELTA, 0, 0, alpha).s;
        std::vector<double> acc(2 * nb, 0.0);
        std::vector<unsigned long long> nm;
        if (nb <= 256 && 2 * ell + 1 <= HG_MAX_PK_TERMS) {
            // every M of this l in one pass over the modes
            PkTerms<T> terms{};
            for (int M = -ell; M <= ell; M++) {
                const int am = M < 0 ? -M : M;
                double Sr = sD[2 * am] + alpha * alpha * sR[2 * am];
                double Si = sD[2 * am + 1] + alpha * alpha * sR[2 * am + 1];
                const Spec<T> f1 = sfield(SF_DELTA, ell, am, alpha).s;
                const double sg = (am % 2) ? -1.0 : 1.0;
                if (M < 0) {
                    Sr = sg * Sr;
                    Si = -sg * Si;
                }
                for (int m1 = -ell; m1 <= ell; m1++) {
                    double w = wigner3j(ell, 0, ell, 0, 0, 0) * wigner3j(ell, 0, ell, m1, 0, M);
                    w *= double(2 * ell + 1) * double(2 * ell + 1);
                    if (std::fabs(w) < 1.0e-10) continue;
                    HG_REQUIRE(terms.n < HG_MAX_PK_TERMS, "too many survey P terms");
                    terms.t[terms.n++] = PkTerm<T>{f1, M < 0 ? 1 : 0, sg, Sr, Si, ell, m1, w};
                }
            }
            std::vector<double> avg;
            pk_bin_terms(terms, f00, avg, nm);
            acc = avg;
        } else {  // more bins or terms than the one-pass kernel holds: one pass per term
        for (int M = -ell; M <= ell; M++) {
            const int am = M < 0 ? -M : M;
            double Sr = sD[2 * am] + alpha * alpha * sR[2 * am];
            double Si = sD[2 * am + 1] + alpha * alpha * sR[2 * am + 1];
            const Spec<T> f1 = sfield(SF_DELTA, ell, am, alpha).s;
            const double sg = (am % 2) ? -1.0 : 1.0;
            if (M < 0) {  // dn_{l,-|M|}(k) = (-1)^|M| conj(dn_{l,|M|}(-k)); likewise S
                Sr = sg * Sr;
                Si = -sg * Si;
            }
            for (int m1 = -ell; m1 <= ell; m1++) {
                double w = wigner3j(ell, 0, ell, 0, 0, 0) * wigner3j(ell, 0, ell, m1, 0, M);
                w *= double(2 * ell + 1) * double(2 * ell + 1);
                if (std::fabs(w) < 1.0e-10) continue;
                std::vector<double> avg;
                if (M < 0)
                    pk_bin2(SpecMirror<T>{f1, sg}, f00, {LM{ell, m1}}, Sr, Si, avg, nm);
                else
                    pk_bin2(f1, f00, {LM{ell, m1}}, Sr, Si, avg, nm);
                for (int i = 0; i < nb; i++) {
                    acc[2 * i] += w * avg[2 * i];
                    acc[2 * i + 1] += w * avg[2 * i + 1];
                }
            }
        }
        }
        for (int i = 0; i < 2 * nb; i++) pk_save[i] = acc[i];
        if (n_mode)
            for (int i = 0; i < nb; i++) n_mode[i] = (int)nm[i];
        if (norm) *norm = vs / wD / wD;  // particle.hpp:303-316
        end();
    }
};

}  // namespace
