// hg_static.cu -- the one entry point of this library that allocates no device memory.
//
// hg_pk_box_spectrum_static bins a power-spectrum multipole out of a density spectrum the
// caller already holds on the device.  It is for callers that cannot call cudaMalloc:
// applications whose own allocator or memory budget owns every byte of the GPU (a library
// allocating behind their back would fail, or break their accounting), and loops that must
// not pay cudaMalloc's cost or its implicit device-wide synchronisation on every call.  It
// runs the same binning kernel as hg_pk_box, but every scratch buffer (the fine-to-coarse
// bin table, the per-axis window and shot-noise tables and the FP64 bin accumulators) lives
// in one file-scope __device__ array of HG_STATIC_SCRATCH_BYTES, which every GPU that loads
// this library holds until the process exits.
//
// Limits (rejected with an error, nothing launched): n_kbin <= 256; n_mesh <= 1024 per
// axis; the fine table needs at most 100000 entries (k bins up to |k| = 10, as in the
// reference's fine histogram).
//
// The first call on each device looks up the array's device address with
// cudaGetSymbolAddress (with that device current) and caches it.  All calls share the one
// array and it keeps the last call's contents: the accumulators are cleared at the start of
// every call, and calls whose work overlaps on the GPU (different streams or threads at the
// same time) race on it.  The call waits for its stream and copies the sums into host
// memory before it returns; it leaves the caller's current device as it found it.
#define HG_TU_NS tu_static
#include "hitomi_gpu.h"
#include "hg_common.cuh"
#include "hg_bin.cuh"

#include <algorithm>
#include <cmath>
#include <mutex>
#include <string>

#define HG_STATIC_SCRATCH_BYTES (1u << 20)
#define HG_STATIC_MAX_KBIN 256
#define HG_STATIC_MAX_MESH 1024
#define HG_STATIC_MAX_FINE 100000

namespace hg {
void set_contextless_error(const std::string &m);
}

using namespace hg;

static __device__ __align__(256) unsigned char g_hg_static_scratch[HG_STATIC_SCRATCH_BYTES];

namespace {

// Byte offsets of the parts of the scratch array.
constexpr size_t kOffAcc = 0;                                                  // double[2 * MAX_KBIN]
constexpr size_t kOffCnt = kOffAcc + sizeof(double) * 2 * HG_STATIC_MAX_KBIN;  // u64[MAX_KBIN]
constexpr size_t kOffTab = kOffCnt + sizeof(unsigned long long) * HG_STATIC_MAX_KBIN;  // double[6][MAX_MESH]
constexpr size_t kOffLut = kOffTab + sizeof(double) * 6 * HG_STATIC_MAX_MESH;           // int2[MAX_FINE]
constexpr size_t kEnd = kOffLut + sizeof(int2) * HG_STATIC_MAX_FINE;
static_assert(kEnd <= HG_STATIC_SCRATCH_BYTES, "static scratch layout exceeds the array");

std::mutex g_mu;
void *g_addr[256] = {nullptr};  // per device ordinal

int fail(const std::string &m) {
    set_contextless_error(m);
    return -1;
}

// Per-axis window / shot-noise tables (the same values k_axis_tables computes).
__global__ void k_static_axis_tables(Grid g, int axis, double *tw, double *ts) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int n = g.n[axis];
    if (i >= n) return;
    double kv = kcomp(wrap_index(i, n), g.dk[axis]);
    int w = window_index(kv, g.dk[axis]);
    tw[i] = sinc_axis(w, n);
    ts[i] = (w != 0) ? sin(HG_PI * (double)w / (double)n) : 0.0;
}

// Fine-bin -> coarse-bin table of field.hpp:823-837 (the host builder's rule, on device).
// Every product and sum is rounded separately, as the reference's host arithmetic is: a
// contracted multiply-add would move fine bins that sit exactly on a coarse edge.
__global__ void k_static_lut(double kmin, double dkk, int n_kbin, int n_fine, int2 *lut) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_fine) return;
    const double kbin0 = __dadd_rn(kmin, __dmul_rn(dkk, 0.0));
    const double kbin1 = __dadd_rn(kmin, __dmul_rn(dkk, 1.0));
    const double dk_bin = __dsub_rn(kbin1, kbin0);
    const double half = __dmul_rn(dk_bin, 0.5);
    const double kt = __dmul_rn(double(i), 0.0001);
    int2 r = make_int2(-1, -1);
    int nb = 0;
    for (int j = 0; j < n_kbin; j++) {
        const double kb = __dadd_rn(kmin, __dmul_rn(dkk, double(j)));
        const double lower = (kb > half) ? __dsub_rn(kb, half) : 0.0;
        const double upper = __dadd_rn(kb, half);
        if ((kt > lower) && (kt <= upper)) {
            if (nb == 0) r.x = j;
            else if (nb == 1) r.y = j;
            nb++;
        }
    }
    lut[i] = r;
}

void *scratch_address(int dev, std::string &err) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (dev < 0 || dev >= 256) {
        err = "device ordinal out of range";
        return nullptr;
    }
    if (g_addr[dev]) return g_addr[dev];
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_hg_static_scratch);
    if (e != cudaSuccess) {
        err = std::string("cudaGetSymbolAddress(static scratch): ") + cudaGetErrorString(e);
        return nullptr;
    }
    g_addr[dev] = p;
    return p;
}

template <typename T>
int run(const hg_config &c, const void *spec, long long n_particles, int ell, double *pk_save, int *n_mode,
        double *norm, cudaStream_t st, unsigned char *base) {
    Grid g;
    for (int a = 0; a < 3; a++) {
        g.n[a] = c.n_mesh[a];
        g.L[a] = c.boxsize[a];
        g.dk[a] = 2.0 * HG_PI / c.boxsize[a];
        g.dr[a] = c.boxsize[a] / double(c.n_mesh[a]);
    }
    g.volume = c.boxsize[0] * c.boxsize[1] * c.boxsize[2];
    g.ntot = (long long)c.n_mesh[0] * c.n_mesh[1] * c.n_mesh[2];
    const int nbin = c.n_kbin;
    const double dkk = (c.kmax - c.kmin) / double(nbin - 1);  // tools.hpp:118-124
    const double kbl = c.kmin + dkk * double(nbin - 1), dk_bin = (c.kmin + dkk) - c.kmin;
    const double kedge = kbl + dk_bin * 0.5;
    int n_fine = (int)std::ceil(kedge / 0.0001) + 2;
    if (n_fine > HG_STATIC_MAX_FINE) n_fine = HG_STATIC_MAX_FINE;
    double *acc = reinterpret_cast<double *>(base + kOffAcc);
    unsigned long long *cnt = reinterpret_cast<unsigned long long *>(base + kOffCnt);
    double *tab = reinterpret_cast<double *>(base + kOffTab);
    int2 *lut = reinterpret_cast<int2 *>(base + kOffLut);
    AxisTabs tabs;
    tabs.interlace = 0;
    for (int a = 0; a < 3; a++) {
        tabs.tc[a] = nullptr;
        tabs.tw[a] = tab + (2 * a) * HG_STATIC_MAX_MESH;
        tabs.ts[a] = tab + (2 * a + 1) * HG_STATIC_MAX_MESH;
        k_static_axis_tables<<<(g.n[a] + 127) / 128, 128, 0, st>>>(g, a, tab + (2 * a) * HG_STATIC_MAX_MESH,
                                                                  tab + (2 * a + 1) * HG_STATIC_MAX_MESH);
    }
    k_static_lut<<<(n_fine + 255) / 256, 256, 0, st>>>(c.kmin, dkk, nbin, n_fine, lut);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(std::string("table launches: ") + cudaGetErrorString(e));
    // the previous call's sums are still in the array
    e = cudaMemsetAsync(acc, 0, sizeof(double) * 2 * nbin, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * nbin, st);
    if (e != cudaSuccess) return fail(std::string("clearing the static accumulators: ") + cudaGetErrorString(e));
    // the mode cube that can reach a bin (as in the context path)
    int3 lo, cn;
    int *lop[3] = {&lo.x, &lo.y, &lo.z};
    int *cnp[3] = {&cn.x, &cn.y, &cn.z};
    for (int a = 0; a < 3; a++) {
        int ca = (int)std::floor(double(n_fine) * 0.0001 / g.dk[a]) + 1;
        int l0 = std::max(-ca, -g.n[a] / 2), h0 = std::min(ca, g.n[a] / 2 - 1);
        *lop[a] = l0;
        *cnp[a] = h0 - l0 + 1;
    }
    LMList lms;
    lms.n = 1;
    lms.lm[0] = LM{ell, 0};
    Spec<T> f{reinterpret_cast<const cplx<T> *>(spec), g.n[0], g.n[1], g.n[2], 1};
    size_t smem = sizeof(double) * 2 * nbin + sizeof(unsigned long long) * nbin;
    e = cudaFuncSetAttribute(k_pk_bin<T, Spec<T>, Spec<T>>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return fail(std::string("binning kernel attribute: ") + cudaGetErrorString(e));
    long long total = (long long)cn.x * cn.y * cn.z;
    unsigned blocks = (unsigned)std::min<long long>((total + 255) / 256, 148 * 8);
    const int wpow = c.assign + 1;
    k_pk_bin<T, Spec<T>, Spec<T>><<<blocks, 256, smem, st>>>(f, f, g, tabs, lo, cn, lut, n_fine, nbin, lms, double(n_particles), 0.0,
                                           c.assign, wpow, acc, cnt, 0, 0.0, 0.0);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(std::string("binning launch: ") + cudaGetErrorString(e));
    double hacc[2 * HG_STATIC_MAX_KBIN];
    unsigned long long hcnt[HG_STATIC_MAX_KBIN];
    e = cudaMemcpyAsync(hacc, acc, sizeof(double) * 2 * nbin, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hcnt, cnt, sizeof(unsigned long long) * nbin, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(std::string("static binning: ") + cudaGetErrorString(e));
    for (int i = 0; i < nbin; i++) {
        double re = 0.0, im = 0.0;
        if (hcnt[i] != 0) {
            re = hacc[2 * i] / double(hcnt[i]);
            im = hacc[2 * i + 1] / double(hcnt[i]);
        }
        pk_save[2 * i] = double(2 * ell + 1) * re;  // powerspec.hpp:307-309
        pk_save[2 * i + 1] = double(2 * ell + 1) * im;
        if (n_mode) n_mode[i] = (int)hcnt[i];
    }
    if (norm) *norm = g.volume / double(n_particles) / double(n_particles);  // powerspec.hpp:316
    return 0;
}

}  // namespace

extern "C" int hg_pk_box_spectrum_static(const hg_config *cfg, const void *d_half_spectrum, long long n_particles,
                                         int ell, double *pk_save, int *n_mode, double *norm, void *stream) {
    if (!cfg || !d_half_spectrum || !pk_save) return fail("hg_pk_box_spectrum_static: null argument");
    const hg_config &c = *cfg;
    if (c.n_kbin < 2 || c.n_kbin > HG_STATIC_MAX_KBIN)
        return fail("hg_pk_box_spectrum_static: n_kbin must be in [2, 256]");
    if (!(c.kmin > 0.0) || !(c.kmax > c.kmin)) return fail("hg_pk_box_spectrum_static: need 0 < kmin < kmax");
    for (int a = 0; a < 3; a++) {
        if (c.n_mesh[a] < 2 || c.n_mesh[a] > HG_STATIC_MAX_MESH)
            return fail("hg_pk_box_spectrum_static: n_mesh must be in [2, 1024] on every axis");
        if (!(c.boxsize[a] > 0.0)) return fail("hg_pk_box_spectrum_static: boxsize must be > 0");
    }
    if (c.assign < 0 || c.assign > 2 || c.interlace)
        return fail("hg_pk_box_spectrum_static: assignment must be NGP, CIC or TSC without interlacing");
    if (n_particles <= 0) return fail("hg_pk_box_spectrum_static: n_particles must be > 0");
    if (ell < 0) return fail("hg_pk_box_spectrum_static: ell must be >= 0");
    {
        const double dkk = (c.kmax - c.kmin) / double(c.n_kbin - 1);
        const double kedge = c.kmax + dkk * 0.5;
        if (std::ceil(kedge / 0.0001) + 2 > HG_STATIC_MAX_FINE)
            return fail("hg_pk_box_spectrum_static: k bins beyond |k| = 10 exceed the fine-bin table");
    }
    if (c.precision != HG_FP64 && c.precision != HG_FP32)
        return fail("hg_pk_box_spectrum_static: precision must be HG_FP64 or HG_FP32");
    int prev_dev = -1;
    cudaError_t e = cudaGetDevice(&prev_dev);
    if (e != cudaSuccess) return fail(std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    e = cudaSetDevice(c.device);
    if (e != cudaSuccess) return fail(std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    std::string err;
    int rc;
    void *base = scratch_address(c.device, err);
    if (!base) {
        rc = fail(err);
    } else {
        cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
        unsigned char *b = reinterpret_cast<unsigned char *>(base);
        rc = (c.precision == HG_FP64) ? run<double>(c, d_half_spectrum, n_particles, ell, pk_save, n_mode, norm, st, b)
                                      : run<float>(c, d_half_spectrum, n_particles, ell, pk_save, n_mode, norm, st, b);
    }
    // the caller's current device, as it was
    if (prev_dev != c.device) {
        e = cudaSetDevice(prev_dev);
        if (e != cudaSuccess && rc == 0) rc = fail(std::string("restoring the current device: ") + cudaGetErrorString(e));
    }
    return rc;
}
