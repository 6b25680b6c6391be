// hg_api.cu -- the C ABI of include/hitomi_gpu.h over the context interface (hg_ctx.hpp).
// Every entry point returns 0 / -1 and keeps the reason for hg_last_error, mirroring the
// reference's int-return convention (src/hitomi_measurement/field.hpp:61,
// powerspec.hpp:12-16); no exception crosses the ABI.
#include "hg_ctx.hpp"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

using hg::HgError;
using hg::MP;

namespace {
thread_local std::string g_create_error;
}  // namespace

namespace hg {
void set_contextless_error(const std::string &m) { g_create_error = m; }
const std::string &contextless_error() { return g_create_error; }
MemBudget *&current_budget() {
    thread_local MemBudget *b = nullptr;
    return b;
}
}  // namespace hg

namespace {
// charges the allocations of one API call to its context
struct BudgetScope {
    hg::MemBudget *prev;
    explicit BudgetScope(hg::MemBudget *b) : prev(hg::current_budget()) {
        b->hit = false;
        hg::current_budget() = b;
    }
    ~BudgetScope() { hg::current_budget() = prev; }
};

std::string with_budget_note(const hg_ctx *ctx, const std::string &m) {
    if (!ctx->budget.hit) return m;
    return m + " [the context's device memory limit of " + std::to_string(ctx->budget.limit) +
           " bytes (hg_set_memory_limit) was reached; it holds " + std::to_string(ctx->budget.used) + " bytes]";
}
}  // namespace

#define HG_CK(x)                                                                                    \
    do {                                                                                            \
        cudaError_t e_ = (x);                                                                       \
        if (e_ != cudaSuccess)                                                                      \
            throw HgError{std::string(#x) + ": " + cudaGetErrorString(e_) + " (" + __FILE__ + ":" + \
                          std::to_string(__LINE__) + ")"};                                          \
    } while (0)

extern "C" {

int hg_create(hg_ctx **out, const hg_config *cfg) {
    if (!out || !cfg) return -1;
    *out = nullptr;
    try {
        if (cfg->precision == HG_FP64) *out = hg::make_engine_fp64(*cfg);
        else if (cfg->precision == HG_FP32) *out = hg::make_engine_fp32(*cfg);
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
    cudaSetDevice(ctx->cfg.device);  // the buffers are freed on the context's GPU
    delete ctx;
    return 0;
}

const char *hg_last_error(const hg_ctx *ctx) {
    if (!ctx) return g_create_error.c_str();
    return ctx->err.c_str();
}

// Every entry point first makes the context's GPU current on the calling host thread, so
// that contexts can be driven from several threads (one per context).
#define HG_GUARD(ctx, body)                                  \
    do {                                                     \
        if (!(ctx)) return -1;                               \
        try {                                                \
            BudgetScope bs_(&(ctx)->budget);                 \
            HG_CK(cudaSetDevice((ctx)->cfg.device));         \
            body;                                            \
            (ctx)->err.clear();                              \
            return 0;                                        \
        } catch (const HgError &e) {                         \
            (ctx)->err = with_budget_note((ctx), e.msg);     \
            return -1;                                       \
        } catch (const std::exception &e) {                  \
            (ctx)->err = with_budget_note((ctx), e.what());  \
            return -1;                                       \
        }                                                    \
    } while (0)

int hg_set_particles(hg_ctx *ctx, int slot, const double *base, long long n, long long stride_bytes, int pos_off,
                     int los_off, int w_off) {
    HG_GUARD(ctx, ctx->set_particles(slot, base, n, stride_bytes, pos_off, los_off, w_off, false));
}

int hg_set_particles_device(hg_ctx *ctx, int slot, const double *dev_base, long long n, long long stride_bytes,
                            int pos_off, int los_off, int w_off) {
    HG_GUARD(ctx, ctx->set_particles(slot, dev_base, n, stride_bytes, pos_off, los_off, w_off, true));
}

int hg_set_memory_limit(hg_ctx *ctx, long long bytes) {
    if (!ctx) return -1;
    if (bytes < 0) {
        ctx->err = "the memory limit must be >= 0 bytes (0: none)";
        return -1;
    }
    ctx->budget.limit = (size_t)bytes;
    ctx->err.clear();
    return 0;
}

long long hg_memory_in_use(const hg_ctx *ctx) { return ctx ? (long long)ctx->budget.used : -1; }

int hg_batch_done(const hg_ctx *ctx) { return ctx ? ctx->batch_done : -1; }

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

int hg_tuning(hg_ctx *ctx, char *buf, long long buflen) {
    if (!ctx || !buf || buflen <= 0) return -1;
    std::string s;
    try {
        s = ctx->tuning();
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
    HG_GUARD(ctx, ctx->bk_box_multi({MP{ell1, ell2, ELL}}, ith_kbin, bk_save, sn_save, norm));
}

int hg_bk_box_multi(hg_ctx *ctx, int n_multipoles, const int *ells, int ith_kbin, double *bk_save, double *sn_save,
                    double *norm) {
    if (!bk_save || !sn_save || !ells || n_multipoles <= 0) return -1;
    std::vector<MP> mps;
    for (int q = 0; q < n_multipoles; q++) mps.push_back(MP{ells[3 * q], ells[3 * q + 1], ells[3 * q + 2]});
    HG_GUARD(ctx, ctx->bk_box_multi(mps, ith_kbin, bk_save, sn_save, norm));
}

int hg_zeta_box(hg_ctx *ctx, int ell1, int ell2, int ELL, int ith_rbin, double *zeta_save, double *sn_save,
                double *norm) {
    if (!zeta_save || !sn_save) return -1;
    HG_GUARD(ctx, ctx->zeta_box_multi({MP{ell1, ell2, ELL}}, ith_rbin, zeta_save, sn_save, norm));
}

int hg_zeta_box_multi(hg_ctx *ctx, int n_multipoles, const int *ells, int ith_rbin, double *zeta_save,
                      double *sn_save, double *norm) {
    if (!zeta_save || !sn_save || !ells || n_multipoles <= 0) return -1;
    std::vector<MP> mps;
    for (int q = 0; q < n_multipoles; q++) mps.push_back(MP{ells[3 * q], ells[3 * q + 1], ells[3 * q + 2]});
    HG_GUARD(ctx, ctx->zeta_box_multi(mps, ith_rbin, zeta_save, sn_save, norm));
}

int hg_bk_survey(hg_ctx *ctx, int ell1, int ell2, int ELL, int ith_kbin, double alpha, double vsurvey,
                 double *bk_save, double *sn_save, double *norm) {
    if (!bk_save || !sn_save) return -1;
    HG_GUARD(ctx, ctx->bk_survey_multi({MP{ell1, ell2, ELL}}, ith_kbin, alpha, vsurvey, bk_save, sn_save, norm));
}

int hg_bk_survey_multi(hg_ctx *ctx, int n_multipoles, const int *ells, int ith_kbin, double alpha, double vsurvey,
                       double *bk_save, double *sn_save, double *norm) {
    if (!bk_save || !sn_save || !ells || n_multipoles <= 0) return -1;
    std::vector<MP> mps;
    for (int q = 0; q < n_multipoles; q++) mps.push_back(MP{ells[3 * q], ells[3 * q + 1], ells[3 * q + 2]});
    HG_GUARD(ctx, ctx->bk_survey_multi(mps, ith_kbin, alpha, vsurvey, bk_save, sn_save, norm));
}

int hg_zeta_survey(hg_ctx *ctx, int ell1, int ell2, int ELL, int ith_rbin, double alpha, double vsurvey,
                   double *zeta_save, double *sn_save, double *norm) {
    if (!zeta_save || !sn_save) return -1;
    HG_GUARD(ctx, ctx->zeta_survey_multi({MP{ell1, ell2, ELL}}, ith_rbin, alpha, vsurvey, zeta_save, sn_save, norm));
}

int hg_zeta_survey_multi(hg_ctx *ctx, int n_multipoles, const int *ells, int ith_rbin, double alpha, double vsurvey,
                         double *zeta_save, double *sn_save, double *norm) {
    if (!zeta_save || !sn_save || !ells || n_multipoles <= 0) return -1;
    std::vector<MP> mps;
    for (int q = 0; q < n_multipoles; q++) mps.push_back(MP{ells[3 * q], ells[3 * q + 1], ells[3 * q + 2]});
    HG_GUARD(ctx, ctx->zeta_survey_multi(mps, ith_rbin, alpha, vsurvey, zeta_save, sn_save, norm));
}

int hg_survey_scalars(hg_ctx *ctx, double *alpha, double *vsurvey, double *nbar, double *wsum_data,
                      double *wsum_rand) {
    HG_GUARD(ctx, ctx->survey_scalars(alpha, vsurvey, nbar, wsum_data, wsum_rand));
}

int hg_pk_survey(hg_ctx *ctx, int ell, double alpha, double vsurvey, double *pk_save, int *n_mode, double *norm) {
    if (!pk_save) return -1;
    HG_GUARD(ctx, ctx->pk_survey(ell, alpha, vsurvey, pk_save, n_mode, norm));
}

int hg_xi_box(hg_ctx *ctx, int ell, double *xi_save, int *n_mode, double *norm) {
    if (!xi_save) return -1;
    HG_GUARD(ctx, ctx->xi_box(ell, xi_save, n_mode, norm));
}

int hg_xi_survey(hg_ctx *ctx, int ell, double alpha, double vsurvey, double *xi_save, int *n_mode, double *norm) {
    if (!xi_save) return -1;
    HG_GUARD(ctx, ctx->xi_survey(ell, false, alpha, vsurvey, xi_save, n_mode, norm));
}

int hg_xi_window(hg_ctx *ctx, int ell, double vsurvey, double *xi_save, int *n_mode, double *norm) {
    if (!xi_save) return -1;
    HG_GUARD(ctx, ctx->xi_survey(ell, true, 0.0, vsurvey, xi_save, n_mode, norm));
}

int hg_zeta_window(hg_ctx *ctx, int ell1, int ell2, int ELL, int ith_rbin, double vsurvey, double *zeta_save,
                   double *sn_save, double *norm) {
    if (!zeta_save || !sn_save) return -1;
    HG_GUARD(ctx, ctx->zeta_window_multi({MP{ell1, ell2, ELL}}, ith_rbin, vsurvey, zeta_save, sn_save, norm));
}

int hg_zeta_window_multi(hg_ctx *ctx, int n_multipoles, const int *ells, int ith_rbin, double vsurvey,
                         double *zeta_save, double *sn_save, double *norm) {
    if (!zeta_save || !sn_save || !ells || n_multipoles <= 0) return -1;
    std::vector<MP> mps;
    for (int q = 0; q < n_multipoles; q++) mps.push_back(MP{ells[3 * q], ells[3 * q + 1], ells[3 * q + 2]});
    HG_GUARD(ctx, ctx->zeta_window_multi(mps, ith_rbin, vsurvey, zeta_save, sn_save, norm));
}

int hg_reconstruct(hg_ctx *ctx, int box, double b1_fid, double RG, double alpha, double vsurvey, double *pos_D,
                   double *pos_R) {
    HG_GUARD(ctx, ctx->reconstruct(box, b1_fid, RG, alpha, vsurvey, pos_D, pos_R));
}

int hg_pk_box_recon(hg_ctx *ctx, int ell, double alpha, double *pk_save, int *n_mode, double *norm) {
    if (!pk_save) return -1;
    HG_GUARD(ctx, ctx->pk_box_recon(ell, alpha, pk_save, n_mode, norm));
}

int hg_xi_box_recon(hg_ctx *ctx, int ell, double alpha, double *xi_save, int *n_mode, double *norm) {
    if (!xi_save) return -1;
    HG_GUARD(ctx, ctx->xi_box_recon(ell, alpha, xi_save, n_mode, norm));
}

int hg_bk_box_recon_multi(hg_ctx *ctx, int n_multipoles, const int *ells, int ith_kbin, double alpha,
                          double *bk_save, double *sn_save, double *norm) {
    if (!bk_save || !sn_save || !ells || n_multipoles <= 0) return -1;
    std::vector<MP> mps;
    for (int q = 0; q < n_multipoles; q++) mps.push_back(MP{ells[3 * q], ells[3 * q + 1], ells[3 * q + 2]});
    HG_GUARD(ctx, ctx->bk_box_recon_multi(mps, ith_kbin, alpha, bk_save, sn_save, norm));
}

int hg_zeta_box_recon_multi(hg_ctx *ctx, int n_multipoles, const int *ells, int ith_rbin, double alpha,
                            double *zeta_save, double *sn_save, double *norm) {
    if (!zeta_save || !sn_save || !ells || n_multipoles <= 0) return -1;
    std::vector<MP> mps;
    for (int q = 0; q < n_multipoles; q++) mps.push_back(MP{ells[3 * q], ells[3 * q + 1], ells[3 * q + 2]});
    HG_GUARD(ctx, ctx->zeta_box_recon_multi(mps, ith_rbin, alpha, zeta_save, sn_save, norm));
}

long long hg_batch_block_len(const hg_ctx *ctx, int n_pk, int n_bk, int n_zeta) {
    if (!ctx || n_pk < 0 || n_bk < 0 || n_zeta < 0) return -1;
    return hg::batch_block_len(ctx->cfg, n_pk, n_bk, n_zeta);
}

int hg_batch_run(hg_ctx *ctx, const hg_mock *mocks, int n_mocks, int n_pk, const int *pk_ells, int n_bk,
                 const int *bk_ells, int n_zeta, const int *zeta_ells, double *out) {
    if (!mocks || n_mocks <= 0 || !out || n_pk < 0 || n_bk < 0 || n_zeta < 0) return -1;
    if ((n_pk && !pk_ells) || (n_bk && !bk_ells) || (n_zeta && !zeta_ells)) return -1;
    std::vector<int> pk(pk_ells, pk_ells + n_pk);
    std::vector<MP> bk, zeta;
    for (int q = 0; q < n_bk; q++) bk.push_back(MP{bk_ells[3 * q], bk_ells[3 * q + 1], bk_ells[3 * q + 2]});
    for (int q = 0; q < n_zeta; q++) zeta.push_back(MP{zeta_ells[3 * q], zeta_ells[3 * q + 1], zeta_ells[3 * q + 2]});
    HG_GUARD(ctx, ctx->batch_run(mocks, n_mocks, pk, bk, zeta, out));
}

int hg_last_timing(const hg_ctx *ctx, double *device_ms, long long *kernel_launches) {
    if (!ctx) return -1;
    if (device_ms) *device_ms = ctx->last_ms;
    if (kernel_launches) *kernel_launches = ctx->last_launches;
    return 0;
}

}  // extern "C"
