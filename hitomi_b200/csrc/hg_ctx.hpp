// hg_ctx.hpp -- the context interface shared by the engine translation units
// (hg_engine_fp32.cu, hg_engine_fp64.cu: one Engine<T> each) and the C ABI (hg_api.cu).
//
// A context is one Engine<T>.  The FP32 form may delegate chosen stages of the periodic-box
// pipeline to an FP64 engine of the same context (hg_config.fp64_stages); the stage_*
// methods are the boundary between the two: the density half spectrum crosses it (converted
// to the receiving engine's precision), and the bispectrum's signal and shot-noise halves
// come back as host FP64 matrices.
#pragma once

#include "hitomi_gpu.h"

#include <mutex>
#include <string>
#include <vector>

namespace hg {

// doubles per mock of hg_batch_run's output
inline long long batch_block_len(const hg_config &c, int n_pk, int n_bk, int n_zeta) {
    long long n = 2LL * n_pk * c.n_kbin + n_pk;
    if (n_bk > 0) n += 4LL * n_bk * c.n_kbin * c.n_kbin + 1;
    if (n_zeta > 0) n += 4LL * n_zeta * c.n_rbin * c.n_rbin + 1;
    return n;
}

struct MP {
    int l1, l2, L;
};

struct HgError {
    std::string msg;
};

// Device memory held by one context's buffers, and the limit set by hg_set_memory_limit
// (0: none).  Every engine allocation made during an API call is charged to the calling
// context (current_budget), and returned to it when the buffer is freed; an allocation that
// would pass the limit fails as cudaMalloc's out-of-memory does, with `hit` set.
struct MemBudget {
    size_t limit = 0;
    size_t used = 0;
    bool hit = false;
    std::mutex m;  // a context's two engines may allocate from two host threads at once
};
// the budget of the API call running on this thread (null outside API calls)
MemBudget *&current_budget();

}  // namespace hg

struct hg_ctx {
    hg_config cfg;
    std::string err;
    hg::MemBudget budget;
    double last_ms = 0.0;
    long long last_launches = 0;
    int batch_done = 0;  // mocks completed by the last batch_run
    virtual ~hg_ctx() {}
    virtual void set_particles(int slot, const double *base, long long n, long long stride, int pos_off, int los_off,
                               int w_off, bool on_device) = 0;
    virtual void set_profiling(bool on) = 0;
    virtual std::string kernel_stats() = 0;
    virtual std::string tuning() = 0;
    virtual void pk_box(int ell, double *pk_save, int *n_mode, double *norm) = 0;
    virtual void bk_box_multi(const std::vector<hg::MP> &mps, int ith, double *bk_save, double *sn_save,
                              double *norm) = 0;
    virtual void zeta_box_multi(const std::vector<hg::MP> &mps, int ith, double *zeta_save, double *sn_save,
                                double *norm) = 0;
    virtual void survey_scalars(double *alpha, double *vs, double *nbar, double *wd, double *wr) = 0;
    virtual void pk_survey(int ell, double alpha, double vs, double *pk_save, int *n_mode, double *norm) = 0;
    virtual void bk_survey_multi(const std::vector<hg::MP> &mps, int ith, double alpha, double vs, double *bk_save,
                                 double *sn_save, double *norm) = 0;
    virtual void zeta_survey_multi(const std::vector<hg::MP> &mps, int ith, double alpha, double vs,
                                   double *zeta_save, double *sn_save, double *norm) = 0;
    virtual void zeta_window_multi(const std::vector<hg::MP> &mps, int ith, double vs, double *zeta_save,
                                   double *sn_save, double *norm) = 0;
    virtual void xi_box(int ell, double *xi_save, int *n_mode, double *norm) = 0;
    virtual void reconstruct(int box, double b1, double RG, double alpha, double vs, double *posD, double *posR) = 0;
    virtual void pk_box_recon(int ell, double alpha, double *pk_save, int *n_mode, double *norm) = 0;
    virtual void xi_box_recon(int ell, double alpha, double *xi_save, int *n_mode, double *norm) = 0;
    virtual void bk_box_recon_multi(const std::vector<hg::MP> &mps, int ith, double alpha, double *bk_save,
                                    double *sn_save, double *norm) = 0;
    virtual void zeta_box_recon_multi(const std::vector<hg::MP> &mps, int ith, double alpha, double *zeta_save,
                                      double *sn_save, double *norm) = 0;
    virtual void batch_run(const hg_mock *mocks, int n_mocks, const std::vector<int> &pk_ells,
                           const std::vector<hg::MP> &bk, const std::vector<hg::MP> &zeta, double *out) = 0;
    virtual void xi_survey(int ell, bool window, double alpha, double vs, double *xi_save, int *n_mode,
                           double *norm) = 0;

    // ---- stages (periodic box), called by the other-precision engine of the same context
    // run every kernel on the caller's stream from now on (the callee's own is released)
    virtual void stage_adopt_stream(void *stream) = 0;
    // the box density half spectrum [n0][n1][n2/2+1] (this engine's precision) and its FP64
    // k = 0 value, particle integral and in-bounds mass; computed if not current
    virtual const void *stage_density(double *delta0, double *N0, double *mass) = 0;
    virtual bool stage_density_ready() const = 0;
    // take a density half spectrum computed by the other engine (fp64: its elements are
    // double pairs, else float pairs) as this engine's current box density
    virtual void stage_import_density(const void *H, bool src_fp64, double delta0, double N0, double mass) = 0;
    // B_raw and the shot noise of the box bispectrum, [q][ns][ns] complex (all rows)
    virtual std::vector<std::vector<double>> stage_bk_signal(const std::vector<hg::MP> &mps) = 0;
    virtual std::vector<std::vector<double>> stage_bk_shot(const std::vector<hg::MP> &mps) = 0;
    // bin averages [nbin][ells.size()] complex of the box density's (|delta|^2 - N C) / W^2
    // Yhat_l0 (the P_l bins before the 2l + 1 factor), from the P cache where those
    // multipoles were binned already
    virtual std::vector<double> stage_pk_terms(const std::vector<int> &ells) = 0;
    // kernels launched since the last call (added to the calling engine's count)
    virtual long long stage_take_launches() = 0;
};

namespace hg {
hg_ctx *make_engine_fp64(const hg_config &c);
hg_ctx *make_engine_fp32(const hg_config &c);
// Error text returned by hg_last_error(NULL) for entry points that have no context.
void set_contextless_error(const std::string &m);
const std::string &contextless_error();
}  // namespace hg
