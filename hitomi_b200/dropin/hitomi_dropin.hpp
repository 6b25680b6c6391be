// hitomi_dropin.hpp -- the reference's estimator entry points with bodies that delegate to
// the B200 library (include/hitomi_gpu.h, libhitomi_b200.so).
//
// A program built on hitomi_measurement includes this header in place of powerspec.hpp and
// bispec.hpp, after the headers that define ParameterClass, ParticleGadgetClass,
// ParticleBOSSClass and ToolClass (parameter.hpp, particleGadget.hpp, particle.hpp,
// tools.hpp), and links -lhitomi_b200.  Each function keeps the reference's signature,
// return convention (0, or -1 after printing the reason) and output file: name, header line
// and fprintf format are those of src/hitomi_measurement/powerspec.hpp and bispec.hpp, and
// the printed numbers are the same products norm * sums.
//
//   calcPowerSpectrumForBOX                  powerspec.hpp:273-332
//   calcTwoPointCorrelationFunctionForBOX    powerspec.hpp:334-393
//   calcBiSpectrumForBOX                     bispec.hpp:877-1203
//   calcThreePointCorrelationFunctionForBOX  bispec.hpp:1205-1424
//   calcPowerSpectrum                        powerspec.hpp:4-91
//   calcTwoPointCorrelationFunction          powerspec.hpp:93-180
//   calcTwoPointWindowCorrelationFunction    powerspec.hpp:182-270
//   calcBiSpectrum                           bispec.hpp:4-352
//   calcThreePointCorrelationFunction        bispec.hpp:355-614
//   calcThreePointWindowCorrelationFunction  bispec.hpp:617-874
//   calcPowerSpectrumForBOXForReconstruction      powerspec.hpp:396-457
//   calcTwoPointFunctionForBOXForReconstruction   powerspec.hpp:459-520
//   calcBiSpectrumForBOXForReconstruction         bispec.hpp:1426-1753
//   calcThreePointCorrelationFunctionForBOXForReconstruction  bispec.hpp:1755-1990
//   calcReconstructionParticles                   particle_reconstruction.hpp:12-208
//   calcReconstructionParticlesForBOX             particle_reconstruction.hpp:210-402
// (the last two in place of particle_reconstruction.hpp, which the program then does not
// include either)
//
// Optional parameter-file keys (hitomi_dropin_configure, one added call after
// ParameterClass::readParameters); absent keys keep the reference's behaviour:
//   gpu_precision   = fp64 (default; matches the reference to 1e-10) | fp32 | chosen
//                     (chosen: FP32 with the density and bispectrum signal in FP64)
//   gpu_interlacing = False (default) | True
//   gpu_scheme      = PCS  (overrides `assignment`, whose check, parameter.hpp:504-510,
//                     admits only NGP / CIC / TSC)
// (The reference's parser matches keys as substrings of the line, parameter.hpp:161-207,
// so no key here contains one of its own key names.)
//   gpu_device      = 0 (CUDA device ordinal)
#ifndef HITOMI_DROPIN_HPP
#define HITOMI_DROPIN_HPP

#include "hitomi_gpu.h"

#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace hitomi_dropin {

struct Options {
    int precision = HG_FP64;
    int fp64_stages = 0;
    int interlace = 0;
    int pcs = 0;
    int device = 0;
};

inline Options &options() {
    static Options o;
    return o;
}

// One context per process, rebuilt when the geometry, bins or scheme change (the reference
// drivers call one estimator per run; a batch program may call several).
struct Cached {
    hg_ctx *ctx = nullptr;
    hg_config cfg;
    ~Cached() {
        if (ctx) hg_destroy(ctx);
    }
};

// recon: the reconstruction mesh n_mesh_recon (its own context, cached separately)
inline hg_ctx *context(ParameterClass &param, bool recon = false) {
    static Cached cache, cache_recon;
    Cached &cc = recon ? cache_recon : cache;
    const Options &o = options();
    hg_config c;
    std::memset(&c, 0, sizeof(c));
    for (int a = 0; a < 3; a++) {
        c.n_mesh[a] = recon ? param.n_mesh_recon[a] : param.n_mesh[a];
        c.boxsize[a] = param.boxsize[a];
    }
    c.assign = o.pcs ? HG_PCS : param.assign == "NGP" ? HG_NGP : param.assign == "CIC" ? HG_CIC : HG_TSC;
    c.interlace = o.interlace;
    c.precision = o.precision;
    c.fp64_stages = o.fp64_stages;
    c.kmin = param.kmin;
    c.kmax = param.kmax;
    c.n_kbin = param.n_kbin;
    c.rmin = param.rmin;
    c.rmax = param.rmax;
    c.n_rbin = param.n_rbin;
    c.periodic = 0;
    c.device = o.device;
    if (cc.ctx && std::memcmp(&cc.cfg, &c, sizeof(c)) == 0) return cc.ctx;
    if (cc.ctx) hg_destroy(cc.ctx);
    cc.ctx = nullptr;
    if (hg_create(&cc.ctx, &c)) {
        printf("hg_create fails: %s\n", hg_last_error(nullptr));
        cc.ctx = nullptr;
        return nullptr;
    }
    cc.cfg = c;
    return cc.ctx;
}

inline int fail(hg_ctx *ctx, const char *what) {
    printf("'%s' fails: %s\n", what, hg_last_error(ctx));
    return -1;
}

// {pos[3], vel[3]} records read in place (particleGadget.hpp:12-15)
inline int set_box(hg_ctx *ctx, ParticleGadgetClass &P) {
    if (hg_set_particles(ctx, 0, &P[0].pos[0], P.n_tot, (long long)sizeof(P[0]), 0, -1, -1))
        return fail(ctx, "hg_set_particles");
    return 0;
}

// the same, randoms in slot 1 (the box with reconstruction)
inline int set_box_randoms(hg_ctx *ctx, ParticleGadgetClass &P) {
    if (hg_set_particles(ctx, 1, &P[0].pos[0], P.n_tot, (long long)sizeof(P[0]), 0, -1, -1))
        return fail(ctx, "hg_set_particles");
    return 0;
}

// {pos[3], los[3], w} records read in place (particle.hpp:12-16); slot 0 data, 1 randoms
inline int set_survey(hg_ctx *ctx, int slot, ParticleBOSSClass &P) {
    if (hg_set_particles(ctx, slot, &P[0].pos[0], P.n_tot, (long long)sizeof(P[0]), 0, 3, 6))
        return fail(ctx, "hg_set_particles");
    return 0;
}

inline bool ell_check(ParameterClass &param) {  // powerspec.hpp:12-16
    if (!((param.ELL == param.ell1) && (param.ell2 == 0))) {
        printf("This multipole combination is not allowed.\n");
        printf("It should be ELL == ell1 and ell2 == 0\n");
        return false;
    }
    return true;
}

inline bool triple_check(ParameterClass &param) {  // bispec.hpp:884-890
    if (std::fabs(wigner_3j(param.ell1, param.ell2, param.ELL, 0, 0, 0)) < 1.0e-10) {
        printf("This multipole combination is not allowed.\n");
        printf("It should be wigner_3j(ell1, ell2, ELL, 0,0,0) != 0\n");
        return false;
    }
    return true;
}

// "" or "_recon" by flag_recon, as the survey writers choose their file names
inline const char *recon_tag(ParameterClass &param) { return param.flag_recon == "True" ? "_recon" : ""; }

inline int write_pk(ParameterClass &param, const char *tag, double *kbin, const std::vector<std::complex<double>> &pk,
                    double norm) {
    char buf[1024];
    sprintf(buf, "%s/pk%d%s.dat", param.output_dir.c_str(), param.ELL, tag);
    FILE *fp = fopen(buf, "w");
    if (!fp) return -1;
    fprintf(fp, "## k [h/Mpc]\t pk_real [(Mpc/h)^3]\t pk_imag [(Mpc/h)^3]\n");
    for (int i = 0; i < param.n_kbin; i++)
        fprintf(fp, "%.5f \t %.7e \t %.7e\n", kbin[i], norm * pk[i].real(), norm * pk[i].imag());
    fclose(fp);
    return 0;
}

inline int write_xi(ParameterClass &param, const char *tag, double *rbin, const std::vector<std::complex<double>> &xi,
                    double norm) {
    char buf[1024];
    sprintf(buf, "%s/xi%d%s.dat", param.output_dir.c_str(), param.ELL, tag);
    FILE *fp = fopen(buf, "w");
    if (!fp) return -1;
    fprintf(fp, "## r [Mpc/h] \t xi\n");
    for (int i = 0; i < param.n_rbin; i++) fprintf(fp, "%.5f \t %.7e\n", rbin[i], norm * xi[i].real());
    fclose(fp);
    return 0;
}

inline int write_bk(ParameterClass &param, const char *tag, double *kbin, const std::vector<std::complex<double>> &bk,
                    const std::vector<std::complex<double>> &sn, double norm) {
    char buf[1024];
    sprintf(buf, "%s/bk%d%d%d_%02d%s.dat", param.output_dir.c_str(), param.ell1, param.ell2, param.ELL, param.ith_kbin,
            tag);
    FILE *fp = fopen(buf, "w");
    if (!fp) return -1;
    fprintf(fp, "## k1 [h/Mpc] \t k2 [h/Mpc] \t bk_real \t bk_imag\n");
    for (int i = 0; i < param.n_kbin; i++)
        fprintf(fp, "%.5f \t %.5f \t %.7e \t %.7e\n", kbin[param.ith_kbin], kbin[i],
                norm * (bk[i].real() - sn[i].real()), norm * (bk[i].imag() - sn[i].imag()));
    fclose(fp);
    return 0;
}

inline int write_zeta(ParameterClass &param, const char *tag, double *rbin,
                      const std::vector<std::complex<double>> &zeta, const std::vector<std::complex<double>> &sn,
                      double norm) {
    char buf[1024];
    sprintf(buf, "%s/zeta%d%d%d_%02d%s.dat", param.output_dir.c_str(), param.ell1, param.ell2, param.ELL,
            param.ith_rbin, tag);
    FILE *fp = fopen(buf, "w");
    if (!fp) return -1;
    fprintf(fp, "## r1 [Mpc/h] \t r2 [Mpc/h] \t zeta \n");
    for (int i = 0; i < param.n_rbin; i++)
        fprintf(fp, "%.5f \t %.5f \t %.7e\n", rbin[param.ith_rbin], rbin[i],
                norm * (zeta[i].real() - sn[i].real()));
    fclose(fp);
    return 0;
}

inline double *dp(std::vector<std::complex<double>> &v) { return reinterpret_cast<double *>(v.data()); }

}  // namespace hitomi_dropin

// Reads the optional gpu_* keys (see above) from the parameter file; 0 on success.
inline int hitomi_dropin_configure(const char *param_file) {
    FILE *fp = fopen(param_file, "r");
    if (!fp) return -1;
    hitomi_dropin::Options &o = hitomi_dropin::options();
    char line[1024];
    while (fgets(line, sizeof(line), fp)) {
        char key[256] = {0}, eq[8] = {0}, val[256] = {0};
        if (sscanf(line, "%255s %7s %255s", key, eq, val) != 3 || strcmp(eq, "=") != 0) continue;
        const std::string k(key), v(val);
        if (k == "gpu_precision") {
            if (v == "fp64") {
                o.precision = HG_FP64;
                o.fp64_stages = 0;
            } else if (v == "fp32") {
                o.precision = HG_FP32;
                o.fp64_stages = 0;
            } else if (v == "chosen") {
                o.precision = HG_FP32;
                o.fp64_stages = HG_STAGE_DENSITY | HG_STAGE_BK_SIGNAL;
            } else {
                printf("gpu_precision must be fp64, fp32 or chosen\n");
                fclose(fp);
                return -1;
            }
        } else if (k == "gpu_interlacing") {
            o.interlace = (v == "True") ? 1 : 0;
        } else if (k == "gpu_scheme") {
            o.pcs = (v == "PCS") ? 1 : 0;
        } else if (k == "gpu_device") {
            o.device = atoi(val);
        }
    }
    fclose(fp);
    return 0;
}

// ---------------------------------------------------------------------------- periodic box

inline int calcPowerSpectrumForBOX(ParticleGadgetClass &P_D, ParameterClass &param, double *kbin) {
    using namespace hitomi_dropin;
    if (!ell_check(param)) return -1;
    hg_ctx *ctx = context(param);
    if (!ctx || set_box(ctx, P_D)) return -1;
    std::vector<std::complex<double>> pk(param.n_kbin);
    double norm;
    if (hg_pk_box(ctx, param.ELL, dp(pk), nullptr, &norm)) return fail(ctx, "hg_pk_box");
    return write_pk(param, "", kbin, pk, norm);
}

inline int calcTwoPointCorrelationFunctionForBOX(ParticleGadgetClass &P_D, ParameterClass &param, double *rbin) {
    using namespace hitomi_dropin;
    if (!ell_check(param)) return -1;
    hg_ctx *ctx = context(param);
    if (!ctx || set_box(ctx, P_D)) return -1;
    std::vector<std::complex<double>> xi(param.n_rbin);
    double norm;
    if (hg_xi_box(ctx, param.ELL, dp(xi), nullptr, &norm)) return fail(ctx, "hg_xi_box");
    return write_xi(param, "", rbin, xi, norm);
}

inline int calcBiSpectrumForBOX(ParticleGadgetClass &P_D, ParameterClass &param, double *kbin) {
    using namespace hitomi_dropin;
    if (!triple_check(param)) return -1;
    hg_ctx *ctx = context(param);
    if (!ctx || set_box(ctx, P_D)) return -1;
    std::vector<std::complex<double>> bk(param.n_kbin), sn(param.n_kbin);
    double norm;
    if (hg_bk_box(ctx, param.ell1, param.ell2, param.ELL, param.ith_kbin, dp(bk), dp(sn), &norm))
        return fail(ctx, "hg_bk_box");
    return write_bk(param, "", kbin, bk, sn, norm);
}

inline int calcThreePointCorrelationFunctionForBOX(ParticleGadgetClass &P_D, ParameterClass &param, double *rbin) {
    using namespace hitomi_dropin;
    if (!triple_check(param)) return -1;
    hg_ctx *ctx = context(param);
    if (!ctx || set_box(ctx, P_D)) return -1;
    std::vector<std::complex<double>> z(param.n_rbin), sn(param.n_rbin);
    double norm;
    if (hg_zeta_box(ctx, param.ell1, param.ell2, param.ELL, param.ith_rbin, dp(z), dp(sn), &norm))
        return fail(ctx, "hg_zeta_box");
    return write_zeta(param, "", rbin, z, sn, norm);
}

// ---------------------------------------------------------------------------- survey geometry
// The caller has prepared both catalogues as main.cpp:129-200 does (calcLOS,
// resetParticleForFFT, alpha, Vsurvey).

inline int calcPowerSpectrum(ParticleBOSSClass &P_D, ParticleBOSSClass &P_R, ParameterClass &param, double alpha,
                             double *kbin, double Vsurvey) {
    using namespace hitomi_dropin;
    if (!ell_check(param)) return -1;
    hg_ctx *ctx = context(param);
    if (!ctx || set_survey(ctx, 0, P_D) || set_survey(ctx, 1, P_R)) return -1;
    std::vector<std::complex<double>> pk(param.n_kbin);
    double norm;
    if (hg_pk_survey(ctx, param.ELL, alpha, Vsurvey, dp(pk), nullptr, &norm)) return fail(ctx, "hg_pk_survey");
    return write_pk(param, recon_tag(param), kbin, pk, norm);
}

inline int calcTwoPointCorrelationFunction(ParticleBOSSClass &P_D, ParticleBOSSClass &P_R, ParameterClass &param,
                                           double alpha, double *rbin, double Vsurvey) {
    using namespace hitomi_dropin;
    if (!ell_check(param)) return -1;
    hg_ctx *ctx = context(param);
    if (!ctx || set_survey(ctx, 0, P_D) || set_survey(ctx, 1, P_R)) return -1;
    std::vector<std::complex<double>> xi(param.n_rbin);
    double norm;
    if (hg_xi_survey(ctx, param.ELL, alpha, Vsurvey, dp(xi), nullptr, &norm)) return fail(ctx, "hg_xi_survey");
    return write_xi(param, recon_tag(param), rbin, xi, norm);
}

inline int calcTwoPointWindowCorrelationFunction(ParticleBOSSClass &P_R, ParameterClass &param, double *rbin,
                                                 double Vsurvey) {
    using namespace hitomi_dropin;
    if (!ell_check(param)) return -1;
    hg_ctx *ctx = context(param);
    if (!ctx || set_survey(ctx, 1, P_R)) return -1;
    std::vector<std::complex<double>> xi(param.n_rbin);
    double norm;
    if (hg_xi_window(ctx, param.ELL, Vsurvey, dp(xi), nullptr, &norm)) return fail(ctx, "hg_xi_window");
    const std::string tag = std::string(recon_tag(param)) + "_window";
    return write_xi(param, tag.c_str(), rbin, xi, norm);
}

inline int calcBiSpectrum(ParticleBOSSClass &P_D, ParticleBOSSClass &P_R, ParameterClass &param, double alpha,
                          double *kbin, double Vsurvey) {
    using namespace hitomi_dropin;
    if (!triple_check(param)) return -1;
    hg_ctx *ctx = context(param);
    if (!ctx || set_survey(ctx, 0, P_D) || set_survey(ctx, 1, P_R)) return -1;
    std::vector<std::complex<double>> bk(param.n_kbin), sn(param.n_kbin);
    double norm;
    if (hg_bk_survey(ctx, param.ell1, param.ell2, param.ELL, param.ith_kbin, alpha, Vsurvey, dp(bk), dp(sn), &norm))
        return fail(ctx, "hg_bk_survey");
    return write_bk(param, recon_tag(param), kbin, bk, sn, norm);
}

inline int calcThreePointCorrelationFunction(ParticleBOSSClass &P_D, ParticleBOSSClass &P_R, ParameterClass &param,
                                             double alpha, double *rbin, double Vsurvey) {
    using namespace hitomi_dropin;
    if (!triple_check(param)) return -1;
    hg_ctx *ctx = context(param);
    if (!ctx || set_survey(ctx, 0, P_D) || set_survey(ctx, 1, P_R)) return -1;
    std::vector<std::complex<double>> z(param.n_rbin), sn(param.n_rbin);
    double norm;
    if (hg_zeta_survey(ctx, param.ell1, param.ell2, param.ELL, param.ith_rbin, alpha, Vsurvey, dp(z), dp(sn), &norm))
        return fail(ctx, "hg_zeta_survey");
    return write_zeta(param, recon_tag(param), rbin, z, sn, norm);
}

inline int calcThreePointWindowCorrelationFunction(ParticleBOSSClass &P_R, ParameterClass &param, double *rbin,
                                                   double Vsurvey) {
    using namespace hitomi_dropin;
    if (!triple_check(param)) return -1;
    hg_ctx *ctx = context(param);
    if (!ctx || set_survey(ctx, 1, P_R)) return -1;
    std::vector<std::complex<double>> z(param.n_rbin), sn(param.n_rbin);
    double norm;
    if (hg_zeta_window(ctx, param.ell1, param.ell2, param.ELL, param.ith_rbin, Vsurvey, dp(z), dp(sn), &norm))
        return fail(ctx, "hg_zeta_window");
    const std::string tag = std::string(recon_tag(param)) + "_window";
    return write_zeta(param, tag.c_str(), rbin, z, sn, norm);
}

// ---------------------------------------------------------------------------- reconstruction

namespace hitomi_dropin {
// the shifted positions written back into the caller's particles, as the reference moves them
template <class P>
inline void write_back(P &part, const std::vector<double> &pos) {
    for (long long i = 0; i < part.n_tot; i++)
        for (int a = 0; a < 3; a++) part[i].pos[a] = pos[3 * i + a];
}
}  // namespace hitomi_dropin

inline int calcReconstructionParticles(ParticleBOSSClass &P_D, ParticleBOSSClass &P_R, ParameterClass &param,
                                       double alpha, double Vsurvey) {
    using namespace hitomi_dropin;
    hg_ctx *ctx = context(param, true);
    if (!ctx || set_survey(ctx, 0, P_D) || set_survey(ctx, 1, P_R)) return -1;
    std::vector<double> pd(3 * P_D.n_tot), pr(3 * P_R.n_tot);
    if (hg_reconstruct(ctx, 0, param.b1_fid, param.RG, alpha, Vsurvey, pd.data(), pr.data()))
        return fail(ctx, "hg_reconstruct");
    write_back(P_D, pd);
    write_back(P_R, pr);
    return 0;
}

inline int calcReconstructionParticlesForBOX(ParticleGadgetClass &P_D, ParticleGadgetClass &P_R, ParameterClass &param) {
    using namespace hitomi_dropin;
    hg_ctx *ctx = context(param, true);
    if (!ctx || set_box(ctx, P_D) || set_box_randoms(ctx, P_R)) return -1;
    std::vector<double> pd(3 * P_D.n_tot), pr(3 * P_R.n_tot);
    if (hg_reconstruct(ctx, 1, param.b1_fid, param.RG, 0.0, param.volume, pd.data(), pr.data()))
        return fail(ctx, "hg_reconstruct");
    write_back(P_D, pd);
    write_back(P_R, pr);
    return 0;
}

inline int calcPowerSpectrumForBOXForReconstruction(ParticleGadgetClass &P_D, ParticleGadgetClass &P_R,
                                                    ParameterClass &param, double alpha, double *kbin) {
    using namespace hitomi_dropin;
    if (!ell_check(param)) return -1;
    hg_ctx *ctx = context(param);
    if (!ctx || set_box(ctx, P_D) || set_box_randoms(ctx, P_R)) return -1;
    std::vector<std::complex<double>> pk(param.n_kbin);
    double norm;
    if (hg_pk_box_recon(ctx, param.ELL, alpha, dp(pk), nullptr, &norm)) return fail(ctx, "hg_pk_box_recon");
    return write_pk(param, "_recon", kbin, pk, norm);
}

inline int calcTwoPointFunctionForBOXForReconstruction(ParticleGadgetClass &P_D, ParticleGadgetClass &P_R,
                                                       ParameterClass &param, double alpha, double *rbin) {
    using namespace hitomi_dropin;
    if (!ell_check(param)) return -1;
    hg_ctx *ctx = context(param);
    if (!ctx || set_box(ctx, P_D) || set_box_randoms(ctx, P_R)) return -1;
    std::vector<std::complex<double>> xi(param.n_rbin);
    double norm;
    if (hg_xi_box_recon(ctx, param.ELL, alpha, dp(xi), nullptr, &norm)) return fail(ctx, "hg_xi_box_recon");
    return write_xi(param, "_recon", rbin, xi, norm);
}

inline int calcBiSpectrumForBOXForReconstruction(ParticleGadgetClass &P_D, ParticleGadgetClass &P_R,
                                                 ParameterClass &param, double alpha, double *kbin) {
    using namespace hitomi_dropin;
    if (!triple_check(param)) return -1;
    hg_ctx *ctx = context(param);
    if (!ctx || set_box(ctx, P_D) || set_box_randoms(ctx, P_R)) return -1;
    std::vector<std::complex<double>> bk(param.n_kbin), sn(param.n_kbin);
    const int ells[3] = {param.ell1, param.ell2, param.ELL};
    double norm;
    if (hg_bk_box_recon_multi(ctx, 1, ells, param.ith_kbin, alpha, dp(bk), dp(sn), &norm))
        return fail(ctx, "hg_bk_box_recon_multi");
    return write_bk(param, "_recon", kbin, bk, sn, norm);
}

inline int calcThreePointCorrelationFunctionForBOXForReconstruction(ParticleGadgetClass &P_D, ParticleGadgetClass &P_R,
                                                                    ParameterClass &param, double alpha,
                                                                    double *rbin) {
    using namespace hitomi_dropin;
    if (!triple_check(param)) return -1;
    hg_ctx *ctx = context(param);
    if (!ctx || set_box(ctx, P_D) || set_box_randoms(ctx, P_R)) return -1;
    std::vector<std::complex<double>> z(param.n_rbin), sn(param.n_rbin);
    const int ells[3] = {param.ell1, param.ell2, param.ELL};
    double norm;
    if (hg_zeta_box_recon_multi(ctx, 1, ells, param.ith_rbin, alpha, dp(z), dp(sn), &norm))
        return fail(ctx, "hg_zeta_box_recon_multi");
    return write_zeta(param, "_recon", rbin, z, sn, norm);
}

#endif  // HITOMI_DROPIN_HPP
