/*
 * oracle/ref_harness.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * Builds the reference's own, unmodified estimator headers
 * (src/hitomi_measurement/{common,parameter,tools,bessel,particle,particleGadget,
 * particle_reconstruction,field,powerspec,bispec}.hpp) against the project-written
 * FFTW/GSL shims in oracle/shim/, and drives them the way the reference's CLI drivers
 * do (src/hitomi_measurement/main_box.cpp:50-230 for the periodic box,
 * src/hitomi_measurement/main.cpp:86-275 for the survey geometry).
 *
 * Only the particle source differs: instead of a Gadget snapshot or an ASCII
 * catalogue, positions (and weights) come from raw float64 files written by the
 * synthetic catalogue generators, so the oracle sees bit-identical inputs to the GPU.
 *
 * Usage:
 *   ref_harness param.ini data.f64 [random.f64] [--all-rows]
 *     box    : data.f64 holds n x 3 doubles (x y z)
 *     survey : data.f64 / random.f64 hold n x 4 doubles (x y z w)
 *   measure = pk | 2PCF | bk | 3PCF (box and survey), window2PCF | window3PCF (survey: the
 *   randoms only, main.cpp:252-270)
 *   --all-rows : for measure = bk / 3PCF, run every ith_kbin / ith_rbin row
 *                (the reference computes one row per process, main.cpp:78-84).
 *   --unit OP  : (box) time one building block of the reference's estimators once and
 *                print "HX_UNIT OP seconds"; OP in assign fft ifft corr bin_l0 bin_l2
 *                xi_ijk ylmk ylmx shell triple snloop spline.
 * Environment:
 *   HX_FULL=1    : result files are written with 17 significant digits instead of
 *                  the reference's %.7e / %.5f (format strings are rewritten at
 *                  fprintf time; the reference sources are untouched).
 *   HX_VERBOSE=1 : keep the reference's progress printf output (stderr).
 *   HX_TIMING=1  : print the wall time of the estimator call(s) to stdout as
 *                  "HX_WALL_SECONDS <t>" (std::chrono; the reference's clock() is CPU time).
 */
#include <chrono>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>

static int hx_printf(const char *fmt, ...) {
    if (!getenv("HX_VERBOSE")) return 0;
    va_list ap;
    va_start(ap, fmt);
    int r = vfprintf(stderr, fmt, ap);
    va_end(ap);
    return r;
}

static int hx_fprintf(FILE *fp, const char *fmt, ...) {
    std::string f(fmt);
    if (getenv("HX_FULL")) {
        std::string out;
        for (size_t i = 0; i < f.size();) {
            if (f.compare(i, 4, "%.7e") == 0) {
                out += "%.17e";
                i += 4;
            } else if (f.compare(i, 4, "%.5f") == 0) {
                out += "%.17g";
                i += 4;
            } else {
                out += f[i++];
            }
        }
        f = out;
    }
    va_list ap;
    va_start(ap, fmt);
    int r = vfprintf(fp, f.c_str(), ap);
    va_end(ap);
    return r;
}

#define printf hx_printf
#define fprintf hx_fprintf

#include "common.hpp"
#include "parameter.hpp"
#include "tools.hpp"
#include "bessel.hpp"
#include "particle.hpp"
#include "particleGadget.hpp"
#include "field.hpp"
#ifdef HX_DROPIN
/* the reference's estimator entry points with bodies over the B200 library: the same driver
 * flow, the same output files (tests/test_gpu_dropin.py compares them) */
#include "hitomi_dropin.hpp"
#else
#include "particle_reconstruction.hpp"
#include "powerspec.hpp"
#include "bispec.hpp"
#endif

#undef printf
#undef fprintf

static std::vector<double> read_f64(const char *path) {
    std::vector<double> v;
    FILE *fp = fopen(path, "rb");
    if (!fp) {
        std::fprintf(stderr, "cannot open %s\n", path);
        exit(2);
    }
    fseek(fp, 0, SEEK_END);
    long sz = ftell(fp);
    fseek(fp, 0, SEEK_SET);
    v.resize(sz / sizeof(double));
    if (fread(v.data(), sizeof(double), v.size(), fp) != v.size()) {
        std::fprintf(stderr, "short read %s\n", path);
        exit(2);
    }
    fclose(fp);
    return v;
}

static void fill_boss(ParticleBOSSClass &P, const std::vector<double> &a) {
    long long n = (long long)(a.size() / 4);
    if (P.initializeParticle(n)) exit(2);
    for (long long i = 0; i < n; i++) {
        P[i].pos[0] = a[4 * i + 0];
        P[i].pos[1] = a[4 * i + 1];
        P[i].pos[2] = a[4 * i + 2];
        P[i].w = a[4 * i + 3];
    }
    P.calcMinAndMax();
}

static int fail(const char *what) {
    std::fprintf(stderr, "'%s' fails.\n", what);
    return 1;
}

/* --unit OP: time one of the reference's periodic-box building blocks once, at the
 * parameter file's mesh, on this process's single core.  Set-up is not timed.  The
 * loops "triple" and "snloop" restate the inline driver loops of bispec.hpp:1158-1166
 * and bispec.hpp:1023-1050 (they are not functions in the reference). */
static volatile double hx_sink = 0.0;

static double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

#ifndef HX_DROPIN
static int unit_op(const std::string &op, ParticleGadgetClass &P_D, ParameterClass &param, std::vector<double> &kbin) {
    double t = 0.0;
    std::complex<double> shotnoise = double(P_D.n_tot);
    double dk = kbin[1] - kbin[0];
    int mid = param.n_kbin / 2;
    if (op == "assign") {
        DensityFieldClass<ParticleGadgetClass> dn(param);
        t = now_s();
        dn.calcNormalDensityFluctuationForBOX(P_D, param);
        t = now_s() - t;
    } else if (op == "fft" || op == "ifft" || op == "corr" || op == "bin_l0" || op == "bin_l2" || op == "xi_ijk") {
        DensityFieldClass<ParticleGadgetClass> dn(param);
        dn.calcNormalDensityFluctuationForBOX(P_D, param);
        if (op == "fft") {
            t = now_s();
            dn.calcFourierTransform();
            t = now_s() - t;
        } else {
            dn.calcFourierTransform();
            TwoPointStatisticsClass<ParticleGadgetClass> stat(param);
            if (op == "ifft") {
                t = now_s();
                dn.calcInverseFourierTransform();
                t = now_s() - t;
            } else if (op == "corr") {
                t = now_s();
                dn.calcAssignmentFunctionCorrection();
                t = now_s() - t;
            } else if (op == "bin_l0" || op == "bin_l2") {
                int ell = (op == "bin_l0") ? 0 : 2;
                t = now_s();
                stat.calcPowerSpectrum(dn, dn, kbin.data(), shotnoise, ell, 0);
                t = now_s() - t;
            } else {
                fftw_complex *xi = fftw_alloc_complex(param.n_mesh_tot);
                for (long long i = 0; i < param.n_mesh_tot; i++) xi[i][0] = xi[i][1] = 0.0;
                t = now_s();
                stat.calcShotNoiseForBispectrum_ijk(dn, dn, shotnoise, 0, 0, xi);
                t = now_s() - t;
                fftw_free(xi);
            }
        }
    } else if (op == "ylmk" || op == "ylmx") {
        std::complex<double> *Y = new std::complex<double>[param.n_mesh_tot];
        t = now_s();
        if (op == "ylmk") ToolClass::storeReducedSphericalHarmonicsInFourierSpace(1, 0, param, Y);
        else ToolClass::storeReducedSphericalHarmonicsInConfigurationSpace(1, 0, param, Y);
        t = now_s() - t;
        delete[] Y;
    } else if (op == "shell") {
        DensityFieldClass<ParticleGadgetClass> dn(param);
        dn.calcNormalDensityFluctuationForBOX(P_D, param);
        dn.calcFourierTransform();
        std::complex<double> *Y = new std::complex<double>[param.n_mesh_tot];
        ToolClass::storeReducedSphericalHarmonicsInFourierSpace(0, 0, param, Y);
        DensityFieldClass<ParticleGadgetClass> tilde(param);
        t = now_s();
        tilde.calcInverseFourierTransformForBispectrum(dn, kbin[mid], dk, Y);
        t = now_s() - t;
        delete[] Y;
    } else if (op == "triple") {
        DensityFieldClass<ParticleGadgetClass> f1(param), f2(param), f3(param);
        f1.calcNormalDensityFluctuationForBOX(P_D, param);
        for (long long i = 0; i < param.n_mesh_tot; i++) {
            f2.field[i][0] = f3.field[i][0] = f1.field[i][0];
            f2.field[i][1] = f3.field[i][1] = 0.5;
        }
        t = now_s();
        std::complex<double> bk_sum = 0.0;
        double fac = param.volume / double(param.n_mesh_tot);
        for (long long coord = 0; coord < param.n_mesh_tot; coord++) {
            std::complex<double> a(f1[coord][0], f1[coord][1]);
            std::complex<double> b(f2[coord][0], f2[coord][1]);
            std::complex<double> c(f3[coord][0], f3[coord][1]);
            bk_sum += (fac * a * b * c);
        }
        t = now_s() - t;
        hx_sink = bk_sum.real() + bk_sum.imag();
    } else if (op == "snloop" || op == "spline") {
        double t0 = now_s();
        SphericalBesselClass sj1(0), sj2(0);
        double tsp = now_s() - t0;
        if (op == "spline") {
            t = tsp / 2.0;
        } else {
            std::complex<double> *Y1 = new std::complex<double>[param.n_mesh_tot];
            std::complex<double> *Y2 = new std::complex<double>[param.n_mesh_tot];
            fftw_complex *xi = fftw_alloc_complex(param.n_mesh_tot);
            for (long long i = 0; i < param.n_mesh_tot; i++) {
                Y1[i] = Y2[i] = 1.0;
                xi[i][0] = 1.0e-3 * double(i % 7);
                xi[i][1] = 0.0;
            }
            double kmag1 = kbin[0], kmag2 = kbin[mid];
            t = now_s();
            std::complex<double> sn_sum = 0.0;
            double dr[3] = {param.boxsize[0] / double(param.n_mesh[0]), param.boxsize[1] / double(param.n_mesh[1]),
                            param.boxsize[2] / double(param.n_mesh[2])};
            for (int i = 0; i < param.n_mesh[0]; i++)
                for (int j = 0; j < param.n_mesh[1]; j++)
                    for (int k = 0; k < param.n_mesh[2]; k++) {
                        long long coord = ((long long)i * param.n_mesh[1] + j) * param.n_mesh[2] + k;
                        double rv0 = (i < param.n_mesh[0] / 2) ? (double)i * dr[0] : (double)(i - param.n_mesh[0]) * dr[0];
                        double rv1 = (j < param.n_mesh[1] / 2) ? (double)j * dr[1] : (double)(j - param.n_mesh[1]) * dr[1];
                        double rv2 = (k < param.n_mesh[2] / 2) ? (double)k * dr[2] : (double)(k - param.n_mesh[2]) * dr[2];
                        double rmag = sqrt(rv0 * rv0 + rv1 * rv1 + rv2 * rv2);
                        std::complex<double> ff(xi[coord][0], xi[coord][1]);
                        double j1 = sj1.getSphericalBessel(kmag1 * rmag);
                        double j2 = sj2.getSphericalBessel(kmag2 * rmag);
                        sn_sum += (j1 * j2 * ff * Y1[coord] * Y2[coord]);
                    }
            t = now_s() - t;
            hx_sink = sn_sum.real() + sn_sum.imag();
            delete[] Y1;
            delete[] Y2;
            fftw_free(xi);
        }
    } else {
        return fail(("unknown unit op " + op).c_str());
    }
    std::printf("HX_UNIT %s %.6f\n", op.c_str(), t);
    return 0;
}

#endif

int main(int argc, char **argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: ref_harness param.ini data.f64 [random.f64] [--all-rows]\n");
        return 2;
    }
    bool all_rows = false, box_recon = false;
    std::string unit;
    std::vector<const char *> pos;
    for (int i = 1; i < argc; i++) {
        if (!strcmp(argv[i], "--all-rows")) all_rows = true;
        else if (!strcmp(argv[i], "--box-recon")) box_recon = true;
        else if (!strcmp(argv[i], "--unit") && i + 1 < argc) unit = argv[++i];
        else pos.push_back(argv[i]);
    }
    /* --read-ascii FILE OUT / --read-gadget BASE OUT: run the reference's readers
     * (particle.hpp:93-154, particleGadget.hpp:211-298) and write what they hold as raw
     * doubles (x y z w / x y z vx vy vz per particle) */
    if (pos.size() == 3 && !strcmp(pos[0], "--read-ascii")) {
        ParticleBOSSClass P;
        std::string fn(pos[1]);
        if (P.readParticleBOSS(fn)) return fail("readParticleBOSS");
        FILE *fo = fopen(pos[2], "wb");
        for (long long i = 0; i < P.n_tot; i++) {
            double r[4] = {P[i].pos[0], P[i].pos[1], P[i].pos[2], P[i].w};
            fwrite(r, sizeof(double), 4, fo);
        }
        fclose(fo);
        return 0;
    }
    if (pos.size() == 3 && !strcmp(pos[0], "--read-gadget")) {
        ParticleGadgetClass P;
        std::string fn(pos[1]);
        if (P.readParticlesFromGagdetSnapshot(fn)) return fail("readParticlesFromGagdetSnapshot");
        FILE *fo = fopen(pos[2], "wb");
        for (long long i = 0; i < P.n_tot; i++) {
            double r[6] = {P[i].pos[0], P[i].pos[1], P[i].pos[2], P[i].vel[0], P[i].vel[1], P[i].vel[2]};
            fwrite(r, sizeof(double), 6, fo);
        }
        fclose(fo);
        return 0;
    }
    char *pargv[2] = {argv[0], (char *)pos[0]};
    ParameterClass param;
    if (param.readParameters(pargv)) return fail("param.readParameters");
#ifdef HX_DROPIN
    if (hitomi_dropin_configure(pos[0])) return fail("hitomi_dropin_configure");
#endif
    if (param.makeOutputDirectory()) return fail("param.makeOutputDirectory");
    if (param.printParameters()) return fail("param.printParameters");
    std::vector<double> kbin(param.n_kbin), rbin(param.n_rbin);
    ToolClass::setKbin(param, kbin.data());
    ToolClass::setRbin(param, rbin.data());

    auto t0 = std::chrono::steady_clock::now();
    int rc = 0;
    if (box_recon && pos.size() == 3) {
        /* periodic box with reconstruction: main_box.cpp:134-152 then the recon estimators
         * (randoms from the second file instead of readRandomParticles); the shifted
         * positions are also written to output_dir/recon_{D,R}.f64 */
        std::vector<double> a = read_f64(pos[1]), b = read_f64(pos[2]);
        ParticleGadgetClass P_D, P_R;
        long long nd = (long long)(a.size() / 3), nr = (long long)(b.size() / 3);
        if (P_D.initializeParticle(nd) || P_R.initializeParticle(nr)) return fail("initializeParticle");
        for (long long i = 0; i < nd; i++)
            for (int ax = 0; ax < 3; ax++) P_D[i].pos[ax] = a[3 * i + ax];
        for (long long i = 0; i < nr; i++)
            for (int ax = 0; ax < 3; ax++) P_R[i].pos[ax] = b[3 * i + ax];
        P_D.calcMinAndMax();
        P_R.calcMinAndMax();
        t0 = std::chrono::steady_clock::now();
        if (calcReconstructionParticlesForBOX(P_D, P_R, param)) return fail("calcReconstructionParticlesForBOX");
        for (int s = 0; s < 2; s++) {
            ParticleGadgetClass &P = s ? P_R : P_D;
            std::string fn = param.output_dir + (s ? "/recon_R.f64" : "/recon_D.f64");
            FILE *fo = fopen(fn.c_str(), "wb");
            for (long long i = 0; i < P.n_tot; i++) fwrite(P[i].pos, sizeof(double), 3, fo);
            fclose(fo);
        }
        P_D.calcPeriodicBoundary(param);
        P_R.calcPeriodicBoundary(param);
        double alpha = double(P_D.n_tot) / double(P_R.n_tot);
        if (param.measure == "pk") rc = calcPowerSpectrumForBOXForReconstruction(P_D, P_R, param, alpha, kbin.data());
        else if (param.measure == "2PCF") rc = calcTwoPointFunctionForBOXForReconstruction(P_D, P_R, param, alpha, rbin.data());
        else if (param.measure == "bk") {  /* main_box.cpp:211-215, one ith_kbin row per run */
            int lo = all_rows ? 0 : param.ith_kbin, hi = all_rows ? param.n_kbin : param.ith_kbin + 1;
            for (int i = lo; i < hi && rc == 0; i++) {
                param.ith_kbin = i;
                rc = calcBiSpectrumForBOXForReconstruction(P_D, P_R, param, alpha, kbin.data());
            }
        } else if (param.measure == "3PCF") {  /* main_box.cpp:216-220 */
            int lo = all_rows ? 0 : param.ith_rbin, hi = all_rows ? param.n_rbin : param.ith_rbin + 1;
            for (int i = lo; i < hi && rc == 0; i++) {
                param.ith_rbin = i;
                rc = calcThreePointCorrelationFunctionForBOXForReconstruction(P_D, P_R, param, alpha, rbin.data());
            }
        } else return fail("measure");
    } else if (pos.size() == 2) {
        /* periodic box: main_box.cpp:96-228 (reader replaced, boxsize from param) */
        std::vector<double> a = read_f64(pos[1]);
        ParticleGadgetClass P_D;
        long long n = (long long)(a.size() / 3);
        if (P_D.initializeParticle(n)) return fail("P_D.initializeParticle");
        for (long long i = 0; i < n; i++)
            for (int ax = 0; ax < 3; ax++) P_D[i].pos[ax] = a[3 * i + ax];
        P_D.calcMinAndMax();
#ifndef HX_DROPIN
        if (!unit.empty()) return unit_op(unit, P_D, param, kbin);
#endif
        t0 = std::chrono::steady_clock::now();
        if (param.measure == "pk") {
            rc = calcPowerSpectrumForBOX(P_D, param, kbin.data());
        } else if (param.measure == "2PCF") {
            rc = calcTwoPointCorrelationFunctionForBOX(P_D, param, rbin.data());
        } else if (param.measure == "bk") {
            int lo = all_rows ? 0 : param.ith_kbin, hi = all_rows ? param.n_kbin : param.ith_kbin + 1;
            for (int i = lo; i < hi && rc == 0; i++) {
                param.ith_kbin = i;
                rc = calcBiSpectrumForBOX(P_D, param, kbin.data());
            }
        } else if (param.measure == "3PCF") {
            int lo = all_rows ? 0 : param.ith_rbin, hi = all_rows ? param.n_rbin : param.ith_rbin + 1;
            for (int i = lo; i < hi && rc == 0; i++) {
                param.ith_rbin = i;
                rc = calcThreePointCorrelationFunctionForBOX(P_D, param, rbin.data());
            }
        } else {
            return fail("measure");
        }
    } else {
        /* survey geometry: main.cpp:129-275 (ASCII reader replaced by raw doubles) */
        ParticleBOSSClass P_D, P_R;
        fill_boss(P_D, read_f64(pos[1]));
        fill_boss(P_R, read_f64(pos[2]));
        if (P_D.calcTotalNumberOfParticlesWithWeights()) return fail("P_D.calcTotalNumberOfParticlesWithWeights");
        if (P_R.calcTotalNumberOfParticlesWithWeights()) return fail("P_R.calcTotalNumberOfParticlesWithWeights");
        if (P_D.calcLOS()) return fail("P_D.calcLOS");
        if (P_R.calcLOS()) return fail("P_R.calcLOS");
        double alpha = ParticleBOSSClass::calcAlpha(P_D, P_R);
        if (alpha < 0.0) return fail("calcAlpha");
        if (ParticleBOSSClass::resetParticleForFFT(P_D, P_R, param)) return fail("resetParticleForFFT");
        t0 = std::chrono::steady_clock::now();
        DensityFieldClass<ParticleBOSSClass> Vol(param);
        double Vsurvey = Vol.calcSurveyVolume(P_R);
        Vol.finalizeDensityField();
        double nbar = ParticleBOSSClass::calcMeanNumberDensity(P_D, Vsurvey);
        if (nbar < 0.0) return fail("calcMeanNumberDensity");
        if (ParticleBOSSClass::printParameters(param, P_D, P_R, alpha, Vsurvey, nbar)) return fail("printParameters");
        if (param.flag_recon == "True") {
            /* main.cpp:215-225; the shifted positions also go to output_dir/recon_{D,R}.f64 */
            if (calcReconstructionParticles(P_D, P_R, param, alpha, Vsurvey)) return fail("calcReconstructionParticles");
            for (int s = 0; s < 2; s++) {
                ParticleBOSSClass &P = s ? P_R : P_D;
                std::string fn = param.output_dir + (s ? "/recon_R.f64" : "/recon_D.f64");
                FILE *fo = fopen(fn.c_str(), "wb");
                for (long long i = 0; i < P.n_tot; i++) fwrite(P[i].pos, sizeof(double), 3, fo);
                fclose(fo);
            }
            ParticleBOSSClass::resetParticleForFFT(P_D, P_R, param);
        }
        {
            /* full-precision survey scalars for the parity tests */
            std::string fn = param.output_dir + "/survey_scalars_full";
            FILE *fp = fopen(fn.c_str(), "w");
            std::fprintf(fp, "%.17e %.17e %.17e %.17e %.17e\n", alpha, Vsurvey, nbar, P_D.n_tot_weight,
                         P_R.n_tot_weight);
            fclose(fp);
        }
        if (param.measure == "pk") {
            rc = calcPowerSpectrum(P_D, P_R, param, alpha, kbin.data(), Vsurvey);
        } else if (param.measure == "2PCF") {
            rc = calcTwoPointCorrelationFunction(P_D, P_R, param, alpha, rbin.data(), Vsurvey);
        } else if (param.measure == "window2PCF") {
            rc = calcTwoPointWindowCorrelationFunction(P_R, param, rbin.data(), Vsurvey);
        } else if (param.measure == "window3PCF") {
            int lo = all_rows ? 0 : param.ith_rbin, hi = all_rows ? param.n_rbin : param.ith_rbin + 1;
            for (int i = lo; i < hi && rc == 0; i++) {
                param.ith_rbin = i;
                rc = calcThreePointWindowCorrelationFunction(P_R, param, rbin.data(), Vsurvey);
            }
        } else if (param.measure == "bk") {
            int lo = all_rows ? 0 : param.ith_kbin, hi = all_rows ? param.n_kbin : param.ith_kbin + 1;
            for (int i = lo; i < hi && rc == 0; i++) {
                param.ith_kbin = i;
                rc = calcBiSpectrum(P_D, P_R, param, alpha, kbin.data(), Vsurvey);
            }
        } else if (param.measure == "3PCF") {
            int lo = all_rows ? 0 : param.ith_rbin, hi = all_rows ? param.n_rbin : param.ith_rbin + 1;
            for (int i = lo; i < hi && rc == 0; i++) {
                param.ith_rbin = i;
                rc = calcThreePointCorrelationFunction(P_D, P_R, param, alpha, rbin.data(), Vsurvey);
            }
        } else {
            return fail("measure");
        }
    }
    double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (getenv("HX_TIMING")) std::printf("HX_WALL_SECONDS %.6f\n", wall);
    if (rc) return fail(param.measure.c_str());
    return 0;
}
