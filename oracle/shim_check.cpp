// oracle/shim_check.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Evaluates the project-written FFTW and GSL shims (oracle/shim/) on inputs read from a
// binary file, so that tests/test_oracle_shims.py can compare them with numpy / scipy.
// Usage:
//   shim_check fft n0 n1 n2 sign in.f64 out.f64     3-D complex DFT (fftw_plan_dft_3d)
//   shim_check plm in.f64 out.f64                    rows (l, m, x) -> gsl_sf_legendre_sphPlm
//   shim_check jl in.f64 out.f64                     rows (l, x) -> gsl_sf_bessel_jl
//   shim_check w3j in.f64 out.f64                    rows (2ja,2jb,2jc,2ma,2mb,2mc) -> 3j
//   shim_check spline n in.f64 out.f64               n knots (x, y), then queries -> cspline
#include <fftw3.h>
#include <gsl/gsl_sf_bessel.h>
#include <gsl/gsl_sf_coupling.h>
#include <gsl/gsl_sf_legendre.h>
#include <gsl/gsl_spline.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

static std::vector<double> read_all(const char *path) {
    std::vector<double> v;
    FILE *fp = fopen(path, "rb");
    if (!fp) {
        fprintf(stderr, "cannot open %s\n", path);
        exit(2);
    }
    double buf[4096];
    size_t got;
    while ((got = fread(buf, sizeof(double), 4096, fp)) > 0) v.insert(v.end(), buf, buf + got);
    fclose(fp);
    return v;
}

static void write_all(const char *path, const std::vector<double> &v) {
    FILE *fp = fopen(path, "wb");
    if (!fp || fwrite(v.data(), sizeof(double), v.size(), fp) != v.size()) {
        fprintf(stderr, "cannot write %s\n", path);
        exit(2);
    }
    fclose(fp);
}

int main(int argc, char **argv) {
    if (argc < 4) {
        fprintf(stderr, "usage: shim_check fft|plm|jl|w3j|spline ...\n");
        return 2;
    }
    const char *op = argv[1];
    std::vector<double> out;
    if (!strcmp(op, "fft") && argc == 8) {
        const int n0 = atoi(argv[2]), n1 = atoi(argv[3]), n2 = atoi(argv[4]), sign = atoi(argv[5]);
        std::vector<double> in = read_all(argv[6]);
        const size_t n = (size_t)n0 * n1 * n2;
        if (in.size() != 2 * n) return 3;
        fftw_complex *a = fftw_alloc_complex(n);
        fftw_complex *b = fftw_alloc_complex(n);
        memcpy(a, in.data(), sizeof(double) * 2 * n);
        fftw_plan p = fftw_plan_dft_3d(n0, n1, n2, a, b, sign > 0 ? FFTW_BACKWARD : FFTW_FORWARD, FFTW_ESTIMATE);
        fftw_execute(p);
        fftw_destroy_plan(p);
        out.assign((double *)b, (double *)b + 2 * n);
        fftw_free(a);
        fftw_free(b);
        write_all(argv[7], out);
    } else if (!strcmp(op, "plm")) {
        std::vector<double> in = read_all(argv[2]);
        for (size_t i = 0; i + 2 < in.size(); i += 3)
            out.push_back(gsl_sf_legendre_sphPlm((int)in[i], (int)in[i + 1], in[i + 2]));
        write_all(argv[3], out);
    } else if (!strcmp(op, "jl")) {
        std::vector<double> in = read_all(argv[2]);
        for (size_t i = 0; i + 1 < in.size(); i += 2) out.push_back(gsl_sf_bessel_jl((int)in[i], in[i + 1]));
        write_all(argv[3], out);
    } else if (!strcmp(op, "w3j")) {
        std::vector<double> in = read_all(argv[2]);
        for (size_t i = 0; i + 5 < in.size(); i += 6)
            out.push_back(gsl_sf_coupling_3j((int)in[i], (int)in[i + 1], (int)in[i + 2], (int)in[i + 3],
                                             (int)in[i + 4], (int)in[i + 5]));
        write_all(argv[3], out);
    } else if (!strcmp(op, "spline") && argc == 5) {
        const size_t n = (size_t)atol(argv[2]);
        std::vector<double> in = read_all(argv[3]);
        if (in.size() < 2 * n) return 3;
        gsl_interp_accel *acc = gsl_interp_accel_alloc();
        gsl_spline *s = gsl_spline_alloc(gsl_interp_cspline, n);
        gsl_spline_init(s, in.data(), in.data() + n, n);
        for (size_t i = 2 * n; i < in.size(); i++) out.push_back(gsl_spline_eval(s, in[i], acc));
        gsl_spline_free(s);
        gsl_interp_accel_free(acc);
        write_all(argv[4], out);
    } else {
        fprintf(stderr, "unknown operation or arguments\n");
        return 2;
    }
    return 0;
}
