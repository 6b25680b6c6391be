// hg_io.cpp -- catalogue ingest for the C ABI (include/hitomi_gpu.h): the reference's
// readers, native and multi-threaded.
//
//   hg_read_ascii   ParticleBOSSClass::readParticleBOSS (particle.hpp:93-154): every line
//                   from which four numbers x y z w can be read (sscanf "%lf %lf %lf %lf") is
//                   one particle; other lines are skipped.  Here the file is memory-read
//                   once and split into byte ranges at line ends, one per thread; each
//                   thread applies the same rule with strtod (the conversion sscanf's %lf
//                   performs) and the ranges are joined in file order.
//   hg_read_gadget  ParticleGadgetClass::readParticlesFromGagdetSnapshot
//                   (particleGadget.hpp:127-168, 211-298): files base.0 .. base.(num_files-1),
//                   each a 256-byte header block then position, velocity and id blocks
//                   (Fortran record markers around each); positions as double, velocities
//                   times sqrt(a) (a = header time).
#include "hitomi_gpu.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

namespace hg {
void set_contextless_error(const std::string &m);
}

namespace {

int io_fail(const std::string &m) {
    hg::set_contextless_error(m);
    return -1;
}

bool read_file(const char *path, std::vector<char> &buf) {
    FILE *fp = fopen(path, "rb");
    if (!fp) return false;
    fseek(fp, 0, SEEK_END);
    const long sz = ftell(fp);
    fseek(fp, 0, SEEK_SET);
    buf.resize((size_t)std::max(sz, 0L) + 1);
    const size_t got = sz > 0 ? fread(buf.data(), 1, (size_t)sz, fp) : 0;
    fclose(fp);
    buf.resize(got + 1);
    buf[got] = '\0';  // strtod stops at the end of the data
    return true;
}

// Parse lines [b, e): one record of `ncols` doubles per line whose first ncols fields read.
// Each line is copied into a terminated scratch string so strtod cannot run past its end
// (sscanf in the reference sees one line at a time, as std::getline returned it).
void parse_range(const char *b, const char *e, int ncols, std::vector<double> &out) {
    std::string line;
    const char *p = b;
    while (p < e) {
        const char *nl = static_cast<const char *>(memchr(p, '\n', (size_t)(e - p)));
        const char *le = nl ? nl : e;
        line.assign(p, (size_t)(le - p));
        const char *q = line.c_str();
        double v[16];
        int k = 0;
        for (; k < ncols; k++) {
            char *end = nullptr;
            v[k] = strtod(q, &end);
            if (end == q) break;
            q = end;
        }
        if (k == ncols) out.insert(out.end(), v, v + ncols);
        p = nl ? nl + 1 : e;
    }
}

}  // namespace

extern "C" {

void hg_free(void *p) { free(p); }

int hg_read_ascii(const char *path, int ncols, double **out, long long *n) {
    if (!path || !out || !n) return io_fail("hg_read_ascii: null argument");
    if (ncols < 1 || ncols > 16) return io_fail("hg_read_ascii: ncols must be in [1, 16]");
    *out = nullptr;
    *n = 0;
    std::vector<char> buf;
    if (!read_file(path, buf)) return io_fail(std::string("Cannot open the file '") + path + "'");
    const size_t size = buf.size() - 1;
    const char *data = buf.data();
    unsigned nt = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    if (size < (1u << 20)) nt = 1;
    // byte ranges that start at a line start
    std::vector<size_t> cut(nt + 1, size);
    cut[0] = 0;
    for (unsigned t = 1; t < nt; t++) {
        size_t c = std::max(cut[t - 1], size * t / nt);
        while (c < size && c > 0 && data[c - 1] != '\n') c++;
        cut[t] = c;
    }
    std::vector<std::vector<double>> part(nt);
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; t++)
        th.emplace_back([&, t] { parse_range(data + cut[t], data + cut[t + 1], ncols, part[t]); });
    for (auto &x : th) x.join();
    size_t total = 0;
    for (auto &p : part) total += p.size();
    double *res = static_cast<double *>(malloc(std::max<size_t>(total, 1) * sizeof(double)));
    if (!res) return io_fail("hg_read_ascii: out of host memory");
    size_t o = 0;
    for (auto &p : part) {
        if (!p.empty()) memcpy(res + o, p.data(), p.size() * sizeof(double));
        o += p.size();
    }
    *out = res;
    *n = (long long)(total / (size_t)ncols);
    return 0;
}

int hg_read_gadget(const char *base, double **out, long long *n, hg_gadget_header *hdr) {
    if (!base || !out || !n) return io_fail("hg_read_gadget: null argument");
    *out = nullptr;
    *n = 0;
    static_assert(sizeof(hg_gadget_header) == 256, "Gadget header block is 256 bytes");
    auto read_header = [&](FILE *fp, hg_gadget_header &h) {
        int mark = 0;
        return fread(&mark, sizeof(int), 1, fp) == 1 && fread(&h, sizeof(h), 1, fp) == 1 &&
               fread(&mark, sizeof(int), 1, fp) == 1;
    };
    std::string f0 = std::string(base) + ".0";
    FILE *fp = fopen(f0.c_str(), "rb");
    if (!fp) return io_fail("can not open " + f0);
    hg_gadget_header h0;
    const bool ok0 = read_header(fp, h0);
    fclose(fp);
    if (!ok0) return io_fail("short Gadget header in " + f0);
    long long ntot = 0;
    for (int k = 0; k < 6; k++) ntot += h0.npartTotal[k];
    if (ntot <= 0) return io_fail("The number of particles should be > 0");
    if (h0.num_files <= 0) return io_fail("Gadget header: num_files <= 0");
    const double sqa = std::sqrt(h0.time);
    double *res = static_cast<double *>(malloc((size_t)ntot * 6 * sizeof(double)));
    if (!res) return io_fail("hg_read_gadget: out of host memory");
    long long pc = 0;
    std::vector<float> block;
    for (int i = 0; i < h0.num_files; i++) {
        const std::string fn = std::string(base) + "." + std::to_string(i);
        FILE *f = fopen(fn.c_str(), "rb");
        if (!f) {
            free(res);
            return io_fail("can not open " + fn);
        }
        hg_gadget_header h;
        long long np = 0;
        bool ok = read_header(f, h);
        for (int k = 0; ok && k < 6; k++) np += h.npart[k];
        ok = ok && np >= 0 && pc + np <= ntot;
        block.resize((size_t)std::max<long long>(np, 1) * 3);
        int mark = 0;
        for (int blk = 0; ok && blk < 2; blk++) {  // positions, velocities
            ok = fread(&mark, sizeof(int), 1, f) == 1 && fread(block.data(), sizeof(float), (size_t)np * 3, f) == (size_t)np * 3 &&
                 fread(&mark, sizeof(int), 1, f) == 1;
            if (!ok) break;
            for (long long p = 0; p < np; p++)
                for (int k = 0; k < 3; k++)
                    res[(size_t)(pc + p) * 6 + 3 * blk + k] =
                        blk == 0 ? (double)block[(size_t)p * 3 + k] : (double)block[(size_t)p * 3 + k] * sqa;
        }
        fclose(f);
        if (!ok) {
            free(res);
            return io_fail("short or inconsistent Gadget file " + fn);
        }
        pc += np;
    }
    if (pc != ntot) {
        free(res);
        return io_fail("readParticlesFromSnapshotOfGadget(std::string & snapshotFileName) fails.");
    }
    if (hdr) *hdr = h0;
    *out = res;
    *n = ntot;
    return 0;
}

}  // extern "C"
