// hg_assign.cuh -- particle-to-mesh assignment (NGP/CIC/TSC, PCS extension) for sm_100a.
//
// Sorted-by-tile scatter with no global float atomics in the particle loop:
//   1. k_bin_count   : per particle, the reference's cell/weight arithmetic in FP64
//                      (field.hpp:80-90 NGP, :117-129 CIC, :158-172 TSC), the set of
//                      output tiles its stencil touches (warp-aggregated counts), and
//                      the FP64 in-bounds mass;
//   2. exclusive scan of the per-tile counts; tiles cut into chunks of <= CH records;
//   3. k_bin_scatter : one compact record per (particle, tile) in tile order;
//   4. k_tile_accum  : one CTA per chunk accumulates its records in a shared-memory tile
//                      (the mesh's precision); a tile with a single chunk is written once, coalesced; the
//                      chunks of a densely populated tile (clustered catalogues) are
//                      zeroed first and add their partial tiles (one add per cell per
//                      chunk, not per particle).
// A particle whose stencil straddles tiles is duplicated into each of them; each CTA
// keeps only the stencil points that fall in its own tile.
//
// Boundary rule.  The reference tests only 0 <= flat < N (field.hpp:92-96): an axis
// index of -1 or n lands in the neighbouring row/plane rather than wrapping, and
// points past either end of the array are dropped.  periodic = 0 reproduces that
// (needed for parity); periodic = 1 wraps each axis (PCS / interlacing extension).
#pragma once

#include "hg_common.cuh"

namespace hg {
// one copy per translation unit: each .cu file names its own HG_TU_NS, so the kernels and
// helpers of this header never collide at link time
inline namespace HG_TU_NS {

struct AssignGeom {
    int n[3];
    double L[3];
    long long ntot;
    int scheme;       // HG_NGP..HG_PCS
    int periodic;     // 0 = reference flat-index rule
    double shift;     // added to the scaled position (0, or 0.5 for the interlaced copy)
    int t[3];         // tile extent per axis
    int tsh[3];       // log2 t[a] when t[a] is a power of two, else -1 (tile_axis)
    int nt[3];        // tiles per axis
    double factor;      // 1/dV (field.hpp:76-77), used for the FP64 in-bounds mass
    double acc_factor;  // factor applied in the mesh accumulation (1/dV, or 1 for a mass mesh)
    float fix_bound;    // bound on |w acc_factor prod(w_axis)| per record (fixed-point accumulation)
    double far[3];      // 2^30 L / n: coordinates at least this far from 0 are "far" (far_reduce)
};

__host__ __device__ __forceinline__ int stencil_width(int scheme) { return scheme + 1; }
__host__ __device__ __forceinline__ int stencil_start(int scheme) { return (scheme >= 2) ? -1 : 0; }

// Anchor index and offset per axis, exactly the reference's FP64 expressions.
__device__ __forceinline__ void anchor(double pos, int n, double L, int scheme, double shift, int &i, double &d) {
    double xp = pos * double(n) / L;
    if (shift != 0.0) xp += shift;
    if (scheme == 0) {          // NGP: iw = int(xp + 0.5)
        i = int(xp + 0.5);
        d = 0.0;
    } else if (scheme == 1) {   // CIC: iw0 = int(xp), dx = xp - iw0
        i = int(xp);
        d = xp - double(i);
    } else if (scheme == 2) {   // TSC: iw1 = int(xp + 0.5), dx = xp - iw1
        i = int(xp + 0.5);
        d = xp - double(i);
    } else {                    // PCS: i = floor(xp), t = xp - i
        i = (int)floor(xp);
        d = xp - double(i);
    }
}

// Stencil weights per axis (index 0 = first stencil point).
template <typename T>
__device__ __forceinline__ void axis_weights(int scheme, T d, T *w) {
    if (scheme == 0) {
        w[0] = (T)1;
    } else if (scheme == 1) {
        w[0] = (T)1 - d;
        w[1] = d;
    } else if (scheme == 2) {
        w[0] = (T)0.5 * ((T)0.5 - d) * ((T)0.5 - d);
        w[1] = (T)0.75 - d * d;
        w[2] = (T)0.5 * ((T)0.5 + d) * ((T)0.5 + d);
    } else {
        T t = d, u = (T)1 - d;
        w[0] = u * u * u / (T)6;
        w[1] = ((T)4 - (T)6 * t * t + (T)3 * t * t * t) / (T)6;
        w[2] = ((T)1 + (T)3 * t + (T)3 * t * t - (T)3 * t * t * t) / (T)6;
        w[3] = t * t * t / (T)6;
    }
}

// i mod n for i within one period of [0, n) (stencil indices of particles inside the
// box), the general remainder otherwise.
__device__ __forceinline__ int wrap_cell(int i, int n) {
    if (i >= -n && i < 2 * n) return i < 0 ? i + n : (i >= n ? i - n : i);
    const int c = i % n;
    return c < 0 ? c + n : c;
}

// Stencil weight j of one axis: the same expressions as axis_weights, without an array
// (for loops whose index is not known at compile time).
template <typename T>
__device__ __forceinline__ T axis_weight_at(int scheme, T d, int j) {
    if (scheme == 0) return (T)1;
    if (scheme == 1) return j == 0 ? (T)1 - d : d;
    if (scheme == 2) {
        if (j == 1) return (T)0.75 - d * d;
        const T e = (j == 0) ? (T)0.5 - d : (T)0.5 + d;
        return (T)0.5 * e * e;
    }
    const T t = d, u = (T)1 - d;
    if (j == 0) return u * u * u / (T)6;
    if (j == 1) return ((T)4 - (T)6 * t * t + (T)3 * t * t * t) / (T)6;
    if (j == 2) return ((T)1 + (T)3 * t + (T)3 * t * t - (T)3 * t * t * t) / (T)6;
    return t * t * t / (T)6;
}

// Effective cell of stencil point (ix, iy, iz); false if the reference drops it.  The
// non-periodic rule decomposes the flat index (ix n1 + iy) n2 + iz: with iz and iy within
// one period of their ranges this is a carry from z into y and from y into x (then
// 0 <= flat < N exactly when the carried ix is in range); a 64-bit division otherwise.
__device__ __forceinline__ bool effective_cell(const AssignGeom &g, int ix, int iy, int iz, int &cx, int &cy, int &cz) {
    if (g.periodic) {
        cx = wrap_cell(ix, g.n[0]);
        cy = wrap_cell(iy, g.n[1]);
        cz = wrap_cell(iz, g.n[2]);
        return true;
    }
    if (ix >= 0 && ix < g.n[0] && iy >= 0 && iy < g.n[1] && iz >= 0 && iz < g.n[2]) {
        cx = ix;
        cy = iy;
        cz = iz;
        return true;
    }
    if (iz >= -g.n[2] && iz < 2 * g.n[2] && iy > -g.n[1] && iy < 2 * g.n[1] - 1) {
        if (iz < 0) {
            iz += g.n[2];
            iy--;
        } else if (iz >= g.n[2]) {
            iz -= g.n[2];
            iy++;
        }
        if (iy < 0) {
            iy += g.n[1];
            ix--;
        } else if (iy >= g.n[1]) {
            iy -= g.n[1];
            ix++;
        }
        if (ix < 0 || ix >= g.n[0]) return false;
        cx = ix;
        cy = iy;
        cz = iz;
        return true;
    }
    long long coord = ((long long)ix * g.n[1] + iy) * (long long)g.n[2] + iz;
    if (coord < 0 || coord >= g.ntot) return false;
    long long nyz = (long long)g.n[1] * g.n[2];
    cx = (int)(coord / nyz);
    long long rem = coord - (long long)cx * nyz;
    cy = (int)(rem / g.n[2]);
    cz = (int)(rem - (long long)cy * g.n[2]);
    return true;
}

struct PartSrc {
    const unsigned char *base;  // device copy of the caller's array of structs
    long long n;
    long long stride;           // bytes
    int pos_off;                // doubles
    int w_off;                  // doubles, < 0: weight 1
    const double2 *cw;          // optional per-particle complex weight, overrides w
    double scale;               // multiplies the weight (e.g. -alpha for randoms)
    int ylm_on;                 // weight *= Yhat_lm(los) (field.hpp:199-216), or conj(Yhat_lm) when ylm_conj
    int ylm_l, ylm_m;
    int los_off;                // doubles
    int wpow;                   // the weight enters as w^wpow (0 or 1: w; 2: the shot-noise fields, field.hpp:249-306)
    int ylm_conj;
};

__device__ __forceinline__ void load_pos(const PartSrc &s, long long p, double pos[3]) {
    const double *rec = reinterpret_cast<const double *>(s.base + p * s.stride);
    pos[0] = rec[s.pos_off + 0];
    pos[1] = rec[s.pos_off + 1];
    pos[2] = rec[s.pos_off + 2];
}

// The particle's assignment weight: w (or 1), times Yhat_lm(los) when requested, times
// the source's scale; (Yhat.re w, Yhat.im w) as in field.hpp:199-216.
__device__ __forceinline__ void load_weight(const PartSrc &s, long long p, double &wr, double &wi) {
    const double *rec = reinterpret_cast<const double *>(s.base + p * s.stride);
    if (s.cw) {
        double2 c = s.cw[p];
        wr = c.x;
        wi = c.y;
    } else {
        double w = (s.w_off >= 0) ? rec[s.w_off] : 1.0;
        if (s.wpow > 1) {  // pow(w, 2) in the reference: w * w
            double w1 = w;
            for (int q = 1; q < s.wpow; q++) w *= w1;
        }
        if (s.ylm_on) {
            zd y = ylm_reduced(s.ylm_l, s.ylm_m, rec[s.los_off], rec[s.los_off + 1], rec[s.los_off + 2]);
            if (s.ylm_conj) y.y = -y.y;
            wr = y.x * w;
            wi = y.y * w;
        } else {
            wr = w;
            wi = 0.0;
        }
    }
    wr *= s.scale;
    wi *= s.scale;
}

__device__ __forceinline__ void load_particle(const PartSrc &s, long long p, double pos[3], double &wr, double &wi) {
    load_pos(s, p, pos);
    load_weight(s, p, wr, wi);
}

template <typename T>
struct PRec {
    int i[3];
    T d[3];
    T wr, wi;
};

// A stencil is separable when its cells follow axis by axis: on a periodic mesh (each axis
// wraps on its own), or when every point lies inside a non-periodic mesh.  Otherwise the
// reference's flat-index rule couples the axes (a point at iz = -1 lands in row iy - 1).
__device__ __forceinline__ bool stencil_separable(const AssignGeom &g, const int anc[3]) {
    if (g.periodic) return true;
    const int W = stencil_width(g.scheme), s0 = stencil_start(g.scheme);
    bool in = true;
    for (int a = 0; a < 3; a++) in &= (anc[a] + s0 >= 0) && (anc[a] + s0 + W - 1 < g.n[a]);
    return in;
}

// Cell index along axis a of stencil index i in a separable stencil.
__device__ __forceinline__ int axis_cell(const AssignGeom &g, int a, int i) {
    return g.periodic ? wrap_cell(i, g.n[a]) : i;
}

// The distinct tiles a particle's stencil touches.  Separable stencils keep, per axis, the
// tiles of the first and last point (the tile extent is at least the stencil width unless
// the axis holds a single tile, so a run of W cells, wrapped or not, meets at most two
// tiles); the q-th tile is a mixed-radix index over the three axes, in registers.  Other
// stencils (non-periodic, straddling the mesh edge: a few per cent of particles) list
// their tiles by deduplicating the effective cells of every point.
struct TileList {
    int f[3], l[3], c[3];  // first / last tile per axis, and how many (1 or 2)
    int n;
    bool sep;
};

// Tile of cell c (>= 0) along axis a: a shift for power-of-two tiles (the usual case), which
// spares the binning passes six integer divisions per particle.
__device__ __forceinline__ int tile_axis(const AssignGeom &g, int a, int c) {
    return g.tsh[a] >= 0 ? (c >> g.tsh[a]) : c / g.t[a];
}

__device__ __forceinline__ int tile_of(const AssignGeom &g, int cx, int cy, int cz) {
    return (tile_axis(g, 0, cx) * g.nt[1] + tile_axis(g, 1, cy)) * g.nt[2] + tile_axis(g, 2, cz);
}

__device__ __forceinline__ void tile_list(const AssignGeom &g, const int anc[3], TileList &tl, int *slow) {
    const int W = stencil_width(g.scheme), s0 = stencil_start(g.scheme);
    tl.sep = stencil_separable(g, anc);
    if (tl.sep) {
        for (int a = 0; a < 3; a++) {
            tl.f[a] = tile_axis(g, a, axis_cell(g, a, anc[a] + s0));
            tl.l[a] = tile_axis(g, a, axis_cell(g, a, anc[a] + s0 + W - 1));
            tl.c[a] = (tl.f[a] != tl.l[a]) ? 2 : 1;
        }
        tl.n = tl.c[0] * tl.c[1] * tl.c[2];
        return;
    }
    int nt = 0;
    for (int a = 0; a < W; a++)
        for (int b = 0; b < W; b++)
            for (int c = 0; c < W; c++) {
                int cx, cy, cz;
                if (!effective_cell(g, anc[0] + s0 + a, anc[1] + s0 + b, anc[2] + s0 + c, cx, cy, cz)) continue;
                int t = tile_of(g, cx, cy, cz);
                bool seen = false;
                for (int q = 0; q < nt; q++) seen |= (slow[q] == t);
                if (!seen) slow[nt++] = t;
            }
    tl.n = nt;
}

__device__ __forceinline__ int tile_at(const AssignGeom &g, const TileList &tl, const int *slow, int q) {
    if (!tl.sep) return slow[q];
    // q as a mixed-radix number over the axes' tile counts (each 1 or 2): bits, no division
    const int sz = tl.c[2] - 1, sy = tl.c[1] - 1;
    const int qc = q & sz, qb = (q >> sz) & sy, qa = q >> (sz + sy);
    const int tx = qa ? tl.l[0] : tl.f[0], ty = qb ? tl.l[1] : tl.f[1], tz = qc ? tl.l[2] : tl.f[2];
    return (tx * g.nt[1] + ty) * g.nt[2] + tz;
}

// Most stencil points a non-separable stencil can have (non-periodic meshes: NGP, CIC, TSC).
#define HG_SLOW_TILES 27


__device__ __forceinline__ double warp_sum_d(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Records that keep the particle instead of its weight, so that one binning serves every
// weighting of the same catalogues (the survey's Yhat_lm-weighted fields): the weight is
// evaluated in the accumulation from the particle's own record.
template <typename T>
struct PRecS {
    int i[3];
    int src;  // which source (0 data, 1 randoms)
    T d[3];
    int p;    // particle index within its source
};

// Record makers for the scatter: weight-carrying records (the box), or particle-index
// records (the survey catalogues, srcid 0 data / 1 randoms).
template <typename T>
struct RecWeight {
    using R = PRec<T>;
    __device__ __forceinline__ R make(const PartSrc &s, long long p, const int anc[3], const double d[3]) const {
        R r;
        double wr, wi;
        load_weight(s, p, wr, wi);
        for (int a = 0; a < 3; a++) {
            r.i[a] = anc[a];
            r.d[a] = (T)d[a];
        }
        r.wr = (T)wr;
        r.wi = (T)wi;
        return r;
    }
};
template <typename T>
struct RecIndex {
    using R = PRecS<T>;
    int srcid;
    __device__ __forceinline__ R make(const PartSrc &, long long p, const int anc[3], const double d[3]) const {
        R r;
        for (int a = 0; a < 3; a++) {
            r.i[a] = anc[a];
            r.d[a] = (T)d[a];
        }
        r.src = srcid;
        r.p = (int)p;
        return r;
    }
};

// Particles whose stencil straddles a non-periodic mesh edge (the reference's flat-index
// rule couples the axes there) take a longer path: deduplicated effective cells, and an
// in-bounds mass point by point.  A warp that met one such lane would idle its other lanes
// for that path, and a catalogue stored in spatial order has some in most warps that touch
// a face; so the main passes hand those particles to a list (Defer) and a second launch
// of the same kernel runs them with every lane on the long path.
struct Defer {
    int *list;          // particle indices, capacity n
    unsigned *count;    // device counter
    int pass;           // 0: main pass (append), 1: the deferred pass (read the list)
    unsigned *bad;      // main pass: counts particles with a non-finite position, weight or line
                        // of sight; they get no tiles and no records (the host rejects the
                        // catalogue when the count is not zero)
    unsigned *neg;      // main pass: set to 1 when some particle has a negative coordinate; the
                        // reference's int() truncates toward zero there, so a CIC or TSC stencil
                        // weight can reach 2 per axis instead of at most 1 (the fixed-point
                        // accumulation then takes 3 more bits of headroom)
};

// A particle whose scaled coordinate n x / L lies 2^30 cells or more from the mesh origin on
// some axis (far outside the box, where the reference's int anchors overflow): on a
// non-periodic mesh it lands in no cell and is dropped (returns true); on a periodic mesh
// (PCS, interlacing) that coordinate is first reduced into [0, L].  Within 2^30 cells every
// anchor and stencil index of the assignment is exact in int.
__device__ __forceinline__ bool far_reduce(const AssignGeom &g, double pos[3]) {
    bool drop = false;
    for (int a = 0; a < 3; a++) {
        if (fabs(pos[a]) < g.far[a]) continue;  // (the threshold's rounding is immaterial at 2^30 cells)
        // separately rounded operations (no fused multiply-add): x - L floor(x / L)
        if (g.periodic) pos[a] = __dsub_rn(pos[a], __dmul_rn(g.L[a], floor(__ddiv_rn(pos[a], g.L[a]))));
        else drop = true;
    }
    return drop;
}

// Position, weight (when the source has one) and line of sight (when it has one) all finite.
// The count and scatter passes apply the same test, so a skipped particle has no records.
__device__ __forceinline__ bool particle_finite(const PartSrc &s, long long p, const double pos[3]) {
    bool ok = isfinite(pos[0]) && isfinite(pos[1]) && isfinite(pos[2]);
    const double *rec = reinterpret_cast<const double *>(s.base + p * s.stride);
    if (s.w_off >= 0) ok = ok && isfinite(rec[s.w_off]);
    if (s.los_off >= 0) ok = ok && isfinite(rec[s.los_off]) && isfinite(rec[s.los_off + 1]) && isfinite(rec[s.los_off + 2]);
    return ok;
}

// Lanes of a warp with `want` set append their particle index to the list.
__device__ __forceinline__ void defer_push(const Defer &df, bool want, long long p) {
    const unsigned m = __ballot_sync(0xffffffffu, want);
    if (!m) return;
    const int lane = threadIdx.x & 31;
    unsigned base = 0;
    if (lane == __ffs(m) - 1) base = atomicAdd(df.count, (unsigned)__popc(m));
    base = __shfl_sync(0xffffffffu, base, __ffs(m) - 1);
    if (want) df.list[base + __popc(m & ((1u << lane) - 1u))] = (int)p;
}

// Pass 1: tile counts + (when mass != null) the FP64 in-bounds mass
// sum_p w_p factor prod(w_axis)  (the field's exact integral, needed for the k = 0 mode
// since boundary drops lose mass).  Clustered catalogues put many lanes of a warp on the
// same tile, so the count is warp-aggregated.  Whole warps stride over the catalogue (the
// main pass) or the deferred list.  The mass is summed in the main pass only, for every
// particle (those deferred for their tiles included), and each block writes its sum to
// mass[2 blockIdx.x] (+1 for the imaginary part): fixed blocks over fixed particles, added
// on the host in block order, so the integral does not depend on scheduling.
__global__ void __launch_bounds__(256, 3) k_bin_count(PartSrc src, AssignGeom g, Defer df, unsigned int *cnt,
                                                      double *mass) {
    __shared__ double red[2][32];
    double m_re = 0.0, m_im = 0.0;
    const int lane = threadIdx.x & 31;
    const long long wstride = (long long)gridDim.x * blockDim.x;
    const long long total = df.pass ? (long long)*df.count : src.n;
    for (long long wbase = (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31); wbase < total;
         wbase += wstride) {
        const long long i = wbase + lane;
        long long p = (i < total) ? (df.pass ? (long long)df.list[i] : i) : -1;
        TileList tl;
        int slow[HG_SLOW_TILES];
        tl.n = 0;
        bool push = false;
        double pos[3];
        if (p >= 0) load_pos(src, p, pos);
        if (p >= 0 && !df.pass && !particle_finite(src, p, pos)) {
            atomicAdd(df.bad, 1u);
            p = -1;
        }
        if (p >= 0 && far_reduce(g, pos)) p = -1;
        if (!df.pass) {  // warp-uniform point: every lane of the warp is here
            const bool negc = p >= 0 && (pos[0] < 0.0 || pos[1] < 0.0 || pos[2] < 0.0);
            if (__any_sync(0xffffffffu, negc) && lane == 0) atomicOr(df.neg, 1u);
        }
        if (p >= 0) {
            double wr = 0.0, wi = 0.0;
            if (mass) load_weight(src, p, wr, wi);
            int anc[3];
            double d[3];
            for (int a = 0; a < 3; a++) anchor(pos[a], g.n[a], g.L[a], g.scheme, g.shift, anc[a], d[a]);
            if (!df.pass && !stencil_separable(g, anc)) {
                push = true;
                if (mass) {  // its in-bounds mass point by point, here (the deferred pass sums none)
                    const int W = stencil_width(g.scheme), s0 = stencil_start(g.scheme);
                    for (int q = 0; q < W * W * W; q++) {
                        const int a = q / (W * W), b = (q / W) % W, c = q % W;
                        int cx, cy, cz;
                        if (!effective_cell(g, anc[0] + s0 + a, anc[1] + s0 + b, anc[2] + s0 + c, cx, cy, cz)) continue;
                        const double wa = axis_weight_at<double>(g.scheme, d[0], a),
                                     wb = axis_weight_at<double>(g.scheme, d[1], b),
                                     wc = axis_weight_at<double>(g.scheme, d[2], c);
                        m_re += wr * g.factor * wa * wb * wc;
                        m_im += wi * g.factor * wa * wb * wc;
                    }
                }
            } else {
                tile_list(g, anc, tl, slow);
                if (!mass || df.pass) {
                } else if (tl.sep) {
                    // every stencil point lands: the weights sum to one per axis
                    m_re += wr * g.factor;
                    m_im += wi * g.factor;
                } else {
                    // in-bounds mass in the reference's product order
                    const int W = stencil_width(g.scheme), s0 = stencil_start(g.scheme);
                    for (int q = 0; q < W * W * W; q++) {
                        const int a = q / (W * W), b = (q / W) % W, c = q % W;
                        int cx, cy, cz;
                        if (!effective_cell(g, anc[0] + s0 + a, anc[1] + s0 + b, anc[2] + s0 + c, cx, cy, cz)) continue;
                        const double wa = axis_weight_at<double>(g.scheme, d[0], a),
                                     wb = axis_weight_at<double>(g.scheme, d[1], b),
                                     wc = axis_weight_at<double>(g.scheme, d[2], c);
                        m_re += wr * g.factor * wa * wb * wc;
                        m_im += wi * g.factor * wa * wb * wc;
                    }
                }
            }
        }
        if (!df.pass) defer_push(df, push, p);
        const int maxnt = __reduce_max_sync(0xffffffffu, tl.n);
        for (int q = 0; q < maxnt; q++) {
            const int t = (q < tl.n) ? tile_at(g, tl, slow, q) : -1;
            const unsigned grp = __match_any_sync(0xffffffffu, t);
            if (t >= 0 && lane == __ffs(grp) - 1) atomicAdd(&cnt[t], (unsigned)__popc(grp));
        }
    }
    if (!mass || df.pass) return;
    m_re = warp_sum_d(m_re);
    m_im = warp_sum_d(m_im);
    if (lane == 0) {
        red[0][threadIdx.x >> 5] = m_re;
        red[1][threadIdx.x >> 5] = m_im;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double sr = 0.0, si = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
            sr += red[0][w];
            si += red[1][w];
        }
        mass[2 * blockIdx.x] = sr;
        mass[2 * blockIdx.x + 1] = si;
    }
}

// Pass 3: one record per (particle, tile).  The main pass fills each tile's range from the
// front (cursor) and skips the deferred particles; the deferred pass fills it from the back
// (cursor_back), so the records of stencils that straddle a mesh edge sit together at the
// end of their tile's range and the accumulation's warps take one path or the other.
template <class MK>
__global__ void __launch_bounds__(256, 3) k_bin_scatter(PartSrc src, AssignGeom g, MK mk, Defer df, const unsigned int *off,
                              unsigned int *cursor, unsigned int *cursor_back, typename MK::R *rec) {
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const long long wstride = (long long)gridDim.x * blockDim.x;
    const long long total = df.pass ? (long long)*df.count : src.n;
    for (long long wbase = (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31); wbase < total;
         wbase += wstride) {
        const long long i = wbase + lane;
        long long p = (i < total) ? (df.pass ? (long long)df.list[i] : i) : -1;
        TileList tl;
        int slow[HG_SLOW_TILES];
        tl.n = 0;
        typename MK::R r;
        double pos[3];
        if (p >= 0) load_pos(src, p, pos);
        if (p >= 0 && !df.pass && !particle_finite(src, p, pos)) p = -1;
        if (p >= 0 && far_reduce(g, pos)) p = -1;
        if (p >= 0) {
            int anc[3];
            double d[3];
            for (int a = 0; a < 3; a++) anchor(pos[a], g.n[a], g.L[a], g.scheme, g.shift, anc[a], d[a]);
            if (df.pass || stencil_separable(g, anc)) {
                tile_list(g, anc, tl, slow);
                r = mk.make(src, p, anc, d);
            }
        }
        const int maxnt = __reduce_max_sync(0xffffffffu, tl.n);
        if (!df.pass) {
            // separable stencils meet at most 8 tiles: every counter atomic of the warp is
            // issued before any result is used, so their round trips overlap
            // (and each tile's range start is read alongside, not after the atomic's return)
            int tq[8];
            unsigned gq[8], bq[8], oq[8];
#pragma unroll
            for (int q = 0; q < 8; q++) {
                tq[q] = -1;
                gq[q] = 0u;
                bq[q] = 0u;
                oq[q] = 0u;
                if (q < maxnt) {
                    tq[q] = (q < tl.n) ? tile_at(g, tl, slow, q) : -1;
                    gq[q] = __match_any_sync(0xffffffffu, tq[q]);
                    if (tq[q] >= 0) oq[q] = __ldg(off + tq[q]);
                    if (tq[q] >= 0 && lane == __ffs(gq[q]) - 1) bq[q] = atomicAdd(&cursor[tq[q]], (unsigned)__popc(gq[q]));
                }
            }
#pragma unroll
            for (int q = 0; q < 8; q++) {
                if (q < maxnt && tq[q] >= 0) {
                    const unsigned base = __shfl_sync(gq[q], bq[q], __ffs(gq[q]) - 1);
                    const unsigned ri = oq[q] + base + __popc(gq[q] & lt);
                    if (HG_IN_BOUNDS(ri < off[tq[q] + 1], HG_SITE_RECORD, ri)) rec[ri] = r;
                }
            }
            continue;
        }
        for (int q = 0; q < maxnt; q++) {
            const int t = (q < tl.n) ? tile_at(g, tl, slow, q) : -1;
            const unsigned grp = __match_any_sync(0xffffffffu, t);
            if (t >= 0) {
                const int leader = __ffs(grp) - 1;
                unsigned base = 0;
                if (lane == leader) base = atomicAdd(&cursor_back[t], (unsigned)__popc(grp));
                base = __shfl_sync(grp, base, leader);
                const unsigned ri = off[t + 1] - 1u - (base + __popc(grp & lt));
                if (HG_IN_BOUNDS(ri >= off[t] && ri < off[t + 1], HG_SITE_RECORD, ri)) rec[ri] = r;
            }
        }
    }
}

// The complex weight of every particle of a source before its scale (load_weight with
// scale 1), in catalogue order: the accumulation then gathers 16 bytes per record instead of
// the particle's weight and line of sight, and evaluates no Yhat_lm.
__global__ void k_make_cw(PartSrc src, double2 *cw) {
    src.scale = 1.0;
    src.cw = nullptr;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < src.n; p += (long long)gridDim.x * blockDim.x) {
        double wr, wi;
        load_weight(src, p, wr, wi);
        cw[p] = make_double2(wr, wi);
    }
}

// max |w| over a catalogue (1 when it has no weights): block partials, maximum on the host
__global__ void k_max_weight(PartSrc src, double *part) {
    __shared__ double red[32];
    double m = 0.0;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < src.n; p += (long long)gridDim.x * blockDim.x) {
        const double *rec = reinterpret_cast<const double *>(src.base + p * src.stride);
        m = fmax(m, (src.w_off >= 0) ? fabs(rec[src.w_off]) : 1.0);
    }
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double v = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) v = fmax(v, red[w]);
        part[blockIdx.x] = v;
    }
}

// Per-particle FP64 sums  out[q] = sum_p scale w_p^pw[q] Yhat_{l_q m_q}(los_p)  (complex), as
// block partials part[block][q] summed on the host in block order (deterministic):
// sum w (particle.hpp:336-352), sum w^2 (particle.hpp:255-258), and the shot-noise sums
// sum w^2 Yhat_LM (field.hpp:1164-1185).
#define HG_PSUM_MAX 16
struct PSumSpec {
    int n;
    int pw[HG_PSUM_MAX];
    int l[HG_PSUM_MAX], m[HG_PSUM_MAX];  // l < 0: no harmonic (weight only)
};
__global__ void k_particle_sums(PartSrc src, PSumSpec q, double *part) {
    __shared__ double red[HG_PSUM_MAX][2][32];
    double acc[HG_PSUM_MAX][2];
    for (int j = 0; j < HG_PSUM_MAX; j++) acc[j][0] = acc[j][1] = 0.0;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < src.n;
         p += (long long)gridDim.x * blockDim.x) {
        const double *rec = reinterpret_cast<const double *>(src.base + p * src.stride);
        const double w = (src.w_off >= 0) ? rec[src.w_off] : 1.0;
        for (int j = 0; j < q.n; j++) {
            double wp = w;
            for (int e = 1; e < q.pw[j]; e++) wp *= w;
            if (q.l[j] < 0) {
                acc[j][0] += wp;
            } else {
                zd y = ylm_reduced(q.l[j], q.m[j], rec[src.los_off], rec[src.los_off + 1], rec[src.los_off + 2]);
                acc[j][0] += wp * y.x;
                acc[j][1] += wp * y.y;
            }
        }
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int j = 0; j < q.n; j++)
        for (int c = 0; c < 2; c++) {
            double v = warp_sum_d(acc[j][c]);
            if (lane == 0) red[j][c][wid] = v;
        }
    __syncthreads();
    if (threadIdx.x < 2 * q.n) {
        const int j = threadIdx.x >> 1, c = threadIdx.x & 1;
        double v = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) v += red[j][c][w];
        part[(long long)blockIdx.x * 2 * HG_PSUM_MAX + 2 * j + c] = v * src.scale;
    }
}

// sum_c m[c]^2 per block (FP64), for V_survey = (sum w_R)^2 / (sum_c rho_R^2 dV) (field.hpp:449-503)
__global__ void k_sum_squares(const double *m, long long n, double *part) {
    __shared__ double red[32];
    double a = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        a += m[i] * m[i];
    a = warp_sum_d(a);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
        double v = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) v += red[w];
        part[blockIdx.x] = v;
    }
}

// Work item of the accumulation: records [r0, r1) of tile `tile`; `multi` when the tile's
// records are split over several chunks (a clustered tile), in which case the tile is
// zeroed first and every chunk adds its partial tile.
struct Chunk {
    int tile;
    unsigned r0, r1;
    int multi;  // 0: sole chunk; 1: first chunk of a split tile; 2: later chunk of a split tile
    unsigned tile_n;  // records of the whole tile
    int slot;         // split tiles: their slot in the integer staging buffer (crowd), else -1
};

__global__ void k_chunk_count(const unsigned int *cnt, int ntiles, unsigned chunk, unsigned int *nch) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t > ntiles) return;
    nch[t] = (t == ntiles) ? 0u : max(1u, (cnt[t] + chunk - 1) / chunk);
}

// nslots: a counter (zeroed by the host) that hands every split tile its staging slot
__global__ void k_chunk_fill(const unsigned int *off, const unsigned int *choff, int ntiles, unsigned chunk, Chunk *ch,
                             unsigned *nslots = nullptr) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntiles) return;
    unsigned b = off[t], e = off[t + 1];
    unsigned n = choff[t + 1] - choff[t];
    const int slot = (n > 1 && nslots) ? (int)atomicAdd(nslots, 1u) : -1;
    for (unsigned c = 0; c < n; c++) {
        Chunk k;
        k.tile = t;
        k.r0 = b + c * chunk;
        k.r1 = min(e, b + (c + 1) * chunk);
        k.multi = (n == 1) ? 0 : (c == 0 ? 1 : 2);
        k.tile_n = e - b;
        k.slot = slot;
        ch[choff[t] + c] = k;
    }
}

// Visit a tile's cells row by row: warp w takes rows w, w + nwarps, ...; a row is t2
// consecutive cells of the mesh, so a warp's stores are contiguous.  f(li, cell) with li
// the cell's index in the tile, (lx t1 + ly) t2 + lz.
template <class F>
__device__ __forceinline__ void for_tile_cells(const AssignGeom &g, int tile, F f) {
    const int tz = tile % g.nt[2];
    const int ty = (tile / g.nt[2]) % g.nt[1];
    const int tx = tile / (g.nt[2] * g.nt[1]);
    const int nw = blockDim.x >> 5, lane = threadIdx.x & 31;
    const int rows = g.t[0] * g.t[1];
    for (int r = threadIdx.x >> 5; r < rows; r += nw) {
        const int lx = r / g.t[1], ly = r - lx * g.t[1];
        const long long base =
            ((long long)(tx * g.t[0] + lx) * g.n[1] + (ty * g.t[1] + ly)) * g.n[2] + tz * g.t[2];
        for (int lz = lane; lz < g.t[2]; lz += 32)
            if (HG_IN_BOUNDS(base + lz >= 0 && base + lz < g.ntot, HG_SITE_MESH_CELL, base + lz)) f(r * g.t[2] + lz, base + lz);
    }
}

// Zero `words` 32-bit words of shared memory (16-byte stores for the bulk).
__device__ __forceinline__ void zero_shared(void *p, int words) {
    int4 *q = reinterpret_cast<int4 *>(p);
    for (int c = threadIdx.x; c < (words >> 2); c += blockDim.x) q[c] = make_int4(0, 0, 0, 0);
    int *w = reinterpret_cast<int *>(p);
    for (int c = (words & ~3) + threadIdx.x; c < words; c += blockDim.x) w[c] = 0;
}

// Zero the cells of every split tile (run before the accumulation), or with crowd != null
// its slot of the integer staging buffer (crowd_words 64-bit words per cell).
template <typename T, bool CPLX>
__global__ void k_zero_split_tiles(const Chunk *ch, AssignGeom g, T *mesh_re, T *mesh_im,
                                   unsigned long long *crowd = nullptr, int crowd_words = 0) {
    Chunk k = ch[blockIdx.x];
    if (k.multi != 1) return;
    if (crowd) {
        const int tcells = g.t[0] * g.t[1] * g.t[2];
        unsigned long long *c = crowd + (size_t)k.slot * tcells * crowd_words;
        for (int i = threadIdx.x; i < tcells * crowd_words; i += blockDim.x) c[i] = 0ull;
        return;
    }
    for_tile_cells(g, k.tile, [&](int, long long cell) {
        mesh_re[cell] = (T)0;
        if (CPLX) mesh_im[cell] = (T)0;
    });
}

// Fixed-point scale of a tile: 2^sc with sc from the tile's record count, the same for every
// chunk of a split tile, so their integer partial sums add exactly.  FP32 (two 32-bit
// words): tile records x bound x 2^sc < 2^50 and bound x 2^sc < 2^42; FP64 (three words):
// tile records x bound x 2^sc <= 2^69.
template <typename T>
__device__ __forceinline__ int fix_exponent(const AssignGeom &g, unsigned tile_n) {
    if (sizeof(T) == 8) {
        int e;
        frexp(double(max(tile_n, 1u)) * (double)g.fix_bound, &e);
        return 69 - e;
    }
    int e, e1;
    frexpf(float(max(tile_n, 1u)) * g.fix_bound, &e);
    frexpf(g.fix_bound, &e1);
    return min(50 - e, 42 - e1);  // the host keeps fix_bound >= 2^-60, so sc <= 102
}

// Split tiles of a fixed-point accumulation: the integer sums their chunks added to the
// staging slot, rounded once to the mesh's type and written (one CTA per split tile).
template <typename T>
__global__ void k_crowd_writeout(const Chunk *ch, AssignGeom g, const unsigned long long *crowd, T *mesh) {
    const Chunk k = ch[blockIdx.x];
    if (k.multi != 1) return;
    const int tcells = g.t[0] * g.t[1] * g.t[2];
    const double inv = ldexp(1.0, -fix_exponent<T>(g, k.tile_n));
    for_tile_cells(g, k.tile, [&](int li, long long cell) {
        if (sizeof(T) == 8) {
            const unsigned long long *c = crowd + (size_t)k.slot * tcells * 2;
            const double hi = (double)(long long)c[li] * 0x1p40;
            mesh[cell] = (T)(__dadd_rn(hi, (double)(long long)c[tcells + li]) * inv);
        } else {
            const unsigned long long *c = crowd + (size_t)k.slot * tcells;
            mesh[cell] = (T)(__ll2float_rn((long long)c[li]) * (float)inv);
        }
    });
}

// Local tile coordinates of a separable stencil along axis a: bit j of the result is set
// when point j (index i0 + j) lies in this CTA's tile, at local index loc[j].
__device__ __forceinline__ unsigned axis_local(const AssignGeom &g, int a, int i0, int o, int W, int loc[4]) {
    unsigned m = 0;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        loc[j] = 0;
        if (j < W) {
            const int l = axis_cell(g, a, i0 + j) - o;
            if ((unsigned)l < (unsigned)g.t[a]) {
                loc[j] = l;
                m |= 1u << j;
            }
        }
    }
    return m;
}

// One CTA per chunk.  The mesh stores the density rho = sum_p w_p (1/dV) prod(w_axis)
// like the reference (the FP32 form: the mass rho dV), in T.
//
// Accumulator.  FIX = false: a shared-memory tile of T with T atomics.  FIX = true (FP32
// real meshes of sources whose per-record weight |w acc_factor| is bounded by
// g.fix_bound, which the host knows for unweighted catalogues): an exact fixed-point sum
// in two 32-bit integer words per cell.  Integer shared-memory atomics run about five
// times faster than FP32 ones on this part (which emulates the latter), and the
// accumulation is bound by them.  Per chunk every stencil weight (an FP32 product) is
// scaled by S = 2^s, exactly, with (records) x fix_bound x S < 2^50 and
// fix_bound x S < 2^42, and split as x = hi 2^20 + lo with hi = round(x / 2^20) and
// |lo| <= 2^19; both parts are formed exactly with FP32 adds against 1.5 x 2^23 (valid
// below 2^22), and lo is rounded to an integer there, the only rounding (below 2^-50 of
// the chunk's bound).  A cell receives at most one add per record (the stencil's points
// are distinct cells when every axis has at least W cells), so |sum hi| < 2^30 + records
// and |sum lo| <= records 2^19 <= 2^30: neither word overflows, the sum is exact and
// independent of the order of the atomics, and it is rounded once, to the mesh's FP32.
//
// Separable stencils (every point inside the mesh, or a periodic mesh) compute their local
// coordinates axis by axis; the few that straddle a non-periodic mesh edge take the
// reference's flat-index rule point by point.
// x = hi 2^20 + lo exactly for |x| < 2^42, hi = round(x / 2^20), lo = round(x - hi 2^20):
// 1.5 x 2^23 + y (|y| < 2^22) is a float of unit spacing whose low bits hold round(y).
__device__ __forceinline__ void fix_split(float x, int &hi, int &lo) {
    const float t = __fmaf_rn(x, 0x1p-20f, 12582912.0f);
    hi = __float_as_int(t) - 0x4B400000;
    const float r = __fmaf_rn(-(t - 12582912.0f), 0x1p20f, x);
    lo = __float_as_int(__fadd_rn(r, 12582912.0f)) - 0x4B400000;
}

// FIX with T = double (real FP64 meshes of weight-bounded sources): three 32-bit integer
// words per cell (64-bit shared-memory atomics measured no faster than FP64 ones here, the
// 32-bit ones are native).  Per chunk every stencil weight (an FP64 product) is scaled by
// S = 2^s, exactly, with (records) x fix_bound x S <= 2^69, and split as
// x = hi 2^40 + mid 2^20 + lo with hi = round(x / 2^40), mid = round((x - hi 2^40) / 2^20);
// both differences are exact, and lo = round(x - hi 2^40 - mid 2^20) is the only rounding
// (below 2^-70 of the chunk's bound, finer than FP64).  |sum lo|, |sum mid| <= records 2^19
// and |sum hi| <= 2^29 + records stay inside 32 bits, so the sum is exact, independent of the
// order of the atomics, and rounded once to the mesh's FP64.
template <typename T, bool CPLX, bool FIX, int SCHEME>
__global__ void k_tile_accum(const PRec<T> *rec, const Chunk *ch, AssignGeom g, T *mesh_re, T *mesh_im,
                             unsigned long long *crowd = nullptr) {
    static_assert(!FIX || !CPLX, "fixed-point accumulation is for real meshes");
    constexpr bool FIX64 = FIX && sizeof(T) == 8;
    constexpr int W = SCHEME + 1, s0 = (SCHEME >= 2) ? -1 : 0;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *acc = reinterpret_cast<T *>(smem_raw);
    const int tcells = g.t[0] * g.t[1] * g.t[2];
    T *acc_im = acc + tcells;
    int *acc_hi = reinterpret_cast<int *>(smem_raw);
    int *acc_lo = acc_hi + tcells;
    int *acc_w3 = reinterpret_cast<int *>(smem_raw);  // FIX64: hi, mid, lo words
    zero_shared(smem_raw, FIX64 ? 3 * tcells : tcells * ((CPLX || FIX) ? 2 : 1) * (int)(sizeof(T) / 4));
    __syncthreads();
    const Chunk k = ch[blockIdx.x];
    const int tile = k.tile;
    const int tz = tile % g.nt[2];
    const int ty = (tile / g.nt[2]) % g.nt[1];
    const int tx = tile / (g.nt[2] * g.nt[1]);
    const int ox = tx * g.t[0], oy = ty * g.t[1], oz = tz * g.t[2];
    float fscale = 1.0f, finv = 1.0f;
    double dscale = 1.0, dinv = 1.0;
    if (FIX) {  // one scale for the whole tile (all its chunks)
        const int sc = fix_exponent<T>(g, k.tile_n);
        dscale = ldexp(1.0, sc);
        dinv = ldexp(1.0, -sc);
        fscale = ldexpf(1.0f, sc);
        finv = ldexpf(1.0f, -sc);
    }
    const T factor = (T)g.acc_factor;
    auto add = [&](int li, T v, T vi) {
        if (!HG_IN_BOUNDS(li >= 0 && li < tcells, HG_SITE_TILE_CELL, li)) return;
        if (FIX64) {
            // (rounding by adding 1.5 2^52 and taking the low word, without conversion
            // instructions, was measured slower: 1.71 -> 1.85 ms per 512^3 mock)
            const double x = (double)v;
            const double hi = rint(x * 0x1p-40);
            const double r1 = x - hi * 0x1p40;  // exact
            const double mid = rint(r1 * 0x1p-20);
            const double r2 = r1 - mid * 0x1p20;  // exact
            atomicAdd(&acc_w3[li], (int)hi);
            atomicAdd(&acc_w3[tcells + li], (int)mid);
            atomicAdd(&acc_w3[2 * tcells + li], __double2int_rn(r2));
        } else if (FIX) {
            int hi, lo;
            fix_split((float)v, hi, lo);
            atomicAdd(&acc_hi[li], hi);
            atomicAdd(&acc_lo[li], lo);
        } else {
            atomicAdd(&acc[li], v);
            if (CPLX) atomicAdd(&acc_im[li], vi);
        }
    };
    for (unsigned r = k.r0 + threadIdx.x; r < k.r1; r += blockDim.x) {
        const PRec<T> pr = rec[r];
        T wr = pr.wr * factor, wi = pr.wi * factor;
        if (FIX64) wr = (T)((double)wr * dscale);
        else if (FIX) wr *= (T)fscale;
        const int anc[3] = {pr.i[0], pr.i[1], pr.i[2]};
        if (stencil_separable(g, anc)) {
            T w[3][W];
            int lx[4], ly[4], lz[4];
#pragma unroll
            for (int a = 0; a < 3; a++)
#pragma unroll
                for (int j = 0; j < W; j++) w[a][j] = axis_weight_at<T>(SCHEME, pr.d[a], j);
            const unsigned mx = axis_local(g, 0, anc[0] + s0, ox, W, lx);
            const unsigned my = axis_local(g, 1, anc[1] + s0, oy, W, ly);
            const unsigned mz = axis_local(g, 2, anc[2] + s0, oz, W, lz);
#pragma unroll
            for (int a = 0; a < W; a++) {
                if (!((mx >> a) & 1u)) continue;
                const T wa = wr * w[0][a], wia = wi * w[0][a];
#pragma unroll
                for (int b = 0; b < W; b++) {
                    if (!((my >> b) & 1u)) continue;
                    const T wab = wa * w[1][b], wiab = wia * w[1][b];
                    const int lab = (lx[a] * g.t[1] + ly[b]) * g.t[2];
#pragma unroll
                    for (int c = 0; c < W; c++) {
                        if (!((mz >> c) & 1u)) continue;
                        add(lab + lz[c], wab * w[2][c], wiab * w[2][c]);
                    }
                }
            }
            continue;
        }
        // a stencil straddling a non-periodic mesh edge (the scatter put these records at the
        // end of the tile's range): point by point, the reference's flat-index rule, weights
        // evaluated per point (no arrays)
#pragma unroll 1
        for (int p = 0; p < W * W * W; p++) {
            const int a = p / (W * W), b = (p / W) % W, c = p % W;
            int cx, cy, cz;
            if (!effective_cell(g, anc[0] + s0 + a, anc[1] + s0 + b, anc[2] + s0 + c, cx, cy, cz)) continue;
            const int lx = cx - ox, ly = cy - oy, lz = cz - oz;
            if ((unsigned)lx >= (unsigned)g.t[0] || (unsigned)ly >= (unsigned)g.t[1] || (unsigned)lz >= (unsigned)g.t[2])
                continue;
            const T wa = axis_weight_at<T>(SCHEME, pr.d[0], a), wb = axis_weight_at<T>(SCHEME, pr.d[1], b),
                    wc = axis_weight_at<T>(SCHEME, pr.d[2], c);
            add((lx * g.t[1] + ly) * g.t[2] + lz, wr * wa * wb * wc, wi * wa * wb * wc);
        }
    }
    __syncthreads();
    if (FIX && k.multi != 0 && crowd) {  // a split tile: this chunk's exact partial sums, added as integers
        for (int li = threadIdx.x; li < tcells; li += blockDim.x) {
            if (FIX64) {
                unsigned long long *c = crowd + (size_t)k.slot * tcells * 2;
                const long long hi = acc_w3[li];
                const long long ml = (long long)acc_w3[tcells + li] * 1048576LL + (long long)acc_w3[2 * tcells + li];
                if (hi) atomicAdd(&c[li], (unsigned long long)hi);
                if (ml) atomicAdd(&c[tcells + li], (unsigned long long)ml);
            } else {
                unsigned long long *c = crowd + (size_t)k.slot * tcells;
                const long long v = (long long)acc_hi[li] * 1048576LL + (long long)acc_lo[li];
                if (v) atomicAdd(&c[li], (unsigned long long)v);
            }
        }
        return;
    }
    // FIX: the exact integer sum rounded once to FP32, then scaled by a power of two (exact)
    for_tile_cells(g, tile, [&](int li, long long cell) {
        const T v = FIX64 ? (T)(__dadd_rn((double)acc_w3[li] * 0x1p40,
                                          (double)((long long)acc_w3[tcells + li] * 1048576LL +
                                                   (long long)acc_w3[2 * tcells + li])) * dinv)
                    : FIX ? (T)(__ll2float_rn((long long)acc_hi[li] * 1048576LL + (long long)acc_lo[li]) * finv)
                          : acc[li];
        if (k.multi == 0) {
            mesh_re[cell] = v;
            if (CPLX) mesh_im[cell] = acc_im[li];
        } else {
            if (v != (T)0) atomicAdd(&mesh_re[cell], v);
            if (CPLX && acc_im[li] != (T)0) atomicAdd(&mesh_im[cell], acc_im[li]);
        }
    });
}

// Weighting of a field: one PartSrc (weight recipe: w^wpow, Yhat_lm(los), scale) per source.
struct FieldW {
    PartSrc s[2];
};

// k_tile_accum on particle-index records: the weight comes from the particle
// (load_weight, the same FP64 expression as the weight-carrying records), and the FP64
// in-bounds mass sum of w factor prod(w_axis) is reduced on the way, for the transform's
// exact k = 0 value.  A separable stencil lands whole, so its mass is w factor (the axis
// weights sum to one), counted by the one record whose tile holds the stencil's first
// point; an edge-straddling stencil (records at the end of the tile's range) adds its
// in-bounds points one by one in the reference's product order.  FIX (FP32 fields whose
// per-record weight is bounded by g.fix_bound: the host takes max |w|^wpow |scale| over the
// catalogues, |Yhat_lm| <= 1): k_tile_accum's exact two-word integer sums, for the real and
// the imaginary part.
template <typename T, bool CPLX, int SCHEME, bool FIX>
__global__ void k_tile_accum_src(const PRecS<T> *rec, const Chunk *ch, AssignGeom g, FieldW fw, T *mesh_re, T *mesh_im,
                                 double *mass) {
    static_assert(!FIX || sizeof(T) == 4, "fixed-point accumulation is for FP32 meshes");
    constexpr int W = SCHEME + 1, s0 = (SCHEME >= 2) ? -1 : 0;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *acc = reinterpret_cast<T *>(smem_raw);
    const int tcells = g.t[0] * g.t[1] * g.t[2];
    T *acc_im = acc + tcells;
    // FIX: (hi, lo) words of the real part, then of the imaginary part (k_tile_accum's scheme)
    int *fx = reinterpret_cast<int *>(smem_raw);
    __shared__ double red[2][32];
    zero_shared(smem_raw, tcells * (CPLX ? 2 : 1) * (FIX ? 2 : 1) * (int)(sizeof(T) / 4));
    __syncthreads();
    const Chunk k = ch[blockIdx.x];
    const int tile = k.tile;
    const int tz = tile % g.nt[2];
    const int ty = (tile / g.nt[2]) % g.nt[1];
    const int tx = tile / (g.nt[2] * g.nt[1]);
    const int ox = tx * g.t[0], oy = ty * g.t[1], oz = tz * g.t[2];
    const T factor = (T)g.acc_factor;
    float fscale = 1.0f, finv = 1.0f;
    if (FIX) {
        int e, e1;
        frexpf(float(k.r1 - k.r0) * g.fix_bound, &e);
        frexpf(g.fix_bound, &e1);
        const int sc = min(50 - e, 42 - e1);  // the host keeps fix_bound >= 2^-60
        fscale = ldexpf(1.0f, sc);
        finv = ldexpf(1.0f, -sc);
    }
    auto add = [&](int li, T v, T vi) {
        if (!HG_IN_BOUNDS(li >= 0 && li < tcells, HG_SITE_TILE_CELL, li)) return;
        if (FIX) {
            int hi, lo;
            fix_split((float)v, hi, lo);
            atomicAdd(&fx[li], hi);
            atomicAdd(&fx[tcells + li], lo);
            if (CPLX) {
                fix_split((float)vi, hi, lo);
                atomicAdd(&fx[2 * tcells + li], hi);
                atomicAdd(&fx[3 * tcells + li], lo);
            }
        } else {
            atomicAdd(&acc[li], v);
            if (CPLX) atomicAdd(&acc_im[li], vi);
        }
    };
    double mr = 0.0, mi = 0.0;
    for (unsigned r = k.r0 + threadIdx.x; r < k.r1; r += blockDim.x) {
        const PRecS<T> pr = rec[r];
        double wr64, wi64;
        load_weight(fw.s[pr.src], pr.p, wr64, wi64);
        T wr = (T)wr64 * factor, wi = (T)wi64 * factor;
        if (FIX) {
            wr *= (T)fscale;
            wi *= (T)fscale;
        }
        const int anc[3] = {pr.i[0], pr.i[1], pr.i[2]};
        if (stencil_separable(g, anc)) {
            T w[3][W];
            int lx[4], ly[4], lz[4];
#pragma unroll
            for (int a = 0; a < 3; a++)
#pragma unroll
                for (int j = 0; j < W; j++) w[a][j] = axis_weight_at<T>(SCHEME, pr.d[a], j);
            const unsigned mx = axis_local(g, 0, anc[0] + s0, ox, W, lx);
            const unsigned my = axis_local(g, 1, anc[1] + s0, oy, W, ly);
            const unsigned mz = axis_local(g, 2, anc[2] + s0, oz, W, lz);
            if (mx & my & mz & 1u) {
                mr += wr64 * g.factor;
                mi += wi64 * g.factor;
            }
#pragma unroll
            for (int a = 0; a < W; a++) {
                if (!((mx >> a) & 1u)) continue;
                const T wa = wr * w[0][a], wia = wi * w[0][a];
#pragma unroll
                for (int b = 0; b < W; b++) {
                    if (!((my >> b) & 1u)) continue;
                    const T wab = wa * w[1][b], wiab = wia * w[1][b];
                    const int lab = (lx[a] * g.t[1] + ly[b]) * g.t[2];
#pragma unroll
                    for (int c = 0; c < W; c++) {
                        if (!((mz >> c) & 1u)) continue;
                        add(lab + lz[c], wab * w[2][c], wiab * w[2][c]);
                    }
                }
            }
            continue;
        }
#pragma unroll 1
        for (int p = 0; p < W * W * W; p++) {
            const int a = p / (W * W), b = (p / W) % W, c = p % W;
            int cx, cy, cz;
            if (!effective_cell(g, anc[0] + s0 + a, anc[1] + s0 + b, anc[2] + s0 + c, cx, cy, cz)) continue;
            const int lx = cx - ox, ly = cy - oy, lz = cz - oz;
            if ((unsigned)lx >= (unsigned)g.t[0] || (unsigned)ly >= (unsigned)g.t[1] || (unsigned)lz >= (unsigned)g.t[2])
                continue;
            const int li = (lx * g.t[1] + ly) * g.t[2] + lz;
            const T wa = axis_weight_at<T>(SCHEME, pr.d[0], a), wb = axis_weight_at<T>(SCHEME, pr.d[1], b),
                    wc = axis_weight_at<T>(SCHEME, pr.d[2], c);
            add(li, wr * wa * wb * wc, wi * wa * wb * wc);
            const double da = axis_weight_at<double>(SCHEME, (double)pr.d[0], a),
                         db = axis_weight_at<double>(SCHEME, (double)pr.d[1], b),
                         dc = axis_weight_at<double>(SCHEME, (double)pr.d[2], c);
            mr += wr64 * g.factor * da * db * dc;
            mi += wi64 * g.factor * da * db * dc;
        }
    }
    mr = warp_sum_d(mr);
    mi = warp_sum_d(mi);
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = mr;
        red[1][threadIdx.x >> 5] = mi;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double sr = 0.0, si = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
            sr += red[0][w];
            si += red[1][w];
        }
        if (sr != 0.0) atomicAdd(&mass[0], sr);
        if (si != 0.0) atomicAdd(&mass[1], si);
    }
    for_tile_cells(g, tile, [&](int li, long long cell) {
        T vr, vi = (T)0;
        if (FIX) {
            vr = (T)(__ll2float_rn((long long)fx[li] * 1048576LL + (long long)fx[tcells + li]) * finv);
            if (CPLX)
                vi = (T)(__ll2float_rn((long long)fx[2 * tcells + li] * 1048576LL + (long long)fx[3 * tcells + li]) * finv);
        } else {
            vr = acc[li];
            if (CPLX) vi = acc_im[li];
        }
        if (k.multi == 0) {
            mesh_re[cell] = vr;
            if (CPLX) mesh_im[cell] = vi;
        } else {
            if (vr != (T)0) atomicAdd(&mesh_re[cell], vr);
            if (CPLX && vi != (T)0) atomicAdd(&mesh_im[cell], vi);
        }
    });
}

}  // namespace HG_TU_NS
}  // namespace hg
