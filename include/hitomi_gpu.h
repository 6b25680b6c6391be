/*
 * hitomi_gpu.h -- C ABI of the B200 (sm_100a) implementation of hitomi_measurement's
 * FFT-based clustering estimators: power-spectrum multipoles P_l(k), bispectrum
 * multipoles B_{l1 l2 L}(k1,k2) and 3PCF multipoles zeta_{l1 l2 L}(r1,r2).
 *
 * The reference has no plugin API: its CLI drivers call free C++ functions
 * (src/hitomi_measurement/main_box.cpp:175-193, main.cpp:242-266).  The entry points
 * below are what the bodies of those functions delegate to; each names the reference
 * function whose arithmetic it replaces.  Plain pointers and sizes only; complex arrays
 * are interleaved (re, im) doubles.
 *
 * Conventions (mirroring the reference, src/hitomi_measurement/field.hpp:61,
 * powerspec.hpp:12-16): every function returns 0 on success and -1 on failure;
 * hg_last_error() gives the reason.  No exception crosses the ABI.  Calls on one context
 * are synchronous and not reentrant.  Several contexts may share a GPU (one host thread
 * each, e.g. to overlap one catalogue's upload with another's statistics); each has its
 * own stream and buffers, and their caches compete for the GPU's memory (a 3PCF field
 * cache that fails to allocate is trimmed and rebuilt in smaller pieces).
 *
 * Results are the reference's RAW FP64 sums before normalisation and printing
 * (pk_save / bk_save / sn_save / zeta_save), plus the normalisation factor the
 * reference multiplies them by, so a caller reproduces the reference's output files.
 */
#ifndef HITOMI_GPU_H
#define HITOMI_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HG_NGP 0
#define HG_CIC 1
#define HG_TSC 2
#define HG_PCS 3 /* project extension: not in the reference (parameter.hpp:504-510 rejects it) */

#define HG_FP64 0 /* plain form: FP64 everywhere */
#define HG_FP32 1 /* chosen form: FP32 mesh/FFT/fields, FP64 sums, scalars and shot noise */

typedef struct hg_ctx hg_ctx;

/* Mirrors the fields of the reference's ParameterClass that the estimators read
 * (parameter.hpp:12-49).  kbin / rbin follow ToolClass::setKbin / setRbin
 * (tools.hpp:118-134): kbin[i] = kmin + i (kmax - kmin)/(n_kbin - 1). */
typedef struct hg_config {
    int n_mesh[3];      /* n_mesh_x/y/z: even, 8..2048, prime factors <= 31 (the 2PCF and the
                           bispectrum / 3PCF shot noise: a power-of-two n_mesh_z <= 1024) */
    double boxsize[3];  /* boxsize_x/y/z */
    int assign;         /* HG_NGP / HG_CIC / HG_TSC / HG_PCS  (parameter "assignment") */
    int interlace;      /* 0/1, project extension (reference has no interlacing) */
    int precision;      /* HG_FP64 or HG_FP32 */
    double kmin, kmax;  /* k bins */
    int n_kbin;
    double rmin, rmax;  /* r bins */
    int n_rbin;
    int periodic;       /* 0: the reference's flat-index bounds rule (field.hpp:92-96);
                           1: periodic wrap (forced for PCS / interlacing) */
    int device;         /* CUDA device ordinal */
    int fp64_stages;    /* HG_FP32 form only: HG_STAGE_* bits of the periodic-box P_l / B_l
                           pipeline to run in FP64 instead (0: none); ignored by HG_FP64 */
} hg_config;

/* Stages of the periodic-box pipeline (hg_pk_box, hg_bk_box*) that an HG_FP32 context can
 * run in FP64 (hg_config.fp64_stages).  The context then also holds an FP64 engine on the
 * same stream; the density spectrum crosses between the two, converted.
 *   HG_STAGE_DENSITY   : assignment and density transform (field.hpp:67-184, 310-325);
 *                        P_l is then binned from the FP64 spectrum
 *   HG_STAGE_BK_SIGNAL : bispectrum signal: G, shell fields, chains, pair sums
 *                        (bispec.hpp:1097-1168)
 *   HG_STAGE_BK_SHOT   : bispectrum shot noise: P terms and the correlation field
 *                        (bispec.hpp:909-1078) */
#define HG_STAGE_DENSITY 1
#define HG_STAGE_BK_SIGNAL 2
#define HG_STAGE_BK_SHOT 4

/* Create / destroy a context.  Replaces the per-call setup the reference does inside
 * each estimator (DensityFieldClass allocation, field.hpp:20-30; FFTW planning,
 * field.hpp:321).  The context owns all device memory, twiddle and bin tables and caches. */
int hg_create(hg_ctx **ctx, const hg_config *cfg);
int hg_destroy(hg_ctx *ctx);
const char *hg_last_error(const hg_ctx *ctx);

/* Hand a particle catalogue to the context.  Reads the caller's array-of-structs in
 * place: particle p's position is the three doubles at base + p*stride_bytes +
 * pos_off*8; its weight the double at w_off*8 (w_off < 0: weight 1).
 *   slot 0 = data  (ParticleGadgetClass {pos[3],vel[3]}: stride 48, pos_off 0, w_off -1,
 *                   particleGadget.hpp:12-15; ParticleBOSSClass {pos[3],los[3],w}:
 *                   stride 56, pos_off 0, los_off 3, w_off 6, particle.hpp:12-16)
 *   slot 1 = randoms (survey geometry only).
 * los_off < 0: no line of sight (periodic box, global LOS along z).
 * Positions must already be in FFT-box coordinates (after the reference's
 * resetParticleForFFT / periodic wrap). */
int hg_set_particles(hg_ctx *ctx, int slot, const double *base, long long n, long long stride_bytes, int pos_off,
                     int los_off, int w_off);

/* As hg_set_particles, but base points to DEVICE memory on the context's GPU that the
 * caller keeps alive and unchanged until the next hg_set_particles* call on this slot or
 * hg_destroy.  Nothing is copied.  (Same reference interface as hg_set_particles.) */
int hg_set_particles_device(hg_ctx *ctx, int slot, const double *dev_base, long long n, long long stride_bytes,
                            int pos_off, int los_off, int w_off);

/* Periodic-box power-spectrum multipole.  Replaces the arithmetic of
 * calcPowerSpectrumForBOX (powerspec.hpp:273-332): TSC/CIC/NGP assignment
 * (field.hpp:67-184), dn = n - N/V (field.hpp:505-525), FFT (field.hpp:310-325) and the
 * binned estimator (field.hpp:765-852) with shot noise N and Y_l0.
 * pk_save[2*n_kbin]: the reference's pk_save = (2l+1) * stat.pk; n_mode[n_kbin] may be
 * NULL; *norm = V / N^2 (powerspec.hpp:316). */
int hg_pk_box(hg_ctx *ctx, int ell, double *pk_save, int *n_mode, double *norm);

/* Periodic-box bispectrum multipole.  Replaces calcBiSpectrumForBOX (bispec.hpp:877-1203).
 * ith_kbin >= 0 computes that k1 row (the reference's one-row-per-run behaviour);
 * ith_kbin = -1 computes all n_kbin rows.  bk_save, sn_save: [rows][n_kbin] complex
 * (2*rows*n_kbin doubles).  Output file value = norm * (bk_save - sn_save)
 * (bispec.hpp:1184-1195). */
int hg_bk_box(hg_ctx *ctx, int ell1, int ell2, int ELL, int ith_kbin, double *bk_save, double *sn_save,
              double *norm);

/* Several periodic-box bispectrum multipoles in one call, sharing the density transform,
 * the shell-field chains and the shot-noise correlation field.  ells = n_multipoles
 * (ell1, ell2, ELL) triples; outputs are n_multipoles consecutive blocks laid out as in
 * hg_bk_box.  Each block equals what calcBiSpectrumForBOX (bispec.hpp:877-1203) computes
 * for that multipole. */
int hg_bk_box_multi(hg_ctx *ctx, int n_multipoles, const int *ells, int ith_kbin, double *bk_save, double *sn_save,
                    double *norm);

/* Periodic-box 3PCF multipole.  Replaces calcThreePointCorrelationFunctionForBOX
 * (bispec.hpp:1205-1424).  ith_rbin >= 0 computes that r1 row, -1 all n_rbin rows;
 * zeta_save, sn_save: [rows][n_rbin] complex.  The shot noise sits only on the diagonal
 * r1 = r2 (bispec.hpp:1279-1285).  Output file value = norm * Re(zeta_save - sn_save)
 * (bispec.hpp:1402-1416), norm = V^3 / N^3. */
int hg_zeta_box(hg_ctx *ctx, int ell1, int ell2, int ELL, int ith_rbin, double *zeta_save, double *sn_save,
                double *norm);

/* Several periodic-box 3PCF multipoles in one call, sharing the density transform, the
 * filtered fields F_lm(r) and the shot-noise correlation field.  ells = n_multipoles
 * (ell1, ell2, ELL) triples; outputs are n_multipoles consecutive blocks laid out as in
 * hg_zeta_box.  Each block equals what calcThreePointCorrelationFunctionForBOX
 * (bispec.hpp:1205-1424) computes for that multipole. */
int hg_zeta_box_multi(hg_ctx *ctx, int n_multipoles, const int *ells, int ith_rbin, double *zeta_save,
                      double *sn_save, double *norm);

/* Survey-geometry bispectrum multipole with local line of sight.  Replaces calcBiSpectrum
 * (bispec.hpp:4-352): shell fields of the data-minus-randoms field, the Yhat_LM-weighted
 * G_LM fields for every M, the (m1, m2, M) sums with Wigner-3j weights, and the shot
 * noise (S3, P and correlation-field terms, bispec.hpp:20-214).  alpha and vsurvey as
 * for hg_pk_survey.  Layout as hg_bk_box; *norm = V_survey^2 / (sum w_D)^3
 * (particle.hpp:319-332).  Needs equal cell sizes on all axes. */
int hg_bk_survey(hg_ctx *ctx, int ell1, int ell2, int ELL, int ith_kbin, double alpha, double vsurvey,
                 double *bk_save, double *sn_save, double *norm);

/* Several survey bispectrum multipoles in one call (layout as hg_bk_box_multi); each block
 * equals what calcBiSpectrum (bispec.hpp:4-352) computes for that multipole. */
int hg_bk_survey_multi(hg_ctx *ctx, int n_multipoles, const int *ells, int ith_kbin, double alpha, double vsurvey,
                       double *bk_save, double *sn_save, double *norm);

/* Survey-geometry 3PCF multipole.  Replaces calcThreePointCorrelationFunction
 * (bispec.hpp:355-614).  Layout as hg_zeta_box; the shot noise sits on the diagonal;
 * *norm = V_survey^2 / (sum w_D)^3. */
int hg_zeta_survey(hg_ctx *ctx, int ell1, int ell2, int ELL, int ith_rbin, double alpha, double vsurvey,
                   double *zeta_save, double *sn_save, double *norm);

/* Several survey 3PCF multipoles in one call (layout as hg_zeta_box_multi). */
int hg_zeta_survey_multi(hg_ctx *ctx, int n_multipoles, const int *ells, int ith_rbin, double alpha, double vsurvey,
                         double *zeta_save, double *sn_save, double *norm);

/* Survey-geometry scalars on the current data (slot 0) and randoms (slot 1):
 * alpha = sum w_D / sum w_R (particle.hpp:268-282), V_survey = (sum w_R)^2 /
 * sum_cells n_R^2 dV (field.hpp:449-503), nbar (particle.hpp:284-300), and the summed
 * weights.  All FP64.  Any output pointer may be NULL. */
int hg_survey_scalars(hg_ctx *ctx, double *alpha, double *vsurvey, double *nbar, double *wsum_data,
                      double *wsum_rand);

/* Survey-geometry (Yamamoto) power-spectrum multipole with local LOS.  Replaces
 * calcPowerSpectrum (powerspec.hpp:4-91): Y_lm-weighted fields
 * (field.hpp:186-228), shot noise (field.hpp:1164-1190) and the (M, m1) sums with
 * Wigner-3j weights.  alpha and vsurvey are the values the caller passes to the
 * reference function.  *norm = V_survey / (sum w_D)^2 (particle.hpp:303-316). */
int hg_pk_survey(hg_ctx *ctx, int ell, double alpha, double vsurvey, double *pk_save, int *n_mode, double *norm);

/* Periodic-box two-point correlation function multipole.  Replaces
 * calcTwoPointCorrelationFunctionForBOX (powerspec.hpp:334-393): xi(x) = FFT_+[(|dn|^2 -
 * N C(k)) / W(k)^2] / V (field.hpp:854-905) averaged over r bins with the Legendre weight
 * L_l(mu) (field.hpp:906-977: fine bins of dr = 0.5, coarse bins (lower, upper]).
 * xi_save[2*n_rbin]: the reference's xi_save = (2l+1) stat.xi; n_mode[n_rbin] (cells per
 * bin) may be NULL; *norm = V / N^2.  Output file value = norm * Re(xi_save)
 * (powerspec.hpp:380-387).  Needs equal cell sizes on all axes. */
int hg_xi_box(hg_ctx *ctx, int ell, double *xi_save, int *n_mode, double *norm);

/* Survey-geometry two-point correlation function multipole with local LOS.  Replaces
 * calcTwoPointCorrelationFunction (powerspec.hpp:93-180): the sum over M and m1 of
 * Wigner-3j-weighted r-binned xi_LM Yhat_{l m1}(r), xi_LM from the Yhat_LM-weighted
 * D - alpha R field against the l = 0 one with the shot noise of field.hpp:1164-1185.
 * *norm = V_survey / (sum w_D)^2.  Layout as hg_xi_box. */
int hg_xi_survey(hg_ctx *ctx, int ell, double alpha, double vsurvey, double *xi_save, int *n_mode, double *norm);

/* Two-point window correlation function multipole.  Replaces
 * calcTwoPointWindowCorrelationFunction (powerspec.hpp:182-270): as hg_xi_survey on the
 * randoms alone (slot 1; calcYlmWeightedDensity field.hpp:230-247, shot noise
 * field.hpp:1202-1217).  *norm = V_survey / (sum w_R)^2.  No data catalogue is needed. */
int hg_xi_window(hg_ctx *ctx, int ell, double vsurvey, double *xi_save, int *n_mode, double *norm);

/* Three-point window correlation function multipole.  Replaces
 * calcThreePointWindowCorrelationFunction (bispec.hpp:617-874): the survey 3PCF of the
 * randoms alone, shot noise from their conj(Yhat) w^2 field minus sum_R w^2 Yhat_LM, on the
 * diagonal.  Layout as hg_zeta_box; *norm = V_survey^2 / (sum w_R)^3.  Output file value =
 * norm * Re(zeta_save - sn_save) (bispec.hpp:863-866). */
int hg_zeta_window(hg_ctx *ctx, int ell1, int ell2, int ELL, int ith_rbin, double vsurvey, double *zeta_save,
                   double *sn_save, double *norm);
int hg_zeta_window_multi(hg_ctx *ctx, int n_multipoles, const int *ells, int ith_rbin, double vsurvey,
                         double *zeta_save, double *sn_save, double *norm);

/* One catalogue of a batch (hg_batch_run): an array of structs in host memory, read as
 * hg_set_particles reads it (positions at pos_off doubles into each record, weight 1). */
typedef struct hg_mock {
    const double *base;
    long long n;
    long long stride_bytes;
    int pos_off;
} hg_mock;

/* Periodic-box statistics of many mock catalogues in one call: the covariance workload
 * that the reference runs as one process per realization (main.cpp:64-76,
 * main_box.cpp:64-90), each process calling calcPowerSpectrumForBOX /
 * calcBiSpectrumForBOX / calcThreePointCorrelationFunctionForBOX.  For every mock, in
 * order: P_l for the n_pk ells, B for the n_bk (l1, l2, L) triples and zeta for the n_zeta
 * triples (all rows).  While one mock is measured, the next one's catalogue is staged
 * through pinned memory by a host thread and copied to the GPU on a second stream.
 * out holds n_mocks blocks of hg_batch_block_len(ctx, n_pk, n_bk, n_zeta) doubles:
 *   pk_save [n_pk][n_kbin] complex, then n_pk norms;
 *   bk_save [n_bk][n_kbin][n_kbin] complex, sn_save likewise, then 1 norm (if n_bk > 0);
 *   zeta_save [n_zeta][n_rbin][n_rbin] complex, sn_save likewise, then 1 norm (if n_zeta > 0).
 * Each block equals what hg_pk_box, hg_bk_box_multi and hg_zeta_box_multi give for that
 * catalogue.  When a mock fails (a catalogue with non-finite positions, a memory limit),
 * the call returns -1 with the mock's index in hg_last_error; the blocks of the mocks
 * before it are complete (hg_batch_done), so a caller resumes from there. */
int hg_batch_run(hg_ctx *ctx, const hg_mock *mocks, int n_mocks, int n_pk, const int *pk_ells, int n_bk,
                 const int *bk_ells, int n_zeta, const int *zeta_ells, double *out);
long long hg_batch_block_len(const hg_ctx *ctx, int n_pk, int n_bk, int n_zeta);
/* How many mocks the last hg_batch_run on this context completed (all of them after a
 * return of 0). */
int hg_batch_done(const hg_ctx *ctx);

/* BAO reconstruction of the current data (slot 0) and randoms (slot 1) on this context's
 * mesh (create the context with the reference's n_mesh_recon) and assignment scheme.
 * Replaces calcReconstructionParticles (particle_reconstruction.hpp:12-208; box = 1:
 * calcReconstructionParticlesForBOX, :210-402): the displacement
 * Psi = FFT_+[-i (W_G(k) / b1_fid) (k / k^2) D(k) / W(k) / V] of the D - alpha R field,
 * W_G = exp(-(k RG)^2 / 2), scaled by vsurvey / sum w_D (box: V / N_D, with alpha taken as
 * double(N_D / N_R) as the reference computes it), TSC-interpolated to every particle.  The
 * shifted positions go to pos_D [n_D][3] and pos_R [n_R][3] (host; either may be NULL); the
 * catalogues the context holds are not changed -- hand the shifted ones back with
 * hg_set_particles, as the reference's drivers continue with the moved particles. */
int hg_reconstruct(hg_ctx *ctx, int box, double b1_fid, double RG, double alpha, double vsurvey, double *pos_D,
                   double *pos_R);

/* Reconstructed periodic-box power-spectrum multipole.  Replaces
 * calcPowerSpectrumForBOXForReconstruction (powerspec.hpp:396-457): dn = n_D - alpha n_R
 * (data slot 0, randoms slot 1, weights 1), shot noise N_D + alpha^2 N_R, Legendre weight;
 * pk_save as hg_pk_box, *norm = V / N_D^2. */
int hg_pk_box_recon(hg_ctx *ctx, int ell, double alpha, double *pk_save, int *n_mode, double *norm);

/* Reconstructed periodic-box 2PCF multipole.  Replaces
 * calcTwoPointFunctionForBOXForReconstruction (powerspec.hpp:459-520): hg_xi_box's estimator
 * on dn = n_D - alpha n_R (weights 1) with shot noise N_D + alpha^2 N_R; *norm = V / N_D^2. */
int hg_xi_box_recon(hg_ctx *ctx, int ell, double alpha, double *xi_save, int *n_mode, double *norm);

/* Reconstructed periodic-box bispectrum multipoles.  Replaces
 * calcBiSpectrumForBOXForReconstruction (bispec.hpp:1426-1753): the estimator of
 * hg_bk_box_multi on dn = n_D - alpha n_R (data slot 0, randoms slot 1, weights 1), its shot
 * noise from the fields dn and n_D + alpha^2 n_R with S3 = N_D - alpha^3 N_R
 * (field.hpp:1242-1250); M = 0 terms only (global line of sight).  ells as
 * hg_bk_box_multi (n_multipoles triples), ith_kbin one row or -1 for all; outputs
 * [n_multipoles][rows][n_kbin] complex; *norm = V^2 / N_D^3.  Output file value =
 * norm * (bk_save - sn_save) (bispec.hpp:1735-1748, file bk{l1}{l2}{L}_{ith}_recon.dat). */
int hg_bk_box_recon_multi(hg_ctx *ctx, int n_multipoles, const int *ells, int ith_kbin, double alpha,
                          double *bk_save, double *sn_save, double *norm);

/* Reconstructed periodic-box 3PCF multipoles.  Replaces
 * calcThreePointCorrelationFunctionForBOXForReconstruction (bispec.hpp:1755-1990): as
 * hg_bk_box_recon_multi for zeta (r bins, shot noise on the diagonal); *norm = V^2 / N_D^3;
 * output file value = norm * Re(zeta_save - sn_save). */
int hg_zeta_box_recon_multi(hg_ctx *ctx, int n_multipoles, const int *ells, int ith_rbin, double alpha,
                            double *zeta_save, double *sn_save, double *norm);

/* ---- catalogue ingest (host side; the reference's readers, native and multi-threaded) */

/* Gadget-2 snapshot header block: 256 bytes, the layout of ParticleGadgetClass::io_header
 * (particleGadget.hpp:33-50), which is the file format. */
typedef struct hg_gadget_header {
    unsigned int npart[6];
    double mass[6];
    double time;
    double redshift;
    int flag_sfr;
    int flag_feedback;
    unsigned int npartTotal[6];
    int flag_cooling;
    int num_files;
    double BoxSize;
    double Omega0;
    double OmegaLambda;
    double HubbleParam;
    char fill[256 - 6 * 4 - 6 * 8 - 2 * 8 - 2 * 4 - 6 * 4 - 2 * 4 - 4 * 8];
} hg_gadget_header;

/* ASCII catalogue.  Replaces ParticleBOSSClass::readParticleBOSS (particle.hpp:93-154):
 * every line from which ncols numbers can be read (as sscanf "%lf %lf ..." reads them:
 * x y z w for ncols = 4) is one record, other lines are skipped.  *out: n x ncols doubles,
 * allocated here, released with hg_free.  Errors: hg_last_error(NULL). */
int hg_read_ascii(const char *path, int ncols, double **out, long long *n);

/* Gadget snapshot base.0 .. base.(num_files-1).  Replaces
 * ParticleGadgetClass::readParticlesFromGagdetSnapshot (particleGadget.hpp:211-298):
 * *out holds n records {pos[3], vel[3] * sqrt(a)} (the ParticleGadgetClass layout, 48-byte
 * stride, for hg_set_particles), allocated here, released with hg_free; *hdr (may be NULL)
 * receives base.0's header. */
int hg_read_gadget(const char *base, double **out, long long *n, hg_gadget_header *hdr);
void hg_free(void *p);

/* Per-kernel device timing: when on, every kernel launch of this library is bracketed by
 * CUDA events on the context's stream.  hg_kernel_stats writes one line per kernel name:
 * "name<TAB>launches<TAB>total_ms<TAB>modelled_bytes".  These replace the reference's
 * clock() progress prints (bispec.hpp:1170-1171, powerspec.hpp:63-66). */
int hg_set_profiling(hg_ctx *ctx, int on);
int hg_kernel_stats(hg_ctx *ctx, char *buf, long long buflen);

/* Device memory of a context.  hg_set_memory_limit caps what the context's buffers may hold
 * (bytes; 0 removes the cap): a statistic that would need more fails with -1 and a message
 * naming the limit, without launching past the failed allocation, and the context stays
 * usable (raise the limit and call again).  Buffers are kept between calls and grow only, so
 * the cap also bounds what a long-lived context keeps.  hg_memory_in_use returns the bytes
 * the context's buffers hold now.  The reference has no counterpart (its global `byte`
 * counter, common.hpp:36, only prints). */
int hg_set_memory_limit(hg_ctx *ctx, long long bytes);
long long hg_memory_in_use(const hg_ctx *ctx);

/* The launch shapes the context's autotuner picked (one line per tuned kernel and grid: the
 * chosen variant and the measured time of every variant).  With HG_CHAIN_VARIANT=v in the
 * environment a context uses chain variant v untimed (every variant gives the same result;
 * an unknown v fails the bispectrum call).  No counterpart in the reference. */
int hg_tuning(hg_ctx *ctx, char *buf, long long buflen);

/* Allocation-free periodic-box power-spectrum multipole.  No counterpart in the reference:
 * it is the binning step of hg_pk_box run on a density spectrum the caller already holds
 * on the device, for callers that cannot call cudaMalloc -- an application whose own
 * allocator or memory budget owns all of the GPU's memory, or a loop that cannot afford
 * cudaMalloc's cost and implicit synchronisation on every call.
 *   d_half_spectrum : device array [n0][n1][n2/2+1] of complex (double pairs for HG_FP64,
 *                     float pairs for HG_FP32, per cfg->precision) holding
 *                     FFT[dV (rho - N/V)], the non-negative-kz half of the reference's
 *                     calcFourierTransform output (field.hpp:310-325) for a real field.
 *   cfg->assign     : NGP, CIC or TSC (the window and shot-noise tables), no interlacing.
 *   outputs as hg_pk_box; stream is a cudaStream_t (NULL: the default stream).
 * All scratch sits in a 1 MiB file-scope __device__ array that every GPU loading this
 * library keeps until exit.  Limits: n_kbin <= 256, n_mesh <= 1024 per axis, k bins
 * below |k| = 10; larger requests fail with an error and launch nothing.  The first call
 * on a device looks up that array's address.  Calls share the array (each clears its
 * accumulators first): calls overlapping on the GPU race.  The call waits for the stream,
 * returns the sums in host memory and restores the caller's current device.
 * Errors: hg_last_error(NULL). */
int hg_pk_box_spectrum_static(const hg_config *cfg, const void *d_half_spectrum, long long n_particles, int ell,
                              double *pk_save, int *n_mode, double *norm, void *stream);

/* Device-side time of the last statistic call in milliseconds (CUDA events on the
 * context's stream), and the number of kernels it launched. */
int hg_last_timing(const hg_ctx *ctx, double *device_ms, long long *kernel_launches);

#ifdef __cplusplus
}
#endif

#endif /* HITOMI_GPU_H */
