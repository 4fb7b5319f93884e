/*
 * cp_oracle.h -- CPU FP64 restatement of the QCD 2->2 hard-process integrator.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker for the CUDA
 * path in cupythia_b200/: only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg may load it.  The product never calls into it, and there is
 * no CPU fallback that routes through it.
 *
 * Every function restates the reference's algorithm and cites the reference
 * file:line it follows (paths relative to the reference project root):
 *   cuPythia/common/rng.cuh            SplitMix64 counter RNG
 *   cuPythia/pipeline/physics.cuh      gg->gg matrix element (reciprocal form)
 *   pythia8317/src/SigmaQCD.cc         the five Sigma2 QCD matrix elements
 *   pythia8317/src/SigmaProcess.cc     flux tables, sigmaPDF, store2Kin scales
 *   pythia8317/src/PartonDistributions.cc  CTEQ5L
 *   pythia8317/src/StandardModel.cc    AlphaStrong (first order)
 *   pythia8317/src/PhaseSpace.cc       tau / y / z limits and Jacobians
 * Philox-4x32-10 is not in the reference; it is restated from Salmon et al.,
 * "Parallel random numbers: as easy as 1, 2, 3" (SC'11).
 */
#ifndef CP_ORACLE_H
#define CP_ORACLE_H
#include <stdint.h>
#include <complex.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------- counter RNGs ---------------- */
uint64_t cpo_splitmix64(uint64_t x);
double   cpo_u01(uint64_t u);
uint64_t cpo_thread_counter(uint64_t seed, uint64_t tid);
uint64_t cpo_event_key(uint64_t base, uint64_t e);
void     cpo_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
/* Philox draws of one integrator point: key = seed, ctr = (point lo, point hi, iter, stream). */
void     cpo_point_words(uint64_t seed, uint64_t point, uint32_t iter, uint32_t stream,
                         uint32_t out[4]);
double   cpo_u24(uint32_t w);          /* (w >> 8) * 2^-24, exact                    */
double   cpo_u53(uint32_t lo, uint32_t hi);

/* ---------------- matrix elements, dsigma/dtHat in GeV^-4 ---------------- */
double cpo_sigma_gg2gg(double sH, double tH, double uH, double alpS);
double cpo_sigma_gg2qqbar(double sH, double tH, double uH, double alpS, int nQuarkNew);
double cpo_sigma_qg2qg(double sH, double tH, double uH, double alpS);
double cpo_sigma_qq2qq(double sH, double tH, double uH, double alpS, int id1, int id2);
double cpo_sigma_qqbar2gg(double sH, double tH, double uH, double alpS);
/* the cuPythia reciprocal form (pipeline/physics.cuh:9-16) */
double cpo_gg2gg_recip(double sH, double tH, double uH, double alpS);

/* ---------------- PDFs and couplings ---------------- */
/* CTEQ5L raw arrays: out = {xd, xu, xg, xubar, xdbar, xs, xc, xb} */
void   cpo_cteq5l_raw(double x, double Q2, double out[8]);
/* proton x*f(id, x, Q2) with Pythia's max(0, .) clamp; id in -5..5 or 21 */
double cpo_pdf_xf(int id, double x, double Q2);

typedef struct {
  double aSmZ;
  double L3_2, L4_2, L5_2, L6_2;
  double mc2, mb2, mt2, scale2Min;
  int nfmax;
} cpo_alphas;
void   cpo_alphas_init(cpo_alphas* a, double aSmZ);
double cpo_alphas_eval(const cpo_alphas* a, double Q2);

/* ---------------- hadronic integrand ---------------- */
enum { CPO_GG2GG = 1, CPO_GG2QQBAR = 2, CPO_QG2QG = 4, CPO_QQ2QQ = 8, CPO_QQBAR2GG = 16,
       CPO_ALLQCD = 31 };

typedef struct {
  double sqrtS;      /* GeV                                           */
  double pTmin;      /* PhaseSpace:pTHatMin                           */
  double aSmZ;       /* SigmaProcess:alphaSvalue (first order)         */
  double kR;         /* renormalisation-scale factor: muR^2 = kR pT^2  */
  double kF;         /* factorisation-scale factor:  muF^2 = kF pT^2   */
  double convert2mb; /* GeV^-2 -> mb                                   */
  int nQuarkIn;      /* PDFinProcess:nQuarkIn                          */
  int nQuarkNew;     /* HardQCD:nQuarkNew                              */
  int procMask;      /* OR of CPO_* process bits                       */
} cpo_had_cfg;

void cpo_had_default(cpo_had_cfg* c);

/* ---------------- operation count (cp_opcount.cc) ---------------- */
/* CTEQ5L coefficient tables: AM [8][9][3], QMIN, ALPHA, UT1, UT2 [8] */
void   cpo_cteq5l_table(const double** am, const double** qmin, const double** alpha, const double** ut1,
                        const double** ut2);
/* the weight of cpo_had_weight_x in the counted (least-arithmetic) form, FP64 */
double cpo_opcount_weight(const cpo_had_cfg* c, const double x[3]);
/* mean add, mul, div, exp, log, sqrt per point over n points x (3n doubles), VEGAS map included;
 * out[6] = largest relative difference of the counted form from cpo_had_weight_x */
void   cpo_opcount_counts(const cpo_had_cfg* c, const double* x, int64_t n, double out[7]);

/* SigmaProcess surface for one phase-space point (Pythia set2Kin + sigmaKin + sigmaPDF).
 * out[0] = sigmaPDF summed over the selected processes (mb), per Pythia's pair loop.
 * out[1] = alpha_s(muR^2), out[2] = Q2Ren, out[3] = Q2Fac, out[4] = uH, out[5] = pT2. */
void cpo_had_sigma_pdf(const cpo_had_cfg* c, double x1, double x2, double sH, double tH,
                       int procMask, double out[6]);

/* Density in (tau, y, z): d sigma / (dtau dy dz) in mb, zero outside the cut region. */
double cpo_had_density(const cpo_had_cfg* c, double tau, double y, double z);

/* Weight of a point x in [0,1]^3 through the analytic base map (tau,y,z)(x):
 * returns f * J_base; fills tyz[3] = (tau, y, z) if non-null. */
/* record picks (process, incoming pair, new flavour, colour flow) of an accepted point at x */
/* pickInState + setIdColAcol of process `code` at given kinematics (x1, x2, sH, tH) */
int    cpo_pick_state(const cpo_had_cfg* c, int code, double x1, double x2, double sH, double tH, double r1,
                      double r3, double rc, double rs, int id[4], int* colour);
int    cpo_pick_record(const cpo_had_cfg* c, const double x[3], double r0, double r1, double r3,
                       double rc, double rs, int id[4], int* colour);
/* the same two picks with *margin = the smallest distance of any draw from a selection
 * boundary, relative to what it selects from (1 when nothing is selected) */
int    cpo_pick_state_margin(const cpo_had_cfg* c, int code, double x1, double x2, double sH, double tH,
                             double r1, double r3, double rc, double rs, int id[4], int* colour, double* margin);
int    cpo_pick_record_margin(const cpo_had_cfg* c, const double x[3], double r0, double r1, double r3,
                              double rc, double rs, int id[4], int* colour, double* margin);
double cpo_had_weight_x(const cpo_had_cfg* c, const double x[3], double tyz[3]);

/* VEGAS map of one point given the three 24-bit uniforms m_d = w_d >> 8:
 * bin_d = (m_d * nb) >> 24, frac_d = ((m_d * nb) & 0xFFFFFF) 2^-24,
 * x_d = e[d][bin] + frac * (e[d][bin+1] - e[d][bin]).  edges is [3][nb+1]. */
double cpo_vegas_map(const double* edges, int nb, const uint32_t w[3], double x[3], int bins[3]);

/* Weight of integrator point `point` of iteration `iter` (Philox stream 0). */
double cpo_had_point_weight(const cpo_had_cfg* c, const double* edges, int nb, uint64_t seed,
                            uint32_t iter, uint64_t point, int bins[3], double x[3]);

/* Accumulate points [p0, p0+n): sums[0]=sum w, sums[1]=sum w^2; hist[3*nb] += w^2 per bin. */
void cpo_had_accumulate(const cpo_had_cfg* c, const double* edges, int nb, uint64_t seed,
                        uint32_t iter, uint64_t p0, uint64_t n, double sums[2], double* hist,
                        int nthreads);

/* Classic VEGAS refinement (Lepage): smooth, compress with exponent alpha, equal-share rebin. */
void cpo_vegas_refine(double* edges, const double* hist, int ndim, int nb, double alpha);
void cpo_vegas_uniform(double* edges, int ndim, int nb);

/* ---------------- partonic gg -> gg (fixed sHat) ---------------- */
double cpo_partonic_weight(double sqrtShat, double alpS, double cMax, double conv, double u);
/* Philox mode: point i uses u53 of words (0,1) of philox(ctr=(i lo, i hi, 0, 0), key=seed). */
void   cpo_partonic_philox(double sqrtShat, double alpS, double cMax, double conv, uint64_t seed,
                           uint64_t p0, uint64_t n, double sums[2], int nthreads);
/* SplitMix64 mode with the reference's per-thread indexing: thread tid draws
 * splitmix64(seed + tid*0x100000001B3 + i) for i < kPer. */
void   cpo_partonic_splitmix(double sqrtShat, double alpS, double cMax, double conv, uint64_t seed,
                             uint64_t nThreads, uint64_t kPer, double sums[2], int nthreads);
double cpo_simpson_gg2gg(int N, double sqrtShat, double alpS, double cMax, double conv);

/* ---------------- derivatives (complex step, FP64) ---------------- */
/* Parameter vector theta = (aSmZ, kR, pTmin).  Returns w and dw/dx_d (d=0..2),
 * dw/dtheta_k (k=0..2) of f*J_base at x, by complex-step differentiation. */
void cpo_had_weight_grad(const cpo_had_cfg* c, const double x[3], double out[7]);

/* Sums over points of the estimator and its gradient for the full VEGAS+base map:
 * g[0]=sum w, g[1]=sum w^2,
 * g[2..4]   = sum dw/dtheta,  g[5..7] = sum w dw/dtheta,
 * g[8 .. 8+E) = sum dw/de,   g[8+E .. 8+2E) = sum w dw/de,  E = 3*(nb+1). */
void cpo_had_adjoint_sums(const cpo_had_cfg* c, const double* edges, int nb, uint64_t seed,
                          uint32_t iter, uint32_t stream, uint64_t p0, uint64_t n, double* g,
                          int nthreads);

/* f * J_base at n points x (3n floats, as doubles), multi-threaded */
void cpo_had_weight_x_batch(const cpo_had_cfg* c, const float* x, int64_t n, double* out, int nthreads);

/* ---------------- learned proposal (flow) ---------------- */
/* FP64 flow forward with the CUDA kernels' BF16 rounding points; P is the FP32 master layout. */
void cpo_flow_forward(const float* P, const double u[3], double v[3], double* logJ);
/* BF16 rounding emulation on (1, default) or off (0: plain FP64, for finite-difference checks) */
void cpo_flow_set_rounding(int on);
/* G = sum_p d(cv_p . v_p + cJ_p lnJ_p)/d params (reverse mode, FP64). */
void cpo_flow_backward_batch(const float* P, int64_t n, const double* u, const double* cv, const double* cJ,
                             double* G, int nthreads);

/* ---------------- unweighting ---------------- */
/* Accept draw of a point: word 3 of its Philox block, as u24. */
int cpo_accept(double w, double wmax, uint32_t w3);

#ifdef __cplusplus
}
#endif
#endif
