/*
 * cupythia_b200.h -- C ABI of the B200 (sm_100a) QCD 2->2 hard-process integrator.
 *
 * Plain pointers and sizes only.  "dev" pointers are CUDA device pointers on the handle's
 * device; "host" pointers are ordinary host memory.  Every entry point returns CP_OK (0) or a
 * nonzero CP_ERR_* code; cp_last_error() gives the message of the handle's last failure.
 *
 * Ownership: the caller owns every input and output buffer; the handle owns its scratch
 * memory, its VEGAS grid and its flow weights.  Threading: one handle per host thread and
 * device; all work of a handle is ordered on its CUDA stream (cp_set_stream).
 *
 * Each entry point names the reference interface it replaces (paths relative to the
 * reference project root: cuPythia/ for the CUDA stages, pythia8317/ for Pythia).
 */
#ifndef CUPYTHIA_B200_H
#define CUPYTHIA_B200_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CP_ABI_VERSION 1

/* status codes */
#define CP_OK 0
#define CP_ERR_INVALID 1  /* invalid argument or configuration                          */
#define CP_ERR_CUDA 2     /* CUDA runtime error (message in cp_last_error)               */
#define CP_ERR_NUMERIC 3  /* non-finite or negative weights were produced and zeroed     */
#define CP_ERR_TIMEOUT 4  /* a bounded device-side wait expired                          */
#define CP_ERR_CAPACITY 5 /* an output buffer was too small (count is still reported)   */
#define CP_ERR_NOMEM 6    /* device allocation failed                                    */

/* process switches (HardQCD:gg2gg ... of pythia8317/share/Pythia8/xmldoc/QCDHardProcesses.xml);
 * Pythia process codes 111..115 (pythia8317/include/Pythia8/SigmaQCD.h:206,242,279,312,344) */
#define CP_PROC_GG2GG 1
#define CP_PROC_GG2QQBAR 2
#define CP_PROC_QG2QG 4
#define CP_PROC_QQ2QQ 8
#define CP_PROC_QQBAR2GG 16
#define CP_PROC_ALL 31

#define CP_MAX_BINS 128   /* VEGAS bins per dimension */

typedef struct cp_handle cp_handle;

/* Physics and sampling configuration; field names follow the Pythia settings they mirror. */
typedef struct cp_config {
  double sqrt_s;       /* Beams:eCM, GeV                                   (13000)  */
  double pt_hat_min;   /* PhaseSpace:pTHatMin, GeV                         (20)     */
  double alphas_mz;    /* SigmaProcess:alphaSvalue, first-order running    (0.13)   */
  double k_ren;        /* SigmaProcess:renormMultFac, muR^2 = k pT^2       (1)      */
  double k_fac;        /* SigmaProcess:factorMultFac, muF^2 = k pT^2       (1)      */
  double convert2mb;   /* GeV^-2 -> mb, SigmaProcess.cc:24                 (0.389380) */
  int n_quark_in;      /* PDFinProcess:nQuarkIn (only 5 supported)         (5)      */
  int n_quark_new;     /* HardQCD:nQuarkNew                                (3)      */
  int proc_mask;       /* OR of CP_PROC_*                                  (ALL)    */
  int n_bins;          /* VEGAS bins per dimension, <= CP_MAX_BINS         (50)     */
  int device;          /* CUDA device ordinal                              (0)      */
  int reserved;
  uint64_t seed;       /* Philox key                                       (42)     */
} cp_config;

typedef struct cp_result {
  double sigma;        /* estimate, mb                                              */
  double sigma_err;    /* standard error, mb                                        */
  double sum_w, sum_w2;
  double w_max;
  uint64_t n_points;
  uint64_t n_bad;      /* non-finite / negative weights (zeroed)                    */
  double eta;          /* <w> / w_max                                               */
} cp_result;

/* 64-byte unweighted event record: 2 incoming + 2 outgoing massless partons. */
typedef struct cp_event {
  int16_t id[4];       /* PDG ids: incoming a (+z), incoming b (-z), outgoing 3, 4  */
  float pz_in[2];      /* incoming momenta along z, GeV (E = |pz|)                  */
  float p3[4];         /* px, py, pz, E of outgoing 3, lab frame, GeV               */
  float p4[4];         /* px, py, pz, E of outgoing 4                               */
  float weight;        /* 1, or w / w_max for overweight events (> 1)               */
  float pt_hat;        /* GeV                                                       */
  uint16_t process;    /* Pythia process code 111..115                              */
  uint16_t colour;     /* colour flow of the process's setIdColAcol: bits 0-1 topology
                          (order of its setColAcol calls), bit 2 swapColAcol, bit 3
                          swapCol1234; cp_colour_tags() expands it to col/acol tags   */
  uint32_t point;      /* low 32 bits of the point index that produced the event    */
} cp_event;

/* Result of a production (unweighting) pass. */
typedef struct cp_unweight_result {
  double sigma, sigma_err;       /* weighted estimate of the pass, mb                    */
  double sigma_unweighted;       /* w_max * (sum of event weights) / n_points, mb        */
  double w_max;                  /* threshold used                                       */
  double w_max_seen;             /* largest weight of the pass                           */
  double eta;                    /* n_accepted / n_points                                */
  uint64_t n_points, n_accepted, n_overweight, n_bad;
} cp_unweight_result;

/* Gradient of the estimator (cp_adjoint). */
typedef struct cp_grad {
  double sigma, var;            /* estimator value and Var[w] of the batch           */
  double dsigma[3], dvar[3];    /* d/d(alpha_s(mZ)), d/d(k_ren), d/d(pT_hat_min)     */
  uint64_t n_points, n_bad;
} cp_grad;

/* ---------------------------------------------------------------- handles ---------- */
int cp_abi_version(void);
int cp_config_default(cp_config* cfg);
/* Adds `offset` to the point index of every integration, production and adjoint pass of this
 * handle (the counter of point p becomes offset + p): the reference's shard offset
 * (cupythia_shard_offset, cuPythia/common/rng.cuh:5-19; the stage drivers read CUPYTHIA_SHARD
 * and CUPYTHIA_SHARD_N into it).  Records carry the low 32 bits of the global index. */
int cp_set_point_offset(cp_handle* h, uint64_t offset);
/* replaces the per-stage cudaMalloc/setup of the cuPythia mains (e.g. 11_vegas_importance/vegas.cu:94-105) */
int cp_create(const cp_config* cfg, cp_handle** out);
int cp_destroy(cp_handle* h);
const char* cp_last_error(const cp_handle* h);
int cp_set_stream(cp_handle* h, void* cuda_stream);
int cp_synchronize(cp_handle* h);
int cp_device_sm_count(cp_handle* h, int* n_sm);

/* ---------------------------------------------------------------- counter RNG ------ */
/* Philox-4x32-10 words of points [point0, point0+n): key = seed, counter = (point, iter, stream);
 * out (dev) holds 4n words.  Replaces the draw of cuPythia/common/rng.cuh:47-57 with the
 * counter layout documented in the product's design notes. */
int cp_philox_words(cp_handle* h, uint64_t seed, uint64_t point0, uint64_t n, uint32_t iter,
                    uint32_t stream, uint32_t* out_dev);
/* SplitMix64 uniforms in the reference's per-thread layout: out[t*k_per + i] =
 * u01(splitmix64(seed + t*0x100000001B3 + i)) (cuPythia/03_fused_resident_me/fused_gg2gg.cu:43-46). */
int cp_splitmix_uniforms(cp_handle* h, uint64_t seed, uint64_t n_threads, uint64_t k_per,
                         double* out_dev);
/* per-event keys splitmix64(base ^ e*0x9E3779B97F4A7C15), e in [e0, e0+n)
 * (cuPythia/05_reproducible_events/repro_events.cu:43, cuPythia/pipeline/generate.cu:33) */
int cp_event_keys(cp_handle* h, uint64_t base, uint64_t e0, uint64_t n, uint64_t* out_dev);

/* ---------------------------------------------------------------- SigmaProcess ----- */
/* Batched Sigma2Process::set2Kin (pythia8317/include/Pythia8/SigmaProcess.h:118,498-501 ->
 * store2Kin, pythia8317/src/SigmaProcess.cc:846-925; massless): stores the batch and its
 * uHat, pT^2, Q2Ren, Q2Fac and alpha_s.  Inputs are dev SoA arrays of n points. */
int cp_set2kin_batch(cp_handle* h, const float* x1, const float* x2, const float* sH,
                     const float* tH, int64_t n);
/* The same from FP64 device arrays, the precision of Pythia's set2Kin arguments: uHat and pT^2
 * are formed in FP64 before the batch is rounded to FP32, so points at large sHat near the pT
 * cut (|uHat| << sHat, where an FP32 sHat + tHat cancels) keep FP32 relative precision. */
int cp_set2kin_batch_f64(cp_handle* h, const double* x1, const double* x2, const double* sH,
                         const double* tH, int64_t n);
/* Batched sigmaKin + sigmaHat of the flavour-independent processes 111, 112, 113, 115
 * (pythia8317/src/SigmaQCD.cc:115-325): dsigmaHat/dtHat in GeV^-4, one value per point. */
int cp_sigma_kin_batch(cp_handle* h, int process_code, float* out_dev);
/* Batched sigmaHat(id1, id2) (SigmaProcess.h:139; Sigma2qq2qq::sigmaHat SigmaQCD.cc:272-286). */
int cp_sigma_hat_batch(cp_handle* h, int process_code, int id1, int id2, float* out_dev);
/* Batched sigmaPDF() (pythia8317/src/SigmaProcess.cc:423-480) summed over the processes of
 * proc_mask: sum over pairs of CONVERT2MB sigmaHat xf_a(x1) xf_b(x2), mb GeV^-2. */
int cp_sigma_pdf_batch(cp_handle* h, int proc_mask, float* out_dev);
/* SigmaProcess::pickInState (SigmaProcess.cc:486-508: the first pair of the initFlux list whose
 * running sum of pdfSigma reaches r x the total) and setIdColAcol (SigmaQCD.cc:135-342) of
 * process `code` over the stored batch, with PDFs at its Q2Fac.  r_dev: 4 uniforms per point
 * (pair, new flavour of g g -> q qbar, colour topology, g g -> g g orientation; 16-byte aligned);
 * ids_dev: 4 PDG ids per point (in a, in b, out 3, out 4; 8-byte aligned); colour_dev: the
 * colour-flow code of the event records (cp_colour_tags). */
int cp_pick_state_batch(cp_handle* h, int code, const float* r_dev, int16_t* ids_dev, uint16_t* colour_dev);
/* Accessors alphaSRen(), Q2Ren(), Q2Fac() of the stored batch (SigmaProcess.h:254-257). */
int cp_scales_batch(cp_handle* h, float* alphas_dev, float* q2ren_dev, float* q2fac_dev);
/* CTEQ5L x f(id, x, Q2) of a proton (PDF::xf, pythia8317/src/PartonDistributions.cc:122-180):
 * out (dev) is n x 11 in id order -5..-1, 1..5, 21. */
int cp_pdf_batch(cp_handle* h, const float* x_dev, const float* q2_dev, int64_t n, float* out_dev);

/* ---------------------------------------------------------------- VEGAS ------------ */
/* Grid: 3 dimensions (tau, y, cos theta) x (n_bins + 1) edges in [0, 1], FP64. */
int cp_grid_reset(cp_handle* h);
int cp_grid_set(cp_handle* h, const double* edges_host);
int cp_grid_get(cp_handle* h, double* edges_host);
/* One VEGAS iteration of n_points points (Philox stream 0, counter iteration = iter):
 * fused draw -> map -> integrand -> Kahan block sums -> FP64 slot reduction -> per-bin w^2
 * histograms, then, if alpha > 0, the FP64 grid refinement on the device.  Replaces the
 * iteration body of cuPythia/11_vegas_importance/vegas.cu:107-124 (3-D, hadronic). */
int cp_vegas_iteration(cp_handle* h, uint64_t n_points, uint32_t iter, double alpha,
                       cp_result* out_host);
/* n_iter iterations back to back on the device, one host read at the end; per_iter (host,
 * n_iter entries, may be NULL) and the inverse-variance combination of the iterations with
 * index >= skip. */
int cp_integrate(cp_handle* h, int n_iter, uint64_t n_points, double alpha, int skip,
                 cp_result* per_iter_host, cp_result* combined_host);
/* Multi-GPU iteration (one process per GPU, contiguous point shards via cp_set_point_offset;
 * the only exchange of a VEGAS iteration across ranks): cp_vegas_accumulate runs this handle's pass over
 * n_points points and writes its CP_SLOT_HEAD + 3 n_bins sums (dev) -- sum w, sum w^2, max w,
 * n_bad, then the per-bin sums of w^2 of each dimension; the caller reduces them over ranks
 * (sum, max for entry 2) and every rank refines identically with cp_vegas_refine_sums
 * (n_total = the points of all ranks).  The reference shards events the same way
 * (cuPythia/common/rng.cuh:5-19) but never exchanges a grid. */
#define CP_SLOT_HEAD 4
int cp_vegas_accumulate(cp_handle* h, uint64_t n_points, uint32_t iter, double* sums_dev);
int cp_vegas_refine_sums(cp_handle* h, const double* sums_dev, double n_total, double alpha, cp_result* out_host);
/* Weight histogram of the last pass (CP_QBINS u64 counts, dev) and the quantile of a histogram
 * reduced (summed) over ranks: every rank then unweights against the same w_max. */
#define CP_QBINS 4096
int cp_weight_histogram(cp_handle* h, unsigned long long* hist_dev);
int cp_weight_quantile_hist(cp_handle* h, const unsigned long long* hist_dev, double q, double* w_q_host);
/* Per-point weights (dev) of points [point0, point0+n) of iteration iter on the current grid,
 * and optionally the mapped x (dev, 3n floats) the integrand was evaluated at. */
int cp_point_weights(cp_handle* h, uint64_t point0, uint64_t n, uint32_t iter, float* w_dev,
                     float* x_dev);
/* FP32 integrand at caller-given x in [0,1]^3 (dev, 3n floats): f * J_base, mb. */
int cp_weight_at(cp_handle* h, const float* x_dev, int64_t n, float* w_dev);

/* Reduced sums of the last VEGAS pass (host, 4 + 3 n_bins doubles): sum w, sum w^2, max w,
 * n_bad, then the per-bin sums of w^2 of each dimension (the refinement's input). */
int cp_last_histogram(cp_handle* h, double* out_host);

/* One VEGAS pass (the body of cp_vegas_iteration, without refinement) that allocates nothing.
 * No counterpart in the reference.  For callers that cannot call cudaMalloc: a host program that
 * owns every device allocation (a caching allocator or pool whose accounting an allocation
 * behind its back would break), a process held to a fixed device-memory budget, or a plugin (a
 * Pythia SigmaProcess) running inside another program's event loop without a handle of its own.
 * No handle is created; the scratch (block partial sums for up to 512 blocks and the weight
 * histogram: 1,622,016 bytes) is a file-scope device array that every GPU
 * loading this library keeps until exit.
 * Inputs: cfg (host), the grid edges_dev (3 x (n_bins + 1) doubles).  Output: sums_dev (4 + 3
 * n_bins doubles, the layout of cp_last_histogram).  n_bins > CP_MAX_BINS is rejected
 * (CP_ERR_INVALID).  The first call on a device looks up the array's device address and the
 * launch shape and should come before any stream capture; later calls re-check the address.
 * Each call clears the weight histogram on the stream (the CTEQ5L records travel in the kernel's
 * parameters); the
 * array keeps the last call's contents, and calls that overlap on the GPU race on it. */
int cp_vegas_pass_noalloc(const cp_config* cfg, uint64_t n_points, uint32_t iter,
                          const double* edges_dev, double* sums_dev, void* cuda_stream);

/* ---------------------------------------------------------------- unweighting ------ */
/* q-quantile of the weights of the last VEGAS pass (integer weight histogram, ~2% bins,
 * rounded up), stored as the handle's unweighting threshold; the production run uses
 * q = 0.999.  Replaces the host w_max scans of cuPythia/07_unweighting_lhe/unweight_lhe.cu:59-63
 * and cuPythia/pipeline/generate.cu:71-76. */
int cp_weight_quantile(cp_handle* h, double q, double* w_q_host);
/* Sets the unweighting threshold explicitly. */
int cp_set_wmax(cp_handle* h, double w_max);
/* Production pass over points [0, n_points) of counter iteration iter: fused draw -> map ->
 * integrand -> accept (u w_max < w; overweight events kept with weight w / w_max) -> compaction
 * of accepted events into records_dev (capacity records).  Replaces the unweighting kernels
 * (cuPythia/07_unweighting_lhe/unweight_lhe.cu:42-57, cuPythia/pipeline/generate.cu:56-62) and
 * the flag + library compaction (cuPythia/10_cub_compaction/cub_compaction.cu:36-46,76-80),
 * with the same output order: the records of the accepted points in point order, the same on
 * every run.  Returns CP_ERR_CAPACITY (with the counts filled in) when more events were accepted
 * than fit; the first `capacity` records in point order are stored.  Device staging: 80 bytes per
 * point of a chunk of at most 2^24 points (1.3 GB), kept in the handle. */
int cp_unweight(cp_handle* h, uint64_t n_points, uint32_t iter, cp_event* records_dev,
                uint64_t capacity, cp_unweight_result* out_host);
/* Scale-variation weights (the fused reweighting of cuPythia/pipeline/reweight.cu:36-51 and
 * pipeline/generate.cu:49-54, extended to mu_F): with a device buffer of capacity >= the record
 * capacity set, cp_unweight also writes 6 floats per record, the event's weight ratios
 * w(muR', muF') / w(muR, muF) for (muR'/muR, muF'/muF) = (2,1), (1/2,1), (1,2), (1,1/2), (2,2),
 * (1/2,1/2), evaluated at the event's own point (alpha_s at the varied mu_R, CTEQ5L at the
 * varied mu_F).  The varied cross section of a sample is w_max / n x sum(event weight x ratio).
 * weights_dev = NULL switches them off; cp_generate_host does not write them. */
int cp_set_scale_weights(cp_handle* h, float* weights_dev, uint64_t capacity);
/* The same production pass delivering the records to HOST memory (pinned for overlap), in
 * chunks of `chunk` points whose device-to-host copies overlap the following chunks' compute
 * (the handle keeps 3 staging buffers of `chunk` records; 2^21 points per chunk keeps the copy
 * engine busy back to back; at most 2^24).  The records arrive in point order, byte-identical
 * to cp_unweight's.  Every copy has finished when the call returns. */
int cp_generate_host(cp_handle* h, uint64_t n_points, uint32_t iter, uint64_t chunk,
                     cp_event* records_host, uint64_t capacity, cp_unweight_result* out_host);

/* ---------------------------------------------------------------- partonic gg->gg --- */
/* Fused resident gg->gg MC in FP64 (cuPythia/03_fused_resident_me/fused_gg2gg.cu:40-51):
 * cos theta = (2u-1) cMax, u from Philox (point i: counter (i, 0, 0, 0), 53-bit uniform of
 * words 0,1); sigma = <w>, w = dsigma/dtHat (2 cMax)(s/2) conv. */
int cp_partonic_integrate(cp_handle* h, double sqrt_shat, double alphas, double cmax,
                          double conv, uint64_t seed, uint64_t n_points, cp_result* out_host);
/* Same integrand on the reference's SplitMix64 per-thread streams (n_threads x k_per draws:
 * reference thread i draws from counter seed + i 0x100000001B3 + k).  The draws are shared out
 * in equal contiguous parts, so the sums are those of the reference's stage in another order;
 * the matrix element is evaluated in its closed form (9/2)(3 - tu/s^2 - su/t^2 - st/u^2), within
 * 1.1e-15 relative of Pythia's bracket form.  Fails with CP_ERR_INVALID when n_threads k_per
 * overflows 64 bits or is below 2. */
int cp_partonic_splitmix(cp_handle* h, double sqrt_shat, double alphas, double cmax,
                         double conv, uint64_t seed, uint64_t n_threads, uint64_t k_per,
                         cp_result* out_host);
/* Per-point FP64 weights of the Philox form, points [point0, point0+n). */
int cp_partonic_weights(cp_handle* h, double sqrt_shat, double alphas, double cmax, double conv,
                        uint64_t seed, uint64_t point0, uint64_t n, double* w_dev);

/* ---------------------------------------------------------------- adjoint ---------- */
/* Gradients of the estimator over points [0, n_points) of counter (iter, stream): d sigma and
 * d Var[w] with respect to alpha_s(mZ), k_ren and pT_hat_min (out), and to the 3 x (n_bins + 1)
 * grid edges (host arrays, may be NULL), exact at fixed random numbers (forward mode, FP32).
 * No reference counterpart (the reference has no derivative code); checked against central
 * finite differences of cp_vegas_iteration / cp_point_weights and the FP64 CPU adjoint. */
int cp_adjoint(cp_handle* h, uint64_t n_points, uint32_t iter, uint32_t stream, cp_grad* out_host,
               double* dsigma_dedges_host, double* dvar_dedges_host);
/* One variance-gradient grid update on the device: the adjoint over n_points points, then
 * ln(bin width) -= lr * G / max|G|, G = dVar/dln(width), per dimension (the most sensitive bin
 * changes by exp(+-lr)); the alternative to the classic refinement of cp_vegas_iteration. */
int cp_vegas_gradient_step(cp_handle* h, uint64_t n_points, uint32_t iter, double lr, cp_grad* out_host);
/* Moment order p of the adjoint passes (2 <= p <= 8; default 2): cp_adjoint, the gradient steps
 * and their data-parallel form differentiate the relative p-th moment <w^p>/<w>^p instead of the
 * variance, and the record's var becomes (<w^p>/<w>^p - 1) sigma^2.  A p above 2 weighs the tail
 * of the weights, which sets the unweighting efficiency at a high-quantile w_max; classic VEGAS
 * refinement (a w^2 histogram) has no such choice.  No reference counterpart. */
int cp_vegas_gradient_objective(cp_handle* h, double p);
/* Adjoint passes with (on != 0, default) or without the three parameter tangents (alpha_s(mZ),
 * k_ren, pT_hat cut).  Off, the pass carries only the x tangents the grid needs: the edge
 * gradients, sigma, Var and every variance-gradient step come out the same bit for bit, the
 * parameter derivatives of cp_grad read zero, and the pass runs about twice as fast. */
int cp_adjoint_parameter_tangents(cp_handle* h, int on);
/* The same step data-parallel, with one exchange (the reference shards its passes by point range,
 * cuPythia/common/rng.cuh:5-19, and merges on the host; here the ranks sum device arrays):
 * cp_adjoint_accumulate writes the adjoint sums of this handle's points [offset, offset +
 * n_points) (cp_set_point_offset) to sums_dev, *n_doubles = cp_adjoint_sums_size of them; the
 * caller reduces them over ranks (entry 8, the largest weight, by max, every other entry by sum);
 * cp_vegas_gradient_apply then forms the gradient record of all n_total points and, with lr > 0,
 * takes the grid step (lr = 0: the record only, as cp_adjoint).  One rank: the two calls are
 * cp_vegas_gradient_step. */
int cp_adjoint_sums_size(cp_handle* h, int* n_doubles);
int cp_adjoint_accumulate(cp_handle* h, uint64_t n_points, uint32_t iter, uint32_t stream, double* sums_dev);
int cp_vegas_gradient_apply(cp_handle* h, const double* sums_dev, uint64_t n_total, double lr, cp_grad* out_host);

/* ---------------------------------------------------------------- learned proposal -- */
/* A RealNVP-style flow on [0,1]^3 after the VEGAS map (between it and the base phase-space map):
 * logit, 4 affine couplings (MLP in -> 64 -> 64 -> out, ReLU, BF16 weights and activations on
 * the tensor cores, FP32 accumulation), sigmoid.  No reference counterpart (the reference has no learned proposal).
 * FP32 master parameters: cp_flow_num_params() floats in the layout of cupythia_b200/csrc/cp_flow.cuh. */
int cp_flow_num_params(void);
/* Xavier-uniform weights from the counter RNG with key `seed` (7 in the production recipe),
 * zero biases, zero output layer (the untrained flow is the identity). */
int cp_flow_init(cp_handle* h, uint64_t seed);
int cp_flow_get_params(cp_handle* h, float* params_host, int n);
int cp_flow_set_params(cp_handle* h, const float* params_host, int n);
/* Checkpoint and resume of training (no reference counterpart: the reference keeps no trained
 * state and regenerates events from their counters, cuPythia/05_reproducible_events/
 * repro_events.cu:3-10): the FP32 master parameters, then Adam's first and second moments
 * (cp_flow_state_size() = 3 x cp_flow_num_params() floats), and the number of updates taken,
 * which is also the counter iteration of the next training batch.  Restoring the state saved
 * after k updates and training m more reproduces k + m uninterrupted updates bit for bit. */
int cp_flow_state_size(void);
int cp_flow_get_state(cp_handle* h, float* state_host, int n, int64_t* updates_host);
int cp_flow_set_state(cp_handle* h, const float* state_host, int n, int64_t updates);
/* Flow samples of points [point0, point0+n), counter (iter, stream): out (dev, 16-byte aligned)
 * holds (v0, v1, v2, ln|dv/du|) per point. */
int cp_flow_sample(cp_handle* h, uint64_t point0, uint64_t n, uint32_t iter, uint32_t stream, float* out_dev);
/* Forward kernel used by cp_flow_sample and the flow-routed passes: 0 = tcgen05 MMAs with TMEM
 * accumulators over 128-point tiles (default), 1 = warp-level mma.sync tiles.  Both compute the
 * same map; CP_ERR_TIMEOUT from a flow-routed call means a bounded tensor-core wait expired.  In
 * production passes the tcgen05 forward also hands each point's accept draw to the accept kernel;
 * with the mma.sync forward the accept kernel draws it itself (same values, slower pass). */
int cp_flow_select_kernel(cp_handle* h, int which);
/* Production passes in the flow form (cp_unweight, cp_generate_host) with the tcgen05 forward:
 * on != 0 runs the flow forward, the integrand and the accept step as one kernel per chunk, the
 * flow's output never leaving the SM (no 20-byte-per-point flow buffer); 0 (default) runs the
 * forward over the pass first and the accept kernel on its stored output, which is faster on
 * B200 (17.9 ms against 19.3 ms per 2^27-point pass of the two kernels' work).  Both give the
 * same records, byte for byte, and the same counts; the sums of w and w^2 differ by their FP64
 * addition order. */
int cp_flow_fuse_production(cp_handle* h, int on);
/* Test hook of the failure path of the tcgen05 forward (no reference counterpart): with on != 0
 * the kernel issues no MMA, every bounded wait expires after about one second, the kernel
 * releases its tensor memory and the call returns CP_ERR_TIMEOUT; the handle stays usable. */
int cp_flow_test_stall(cp_handle* h, int on);
/* Routes cp_vegas_iteration / cp_integrate / cp_point_weights / cp_unweight / cp_generate_host
 * through the flow (on = 1) or the Philox words directly (on = 0). */
int cp_flow_enable(cp_handle* h, int on);
/* n_steps Adam steps (learning rate lr) on batches of `batch` points (counter stream 2) drawn
 * through the current flow and VEGAS grid, minimising <w^2>/<w>^2; loss_host (n_steps doubles,
 * may be NULL) receives each batch's value before its update. */
int cp_flow_train(cp_handle* h, int n_steps, uint64_t batch, double lr, double* loss_host);
/* Training objective of cp_flow_train and the data-parallel steps: the relative p-th moment of
 * the weights <w^p>/<w>^p, 2 <= p <= 8 (default 2: <w^2>/<w>^2 = 1 + Var[w]/sigma^2, the weight
 * variance).  A larger p weighs the tail of the weights, which sets the unweighting efficiency at
 * a high-quantile w_max.  The reported batch loss stays <w^2>/<w>^2. */
int cp_flow_set_objective(cp_handle* h, double p);
/* The training gradient of one batch (counter iteration iter, stream 2) without an update. */
int cp_flow_loss_grad(cp_handle* h, uint64_t batch, uint32_t iter, float* grad_host, double* loss_host);
/* Data-parallel training (no reference counterpart): one step of cp_flow_train in three calls,
 * the ranks summing device arrays between them.  The step's batch is points [0, batch_total) of
 * counter iteration = updates so far, stream 2; each rank takes a contiguous share.
 *  1. cp_flow_step_moments: forward and integrand over the batch points [point0, point0 + count);
 *     moments_dev[0..1] = (sum w, sum w^2) over them.  Sum moments_dev over ranks.
 *  2. cp_flow_step_gradient: these points' part of the gradient of the batch loss
 *     <w^2>/<w>^2 (from the summed moments over batch_total points) into grad_dev
 *     (cp_flow_num_params() floats, may be NULL); loss_host (may be NULL) = the batch loss.
 *     Sum grad_dev over ranks.
 *  3. cp_flow_step_update: Adam step (learning rate lr) with the summed gradient (grad_dev NULL:
 *     the handle's own gradient of step 2) and the BF16 repack.
 * The per-point state of step 1 stays in the handle until step 2.  One rank with point0 = 0 and
 * count = batch_total reproduces a step of cp_flow_train bit for bit. */
int cp_flow_step_moments(cp_handle* h, uint64_t point0, uint64_t count, double* moments_dev);
int cp_flow_step_gradient(cp_handle* h, const double* moments_dev, uint64_t batch_total, float* grad_dev,
                          double* loss_host);
int cp_flow_step_update(cp_handle* h, const float* grad_dev, double lr);

/* ---------------------------------------------------------------- device hand-off --- */
/* The reference pipeline's device-resident event record (cuPythia/pipeline/event.cuh:20-31,
 * struct DeviceEvents): the same members in the same order and types, so a DeviceEvents built by
 * the reference's allocEvents (event.cuh:33-48) can be passed by address.  Particle p of event e
 * is at e * maxPart + p; every pointer is device memory owned by the caller. */
typedef struct cp_device_events {
  int nEvents, maxPart, nVar;          /* nVar >= 1 weights per event (slot 0 nominal)      */
  double *px, *py, *pz, *e, *m;        /* [nEvents * maxPart]                               */
  int *pdg, *status, *col, *acol, *mo1, *mo2, *d1, *d2;
  int *nPart;                          /* [nEvents]                                         */
  uint64_t *seed;
  double *scale, *x1, *x2;
  int *flavA, *flavB;
  unsigned char *active;
  double *weight;                      /* [nEvents * nVar]                                  */
} cp_device_events;
/* Hands n records (dev) over to events [e0, e0 + n) of `ev`, on the device, as the reference's
 * hard-process stage fills an event with addParticle (cuPythia/pipeline/generate.cu:30-48,
 * event.cuh:59-71): the two incoming partons (status -21, mothers -1, momentum (0, 0, pz, |pz|))
 * and the two outgoing ones (status 23, mothers 0 and 1), massless, daughters -1, colour tags
 * 500 + the record's colour flow tags (0 = none); nPart = 4, seed = the event key
 * splitmix64(config seed ^ point * 0x9E3779B97F4A7C15) of the record's point (the per-event key
 * of cuPythia/pipeline/generate.cu:33), scale = sqrt(k_fac) pT_hat (the factorisation scale),
 * x1, x2 = the incoming energies over sqrt(s)/2, flavA, flavB = the incoming ids, active = 1, and
 * weight slot 0 = the record weight.  With scale_ratios_dev (6 floats per record, as
 * cp_set_scale_weights writes them) slots 1 .. nVar-1 (nVar <= 7) hold weight x ratio k-1;
 * without it nVar must be 1.  Requires maxPart >= 4 and e0 + n <= nEvents. */
int cp_records_to_device_events(cp_handle* h, const cp_event* records_dev, uint64_t n,
                                const float* scale_ratios_dev, const cp_device_events* ev, uint64_t e0);

/* ---------------------------------------------------------------- record consumers -- */
/* Host-only (no GPU needed).  Colour tags (1..4, 0 = none) of the four partons of a record from
 * its process code and encoded colour flow, as the process's setIdColAcol sets them
 * (pythia8317/src/SigmaQCD.cc:135-342, setColAcol + swapColAcol / swapCol1234). */
int cp_colour_tags(uint16_t process, uint16_t colour, int col[4], int acol[4]);
/* Host-only (no GPU needed).  One event's Sigma2*::setIdColAcol (pythia8317/src/SigmaQCD.cc:
 * 135-148, 195-205, 232-244, 292-304, 331-342) for process `code` 111..115 with incoming
 * (id1, id2): the outgoing flavours (g g -> q qbar: 1 + int(n_quark_new r_flavour), the new
 * flavour its sigmaKin draws) and the colour tags (1..4, 0 = none) of the topology drawn with
 * r_colour in proportion to its kinematic term at tHat/sHat, uHat/sHat, g g -> g g oriented by
 * r_swap, then the swaps for antiquarks and a leading gluon.  The same code as the record
 * builder's colour flow; the Pythia adapter's setIdColAcol calls it with Pythia's own draws.
 * CP_ERR_INVALID for a pair the process does not accept. */
int cp_set_id_col_acol(int code, int id1, int id2, double t_over_s, double u_over_s, int n_quark_new,
                       double r_flavour, double r_colour, double r_swap, int ids_out[4], int col[4], int acol[4]);
/* Writes n host records as a Les Houches Event File 3.0 (the reference's LHE writers:
 * cuPythia/pipeline/lhe_writer.cu:46-70, cuPythia/07_unweighting_lhe/unweight_lhe.cu:74-102):
 * beams and PDF set from cfg, one <init> line per process present with XSECUP = sigma x its
 * share of the event weights (pb), IDWTUP 3; per event IDPRUP = process code, XWGTUP = the
 * record weight (1, or w / w_max for overweight events), SCALUP = sqrt(k_fac) pT_hat,
 * AQCDUP = alpha_s(k_ren pT_hat^2) at first order, colour tags 501.. from cp_colour_tags. */
int cp_write_lhef(const cp_config* cfg, const cp_event* events_host, uint64_t n, double sigma_mb,
                  double sigma_err_mb, const char* path);

/* ---------------------------------------------------------------- measurement ------ */
/* Per-kernel CUDA-event timing of cp_unweight: slot 0 the flow forward, 1 the accept kernel,
 * 2 the record builder (with the slot reduction and the output-offset scan), summed over the
 * pass's chunks; launches3 counts the passes that ran each kernel.  With the fused flow form
 * (cp_flow_fuse_production) slot 1 is the fused forward + accept kernel and slot 0 stays empty.
 * No reference counterpart (the reference times whole stages with a host clock,
 * cuPythia/03_fused_resident_me/fused_gg2gg.cu:93-100). */
int cp_set_kernel_timing(cp_handle* h, int on);
int cp_kernel_times(cp_handle* h, double* ms3_host, uint64_t* launches3_host, int reset);
/* FP32 FMA and MUFU (ex2) throughput of the device from dependency-free microbenchmarks:
 * TFLOP/s (2 per FMA) and Tops/s.  No reference counterpart: the integrand's roofline
 * denominators (it is SIMT FP32 / SFU work). */
int cp_measure_peaks(cp_handle* h, double* fp32_tflops_host, double* mufu_tops_host);

#ifdef __cplusplus
}
#endif
#endif
