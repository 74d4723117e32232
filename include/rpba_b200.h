/*
 * rpba_b200.h -- C ABI of the B200 robust bundle adjuster.
 *
 * The library replaces the global robust bundle adjustment of RPBA
 * (class LSA, rbacore.cpp) behind the reference's own entry points:
 *
 *   InputBlock   rpba.cpp:180-284      -> rpba_input_block
 *   OutputBlock  rpba.cpp:288-338      -> rpba_output_block
 *   CalcPLSA     rpba.h:693-703,
 *                rpbacore.cpp:28-531   -> rpba_calc_plsa
 *   EvalLSA      rpbacore.cpp:882-941  -> rpba_calc_plsa with exteval=1
 *
 * plus a handle API (rpba_create / rpba_solve / rpba_get_state /
 * rpba_destroy) that keeps a problem resident on the GPU between solves.
 *
 * Every signature uses plain C types: pointers, sizes and status codes.
 * No exception crosses the boundary.  All host buffers belong to the
 * caller; device memory belongs to the handle.
 *
 * Data layout of a block (mirrors the containers CalcPLSA takes):
 *   pmat        [n_images][3][4]  float, row major, PMat = [R | t]
 *   K           [n_images][3][3]  float, row major, Camera::K
 *   distpara    [n_images][2]     float, Camera::distpara (k1', k2')
 *   XX          [n_points][3]     float, point coordinates (XX rows 0..2)
 *   img_obs_off [n_images+1]      offsets of image slots (xg columns)
 *   xg          [n_slots][2]      float, xg(0..1, slot), already negated
 *                                 as InputBlock stores them (rpba.cpp:268-272)
 *   wx, wy, wxy [n_slots]         float weights per slot
 *   pt_obs_off  [n_points+1]      offsets into the per-point track lists
 *   pt_obs_image, pt_obs_slot     [pt_obs_off[n_points]] IMAPNR entries
 *                                 (image, pointnr) of pointXXv (rpba.h:88-93)
 * n_slots = img_obs_off[n_images].  The track lists are rewritten in place by
 * a solve (robustly deleted observations are removed, dropped points get an
 * empty list), exactly as CalcPLSA rewrites pointXXvio.
 */
#ifndef RPBA_B200_H_
#define RPBA_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The reference reports errors as "BA-Error: ..." text in its
 * log stream and returns; the codes name the same cases. */
typedef enum rpba_status {
  RPBA_OK = 0,
  RPBA_ERR_ARG = 1,             /* invalid argument or inconsistent block   */
  RPBA_ERR_CUDA = 2,            /* CUDA runtime error                       */
  RPBA_ERR_NO_OBS_IMAGE = 3,    /* image without observations, rbacore.cpp:415-424 */
  RPBA_ERR_LOW_REDUNDANCY = 4,  /* redundancy < 0, rbacore.cpp:470-476      */
  RPBA_ERR_NAN_STEP = 5,        /* NaN/Inf in the step, rbacore.cpp:541-546 */
  RPBA_ERR_DEVICE_TIMEOUT = 6,  /* a bounded device-side wait expired       */
  RPBA_ERR_IO = 7,              /* file could not be read or written        */
  RPBA_ERR_UNSUPPORTED = 8,     /* input the GPU path does not accept       */
  RPBA_ERR_NO_DEVICE = 9,       /* no CUDA device / library not usable      */
  RPBA_ERR_SOLVER = 10,         /* direct factorisation failed (not SPD)    */
  RPBA_ERR_TOO_LARGE = 11,      /* input exceeds a fixed-size scratch area  */
  RPBA_ERR_COMM = 12            /* a collective between ranks failed        */
} rpba_status;

typedef struct rpba_block {
  int32_t n_images;
  int32_t n_points;
  float *pmat;
  float *K;
  float *distpara;
  float *XX;
  int32_t *img_obs_off;
  float *xg;
  float *wx;
  float *wy;
  float *wxy;
  int32_t *pt_obs_off;
  int32_t *pt_obs_image;
  int32_t *pt_obs_slot;
} rpba_block;

/* Linear solver for the reduced camera system. */
enum {
  RPBA_SOLVER_PCG = 0,      /* block-Jacobi PCG with the reference's stop rule
                               (SparsePCG, rbacore.cpp:1807-1914): the drop-in */
  RPBA_SOLVER_DIRECT = 1,   /* dense Cholesky of the reduced camera system     */
  RPBA_SOLVER_LEARNED = 2   /* PCG with a learned block-preconditioner correction */
};

/* Arithmetic of the assembly kernels. */
enum {
  RPBA_PREC_FP64 = 0,
  RPBA_PREC_MIXED = 1       /* FP32 Jacobians / Schur assembly, FP64 cost and refinement */
};

typedef struct rpba_options {
  int32_t robust;        /* parameters: Robust                              */
  int32_t exteval;       /* parameters: Exteval (evaluate only, EvalLSA)    */
  int32_t threads;       /* parameters: Threads: selects the partitioned or the
                            global branch as the reference does (see
                            rpba_calc_plsa); < 1: the host's threads        */
  int32_t k2, k4, f;     /* parameters: k2, k4, f  -> addflags[0..2]        */
  int32_t solver;        /* RPBA_SOLVER_*                                   */
  int32_t precision;     /* RPBA_PREC_*                                     */
  int32_t max_lm_iterations; /* < 0: the reference's own stop rule only;
                                >= 0: additionally stop after this many
                                linear solves in total                      */
  int32_t pcg_max_iterations; /* <= 0: the reference's cap max(n_unknowns, 1000) */
  double pcg_tolerance;  /* learned/direct-checked PCG relative tolerance
                            (0: the reference's 1e5 decrease rule)          */
  int32_t device;        /* CUDA device ordinal                             */
  int32_t verbose;
  int32_t coarse_aggregates; /* learned solver's coarse space: 0 = default
                                (up to 148 camera aggregates), > 0 = at most
                                this many (<= 200), < 0 = none (block-Jacobi
                                part only)                                  */
} rpba_options;

/* Per-pass summary; index 0 = robust pass, 1 = refinement pass. */
typedef struct rpba_report {
  float sigma0_in[2];    /* sqrtf(sig0in * ihw2)                            */
  float sigma0_out[2];   /* sqrtf(sig0old * ihw2)                           */
  int32_t redundancy[2];
  int32_t nrobs[2];
  int32_t nrunknowns[2];
  int32_t itt[2];        /* the reference's ITT counter at the end of a pass */
  int32_t passes_done;
  int32_t linear_solves; /* CalcBundleSep calls                             */
  int64_t pcg_iterations;/* total PCG iterations                            */
  int32_t pcg_fallbacks; /* learned PCG runs that fell back to the direct solve */
  int32_t coarse_rebuilds; /* learned PCG solves repeated with a rebuilt coarse operator */
  int32_t obs_deleted;   /* observations removed by RobustDelete            */
  int32_t points_deleted;
  int32_t points_used;   /* points kept by PointXXvIn                       */
  double cost;           /* FP64 sum of w-weighted squared residuals, final state */
  double rms;            /* sqrt(sum |r|^2 / n_alive) in pixels, final state */
  float exteval_sigma0;  /* ITTTT value, rpbacore.cpp:938                   */
  int64_t exteval_nrobs;
  int64_t exteval_redundancy;
  double solve_seconds;  /* device time of the solve (CUDA events)          */
  double setup_seconds;  /* host+device time before the first LM iteration  */
  int32_t status;
  int64_t kernel_launches; /* launches of this library's kernels in the solve */
} rpba_report;

typedef struct rpba_handle rpba_handle;

/* Human-readable name of a status code (the reference reports its errors
 * as "BA-Error: ..." lines instead, rbacore.cpp:415-424, 470-476, 541-548). */
const char *rpba_status_string(int32_t status);

/* Version string of the library build (no counterpart in the reference). */
const char *rpba_version(void);

/* The reference's branch rule of CalcPLSA (rpbacore.cpp:79-92): the
 * partition count min(threads, iround(n_images / 70)) when it is above 1,
 * there are more than five images and exteval is 0; otherwise 1 (the global
 * LSA).  threads < 1: the host's hardware threads.  Host code, no device. */
int32_t rpba_partition_count(int32_t n_images, int32_t threads, int32_t exteval);

/* InputBlock (rpba.cpp:180-284): parse a BAL text file into a block whose
 * arrays are allocated by the library (free with rpba_block_free).  Same
 * float quantisation, sign flip of the observations and k24out scaling. */
int32_t rpba_input_block(const char *path, int32_t nraddpar, int32_t k24out,
                         rpba_block *out);
/* Frees the arrays rpba_input_block allocated (no counterpart in the
 * reference, whose block lives in std::vector and Eigen members). */
void rpba_block_free(rpba_block *blk);

/* OutputBlock (rpba.cpp:288-338): write a block as BAL text. The per-point
 * track lists are sorted by image in place, as the reference does. */
int32_t rpba_output_block(const char *path, rpba_block *blk, int32_t k24out);

/* CalcPLSA (rpbacore.cpp:28-531): adjust (or, with opt->exteval, evaluate)
 * the block in place on the GPU.  The log receives the lines the reference
 * writes to its ostream ("Sigma0: ...", "BA-Error: ...", "ITTTT: ...");
 * pass log=NULL to skip it.  rep may be NULL.  The branch follows the
 * reference's rule (rpbacore.cpp:79-92, rpba_partition_count below): with
 * min(threads, iround(n_images / 70)) > 1 and more than five images the
 * partitioned RPBA runs (rpba_calc_plsa_parallel over rpba_partition_images,
 * the reference's "#threads", "Partitioning runtime" and "Thread:" lines at
 * the head of the log; rep then carries only the status), else the global
 * LSA.  threads < 1 means the host's hardware threads, as Threads = 0 does
 * in the reference's parameters file (rpba.cpp:88-89).  The partitioned
 * branch runs the drop-in form (FP64, PCG or direct); the mixed and learned
 * forms always solve the whole block. */
int32_t rpba_calc_plsa(rpba_block *blk, const rpba_options *opt, char *log,
                       size_t log_cap, rpba_report *rep);

/* Handle API: upload once, solve many times from the uploaded state.  The
 * global branch of CalcPLSA in steps (rpbacore.cpp:514-527): rpba_create is
 * `new LSA(...)` (the constructor with PointXXvIn and PrepareCameras,
 * rbacore.cpp:37-125, 670-700, 1918-1974), the problem copied to the GPU. */
int32_t rpba_create(rpba_handle **h, const rpba_block *blk,
                    const rpba_options *opt);
/* LSA::Adjust (rbacore.cpp:333-616) from the uploaded state. */
int32_t rpba_solve(rpba_handle *h, rpba_report *rep);
/* Copy the adjusted state into blk (pmat, K, distpara, XX, track lists):
 * OutputLSAc with PointXXvOut (rbacore.cpp:644-666, 1978-2010). */
int32_t rpba_get_state(rpba_handle *h, rpba_block *blk);
/* Copy the log of the last solve (NUL terminated, truncated to cap): what
 * Adjust writes to CalcPLSA's ostream (rpbacore.cpp:28-39). */
int32_t rpba_get_log(rpba_handle *h, char *log, size_t cap);
/* Per-observation back-projection errors of the uploaded block, in track
 * order (dx, dy as double), as EvalLSA/CalcCorrPointMulti compute them
 * (rpbacore.cpp:778-837, 882-941).  resid has 2*pt_obs_off[n_points]
 * entries; entries of points with fewer than two observations are 0.
 * The handle must have been created with opt->exteval = 1 (RPBA_ERR_ARG
 * otherwise), as Exteval is a mode of CalcPLSA (extevalflag). */
int32_t rpba_exteval(rpba_handle *h, double *resid, rpba_report *rep);
/* The float sum of v[0..n) accumulated left to right, one rounding per
 * addition -- the way the reference accumulates its cost and weight sums
 * (rbacore.cpp:727, 881, 1327) -- computed on the GPU with a bitwise equal
 * result (values must be finite and >= 0).  No counterpart in the reference;
 * exposed for verification. */
int32_t rpba_float_sequential_sum(const float *v, int64_t n, int32_t device, float *out);

/* ---- learned block-Jacobi correction (RPBA_SOLVER_LEARNED) ----
 * The reference preconditions its PCG with the inverse diagonal blocks of
 * the reduced camera system (rbacore.cpp:1841).  The learned form scales
 * each block's inverse per parameter, C_k = diag(s) S_kk^-1 diag(s), with s
 * from a 2-layer network (19 -> 64 tanh -> 9) over scale-free features of
 * the assembled system; weights are BF16-rounded for inference. */
#define RPBA_PRECOND_WEIGHTS 1865 /* W1[64][19], b1[64], W2[9][64], b2[9] */

typedef struct rpba_train_options {
  int32_t steps;        /* Adam steps (0: 300)                           */
  int32_t batch;        /* unused: every step uses the whole set         */
  float lr;             /* learning rate (0: 3e-3)                       */
  int32_t probes;       /* random right-hand sides per system besides the
                           LM step's own                                 */
  int32_t max_samples;  /* block-row capacity of the training set (0: 2^18) */
  uint64_t seed;
} rpba_train_options;

typedef struct rpba_train_report {
  int32_t samples;      /* block rows in the training set                */
  int32_t steps;
  float loss_initial;   /* mean of ln(u^T S u) - 2 ln(b^T u), untrained (s = 1) */
  float loss_final;
  int32_t systems;      /* recorded reduced camera systems              */
  float err_initial;    /* mean relative A-norm error after one
                           preconditioned step on the LM right-hand sides */
  float err_final;
} rpba_train_report;

/* Train the preconditioner network on the reduced camera systems that the
 * direct solver's own LM iterations assemble on the given scenes (solved with
 * *opt, solver forced to DIRECT).  Objective: the relative A-norm error left
 * after one preconditioned step, over the LM right-hand sides and random
 * ones.  weights receives RPBA_PRECOND_WEIGHTS floats.  No counterpart in the
 * reference. */
int32_t rpba_train_preconditioner(const rpba_block *scenes, int32_t nscenes, const rpba_options *opt,
                                  const rpba_train_options *topt, float *weights,
                                  rpba_train_report *rep);
/* Use these weights in the handle's RPBA_SOLVER_LEARNED solves (NULL: plain
 * block-Jacobi under the same stopping rule).  n = RPBA_PRECOND_WEIGHTS.
 * No counterpart in the reference. */
int32_t rpba_set_preconditioner(rpba_handle *h, const float *weights, int32_t n);

/* A training set in host memory (diagonally scaled, block-diagonal union of
 * systems) for rpba_precond_loss_grad. */
typedef struct rpba_precond_set {
  int32_t rows, systems, probes, nent, nblocks;
  const float *features;   /* [rows][19]                                  */
  const float *sinv;       /* [rows][81] D^1/2 S_kk^-1 D^1/2             */
  const float *b;          /* [probes][rows][9]                           */
  const float *xs;         /* [rows][9] solution of right-hand side 0     */
  const int32_t *np, *sys; /* [rows] parameter count, system index        */
  const int32_t *rowoff;   /* [rows + 1]                                  */
  const int32_t *ent_col;  /* [nent] column row                           */
  const int32_t *ent_blk;  /* [nent] block index, bit 31: transposed      */
  const float *blocks;     /* [nblocks][81] D^-1/2 S D^-1/2               */
  const int32_t *sys_row;  /* [systems + 1]                               */
  const float *uc;         /* [probes][rows][9] coarse part of the
                              preconditioned right-hand sides, or NULL     */
} rpba_precond_set;
/* Caller-allocated host buffers for rpba_record_systems: capacities in,
 * counts out; the arrays have the layout of rpba_precond_set; NULL arrays
 * are skipped. */
typedef struct rpba_precond_buffers {
  int32_t rows_cap, ents_cap, blocks_cap, systems_cap;
  int32_t rows, systems, probes, nent, nblocks;
  float *features, *sinv, *b, *xs, *blocks, *uc;
  int32_t *np, *sys, *rowoff, *ent_col, *ent_blk, *sys_row;
} rpba_precond_buffers;
/* The training set rpba_train_preconditioner would train on (the direct
 * solver's systems for the scenes, diagonally scaled), copied to the host:
 * for checking the recording and the training objective independently.
 * RPBA_ERR_TOO_LARGE when a capacity is short (the counts say how much is
 * needed).  No counterpart in the reference. */
int32_t rpba_record_systems(const rpba_block *scenes, int32_t nscenes, const rpba_options *opt,
                            const rpba_train_options *topt, rpba_precond_buffers *out);

/* Training loss and its gradient for `weights`, computed by the GPU's
 * training kernels (for checking against an independent implementation).
 * No counterpart in the reference. */
int32_t rpba_precond_loss_grad(const rpba_precond_set *set, const float *weights, float *loss, float *grad);

/* Allocation-free form of rpba_float_sequential_sum, for callers that must
 * not have a library call cudaMalloc or cudaFree -- an application that hands
 * out all device memory from its own fixed-budget pool, or a latency-critical
 * loop that cannot take the device-wide synchronisation cudaFree implies.
 * d_v and d_out are device pointers on the calling thread's current device;
 * the work is enqueued on `stream` (a cudaStream_t; NULL = legacy default
 * stream) and the call returns without waiting for it.  Scratch lives in one
 * static device array of the library (about 20 KB, held by every GPU that
 * loads the library until the process exits), which caps n at 4,194,304 on
 * every device: larger n returns RPBA_ERR_TOO_LARGE.  The first call on a
 * device (and the first after cudaDeviceReset or with another context
 * current) looks up that array's device address (a blocking runtime query),
 * so make the first call on each device before any stream capture.
 * The call first sets *d_out to NaN; the kernel overwrites it with the sum.
 * A NaN left in *d_out after the stream has run means the call failed on the
 * device (a bounded grid-barrier wait ran out); a valid sum of finite inputs
 * >= 0 is never NaN.  All calls share the one array: calls that overlap on
 * the GPU (different streams, or different host threads, on the same
 * device) race and must be serialised by the caller.  No counterpart in the
 * reference. */
int32_t rpba_float_sequential_sum_noalloc(const float *d_v, int64_t n, float *d_out, void *stream);

/* Per-point refinement against fixed cameras: CalcLSAXMulti
 * (rpbacore.cpp:536-773), the per-point bundle adjustment of the
 * reference's parallel RPBA, for every point of the block at once on the GPU
 * (one thread per point).  robustmode 0: plain; 1: also return each
 * observation's weighted squared residual in sig0v (the statistic of the
 * per-image thresholds); 2: observations whose residual exceeds 16 x the
 * image's threshold sig0w[image] are down-weighted and dropped (keep = 0).
 * weight_only: evaluate and accumulate only (the reference's first pass).
 * Outputs per point: the refined point (XX_out, 3 doubles; the input when the
 * point did not converge) and conv; per track entry (pt_obs_off order): keep
 * and sig0v; totals: sig0io and redundancy as the reference accumulates them.
 * rpba_triangulate_parts below also forms the per-partition weight blocks. */
typedef struct rpba_tri_options {
  int32_t robustmode;   /* 0, 1 or 2                                        */
  int32_t weight_only;  /* weightonlyflag                                   */
  int32_t device;
} rpba_tri_options;
/* CalcLSAXMulti (rpbacore.cpp:536-773) for every point, as described above. */
int32_t rpba_triangulate(const rpba_block *blk, const float *sig0w, const rpba_tri_options *opt, double *XX_out,
                         uint8_t *keep, float *sig0v, uint8_t *conv, double *sig0io, int64_t *redundancy);

/* rpba_triangulate with the camera partition of the parallel RPBA
 * (part[image] in 0 .. nparts - 1, e.g. from rpba_partition_images): also the
 * per-partition weight blocks CalcLSAXMulti forms with wxyflag
 * (rpbacore.cpp:579-590, 612-622, 663-672, the w3dvivv of rpbacore.cpp:
 * 370-380): w3d[n_points][nparts][6] = (XX, YY, ZZ, XY, XZ, YZ) of the
 * normal matrix of the point's observations outside partition i, for every
 * partition i that sees the point (one partition: all observations),
 * undamped, from the accepted iteration; zero elsewhere. */
int32_t rpba_triangulate_parts(const rpba_block *blk, const float *sig0w, const rpba_tri_options *opt,
                               const int32_t *part, int32_t nparts, double *XX_out, uint8_t *keep, float *sig0v,
                               uint8_t *conv, double *sig0io, int64_t *redundancy, float *w3d);

/* One GCP-mode step of the LSA: the per-partition call of the parallel
 * RPBA, replacing LSA::InputLSAP + Adjust(false, os, true, 0, W3ijiv[it],
 * true, gcpdatav[it]) + OutputLSAP (rpbacore.cpp:212-229; rbacore.cpp:
 * 233-331, 333-616, 620-639).  blk holds the partition's images and its
 * points; every camera is free (no scale camera); point p with
 * gcpinfo[p] > -1 is held at gcpdata[gcpinfo[p]] (3 doubles) by a 3-D prior
 * whose weight block (6 floats: XX YY ZZ XY XZ YZ) is the next row of W3 in
 * the order of the points the LSA keeps (the reference's gcpnum); a point
 * is kept with two or more observations, or with one and gcpinfo > 0.  The
 * additional parameters count ncam_total times in the redundancy (the
 * reference's nrcameras).  pmat_d: the cameras in double precision (null:
 * blk->pmat).  One damped step (multfact 1e-4), stored unconditionally,
 * without robust reweighting; the log gets the Sigma0 and Sigma0AO lines.
 * Outputs: blk (cameras, points, tracks as rpba_get_state), pmat_d_out
 * (12 doubles per image) and point_used (1 for the points the step took),
 * each optional.  FP64 only (RPBA_PREC_FP64; RPBA_SOLVER_PCG with the
 * reference's stop rule, or RPBA_SOLVER_DIRECT).  Calls from several host
 * threads may overlap: each has its own device memory and stream, and their
 * cooperative kernels take turns (one process-wide lock). */
int32_t rpba_lsa_gcp_step(rpba_block *blk, const rpba_options *opt, const int32_t *gcpinfo, const float *W3,
                          int32_t n_w3, const double *gcpdata, int32_t n_gcp, int32_t ncam_total,
                          const double *pmat_d, double *pmat_d_out, uint8_t *point_used, rpba_report *rep,
                          char *log, size_t cap);

/* The parallel RPBA: the partitioned branch of CalcPLSA (rpbacore.cpp:
 * 100-510), which the reference takes when min(Threads, iround(images /
 * 70)) > 1.  part[image] in 0 .. nthreads - 1 (rpba_partition_images
 * replaces the reference's METIS cut).  Each outer iteration after the
 * first takes one rpba_lsa_gcp_step per partition -- concurrently, on host
 * threads (at most one per core), as the reference's OpenMP loop does; the
 * result does not depend on their order -- and merges with
 * CalcLSAXMulti on the GPU (robust thresholds when the robust stage starts,
 * robust deletion, weight blocks of the shared points); the best iteration
 * (lowest sigma0) is written back to blk (cameras, points, tracks), as the
 * reference writes pointXXvold, PMatricesdold, XXdold and camerasold
 * (rpbacore.cpp:498-507).  stats (optional): {sigma0 of the best
 * iteration, outer iterations}.  FP64 only, like rpba_lsa_gcp_step. */
int32_t rpba_calc_plsa_parallel(rpba_block *blk, const rpba_options *opt, int32_t nthreads, const int32_t *part,
                                char *log, size_t cap, double *stats);

/* The two steps of the parallel RPBA's loop: the partition step (the
 * signature of rpba_lsa_gcp_step) and the merge pass (CalcLSAXMulti over
 * every point of b with the cameras Pd, 12 doubles per image; part null:
 * no weight blocks; s0_pt / red_pt: every point's contribution to the sum
 * and to the redundancy, as the reference's per-thread sums take them). */
typedef int32_t (*rpba_gcp_step_fn)(rpba_block *blk, const rpba_options *opt, const int32_t *gcpinfo,
                                    const float *W3, int32_t n_w3, const double *gcpdata, int32_t n_gcp,
                                    int32_t ncam_total, const double *pmat_d, double *pmat_d_out,
                                    uint8_t *point_used, rpba_report *rep, char *log, size_t cap);
typedef int32_t (*rpba_merge_fn)(const rpba_block *b, const double *Pd, const float *sig0w, int32_t robustmode,
                                 int32_t weight_only, const int32_t *part, int32_t nparts, int32_t device,
                                 double *XX_out, uint8_t *keep, float *sig0v, uint8_t *conv, float *w3d,
                                 double *s0_pt, int32_t *red_pt);
/* rpba_calc_plsa_parallel's loop with both steps supplied by the caller
 * (the host-side check of the loop binds CPU implementations of them); no
 * counterpart in the reference. */
int32_t rpba_calc_plsa_parallel_hosted(rpba_block *blk, const rpba_options *opt, int32_t nthreads,
                                       const int32_t *part, char *log, size_t cap, double *stats,
                                       rpba_gcp_step_fn step, rpba_merge_fn merge);

/* All-gather between the ranks of a multi-rank call: every rank passes
 * `bytes` bytes (the same count on every rank) and receives every rank's,
 * in rank order, at recv (world x bytes); returns 0 on success.  Every rank
 * calls it the same number of times.  The caller supplies it (over
 * torch.distributed, MPI, ...): the library has no transport of its own. */
typedef int32_t (*rpba_allgather_fn)(void *ctx, const void *send, uint64_t bytes, void *recv);

/* rpba_calc_plsa_parallel over several ranks (one process per GPU; this
 * rank's GPU is opt->device): one scene, its partitions dealt to the ranks
 * (largest first to the least-loaded rank).  Every rank holds the whole
 * block and runs the whole loop: the partition steps of its own partitions
 * on its GPU, then, after each round of steps, two all-gathers (the sizes,
 * then the steps' results: status, log, the partitions' cameras, which
 * points each step took), after which every rank merges all points on its
 * GPU and takes the same decisions.  Every rank ends with the same block,
 * log and stats, equal to the one-rank call's.  A failed all-gather returns
 * RPBA_ERR_COMM (on every rank whose collective failed); a partition step's
 * failure is returned by every rank, after the exchange that reports it.
 * Like the reference's partitioned branch (rpbacore.cpp:100-510), with its
 * OpenMP threads replaced by ranks and threads; no single counterpart. */
int32_t rpba_calc_plsa_parallel_ranks(rpba_block *blk, const rpba_options *opt, int32_t nthreads,
                                      const int32_t *part, char *log, size_t cap, double *stats, int32_t rank,
                                      int32_t world, rpba_allgather_fn allgather, void *ctx);
/* The same with both steps supplied by the caller (the host-side check of
 * the multi-rank loop); no counterpart in the reference. */
int32_t rpba_calc_plsa_parallel_ranks_hosted(rpba_block *blk, const rpba_options *opt, int32_t nthreads,
                                             const int32_t *part, char *log, size_t cap, double *stats,
                                             rpba_gcp_step_fn step, rpba_merge_fn merge, int32_t rank,
                                             int32_t world, rpba_allgather_fn allgather, void *ctx);

/* Camera partition of the reference's parallel RPBA: replaces
 * PartitionpointXXv (rpbacore.cpp:945-1037), which cuts the images'
 * covisibility graph (an edge where two images share a point observed at
 * least twice; vertex weight floor(BM^0.3333), BM the sum of the track
 * lengths of the image's points) with METIS_PartGraphRecursive and
 * METIS_OPTION_CONTIG.  METIS is not available here: the cut is this
 * library's own deterministic recursive bisection, every part contiguous on
 * a connected graph.  part[n_images] receives each image's part,
 * 0 .. nparts - 1.  Host code; needs no GPU. */
int32_t rpba_partition_images(const rpba_block *blk, int32_t nparts, int32_t *part);

/* Batched form: many independent scenes of uneven size on one GPU.  Every
 * scene is solved as rpba_calc_plsa would solve it (in place; reports[i] and
 * status[i] per scene); `workers` scenes run at once, each on its own stream,
 * so that the kernels of small scenes fill the GPU together (workers <= 0:
 * chosen by timing a sample of the batch, reported in br->workers).  The
 * cooperative kernels of different scenes run one at a time.  Returns
 * RPBA_ERR_SOLVER when any scene failed (see status).  No counterpart in the
 * reference (its parallel form partitions one scene, rpbacore.cpp:100-510). */
typedef struct rpba_batch_report {
  double seconds;            /* wall time of the batch, tuning excluded       */
  double scenes_per_second;
  double tune_seconds;       /* wall time spent choosing the worker count     */
  int32_t workers;           /* scenes solved concurrently                    */
  int32_t failed;            /* scenes whose status is not RPBA_OK            */
} rpba_batch_report;
/* The batched form described above (no counterpart in the reference). */
int32_t rpba_solve_batch(rpba_block *blocks, int32_t n, const rpba_options *opt, int32_t workers,
                         rpba_report *reports, int32_t *status, rpba_batch_report *br);

/* Per-kernel device time of the last solve as a JSON object
 * {"name": {"launches": n, "ms": t}, ...}; filled only when the handle was
 * created with rpba_options.verbose bit 1 (value 2) set.  No counterpart in
 * the reference (its only instrument is a wall-clock print, rpba.cpp:140). */
int32_t rpba_kernel_stats(rpba_handle *h, char *json, size_t cap);
/* The inverse of a dense symmetric positive definite n x n matrix (row
 * major, host buffers; the lower triangle of A is read), computed by the
 * library's tiled Cholesky factorisation and inverse on the FP64 tensor
 * cores -- the kernel that inverts the learned solver's coarse operator --
 * for checking it against an independent implementation.
 * RPBA_ERR_SOLVER when A is not positive definite.  No counterpart in the
 * reference. */
int32_t rpba_spd_inverse(const double *A, int32_t n, double *Ainv, int32_t device);
/* Test hook of the bounded device waits.  With extra_ctas = 1 every grid
 * barrier of the handle's persistent PCG waits for one CTA more than the
 * launch has -- an arrival that never comes -- for at most timeout_ns
 * (1 ms .. 2 s), so the wait runs out, the kernel sets the error word and
 * returns, and the solve ends with RPBA_ERR_DEVICE_TIMEOUT; the handle stays
 * usable.  (0, 0) restores normal operation (the default 2 s limit).  The
 * reference has no device waits and no counterpart; its error exits are
 * the BA-Error lines of rbacore.cpp:415-424, 470-476 and 541-546. */
int32_t rpba_debug_barrier_timeout(rpba_handle *h, int32_t extra_ctas, int64_t timeout_ns);
/* Releases a handle and its device memory (`delete LSA1`,
 * rpbacore.cpp:525). */
void rpba_destroy(rpba_handle *h);

#ifdef __cplusplus
}
#endif

#endif /* RPBA_B200_H_ */
