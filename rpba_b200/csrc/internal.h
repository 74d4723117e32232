// internal.h -- device-side state of one global LSA and the launchers of
// its kernels.  Host code (solver.cu) owns the buffers; kernels receive the
// plain-pointer view DevLSA by value.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "../../include/rpba_b200.h"
#include "common.cuh"

namespace rpba {

// Per-observation linearisation record (doubles):
//   [0..17]  Bc (2 x 9 camera Jacobian, row major)
//   [18..23] G  = W Jp (2 x 3); in the FP32 form H = G L^-T, V = L L^T
//   [24..25] e  = W d
//   [26..28] M  = W - G V^-1 G^T  (M00, M01, M11)
//   [29..30] m  = e - G V^-1 g
constexpr int REC = 32;
// Per-point record: V^-1 (9, row major) and g (3); in the FP32 form L^-1
// (9, row major, lower) and q = L^-1 g.
constexpr int PREC = 12;

struct DevLSA {
  int nimg, npts, nobs;
  int nrioff, begini, normcamera, addmask, nadd, robust;
  int minimagenrdel;
  double defdiff;
  const int *camparv;  // [nimg+1]
  int *gauge;          // [4] esvm0, esvm1, esvmaxm
  double *Pacc;        // [nimg*12] accepted PMatrices
  double *Kc;          // [nimg*9]  accepted intrinsics (cameras)
  double *dc;          // [nimg*2]
  CamState *camn;      // [nimg]    trial cameras (camerasnew, eRMnew, ePCnew)
  double *Rb, *PCb;    // [nimg*9], [nimg*3] pass-start eRM / ePC
  // observations in track order (point major)
  int *o_cam, *o_slot, *o_pt;
  float2 *o_xg;
  float4 *o_wold, *o_w;
  float *o_s0rmv, *o_cost, *o_wterm;
  uint8_t *o_flag, *o_flagnew;
  int *pt_off, *pt_id;
  // state
  double *XPM, *XPMn, *x;
  // linearisation
  double *rec, *ptV;
  // camera-grouped observation order (the reference's nro order)
  int *camlist, *coff;
  // mixed-precision form: FP32 records, point blocks and reduced camera
  // system (the FP64 arrays above and below are then unused)
  float *rec32, *ptV32, *blocks32;
  // reduced camera system
  double *blocks;  // [(nimg + nboff) * 81], diagonal blocks first
  double *rhs;     // [nimg * 9]
  int nboff;
  const int *boff;     // [nboff + 1] contribution ranges of the off-diagonal blocks
  const int2 *contrib; // (obs in the row camera, obs in the column camera)
  const int *rowoff;   // [nimg + 1]
  const int2 *ent;     // (column camera, block index | 0x80000000 if transposed)
  // SpMV work items: runs of <= 3 entries of one row.  In the FP32 form the
  // items cover each row's diagonal and normal entries only: the SpMV reads
  // every off-diagonal block once and forms both of its products.
  int nitems;
  const int *row_item_off;  // [nimg + 1]
  const int4 *item_meta;    // (row, first entry, end entry, 0)
  const int2 *rowspan;      // [nimg] (diagonal entry, end entry) of each row
  float *tpart;             // [nboff * 16] FP32 form: transposed block products, column order
  const int4 *bidx;         // FP32 form: (row, column, transposed slot, 0) of every block, storage order
  const int *firstN;        // [nimg + 1] first off-diagonal block of every row
  const int *firstT;        // [nimg + 1] first transposed slot of every row (blocks in its column)
  int *err;            // device error word
  // Test hook of the bounded waits (rpba_debug_barrier_timeout): the PCG's
  // grid barriers wait for bar_extra CTAs more than the launch has, for at
  // most bar_timeout_ns (0: the default limit).  Both 0 in normal use.
  unsigned bar_extra = 0;
  unsigned long long bar_timeout_ns = 0;
  // GCP mode of the parallel RPBA's per-partition LSA (ao = 1): every
  // camera free (no scale camera, camera 0 with a full block), and the
  // points shared with other partitions held by 3-D priors.  Per point
  // (local order): the GCP index into gcpdata, or -1, and the row of its
  // weight block in W3 (6 floats: XX YY ZZ XY XZ YZ).  ao = 0 leaves every
  // kernel as in the global LSA.
  int ao = 0;
  int n_w3 = 0;
  const int *pt_gcp = nullptr, *pt_w3row = nullptr;
  const float *W3 = nullptr;
  const double *gcpdata = nullptr;
};

// Storage stride (elements) of one 9x9 block of the reduced camera system in
// the FP64 and the FP32 form (row major, packed).
constexpr int BS64 = 81, BS32 = 81;

// Element e of block b of the reduced camera system in either form (for
// set-up kernels; the PCG's SpMV is compiled for each form).
__device__ __forceinline__ double blk_at(const DevLSA &L, size_t b, int e) {
  return L.blocks32 ? (double)L.blocks32[b * BS32 + e] : L.blocks[b * BS64 + e];
}
__device__ __forceinline__ void load_block(const DevLSA &L, size_t b, double out[81]) {
  if (L.blocks32)
    for (int e = 0; e < 81; ++e) out[e] = (double)L.blocks32[b * BS32 + e];
  else
    for (int e = 0; e < 81; ++e) out[e] = L.blocks[b * BS64 + e];
}

// ---- launchers (kernels.cu)
void launch_cost(const DevLSA &L, const double *XM, bool srmv, cudaStream_t s);
void launch_seq_sum(const float *v, int n, float *out, cudaStream_t s);
void launch_point_pass(const DevLSA &L, double multfact1, cudaStream_t s);
void launch_camera_pass(const DevLSA &L, double multfact1, cudaStream_t s);
void launch_pair_pass(const DevLSA &L, cudaStream_t s);
void launch_backsub(const DevLSA &L, const double *xsol, cudaStream_t s);
void launch_xcam(const DevLSA &L, const double *xsol, cudaStream_t s);
void launch_update(const DevLSA &L, int nunk, cudaStream_t s);
void launch_decode(const DevLSA &L, const double *XM, cudaStream_t s);
void launch_encode(const DevLSA &L, cudaStream_t s);
void launch_store(const DevLSA &L, int xpmsize, cudaStream_t s);
void launch_prepare_weights(const DevLSA &L, cudaStream_t s);
void launch_reweight(const DevLSA &L, int iflag, float *vals_scratch, float *sig00v, int *nflag,
                     cudaStream_t s);
void launch_final_cost(const DevLSA &L, double *partials, int nparts, cudaStream_t s);
// GCP mode: the prior cost term of every point at the state XM (0 for a
// point without a prior), out[0 .. npts)
void launch_gcp_cost(const DevLSA &L, const double *XM, float *out, cudaStream_t s);
void launch_exteval(int n_points, const int *pt_off, const int *pt_img, const int *pt_slot,
                    const int *img_off, const float *pmat, const float *K, const float *dist,
                    const float *XX, const float *xg, const float *wx, const float *wy,
                    const float *wxy, double *resid, float *ptterm, int *ptred,
                    cudaStream_t s);
// robust deletion: marks, then compacts into the *_n buffers
void launch_delete_mark(const DevLSA &L, int *okeep, int *pkeep, cudaStream_t s);
void launch_delete_compact(const DevLSA &L, const int *oidx, const int *pidx, const int *okeep,
                           const int *pkeep, int nobs_new, int npts_new, int *o_cam_n,
                           int *o_slot_n, int *o_pt_n, float2 *o_xg_n, float4 *o_wold_n,
                           int *pt_off_n, int *pt_id_n, double *X_n, cudaStream_t s);

// ---- exact sequential float sums (exactsum.cu)
struct ExactSumWork {
  long long *Rc, *Mc;
  int *Tc;
  void *ctl;
  unsigned *bar;
  int *err;
  int max_grid;
};
int exact_sum_max_grid(int device);
void launch_exact_sum(const float *v, int n, float *out, const ExactSumWork &W, cudaStream_t s);

// ---- dense direct solve (direct.cu)
struct DirectWork {
  int n = 0;              // unknowns of the reduced camera system
  int nt = 0;             // 64-wide tile rows
  long long ntiles = 0;   // tiles of the envelope
  size_t env_bytes = 0;   // device bytes the envelope and its inverses take
  double *tiles = nullptr;         // [ntiles][64 * 64] lower envelope, then L
  double *Linv = nullptr;          // [nt][64 * 64] inverses of the diagonal tiles
  double *y = nullptr;             // [nt * 64] right-hand side / solution, factor order
  long long *toff = nullptr;       // [nt] first tile of each tile row
  int *fcol = nullptr, *hrow = nullptr;  // [nt] first tile column of a row, last tile row of a column
  int *pos = nullptr;              // [nimg] first unknown of each camera in factor order
  unsigned *bar = nullptr;         // grid-barrier words
  const unsigned *bkey = nullptr;  // (row * nimg + column) of each off-diagonal block
  size_t cap_tiles = 0;
  int cap_nt = 0;
};
// Camera order (reverse Cuthill-McKee) and envelope of the current structure
// (host), device buffers sized for it; false when the envelope would take
// more than max_bytes.
bool direct_analyse(const DevLSA &L, const unsigned *d_bkey, const std::vector<int> &camparv, size_t max_bytes,
                    DirectWork &W, std::vector<void *> &owned, cudaStream_t s);
void direct_solve(const DevLSA &L, const DirectWork &W, double *xsol, cudaStream_t s);
void direct_factor(const DevLSA &L, const DirectWork &W, cudaStream_t s);
void direct_resolve(const DevLSA &L, const DirectWork &W, const double *b, double *xsol, cudaStream_t s);
// Tiled Cholesky of a lower envelope of 64 x 64 tiles in place, with the
// inverses of the diagonal tiles (chol.cu; one cooperative launch).
void tile_cholesky(double *tiles, const long long *toff, const int *fcol, const int *hrow, double *Linv, int nt,
                   unsigned *bar, int *err, cudaStream_t s);
// A^-1 of (D A D + eps I), scaled back by D = diag(dsc), for a dense SPD
// matrix (row major n x n, lower triangle used): tiled Cholesky and inverse
// in one cooperative launch on the FP64 tensor cores (chol.cu).  work:
// spd_inverse_bytes(n); bar: two barrier words; err bit 4: not SPD.
size_t spd_inverse_bytes(int n);
void spd_inverse_scaled(const double *A, const double *dsc, double eps, int n, double *Ainv, void *work,
                        unsigned *bar, int *err, cudaStream_t s);

// ---- coarse space of the two-level preconditioner (coarse.cu)
// Cameras are grouped into spatially compact aggregates; each aggregate
// contributes CO_M coarse unknowns: a small rigid motion of its cameras
// (rotation 3, translation 3), a scale about its centre, and common shifts
// of the three intrinsics.  P_k (9 x CO_M) maps them onto camera k's block.
constexpr int CO_M = 10;
struct CoarseWork {
  int nagg = 0, nc = 0;          // aggregates, coarse unknowns (CO_M each)
  int *agg_off = nullptr;        // [nagg + 1]
  int *agg_rows = nullptr;       // rows of the system grouped by aggregate
  int *row_agg = nullptr;        // [nimg] aggregate of a row, -1 outside
  double *P = nullptr;           // [nimg * 9 * CO_M]
  double *Ac = nullptr, *Ainv = nullptr;
  double *rc = nullptr;          // [nc] restricted residual
  double *dsc = nullptr;         // [nc] Jacobi scaling of A_c
  double *hj = nullptr;          // [nimg * 9] fine part of the preconditioned residual
  int *err = nullptr;            // bit 4: coarse matrix not positive definite
  void *work = nullptr;          // spd_inverse_bytes(nc)
  unsigned *bar = nullptr;       // grid-barrier words of the factorisation
  // Galerkin assembly (grown on demand, released by coarse_release)
  int built_version = -1, nruns = 0, nsegs = 0;
  unsigned *ekey = nullptr, *ekey2 = nullptr, *run_key = nullptr, *rkey = nullptr, *rkey2 = nullptr,
           *seg_key = nullptr;
  int *eval = nullptr, *ent_sorted = nullptr, *run_cnt = nullptr, *run_off = nullptr, *counts = nullptr,
      *ridx = nullptr, *run_sorted = nullptr, *seg_cnt = nullptr, *seg_off = nullptr;
  double *Z = nullptr;           // [nruns][CO_M * CO_M]
  unsigned char *cub_tmp = nullptr;
  size_t ekey_cap = 0, ekey2_cap = 0, eval_cap = 0, ent_sorted_cap = 0, run_key_cap = 0, run_cnt_cap = 0,
         run_off_cap = 0, counts_cap = 0, rkey_cap = 0, rkey2_cap = 0, ridx_cap = 0, run_sorted_cap = 0,
         seg_key_cap = 0, seg_cnt_cap = 0, seg_off_cap = 0, Z_cap = 0, cub_tmp_cap = 0;
};
// Aggregates from the cameras' projection centres (recursive coordinate
// bisection into at most max_aggs groups of about 16 cameras or more).
void coarse_build(const DevLSA &L, int max_aggs, CoarseWork &C, std::vector<void *> &owned, cudaStream_t s);
// Per linear system: P, the Galerkin matrix P^T S P and its inverse (the
// run structure of the assembly is rebuilt when structure_version changes).
void coarse_setup(const DevLSA &L, CoarseWork &C, int structure_version, cudaStream_t s);
// the two halves of coarse_setup: P and P^T S P; the factorisation and inverse
void coarse_assemble(const DevLSA &L, CoarseWork &C, int structure_version, cudaStream_t s);
void coarse_factor(CoarseWork &C, cudaStream_t s);
void coarse_release(CoarseWork &C);
// h += P A_c^-1 P^T r over the rows of the system.
void coarse_apply(const DevLSA &L, const CoarseWork &C, const double *r, double *h, cudaStream_t s);

// ---- learned preconditioner (learned.cu)
constexpr int NN_F = 19, NN_H = 64, NN_O = 9;
constexpr int NN_WEIGHTS = NN_H * NN_F + NN_H + NN_O * NN_H + NN_O;  // 1865
// Training set: recorded reduced camera systems, diagonally scaled and
// concatenated into one block-diagonal system (device arrays).
struct TrainSet {
  int rows, rows_cap, systems, probes;
  float *f;          // [rows_cap][NN_F]
  float *sinv;       // [rows_cap][81]  D^1/2 S_kk^-1 D^1/2
  float *b;          // [probes][rows_cap][9] right-hand sides (D^-1/2 b)
  float *xs;         // [rows_cap][9]   D^1/2 x* of right-hand side 0
  int *np, *sys;     // [rows_cap]
  int *rowoff;       // [rows_cap + 1]
  int2 *ent;         // (row, block | 0x80000000 if transposed)
  float *blocks;     // [.][81]        D^-1/2 S D^-1/2
  int *sys_row;      // [systems + 1]
  float *uc;         // [probes][rows_cap][9] coarse part D^1/2 P A_c^-1 P^T b
                     // of the preconditioned right-hand sides (nullptr: none)
};
struct TrainHost {  // host-side capacities and fill levels
  int ents, ents_cap, blocks, blocks_cap, sys_cap;
  int2 *rc;  // device scratch: (row, col) of a system's off-diagonal blocks
  double *vb, *vz;  // device scratch: [nimg * 9] right-hand side, coarse part
  std::vector<int> sys_row;
};
struct TrainBufs {
  float *sv, *ov, *hv, *u, *v, *d2, *d1, *grad;
  double *pq;
};
struct PcgWork;
void learned_pcg_setup(const DevLSA &L, const PcgWork &W, const float *weights, cudaStream_t s);
struct CoarseWork;
// scratch: [nimg * 81] doubles
void learned_record(const DevLSA &L, const CoarseWork *coarse, const double *xstar, double *scratch, double *drs,
                    unsigned long long seed, TrainSet &T, TrainHost &H, cudaStream_t s);
void learned_loss_grad(const TrainSet &T, const float *W, TrainBufs &B, float *loss, float *err, cudaStream_t s);
void learned_adam(float *W, float *m, float *v, const float *grad, float lr, int t, cudaStream_t s);

// ---- PCG (pcg.cu)
struct PcgWork {
  double *r, *d, *q, *h, *x, *xbest, *Cinv, *partials, *part;
  // FP32 form: d^k in FP32 ([nimg * 12]), and the SpMV's row sums of the
  // diagonal blocks, of the rows' first runs, and of the chunk runs that
  // start inside a row ([nimg * 9], [nimg * 9], [groups * 9]); per chunk its
  // share of d^T A d ([groups]); the chunk counter
  float *d32;
  double *pdiag, *prow, *pw, *pdqc;
  unsigned *ctr;  // [2] next phase-1 chunk, next phase-2 row
  double *rowc;   // [nimg * 12] with the coarse space: per row P_k^T r and its share of |dr|^2
  double *drs;  // [nimg * 9] 1 / sqrt of the camera blocks' diagonal entries (learned features)
  float *feat;  // [nimg * 20] the learned preconditioner's features per camera row
  unsigned *bar;
  int *iters;
};
// A PCG solve is pcg_prepare (the preconditioner and the start vectors;
// returns its launch count) followed by pcg_iterate (the persistent kernel).
// mode 0: the reference's stop rule; mode 1: stop when r^T M^-1 r falls
// below tol^2 times its start value (W.iters[1] = 1 when it did), with the
// learned preconditioner `weights` (nullptr: plain block-Jacobi).
// With `coarse` the preconditioner is two-level: the (learned) block
// Jacobi part plus the coarse correction P A_c^-1 P^T.
int pcg_prepare(const DevLSA &L, const PcgWork &W, int mode, const float *weights, const CoarseWork *coarse,
                cudaStream_t s);
int pcg_iterate(const DevLSA &L, const PcgWork &W, int msize, int grid, cudaStream_t s, int mode, double tol,
                const CoarseWork *coarse);
int pcg_max_grid(int device);

// ---- structure (structure.cu)
struct StructWork {
  void *cub_tmp;
  size_t cub_bytes;
  unsigned *pkey, *pkey2;
  unsigned long long *pval, *pval2;
  int *pcnt, *poff;
  int *ccnt;
  unsigned *bkey;
  int *bcnt, *boff;
  int *nrun;
  int *cntN, *cntT, *firstN, *firstT, *rowtmp;
  int4 *bidx;  // FP32 form: (row, column, transposed slot, 0) of every block in storage order
  unsigned *tkey, *tkey2;
  int *tidx, *tidx2;
  int2 *contrib;
  int *rowoff;
  int2 *ent;
  int *iota, *iota2;
  unsigned *ckey, *ckey2;
  int *row_items, *row_item_off;
  int4 *item_meta;
  int2 *rowspan;
};
size_t structure_cub_bytes(int nobs, long long npairs, int nimg);
// PointXXvIn on the device (structure.cu): the caller's block in device
// memory, the scan scratch, and the track-ordered outputs.
struct TrackIn {
  const int *pt_off, *pt_img, *pt_slot, *img_off;
  const float *xg, *wx, *wy, *wxy, *XX;
  int np, n;
  // GCP mode: per point its GCP index or -1; a point with a GCP index above
  // 0 is kept with a single observation (rbacore.cpp:1954-1956)
  const int *gcp = nullptr;
};
struct TrackScan {
  int *cnt, *pval, *ooff, *pidx, *err;  // [np + 1]
  long long *pairs, *psum;              // [np], [1]
};
struct TrackOut {
  int *o_cam, *o_slot, *o_pt, *pt_off, *pt_id;
  float2 *o_xg;
  float4 *o_w;
  double *X;
  int *gcp = nullptr;  // GCP mode: the GCP index of every kept point
};
// returns the error bits (1: an index out of range, 2: an image twice in a track)
int track_count(const TrackIn &T, TrackScan &W, int *nobs, int *npts, long long *max_pairs, cudaStream_t s);
void track_scatter(const TrackIn &T, const TrackScan &W, const TrackOut &O, int nobs, int npts, cudaStream_t s);
// camera grouping: returns 0, fills camlist/coff; counts in ccnt
void build_camera_order(DevLSA &L, StructWork &S, cudaStream_t s);
// pair structure: returns number of off-diagonal blocks (syncs the stream)
int build_pairs(DevLSA &L, StructWork &S, long long max_pairs, long long *npairs_out,
                cudaStream_t s);
void build_bsr(DevLSA &L, StructWork &S, cudaStream_t s);
cudaError_t cub_exclusive_sum_int(void *tmp, size_t &bytes, const int *in, int *out, int n, cudaStream_t s);
// CalcLSAXMulti for every point of b (triangulate.cu): the cameras Pd in
// double precision (null: b->pmat), the other arguments as
// rpba_triangulate_parts (part null: no weight blocks); s0_pt / red_pt
// (optional): every point's contribution to sig0io and the redundancy
int32_t triangulate_impl(const rpba_block *b, const double *Pd, const float *sig0w, const rpba_tri_options *opt,
                         const int32_t *part, int32_t nparts, double *XX_out, uint8_t *keep, float *sig0v,
                         uint8_t *conv, double *sig0io, int64_t *redundancy, float *w3d, double *s0_pt,
                         int32_t *red_pt);

}  // namespace rpba

#define RPBA_CUDA_CHECK(x)                                  \
  do {                                                      \
    cudaError_t e__ = (x);                                  \
    if (e__ != cudaSuccess) throw rpba::CudaError(e__, #x); \
  } while (0)

namespace rpba {
struct CudaError {
  cudaError_t code;
  const char *what;
  CudaError(cudaError_t c, const char *w) : code(c), what(w) {}
};
}  // namespace rpba
