// solver.cu -- host driver of the GPU global LSA and the C ABI.
//
// The control flow is LSA::Adjust (rbacore.cpp:333-616) and
// LSA::CalcBundleSep (rbacore.cpp:1094-1195): two passes (damping 1e-3 with
// robust reweighting, then 1e-6), acceptance on the float sigma0, the
// reference's stop counter.  Every O(observations) step runs on the GPU;
// the host only takes the scalar decisions (one small device->host copy per
// LM iteration).  Set-up that the reference does in its constructor
// (PointXXvIn, PrepareCameras, PrepareIteration, rbacore.cpp:37-229,
// 670-700, 1918-1974) runs once in rpba_create.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/rpba_b200.h"
#include "internal.h"

using namespace rpba;

namespace {

// A handle's device memory comes from the device's stream-ordered pool
// (cudaMallocAsync on the handle's stream, retained by the pool after
// cudaFreeAsync): creating and destroying handles then never waits for the
// whole device, as cudaFree does, so handles on other streams -- the batched
// form, or an application's own work -- keep running.  The scope below,
// active while a handle allocates, routes dalloc(n, handle->owned) there;
// other lists (training sets) keep plain cudaMalloc.
struct AsyncAlloc {
  cudaStream_t s = nullptr;
  std::vector<void *> *sync_list = nullptr;   // the handle's `owned`
  std::vector<void *> *async_list = nullptr;  // where pool allocations are recorded
};
thread_local AsyncAlloc g_aa;
struct AsyncScope {
  AsyncAlloc prev;
  AsyncScope(cudaStream_t s, std::vector<void *> &sync_list, std::vector<void *> &async_list) : prev(g_aa) {
    g_aa.s = s;
    g_aa.sync_list = &sync_list;
    g_aa.async_list = &async_list;
  }
  ~AsyncScope() { g_aa = prev; }
};

void retain_pool(int dev) {
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    unsigned long long thr = ~0ull;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
}

template <typename T>
T *dalloc(size_t n, std::vector<void *> &owned) {
  void *p = nullptr;
  const size_t bytes = sizeof(T) * (n ? n : 1);
  if (g_aa.s && &owned == g_aa.sync_list) {
    RPBA_CUDA_CHECK(cudaMallocAsync(&p, bytes, g_aa.s));
    g_aa.async_list->push_back(p);
  } else {
    RPBA_CUDA_CHECK(cudaMalloc(&p, bytes));
    owned.push_back(p);
  }
  return (T *)p;
}

std::string fmt_g(double v) {
  char b[64];
  std::snprintf(b, sizeof b, "%g", v);
  return b;
}

// RectifyRotationMatrix4 on the host (rpba.h:923-960), for PrepareIteration.
void rectify_host(double *R, int rs) {
  double a[3] = {R[2 * rs + 1] - R[rs + 2], R[2] - R[2 * rs], R[rs] - R[1]};
  for (double &v : a)
    if (std::fabs(v) < 1.e-20) v = 1.e-20;
  const double al = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
  for (double &v : a) v /= al;
  const double phi = std::atan2(al, R[0] + R[rs + 1] + R[2 * rs + 2] - 1.);
  const double q0 = std::cos(phi * 0.5), s = std::sin(phi * 0.5);
  const double q1 = a[0] * s, q2 = a[1] * s, q3 = a[2] * s;
  R[0] = q0 * q0 + q1 * q1 - q2 * q2 - q3 * q3;
  R[1] = 2 * (q1 * q2 - q0 * q3);
  R[2] = 2 * (q1 * q3 + q0 * q2);
  R[rs] = 2 * (q2 * q1 + q0 * q3);
  R[rs + 1] = q0 * q0 - q1 * q1 + q2 * q2 - q3 * q3;
  R[rs + 2] = 2 * (q2 * q3 - q0 * q1);
  R[2 * rs] = 2 * (q3 * q1 - q0 * q2);
  R[2 * rs + 1] = 2 * (q3 * q2 + q0 * q1);
  R[2 * rs + 2] = q0 * q0 - q1 * q1 - q2 * q2 + q3 * q3;
}

}  // namespace

// Per-kernel device timing (CUDA events around each launch on the solve's
// stream), enabled by rpba_options.verbose bit 1; launch counts always.
struct KernelProf {
  struct Rec {
    const char *name;
    cudaEvent_t a, b;
    double bytes;
  };
  bool on = false;
  cudaStream_t s = nullptr;
  std::vector<Rec> pending;
  std::vector<cudaEvent_t> pool;
  struct Stat {
    std::string name;
    long long launches;
    double ms, bytes;
  };
  std::vector<Stat> stats;
  double next_bytes = 0.;
  long long launches = 0, lib_launches = 0;
  const char *cur = nullptr;
  cudaEvent_t ev() {
    if (pool.empty()) {
      cudaEvent_t e;
      RPBA_CUDA_CHECK(cudaEventCreate(&e));
      return e;
    }
    cudaEvent_t e = pool.back();
    pool.pop_back();
    return e;
  }
  void begin(const char *name, int n = 1) {
    launches += n;
    if (!on) return;
    Rec r{name, ev(), ev(), next_bytes};
    next_bytes = 0.;
    RPBA_CUDA_CHECK(cudaEventRecord(r.a, s));
    pending.push_back(r);
  }
  void end() {
    if (!on) return;
    RPBA_CUDA_CHECK(cudaEventRecord(pending.back().b, s));
  }
  void add(const char *name, long long n, double ms, double bytes) {
    for (auto &st : stats)
      if (st.name == name) {
        st.launches += n;
        st.ms += ms;
        st.bytes += bytes;
        return;
      }
    stats.push_back({name, n, ms, bytes});
  }
  void resolve() {
    for (auto &r : pending) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, r.a, r.b);
      add(r.name, 1, ms, r.bytes);
      pool.push_back(r.a);
      pool.push_back(r.b);
    }
    pending.clear();
  }
  void reset() {
    resolve();
    stats.clear();
    launches = lib_launches = 0;
  }
  ~KernelProf() {
    for (auto e : pool) cudaEventDestroy(e);
    for (auto &r : pending) {
      cudaEventDestroy(r.a);
      cudaEventDestroy(r.b);
    }
  }
};

#define PROF(name, n, call) \
  do {                          \
    prof.begin(name, n);        \
    call;                       \
    prof.end();                 \
  } while (0)

struct rpba_handle {
  rpba_options opt{};
  KernelProf prof;
  int dev = 0;
  cudaStream_t s = nullptr;
  std::vector<void *> owned;

  // problem
  int nimg = 0, XXnr = 0, n_slots = 0, n_track_in = 0;
  std::vector<float> K_in, XX_in;
  std::vector<int32_t> img_off_in;
  rpba_block raw{};  // device copy of the caller's block (Exteval)
  bool raw_uploaded = false;
  std::vector<float> h_pmat, h_K, h_dist, h_XX, h_xg, h_wx, h_wy, h_wxy;
  std::vector<int32_t> h_img_off, h_pt_off, h_pt_img, h_pt_slot;

  // GCP mode (the parallel RPBA's per-partition LSA): the scene's camera
  // count (unknowns of the additional parameters), the kept points with a
  // prior, the float sum of their weight diagonals (PrepareWeights3D), and
  // three segments of per-point prior cost terms
  bool ao = false;
  int ncam_total = 0, nrgcp = 0;
  float w3diag_sum = 0.f;
  float *aoterm = nullptr;

  // static parameterisation
  int nadd = 0, addmask = 0, nrpari = 0, nrparir = 0, nrioff = 0, normcamera = -1, begini = 1;
  int minimagenrdel = 2, xpmsize = 0, npts0 = 0, nobs0 = 0;
  bool lflflag = false, robust = true;
  float ihw2 = 1.f;
  double defdiff = 5000.;
  std::vector<int> camparv;
  long long max_pairs = 0, npairs_cur = 0, learned_iters = 0;
  int pcg_grid = 1;
  bool pcg_pending = false;

  // original state (restored by every solve)
  int *d0_o_cam, *d0_o_slot, *d0_o_pt, *d0_pt_off, *d0_pt_id;
  float2 *d0_o_xg;
  float4 *d0_o_wold;
  double *d0_P, *d0_Kc, *d0_dc, *d0_X;
  CamState *d0_camn;
  float *d_XXin = nullptr;  // the caller's points as given (rpba_get_state keeps the unused ones)

  // working state
  DevLSA L{};
  int *o_cam_n, *o_slot_n, *o_pt_n, *pt_off_n, *pt_id_n;
  float2 *o_xg_n;
  float4 *o_wold_n;
  double *X_n;
  int *okeep, *oidx, *pkeep, *pidx;
  float *vals, *sig00v, *sums;
  int *nflag;
  double *fc_part;
  int fc_nparts = 0;
  StructWork S{};
  PcgWork W{};
  ExactSumWork ES{};
  DirectWork DW{};
  // learned preconditioner (device copy of the weights; nullptr: none)
  float *d_weights = nullptr;
  // training-data recording (set by rpba_train_preconditioner)
  TrainSet *rec_T = nullptr;
  TrainHost *rec_H = nullptr;
  unsigned long long rec_seed = 1;
  int blocks_cap = 0;
  cudaEvent_t ev0, ev1;

  std::string log;
  rpba_report rep{};

  std::vector<void *> owned_async;  // pool allocations on stream s

  ~rpba_handle() {
    coarse_release(CW);
    if (s) {
      for (void *p : owned_async) cudaFreeAsync(p, s);
      cudaStreamSynchronize(s);
    }
    for (void *p : owned) cudaFree(p);
    if (s) {
      cudaEventDestroy(ev0);
      cudaEventDestroy(ev1);
      cudaStreamDestroy(s);
    }
  }

  // Algorithmic bytes of one PCG iteration.  FP64 form: every block read from
  // both sides with its entry (648 + 8 B per side).  FP32 form (symmetric):
  // every block read once with its index (324 + 16 B), and per off-diagonal
  // block the transposed product written and read (a 64 B slot each way).  Per camera row: the preconditioner (648 B) and
  // 22 reads/writes of 9-vectors (72 B each); with the coarse space P_k twice
  // (720 B each) and the block part of h twice; A_c^-1 stays in L2 and is
  // not counted.
  double pcg_bytes_per_iteration(bool coarse) const {
    const double Nc = nimg - begini, Nb = L.nboff;
    const double row = 648. + 22. * 72. + (coarse ? 2. * 720. + 2. * 72. : 0.);
    const double blocks = L.blocks32 ? 340. * (Nc + Nb) + 128. * Nb : 656. * (Nc + 2. * Nb);
    return blocks + Nc * row;
  }

  // Algorithmic bytes of the PCG set-up: per camera row its diagonal block,
  // C_k out (648 B) and five 9-vectors (r, h, x, best, rhs); with the
  // learned preconditioner also the features, every block of every row read
  // from both sides with its entry and the column's parameter count.
  double setup_bytes(bool features) const {
    const double Nc = nimg - begini, Nb = L.nboff, Eb = L.blocks32 ? 4. : 8.;
    return Nc * (81. * Eb + 648. + 5. * 72.) + (features ? (Nc + 2. * Nb) * (81. * Eb + 8. + 8.) : 0.);
  }

  // reduced camera system storage: FP64, or FP32 in the mixed form
  void ensure_blocks(int nb) {
    const bool mixed = opt.precision == RPBA_PREC_MIXED;
    void *cur = mixed ? (void *)L.blocks32 : (void *)L.blocks;
    if (nb <= blocks_cap && cur) return;
    const int cap = std::max(nb, 1);
    if (cur) {
      for (void *p : {cur, (void *)S.ent, (void *)S.item_meta, (void *)W.part, (void *)L.tpart, (void *)S.bidx,
                      (void *)W.pw, (void *)W.pdqc}) {
        if (!p) continue;
        auto it = std::find(owned_async.begin(), owned_async.end(), p);
        if (it != owned_async.end()) {
          cudaFreeAsync(p, s);
          owned_async.erase(it);
        } else {
          cudaFree(p);
          owned.erase(std::remove(owned.begin(), owned.end(), p), owned.end());
        }
      }
    }
    if (mixed) {
      // slack past the last block, row pair and transposed product: the
      // FP32 PCG's bulk copies round their sizes up to 16 bytes
      L.blocks32 = dalloc<float>((size_t)(nimg + cap) * BS32 + 16, owned);
      L.tpart = dalloc<float>((size_t)cap * 16 + 16, owned);
      S.bidx = dalloc<int4>((size_t)nimg + cap + 4, owned);
      // phase-1 chunks of the FP32 PCG: at most one per group of 32 blocks
      const size_t groups = ((size_t)nimg + cap) / 32 + 4;
      W.pw = dalloc<double>(9 * groups, owned);
      W.pdqc = dalloc<double>(groups, owned);
    } else
      L.blocks = dalloc<double>((size_t)(nimg + cap) * BS64, owned);
    S.ent = dalloc<int2>((size_t)nimg + 2 * (size_t)cap, owned);
    // SpMV work items: at most ceil(entries / 3) per row
    const size_t items = (size_t)nimg + ((size_t)nimg + 2 * (size_t)cap) / 3 + 1;
    S.item_meta = dalloc<int4>(items, owned);
    W.part = dalloc<double>(items * 9, owned);
    blocks_cap = cap;
  }

  // dense direct-solve buffers, allocated on first use
  // coarse space of the learned solver, built once per handle from the
  // cameras of the first linear system (nullptr: none)
  CoarseWork CW{};
  bool coarse_built = false, coarse_stale = true;
  int structure_version = 0;
  int coarse_ref_iters = 0;
  const CoarseWork *ensure_coarse() {
    if (opt.coarse_aggregates < 0) return nullptr;
    if (!coarse_built) {
      coarse_built = true;
      const int want = opt.coarse_aggregates > 0 ? opt.coarse_aggregates : 148;
      coarse_build(L, want, CW, owned, s);
    }
    return CW.nagg > 0 ? &CW : nullptr;
  }

  // Direct-solve structure (camera order and envelope), rebuilt when the
  // pair structure changes; false when the envelope does not fit in device
  // memory (the reduced camera system is too dense for the direct form).
  int direct_version = -1;
  bool direct_ok = false;
  bool ensure_direct() {
    if (direct_version == structure_version) return direct_ok;
    size_t fr = 0, tot = 0;
    RPBA_CUDA_CHECK(cudaMemGetInfo(&fr, &tot));
    const size_t reuse = DW.cap_tiles * 64 * 64 * sizeof(double);
    direct_ok = direct_analyse(L, S.bkey, camparv, (fr + reuse) / 10 * 7, DW, owned, s);
    direct_version = structure_version;
    return direct_ok;
  }
  bool direct_too_large = false;

  // Batched solves (rpba_solve_batch) run many handles on one GPU at once.
  // Cooperative kernels (the persistent PCG, the exact sums) need all their
  // CTAs resident together; two of them from different scenes could each
  // hold part of the SMs and wait for the rest.  In a batch they are
  // therefore run one at a time: the launch takes `coop` and releases it
  // once the kernel has finished.  Ordinary kernels of other scenes keep
  // running meanwhile.
  std::mutex *coop = nullptr;
  struct CoopLock {
    rpba_handle *H;
    explicit CoopLock(rpba_handle *h) : H(h) {
      if (H->coop) H->coop->lock();
    }
    ~CoopLock() {
      if (H->coop) {
        cudaStreamSynchronize(H->s);
        H->coop->unlock();
      }
    }
  };

  float seq_sum(const float *v, int n) {
    {
      CoopLock lk(this);
      prof.next_bytes = 4. * n;  // each element read once
      PROF("seq_sum", 1, launch_exact_sum(v, n, sums, ES, s));
    }
    float out = 0.f;
    RPBA_CUDA_CHECK(cudaMemcpyAsync(&out, sums, sizeof(float), cudaMemcpyDeviceToHost, s));
    RPBA_CUDA_CHECK(cudaStreamSynchronize(s));
    return out;
  }

  void reset();
  int adjust();
  int adjust_gcp_step();
  bool calc_bundle_sep(double multfact, int nrunknowns);
  void robust_delete();
  void structure();
};

// ------------------------------------------------------------- create

// The GCP-mode inputs of rpba_lsa_gcp_step.
struct GcpSetup {
  const int32_t *gcpinfo;  // [n_points] GCP index or -1
  const float *W3;         // [n_w3 x 6]
  int32_t n_w3;
  const double *gcpdata;   // [n_gcp x 3]
  int32_t n_gcp;
  int32_t ncam_total;
  const double *Pd;        // [n_images x 12] cameras in double precision, or null
};

static int create_impl(rpba_handle *H, const rpba_block *b, const rpba_options *o, const GcpSetup *gs = nullptr) {
  H->opt = *o;
  H->dev = o->device;
  RPBA_CUDA_CHECK(cudaSetDevice(H->dev));
  RPBA_CUDA_CHECK(cudaStreamCreateWithFlags(&H->s, cudaStreamNonBlocking));
  RPBA_CUDA_CHECK(cudaEventCreate(&H->ev0));
  RPBA_CUDA_CHECK(cudaEventCreate(&H->ev1));
  retain_pool(H->dev);
  AsyncScope scope(H->s, H->owned, H->owned_async);
  auto &own = H->owned;
  const int n = b->n_images, np = b->n_points;
  H->nimg = n;
  H->XXnr = np;
  H->n_slots = b->img_obs_off[n];
  H->n_track_in = b->pt_obs_off[np];
  H->robust = o->robust != 0 && !gs;  // the partition LSAs run without robust reweighting
  H->ao = gs != nullptr;
  H->ncam_total = gs ? gs->ncam_total : n;
  H->addmask = (o->k2 ? 1 : 0) | (o->k4 ? 2 : 0) | (o->f ? 4 : 0);
  H->nadd = (o->k2 ? 1 : 0) + (o->k4 ? 1 : 0) + (o->f ? 1 : 0);
  if (n > 65535) return RPBA_ERR_UNSUPPORTED;
  // host copies of the caller's cameras and points (the output keeps the
  // input values of points the solve does not use); the observations and
  // tracks only for an Exteval handle, whose rpba_exteval reads them (a
  // solve handle takes them straight from the caller's arrays to the device)
  H->h_pmat.assign(b->pmat, b->pmat + 12 * n);
  H->h_K.assign(b->K, b->K + 9 * n);
  H->h_dist.assign(b->distpara, b->distpara + 2 * n);
  H->h_XX.assign(b->XX, b->XX + 3 * np);
  H->d_XXin = dalloc<float>(3 * (size_t)std::max(np, 1), own);
  if (np) RPBA_CUDA_CHECK(cudaMemcpyAsync(H->d_XXin, b->XX, sizeof(float) * 3 * np, cudaMemcpyHostToDevice, H->s));
  if (o->exteval) {
    H->h_img_off.assign(b->img_obs_off, b->img_obs_off + n + 1);
    H->h_xg.assign(b->xg, b->xg + 2 * H->n_slots);
    H->h_wx.assign(b->wx, b->wx + H->n_slots);
    H->h_wy.assign(b->wy, b->wy + H->n_slots);
    H->h_wxy.assign(b->wxy, b->wxy + H->n_slots);
    H->h_pt_off.assign(b->pt_obs_off, b->pt_obs_off + np + 1);
    H->h_pt_img.assign(b->pt_obs_image, b->pt_obs_image + H->n_track_in);
    H->h_pt_slot.assign(b->pt_obs_slot, b->pt_obs_slot + H->n_track_in);
  }
  {
    H->ES.max_grid = exact_sum_max_grid(H->dev);
    H->ES.Rc = dalloc<long long>(2 * (size_t)H->ES.max_grid, own);
    H->ES.Mc = dalloc<long long>(2 * (size_t)H->ES.max_grid, own);
    H->ES.Tc = dalloc<int>(2 * (size_t)H->ES.max_grid, own);
    H->ES.ctl = dalloc<char>(16, own);
    H->ES.bar = dalloc<unsigned>(2, own);
    H->ES.err = dalloc<int>(4, own);
    RPBA_CUDA_CHECK(cudaMemsetAsync(H->ES.err, 0, 4 * sizeof(int), H->s));
  }
  if (o->exteval) {
    RPBA_CUDA_CHECK(cudaStreamSynchronize(H->s));
    for (int i = 0; i < H->n_track_in; ++i) {
      const int im = H->h_pt_img[i];
      if (im < 0 || im >= n || H->h_pt_slot[i] < 0 || H->h_pt_slot[i] >= H->h_img_off[im + 1] - H->h_img_off[im])
        return RPBA_ERR_ARG;
    }
    return RPBA_OK;
  }

  // ihw2 / defdiff for iwidth = iheight = 1 (rpba.cpp:264-265, rpbacore.cpp:87-90, rbacore.cpp:48)
  float ihw2 = 0.f;
  for (int i = 0; i < n; ++i) ihw2 += (float)((1 + 1) * (1 + 1)) * 0.25f;
  ihw2 /= (float)n;
  H->ihw2 = ihw2;
  H->defdiff = 5000. / (double)std::sqrt(ihw2);
  H->minimagenrdel = n > 2 ? 3 : 2;

  // PointXXvIn (rbacore.cpp:1918-1974): points with >= 2 observations and
  // |Z| > 1e-8, track order, compacted on the device from the caller's
  // arrays (also validated there: image and slot indices in range, no image
  // twice in one track)
  std::vector<void *> tmp;
  auto tmalloc = [&](size_t bytes) {
    void *p = nullptr;
    RPBA_CUDA_CHECK(cudaMallocAsync(&p, std::max<size_t>(bytes, 16), H->s));
    tmp.push_back(p);
    return p;
  };
  struct TmpFree {
    std::vector<void *> &v;
    cudaStream_t s;
    ~TmpFree() {
      for (void *p : v) cudaFreeAsync(p, s);
    }
  } tmp_free{tmp, H->s};
  auto upt = [&](const void *h, size_t bytes) {
    void *d = tmalloc(bytes);
    if (bytes) RPBA_CUDA_CHECK(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, H->s));
    return d;
  };
  TrackIn TI;
  TI.np = np;
  TI.n = n;
  TI.pt_off = (const int *)upt(b->pt_obs_off, sizeof(int) * (np + 1));
  TI.pt_img = (const int *)upt(b->pt_obs_image, sizeof(int) * H->n_track_in);
  TI.pt_slot = (const int *)upt(b->pt_obs_slot, sizeof(int) * H->n_track_in);
  TI.img_off = (const int *)upt(b->img_obs_off, sizeof(int) * (n + 1));
  TI.xg = (const float *)upt(b->xg, sizeof(float) * 2 * H->n_slots);
  TI.wx = (const float *)upt(b->wx, sizeof(float) * H->n_slots);
  TI.wy = (const float *)upt(b->wy, sizeof(float) * H->n_slots);
  TI.wxy = (const float *)upt(b->wxy, sizeof(float) * H->n_slots);
  TI.XX = (const float *)upt(b->XX, sizeof(float) * 3 * np);
  if (gs) TI.gcp = (const int *)upt(gs->gcpinfo, sizeof(int) * np);
  TrackScan TW;
  TW.cnt = (int *)tmalloc(sizeof(int) * (np + 1));
  TW.pval = (int *)tmalloc(sizeof(int) * (np + 1));
  TW.ooff = (int *)tmalloc(sizeof(int) * (np + 1));
  TW.pidx = (int *)tmalloc(sizeof(int) * (np + 1));
  TW.err = (int *)tmalloc(sizeof(int));
  TW.pairs = (long long *)tmalloc(sizeof(long long) * std::max(np, 1));
  TW.psum = (long long *)tmalloc(sizeof(long long));
  int nobs = 0, npts = 0;
  long long max_pairs = 0;
  const int terr = track_count(TI, TW, &nobs, &npts, &max_pairs, H->s);
  if (terr & 1) return RPBA_ERR_ARG;
  if (terr & 2) return RPBA_ERR_UNSUPPORTED;
  H->npts0 = npts;
  H->nobs0 = nobs;
  H->max_pairs = max_pairs;
  if (H->max_pairs > 0x7fffffffll) return RPBA_ERR_UNSUPPORTED;

  // PrepareCameras (rbacore.cpp:670-700)
  std::vector<double> P(12 * (size_t)n);
  for (size_t i = 0; i < P.size(); ++i) P[i] = gs && gs->Pd ? gs->Pd[i] : (double)b->pmat[i];
  {
    std::vector<double> Tv(3 * (size_t)n);
    for (int i = 0; i < n; ++i)
      for (int r = 0; r < 3; ++r)
        Tv[3 * i + r] = P[12 * i + r * 4] * P[12 * i + 3] + P[12 * i + r * 4 + 1] * P[12 * i + 7] +
                        P[12 * i + r * 4 + 2] * P[12 * i + 11];
    double nd = 0.;
    H->normcamera = -1;
    for (int i = 1; i < n; ++i) {
      double d = 0.;
      for (int j = 0; j < 3; ++j) d += (Tv[3 * i + j] - Tv[j]) * (Tv[3 * i + j] - Tv[j]);
      if (d > nd) {
        nd = d;
        H->normcamera = i;
      }
    }
  }
  if (gs)
    H->normcamera = -1;  // every camera free (rbacore.cpp:697-698)
  else if (n < 2 || H->normcamera < 1)
    return RPBA_ERR_ARG;
  // PrepareIteration (rbacore.cpp:127-229)
  rectify_host(&P[0], 4);
  CamState c0{};
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) c0.R[r * 3 + c] = P[r * 4 + c];
  for (int i = 0; i < 3; ++i) c0.PC[i] = c0.R[i] * P[3] + c0.R[3 + i] * P[7] + c0.R[6 + i] * P[11];
  H->nrparir = 5 + H->nadd;
  H->nrpari = 6 + H->nadd;
  H->lflflag = false;
  for (int i = 0; i < n; ++i)
    if (b->K[9 * i] > 2.f || b->K[9 * i + 4] > 2.f) {
      H->lflflag = true;
      break;
    }
  // camparv as EncodeCameras lays it out (rbacore.cpp:999-1087); in GCP
  // mode every camera has the full block and the state vector has room for
  // the scene's cameras (xpmsize with nrcameras, rbacore.cpp:324)
  H->camparv.assign(n + 1, 0);
  if (gs) {
    H->nrioff = H->nrpari * n;
    H->begini = 0;
    H->xpmsize = n * 6 + 3 * np + 7 * std::max(H->ncam_total, n);
    for (int k = 0; k < n; ++k) H->camparv[k + 1] = H->camparv[k] + H->nrpari;
  } else {
    H->nrioff = H->nadd + H->nrparir + H->nrpari * (n - 2);
    H->begini = H->nadd > 0 ? 0 : 1;
    H->xpmsize = n * 6 + 3 * np + 7 * n;
    H->camparv[1] = H->nadd;
    for (int k = 1; k < n; ++k) H->camparv[k + 1] = H->camparv[k] + (k == H->normcamera ? H->nrparir : H->nrpari);
  }

  std::vector<CamState> cams(n);
  std::vector<double> Kc(9 * (size_t)n), dc(2 * (size_t)n);
  for (int i = 0; i < n; ++i) {
    CamState &c = cams[i];
    c = i == 0 ? c0 : CamState{};
    c.K00 = b->K[9 * i];
    c.K01 = b->K[9 * i + 1];
    c.K02 = b->K[9 * i + 2];
    c.K11 = b->K[9 * i + 4];
    c.K12 = b->K[9 * i + 5];
    c.d0 = b->distpara[2 * i];
    c.d1 = b->distpara[2 * i + 1];
    for (int j = 0; j < 9; ++j) Kc[9 * i + j] = b->K[9 * i + j];
    dc[2 * i] = b->distpara[2 * i];
    dc[2 * i + 1] = b->distpara[2 * i + 1];
  }

  // ---- device buffers
  const int no = std::max(nobs, 1), npp = std::max(npts, 1);
  H->d0_o_cam = dalloc<int>(no, own);
  H->d0_o_slot = dalloc<int>(no, own);
  H->d0_o_pt = dalloc<int>(no, own);
  H->d0_o_xg = dalloc<float2>(no, own);
  H->d0_o_wold = dalloc<float4>(no, own);
  H->d0_pt_off = dalloc<int>(npp + 1, own);
  H->d0_pt_id = dalloc<int>(npp, own);
  H->d0_P = dalloc<double>(12 * (size_t)n, own);
  H->d0_Kc = dalloc<double>(9 * (size_t)n, own);
  H->d0_dc = dalloc<double>(2 * (size_t)n, own);
  H->d0_X = dalloc<double>(3 * (size_t)npp, own);
  H->d0_camn = dalloc<CamState>(n, own);
  auto up = [&](void *d, const void *h, size_t bytes) {
    if (bytes) RPBA_CUDA_CHECK(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, H->s));
  };
  {
    TrackOut TO;
    TO.o_cam = H->d0_o_cam;
    TO.o_slot = H->d0_o_slot;
    TO.o_pt = H->d0_o_pt;
    TO.o_xg = H->d0_o_xg;
    TO.o_w = H->d0_o_wold;
    TO.pt_off = H->d0_pt_off;
    TO.pt_id = H->d0_pt_id;
    TO.X = H->d0_X;
    if (gs) TO.gcp = dalloc<int>(npp, own);
    track_scatter(TI, TW, TO, nobs, npts, H->s);
    if (gs) {
      // the weight-block row of every kept point with a prior: they are
      // numbered in point order (gcpnum, rbacore.cpp:1677-1729)
      std::vector<int> kg(npts), rows(npp, -1);
      if (npts) RPBA_CUDA_CHECK(cudaMemcpyAsync(kg.data(), TO.gcp, sizeof(int) * npts, cudaMemcpyDeviceToHost, H->s));
      RPBA_CUDA_CHECK(cudaStreamSynchronize(H->s));
      int nr = 0;
      for (int q = 0; q < npts; ++q) {
        if (kg[q] < -1 || kg[q] >= gs->n_gcp) return RPBA_ERR_ARG;
        if (kg[q] > -1) rows[q] = nr++;
      }
      if (nr > gs->n_w3) return RPBA_ERR_ARG;
      H->nrgcp = nr;
      // PrepareWeights3D: the float sum of the weight diagonals of the
      // kept priors, row by row (rbacore.cpp:787-818)
      float ws = 0.f;
      for (int i = 0; i < nr; ++i) ws += gs->W3[6 * i] + gs->W3[6 * i + 1] + gs->W3[6 * i + 2];
      H->w3diag_sum = ws;
      int *drows = dalloc<int>(npp, own);
      float *dW3 = dalloc<float>(6 * (size_t)std::max(gs->n_w3, 1), own);
      double *dG = dalloc<double>(3 * (size_t)std::max(gs->n_gcp, 1), own);
      up(drows, rows.data(), sizeof(int) * npp);
      up(dW3, gs->W3, sizeof(float) * 6 * (size_t)gs->n_w3);
      up(dG, gs->gcpdata, sizeof(double) * 3 * (size_t)gs->n_gcp);
      H->L.ao = 1;
      H->L.n_w3 = gs->n_w3;
      H->L.pt_gcp = TO.gcp;
      H->L.pt_w3row = drows;
      H->L.W3 = dW3;
      H->L.gcpdata = dG;
      H->aoterm = dalloc<float>(3 * (size_t)npp, own);
    }
  }
  up(H->d0_P, P.data(), sizeof(double) * P.size());
  up(H->d0_Kc, Kc.data(), sizeof(double) * Kc.size());
  up(H->d0_dc, dc.data(), sizeof(double) * dc.size());
  up(H->d0_camn, cams.data(), sizeof(CamState) * n);

  DevLSA &L = H->L;
  L.nimg = n;
  L.nrioff = H->nrioff;
  L.begini = H->begini;
  L.normcamera = H->normcamera;
  L.addmask = H->addmask;
  L.nadd = H->nadd;
  L.robust = H->robust ? 1 : 0;
  L.minimagenrdel = H->minimagenrdel;
  L.defdiff = H->defdiff;
  int *cp = dalloc<int>(n + 1, own);
  up(cp, H->camparv.data(), sizeof(int) * (n + 1));
  L.camparv = cp;
  L.gauge = dalloc<int>(4, own);
  L.Pacc = dalloc<double>(12 * (size_t)n, own);
  L.Kc = dalloc<double>(9 * (size_t)n, own);
  L.dc = dalloc<double>(2 * (size_t)n, own);
  L.camn = dalloc<CamState>(n, own);
  L.Rb = dalloc<double>(9 * (size_t)n, own);
  L.PCb = dalloc<double>(3 * (size_t)n, own);
  L.o_cam = dalloc<int>(no, own);
  L.o_slot = dalloc<int>(no, own);
  L.o_pt = dalloc<int>(no, own);
  L.o_xg = dalloc<float2>(no, own);
  L.o_wold = dalloc<float4>(no, own);
  L.o_w = dalloc<float4>(no, own);
  L.o_s0rmv = dalloc<float>(no, own);
  L.o_cost = dalloc<float>(no, own);
  L.o_wterm = dalloc<float>(no, own);
  L.o_flag = dalloc<uint8_t>(no, own);
  L.o_flagnew = dalloc<uint8_t>(no, own);
  L.pt_off = dalloc<int>(npp + 1, own);
  L.pt_id = dalloc<int>(npp, own);
  L.XPM = dalloc<double>(H->xpmsize, own);
  L.XPMn = dalloc<double>(H->xpmsize, own);
  L.x = dalloc<double>(H->xpmsize, own);
  if (H->opt.precision == RPBA_PREC_MIXED) {
    L.rec32 = dalloc<float>((size_t)no * REC, own);
    L.ptV32 = dalloc<float>((size_t)npp * PREC, own);
  } else {
    L.rec = dalloc<double>((size_t)no * REC, own);
    L.ptV = dalloc<double>((size_t)npp * PREC, own);
  }
  L.camlist = dalloc<int>(no, own);
  L.coff = dalloc<int>(n + 1, own);
  L.rhs = dalloc<double>(9 * (size_t)n, own);
  L.err = dalloc<int>(4, own);
  H->o_cam_n = dalloc<int>(no, own);
  H->o_slot_n = dalloc<int>(no, own);
  H->o_pt_n = dalloc<int>(no, own);
  H->o_xg_n = dalloc<float2>(no, own);
  H->o_wold_n = dalloc<float4>(no, own);
  H->pt_off_n = dalloc<int>(npp + 1, own);
  H->pt_id_n = dalloc<int>(npp, own);
  H->X_n = dalloc<double>(3 * (size_t)npp, own);
  H->okeep = dalloc<int>(no + 1, own);
  H->oidx = dalloc<int>(no + 1, own);
  H->pkeep = dalloc<int>(npp + 1, own);
  H->pidx = dalloc<int>(npp + 1, own);
  H->vals = dalloc<float>(no, own);
  H->sig00v = dalloc<float>(n, own);
  H->sums = dalloc<float>(4, own);
  H->nflag = dalloc<int>(4, own);
  H->fc_nparts = 296;
  H->fc_part = dalloc<double>(2 * H->fc_nparts, own);
  // structure work
  StructWork &S = H->S;
  const long long mp = std::max(H->max_pairs, 1ll);
  const long long mb = std::min(mp, (long long)n * (n - 1) / 2 + 1);
  S.cub_bytes = structure_cub_bytes(nobs, mp, n);
  S.cub_tmp = dalloc<char>(S.cub_bytes, own);
  S.pkey = dalloc<unsigned>(mp, own);
  S.pkey2 = dalloc<unsigned>(mp, own);
  S.pval = dalloc<unsigned long long>(mp, own);
  S.pval2 = dalloc<unsigned long long>(mp, own);
  S.contrib = dalloc<int2>(mp, own);
  S.pcnt = dalloc<int>(npp + 1, own);
  S.poff = dalloc<int>(npp + 1, own);
  S.ccnt = dalloc<int>(n + 1, own);
  S.bkey = dalloc<unsigned>(mb, own);
  S.bcnt = dalloc<int>(mb + 1, own);
  S.boff = dalloc<int>(mb + 1, own);
  S.nrun = dalloc<int>(1, own);
  S.cntN = dalloc<int>(n + 1, own);
  S.cntT = dalloc<int>(n + 1, own);
  S.firstN = dalloc<int>(n + 1, own);
  S.firstT = dalloc<int>(n + 1, own);
  S.rowtmp = dalloc<int>(n + 1, own);
  S.rowoff = dalloc<int>(n + 1, own);
  S.tkey = dalloc<unsigned>(mb, own);
  S.tkey2 = dalloc<unsigned>(mb, own);
  S.tidx = dalloc<int>(mb, own);
  S.tidx2 = dalloc<int>(mb, own);
  S.iota = dalloc<int>(no, own);
  S.row_items = dalloc<int>(n + 1, own);
  S.row_item_off = dalloc<int>(n + 1, own);
  S.rowspan = dalloc<int2>(n + 1, own);
  S.ckey = dalloc<unsigned>(no, own);
  S.ckey2 = dalloc<unsigned>(no, own);
  H->ES.err = L.err;  // a barrier timeout in a sum surfaces in the LSA's error word
  // PCG work
  H->pcg_grid = pcg_max_grid(H->dev);
  PcgWork &W = H->W;
  const size_t nv = 9 * (size_t)n;
  W.r = dalloc<double>(nv, own);
  W.d = dalloc<double>(nv, own);
  W.q = dalloc<double>(nv, own);
  W.h = dalloc<double>(nv, own);
  W.drs = dalloc<double>(nv, own);
  W.feat = dalloc<float>(20 * (size_t)n, own);
  W.x = dalloc<double>(nv, own);
  W.xbest = dalloc<double>(nv, own);
  W.Cinv = dalloc<double>(81 * (size_t)n, own);
  W.partials = dalloc<double>(8 * (size_t)H->pcg_grid, own);
  W.bar = dalloc<unsigned>(2, own);
  W.iters = dalloc<int>(2, own);
  if (o->precision == RPBA_PREC_MIXED) {
    W.d32 = dalloc<float>(12 * (size_t)n + 4, own);
    W.pdiag = dalloc<double>(nv, own);
    W.prow = dalloc<double>(nv, own);
    W.ctr = dalloc<unsigned>(4, own);
    W.rowc = dalloc<double>(12 * (size_t)n, own);
  }
  RPBA_CUDA_CHECK(cudaMemsetAsync(W.q, 0, sizeof(double) * nv, H->s));
  RPBA_CUDA_CHECK(cudaStreamSynchronize(H->s));
  return RPBA_OK;
}

// Restore the uploaded input state (the LSA after its constructor).
void rpba_handle::reset() {
  direct_too_large = false;
  L.nobs = nobs0;
  L.npts = npts0;
  auto cp = [&](void *d, const void *src, size_t bytes) {
    if (bytes) RPBA_CUDA_CHECK(cudaMemcpyAsync(d, src, bytes, cudaMemcpyDeviceToDevice, s));
  };
  cp(L.o_cam, d0_o_cam, sizeof(int) * nobs0);
  cp(L.o_slot, d0_o_slot, sizeof(int) * nobs0);
  cp(L.o_pt, d0_o_pt, sizeof(int) * nobs0);
  cp(L.o_xg, d0_o_xg, sizeof(float2) * nobs0);
  cp(L.o_wold, d0_o_wold, sizeof(float4) * nobs0);
  cp(L.pt_off, d0_pt_off, sizeof(int) * (npts0 + 1));
  cp(L.pt_id, d0_pt_id, sizeof(int) * npts0);
  cp(L.Pacc, d0_P, sizeof(double) * 12 * nimg);
  cp(L.Kc, d0_Kc, sizeof(double) * 9 * nimg);
  cp(L.dc, d0_dc, sizeof(double) * 2 * nimg);
  cp(L.camn, d0_camn, sizeof(CamState) * nimg);
  RPBA_CUDA_CHECK(cudaMemsetAsync(L.XPM, 0, sizeof(double) * xpmsize, s));
  RPBA_CUDA_CHECK(cudaMemsetAsync(L.XPMn, 0, sizeof(double) * xpmsize, s));
  RPBA_CUDA_CHECK(cudaMemsetAsync(L.x, 0, sizeof(double) * xpmsize, s));
  cp(L.XPM + nrioff, d0_X, sizeof(double) * 3 * npts0);
  RPBA_CUDA_CHECK(cudaMemsetAsync(L.err, 0, sizeof(int) * 4, s));
  RPBA_CUDA_CHECK(cudaMemsetAsync(L.gauge, 0, sizeof(int) * 4, s));
  RPBA_CUDA_CHECK(cudaMemsetAsync(L.o_flag, 0, nobs0 ? nobs0 : 1, s));
  RPBA_CUDA_CHECK(cudaMemsetAsync(L.o_flagnew, 0, nobs0 ? nobs0 : 1, s));
}

void rpba_handle::structure() {
  coarse_stale = true;
  ++structure_version;
  long long npairs = 0;
  int nb = 0;
  PROF("structure_pairs", 3, nb = build_pairs(L, S, max_pairs, &npairs, s));
  npairs_cur = npairs;
  ensure_blocks(nb);
  PROF("structure_bsr", 6, build_bsr(L, S, s));
  if (opt.verbose & 4) {
    char line[160];
    std::snprintf(line, sizeof line, "Structure: cameras %d points %d observations %d pair contributions %lld "
                  "off-diagonal blocks %d work items %d\n", L.nimg, L.npts, L.nobs, npairs, L.nboff, L.nitems);
    log += line;
  }
}

// CalcBundleSep (rbacore.cpp:1094-1195): assemble, solve, back-substitute.
bool rpba_handle::calc_bundle_sep(double multfact, int nrunknowns) {
  const double multfact1 = 1. + multfact;
  // Algorithmic bytes of each launch (inputs read once, outputs written once;
  // E = 8 or 4 bytes per record entry in the FP64 or FP32 form):
  //  point : obs (cam 4, xg 8, w 16, record 31 E out) + point (X 24, off 8,
  //          point record 12 E out) + trial cameras 160
  //  camera: obs (list 4, record part 23 E) + camera (block 81 E + rhs 72 out)
  //  pair  : obs records (Bc G, 24 E) + points (V^-1, 9 E; not read in the
  //          FP32 form) + contributions (8) + off-diagonal blocks out (81 E)
  const double No = L.nobs, Np = L.npts, Nc = nimg, Nb = L.nboff;
  const double E = L.rec32 ? 4. : 8.;
  prof.next_bytes = No * (4 + 8 + 16 + 31 * E) + Np * (24 + 8 + 12 * E) + Nc * 160;
  PROF("point", 1, launch_point_pass(L, multfact1, s));
  prof.next_bytes = No * (4 + 23 * E) + (Nc - begini) * (81 * E + 72);
  PROF("camera", 1, launch_camera_pass(L, multfact1, s));
  prof.next_bytes = No * 24 * E + (L.rec32 ? 0. : Np * 72) + npairs_cur * 8. + Nb * 81 * E;
  PROF("pair", 1, launch_pair_pass(L, s));
  int msize = 0;
  for (int k = begini; k < nimg; ++k) msize += camparv[k + 1] - camparv[k];
  if (msize < 1000) msize = 1000;
  if (opt.pcg_max_iterations > 0) msize = opt.pcg_max_iterations;
  if (opt.solver == RPBA_SOLVER_DIRECT) {
    if (!ensure_direct()) {
      direct_too_large = true;
      return true;
    }
    CoopLock lk(this);
    PROF("direct", 3, direct_solve(L, DW, W.xbest, s));
  } else if (opt.solver == RPBA_SOLVER_LEARNED) {
    // PCG with the two-level preconditioner: the learned block-Jacobi part
    // plus the aggregate coarse space.  Stop rule: the reference's
    // (pcg_tolerance == 0) or a relative preconditioned residual; past the
    // iteration cap the direct solve takes over
    const int mode = opt.pcg_tolerance > 0. ? 1 : 0;
    const int cap = opt.pcg_max_iterations > 0 ? opt.pcg_max_iterations : msize;
    // The coarse operator is rebuilt whenever the observation weights or
    // the structure changed (every step of the robust pass: reweighting
    // rescales S); in the refinement pass the operator of an earlier
    // linearisation is reused -- any SPD coarse operator keeps M SPD -- with
    // the iteration cap cut to three times the iterations of its first use.
    // If a reused operator misses that cap, it is rebuilt and the solve
    // repeated.
    const CoarseWork *cw = ensure_coarse();
    int it[3] = {0, 0, 0};
    bool fresh = false;
    for (int attempt = 0; attempt < 2; ++attempt) {
      if (cw && (coarse_stale || attempt > 0)) {
        const double nc = CW.nc;
        prof.next_bytes = (Nc + 2. * Nb) * (L.blocks32 ? 324. : 648.) + nc * nc * 8;
        PROF("coarse_assemble", 4, coarse_assemble(L, CW, structure_version, s));
        prof.next_bytes = 4. * nc * nc * 8;
        {
          CoopLock lk(this);
          // diagonal scaling, tile metadata, packing, the factorisation and
          // inverse, unpacking
          PROF("coarse_factor", 5, coarse_factor(CW, s));
        }
        coarse_stale = false;
        fresh = true;
      }
      const int cap_try = (cw && !fresh) ? std::min(cap, 3 * coarse_ref_iters + 20) : cap;
      {
        CoopLock lk(this);
        prof.next_bytes = setup_bytes(d_weights != nullptr);
        // set-up kernels: rsqrt, features and set-up with weights (else the
        // set-up alone), the coarse restriction and prolongation
        PROF("pcg_setup", (d_weights ? 3 : 1) + (cw ? 2 : 0), pcg_prepare(L, W, mode, d_weights, cw, s));
        PROF("pcg", 1, pcg_iterate(L, W, cap_try, pcg_grid, s, mode, opt.pcg_tolerance, cw));
      }
      RPBA_CUDA_CHECK(cudaMemcpyAsync(it, W.iters, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
      if (cw) RPBA_CUDA_CHECK(cudaMemcpyAsync(it + 2, CW.err, sizeof(int), cudaMemcpyDeviceToHost, s));
      RPBA_CUDA_CHECK(cudaStreamSynchronize(s));
      learned_iters += it[0];
      if (prof.on)
        for (auto itp = prof.pending.rbegin(); itp != prof.pending.rend(); ++itp)
          if (std::string(itp->name) == "pcg") {
            itp->bytes = (double)it[0] * pcg_bytes_per_iteration(cw != nullptr);
            break;
          }
      if (fresh) coarse_ref_iters = it[0];
      const bool conv = (mode == 1 ? it[1] != 0 : it[0] < cap_try) && it[2] == 0;
      if (conv || fresh || !cw) break;
      ++rep.coarse_rebuilds;
    }
    const bool ok = (mode == 1 ? it[1] != 0 : it[0] < cap) && it[2] == 0;
    if (opt.verbose & 4) {
      char line[128];
      std::snprintf(line, sizeof line, "PCG: iterations %d converged %d coarse %d status %d\n", it[0], it[1],
                    cw ? CW.nagg : 0, it[2]);
      log += line;
    }
    if (!ok) {
      // fallbacks: block-Jacobi PCG alone (no coarse space, no network) to
      // the same tolerance and the reference's cap; then the dense direct
      // solve where it fits (the dense matrix of 40k unknowns is 12.8 GB);
      // past that the block-Jacobi PCG's best iterate is used
      ++rep.pcg_fallbacks;
      int it2[2] = {0, 0};
      {
        CoopLock lk(this);
        prof.next_bytes = setup_bytes(false);
        PROF("pcg_setup", 1, pcg_prepare(L, W, 1, nullptr, nullptr, s));
        PROF("pcg", 1, pcg_iterate(L, W, msize, pcg_grid, s, 1, opt.pcg_tolerance > 0. ? opt.pcg_tolerance : 1e-6,
                                    nullptr));
      }
      RPBA_CUDA_CHECK(cudaMemcpyAsync(it2, W.iters, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
      RPBA_CUDA_CHECK(cudaStreamSynchronize(s));
      learned_iters += it2[0];
      if (opt.verbose & 4) {
        char line[128];
        std::snprintf(line, sizeof line, "PCG fallback (block-Jacobi): iterations %d converged %d\n", it2[0], it2[1]);
        log += line;
      }
      if (it2[1] == 0 && ensure_direct()) {
        CoopLock lk(this);
        PROF("direct", 3, direct_solve(L, DW, W.xbest, s));
      }
    }
  } else {
    {
      CoopLock lk(this);
      prof.next_bytes = setup_bytes(false);
      PROF("pcg_setup", 1, pcg_prepare(L, W, 0, nullptr, nullptr, s));
      PROF("pcg", 1, pcg_iterate(L, W, msize, pcg_grid, s, 0, 0., nullptr));
    }
    pcg_pending = true;
  }
  if (rec_T) {
    const CoarseWork *cw = ensure_coarse();
    if (cw) coarse_setup(L, CW, structure_version, s);
    learned_record(L, cw, W.xbest, W.Cinv, W.drs, rec_seed + 104729ull * (unsigned long long)rep.linear_solves, *rec_T,
                   *rec_H, s);
  }
  // back-substitution: obs (camera 4, record 24 E) + the cameras' steps
  // (72, read once) + point (point record 12 E, offsets 8, step 24 out)
  prof.next_bytes = No * (4 + 24 * E) + Nc * 72 + Np * (12 * E + 8 + 24);
  PROF("backsub", 1, launch_backsub(L, W.xbest, s));
  PROF("xcam", 1, launch_xcam(L, W.xbest, s));
  PROF("update", 1, launch_update(L, nrunknowns, s));
  RPBA_CUDA_CHECK(cudaGetLastError());
  return false;
}

// RobustDelete (rbacore.cpp:922-995) as a device compaction.
void rpba_handle::robust_delete() {
  const int no = L.nobs, np = L.npts;
  RPBA_CUDA_CHECK(cudaMemsetAsync(okeep + no, 0, sizeof(int), s));
  RPBA_CUDA_CHECK(cudaMemsetAsync(pkeep + np, 0, sizeof(int), s));
  PROF("delete", 1, launch_delete_mark(L, okeep, pkeep, s));
  size_t bytes = S.cub_bytes;
  RPBA_CUDA_CHECK(cub_exclusive_sum_int(S.cub_tmp, bytes, okeep, oidx, no + 1, s));
  bytes = S.cub_bytes;
  RPBA_CUDA_CHECK(cub_exclusive_sum_int(S.cub_tmp, bytes, pkeep, pidx, np + 1, s));
  int tot[2];
  RPBA_CUDA_CHECK(cudaMemcpyAsync(&tot[0], oidx + no, sizeof(int), cudaMemcpyDeviceToHost, s));
  RPBA_CUDA_CHECK(cudaMemcpyAsync(&tot[1], pidx + np, sizeof(int), cudaMemcpyDeviceToHost, s));
  RPBA_CUDA_CHECK(cudaStreamSynchronize(s));
  const int nobs_new = tot[0], npts_new = tot[1];
  PROF("delete", 2, launch_delete_compact(L, oidx, pidx, okeep, pkeep, nobs_new, npts_new, o_cam_n, o_slot_n, o_pt_n,
                                          o_xg_n, o_wold_n, pt_off_n, pt_id_n, X_n, s));
  std::swap(L.o_cam, o_cam_n);
  std::swap(L.o_slot, o_slot_n);
  std::swap(L.o_pt, o_pt_n);
  std::swap(L.o_xg, o_xg_n);
  std::swap(L.o_wold, o_wold_n);
  std::swap(L.pt_off, pt_off_n);
  std::swap(L.pt_id, pt_id_n);
  if (npts_new > 0)
    RPBA_CUDA_CHECK(cudaMemcpyAsync(L.XPM + nrioff, X_n, sizeof(double) * 3 * npts_new, cudaMemcpyDeviceToDevice, s));
  rep.obs_deleted += no - nobs_new;
  rep.points_deleted += np - npts_new;
  L.nobs = nobs_new;
  L.npts = npts_new;
}

// Adjust (rbacore.cpp:333-616, itbreakflag false, no GCPs).
int rpba_handle::adjust() {
  int itt = 0;
  const float sig0frac = lflflag ? 1.01f : 1.05f;
  double multfact = 1.e-3;
  int solves = 0;
  bool cap_hit = false;
  float sig0old = 0.f, sig0in = 0.f, wsum = 0.f, wsumg = 0.f;
  int nrobsnew = 0, nrunknownsnew = 0, redundancynew = 0;
  std::vector<int> cnt(nimg + 1);
  for (int it = 0; it < 2; ++it) {
    if (cap_hit) break;
    sig0old = 1.e20f;
    if (it > 0) multfact = 1.e-6;
    const int imagepointnr = L.nobs;
    int nrobs = 2 * imagepointnr;
    PROF("structure_cam", 2, build_camera_order(L, S, s));
    RPBA_CUDA_CHECK(cudaMemcpyAsync(cnt.data(), S.ccnt, sizeof(int) * nimg, cudaMemcpyDeviceToHost, s));
    RPBA_CUDA_CHECK(cudaStreamSynchronize(s));
    for (int i = 0; i < nimg; ++i)
      if (cnt[i] == 0) {
        if (nimg > 3) log += "BA-Error: No observations in image " + std::to_string(i) + " (image index)\n";
        return RPBA_ERR_NO_OBS_IMAGE;
      }
    PROF("weights", 1, launch_prepare_weights(L, s));
    wsum = seq_sum(L.o_wterm, L.nobs);
    wsum = (float)(2 * imagepointnr) / wsum;
    wsumg = wsum;
    PROF("encode", 1, launch_encode(L, s));
    const int nrioff3 = nrioff + 3 * L.npts;
    int nrunknowns = nrioff3 + nadd * nimg;
    int redundancy = nrobs - nrunknowns;
    if (redundancy < 0) {
      if (nimg > 3) log += "BA-Error: Low redundancy\n";
      return RPBA_ERR_LOW_REDUNDANCY;
    }
    RPBA_CUDA_CHECK(cudaMemsetAsync(L.x, 0, sizeof(double) * xpmsize, s));
    structure();
    if (it == 0) {
      PROF("decode", 1, launch_decode(L, L.XPM, s));
      PROF("cost", 1, launch_cost(L, L.XPM, true, s));
      float sig0 = seq_sum(L.o_cost, L.nobs);
      sig0 = sig0 * wsumg / (float)redundancy;
      sig0in = sig0old = sig0;
    } else {
      sig0in = sig0old;
    }
    int iflag = robust ? 2 : 1;
    int iter = 1;
    const int nunk_given = nrunknowns, nobs_given = nrobs;
    while (iflag > 0) {
      if (it == 0 && robust) {
        nrunknowns = nunk_given;
        nrobs = nobs_given;
        PROF("reweight", 3, launch_reweight(L, iflag, vals, sig00v, nflag, s));
        coarse_stale = true;
        int nf = 0;
        RPBA_CUDA_CHECK(cudaMemcpyAsync(&nf, nflag, sizeof(int), cudaMemcpyDeviceToHost, s));
        wsum = seq_sum(L.o_wterm, L.nobs);
        nrobs -= 2 * nf;
        redundancy = nrobs - nrunknowns;
        wsum = (float)(2 * imagepointnr) / wsum;
        wsumg = wsum;
      }
      calc_bundle_sep(multfact, nrunknowns);
      if (direct_too_large) return RPBA_ERR_TOO_LARGE;
      ++solves;
      rep.linear_solves = solves;
      PROF("decode", 1, launch_decode(L, L.XPMn, s));
      PROF("cost", 1, launch_cost(L, L.XPMn, true, s));
      {
        CoopLock lk(this);
        prof.next_bytes = 4. * L.nobs;
        PROF("seq_sum", 1, launch_exact_sum(L.o_cost, L.nobs, sums, ES, s));
      }
      struct {
        float sig0;
        int err;
        int iters;
      } hv;
      RPBA_CUDA_CHECK(cudaMemcpyAsync(&hv.sig0, sums, sizeof(float), cudaMemcpyDeviceToHost, s));
      RPBA_CUDA_CHECK(cudaMemcpyAsync(&hv.err, L.err, sizeof(int), cudaMemcpyDeviceToHost, s));
      RPBA_CUDA_CHECK(cudaMemcpyAsync(&hv.iters, W.iters, sizeof(int), cudaMemcpyDeviceToHost, s));
      RPBA_CUDA_CHECK(cudaStreamSynchronize(s));
      rep.pcg_iterations += opt.solver == RPBA_SOLVER_PCG ? hv.iters : 0;
      if (prof.on && pcg_pending)
        for (auto it = prof.pending.rbegin(); it != prof.pending.rend(); ++it)
          if (std::string(it->name) == "pcg") {
            it->bytes = (double)hv.iters * pcg_bytes_per_iteration(false);
            break;
          }
      pcg_pending = false;
      if (hv.err & 2) return RPBA_ERR_DEVICE_TIMEOUT;
      if (hv.err & 4) return RPBA_ERR_SOLVER;
      if (hv.err & 1) return RPBA_ERR_NAN_STEP;
      float sig0 = hv.sig0 * wsumg / (float)redundancy;
      if (sig0old < sig0 * sig0frac) --iflag;
      if (sig0 <= sig0old || iter == 1) {
        PROF("store", 1, launch_store(L, xpmsize, s));
        sig0old = sig0;
        nrobsnew = nrobs;
        nrunknownsnew = nrunknowns;
        redundancynew = redundancy;
      }
      if (itt > 200) break;
      ++itt;
      ++iter;
      if (opt.max_lm_iterations >= 0 && solves >= opt.max_lm_iterations) {
        cap_hit = true;
        break;
      }
    }
    const float s_in = std::sqrt(sig0in * ihw2), s_out = std::sqrt(sig0old * ihw2);
    int red = redundancy, nob = nrobs, nun = nrunknowns;
    if (it == 0 && robust) {
      red = redundancynew;
      nob = nrobsnew;
      nun = nrunknownsnew;
    }
    log += "Sigma0: " + fmt_g(s_in) + ' ' + fmt_g(s_out) + "  " + std::to_string(red) + ' ' + std::to_string(nob) +
           ' ' + std::to_string(nun) + "  IT: " + std::to_string(it) + "  ITT: " + std::to_string(itt) + '\n';
    rep.sigma0_in[it] = s_in;
    rep.sigma0_out[it] = s_out;
    rep.redundancy[it] = red;
    rep.nrobs[it] = nob;
    rep.nrunknowns[it] = nun;
    rep.itt[it] = itt;
    rep.passes_done = it + 1;
    if (robust && it == 0) robust_delete();
  }
  rep.linear_solves = solves;
  if (opt.solver == RPBA_SOLVER_LEARNED) rep.pcg_iterations = learned_iters;
  return RPBA_OK;
}

// Adjust in GCP mode (rbacore.cpp:333-616 with robust = false, itbreakflag
// = true, itmaxnum = 0, gcpflag = true): the per-partition call of the
// parallel RPBA (rpbacore.cpp:225-229).  The cost with the priors, one damped
// step (multfact 1e-4) stored unconditionally, and the Sigma0 / Sigma0AO
// lines.  sig0ao is reset only by the first cost evaluation and by
// CalcBundleSep, so the post-step value accumulates the prior terms of the
// assembly pass and the back-substitution pass (both at the start state) and
// of the trial cost pass, in that order: one sequential float sum over three
// segments of per-point terms.
int rpba_handle::adjust_gcp_step() {
  const double multfact = 1.e-4;
  const int imagepointnr = L.nobs, np = L.npts;
  const int nrobsao = 3 * nrgcp;
  const int nrobs = 2 * imagepointnr + nrobsao;
  std::vector<int> cnt(nimg + 1);
  PROF("structure_cam", 2, build_camera_order(L, S, s));
  RPBA_CUDA_CHECK(cudaMemcpyAsync(cnt.data(), S.ccnt, sizeof(int) * nimg, cudaMemcpyDeviceToHost, s));
  RPBA_CUDA_CHECK(cudaStreamSynchronize(s));
  for (int i = 0; i < nimg; ++i)
    if (cnt[i] == 0) {
      if (nimg > 3) log += "BA-Error: No observations in image " + std::to_string(i) + " (image index)\n";
      return RPBA_ERR_NO_OBS_IMAGE;
    }
  // a float sum of terms of either sign, in array order
  auto seq_sum_any = [&](const float *v, int n) {
    float out = 0.f;
    if (n > 0) {
      launch_seq_sum(v, n, sums + 1, s);
      RPBA_CUDA_CHECK(cudaMemcpyAsync(&out, sums + 1, sizeof(float), cudaMemcpyDeviceToHost, s));
      RPBA_CUDA_CHECK(cudaStreamSynchronize(s));
    }
    return out;
  };
  // PrepareWeights2D / PrepareWeights3D (rbacore.cpp:704-818)
  PROF("weights", 1, launch_prepare_weights(L, s));
  float wsum = seq_sum(L.o_wterm, L.nobs);
  float wsumao = w3diag_sum;
  const float wsumg = (float)(2 * imagepointnr + nrobsao) / (wsumao + wsum);
  wsumao = (float)nrobsao / wsumao;
  wsum = (float)(2 * imagepointnr) / wsum;
  PROF("encode", 1, launch_encode(L, s));
  // the additional parameters count once per camera of the scene
  const int nrunknowns = nrioff + 3 * np + nadd * ncam_total;
  const int redundancy = nrobs - nrunknowns;
  if (redundancy < 0) {
    if (nimg > 3) log += "BA-Error: Low redundancy\n";
    return RPBA_ERR_LOW_REDUNDANCY;
  }
  RPBA_CUDA_CHECK(cudaMemsetAsync(L.x, 0, sizeof(double) * xpmsize, s));
  structure();
  // the cost at the start state
  PROF("decode", 1, launch_decode(L, L.XPM, s));
  PROF("cost", 1, launch_cost(L, L.XPM, true, s));
  float sig0 = seq_sum(L.o_cost, L.nobs);
  launch_gcp_cost(L, L.XPM, aoterm, s);
  float sig0ao = seq_sum_any(aoterm, np);
  const float sig0aoin = sig0 * wsumg / (float)redundancy;
  sig0 = (sig0 + sig0ao) * wsumg / (float)(redundancy + nrobsao - 7);
  const float sig0in = sig0;
  // one damped step; its two passes see the priors at the start state
  if (np > 0) {
    RPBA_CUDA_CHECK(cudaMemcpyAsync(aoterm + np, aoterm, sizeof(float) * np, cudaMemcpyDeviceToDevice, s));
  }
  calc_bundle_sep(multfact, nrunknowns);
  if (direct_too_large) return RPBA_ERR_TOO_LARGE;
  rep.linear_solves = 1;
  PROF("decode", 1, launch_decode(L, L.XPMn, s));
  PROF("cost", 1, launch_cost(L, L.XPMn, true, s));
  launch_gcp_cost(L, L.XPMn, aoterm + 2 * (size_t)np, s);
  {
    CoopLock lk(this);
    prof.next_bytes = 4. * L.nobs;
    PROF("seq_sum", 1, launch_exact_sum(L.o_cost, L.nobs, sums, ES, s));
  }
  struct {
    float sig0;
    int err;
    int iters;
  } hv;
  RPBA_CUDA_CHECK(cudaMemcpyAsync(&hv.sig0, sums, sizeof(float), cudaMemcpyDeviceToHost, s));
  RPBA_CUDA_CHECK(cudaMemcpyAsync(&hv.err, L.err, sizeof(int), cudaMemcpyDeviceToHost, s));
  RPBA_CUDA_CHECK(cudaMemcpyAsync(&hv.iters, W.iters, sizeof(int), cudaMemcpyDeviceToHost, s));
  RPBA_CUDA_CHECK(cudaStreamSynchronize(s));
  pcg_pending = false;
  rep.pcg_iterations = opt.solver == RPBA_SOLVER_PCG ? hv.iters : 0;
  if (hv.err & 2) return RPBA_ERR_DEVICE_TIMEOUT;
  if (hv.err & 4) return RPBA_ERR_SOLVER;
  if (hv.err & 1) return RPBA_ERR_NAN_STEP;
  // the post-step sig0ao: one running float sum over the three passes'
  // terms (the start state twice, the trial state once)
  sig0ao = seq_sum_any(aoterm, 3 * np);
  const float sig0aoiold = hv.sig0 * wsumg / (float)redundancy;
  const float sig0old = (hv.sig0 + sig0ao) * wsumg / (float)(redundancy + nrobsao - 7);
  PROF("store", 1, launch_store(L, xpmsize, s));
  const float s_in = std::sqrt(sig0in * ihw2), s_out = std::sqrt(sig0old * ihw2);
  log += "Sigma0: " + fmt_g(std::sqrt(sig0aoin * ihw2)) + ' ' + fmt_g(std::sqrt(sig0aoiold * ihw2)) + "  " +
         std::to_string(redundancy) + ' ' + std::to_string(nrobs) + ' ' + std::to_string(nrunknowns) +
         "  IT: 0  ITT: 0\n";
  log += "Sigma0AO: " + fmt_g(std::sqrt(sig0ao * wsumao / (float)(nrobsao - 7))) + "  " + fmt_g(s_in) + ' ' +
         fmt_g(s_out) + "  " + std::to_string(nrobsao) + " " + fmt_g(wsumao) + '\n';
  rep.sigma0_in[0] = s_in;
  rep.sigma0_out[0] = s_out;
  rep.redundancy[0] = redundancy;
  rep.nrobs[0] = nrobs;
  rep.nrunknowns[0] = nrunknowns;
  rep.passes_done = 1;
  return RPBA_OK;
}

// ------------------------------------------------------------ C ABI

namespace {

int guard(int (*fn)(void *), void *arg) {
  try {
    return fn(arg);
  } catch (const CudaError &e) {
    std::fprintf(stderr, "rpba_b200: CUDA error %s at %s\n", cudaGetErrorString(e.code), e.what);
    return RPBA_ERR_CUDA;
  } catch (const std::bad_alloc &) {
    return RPBA_ERR_CUDA;
  }
}

// taken by the cooperative launches of every rpba_lsa_gcp_step in the process
std::mutex g_gcp_coop;

}  // namespace

extern "C" {

const char *rpba_status_string(int32_t st) {
  switch (st) {
    case RPBA_OK: return "ok";
    case RPBA_ERR_ARG: return "invalid argument";
    case RPBA_ERR_CUDA: return "CUDA error";
    case RPBA_ERR_NO_OBS_IMAGE: return "BA-Error: No observations in image";
    case RPBA_ERR_LOW_REDUNDANCY: return "BA-Error: Low redundancy";
    case RPBA_ERR_NAN_STEP: return "BA-Error: NANs in result vector";
    case RPBA_ERR_DEVICE_TIMEOUT: return "device wait timed out";
    case RPBA_ERR_IO: return "I/O error";
    case RPBA_ERR_UNSUPPORTED: return "unsupported input";
    case RPBA_ERR_NO_DEVICE: return "no CUDA device";
    case RPBA_ERR_SOLVER: return "direct solve failed";
    case RPBA_ERR_TOO_LARGE: return "input exceeds the fixed scratch of an allocation-free call";
    case RPBA_ERR_COMM: return "a collective between ranks failed";
    default: return "unknown status";
  }
}

const char *rpba_version(void) { return "rpba_b200 0.1 (sm_100a)"; }

int32_t rpba_create(rpba_handle **h, const rpba_block *blk, const rpba_options *opt) {
  if (!h || !blk || !opt) return RPBA_ERR_ARG;
  *h = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= opt->device) return RPBA_ERR_NO_DEVICE;
  if (blk->n_images < 1 || blk->n_points < 0) return RPBA_ERR_ARG;
  rpba_handle *H = new rpba_handle();
  struct A {
    rpba_handle *H;
    const rpba_block *b;
    const rpba_options *o;
  } a{H, blk, opt};
  const int st = guard([](void *p) {
    A *a = (A *)p;
    return create_impl(a->H, a->b, a->o);
  }, &a);
  if (st != RPBA_OK) {
    delete H;
    return st;
  }
  *h = H;
  return RPBA_OK;
}

int32_t rpba_solve(rpba_handle *H, rpba_report *rep) {
  if (!H || H->opt.exteval) return RPBA_ERR_ARG;
  const int st = guard([](void *p) {
    rpba_handle *H = (rpba_handle *)p;
    RPBA_CUDA_CHECK(cudaSetDevice(H->dev));
    AsyncScope scope(H->s, H->owned, H->owned_async);
    H->log.clear();
    std::memset(&H->rep, 0, sizeof H->rep);
    H->learned_iters = 0;
    H->prof.s = H->s;
    H->prof.on = (H->opt.verbose & 2) != 0;
    H->prof.reset();
    H->rep.points_used = H->npts0;
    RPBA_CUDA_CHECK(cudaEventRecord(H->ev0, H->s));
    H->reset();
    const int r = H->adjust();
    RPBA_CUDA_CHECK(cudaEventRecord(H->ev1, H->s));
    RPBA_CUDA_CHECK(cudaEventSynchronize(H->ev1));
    float ms = 0.f;
    RPBA_CUDA_CHECK(cudaEventElapsedTime(&ms, H->ev0, H->ev1));
    H->rep.solve_seconds = ms * 1e-3;
    H->prof.resolve();
    H->rep.kernel_launches = H->prof.launches;
    launch_final_cost(H->L, H->fc_part, H->fc_nparts, H->s);
    std::vector<double> part(2 * H->fc_nparts);
    RPBA_CUDA_CHECK(cudaMemcpyAsync(part.data(), H->fc_part, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, H->s));
    RPBA_CUDA_CHECK(cudaStreamSynchronize(H->s));
    double c = 0., q = 0.;
    for (int i = 0; i < H->fc_nparts; ++i) {
      c += part[2 * i];
      q += part[2 * i + 1];
    }
    H->rep.cost = c;
    H->rep.rms = H->L.nobs > 0 ? std::sqrt(q / H->L.nobs) : 0.;
    H->rep.status = r;
    return r;
  }, H);
  if (rep) *rep = H->rep;
  if (rep) rep->status = st;
  return st;
}

int32_t rpba_get_log(rpba_handle *H, char *log, size_t cap) {
  if (!H || !log || cap == 0) return RPBA_ERR_ARG;
  const size_t n = std::min(cap - 1, H->log.size());
  std::memcpy(log, H->log.data(), n);
  log[n] = 0;
  return RPBA_OK;
}

namespace {
// rpba_get_state on the device, for tracks kept as one CSR over strictly
// increasing point ids (the layout the solver keeps).  Violations of that
// layout set *bad.
__global__ void k_state_check(const int *pt_off, const int *pt_id, int np, int nall, int *bad) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= np) return;
  if (pt_off[q] > pt_off[q + 1] || pt_id[q] < 0 || pt_id[q] >= nall || (q > 0 && pt_id[q - 1] >= pt_id[q]))
    atomicOr(bad, 1);
}
// The solved points into the caller's point array (the others keep their
// input values, already in XXf).
__global__ void k_state_xx(const double *X, const int *pt_id, int np, float *XXf) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= np) return;
  const size_t i = (size_t)pt_id[q];
#pragma unroll
  for (int j = 0; j < 3; ++j) XXf[3 * i + j] = (float)X[3 * (size_t)q + j];
}
// Track offsets over all nall input points: point ids from that of kept
// point q - 1 up to (not including) that of kept point q end where kept
// point q - 1 ends (pt_off[q]); off[0] = 0.  Thread q in 0 .. np.
__global__ void k_state_off(const int *pt_off, const int *pt_id, int np, int nall, int *off) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q > np) return;
  if (q == 0) off[0] = 0;
  const int lo = q == 0 ? 0 : pt_id[q - 1], hi = q == np ? nall : pt_id[q];
  const int v = pt_off[q];
  for (int i = lo; i < hi; ++i) off[i + 1] = v;
}
}  // namespace

// OutputLSAc + PointXXvOut (rbacore.cpp:644-666, 1978-2010).
int32_t rpba_get_state(rpba_handle *H, rpba_block *blk) {
  if (!H || !blk || H->opt.exteval) return RPBA_ERR_ARG;
  if (blk->n_images != H->nimg || blk->n_points != H->XXnr) return RPBA_ERR_ARG;
  struct A {
    rpba_handle *H;
    rpba_block *b;
  } a{H, blk};
  return guard([](void *p) {
    A *a = (A *)p;
    rpba_handle *H = a->H;
    rpba_block *b = a->b;
    RPBA_CUDA_CHECK(cudaSetDevice(H->dev));
    const int n = H->nimg, no = H->L.nobs, np = H->L.npts, nall = H->XXnr;
    std::vector<double> P(12 * (size_t)n);
    std::vector<CamState> cams(n);
    auto dn = [&](void *h, const void *d, size_t bytes) {
      if (bytes) RPBA_CUDA_CHECK(cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, H->s));
    };
    auto cameras_out = [&]() {
      for (size_t i = 0; i < P.size(); ++i) b->pmat[i] = (float)P[i];
      for (int i = 0; i < n; ++i) {
        const CamState &c = cams[i];
        float *K = b->K + 9 * i;
        const float *Ki = H->h_K.data() + 9 * i;
        K[0] = (float)c.K00;
        K[1] = (float)c.K01;
        K[2] = (float)c.K02;
        K[3] = Ki[3];
        K[4] = (float)c.K11;
        K[5] = (float)c.K12;
        K[6] = Ki[6];
        K[7] = Ki[7];
        K[8] = 1.f;
        b->distpara[2 * i] = (float)c.d0;
        b->distpara[2 * i + 1] = (float)c.d1;
      }
    };
    dn(P.data(), H->L.Pacc, sizeof(double) * P.size());
    dn(cams.data(), H->L.camn, sizeof(CamState) * n);
    // The output tracks are the device's, point by point in increasing
    // point order.  When the device lists are one CSR from 0 to nobs over
    // strictly increasing point ids (the layout the solver keeps), that
    // concatenation is the device arrays as they are, and the points and
    // offsets are formed on the device: everything goes straight into the
    // caller's arrays.  Otherwise the tracks are gathered point by point on
    // the host.
    {
      int *dbad = nullptr, *doff = nullptr;
      float *dxx = nullptr;
      RPBA_CUDA_CHECK(cudaMallocAsync(&dbad, sizeof(int) * 4, H->s));
      RPBA_CUDA_CHECK(cudaMemsetAsync(dbad, 0, sizeof(int) * 4, H->s));
      if (np > 0) k_state_check<<<(np + 255) / 256, 256, 0, H->s>>>(H->L.pt_off, H->L.pt_id, np, nall, dbad);
      int ends[2] = {0, 0}, bad = 0;
      dn(&ends[0], H->L.pt_off, sizeof(int));
      dn(&ends[1], H->L.pt_off + np, sizeof(int));
      dn(&bad, dbad, sizeof(int));
      RPBA_CUDA_CHECK(cudaStreamSynchronize(H->s));
      const bool fast = bad == 0 && ends[0] == 0 && ends[1] == no && no <= H->n_track_in;
      if (fast) {
        RPBA_CUDA_CHECK(cudaMallocAsync(&dxx, sizeof(float) * 3 * std::max(nall, 1), H->s));
        RPBA_CUDA_CHECK(cudaMallocAsync(&doff, sizeof(int) * (nall + 1), H->s));
        if (nall)
          RPBA_CUDA_CHECK(cudaMemcpyAsync(dxx, H->d_XXin, sizeof(float) * 3 * nall, cudaMemcpyDeviceToDevice, H->s));
        if (np > 0) k_state_xx<<<(np + 255) / 256, 256, 0, H->s>>>(H->L.XPM + H->nrioff, H->L.pt_id, np, dxx);
        k_state_off<<<(np + 1 + 255) / 256, 256, 0, H->s>>>(H->L.pt_off, H->L.pt_id, np, nall, doff);
        RPBA_CUDA_CHECK(cudaGetLastError());
        dn(b->XX, dxx, sizeof(float) * 3 * nall);
        dn(b->pt_obs_off, doff, sizeof(int) * (nall + 1));
        dn(b->pt_obs_image, H->L.o_cam, sizeof(int) * no);
        dn(b->pt_obs_slot, H->L.o_slot, sizeof(int) * no);
        RPBA_CUDA_CHECK(cudaFreeAsync(dxx, H->s));
        RPBA_CUDA_CHECK(cudaFreeAsync(doff, H->s));
      }
      RPBA_CUDA_CHECK(cudaFreeAsync(dbad, H->s));
      if (fast) {
        RPBA_CUDA_CHECK(cudaStreamSynchronize(H->s));
        cameras_out();
        // entries past the kept observations are 0
        if (H->n_track_in > no) {
          std::memset(b->pt_obs_image + no, 0, sizeof(int) * (size_t)(H->n_track_in - no));
          std::memset(b->pt_obs_slot + no, 0, sizeof(int) * (size_t)(H->n_track_in - no));
        }
        return (int)RPBA_OK;
      }
    }
    std::vector<int> pt_off(np + 1), pt_id(np);
    std::vector<double> X(3 * (size_t)np);
    dn(pt_off.data(), H->L.pt_off, sizeof(int) * (np + 1));
    dn(pt_id.data(), H->L.pt_id, sizeof(int) * np);
    dn(X.data(), H->L.XPM + H->nrioff, sizeof(double) * 3 * np);
    RPBA_CUDA_CHECK(cudaStreamSynchronize(H->s));
    bool direct = pt_off[0] == 0 && pt_off[np] == no && no <= H->n_track_in;
    for (int q = 0; q < np && direct; ++q)
      direct = pt_off[q] <= pt_off[q + 1] && pt_id[q] >= 0 && pt_id[q] < H->XXnr && (q == 0 || pt_id[q - 1] < pt_id[q]);
    std::vector<int> o_cam, o_slot;
    if (direct) {
      dn(b->pt_obs_image, H->L.o_cam, sizeof(int) * no);
      dn(b->pt_obs_slot, H->L.o_slot, sizeof(int) * no);
    } else {
      o_cam.resize(no);
      o_slot.resize(no);
      dn(o_cam.data(), H->L.o_cam, sizeof(int) * no);
      dn(o_slot.data(), H->L.o_slot, sizeof(int) * no);
    }
    RPBA_CUDA_CHECK(cudaStreamSynchronize(H->s));
    cameras_out();
    std::memcpy(b->XX, H->h_XX.data(), sizeof(float) * H->h_XX.size());
    int w = 0, q = 0;
    b->pt_obs_off[0] = 0;
    for (int i = 0; i < H->XXnr; ++i) {
      if (q < np && pt_id[q] == i) {
        if (direct) {
          w = pt_off[q + 1];
        } else {
          for (int o = pt_off[q]; o < pt_off[q + 1]; ++o, ++w) {
            b->pt_obs_image[w] = o_cam[o];
            b->pt_obs_slot[w] = o_slot[o];
          }
        }
        for (int j = 0; j < 3; ++j) b->XX[3 * i + j] = (float)X[3 * q + j];
        ++q;
      }
      b->pt_obs_off[i + 1] = w;
    }
    if (H->n_track_in > w) {
      std::memset(b->pt_obs_image + w, 0, sizeof(int) * (size_t)(H->n_track_in - w));
      std::memset(b->pt_obs_slot + w, 0, sizeof(int) * (size_t)(H->n_track_in - w));
    }
    return (int)RPBA_OK;
  }, &a);
}

// EvalLSA on the uploaded block (rpbacore.cpp:882-941).
int32_t rpba_exteval(rpba_handle *H, double *resid, rpba_report *rep) {
  if (!H || !H->opt.exteval) return RPBA_ERR_ARG;
  struct A {
    rpba_handle *H;
    double *resid;
    rpba_report *rep;
  } a{H, resid, rep};
  return guard([](void *p) {
    A *a = (A *)p;
    rpba_handle *H = a->H;
    RPBA_CUDA_CHECK(cudaSetDevice(H->dev));
    auto &own = H->owned;
    const int n = H->nimg, np = H->XXnr, ns = H->n_slots, nt = H->n_track_in;
    float *pm = dalloc<float>(12 * (size_t)n, own), *K = dalloc<float>(9 * (size_t)n, own);
    float *ds = dalloc<float>(2 * (size_t)n, own), *XX = dalloc<float>(3 * (size_t)std::max(np, 1), own);
    float *xg = dalloc<float>(2 * (size_t)std::max(ns, 1), own), *wx = dalloc<float>(std::max(ns, 1), own);
    float *wy = dalloc<float>(std::max(ns, 1), own), *wxy = dalloc<float>(std::max(ns, 1), own);
    int *io = dalloc<int>(n + 1, own), *po = dalloc<int>(np + 1, own);
    int *pi = dalloc<int>(std::max(nt, 1), own), *ps = dalloc<int>(std::max(nt, 1), own);
    double *res = dalloc<double>(2 * (size_t)std::max(nt, 1), own);
    float *term = dalloc<float>(std::max(np, 1), own), *sum = dalloc<float>(1, own);
    int *red = dalloc<int>(std::max(np, 1), own);
    auto up = [&](void *d, const void *h, size_t bytes) {
      if (bytes) RPBA_CUDA_CHECK(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, H->s));
    };
    up(pm, H->h_pmat.data(), sizeof(float) * 12 * n);
    up(K, H->h_K.data(), sizeof(float) * 9 * n);
    up(ds, H->h_dist.data(), sizeof(float) * 2 * n);
    up(XX, H->h_XX.data(), sizeof(float) * 3 * np);
    up(xg, H->h_xg.data(), sizeof(float) * 2 * ns);
    up(wx, H->h_wx.data(), sizeof(float) * ns);
    up(wy, H->h_wy.data(), sizeof(float) * ns);
    up(wxy, H->h_wxy.data(), sizeof(float) * ns);
    up(io, H->h_img_off.data(), sizeof(int) * (n + 1));
    up(po, H->h_pt_off.data(), sizeof(int) * (np + 1));
    up(pi, H->h_pt_img.data(), sizeof(int) * nt);
    up(ps, H->h_pt_slot.data(), sizeof(int) * nt);
    launch_exteval(np, po, pi, ps, io, pm, K, ds, XX, xg, wx, wy, wxy, res, term, red, H->s);
    launch_exact_sum(term, np, sum, H->ES, H->s);
    std::vector<int> hred(np);
    float s = 0.f;
    if (np) RPBA_CUDA_CHECK(cudaMemcpyAsync(hred.data(), red, sizeof(int) * np, cudaMemcpyDeviceToHost, H->s));
    RPBA_CUDA_CHECK(cudaMemcpyAsync(&s, sum, sizeof(float), cudaMemcpyDeviceToHost, H->s));
    if (a->resid && nt)
      RPBA_CUDA_CHECK(cudaMemcpyAsync(a->resid, res, sizeof(double) * 2 * nt, cudaMemcpyDeviceToHost, H->s));
    RPBA_CUDA_CHECK(cudaStreamSynchronize(H->s));
    long redundancy = 0, nrobs = 0;
    for (int i = 0; i < np; ++i) {
      redundancy += hred[i];
      if (hred[i] > 0) nrobs += hred[i] + 3;
    }
    const long r = redundancy - (long)(n - 2) * 6 - 5 - (long)n * H->nadd;
    float sig0g = s;
    sig0g *= 1.f / (float)r;
    float ihw2 = 0.f;
    for (int i = 0; i < n; ++i) ihw2 += (float)((1 + 1) * (1 + 1)) * 0.25f;
    ihw2 /= (float)n;
    const float v = std::sqrt(sig0g * ihw2);
    H->log += "ITTTT: " + fmt_g(v) + ' ' + std::to_string(nrobs) + " " + std::to_string(r) + '\n';
    if (a->rep) {
      a->rep->exteval_sigma0 = v;
      a->rep->exteval_nrobs = nrobs;
      a->rep->exteval_redundancy = r;
    }
    return (int)RPBA_OK;
  }, &a);
}

int32_t rpba_float_sequential_sum(const float *v, int64_t n, int32_t device, float *out) {
  if (!out || n < 0 || n > 0x7fffffff || (n > 0 && !v)) return RPBA_ERR_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= device) return RPBA_ERR_NO_DEVICE;
  struct A {
    const float *v;
    int n, dev;
    float *out;
  } a{v, (int)n, device, out};
  return guard([](void *p) {
    A *a = (A *)p;
    RPBA_CUDA_CHECK(cudaSetDevice(a->dev));
    std::vector<void *> own;
    struct Free {
      std::vector<void *> &o;
      ~Free() {
        for (void *q : o) cudaFree(q);
      }
    } fr{own};
    cudaStream_t s = 0;
    ExactSumWork W{};
    W.max_grid = exact_sum_max_grid(a->dev);
    W.Rc = dalloc<long long>(2 * (size_t)W.max_grid, own);
    W.Mc = dalloc<long long>(2 * (size_t)W.max_grid, own);
    W.Tc = dalloc<int>(2 * (size_t)W.max_grid, own);
    W.ctl = dalloc<char>(16, own);
    W.bar = dalloc<unsigned>(2, own);
    W.err = dalloc<int>(1, own);
    float *dv = dalloc<float>(std::max(a->n, 1), own), *dout = dalloc<float>(1, own);
    RPBA_CUDA_CHECK(cudaMemset(W.err, 0, sizeof(int)));
    if (a->n) RPBA_CUDA_CHECK(cudaMemcpy(dv, a->v, sizeof(float) * a->n, cudaMemcpyHostToDevice));
    launch_exact_sum(dv, a->n, dout, W, s);
    int err = 0;
    RPBA_CUDA_CHECK(cudaMemcpy(a->out, dout, sizeof(float), cudaMemcpyDeviceToHost));
    RPBA_CUDA_CHECK(cudaMemcpy(&err, W.err, sizeof(int), cudaMemcpyDeviceToHost));
    return err ? (int)RPBA_ERR_DEVICE_TIMEOUT : (int)RPBA_OK;
  }, &a);
}

int32_t rpba_set_preconditioner(rpba_handle *H, const float *weights, int32_t n) {
  if (!H || H->opt.exteval) return RPBA_ERR_ARG;
  if (weights && n != RPBA_PRECOND_WEIGHTS) return RPBA_ERR_ARG;
  struct A {
    rpba_handle *H;
    const float *w;
  } a{H, weights};
  return guard([](void *p) {
    A *a = (A *)p;
    rpba_handle *H = a->H;
    RPBA_CUDA_CHECK(cudaSetDevice(H->dev));
    if (!a->w) {
      H->d_weights = nullptr;
      return (int)RPBA_OK;
    }
    static_assert(NN_WEIGHTS == RPBA_PRECOND_WEIGHTS, "weight count");
    if (!H->d_weights) {
      float *d = dalloc<float>(NN_WEIGHTS, H->owned);
      H->d_weights = d;
    }
    RPBA_CUDA_CHECK(cudaMemcpyAsync(H->d_weights, a->w, sizeof(float) * NN_WEIGHTS, cudaMemcpyHostToDevice, H->s));
    RPBA_CUDA_CHECK(cudaStreamSynchronize(H->s));
    return (int)RPBA_OK;
  }, &a);
}

namespace {

// device training set with the given capacities
struct TrainAlloc {
  TrainSet T{};
  TrainHost H{};
  TrainBufs B{};
  std::vector<void *> own;
  ~TrainAlloc() {
    for (void *q : own) cudaFree(q);
  }
  void alloc(int rows_cap, int ents_cap, int blocks_cap, int sys_cap, int probes) {
    T.rows_cap = rows_cap;
    T.probes = probes;
    T.f = dalloc<float>((size_t)rows_cap * NN_F, own);
    T.sinv = dalloc<float>((size_t)rows_cap * 81, own);
    T.b = dalloc<float>((size_t)probes * rows_cap * 9, own);
    T.xs = dalloc<float>((size_t)rows_cap * 9, own);
    T.np = dalloc<int>(rows_cap, own);
    T.sys = dalloc<int>(rows_cap, own);
    T.rowoff = dalloc<int>((size_t)rows_cap + 1, own);
    T.ent = dalloc<int2>(ents_cap, own);
    T.blocks = dalloc<float>((size_t)blocks_cap * 81, own);
    T.sys_row = dalloc<int>((size_t)sys_cap + 1, own);
    T.uc = nullptr;
    H.ents_cap = ents_cap;
    H.blocks_cap = blocks_cap;
    H.sys_cap = sys_cap;
    H.sys_row.assign(1, 0);
  }
  void bufs() {
    const size_t R = T.rows, P = T.probes;
    B.sv = dalloc<float>(R * NN_O, own);
    B.ov = dalloc<float>(R * NN_O, own);
    B.hv = dalloc<float>(R * NN_H, own);
    B.u = dalloc<float>(P * R * 9, own);
    B.v = dalloc<float>(P * R * 9, own);
    B.d2 = dalloc<float>(R * NN_O, own);
    B.d1 = dalloc<float>(R * NN_H, own);
    B.grad = dalloc<float>(NN_WEIGHTS, own);
    B.pq = dalloc<double>(3 * (size_t)T.systems * P, own);
  }
};

}  // namespace

int32_t rpba_precond_loss_grad(const rpba_precond_set *set, const float *weights, float *loss, float *grad) {
  if (!set || !weights || !grad || set->rows <= 0 || set->systems <= 0 || set->probes <= 0) return RPBA_ERR_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return RPBA_ERR_NO_DEVICE;
  struct A {
    const rpba_precond_set *st;
    const float *w;
    float *loss, *grad;
  } a{set, weights, loss, grad};
  return guard([](void *p) {
    A *a = (A *)p;
    const rpba_precond_set &S = *a->st;
    TrainAlloc TA;
    TA.alloc(S.rows, std::max(S.nent, 1), std::max(S.nblocks, 1), S.systems, S.probes);
    TrainSet &T = TA.T;
    T.rows = S.rows;
    T.systems = S.systems;
    // a given set is laid out with rows_cap == rows
    auto up = [](void *d, const void *h, size_t n) { RPBA_CUDA_CHECK(cudaMemcpy(d, h, n, cudaMemcpyHostToDevice)); };
    up(T.f, S.features, sizeof(float) * S.rows * NN_F);
    up(T.sinv, S.sinv, sizeof(float) * S.rows * 81);
    up(T.b, S.b, sizeof(float) * (size_t)S.probes * S.rows * 9);
    up(T.xs, S.xs, sizeof(float) * S.rows * 9);
    up(T.np, S.np, sizeof(int) * S.rows);
    up(T.sys, S.sys, sizeof(int) * S.rows);
    up(T.rowoff, S.rowoff, sizeof(int) * (S.rows + 1));
    std::vector<int2> ent(std::max(S.nent, 1));
    for (int i = 0; i < S.nent; ++i) ent[i] = make_int2(S.ent_col[i], S.ent_blk[i]);
    up(T.ent, ent.data(), sizeof(int2) * S.nent);
    up(T.blocks, S.blocks, sizeof(float) * (size_t)S.nblocks * 81);
    up(T.sys_row, S.sys_row, sizeof(int) * (S.systems + 1));
    if (S.uc) {
      T.uc = dalloc<float>((size_t)S.probes * S.rows * 9, TA.own);
      up(T.uc, S.uc, sizeof(float) * (size_t)S.probes * S.rows * 9);
    }
    TA.bufs();
    float *dw = dalloc<float>(NN_WEIGHTS, TA.own);
    up(dw, a->w, sizeof(float) * NN_WEIGHTS);
    float l = 0.f;
    learned_loss_grad(T, dw, TA.B, &l, nullptr, 0);
    RPBA_CUDA_CHECK(cudaMemcpy(a->grad, TA.B.grad, sizeof(float) * NN_WEIGHTS, cudaMemcpyDeviceToHost));
    if (a->loss) *a->loss = l;
    return (int)RPBA_OK;
  }, &a);
}

namespace {

// Record the systems of the direct solver's own LM iterations on the scenes
// into TA (allocated here).
int record_systems(const rpba_block *sc, int ns, const rpba_options *opt, const rpba_train_options &t,
                   TrainAlloc &TA) {
  RPBA_CUDA_CHECK(cudaSetDevice(opt->device));
  const int probes = 1 + std::max(0, t.probes);
  const int rows_cap = t.max_samples > 0 ? t.max_samples : 1 << 18;
  TA.alloc(rows_cap, rows_cap * 96, rows_cap * 48, 4096, probes);
  TA.T.uc = dalloc<float>((size_t)probes * rows_cap * 9, TA.own);
  TA.H.vb = dalloc<double>(((size_t)rows_cap + 1) * 9, TA.own);
  TA.H.vz = dalloc<double>(((size_t)rows_cap + 1) * 9, TA.own);
  TA.H.rc = dalloc<int2>((size_t)rows_cap * 48, TA.own);
  for (int i = 0; i < ns; ++i) {
    rpba_options o = *opt;
    o.solver = RPBA_SOLVER_DIRECT;
    o.precision = RPBA_PREC_FP64;
    o.exteval = 0;
    rpba_handle *H = nullptr;
    int st = rpba_create(&H, &sc[i], &o);
    if (st != RPBA_OK) return st;
    H->rec_T = &TA.T;
    H->rec_H = &TA.H;
    H->rec_seed = t.seed * 1000003ull + (unsigned long long)i;
    rpba_report r{};
    st = rpba_solve(H, &r);
    rpba_destroy(H);
    if (st != RPBA_OK) return st;
  }
  if (TA.T.systems <= 0) return (int)RPBA_ERR_ARG;
  RPBA_CUDA_CHECK(cudaMemcpy(TA.T.sys_row, TA.H.sys_row.data(), sizeof(int) * (TA.T.systems + 1),
                             cudaMemcpyHostToDevice));
  return RPBA_OK;
}

}  // namespace

int32_t rpba_record_systems(const rpba_block *scenes, int32_t nscenes, const rpba_options *opt,
                            const rpba_train_options *topt, rpba_precond_buffers *out) {
  if (!scenes || nscenes <= 0 || !opt || !topt || !out) return RPBA_ERR_ARG;
  struct A {
    const rpba_block *sc;
    int ns;
    const rpba_options *o;
    const rpba_train_options *t;
    rpba_precond_buffers *out;
  } a{scenes, nscenes, opt, topt, out};
  return guard([](void *p) {
    A *a = (A *)p;
    TrainAlloc TA;
    const int st = record_systems(a->sc, a->ns, a->o, *a->t, TA);
    if (st != RPBA_OK) return st;
    const TrainSet &T = TA.T;
    rpba_precond_buffers &o = *a->out;
    const int rows = T.rows, nent = TA.H.ents, nb = TA.H.blocks, P = T.probes;
    o.rows = rows;
    o.systems = T.systems;
    o.probes = P;
    o.nent = nent;
    o.nblocks = nb;
    if (rows > o.rows_cap || nent > o.ents_cap || nb > o.blocks_cap || T.systems > o.systems_cap)
      return (int)RPBA_ERR_TOO_LARGE;
    auto down = [](void *h, const void *d, size_t n) {
      if (h && n) RPBA_CUDA_CHECK(cudaMemcpy(h, d, n, cudaMemcpyDeviceToHost));
    };
    down(o.features, T.f, sizeof(float) * rows * NN_F);
    down(o.sinv, T.sinv, sizeof(float) * rows * 81);
    for (int pr = 0; pr < P; ++pr) {
      down(o.b ? o.b + (size_t)pr * rows * 9 : nullptr, T.b + (size_t)pr * T.rows_cap * 9, sizeof(float) * rows * 9);
      down(o.uc ? o.uc + (size_t)pr * rows * 9 : nullptr, T.uc + (size_t)pr * T.rows_cap * 9,
           sizeof(float) * rows * 9);
    }
    down(o.xs, T.xs, sizeof(float) * rows * 9);
    down(o.np, T.np, sizeof(int) * rows);
    down(o.sys, T.sys, sizeof(int) * rows);
    down(o.rowoff, T.rowoff, sizeof(int) * (rows + 1));
    std::vector<int2> ent(std::max(nent, 1));
    down(ent.data(), T.ent, sizeof(int2) * nent);
    for (int i = 0; i < nent; ++i) {
      if (o.ent_col) o.ent_col[i] = ent[i].x;
      if (o.ent_blk) o.ent_blk[i] = ent[i].y;
    }
    down(o.blocks, T.blocks, sizeof(float) * (size_t)nb * 81);
    if (o.sys_row)
      for (int i = 0; i <= T.systems; ++i) o.sys_row[i] = TA.H.sys_row[i];
    return (int)RPBA_OK;
  }, &a);
}

int32_t rpba_train_preconditioner(const rpba_block *scenes, int32_t nscenes, const rpba_options *opt,
                                  const rpba_train_options *topt, float *weights, rpba_train_report *rep) {
  if (!scenes || nscenes <= 0 || !opt || !topt || !weights) return RPBA_ERR_ARG;
  if (rep) std::memset(rep, 0, sizeof *rep);
  struct A {
    const rpba_block *sc;
    int ns;
    const rpba_options *o;
    const rpba_train_options *t;
    float *w;
    rpba_train_report *rep;
  } a{scenes, nscenes, opt, topt, weights, rep};
  return guard([](void *p) {
    A *a = (A *)p;
    const rpba_train_options &t = *a->t;
    TrainAlloc TA;
    // 1. systems of the direct solver's own LM iterations
    const int st = record_systems(a->sc, a->ns, a->o, t, TA);
    if (st != RPBA_OK) return st;
    TrainSet &T = TA.T;
    TA.bufs();
    // 2. Adam on the one-step objective
    float *W = dalloc<float>(NN_WEIGHTS, TA.own), *m = dalloc<float>(NN_WEIGHTS, TA.own);
    float *v = dalloc<float>(NN_WEIGHTS, TA.own);
    std::vector<float> w0(NN_WEIGHTS, 0.f);
    {
      // W1 ~ U(-1/sqrt(F), 1/sqrt(F)), everything else 0: the untrained
      // network gives s = 1, i.e. plain block-Jacobi
      unsigned long long z = t.seed ^ 0x2545f4914f6cdd1dull;
      for (int i = 0; i < NN_H * NN_F; ++i) {
        z ^= z << 13;
        z ^= z >> 7;
        z ^= z << 17;
        w0[i] = (float)(((double)(z >> 11) / 9007199254740992.0 * 2. - 1.) / std::sqrt((double)NN_F));
      }
    }
    RPBA_CUDA_CHECK(cudaMemcpy(W, w0.data(), sizeof(float) * NN_WEIGHTS, cudaMemcpyHostToDevice));
    RPBA_CUDA_CHECK(cudaMemset(m, 0, sizeof(float) * NN_WEIGHTS));
    RPBA_CUDA_CHECK(cudaMemset(v, 0, sizeof(float) * NN_WEIGHTS));
    // Adam with a cosine learning-rate decay; the weights with the lowest
    // training loss seen are returned (the untrained network, plain
    // block-Jacobi, is the first candidate)
    float *Wbest = dalloc<float>(NN_WEIGHTS, TA.own);
    float loss0 = 0.f, err0 = 0.f, loss1 = 0.f, err1 = 0.f;
    learned_loss_grad(T, W, TA.B, &loss0, &err0, 0);
    RPBA_CUDA_CHECK(cudaMemcpy(Wbest, W, sizeof(float) * NN_WEIGHTS, cudaMemcpyDeviceToDevice));
    float best = loss0;
    const int steps = t.steps > 0 ? t.steps : 300;
    const float lr = t.lr > 0.f ? t.lr : 3e-3f;
    for (int st = 0; st < steps; ++st) {
      float l = 0.f;
      learned_loss_grad(T, W, TA.B, &l, nullptr, 0);
      if (st > 0 && l < best) {
        best = l;
        RPBA_CUDA_CHECK(cudaMemcpy(Wbest, W, sizeof(float) * NN_WEIGHTS, cudaMemcpyDeviceToDevice));
      }
      const float lr_t = lr * 0.5f * (1.f + std::cos(3.14159265f * (float)st / (float)steps));
      learned_adam(W, m, v, TA.B.grad, lr_t, st + 1, 0);
    }
    {
      float l = 0.f;
      learned_loss_grad(T, W, TA.B, &l, nullptr, 0);
      if (l < best) RPBA_CUDA_CHECK(cudaMemcpy(Wbest, W, sizeof(float) * NN_WEIGHTS, cudaMemcpyDeviceToDevice));
    }
    W = Wbest;
    learned_loss_grad(T, W, TA.B, &loss1, &err1, 0);
    std::vector<float> wout(NN_WEIGHTS);
    RPBA_CUDA_CHECK(cudaMemcpy(wout.data(), W, sizeof(float) * NN_WEIGHTS, cudaMemcpyDeviceToHost));
    for (int i = 0; i < NN_WEIGHTS; ++i) a->w[i] = wout[i];
    if (a->rep) {
      a->rep->samples = T.rows;
      a->rep->systems = T.systems;
      a->rep->steps = steps;
      a->rep->loss_initial = loss0;
      a->rep->loss_final = loss1;
      a->rep->err_initial = err0;
      a->rep->err_final = err1;
    }
    return (int)RPBA_OK;
  }, &a);
}

int32_t rpba_kernel_stats(rpba_handle *H, char *json, size_t cap) {
  if (!H || !json || cap == 0) return RPBA_ERR_ARG;
  std::string o = "{";
  bool first = true;
  for (auto &st : H->prof.stats) {
    char b[200];
    std::snprintf(b, sizeof b, "%s\"%s\": {\"launches\": %lld, \"ms\": %.6f, \"bytes\": %.0f}", first ? "" : ", ",
                  st.name.c_str(), st.launches, st.ms, st.bytes);
    o += b;
    first = false;
  }
  // the reduced camera system's size, for per-iteration byte counts
  char b[160];
  std::snprintf(b, sizeof b, "%s\"_rcs\": {\"rows\": %d, \"offdiag_blocks\": %d, \"fp32\": %d}", first ? "" : ", ",
                H->nimg - H->begini, H->L.nboff, H->L.blocks32 ? 1 : 0);
  o += b;
  o += "}";
  const size_t n = std::min(cap - 1, o.size());
  std::memcpy(json, o.data(), n);
  json[n] = 0;
  return RPBA_OK;
}

int32_t rpba_spd_inverse(const double *A, int32_t n, double *Ainv, int32_t device) {
  if (!A || !Ainv || n <= 0) return RPBA_ERR_ARG;
  if (n > 16384) return RPBA_ERR_TOO_LARGE;
  struct Args {
    const double *A;
    int n;
    double *Ainv;
    int device;
  } args{A, n, Ainv, device};
  return guard(
      [](void *p) -> int {
        const Args &a = *(const Args *)p;
        RPBA_CUDA_CHECK(cudaSetDevice(a.device));
        const size_t bytes = sizeof(double) * (size_t)a.n * a.n;
        std::vector<void *> owned;  // freed on every return
        struct Free {
          std::vector<void *> &v;
          ~Free() {
            for (void *q : v) cudaFree(q);
          }
        } fr{owned};
        auto dal = [&](size_t b) {
          void *q = nullptr;
          RPBA_CUDA_CHECK(cudaMalloc(&q, std::max<size_t>(b, 16)));
          owned.push_back(q);
          return q;
        };
        double *dA = (double *)dal(bytes), *dI = (double *)dal(bytes), *dd = (double *)dal(sizeof(double) * a.n);
        void *work = dal(spd_inverse_bytes(a.n));
        unsigned *bar = (unsigned *)dal(2 * sizeof(unsigned));
        int *err = (int *)dal(sizeof(int));
        const std::vector<double> ones(a.n, 1.);
        RPBA_CUDA_CHECK(cudaMemcpy(dA, a.A, bytes, cudaMemcpyHostToDevice));
        RPBA_CUDA_CHECK(cudaMemcpy(dd, ones.data(), sizeof(double) * a.n, cudaMemcpyHostToDevice));
        RPBA_CUDA_CHECK(cudaMemset(err, 0, sizeof(int)));
        spd_inverse_scaled(dA, dd, 0., a.n, dI, work, bar, err, 0);
        int e = 0;
        RPBA_CUDA_CHECK(cudaMemcpy(a.Ainv, dI, bytes, cudaMemcpyDeviceToHost));
        RPBA_CUDA_CHECK(cudaMemcpy(&e, err, sizeof(int), cudaMemcpyDeviceToHost));
        if (e & 2) return RPBA_ERR_DEVICE_TIMEOUT;
        return (e & 4) ? RPBA_ERR_SOLVER : RPBA_OK;
      },
      &args);
}

int32_t rpba_debug_barrier_timeout(rpba_handle *H, int32_t extra_ctas, int64_t timeout_ns) {
  if (!H || extra_ctas < 0 || extra_ctas > 1 || timeout_ns < 0 || timeout_ns > 2000000000ll ||
      (extra_ctas > 0 && timeout_ns < 1000000))
    return RPBA_ERR_ARG;
  H->L.bar_extra = (unsigned)extra_ctas;
  H->L.bar_timeout_ns = (unsigned long long)timeout_ns;
  return RPBA_OK;
}

void rpba_destroy(rpba_handle *H) { delete H; }

int32_t rpba_partition_count(int32_t n_images, int32_t threads, int32_t exteval) {
  int mt = threads;
  if (mt < 1) mt = std::max(1, (int)std::thread::hardware_concurrency());
  // boost::math::iround: nearest, halves away from zero
  const int minnrthreads = (int)std::lround((float)n_images / 70.f);
  const int nr = std::min(mt, minnrthreads);
  return (!exteval && nr > 1 && n_images > 5) ? nr : 1;
}

namespace {
// CalcPLSA's partitioned branch (rpbacore.cpp:100-510): the reference's
// console lines (rpbacore.cpp:110, 140, 157) at the head of the log, the
// partition, and the loop.
int32_t calc_plsa_partitioned(rpba_block *blk, const rpba_options *opt, int nrthreads, char *log, size_t cap,
                              rpba_report *rep) {
  std::string head = "#threads: " + std::to_string(nrthreads) + " " +
                     std::to_string((int)std::lround((float)blk->n_images / 70.f)) + "\n";
  std::vector<int32_t> part(blk->n_images);
  const auto tp = std::chrono::steady_clock::now();
  int32_t st = rpba_partition_images(blk, nrthreads, part.data());
  char line[160];
  std::snprintf(line, sizeof line, "\n\nPartitioning runtime: %gs\n\n",
                (float)std::chrono::duration<double>(std::chrono::steady_clock::now() - tp).count());
  head += line;
  if (st == RPBA_OK) {
    std::vector<int> cnt(nrthreads, 0);
    for (int32_t q : part) ++cnt[q];
    for (int it = 0, a = 0; it < nrthreads; a += cnt[it], ++it) {
      std::snprintf(line, sizeof line, "Thread: %d #images %d indices %d %d\n", it, cnt[it], a, a + cnt[it]);
      head += line;
    }
  }
  size_t used = 0;
  if (log && cap) {
    used = std::min(cap - 1, head.size());
    std::memcpy(log, head.data(), used);
    log[used] = 0;
  }
  if (st == RPBA_OK) {
    double stats[2] = {0., 0.};
    st = rpba_calc_plsa_parallel(blk, opt, nrthreads, part.data(), log ? log + used : nullptr,
                                 log ? cap - used : 0, stats);
  }
  if (rep) rep->status = st;
  return st;
}
}  // namespace

int32_t rpba_calc_plsa(rpba_block *blk, const rpba_options *opt, char *log, size_t cap, rpba_report *rep) {
  if (!blk || !opt) return RPBA_ERR_ARG;
  if (rep) std::memset(rep, 0, sizeof *rep);
  // the reference's branch rule (rpbacore.cpp:79-92); the partitioned branch
  // runs the drop-in FP64 form, the other forms always solve the whole block
  const int nrthreads = rpba_partition_count(blk->n_images, opt->threads, opt->exteval);
  if (nrthreads > 1 && opt->precision == RPBA_PREC_FP64 &&
      (opt->solver == RPBA_SOLVER_PCG || opt->solver == RPBA_SOLVER_DIRECT))
    return calc_plsa_partitioned(blk, opt, nrthreads, log, cap, rep);
  rpba_handle *H = nullptr;
  int st = rpba_create(&H, blk, opt);
  if (st != RPBA_OK) return st;
  if (opt->exteval) {
    st = rpba_exteval(H, nullptr, rep);
  } else {
    st = rpba_solve(H, rep);
    if (st == RPBA_OK || st == RPBA_ERR_NO_OBS_IMAGE || st == RPBA_ERR_LOW_REDUNDANCY || st == RPBA_ERR_NAN_STEP) {
      const int st2 = rpba_get_state(H, blk);
      if (st == RPBA_OK) st = st2;
    }
  }
  if (log && cap) rpba_get_log(H, log, cap);
  rpba_destroy(H);
  return st;
}

int32_t rpba_lsa_gcp_step(rpba_block *blk, const rpba_options *opt, const int32_t *gcpinfo, const float *W3,
                          int32_t n_w3, const double *gcpdata, int32_t n_gcp, int32_t ncam_total,
                          const double *pmat_d, double *pmat_d_out, uint8_t *point_used, rpba_report *rep,
                          char *log, size_t cap) {
  if (!blk || !opt || !gcpinfo || n_w3 < 0 || n_gcp < 0 || (n_w3 > 0 && !W3) || (n_gcp > 0 && !gcpdata) ||
      blk->n_images < 1 || blk->n_points < 0 || ncam_total < blk->n_images)
    return RPBA_ERR_ARG;
  if (opt->exteval || opt->precision != RPBA_PREC_FP64 ||
      (opt->solver != RPBA_SOLVER_PCG && opt->solver != RPBA_SOLVER_DIRECT))
    return RPBA_ERR_UNSUPPORTED;
  if (rep) std::memset(rep, 0, sizeof *rep);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= opt->device) return RPBA_ERR_NO_DEVICE;
  rpba_handle *H = new rpba_handle();
  // the partition steps of one outer iteration run concurrently (the
  // reference's OpenMP loop, rpbacore.cpp:219-235); their cooperative
  // kernels take one process-wide lock, as a batch's do
  H->coop = &g_gcp_coop;
  const GcpSetup gs{gcpinfo, W3, n_w3, gcpdata, n_gcp, ncam_total, pmat_d};
  struct A {
    rpba_handle *H;
    const rpba_block *b;
    const rpba_options *o;
    const GcpSetup *g;
  } a{H, blk, opt, &gs};
  int st = guard([](void *p) {
    A *a = (A *)p;
    return create_impl(a->H, a->b, a->o, a->g);
  }, &a);
  if (st != RPBA_OK) {
    delete H;
    return st;
  }
  st = guard([](void *p) {
    rpba_handle *H = (rpba_handle *)p;
    RPBA_CUDA_CHECK(cudaSetDevice(H->dev));
    AsyncScope scope(H->s, H->owned, H->owned_async);
    H->log.clear();
    std::memset(&H->rep, 0, sizeof H->rep);
    H->rep.points_used = H->npts0;
    H->reset();
    return H->adjust_gcp_step();
  }, H);
  if (st == RPBA_OK || st == RPBA_ERR_NO_OBS_IMAGE || st == RPBA_ERR_LOW_REDUNDANCY || st == RPBA_ERR_NAN_STEP) {
    int st2 = rpba_get_state(H, blk);
    if (st2 == RPBA_OK && (pmat_d_out || point_used)) {
      // OutputLSAP (rbacore.cpp:620-639): the cameras in double precision
      // and the points PointXXvIn took (the others' lists are cleared)
      struct B {
        rpba_handle *H;
        double *P;
        uint8_t *used;
      } bb{H, pmat_d_out, point_used};
      st2 = guard([](void *p) {
        B *b = (B *)p;
        rpba_handle *H = b->H;
        RPBA_CUDA_CHECK(cudaSetDevice(H->dev));
        if (b->P)
          RPBA_CUDA_CHECK(cudaMemcpyAsync(b->P, H->L.Pacc, sizeof(double) * 12 * H->nimg, cudaMemcpyDeviceToHost, H->s));
        std::vector<int> ids(H->L.npts);
        if (b->used && H->L.npts)
          RPBA_CUDA_CHECK(
              cudaMemcpyAsync(ids.data(), H->L.pt_id, sizeof(int) * H->L.npts, cudaMemcpyDeviceToHost, H->s));
        RPBA_CUDA_CHECK(cudaStreamSynchronize(H->s));
        if (b->used) {
          std::memset(b->used, 0, (size_t)H->XXnr);
          for (int q : ids) b->used[q] = 1;
        }
        return (int)RPBA_OK;
      }, &bb);
    }
    if (st == RPBA_OK) st = st2;
  }
  if (rep) *rep = H->rep;
  if (log && cap) rpba_get_log(H, log, cap);
  delete H;
  return st;
}

int32_t rpba_solve_batch(rpba_block *blocks, int32_t n, const rpba_options *opt, int32_t workers,
                         rpba_report *reports, int32_t *status, rpba_batch_report *br) {
  if (!blocks || n <= 0 || !opt || !status || opt->exteval) return RPBA_ERR_ARG;
  if (br) std::memset(br, 0, sizeof *br);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= opt->device) return RPBA_ERR_NO_DEVICE;
  // largest scenes first: the tail of the batch is made of small scenes
  std::vector<int> order(n);
  for (int i = 0; i < n; ++i) order[i] = i;
  auto obs = [&](int i) { return blocks[i].pt_obs_off ? (long long)blocks[i].pt_obs_off[blocks[i].n_points] : 0ll; };
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return obs(a) > obs(b); });
  std::mutex coop;
  std::vector<rpba_report> reps(n);
  // solve the scenes of `ord` with `w` concurrent workers, each driving its
  // own handle (and stream; handle memory comes from the stream-ordered
  // pool, so creating and destroying handles does not stall the others);
  // returns the wall time
  auto run = [&](const std::vector<int> &ord, int w, bool keep) {
    std::atomic<int> next{0};
    auto body = [&]() {
      cudaSetDevice(opt->device);
      for (;;) {
        const int q = next.fetch_add(1);
        if (q >= (int)ord.size()) break;
        const int i = ord[q];
        rpba_report r{};
        rpba_handle *H = nullptr;
        int st = rpba_create(&H, &blocks[i], opt);
        if (st == RPBA_OK) {
          H->coop = &coop;
          st = rpba_solve(H, &r);
          if (keep && (st == RPBA_OK || st == RPBA_ERR_NO_OBS_IMAGE || st == RPBA_ERR_LOW_REDUNDANCY ||
                       st == RPBA_ERR_NAN_STEP)) {
            const int st2 = rpba_get_state(H, &blocks[i]);
            if (st == RPBA_OK) st = st2;
          }
          rpba_destroy(H);
        }
        if (keep) {
          status[i] = st;
          reps[i] = r;
        }
      }
    };
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<std::thread> th;
    for (int k = 1; k < w; ++k) th.emplace_back(body);
    body();
    for (auto &t : th) t.join();
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  };
  int w = workers;
  double tune = 0.;
  if (w <= 0) {
    // autotune the number of concurrent scenes on a sample spread over the
    // size order (the solutions are discarded)
    std::vector<int> sample;
    const int ns = std::min(n, 24);
    for (int j = 0; j < ns; ++j) sample.push_back(order[(long long)j * n / ns]);
    const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
    double best = 1e300;
    w = 1;
    for (int cand : {1, 2, 4, 8, 16, 32}) {
      if (cand > ns || cand > hw) break;
      const double t = run(sample, cand, false);
      tune += t;
      if (t < best * 0.97) {
        best = t;
        w = cand;
      }
    }
  }
  const double secs = run(order, w, true);
  int failed = 0;
  for (int i = 0; i < n; ++i) {
    if (reports) reports[i] = reps[i];
    if (status[i] != RPBA_OK) ++failed;
  }
  if (br) {
    br->seconds = secs;
    br->scenes_per_second = n / secs;
    br->tune_seconds = tune;
    br->workers = w;
    br->failed = failed;
  }
  return failed ? RPBA_ERR_SOLVER : RPBA_OK;
}

}  // extern "C"
