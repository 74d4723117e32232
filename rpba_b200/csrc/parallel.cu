// parallel.cu -- the parallel RPBA (the partitioned branch of CalcPLSA,
// rpbacore.cpp:100-510) on the GPU: host control, device work.
//
// The images are cut into nthreads partitions (part[image]; the reference
// cuts the covisibility graph with METIS, rpba_partition_images replaces
// it).  Outer iteration `iter`:
//   iter > 1: every partition takes one GCP-mode LSA step on its images and
//     the observations in them (rpba_lsa_gcp_step): the points it shares
//     with other partitions are held by 3-D priors with the weight blocks of
//     the last merge; the additional parameters stay fixed at iter 2; its
//     cameras replace the scene's;
//   the merge: every point is refined against the new cameras by
//   CalcLSAXMulti on the GPU (one launch over all points): first a robust
//   pass that gives the per-image thresholds when the robust stage starts,
//   then the main pass (robust deletion, weight-only at iter 1, the
//   per-partition weight blocks).  The reference sums its per-thread point
//   chunks and then the chunks; the per-point contributions are summed here
//   the same way, so sigma0 and every decision follow it;
//   sigma0 = sum / (redundancy - unknowns); the best state is kept, and the
//   points seen by more than one partition become the next GCPs at their
//   refined positions;
// until iflag runs out (the sig0frac rule) or 50 iterations.  The partition
// steps of an outer iteration run concurrently on host threads, each on its
// own handle and stream (their cooperative kernels one at a time: the
// persistent PCG and the exact sums need every SM); each step's result does
// not depend on the others, so neither does the loop's.
//
// Over several ranks (one process per GPU, rpba_calc_plsa_parallel_ranks)
// every rank keeps the whole loop, runs the steps of the partitions it owns
// and all-gathers the steps' results with the others after every round of
// steps, through the caller's transport; the merge and the bookkeeping are
// repeated on every rank, so every rank takes the same decisions.
//
// The loop is host code over two steps, the partition step and the merge
// pass; rpba_calc_plsa_parallel(_ranks) binds them to the GPU
// (rpba_lsa_gcp_step and the CalcLSAXMulti kernel), the _hosted forms take
// them from the caller, so that the loop itself can be checked without a
// GPU.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <exception>
#include <mutex>
#include <string>
#include <system_error>
#include <thread>
#include <vector>

#include "../../include/rpba_b200.h"
#include "internal.h"

namespace {

// observation lists of points (the reference's pointXXv: a list of (image,
// slot) per point) in CSR form: point p's observations are entries
// off[p] .. off[p + 1] - 1 of img and slot
struct Tracks {
  std::vector<int32_t> off, img, slot;
  int len(int p) const { return off[p + 1] - off[p]; }
  void start(int npts) {
    off.assign(1, 0);
    off.reserve(npts + 1);
    img.clear();
    slot.clear();
  }
  void add(int32_t i, int32_t s) {
    img.push_back(i);
    slot.push_back(s);
  }
  void close_point() { off.push_back((int32_t)img.size()); }
};
// a partition's points (the reference's pointXXvv[it] and pindv[it]):
// global point index, the observations in the partition's images (global
// image indices), and whether the partition's last step took the point
struct PartTracks {
  std::vector<int> pind;
  Tracks tr;
  std::vector<uint8_t> used;
};
struct PCam {
  float K[9], d[2];
};

std::string fmt_g(double v) {
  char b[64];
  std::snprintf(b, sizeof b, "%g", v);
  return b;
}

// a block over given cameras and point lists (views into its own vectors)
struct TmpBlock {
  rpba_block b{};
  std::vector<int32_t> off, img, slot, ioff;
  std::vector<float> XX, pmat, K, dist, xg, wx, wy, wxy;
};

// host threads for the partition steps (the reference runs one OpenMP
// thread per partition, rpbacore.cpp:219-235; here at most one per core)
int host_workers() { return (int)std::max(1u, std::thread::hardware_concurrency()); }

// Host-side passes over points, observations or partitions run on host
// threads in W contiguous ranges; where the output is a list in item order,
// a first pass counts per range and a second writes at the prefix sums, so
// the result does not depend on W.
//   nranges: at most `workers` ranges of at least `grain` items
//   parallel_ranges: f(k, lo, hi) for range k = [n k / W, n (k + 1) / W)
int nranges(long long n, int workers, int grain) {
  return (int)std::max(1ll, std::min((long long)workers, n / grain));
}
//   (a range whose thread cannot be created runs on the calling thread; an
//   exception in a range is rethrown on the calling thread after the join)
template <class F>
void parallel_ranges(int n, int W, F &&f) {
  std::exception_ptr err;
  std::mutex em;
  auto body = [&](int k) {
    try {
      f(k, (int)((long long)n * k / W), (int)((long long)n * (k + 1) / W));
    } catch (...) {
      std::lock_guard<std::mutex> lock(em);
      if (!err) err = std::current_exception();
    }
  };
  std::vector<std::thread> th;
  int k = 1;
  try {
    for (; k < W; ++k) th.emplace_back(body, k);
  } catch (const std::system_error &) {
  }
  for (int j = k; j < W; ++j) body(j);
  body(0);
  for (auto &t : th) t.join();
  if (err) std::rethrow_exception(err);
}

// the merge pass on the GPU
int32_t gpu_merge(const rpba_block *b, const double *Pd, const float *sig0w, int32_t robustmode, int32_t weight_only,
                  const int32_t *part, int32_t nparts, int32_t device, double *XX_out, uint8_t *keep, float *sig0v,
                  uint8_t *conv, float *w3d, double *s0_pt, int32_t *red_pt) {
  rpba_tri_options to{};
  to.robustmode = robustmode;
  to.weight_only = weight_only;
  to.device = device;
  double a = 0.;
  int64_t r = 0;
  return rpba::triangulate_impl(b, Pd, sig0w, &to, part, nparts, XX_out, keep, sig0v, conv, &a, &r, w3d, s0_pt,
                                red_pt);
}

// Ranks of a multi-rank loop (one process per GPU): every rank holds the
// whole scene and keeps the whole loop state; it runs the partition steps
// of the partitions it owns, and after each round of steps the ranks
// exchange the steps' results through `ag` (an all-gather supplied by the
// caller), so that every rank continues from the same state.  ag null: one
// rank, no exchange.
struct Ranks {
  int rank = 0, world = 1;
  rpba_allgather_fn ag = nullptr;
  void *ctx = nullptr;
};

// byte records of the exchange
void put(std::vector<uint8_t> &b, const void *p, size_t n) {
  const uint8_t *c = (const uint8_t *)p;
  b.insert(b.end(), c, c + n);
}
template <class V>
void put_v(std::vector<uint8_t> &b, const V &v) {
  put(b, &v, sizeof v);
}
struct Reader {
  const uint8_t *p, *end;
  bool ok = true;
  void get(void *d, size_t n) {
    if ((size_t)(end - p) < n) {
      ok = false;
      return;
    }
    std::memcpy(d, p, n);
    p += n;
  }
  template <class V>
  V get_v() {
    V v{};
    get(&v, sizeof v);
    return v;
  }
};

int32_t plsa_parallel(rpba_block *blk, const rpba_options *opt, int32_t nthreads, const int32_t *part, char *log,
                      size_t cap, double *stats, rpba_gcp_step_fn step_fn, rpba_merge_fn merge_fn, int workers,
                      const Ranks &rk = Ranks()) {
  if (!blk || !opt || !part || nthreads < 2 || blk->n_images < 1 || blk->n_points < 0) return RPBA_ERR_ARG;
  if (rk.world < 1 || rk.rank < 0 || rk.rank >= rk.world || (rk.world > 1 && !rk.ag)) return RPBA_ERR_ARG;
  const int nrimages = blk->n_images, pxs = blk->n_points, T = nthreads;
  for (int i = 0; i < nrimages; ++i)
    if (part[i] < 0 || part[i] >= T) return RPBA_ERR_ARG;
  std::string os;
  const bool robustflag = opt->robust != 0;
  const int nraddp = (opt->k2 ? 1 : 0) + (opt->k4 ? 1 : 0) + (opt->f ? 1 : 0);
  // partitions: images in index order
  std::vector<std::vector<int>> imgindv(T);
  std::vector<int32_t> imgindbv(nrimages);
  for (int i = 0; i < nrimages; ++i) {
    imgindv[part[i]].push_back(i);
    imgindbv[i] = part[i];
  }
  for (int it = 0; it < T; ++it)
    if (imgindv[it].empty()) return RPBA_ERR_ARG;
  // the owner rank of every partition: largest (observation slots) first to
  // the least-loaded rank, ties to the lower index and rank -- the same on
  // every rank
  std::vector<int> owner(T, 0);
  {
    std::vector<long long> cost(T, 0), load(rk.world, 0);
    for (int i = 0; i < nrimages; ++i) cost[part[i]] += blk->img_obs_off[i + 1] - blk->img_obs_off[i];
    std::vector<int> order(T);
    for (int it = 0; it < T; ++it) order[it] = it;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] > cost[b]; });
    for (int it : order) {
      const int r = (int)(std::min_element(load.begin(), load.end()) - load.begin());
      owner[it] = r;
      load[r] += cost[it];
    }
  }
  for (int p = 0; p < pxs; ++p)
    for (int t = blk->pt_obs_off[p]; t < blk->pt_obs_off[p + 1]; ++t) {
      const int im = blk->pt_obs_image[t];
      if (im < 0 || im >= nrimages || blk->pt_obs_slot[t] < 0 ||
          blk->pt_obs_slot[t] >= blk->img_obs_off[im + 1] - blk->img_obs_off[im])
        return RPBA_ERR_ARG;
    }
  // state: points and cameras in double precision, cameras' intrinsics
  std::vector<double> XXd(3 * (size_t)pxs), XXdold, PMd(12 * (size_t)nrimages), PMdold;
  for (size_t i = 0; i < XXd.size(); ++i) XXd[i] = (double)blk->XX[i];
  for (size_t i = 0; i < PMd.size(); ++i) PMd[i] = (double)blk->pmat[i];
  PMdold = PMd;
  XXdold = XXd;
  std::vector<PCam> cameras(nrimages), cameraps, camerasnew(nrimages), camerasold(nrimages);
  for (int i = 0; i < nrimages; ++i) {
    for (int c = 0; c < 9; ++c) cameras[i].K[c] = blk->K[9 * i + c];
    cameras[i].d[0] = blk->distpara[2 * i];
    cameras[i].d[1] = blk->distpara[2 * i + 1];
  }
  cameraps = cameras;
  Tracks pointXXv, pointXXvold;
  pointXXv.start(pxs);
  for (int p = 0; p < pxs; ++p) {
    for (int t = blk->pt_obs_off[p]; t < blk->pt_obs_off[p + 1]; ++t)
      pointXXv.add(blk->pt_obs_image[t], blk->pt_obs_slot[t]);
    pointXXv.close_point();
  }
  pointXXvold = pointXXv;
  // the reference's pitflagsv: the partitions each point's observations
  // fall in at the start of the outer iteration, distinct, in order of
  // first appearance (CSR: point p's are pitp[pitp_off[p] ..
  // pitp_off[p + 1]))
  std::vector<int32_t> pitp_off(pxs + 1, 0), pitp;
  std::vector<int> gcpinfo(pxs, -1);
  std::vector<std::vector<PCam>> camerasoit(T, cameras);
  std::vector<std::vector<double>> PMdd(T, PMd);
  std::vector<PartTracks> pointXXvv(T);
  std::vector<std::vector<int32_t>> gcpinfov(T);
  std::vector<std::vector<float>> W3ijiv(T);
  std::vector<double> gcpdatav;
  std::vector<float> sig0wv(nrimages, 0.f);
  const int nrparimages = (nrimages - 2) * 6 + 5 + nrimages * nraddp;
  const int nrppt = pxs / T;
  std::vector<int> beginv(T), endv(T);
  for (int c = 0; c < T; ++c) {
    beginv[c] = nrppt * c;
    endv[c] = c == T - 1 ? pxs : nrppt * (c + 1);
  }
  double sig0opt = 1.e20, sig0g = 0.;
  int iflag = robustflag ? 2 : 1, iter = 1;
  float sig0frac = 1.01f;
  // the weight blocks of the last main pass, per point and partition (only
  // points that converged in it keep two or more observations, and only
  // those become GCPs)
  std::vector<float> w3d((size_t)pxs * T * 6, 0.f);

  // one CalcLSAXMulti pass over all points with the current cameras; applies
  // the refined points and the deletions; returns (sum, redundancy) with the
  // per-point contributions summed chunk by chunk
  int status = RPBA_OK;
  std::vector<double> XXo(3 * (size_t)pxs), s0pt(pxs);
  std::vector<uint8_t> keep, conv(std::max(pxs, 1));
  std::vector<float> sv;
  std::vector<int32_t> redpt(pxs);
  auto sweep = [&](int robustmode, bool weightonly, bool wxy, std::vector<std::vector<float>> *sig0vv,
                   double *sum, long long *redund) {
    TmpBlock tb;
    tb.b = *blk;
    tb.XX.resize(3 * (size_t)pxs);
    for (size_t i = 0; i < tb.XX.size(); ++i) tb.XX[i] = (float)XXd[i];
    tb.K.resize(9 * (size_t)nrimages);
    tb.dist.resize(2 * (size_t)nrimages);
    for (int i = 0; i < nrimages; ++i) {
      std::memcpy(&tb.K[9 * (size_t)i], cameraps[i].K, sizeof(float) * 9);
      tb.dist[2 * i] = cameraps[i].d[0];
      tb.dist[2 * i + 1] = cameraps[i].d[1];
    }
    tb.b.pt_obs_off = pointXXv.off.data();
    tb.b.pt_obs_image = pointXXv.img.data();
    tb.b.pt_obs_slot = pointXXv.slot.data();
    tb.b.XX = tb.XX.data();
    tb.b.K = tb.K.data();
    tb.b.distpara = tb.dist.data();
    const size_t nt = pointXXv.img.size();
    // the merge's outputs (it writes every point's and every track entry's;
    // the buffers are kept from sweep to sweep: the track only shrinks)
    if (keep.size() < std::max<size_t>(nt, 1)) {
      keep.resize(std::max<size_t>(nt, 1));
      sv.resize(std::max<size_t>(nt, 1));
    }
    status = merge_fn(&tb.b, PMd.data(), sig0wv.data(), robustmode, weightonly ? 1 : 0, wxy ? imgindbv.data() : nullptr,
                      wxy ? T : 1, opt->device, XXo.data(), keep.data(), sv.data(), conv.data(),
                      wxy ? w3d.data() : nullptr, s0pt.data(), redpt.data());
    if (status != RPBA_OK) return false;
    if (sig0vv)  // every image's statistics in track order (image ranges on host threads)
      parallel_ranges(nrimages, nranges(nrimages, workers, 64), [&](int, int i0, int i1) {
        for (size_t t = 0; t < nt; ++t) {
          const int i = pointXXv.img[t];
          if (i >= i0 && i < i1) (*sig0vv)[i].push_back(sv[t]);
        }
      });
    // the refined points, and every list without the deleted observations
    // (point ranges on host threads: the kept observations counted, then
    // written at the ranges' prefix sums)
    const int W = nranges(pxs, workers, 4096);
    std::vector<int32_t> kc(W + 1, 0);
    parallel_ranges(pxs, W, [&](int k, int p0, int p1) {
      int32_t c = 0;
      for (int p = p0; p < p1; ++p)
        if (pointXXv.len(p) > 0)
          for (int t = pointXXv.off[p]; t < pointXXv.off[p + 1]; ++t) c += keep[t] ? 1 : 0;
      kc[k + 1] = c;
    });
    for (int k = 0; k < W; ++k) kc[k + 1] += kc[k];
    Tracks kept;
    kept.off.resize(pxs + 1);
    kept.img.resize(kc[W]);
    kept.slot.resize(kc[W]);
    parallel_ranges(pxs, W, [&](int k, int p0, int p1) {
      int32_t o = kc[k];
      for (int p = p0; p < p1; ++p) {
        kept.off[p] = o;
        if (pointXXv.len(p) == 0) continue;
        for (int q = 0; q < 3; ++q) XXd[3 * (size_t)p + q] = XXo[3 * (size_t)p + q];
        for (int t = pointXXv.off[p]; t < pointXXv.off[p + 1]; ++t)
          if (keep[t]) {
            kept.img[o] = pointXXv.img[t];
            kept.slot[o++] = pointXXv.slot[t];
          }
      }
    });
    kept.off[pxs] = kc[W];
    pointXXv = std::move(kept);
    double a = 0.;
    long long r = 0;
    for (int c = 0; c < T; ++c) {
      double ac = 0.;
      long long rc = 0;
      for (int p = beginv[c]; p < endv[c]; ++p) {
        ac += s0pt[p];
        rc += redpt[p];
      }
      a += ac;
      r += rc;
    }
    *sum = a;
    *redund = r;
    return true;
  };

  while (iflag > 0 && iter < 51) {
    bool robustflagit = false;
    if (iter > 1) {
      rpba_options ol = *opt;
      ol.robust = 0;
      if (iter < 3) ol.k2 = ol.k4 = ol.f = 0;
      // the step of partition `it`: its log goes to plog, its results to
      // the partition's own state (PMdd[it], camerasoit[it],
      // pointXXvv[it].used)
      auto part_step = [&](int it, std::string &plog) -> int {
        const std::vector<int> &imgs = imgindv[it];
        const int m = (int)imgs.size();
        TmpBlock tb;
        std::vector<int> loc(nrimages, -1);
        std::vector<double> Pd(12 * (size_t)m), Pout(12 * (size_t)m);
        tb.pmat.resize(12 * (size_t)m);
        tb.K.resize(9 * (size_t)m);
        tb.dist.resize(2 * (size_t)m);
        tb.ioff.assign(m + 1, 0);
        for (int li = 0; li < m; ++li) {
          const int g = imgs[li];
          loc[g] = li;
          for (int c = 0; c < 12; ++c) {
            Pd[12 * li + c] = PMdd[it][12 * (size_t)g + c];
            tb.pmat[12 * li + c] = (float)Pd[12 * li + c];
          }
          std::memcpy(&tb.K[9 * (size_t)li], camerasoit[it][g].K, sizeof(float) * 9);
          tb.dist[2 * li] = camerasoit[it][g].d[0];
          tb.dist[2 * li + 1] = camerasoit[it][g].d[1];
          // the image's observation slots are contiguous in the block
          const int s0 = blk->img_obs_off[g], s1 = blk->img_obs_off[g + 1];
          tb.xg.insert(tb.xg.end(), blk->xg + 2 * (size_t)s0, blk->xg + 2 * (size_t)s1);
          tb.wx.insert(tb.wx.end(), blk->wx + s0, blk->wx + s1);
          tb.wy.insert(tb.wy.end(), blk->wy + s0, blk->wy + s1);
          tb.wxy.insert(tb.wxy.end(), blk->wxy + s0, blk->wxy + s1);
          tb.ioff[li + 1] = (int32_t)tb.wx.size();
        }
        PartTracks &pt = pointXXvv[it];
        const int np = (int)pt.pind.size();
        tb.off = pt.tr.off;  // copies: the step writes its tracks back into the block
        tb.slot = pt.tr.slot;
        tb.img.resize(pt.tr.img.size());
        for (size_t t = 0; t < pt.tr.img.size(); ++t) tb.img[t] = loc[pt.tr.img[t]];
        tb.XX.resize(3 * (size_t)np);
        for (int j = 0; j < np; ++j)
          for (int c = 0; c < 3; ++c) tb.XX[3 * j + c] = (float)XXd[3 * (size_t)pt.pind[j] + c];
        rpba_block &b = tb.b;
        b.n_images = m;
        b.n_points = np;
        b.pmat = tb.pmat.data();
        b.K = tb.K.data();
        b.distpara = tb.dist.data();
        b.XX = tb.XX.data();
        b.img_obs_off = tb.ioff.data();
        b.xg = tb.xg.data();
        b.wx = tb.wx.data();
        b.wy = tb.wy.data();
        b.wxy = tb.wxy.data();
        b.pt_obs_off = tb.off.data();
        b.pt_obs_image = tb.img.data();
        b.pt_obs_slot = tb.slot.data();
        std::vector<uint8_t> used(std::max(np, 1), 0);
        std::vector<char> lg(1 << 12);
        const int st = step_fn(&b, &ol, gcpinfov[it].data(), W3ijiv[it].data(),
                                         (int32_t)(W3ijiv[it].size() / 6), gcpdatav.data(),
                                         (int32_t)(gcpdatav.size() / 3), nrimages, Pd.data(), Pout.data(),
                                         used.data(), nullptr, lg.data(), lg.size());
        if (st != RPBA_OK && st != RPBA_ERR_NO_OBS_IMAGE && st != RPBA_ERR_LOW_REDUNDANCY &&
            st != RPBA_ERR_NAN_STEP)
          return st;
        plog = lg.data();
        // OutputLSAP: PointXXvOut clears the lists of the points that
        // PointXXvIn did not take; the stored cameras and camerasnew
        pt.used.assign(used.begin(), used.begin() + np);
        for (int li = 0; li < m; ++li) {
          const int gi = imgs[li];
          std::memcpy(&PMdd[it][12 * (size_t)gi], &Pout[12 * (size_t)li], sizeof(double) * 12);
          std::memcpy(camerasoit[it][gi].K, &tb.K[9 * (size_t)li], sizeof(float) * 9);
          camerasoit[it][gi].d[0] = tb.dist[2 * li];
          camerasoit[it][gi].d[1] = tb.dist[2 * li + 1];
        }
        return (int)RPBA_OK;
      };
      // the partitions' steps are independent: run this rank's on `workers`
      // host threads (partitions taken from a counter), exchange the results
      // between ranks, then take the logs and the first failure in
      // partition order, as a sequential loop would
      std::vector<int> pst(T, RPBA_OK), mine;
      for (int it = 0; it < T; ++it)
        if (owner[it] == rk.rank) mine.push_back(it);
      std::vector<std::string> plogs(T);
      std::atomic<int> next{0};
      auto body = [&]() {
        for (;;) {
          const int q = next.fetch_add(1);
          if (q >= (int)mine.size()) break;
          const int it = mine[q];
          try {
            pst[it] = part_step(it, plogs[it]);
          } catch (const std::exception &) {  // allocation: reported as the step's failure
            pst[it] = RPBA_ERR_CUDA;
          }
        }
      };
      std::vector<std::thread> th;
      try {  // fewer workers if the host refuses a thread: the counter hands out the rest
        for (int k = 1; k < std::min(workers, (int)mine.size()); ++k) th.emplace_back(body);
      } catch (const std::system_error &) {
      }
      body();
      for (auto &t : th) t.join();
      if (rk.ag) {
        // this rank's partitions: status, log, cameras (double matrices,
        // intrinsics) of their images, and which of their points the step
        // took
        std::vector<uint8_t> pay;
        for (int it : mine) {
          put_v(pay, (int32_t)it);
          put_v(pay, (int32_t)pst[it]);
          put_v(pay, (uint64_t)plogs[it].size());
          put(pay, plogs[it].data(), plogs[it].size());
          for (int gi : imgindv[it]) {
            put(pay, &PMdd[it][12 * (size_t)gi], sizeof(double) * 12);
            put_v(pay, camerasoit[it][gi]);
          }
          const std::vector<uint8_t> &u = pointXXvv[it].used;
          put_v(pay, (uint64_t)u.size());
          put(pay, u.data(), u.size());
        }
        // sizes first, then the records padded to the largest
        const uint64_t sz = pay.size();
        std::vector<uint64_t> szs(rk.world);
        if (rk.ag(rk.ctx, &sz, sizeof sz, szs.data()) != 0) return RPBA_ERR_COMM;
        const uint64_t mx = std::max<uint64_t>(1, *std::max_element(szs.begin(), szs.end()));
        pay.resize(mx);
        std::vector<uint8_t> all(mx * rk.world);
        if (rk.ag(rk.ctx, pay.data(), mx, all.data()) != 0) return RPBA_ERR_COMM;
        for (int r = 0; r < rk.world; ++r) {
          if (r == rk.rank) continue;
          Reader rd{all.data() + mx * r, all.data() + mx * r + szs[r]};
          while (rd.ok && rd.p < rd.end) {
            const int it = rd.get_v<int32_t>();
            if (!rd.ok || it < 0 || it >= T || owner[it] != r) return RPBA_ERR_COMM;
            pst[it] = rd.get_v<int32_t>();
            const uint64_t nlog = rd.get_v<uint64_t>();
            if (!rd.ok || nlog > (uint64_t)(rd.end - rd.p)) return RPBA_ERR_COMM;
            plogs[it].assign((const char *)rd.p, (size_t)nlog);
            rd.p += nlog;
            for (int gi : imgindv[it]) {
              rd.get(&PMdd[it][12 * (size_t)gi], sizeof(double) * 12);
              camerasoit[it][gi] = rd.get_v<PCam>();
            }
            std::vector<uint8_t> &u = pointXXvv[it].used;
            if (rd.get_v<uint64_t>() != u.size()) return RPBA_ERR_COMM;
            rd.get(u.data(), u.size());
          }
          if (!rd.ok) return RPBA_ERR_COMM;
        }
      }
      for (int it = 0; it < T; ++it) {
        if (pst[it] != RPBA_OK) return pst[it];
        os += plogs[it];
      }
      for (int it = 0; it < T; ++it)
        for (int gi : imgindv[it]) {
          std::memcpy(&PMd[12 * (size_t)gi], &PMdd[it][12 * (size_t)gi], sizeof(double) * 12);
          cameraps[gi] = camerasoit[it][gi];
          camerasnew[gi] = camerasoit[it][gi];
        }
    }
    if (iflag == 1) {
      robustflagit = robustflag;
      if (robustflag) sig0frac = 1.02f;
    }
    if (iter > 1) {
      // every point's list: its lists in the partitions that took it, in
      // partition order; lists of fewer than two observations are cleared
      // (each partition list's place in its point's list is counted in
      // partition order; the lists are then copied by partitions on host
      // threads)
      std::vector<int32_t> cnt(pxs + 1, 0);
      std::vector<std::vector<int32_t>> dst(T);
      for (int it = 0; it < T; ++it) {
        const PartTracks &pt = pointXXvv[it];
        dst[it].resize(pt.pind.size());
        for (size_t j = 0; j < pt.pind.size(); ++j) {
          dst[it][j] = cnt[pt.pind[j]];
          if (pt.used[j]) cnt[pt.pind[j]] += pt.tr.len((int)j);
        }
      }
      Tracks nl;
      nl.off.assign(pxs + 1, 0);
      for (int p = 0; p < pxs; ++p) nl.off[p + 1] = nl.off[p] + (cnt[p] < 2 ? 0 : cnt[p]);
      nl.img.resize(nl.off[pxs]);
      nl.slot.resize(nl.off[pxs]);
      parallel_ranges(T, nranges(T, workers, 1), [&](int, int i0, int i1) {
        for (int it = i0; it < i1; ++it) {
          const PartTracks &pt = pointXXvv[it];
          for (size_t j = 0; j < pt.pind.size(); ++j) {
            const int p = pt.pind[j];
            if (!pt.used[j] || cnt[p] < 2) continue;
            int32_t o = nl.off[p] + dst[it][j];
            for (int t = pt.tr.off[j]; t < pt.tr.off[j + 1]; ++t, ++o) {
              nl.img[o] = pt.tr.img[t];
              nl.slot[o] = pt.tr.slot[t];
            }
          }
        }
      });
      pointXXv = std::move(nl);
    } else {
      for (int i = 0; i < nrimages; ++i) cameraps[i] = camerasnew[i] = cameras[i];
    }
    {
      // (point ranges on host threads: counts, then entries at the prefix
      // sums)
      const int W = nranges(pxs, workers, 4096);
      std::vector<int32_t> cr(W + 1, 0);
      auto distinct = [&](int p, std::vector<int> &seen, auto &&emit) {
        for (int t = pointXXv.off[p]; t < pointXXv.off[p + 1]; ++t) {
          const int it = imgindbv[pointXXv.img[t]];
          if (seen[it] != p) {
            seen[it] = p;
            emit(it);
          }
        }
      };
      parallel_ranges(pxs, W, [&](int k, int p0, int p1) {
        std::vector<int> seen(T, -1);
        int32_t c = 0;
        for (int p = p0; p < p1; ++p) {
          int32_t n = 0;
          distinct(p, seen, [&](int) { ++n; });
          pitp_off[p + 1] = n;
          c += n;
        }
        cr[k + 1] = c;
      });
      for (int k = 0; k < W; ++k) cr[k + 1] += cr[k];
      pitp.resize(cr[W]);
      parallel_ranges(pxs, W, [&](int k, int p0, int p1) {
        std::vector<int> seen(T, -1);
        int32_t o = cr[k];
        for (int p = p0; p < p1; ++p) {
          const int32_t n = pitp_off[p + 1];
          pitp_off[p + 1] = o + n;  // the end of p's entries (its start is the previous point's end)
          distinct(p, seen, [&](int it) { pitp[o++] = it; });
        }
      });
      pitp_off[0] = 0;
    }
    double sum = 0.;
    long long redundancy = 0;
    if (robustflagit) {
      std::vector<std::vector<float>> sig0vvs(nrimages);
      if (!sweep(1, false, false, &sig0vvs, &sum, &redundancy)) return status;
      // every image's median statistic (images on host threads)
      parallel_ranges(nrimages, nranges(nrimages, workers, 16), [&](int, int i0, int i1) {
        for (int i = i0; i < i1; ++i) {
          if (sig0vvs[i].empty()) {
            sig0wv[i] = 0.f;
          } else {
            std::sort(sig0vvs[i].begin(), sig0vvs[i].end());
            sig0wv[i] = 1.f / (sig0vvs[i][(int)sig0vvs[i].size() / 2] * 2.1981f);
          }
        }
      });
    }
    if (!sweep(robustflagit ? 2 : 0, iter == 1, true, nullptr, &sum, &redundancy)) return status;
    sig0g = sum / (double)(redundancy - nrparimages);
    {
      // the progress line (rpbacore.cpp:377-389; ihw2 = 1 for unit image sizes)
      const long long nrobs = 2 * (long long)pointXXv.img.size();
      const float ihw2 = 1.f;
      os += "IT: " + std::to_string(iter) + " " + std::to_string(iflag) + "  " + fmt_g(std::sqrt(sig0g * ihw2)) + ' ' +
            fmt_g(sig0opt / sig0g) + "  " + fmt_g(sig0g) + " " + std::to_string(redundancy) + " " +
            std::to_string(nrobs) + " " + std::to_string(nrparimages) + " " + std::to_string(nraddp) + "  " +
            std::to_string(redundancy - nrparimages) + "\n";
    }
    if (sig0g <= sig0opt) {
      XXdold = XXd;
      PMdold = PMd;
      pointXXvold = pointXXv;
      camerasold = camerasnew;
    }
    for (int it = 0; it < T; ++it) {
      camerasoit[it] = camerasnew;
      for (int gi : imgindv[it])
        std::memcpy(&PMdd[it][12 * (size_t)gi], &PMd[12 * (size_t)gi], sizeof(double) * 12);
      W3ijiv[it].clear();
    }
    // the next GCPs: points (tracks of 2 or more) seen by more than one partition
    // (the point chunks beginv[c] .. endv[c] of the reference's threads
    // cover the points in order).  Point ranges on host threads: a point
    // with a list of two or more observations whose observations fell in
    // two or more partitions at the start of the iteration becomes GCP
    // number g (in point order) and adds its weight block for each of
    // those partitions to the partition's W3 rows (in point order); the
    // other points with such lists get -1.  First pass: the counts per
    // range; second: the entries at the ranges' prefix sums.
    {
      const int W = nranges(pxs, workers, 4096);
      std::vector<int8_t> isg(pxs, -1);
      std::vector<int32_t> ng(W + 1, 0), nw((size_t)(W + 1) * T, 0);
      // the distinct partitions of the point's start-of-iteration list
      auto parts_of = [&](int p, std::vector<int> &, std::vector<int> &parts) {
        parts.assign(pitp.begin() + pitp_off[p], pitp.begin() + pitp_off[p + 1]);
      };
      parallel_ranges(pxs, W, [&](int k, int p0, int p1) {
        std::vector<int> seen(T, -1), parts;
        std::vector<int32_t> w(T, 0);  // counted locally: the ranges' counts share cache lines
        int32_t g = 0;
        for (int p = p0; p < p1; ++p) {
          if (pointXXv.len(p) < 2) continue;
          parts_of(p, seen, parts);
          isg[p] = parts.size() > 1 ? 1 : 0;
          if (!isg[p]) continue;
          ++g;
          for (int it : parts) ++w[it];
        }
        ng[k + 1] = g;
        std::copy(w.begin(), w.end(), nw.begin() + (size_t)(k + 1) * T);
      });
      for (int k = 0; k < W; ++k) {
        ng[k + 1] += ng[k];
        for (int it = 0; it < T; ++it) nw[(size_t)(k + 1) * T + it] += nw[(size_t)k * T + it];
      }
      gcpdatav.assign(3 * (size_t)ng[W], 0.);
      for (int it = 0; it < T; ++it) W3ijiv[it].assign(6 * (size_t)nw[(size_t)W * T + it], 0.f);
      parallel_ranges(pxs, W, [&](int k, int p0, int p1) {
        std::vector<int> seen(T, -1), parts;
        std::vector<int32_t> wp(nw.begin() + (size_t)k * T, nw.begin() + (size_t)(k + 1) * T);
        int32_t g = ng[k];
        for (int p = p0; p < p1; ++p) {
          if (isg[p] < 0) continue;
          if (!isg[p]) {
            gcpinfo[p] = -1;
            continue;
          }
          gcpinfo[p] = g;
          for (int q = 0; q < 3; ++q) gcpdatav[3 * (size_t)g + q] = XXd[3 * (size_t)p + q];
          parts_of(p, seen, parts);
          for (int it : parts)
            std::memcpy(&W3ijiv[it][6 * (size_t)wp[it]++], &w3d[((size_t)p * T + it) * 6], sizeof(float) * 6);
          ++g;
        }
      });
    }
    // every partition's points, in point order, with their observations in
    // the partition's images (point ranges on host threads: points and
    // observations counted per range and partition, then written at the
    // prefix sums)
    {
      const int W = nranges(pxs, workers, 4096);
      std::vector<int32_t> cp((size_t)(W + 1) * T, 0), co((size_t)(W + 1) * T, 0);
      parallel_ranges(pxs, W, [&](int k, int p0, int p1) {
        std::vector<int> lastp(T, -1);
        std::vector<int32_t> np_(T, 0), no_(T, 0);  // counted locally, as above
        for (int p = p0; p < p1; ++p)
          for (int t = pointXXv.off[p]; t < pointXXv.off[p + 1]; ++t) {
            const int it = imgindbv[pointXXv.img[t]];
            if (lastp[it] != p) {
              lastp[it] = p;
              ++np_[it];
            }
            ++no_[it];
          }
        std::copy(np_.begin(), np_.end(), cp.begin() + (size_t)(k + 1) * T);
        std::copy(no_.begin(), no_.end(), co.begin() + (size_t)(k + 1) * T);
      });
      for (int k = 0; k < W; ++k)
        for (int it = 0; it < T; ++it) {
          cp[(size_t)(k + 1) * T + it] += cp[(size_t)k * T + it];
          co[(size_t)(k + 1) * T + it] += co[(size_t)k * T + it];
        }
      for (int it = 0; it < T; ++it) {
        PartTracks &pt = pointXXvv[it];
        const int32_t npt = cp[(size_t)W * T + it], nob = co[(size_t)W * T + it];
        pt.pind.resize(npt);
        pt.tr.off.resize(npt + 1);
        pt.tr.off[npt] = nob;
        pt.tr.img.resize(nob);
        pt.tr.slot.resize(nob);
      }
      parallel_ranges(pxs, W, [&](int k, int p0, int p1) {
        std::vector<int> lastp(T, -1);
        std::vector<int32_t> pp(cp.begin() + (size_t)k * T, cp.begin() + (size_t)(k + 1) * T);
        std::vector<int32_t> oo(co.begin() + (size_t)k * T, co.begin() + (size_t)(k + 1) * T);
        for (int p = p0; p < p1; ++p)
          for (int t = pointXXv.off[p]; t < pointXXv.off[p + 1]; ++t) {
            const int it = imgindbv[pointXXv.img[t]];
            PartTracks &pt = pointXXvv[it];
            if (lastp[it] != p) {
              lastp[it] = p;
              pt.pind[pp[it]] = p;
              pt.tr.off[pp[it]++] = oo[it];
            }
            pt.tr.img[oo[it]] = pointXXv.img[t];
            pt.tr.slot[oo[it]++] = pointXXv.slot[t];
          }
      });
    }
    for (int it = 0; it < T; ++it) {
      PartTracks &pt = pointXXvv[it];
      pt.used.assign(pt.pind.size(), 1);
      gcpinfov[it].resize(pt.pind.size());
      for (size_t j = 0; j < pt.pind.size(); ++j) gcpinfov[it][j] = gcpinfo[pt.pind[j]];
    }
    if (iter > 1) {
      if (sig0g <= sig0opt) {
        if (sig0opt < sig0g * sig0frac && iter > 3)
          --iflag;
        else
          sig0opt = sig0g;
      } else if (iter > 3) {
        --iflag;
      }
    }
    ++iter;
  }
  // pointXXvio = pointXXvold, PMatrices, XX, cameras (rpbacore.cpp:498-507)
  for (int p = 0; p <= pxs; ++p) blk->pt_obs_off[p] = pointXXvold.off[p];
  std::copy(pointXXvold.img.begin(), pointXXvold.img.end(), blk->pt_obs_image);
  std::copy(pointXXvold.slot.begin(), pointXXvold.slot.end(), blk->pt_obs_slot);
  for (size_t i = 0; i < PMdold.size(); ++i) blk->pmat[i] = (float)PMdold[i];
  for (size_t i = 0; i < XXdold.size(); ++i) blk->XX[i] = (float)XXdold[i];
  for (int i = 0; i < nrimages; ++i) {
    std::memcpy(blk->K + 9 * (size_t)i, camerasold[i].K, sizeof(float) * 9);
    blk->distpara[2 * i] = camerasold[i].d[0];
    blk->distpara[2 * i + 1] = camerasold[i].d[1];
  }
  if (stats) {
    stats[0] = sig0opt;
    stats[1] = iter - 1;
  }
  if (log && cap) {
    const size_t n = std::min(cap - 1, os.size());
    std::memcpy(log, os.data(), n);
    log[n] = 0;
  }
  return RPBA_OK;
}

}  // namespace

// The loop's host containers may throw (allocation, thread creation); no
// exception crosses the C ABI.
template <class F>
int32_t no_throw(F &&f) {
  try {
    return f();
  } catch (const std::exception &) {
    return RPBA_ERR_CUDA;
  }
}

extern "C" int32_t rpba_calc_plsa_parallel(rpba_block *blk, const rpba_options *opt, int32_t nthreads,
                                           const int32_t *part, char *log, size_t cap, double *stats) {
  if (opt && (opt->exteval || opt->precision != RPBA_PREC_FP64 ||
              (opt->solver != RPBA_SOLVER_PCG && opt->solver != RPBA_SOLVER_DIRECT)))
    return RPBA_ERR_UNSUPPORTED;
  return no_throw([&] {
    return plsa_parallel(blk, opt, nthreads, part, log, cap, stats, rpba_lsa_gcp_step, gpu_merge, host_workers());
  });
}

extern "C" int32_t rpba_calc_plsa_parallel_hosted(rpba_block *blk, const rpba_options *opt, int32_t nthreads,
                                                  const int32_t *part, char *log, size_t cap, double *stats,
                                                  rpba_gcp_step_fn step, rpba_merge_fn merge) {
  if (!step || !merge) return RPBA_ERR_ARG;
  return no_throw([&] {
    return plsa_parallel(blk, opt, nthreads, part, log, cap, stats, step, merge, host_workers());
  });
}

extern "C" int32_t rpba_calc_plsa_parallel_ranks(rpba_block *blk, const rpba_options *opt, int32_t nthreads,
                                                 const int32_t *part, char *log, size_t cap, double *stats,
                                                 int32_t rank, int32_t world, rpba_allgather_fn allgather,
                                                 void *ctx) {
  if (opt && (opt->exteval || opt->precision != RPBA_PREC_FP64 ||
              (opt->solver != RPBA_SOLVER_PCG && opt->solver != RPBA_SOLVER_DIRECT)))
    return RPBA_ERR_UNSUPPORTED;
  if (!allgather) return RPBA_ERR_ARG;
  Ranks rk;
  rk.rank = rank;
  rk.world = world;
  rk.ag = allgather;
  rk.ctx = ctx;
  return no_throw([&] {
    return plsa_parallel(blk, opt, nthreads, part, log, cap, stats, rpba_lsa_gcp_step, gpu_merge, host_workers(), rk);
  });
}

extern "C" int32_t rpba_calc_plsa_parallel_ranks_hosted(rpba_block *blk, const rpba_options *opt,
                                                        int32_t nthreads, const int32_t *part, char *log,
                                                        size_t cap, double *stats, rpba_gcp_step_fn step,
                                                        rpba_merge_fn merge, int32_t rank, int32_t world,
                                                        rpba_allgather_fn allgather, void *ctx) {
  if (!step || !merge || !allgather) return RPBA_ERR_ARG;
  Ranks rk;
  rk.rank = rank;
  rk.world = world;
  rk.ag = allgather;
  rk.ctx = ctx;
  return no_throw([&] {
    return plsa_parallel(blk, opt, nthreads, part, log, cap, stats, step, merge, host_workers(), rk);
  });
}
