// partition.cpp -- camera partition of the reference's parallel RPBA
// (PartitionpointXXv, rpbacore.cpp:945-1037), host code.
//
// The reference builds the images' covisibility graph (an edge wherever two
// images share a point observed at least twice; unweighted), weights every
// image by floor(BM^0.3333) with BM the sum of the track lengths of its
// points, and cuts it into nrthreads contiguous parts with
// METIS_PartGraphRecursive and METIS_OPTION_CONTIG.  METIS is not available
// here, so the cut is a deterministic recursive bisection of this library's
// own: each half is grown breadth-first from a pseudo-peripheral vertex until
// it holds its share of the weight, and the components that this leaves
// detached from the rest join the grown half.  On a connected graph both
// halves stay connected at every level, so every part is contiguous.
// The graph is kept as sorted adjacency lists (the reference's dense
// N_img x N_img matrix would take 750 MB at 13,700 images).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <system_error>
#include <thread>
#include <vector>

#include "../../include/rpba_b200.h"

namespace {

struct Graph {
  std::vector<int> off, adj;  // CSR adjacency, neighbours sorted by index
  std::vector<long long> w;   // vertex weights
};

Graph build_graph(const rpba_block *b) {
  const int n = b->n_images;
  Graph g;
  g.w.assign(n, 0);
  // BM[i]: sum of the track lengths of the image's points (tracks of >= 2)
  std::vector<long long> bm(n, 0);
  for (int p = 0; p < b->n_points; ++p) {
    const int t0 = b->pt_obs_off[p], t1 = b->pt_obs_off[p + 1];
    if (t1 - t0 < 2) continue;
    for (int t = t0; t < t1; ++t) bm[b->pt_obs_image[t]] += t1 - t0;
  }
  for (int i = 0; i < n; ++i) g.w[i] = (long long)std::pow((double)bm[i], 0.3333);
  g.off.assign(n + 1, 0);
  const int T = n >= 256 ? (int)std::min(32u, std::max(1u, std::thread::hardware_concurrency())) : 1;
  // work(k) for k < T, one thread each (a k whose thread cannot be created
  // runs on the calling thread: the ranges are independent)
  auto run = [&](auto &&work) {
    std::vector<std::thread> th;
    int k = 1;
    try {
      for (; k < T; ++k) th.emplace_back(work, k);
    } catch (const std::system_error &) {
    }
    for (int j = k; j < T; ++j) work(j);
    work(0);
    for (auto &t : th) t.join();
  };
  if (n <= 32768) {
    // neighbours of every image as a bit row (n bits; at most 128 MB in
    // all), images split over host threads in contiguous ranges: each
    // thread streams every track in order and sets, for each of its images
    // in the track, the bits of the track's other images; the rows are then
    // read out in index order, so the lists come out sorted
    const size_t words = ((size_t)n + 63) / 64;
    std::vector<uint64_t> bits((size_t)n * words, 0);
    run([&](int k) {
      const int lo = (int)((long long)n * k / T), hi = (int)((long long)n * (k + 1) / T);
      for (int p = 0; p < b->n_points; ++p) {
        const int t0 = b->pt_obs_off[p], t1 = b->pt_obs_off[p + 1];
        if (t1 - t0 < 2) continue;
        for (int t = t0; t < t1; ++t) {
          const int i = b->pt_obs_image[t];
          if (i < lo || i >= hi) continue;
          uint64_t *row = &bits[(size_t)i * words];
          for (int u = t0; u < t1; ++u) {
            const int j = b->pt_obs_image[u];
            if (j != i) row[j >> 6] |= 1ull << (j & 63);
          }
        }
      }
    });
    for (int i = 0; i < n; ++i) {
      int c = 0;
      for (size_t w = 0; w < words; ++w) c += __builtin_popcountll(bits[(size_t)i * words + w]);
      g.off[i + 1] = g.off[i] + c;
    }
    g.adj.resize(g.off[n]);
    run([&](int k) {
      for (int i = (int)((long long)n * k / T); i < (int)((long long)n * (k + 1) / T); ++i) {
        int o = g.off[i];
        for (size_t w = 0; w < words; ++w)
          for (uint64_t v = bits[(size_t)i * words + w]; v; v &= v - 1) g.adj[o++] = (int)(w * 64) + __builtin_ctzll(v);
      }
    });
    return g;
  }
  // larger scenes: neighbours of every image through its points (a stamp
  // array per thread marks the ones already listed), images split over host
  // threads in contiguous ranges; each list is sorted, so the result does not
  // depend on the thread count
  std::vector<int> ipo(n + 1, 0);  // image -> points (CSR)
  for (int p = 0; p < b->n_points; ++p) {
    const int t0 = b->pt_obs_off[p], t1 = b->pt_obs_off[p + 1];
    if (t1 - t0 < 2) continue;
    for (int t = t0; t < t1; ++t) ++ipo[b->pt_obs_image[t] + 1];
  }
  for (int i = 0; i < n; ++i) ipo[i + 1] += ipo[i];
  std::vector<int> ipts(ipo[n]), fill(ipo.begin(), ipo.end() - 1);
  for (int p = 0; p < b->n_points; ++p) {
    const int t0 = b->pt_obs_off[p], t1 = b->pt_obs_off[p + 1];
    if (t1 - t0 < 2) continue;
    for (int t = t0; t < t1; ++t) ipts[fill[b->pt_obs_image[t]]++] = p;
  }
  std::vector<std::vector<int>> nbr(n);
  run([&](int k) {
    std::vector<int> stamp(n, -1);
    for (int i = (int)((long long)n * k / T); i < (int)((long long)n * (k + 1) / T); ++i) {
      std::vector<int> &out = nbr[i];
      for (int q = ipo[i]; q < ipo[i + 1]; ++q) {
        const int p = ipts[q];
        for (int t = b->pt_obs_off[p]; t < b->pt_obs_off[p + 1]; ++t) {
          const int j = b->pt_obs_image[t];
          if (j != i && stamp[j] != i) {
            stamp[j] = i;
            out.push_back(j);
          }
        }
      }
      std::sort(out.begin(), out.end());
    }
  });
  for (int i = 0; i < n; ++i) g.off[i + 1] = g.off[i] + (int)nbr[i].size();
  g.adj.resize(g.off[n]);
  for (int i = 0; i < n; ++i) std::copy(nbr[i].begin(), nbr[i].end(), g.adj.begin() + g.off[i]);
  return g;
}

class Bisector {
 public:
  // spawn_depth: levels of the recursion whose first half is cut on a
  // thread of its own (with its own Bisector: its own scratch arrays, so
  // the halves share nothing but the graph; a cut depends only on its set,
  // so the parts do not depend on the threads)
  Bisector(const Graph &g, int32_t *part, int spawn_depth = 0)
      : g_(g), part_(part), spawn_depth_(spawn_depth), in_(g.w.size(), 0), mark_(g.w.size(), 0) {}

  // Cuts `verts` (sorted) into k parts numbered base .. base + k - 1.
  void cut(std::vector<int> verts, int k, int base, int depth = 0) {
    if (k <= 1 || verts.size() <= 1) {
      for (int v : verts) part_[v] = base;
      return;
    }
    const int k1 = k / 2;
    long long total = 0;
    for (int v : verts) total += g_.w[v];
    const long long target = (total * k1 + k / 2) / k;
    const int tag = ++tag_;
    for (int v : verts) in_[v] = tag;
    // grow the first half breadth-first from a pseudo-peripheral vertex;
    // a component exhausted before the target continues from the next
    // unvisited vertex of the set
    const int side1 = ++tag_;
    long long w1 = 0;
    size_t n1 = 0;
    int last_added = -1;
    std::vector<int> queue;
    int seed = peripheral(verts.front(), tag);
    size_t next_unvisited = 0;
    while (w1 < target || n1 == 0) {
      if (queue.empty()) {
        if (mark_[seed] == side1) {
          while (next_unvisited < verts.size() && mark_[verts[next_unvisited]] == side1) ++next_unvisited;
          if (next_unvisited == verts.size()) break;
          seed = verts[next_unvisited];
        }
        mark_[seed] = side1;
        w1 += g_.w[seed];
        ++n1;
        last_added = seed;
        queue.assign(1, seed);
        continue;
      }
      std::vector<int> nextq;
      for (size_t qi = 0; qi < queue.size() && (w1 < target); ++qi) {
        const int v = queue[qi];
        for (int e = g_.off[v]; e < g_.off[v + 1] && w1 < target; ++e) {
          const int u = g_.adj[e];
          if (in_[u] != tag || mark_[u] == side1) continue;
          mark_[u] = side1;
          w1 += g_.w[u];
          ++n1;
          last_added = u;
          nextq.push_back(u);
        }
      }
      queue.swap(nextq);
    }
    if (n1 == verts.size()) {  // nothing left for the second half
      mark_[last_added] = 0;
      --n1;
    }
    // the rest: keep its heaviest component, the others join the first half
    std::vector<int> rest;
    for (int v : verts)
      if (mark_[v] != side1) rest.push_back(v);
    const int comp_tag = ++tag_;
    std::vector<int> best;
    long long best_w = -1;
    for (int r : rest) {
      if (mark_[r] == comp_tag) continue;
      std::vector<int> comp(1, r);
      mark_[r] = comp_tag;
      long long cw = g_.w[r];
      for (size_t qi = 0; qi < comp.size(); ++qi) {
        const int v = comp[qi];
        for (int e = g_.off[v]; e < g_.off[v + 1]; ++e) {
          const int u = g_.adj[e];
          if (in_[u] != tag || mark_[u] == side1 || mark_[u] == comp_tag) continue;
          mark_[u] = comp_tag;
          cw += g_.w[u];
          comp.push_back(u);
        }
      }
      if (cw > best_w) {
        best_w = cw;
        best = comp;
      }
    }
    std::vector<int> h1, h2;
    const int keep = ++tag_;
    for (int v : best) mark_[v] = keep;
    for (int v : verts) (mark_[v] == keep ? h2 : h1).push_back(v);
    std::thread t;
    if (depth < spawn_depth_ && h1.size() >= 256 && h2.size() >= 256) {
      try {
        t = std::thread([&] { Bisector(g_, part_, spawn_depth_).cut(std::move(h1), k1, base, depth + 1); });
      } catch (const std::system_error &) {  // no thread: both halves here
      }
    }
    if (t.joinable()) {
      cut(std::move(h2), k - k1, base + k1, depth + 1);
      t.join();
    } else {
      cut(std::move(h1), k1, base, depth + 1);
      cut(std::move(h2), k - k1, base + k1, depth + 1);
    }
  }

 private:
  // a pseudo-peripheral vertex of the set: the farthest vertex of a
  // breadth-first search from the farthest vertex of one from `start`
  int peripheral(int start, int tag) {
    int v = start;
    for (int round = 0; round < 2; ++round) {
      const int seen = ++tag_;
      std::vector<int> q(1, v);
      mark_[v] = seen;
      for (size_t qi = 0; qi < q.size(); ++qi) {
        const int x = q[qi];
        for (int e = g_.off[x]; e < g_.off[x + 1]; ++e) {
          const int u = g_.adj[e];
          if (in_[u] != tag || mark_[u] == seen) continue;
          mark_[u] = seen;
          q.push_back(u);
        }
      }
      v = q.back();
    }
    return v;
  }

  const Graph &g_;
  int32_t *part_;
  int spawn_depth_;
  std::vector<int> in_, mark_;
  int tag_ = 0;
};

}  // namespace

extern "C" int32_t rpba_partition_images(const rpba_block *blk, int32_t nparts, int32_t *part) {
  if (!blk || !part || nparts < 1 || blk->n_images < 1) return RPBA_ERR_ARG;
  const Graph g = build_graph(blk);
  std::vector<int> all(blk->n_images);
  for (int i = 0; i < blk->n_images; ++i) all[i] = i;
  int depth = 0;  // about one thread per host core at the deepest spawning level
  for (unsigned c = std::max(1u, std::thread::hardware_concurrency()); c > 1 && depth < 6; c >>= 1) ++depth;
  Bisector(g, part, depth).cut(all, nparts, 0);
  return RPBA_OK;
}
