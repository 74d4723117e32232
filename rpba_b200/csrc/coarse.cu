// coarse.cu -- coarse space of the two-level preconditioner of the reduced
// camera system (RCS).
//
// Block-Jacobi (rbacore.cpp:1841) removes the error of each camera block
// against its own diagonal, but not the smooth error in which neighbouring
// cameras move together: on a long street or a city those modes take CG
// hundreds of iterations.  The near-null space of the RCS is known: a small
// similarity transform of the world (all cameras and, through the Schur
// complement, all points) changes no residual, so it is opposed only by the
// gauge and by damping.  Grouping cameras into spatially compact aggregates
// and giving each aggregate its own small similarity transform spans the
// smooth modes; with P the prolongation and A_c = P^T S P the Galerkin
// matrix, the preconditioner is
//     M^-1 = C + P A_c^-1 P^T          (C: the (learned) block-Jacobi part)
//
// Per camera k (x = R (X + PC), R_new = Cayley(w) R), a world motion
// X' = (I + [d]x) X + t seen by unchanged images needs
//     w = -R d,   dPC = d x (PC - c_a) - t',   and a scale s: dPC = s (PC - c_a)
// (c_a the aggregate's mean PC).  The coarse unknowns of aggregate a are
// (d 3, t 3, s, and common shifts of k1, k2, f): CO_M = 10.
//
// Everything here is deterministic: every sum has a fixed order.
#include <cub/cub.cuh>

#include <algorithm>
#include <numeric>
#include <vector>

#include "internal.h"

namespace rpba {

namespace {

constexpr int CP = CO_M * 9;  // P_k entries

// P_k for the rows of aggregate blockIdx.x (row major, 9 x CO_M).
__global__ void k_coarse_P(DevLSA L, CoarseWork C) {
  const int a = blockIdx.x;
  const int t0 = C.agg_off[a], t1 = C.agg_off[a + 1];
  __shared__ double cen[3], rho_inv;
  if (threadIdx.x == 0) {
    double c[3] = {0., 0., 0.};
    int n = 0;
    for (int t = t0; t < t1; ++t) {
      const int k = C.agg_rows[t];
      if (k < 1) continue;
      for (int j = 0; j < 3; ++j) c[j] += L.camn[k].PC[j];
      ++n;
    }
    for (int j = 0; j < 3; ++j) c[j] /= (n > 0 ? n : 1);
    double r2 = 0.;
    for (int t = t0; t < t1; ++t) {
      const int k = C.agg_rows[t];
      if (k < 1) continue;
      for (int j = 0; j < 3; ++j) {
        const double d = L.camn[k].PC[j] - c[j];
        r2 += d * d;
      }
    }
    const double rho = sqrt(r2 / (n > 0 ? n : 1));
    for (int j = 0; j < 3; ++j) cen[j] = c[j];
    rho_inv = rho > 0. ? 1. / rho : 0.;
  }
  __syncthreads();
  for (int t = t0 + threadIdx.x; t < t1; t += blockDim.x) {
    const int k = C.agg_rows[t];
    double *P = C.P + (size_t)k * CP;
    for (int i = 0; i < CP; ++i) P[i] = 0.;
    if (k < 1) continue;  // camera 0's intrinsics row: block-Jacobi only
    const CamState &cs = L.camn[k];
    for (int r = 0; r < 3; ++r)
      for (int j = 0; j < 3; ++j) P[r * CO_M + j] = -cs.R[r * 3 + j];
    const double lev[3] = {cs.PC[0] - cen[0], cs.PC[1] - cen[1], cs.PC[2] - cen[2]};
    // cr[j][c] = (e_j x lev)_c
    const double cr[3][3] = {{0., -lev[2], lev[1]}, {lev[2], 0., -lev[0]}, {-lev[1], lev[0], 0.}};
    int comp[3] = {0, 1, 2}, npc = 3;
    if (k == L.normcamera) {
      comp[0] = L.gauge[0];
      comp[1] = L.gauge[1];
      npc = 2;
    }
    for (int q = 0; q < npc; ++q) {
      const int c = comp[q], r = 3 + q;
      for (int j = 0; j < 3; ++j) P[r * CO_M + j] = cr[j][c];
      P[r * CO_M + 3 + c] = 1.;
      P[r * CO_M + 6] = lev[c] * rho_inv;
    }
    int r = 3 + npc;
    if (L.addmask & 1) P[(r++) * CO_M + 7] = 1.;
    if (L.addmask & 2) P[(r++) * CO_M + 8] = 1.;
    if (L.addmask & 4) P[(r++) * CO_M + 9] = 1.;
  }
}

// Galerkin matrix A_c = P^T S P in three deterministic steps.
//  1. The entries (k, l) of every row are sorted by (k, aggregate of l)
//     (a stable sort: entry order inside a run), once per structure.
//  2. One warp per run (row k, aggregate b): Y = sum_l S_kl P_l (9 x 10),
//     Z = P_k^T Y (10 x 10).
//  3. The runs sorted by (aggregate of k, b) (stable: row order); one warp
//     per coarse block (a, b) sums its runs' Z in that order.
// A_c is symmetric (S is): only the blocks (a, b) with b >= a are summed,
// and each block with b > a is written to (b, a) transposed as well, so
// the entries (k, l) whose column's aggregate precedes the row's are left
// out of the runs.
__global__ void k_entry_keys(DevLSA L, CoarseWork C, unsigned *key, int *val) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= L.nimg) return;
  const int a = C.row_agg[k];
  for (int e = L.rowoff[k]; e < L.rowoff[k + 1]; ++e) {
    const int b = C.row_agg[L.ent[e].x];
    key[e] = (b < 0 || b < a) ? 0xffffffffu : (unsigned)k * (unsigned)C.nagg + (unsigned)b;
    val[e] = e;
  }
}

// Step 2, one warp per run.  Per entry (l, S_kl) the warp stages S_kl in the
// run's orientation (row p of k, column q of l) and P_l^T in shared memory,
// the global loads of the next entry already in flight; lane (j, s) < 30
// then owns Y[3 s .. 3 s + 2][j] and reads row p of S and column j of P_l as
// 16-byte pairs.  Each Y entry sums q = 0 .. npl - 1 per entry, the entries
// in run order (the same operations in the same order as a lane per Y entry
// reading both operands from global memory).
constexpr int RS_T = 256, RS_W = RS_T / 32;
__global__ void __launch_bounds__(RS_T) k_coarse_runs(DevLSA L, CoarseWork C, int nruns) {
  __shared__ __align__(16) double Ssh[RS_W][90];   // S_kl[p][q] at 10 p + q
  __shared__ __align__(16) double Psh[RS_W][100];  // P_l[q][j] at 10 j + q
  __shared__ double Ysh[RS_W][9 * CO_M];
  const int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
  if (r >= nruns) return;
  double *Ss = Ssh[wl], *Ps = Psh[wl];
  const int k = (int)(C.run_key[r] / (unsigned)C.nagg);
  const int npk = L.camparv[k + 1] - L.camparv[k];
  const int jc = lane % 10, s3 = lane < 30 ? lane / 10 : 0;
  double y[3] = {0., 0., 0.};
  const int t0 = C.run_off[r], t1 = C.run_off[r + 1];
  int2 en = make_int2(0, 0);
  double sv[3], pv[3];
  auto fetch = [&](int t) {
    en = L.ent[C.ent_sorted[t]];
    const size_t B = (size_t)(en.y & 0x7fffffff);
    const double *Pl = C.P + (size_t)en.x * CP;
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      const int e = lane + 32 * m;
      sv[m] = e < 81 ? blk_at(L, B, e) : 0.;
      pv[m] = e < CP ? __ldg(Pl + e) : 0.;
    }
  };
  if (t0 < t1) fetch(t0);
  for (int t = t0; t < t1; ++t) {
    const bool tr = en.y < 0;
    const int l = en.x;
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      const int e = lane + 32 * m;
      if (e < 81) {
        const int i = e / 9, c = e - 9 * (e / 9);
        Ss[tr ? c * 10 + i : i * 10 + c] = sv[m];
      }
      if (e < CP) {
        const int q = e / CO_M, j = e - CO_M * (e / CO_M);
        Ps[j * 10 + q] = pv[m];
      }
    }
    const int npl = L.camparv[l + 1] - L.camparv[l];
    __syncwarp();
    if (t + 1 < t1) fetch(t + 1);
    double pc[10];
#pragma unroll
    for (int h = 0; h < 5; ++h) {
      const double2 v = *(const double2 *)(Ps + jc * 10 + 2 * h);
      pc[2 * h] = v.x;
      pc[2 * h + 1] = v.y;
    }
#pragma unroll
    for (int u = 0; u < 3; ++u) {
      const int p = 3 * s3 + u;
      double sr[10];
#pragma unroll
      for (int h = 0; h < 5; ++h) {
        const double2 v = *(const double2 *)(Ss + p * 10 + 2 * h);
        sr[2 * h] = v.x;
        sr[2 * h + 1] = v.y;
      }
      if (lane < 30 && p < npk) {
#pragma unroll
        for (int q = 0; q < 9; ++q)
          if (q < npl) y[u] += sr[q] * pc[q];
      }
    }
    __syncwarp();
  }
  if (lane < 30)
#pragma unroll
    for (int u = 0; u < 3; ++u) Ysh[wl][(3 * s3 + u) * CO_M + jc] = y[u];
  __syncwarp();
  const double *Pk = C.P + (size_t)k * CP;
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    const int o = lane + 32 * m, i = o / CO_M, j = o % CO_M;
    if (o < CO_M * CO_M) {
      double z = 0.;
      for (int p = 0; p < npk; ++p) z += Pk[p * CO_M + i] * Ysh[wl][p * CO_M + j];
      C.Z[(size_t)r * CO_M * CO_M + o] = z;
    }
  }
}

__global__ void k_run_keys2(CoarseWork C, int nruns, unsigned *key2, int *idx) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nruns) return;
  const unsigned key = C.run_key[r];
  const int k = (int)(key / (unsigned)C.nagg), b = (int)(key % (unsigned)C.nagg);
  key2[r] = (unsigned)C.row_agg[k] * (unsigned)C.nagg + (unsigned)b;
  idx[r] = r;
}

__global__ void k_coarse_blocks(CoarseWork C, int nsegs) {
  const int sg = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (sg >= nsegs) return;
  const unsigned key = C.seg_key[sg];
  const int a = (int)(key / (unsigned)C.nagg), b = (int)(key % (unsigned)C.nagg);
  double acc[4] = {0., 0., 0., 0.};
  for (int t = C.seg_off[sg]; t < C.seg_off[sg + 1]; ++t) {
    const double *Z = C.Z + (size_t)C.run_sorted[t] * CO_M * CO_M;
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      const int o = lane + 32 * m;
      if (o < CO_M * CO_M) acc[m] += Z[o];
    }
  }
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    const int o = lane + 32 * m, i = o / CO_M, j = o % CO_M;
    if (o < CO_M * CO_M) {
      C.Ac[(size_t)(a * CO_M + i) * C.nc + b * CO_M + j] = acc[m];
      if (b != a) C.Ac[(size_t)(b * CO_M + j) * C.nc + a * CO_M + i] = acc[m];
    }
  }
}

// a coarse unknown that no parameter carries (an intrinsic that is not
// estimated) has an empty row and column: give it a unit diagonal
__global__ void k_coarse_fixdiag(CoarseWork C) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= C.nc) return;
  double &d = C.Ac[(size_t)i * C.nc + i];
  if (d == 0.) d = 1.;
}

// Symmetric Jacobi scaling of A_c before the factorisation (the coarse
// unknowns mix radians, metres, pixels and distortion coefficients, whose
// diagonal entries span many decades): dsc = diag^-1/2, A <- D A D with a
// unit diagonal (+1e-6: an aggregate whose cameras barely fix one of its
// coarse unknowns leaves A_c nearly singular, and a preconditioner needs
// only to stay SPD); the same kernel without the
// diagonal term maps the inverse back (A^-1 = D (D A D)^-1 D).
__global__ void k_coarse_diag(CoarseWork C) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= C.nc) return;
  const double d = C.Ac[(size_t)i * C.nc + i];
  C.dsc[i] = d > 0. ? 1. / sqrt(d) : 1.;
}

// rc_a = sum_{k in a} P_k^T r_k (rows in order)
__global__ void k_coarse_restrict(CoarseWork C, const double *r) {
  const int a = blockIdx.x, j = threadIdx.x;
  if (j >= CO_M) return;
  double s = 0.;
  for (int t = C.agg_off[a]; t < C.agg_off[a + 1]; ++t) {
    const int k = C.agg_rows[t];
    const double *P = C.P + (size_t)k * CP;
    for (int c = 0; c < 9; ++c) s += P[c * CO_M + j] * r[(size_t)k * 9 + c];
  }
  C.rc[a * CO_M + j] = s;
}

// z_a = A_c^-1[a rows] rc; h_k += P_k z_a for the rows of a
constexpr int PR_T = 256;
__global__ void __launch_bounds__(PR_T) k_coarse_prolong(CoarseWork C, double *h) {
  const int a = blockIdx.x, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __shared__ double part[PR_T / 32][CO_M];
  __shared__ double z[CO_M];
  double zz[CO_M];
#pragma unroll
  for (int j = 0; j < CO_M; ++j) zz[j] = 0.;
  for (int i = threadIdx.x; i < C.nc; i += PR_T) {
    const double rv = C.rc[i];
#pragma unroll
    for (int j = 0; j < CO_M; ++j) zz[j] += C.Ainv[(size_t)(a * CO_M + j) * C.nc + i] * rv;
  }
#pragma unroll
  for (int j = 0; j < CO_M; ++j) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) zz[j] += __shfl_xor_sync(0xffffffffu, zz[j], o);
    if (lane == 0) part[warp][j] = zz[j];
  }
  __syncthreads();
  if (threadIdx.x < CO_M) {
    double s = 0.;
    for (int w = 0; w < PR_T / 32; ++w) s += part[w][threadIdx.x];
    z[threadIdx.x] = s;
  }
  __syncthreads();
  for (int t = C.agg_off[a] + threadIdx.x; t < C.agg_off[a + 1]; t += PR_T) {
    const int k = C.agg_rows[t];
    const double *P = C.P + (size_t)k * CP;
    for (int c = 0; c < 9; ++c) {
      double s = 0.;
#pragma unroll
      for (int j = 0; j < CO_M; ++j) s += P[c * CO_M + j] * z[j];
      h[(size_t)k * 9 + c] += s;
    }
  }
}

// Recursive coordinate bisection of idx[lo, hi) into K groups: split along
// the widest axis at the share of the first half's groups.
void rcb(const std::vector<double> &pc, std::vector<int> &idx, int lo, int hi, int K, std::vector<int> &cuts) {
  if (K <= 1 || hi - lo <= 1) {
    cuts.push_back(hi);
    return;
  }
  double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
  for (int i = lo; i < hi; ++i)
    for (int j = 0; j < 3; ++j) {
      mn[j] = std::min(mn[j], pc[3 * idx[i] + j]);
      mx[j] = std::max(mx[j], pc[3 * idx[i] + j]);
    }
  int ax = 0;
  for (int j = 1; j < 3; ++j)
    if (mx[j] - mn[j] > mx[ax] - mn[ax]) ax = j;
  const int K1 = K / 2;
  const int mid = lo + (int)((long long)(hi - lo) * K1 / K);
  std::nth_element(idx.begin() + lo, idx.begin() + mid, idx.begin() + hi, [&](int u, int v) {
    const double a = pc[3 * u + ax], b = pc[3 * v + ax];
    return a < b || (a == b && u < v);
  });
  rcb(pc, idx, lo, mid, K1, cuts);
  rcb(pc, idx, mid, hi, K - K1, cuts);
}

template <class T>
T *calloc_dev(size_t n, std::vector<void *> &owned) {
  void *p = nullptr;
  RPBA_CUDA_CHECK(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)));
  owned.push_back(p);
  return (T *)p;
}

}  // namespace

void coarse_build(const DevLSA &L, int max_aggs, CoarseWork &C, std::vector<void *> &owned, cudaStream_t s) {
  C.nagg = C.nc = 0;
  const int nimg = L.nimg;
  const int ncam = nimg - 1;  // camera rows k >= 1
  if (ncam < 8) return;
  std::vector<CamState> cams(nimg);
  RPBA_CUDA_CHECK(cudaMemcpyAsync(cams.data(), L.camn, sizeof(CamState) * nimg, cudaMemcpyDeviceToHost, s));
  RPBA_CUDA_CHECK(cudaStreamSynchronize(s));
  std::vector<double> pc(3 * (size_t)nimg);
  for (int k = 0; k < nimg; ++k)
    for (int j = 0; j < 3; ++j) pc[3 * k + j] = cams[k].PC[j];
  const int K = std::max(1, std::min(std::min(max_aggs, 200), ncam / 16));
  std::vector<int> idx(ncam);
  std::iota(idx.begin(), idx.end(), 1);
  std::vector<int> cuts;
  rcb(pc, idx, 0, ncam, K, cuts);
  const int nagg = (int)cuts.size();
  std::vector<int> off(nagg + 1, 0), rows, row_agg(nimg, -1);
  for (int a = 0, lo = 0; a < nagg; ++a) {
    const int hi = cuts[a];
    std::vector<int> g(idx.begin() + lo, idx.begin() + hi);
    if (a == 0 && L.begini == 0) g.push_back(0);  // camera 0's intrinsics row rides along
    std::sort(g.begin(), g.end());
    for (int k : g) {
      rows.push_back(k);
      row_agg[k] = a;
    }
    off[a + 1] = (int)rows.size();
    lo = hi;
  }
  C.nagg = nagg;
  C.nc = nagg * CO_M;
  const size_t nc = C.nc;
  C.agg_off = calloc_dev<int>(nagg + 1, owned);
  C.agg_rows = calloc_dev<int>(rows.size(), owned);
  C.row_agg = calloc_dev<int>(nimg, owned);
  C.P = calloc_dev<double>((size_t)nimg * CP, owned);
  C.Ac = calloc_dev<double>(nc * nc, owned);
  C.Ainv = calloc_dev<double>(nc * nc, owned);
  C.rc = calloc_dev<double>(nc, owned);
  C.dsc = calloc_dev<double>(nc, owned);
  C.hj = calloc_dev<double>((size_t)nimg * 9, owned);
  C.err = calloc_dev<int>(1, owned);
  C.work = calloc_dev<char>(spd_inverse_bytes((int)nc), owned);
  C.bar = calloc_dev<unsigned>(2, owned);
  RPBA_CUDA_CHECK(cudaMemcpyAsync(C.agg_off, off.data(), sizeof(int) * (nagg + 1), cudaMemcpyHostToDevice, s));
  RPBA_CUDA_CHECK(cudaMemcpyAsync(C.agg_rows, rows.data(), sizeof(int) * rows.size(), cudaMemcpyHostToDevice, s));
  RPBA_CUDA_CHECK(cudaMemcpyAsync(C.row_agg, row_agg.data(), sizeof(int) * nimg, cudaMemcpyHostToDevice, s));
  RPBA_CUDA_CHECK(cudaMemsetAsync(C.P, 0, sizeof(double) * (size_t)nimg * CP, s));
  RPBA_CUDA_CHECK(cudaStreamSynchronize(s));
}

template <class T>
T *grow(T *&p, size_t &cap, size_t n) {
  if (n > cap) {
    if (p) cudaFree(p);
    p = nullptr;
    RPBA_CUDA_CHECK(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)));
    cap = n;
  }
  return p;
}

void coarse_assemble(const DevLSA &L, CoarseWork &C, int structure_version, cudaStream_t s) {
  if (C.nagg <= 0) return;
  RPBA_CUDA_CHECK(cudaMemsetAsync(C.err, 0, sizeof(int), s));
  k_coarse_P<<<C.nagg, 128, 0, s>>>(L, C);
  if (C.built_version != structure_version) {
    // runs (row, aggregate of the column) and coarse blocks (a, b): once per
    // structure
    int nent = 0;
    RPBA_CUDA_CHECK(cudaMemcpyAsync(&nent, L.rowoff + L.nimg, sizeof(int), cudaMemcpyDeviceToHost, s));
    RPBA_CUDA_CHECK(cudaStreamSynchronize(s));
    unsigned *k1 = grow(C.ekey, C.ekey_cap, (size_t)nent), *k2 = grow(C.ekey2, C.ekey2_cap, (size_t)nent);
    int *v1 = grow(C.eval, C.eval_cap, (size_t)nent);
    grow(C.ent_sorted, C.ent_sorted_cap, (size_t)nent);
    grow(C.run_key, C.run_key_cap, (size_t)nent);
    grow(C.run_cnt, C.run_cnt_cap, (size_t)nent + 1);
    grow(C.run_off, C.run_off_cap, (size_t)nent + 1);
    grow(C.counts, C.counts_cap, 2);
    k_entry_keys<<<(L.nimg + 127) / 128, 128, 0, s>>>(L, C, k1, v1);
    size_t need = 0, b1 = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, b1, k1, k2, v1, C.ent_sorted, nent, 0, 32, s);
    need = std::max(need, b1);
    cub::DeviceRunLengthEncode::Encode(nullptr, b1, k2, C.run_key, C.run_cnt, C.counts, nent, s);
    need = std::max(need, b1);
    cub::DeviceScan::ExclusiveSum(nullptr, b1, C.run_cnt, C.run_off, nent + 1, s);
    need = std::max(need, b1);
    void *tmp = grow(C.cub_tmp, C.cub_tmp_cap, need);
    RPBA_CUDA_CHECK(cub::DeviceRadixSort::SortPairs(tmp, need, k1, k2, v1, C.ent_sorted, nent, 0, 32, s));
    size_t bb = C.cub_tmp_cap;
    RPBA_CUDA_CHECK(cub::DeviceRunLengthEncode::Encode(tmp, bb, k2, C.run_key, C.run_cnt, C.counts, nent, s));
    int nr = 0;
    RPBA_CUDA_CHECK(cudaMemcpyAsync(&nr, C.counts, sizeof(int), cudaMemcpyDeviceToHost, s));
    RPBA_CUDA_CHECK(cudaStreamSynchronize(s));
    // the entries whose column lies outside the coarse space sort last
    unsigned lastkey = 0;
    if (nr > 0)
      RPBA_CUDA_CHECK(cudaMemcpy(&lastkey, C.run_key + nr - 1, sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (nr > 0 && lastkey == 0xffffffffu) --nr;
    RPBA_CUDA_CHECK(cudaMemsetAsync(C.run_cnt + nr, 0, sizeof(int), s));
    bb = C.cub_tmp_cap;
    RPBA_CUDA_CHECK(cub::DeviceScan::ExclusiveSum(tmp, bb, C.run_cnt, C.run_off, nr + 1, s));
    C.nruns = nr;
    // coarse blocks
    unsigned *q1 = grow(C.rkey, C.rkey_cap, (size_t)nr), *q2 = grow(C.rkey2, C.rkey2_cap, (size_t)nr);
    int *w1 = grow(C.ridx, C.ridx_cap, (size_t)nr);
    grow(C.run_sorted, C.run_sorted_cap, (size_t)nr);
    grow(C.seg_key, C.seg_key_cap, (size_t)nr);
    grow(C.seg_cnt, C.seg_cnt_cap, (size_t)nr + 1);
    grow(C.seg_off, C.seg_off_cap, (size_t)nr + 1);
    grow(C.Z, C.Z_cap, (size_t)std::max(nr, 1) * CO_M * CO_M);
    if (nr > 0) {
      k_run_keys2<<<(nr + 255) / 256, 256, 0, s>>>(C, nr, q1, w1);
      need = 0;
      cub::DeviceRadixSort::SortPairs(nullptr, b1, q1, q2, w1, C.run_sorted, nr, 0, 32, s);
      need = std::max(need, b1);
      cub::DeviceRunLengthEncode::Encode(nullptr, b1, q2, C.seg_key, C.seg_cnt, C.counts + 1, nr, s);
      need = std::max(need, b1);
      cub::DeviceScan::ExclusiveSum(nullptr, b1, C.seg_cnt, C.seg_off, nr + 1, s);
      need = std::max(need, b1);
      tmp = grow(C.cub_tmp, C.cub_tmp_cap, need);
      bb = C.cub_tmp_cap;
      RPBA_CUDA_CHECK(cub::DeviceRadixSort::SortPairs(tmp, bb, q1, q2, w1, C.run_sorted, nr, 0, 32, s));
      bb = C.cub_tmp_cap;
      RPBA_CUDA_CHECK(cub::DeviceRunLengthEncode::Encode(tmp, bb, q2, C.seg_key, C.seg_cnt, C.counts + 1, nr, s));
      int ns = 0;
      RPBA_CUDA_CHECK(cudaMemcpyAsync(&ns, C.counts + 1, sizeof(int), cudaMemcpyDeviceToHost, s));
      RPBA_CUDA_CHECK(cudaStreamSynchronize(s));
      RPBA_CUDA_CHECK(cudaMemsetAsync(C.seg_cnt + ns, 0, sizeof(int), s));
      bb = C.cub_tmp_cap;
      RPBA_CUDA_CHECK(cub::DeviceScan::ExclusiveSum(tmp, bb, C.seg_cnt, C.seg_off, ns + 1, s));
      C.nsegs = ns;
    } else {
      C.nsegs = 0;
    }
    C.built_version = structure_version;
  }
  const size_t nn = (size_t)C.nc * C.nc;
  RPBA_CUDA_CHECK(cudaMemsetAsync(C.Ac, 0, sizeof(double) * nn, s));
  if (C.nruns > 0) {
    k_coarse_runs<<<(C.nruns + RS_T / 32 - 1) / (RS_T / 32), RS_T, 0, s>>>(L, C, C.nruns);
    k_coarse_blocks<<<(C.nsegs + 7) / 8, 256, 0, s>>>(C, C.nsegs);
  }
  k_coarse_fixdiag<<<(C.nc + 255) / 256, 256, 0, s>>>(C);
  RPBA_CUDA_CHECK(cudaGetLastError());
}

void coarse_factor(CoarseWork &C, cudaStream_t s) {
  if (C.nagg <= 0) return;
  // Jacobi scaling, then the scaled matrix plus 1e-6 on its diagonal is
  // factored and inverted in one launch, and the inverse scaled back
  k_coarse_diag<<<(C.nc + 255) / 256, 256, 0, s>>>(C);
  spd_inverse_scaled(C.Ac, C.dsc, 1e-6, C.nc, C.Ainv, C.work, C.bar, C.err, s);
  RPBA_CUDA_CHECK(cudaGetLastError());
}

void coarse_setup(const DevLSA &L, CoarseWork &C, int structure_version, cudaStream_t s) {
  coarse_assemble(L, C, structure_version, s);
  coarse_factor(C, s);
}

void coarse_release(CoarseWork &C) {
  for (void *p : {(void *)C.ekey, (void *)C.ekey2, (void *)C.eval, (void *)C.ent_sorted, (void *)C.run_key,
                  (void *)C.run_cnt, (void *)C.run_off, (void *)C.counts, (void *)C.rkey, (void *)C.rkey2,
                  (void *)C.ridx, (void *)C.run_sorted, (void *)C.seg_key, (void *)C.seg_cnt, (void *)C.seg_off,
                  (void *)C.Z, (void *)C.cub_tmp})
    if (p) cudaFree(p);
  C = CoarseWork{};
}

void coarse_apply(const DevLSA &L, const CoarseWork &C, const double *r, double *h, cudaStream_t s) {
  (void)L;
  if (C.nagg <= 0) return;
  k_coarse_restrict<<<C.nagg, 32, 0, s>>>(C, r);
  k_coarse_prolong<<<C.nagg, PR_T, 0, s>>>(C, h);
}

}  // namespace rpba
