// direct.cu -- sparse direct Cholesky solve of the reduced camera system (the
// plain direct form; the reference itself only runs PCG, rbacore.cpp:1176).
//
// Symbolic part (host, once per structure): the cameras of the system are
// ordered by reverse Cuthill-McKee on their covisibility graph, which keeps
// the nonzeros near the diagonal on chain-like (street) and grid-like
// (aerial) scenes.  In that order the unknowns' envelope -- for every row
// the first column any covisible camera reaches -- holds the Cholesky factor
// exactly (a factor has no fill outside the envelope of its matrix).  The
// envelope is kept at 64 x 64 tile granularity, its left edge made
// nondecreasing (rows with a longer reach widen the rows above them).
//
// Numeric part (device, per linear system): the blocks are scattered into
// the envelope tiles, the tiles factored in one cooperative launch
// (chol.cu: right-looking, tile products on the FP64 tensor cores), and the
// system solved by forward and back substitution over the tiles in one more
// cooperative launch (one grid barrier per tile row and direction).  A
// non-positive pivot sets bit 4 of the error word (RPBA_ERR_SOLVER).
#include <algorithm>
#include <numeric>
#include <vector>

#include "gridsync.cuh"
#include "internal.h"

namespace rpba {

namespace {

constexpr int T = 64;
constexpr int TS = T * T;
constexpr int ST = 256;  // threads per CTA of the solve

__global__ void k_env_diag_pad(double *tiles, const long long *toff, const int *fcol, int nt, int n) {
  const int r = n + blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nt * T) return;
  const int I = r / T, a = r % T;
  tiles[(size_t)(toff[I] + (I - fcol[I])) * TS + a * T + a] = 1.;
}

__device__ __forceinline__ void env_put(double *tiles, const long long *toff, const int *fcol, int R, int C,
                                        double v) {
  if (C > R) {
    const int t = R;
    R = C;
    C = t;
  }
  const int I = R / T, J = C / T;
  tiles[(size_t)(toff[I] + (J - fcol[I])) * TS + (R % T) * T + (C % T)] = v;
}

// diagonal blocks: entries on and below the diagonal (as assembled)
__global__ void k_env_fill_diag(DevLSA L, const int *pos, double *tiles, const long long *toff, const int *fcol) {
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int r = (int)(gid / 81) + L.begini;
  if (r >= L.nimg) return;
  const int e = (int)(gid % 81), i = e / 9, j = e % 9;
  const int nr = L.camparv[r + 1] - L.camparv[r];
  if (i >= nr || j > i) return;
  env_put(tiles, toff, fcol, pos[r] + i, pos[r] + j, blk_at(L, (size_t)r, e));
}

// off-diagonal blocks (row r, column c > r, stored r params x c params)
__global__ void k_env_fill_off(DevLSA L, const unsigned *bkey, const int *pos, double *tiles, const long long *toff,
                               const int *fcol) {
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long b = gid / 81;
  if (b >= L.nboff) return;
  const int e = (int)(gid % 81), i = e / 9, j = e % 9;
  const unsigned key = bkey[b];
  const int r = (int)(key / (unsigned)L.nimg), c = (int)(key % (unsigned)L.nimg);
  const int nr = L.camparv[r + 1] - L.camparv[r], nc = L.camparv[c + 1] - L.camparv[c];
  if (i >= nr || j >= nc) return;
  env_put(tiles, toff, fcol, pos[r] + i, pos[c] + j, blk_at(L, (size_t)L.nimg + b, e));
}

__global__ void k_env_gather(DevLSA L, const int *pos, const double *b, double *y) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x + L.begini;
  if (k >= L.nimg) return;
  const int np = L.camparv[k + 1] - L.camparv[k];
  const double *src = b ? b + (size_t)k * 9 : L.rhs + (size_t)k * 9;
  for (int a = 0; a < np; ++a) y[pos[k] + a] = src[a];
}

__global__ void k_env_scatter(DevLSA L, const int *pos, const double *y, double *xsol) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= L.nimg) return;
  const int np = L.camparv[k + 1] - L.camparv[k];
  for (int a = 0; a < 9; ++a) xsol[(size_t)k * 9 + a] = (k >= L.begini && a < np) ? y[pos[k] + a] : 0.;
}

struct SolveArgs {
  const double *tiles, *Linv;
  const long long *toff;
  const int *fcol, *hrow;
  double *y;
  int nt;
  unsigned *bar;
  int *err;
  unsigned long long bar_ns;
};

__device__ __forceinline__ const double *etile(const SolveArgs &A, int I, int J) {
  return A.tiles + (size_t)(A.toff[I] + (J - A.fcol[I])) * TS;
}

// y_I -= M y_J (trans = 0) or y_I -= M^T y_J (trans = 1) for a 64 x 64 tile M
__device__ void tile_gemv_sub(const double *M, const double *yj, double *yi, bool trans, double *sv, double *sp) {
  const int t = threadIdx.x;
  __syncthreads();
  if (t < T) sv[t] = __ldcg(yj + t);
  __syncthreads();
  if (!trans) {
    // row r = t / 4, columns 16 (t % 4) .. + 16
    const int r = t >> 2, c0 = (t & 3) * 16;
    double s = 0.;
#pragma unroll
    for (int c = 0; c < 16; ++c) s += __ldcg(M + r * T + c0 + c) * sv[c0 + c];
    s += __shfl_xor_sync(0xffffffffu, s, 1);
    s += __shfl_xor_sync(0xffffffffu, s, 2);
    if ((t & 3) == 0) yi[r] = __ldcg(yi + r) - s;
  } else {
    // column c = t % 64, rows 16 (t / 64) .. + 16
    const int c = t & 63, r0 = (t >> 6) * 16;
    double s = 0.;
#pragma unroll
    for (int r = 0; r < 16; ++r) s += __ldcg(M + (r0 + r) * T + c) * sv[r0 + r];
    sp[t] = s;
    __syncthreads();
    if (t < T) yi[t] = __ldcg(yi + t) - ((sp[t] + sp[t + 64]) + (sp[t + 128] + sp[t + 192]));
  }
  __syncthreads();
}

// y_J = Linv_J y_J (trans = 0) or Linv_J^T y_J (trans = 1)
__device__ void tile_gemv_set(const double *Li, double *yj, bool trans, double *sv, double *sp) {
  const int t = threadIdx.x;
  __syncthreads();
  if (t < T) sv[t] = __ldcg(yj + t);
  __syncthreads();
  const int c = t & 63, q = t >> 6;
  double s = 0.;
  if (!trans) {
    // output row c, columns 16 q .. + 16
#pragma unroll
    for (int m = 0; m < 16; ++m) s += __ldcg(Li + c * T + 16 * q + m) * sv[16 * q + m];
  } else {
    // output column c: sum over rows 16 q .. + 16
#pragma unroll
    for (int m = 0; m < 16; ++m) s += __ldcg(Li + (16 * q + m) * T + c) * sv[16 * q + m];
  }
  sp[t] = s;
  __syncthreads();
  if (t < T) yj[t] = (sp[t] + sp[t + 64]) + (sp[t + 128] + sp[t + 192]);
  __syncthreads();
}

// Forward then back substitution over the envelope tiles.  A tile row's
// diagonal solve is done by the CTA that applies the row's last update, so
// every step costs one grid barrier.
__global__ void __launch_bounds__(ST) k_env_solve(SolveArgs A) {
  __shared__ double sv[T], sp[ST];
  const int G = gridDim.x, nt = A.nt;
  // forward: L y = b
  if (blockIdx.x == 0) tile_gemv_set(A.Linv, A.y, false, sv, sp);
  if (!grid_barrier(A.bar, G, A.err, A.bar_ns)) return;
  for (int J = 0; J < nt - 1; ++J) {
    const int m = A.hrow[J] - J;
    for (int t = blockIdx.x; t < m; t += G) {
      const int I = J + 1 + t;
      tile_gemv_sub(etile(A, I, J), A.y + (size_t)J * T, A.y + (size_t)I * T, false, sv, sp);
      if (t == 0) tile_gemv_set(A.Linv + (size_t)I * TS, A.y + (size_t)I * T, false, sv, sp);
    }
    if (m == 0 && blockIdx.x == (J + 1) % G)
      tile_gemv_set(A.Linv + (size_t)(J + 1) * TS, A.y + (size_t)(J + 1) * T, false, sv, sp);
    if (!grid_barrier(A.bar, G, A.err, A.bar_ns)) return;
  }
  // backward: L^T x = y
  if (blockIdx.x == 0) tile_gemv_set(A.Linv + (size_t)(nt - 1) * TS, A.y + (size_t)(nt - 1) * T, true, sv, sp);
  if (!grid_barrier(A.bar, G, A.err, A.bar_ns)) return;
  for (int J = nt - 1; J > 0; --J) {
    const int m = J - A.fcol[J];
    for (int t = blockIdx.x; t < m; t += G) {
      const int K = J - 1 - t;
      tile_gemv_sub(etile(A, J, K), A.y + (size_t)J * T, A.y + (size_t)K * T, true, sv, sp);
      if (t == 0) tile_gemv_set(A.Linv + (size_t)K * TS, A.y + (size_t)K * T, true, sv, sp);
    }
    if (m == 0 && blockIdx.x == (J - 1) % G)
      tile_gemv_set(A.Linv + (size_t)(J - 1) * TS, A.y + (size_t)(J - 1) * T, true, sv, sp);
    if (!grid_barrier(A.bar, G, A.err, A.bar_ns)) return;
  }
}

// Reverse Cuthill-McKee order of the vertices of a graph (CSR, neighbours
// of every vertex), every component from a pseudo-peripheral vertex.
std::vector<int> rcm_order(int n, const std::vector<int> &off, const std::vector<int> &adj) {
  std::vector<int> deg(n), order;
  order.reserve(n);
  for (int v = 0; v < n; ++v) deg[v] = off[v + 1] - off[v];
  std::vector<char> seen(n, 0);
  std::vector<int> lvl(n, -1), q;
  auto bfs_last = [&](int s, int &ecc) {
    // level structure from s: a vertex of least degree in the last level
    q.assign(1, s);
    lvl[s] = 0;
    for (size_t h = 0; h < q.size(); ++h) {
      const int v = q[h];
      for (int e = off[v]; e < off[v + 1]; ++e)
        if (lvl[adj[e]] < 0) {
          lvl[adj[e]] = lvl[v] + 1;
          q.push_back(adj[e]);
        }
    }
    ecc = lvl[q.back()];
    int best = q.back();
    for (int v : q)
      if (lvl[v] == ecc && (deg[v] < deg[best] || (deg[v] == deg[best] && v < best))) best = v;
    for (int v : q) lvl[v] = -1;
    return best;
  };
  std::vector<int> byd(n);
  std::iota(byd.begin(), byd.end(), 0);
  std::stable_sort(byd.begin(), byd.end(), [&](int a, int b) { return deg[a] < deg[b]; });
  std::vector<int> nb;
  for (int s0 : byd) {
    if (seen[s0]) continue;
    int s = s0, ecc = -1;
    for (int it = 0; it < 6; ++it) {
      int e2 = 0;
      const int c = bfs_last(s, e2);
      if (e2 <= ecc) break;
      ecc = e2;
      s = c;
    }
    const size_t base = order.size();
    order.push_back(s);
    seen[s] = 1;
    for (size_t h = base; h < order.size(); ++h) {
      const int v = order[h];
      nb.clear();
      for (int e = off[v]; e < off[v + 1]; ++e)
        if (!seen[adj[e]]) nb.push_back(adj[e]);
      std::sort(nb.begin(), nb.end(), [&](int a, int b) { return deg[a] < deg[b] || (deg[a] == deg[b] && a < b); });
      for (int w : nb) {
        seen[w] = 1;
        order.push_back(w);
      }
    }
  }
  std::reverse(order.begin(), order.end());
  return order;
}

int solve_grid() {
  int dev = 0, nsm = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_env_solve, ST, 0);
  return per >= 1 ? nsm : 0;
}

}  // namespace

// Ordering and envelope of the current structure (host); device buffers
// sized for it.  Returns false when the envelope's tiles exceed max_bytes.
bool direct_analyse(const DevLSA &L, const unsigned *d_bkey, const std::vector<int> &camparv, size_t max_bytes,
                    DirectWork &W, std::vector<void *> &owned, cudaStream_t s) {
  const int nimg = L.nimg, b0 = L.begini, nc = nimg - b0, nb = L.nboff;
  std::vector<unsigned> key(std::max(nb, 1));
  if (nb) RPBA_CUDA_CHECK(cudaMemcpyAsync(key.data(), d_bkey, sizeof(unsigned) * nb, cudaMemcpyDeviceToHost, s));
  RPBA_CUDA_CHECK(cudaStreamSynchronize(s));
  // covisibility graph of the system's cameras (local index k - begini)
  std::vector<int> off(nc + 1, 0), adj(2 * (size_t)nb);
  for (int b = 0; b < nb; ++b) {
    ++off[key[b] / nimg - b0 + 1];
    ++off[key[b] % nimg - b0 + 1];
  }
  for (int v = 0; v < nc; ++v) off[v + 1] += off[v];
  {
    std::vector<int> fill(off.begin(), off.end() - 1);
    for (int b = 0; b < nb; ++b) {
      const int r = (int)(key[b] / nimg) - b0, c = (int)(key[b] % nimg) - b0;
      adj[fill[r]++] = c;
      adj[fill[c]++] = r;
    }
  }
  const std::vector<int> order = rcm_order(nc, off, adj);
  // first unknown of every camera in the order
  std::vector<int> pos(nimg, 0);
  int n = 0;
  for (int v : order) {
    pos[v + b0] = n;
    n += camparv[v + b0 + 1] - camparv[v + b0];
  }
  const int nt = (n + T - 1) / T;
  // envelope: first column of every camera's rows, then per tile row
  std::vector<int> fc(std::max(nt, 1), 0);
  for (int I = 0; I < nt; ++I) fc[I] = I;
  for (int v = 0; v < nc; ++v) {
    int first = pos[v + b0];
    for (int e = off[v]; e < off[v + 1]; ++e) first = std::min(first, pos[adj[e] + b0]);
    const int np = camparv[v + b0 + 1] - camparv[v + b0];
    for (int a = 0; a < np; ++a) {
      const int I = (pos[v + b0] + a) / T;
      fc[I] = std::min(fc[I], first / T);
    }
  }
  for (int I = nt - 2; I >= 0; --I) fc[I] = std::min(fc[I], fc[I + 1]);
  std::vector<long long> toff(std::max(nt, 1), 0);
  long long ntiles = 0;
  for (int I = 0; I < nt; ++I) {
    toff[I] = ntiles;
    ntiles += I - fc[I] + 1;
  }
  std::vector<int> hrow(std::max(nt, 1), 0);
  for (int J = 0, I = 0; J < nt; ++J) {
    while (I + 1 < nt && fc[I + 1] <= J) ++I;
    hrow[J] = std::max(I, J);
  }
  const size_t bytes = (size_t)(ntiles + nt) * TS * sizeof(double);
  W.n = n;
  W.nt = nt;
  W.ntiles = ntiles;
  W.env_bytes = bytes;
  if (bytes > max_bytes) return false;
  auto dal = [&](size_t b) {
    void *p = nullptr;
    RPBA_CUDA_CHECK(cudaMalloc(&p, std::max<size_t>(b, 16)));
    owned.push_back(p);
    return p;
  };
  if ((size_t)ntiles > W.cap_tiles) {
    W.tiles = (double *)dal((size_t)ntiles * TS * sizeof(double));
    W.cap_tiles = (size_t)ntiles;
  }
  if (nt > W.cap_nt) {
    W.Linv = (double *)dal((size_t)nt * TS * sizeof(double));
    W.y = (double *)dal((size_t)nt * T * sizeof(double));
    W.toff = (long long *)dal(sizeof(long long) * nt);
    W.fcol = (int *)dal(sizeof(int) * nt);
    W.hrow = (int *)dal(sizeof(int) * nt);
    W.cap_nt = nt;
  }
  if (!W.pos) {
    W.pos = (int *)dal(sizeof(int) * nimg);
    W.bar = (unsigned *)dal(2 * sizeof(unsigned));
  }
  W.bkey = d_bkey;
  RPBA_CUDA_CHECK(cudaMemcpyAsync(W.pos, pos.data(), sizeof(int) * nimg, cudaMemcpyHostToDevice, s));
  if (nt) {
    RPBA_CUDA_CHECK(cudaMemcpyAsync(W.toff, toff.data(), sizeof(long long) * nt, cudaMemcpyHostToDevice, s));
    RPBA_CUDA_CHECK(cudaMemcpyAsync(W.fcol, fc.data(), sizeof(int) * nt, cudaMemcpyHostToDevice, s));
    RPBA_CUDA_CHECK(cudaMemcpyAsync(W.hrow, hrow.data(), sizeof(int) * nt, cudaMemcpyHostToDevice, s));
  }
  RPBA_CUDA_CHECK(cudaStreamSynchronize(s));  // the host vectors go out of scope
  return true;
}

// Factor the reduced camera system into the envelope tiles.
void direct_factor(const DevLSA &L, const DirectWork &W, cudaStream_t s) {
  if (W.n <= 0) return;
  RPBA_CUDA_CHECK(cudaMemsetAsync(W.tiles, 0, (size_t)W.ntiles * TS * sizeof(double), s));
  const int pad = W.nt * T - W.n;
  if (pad > 0) k_env_diag_pad<<<(pad + 127) / 128, 128, 0, s>>>(W.tiles, W.toff, W.fcol, W.nt, W.n);
  const long long nd = (long long)(L.nimg - L.begini) * 81;
  if (nd > 0) k_env_fill_diag<<<(int)((nd + 255) / 256), 256, 0, s>>>(L, W.pos, W.tiles, W.toff, W.fcol);
  const long long no = (long long)L.nboff * 81;
  if (no > 0) k_env_fill_off<<<(int)((no + 255) / 256), 256, 0, s>>>(L, W.bkey, W.pos, W.tiles, W.toff, W.fcol);
  tile_cholesky(W.tiles, W.toff, W.fcol, W.hrow, W.Linv, W.nt, W.bar, L.err, s);
}

// x = S^-1 b with the factor from direct_factor; b and x padded 9 per camera
// (b == nullptr: the assembled right-hand side L.rhs).
void direct_resolve(const DevLSA &L, const DirectWork &W, const double *b, double *xsol, cudaStream_t s) {
  if (W.n <= 0) return;
  const int pad = W.nt * T - W.n;
  if (pad > 0) RPBA_CUDA_CHECK(cudaMemsetAsync(W.y + W.n, 0, sizeof(double) * pad, s));
  k_env_gather<<<(L.nimg + 127) / 128, 128, 0, s>>>(L, W.pos, b, W.y);
  SolveArgs A;
  A.tiles = W.tiles;
  A.Linv = W.Linv;
  A.toff = W.toff;
  A.fcol = W.fcol;
  A.hrow = W.hrow;
  A.y = W.y;
  A.nt = W.nt;
  A.bar = W.bar;
  A.err = L.err;
  A.bar_ns = BAR_TIMEOUT_NS;
  const int g = std::max(1, std::min(solve_grid(), W.nt));
  RPBA_CUDA_CHECK(cudaMemsetAsync(W.bar, 0, 2 * sizeof(unsigned), s));
  void *args[] = {&A};
  RPBA_CUDA_CHECK(cudaLaunchCooperativeKernel((const void *)k_env_solve, dim3(g), dim3(ST), args, 0, s));
  k_env_scatter<<<(L.nimg + 127) / 128, 128, 0, s>>>(L, W.pos, W.y, xsol);
  RPBA_CUDA_CHECK(cudaGetLastError());
}

void direct_solve(const DevLSA &L, const DirectWork &W, double *xsol, cudaStream_t s) {
  direct_factor(L, W, s);
  direct_resolve(L, W, nullptr, xsol, s);
}

}  // namespace rpba
