// direct.cu -- dense FP64 Cholesky solve of the reduced camera system (the
// plain direct form; the reference itself only runs PCG, rbacore.cpp:1176).
//
// The system (camera blocks k >= begini, sizes np_k, compact offsets) is
// expanded into a dense row-major n x n lower triangle, factored L L^T by a
// right-looking blocked algorithm with T x T tiles:
//   potrf   one CTA factors the diagonal tile in shared memory and writes
//           L_jj^-1 (also a lower triangle)
//   trsm    every tile below it: A_ij <- A_ij L_jj^-T (a T x T x T product)
//   syrk    trailing lower triangle: A_ik -= A_ij A_kj^T
// then solved by blocked forward and back substitution.  A non-positive
// pivot sets an error bit; the host reports RPBA_ERR_SOLVER.
#include "internal.h"

namespace rpba {

namespace {

constexpr int T = 64;
constexpr int DT = 256;

// diagonal blocks into the dense lower triangle
__global__ void k_dense_fill(DevLSA L, const int *coff, int n, double *A) {
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int r = (int)(gid / 81) + L.begini;
  if (r >= L.nimg) return;
  const int e = (int)(gid % 81);
  const int nr = L.camparv[r + 1] - L.camparv[r];
  const int i = e / 9, j = e % 9;
  if (i >= nr || j > i) return;
  A[(size_t)(coff[r] + i) * n + coff[r] + j] = blk_at(L, (size_t)r, e);
}

// off-diagonal blocks through the row entries: row r, column c > r,
// block (r, c) stored row major (r params x c params); the dense lower
// triangle gets its transpose at (c, r)
__global__ void k_dense_fill_off(DevLSA L, const int *coff, int n, double *A) {
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int row = (int)(gid / 81) + L.begini;
  if (row >= L.nimg) return;
  const int e = (int)(gid % 81);
  const int i = e / 9, j = e % 9;
  const int nr = L.camparv[row + 1] - L.camparv[row];
  if (i >= nr) return;
  for (int t = L.rowoff[row]; t < L.rowoff[row + 1]; ++t) {
    const int2 en = L.ent[t];
    if (en.y < 0 || en.x <= row) continue;  // normal entries right of the diagonal
    const int col = en.x;
    const int nc = L.camparv[col + 1] - L.camparv[col];
    if (j >= nc) continue;
    A[(size_t)(coff[col] + j) * n + coff[row] + i] = blk_at(L, (size_t)en.y, i * 9 + j);
  }
}

__global__ void k_gather_rhs(DevLSA L, const int *coff, double *y) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x + L.begini;
  if (k >= L.nimg) return;
  const int np = L.camparv[k + 1] - L.camparv[k];
  for (int a = 0; a < np; ++a) y[coff[k] + a] = L.rhs[(size_t)k * 9 + a];
}

__global__ void k_gather_vec(DevLSA L, const int *coff, const double *b, double *y) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x + L.begini;
  if (k >= L.nimg) return;
  const int np = L.camparv[k + 1] - L.camparv[k];
  for (int a = 0; a < np; ++a) y[coff[k] + a] = b[(size_t)k * 9 + a];
}

__global__ void k_scatter_solution(DevLSA L, const int *coff, const double *y, double *xsol) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= L.nimg) return;
  for (int a = 0; a < 9; ++a) {
    const int np = L.camparv[k + 1] - L.camparv[k];
    xsol[(size_t)k * 9 + a] = (k >= L.begini && a < np) ? y[coff[k] + a] : 0.;
  }
}

// Factor the diagonal tile at j0 (size tb <= T) in shared memory; writes
// L back into A and L^-1 into Linv (T x T, row major).
constexpr int SMEM2 = 2 * T * (T + 1) * sizeof(double);  // two padded tiles (66.5 KB)

__global__ void __launch_bounds__(DT) k_potrf(double *A, int n, int j0, int tb, double *Linv, int *err) {
  extern __shared__ double dyn[];
  double(*s)[T + 1] = reinterpret_cast<double(*)[T + 1]>(dyn);
  double(*inv)[T + 1] = reinterpret_cast<double(*)[T + 1]>(dyn + T * (T + 1));
  const int tid = threadIdx.x;
  for (int idx = tid; idx < T * T; idx += DT) {
    const int i = idx / T, j = idx % T;
    s[i][j] = (i < tb && j <= i) ? A[(size_t)(j0 + i) * n + j0 + j] : (i == j ? 1. : 0.);
  }
  __syncthreads();
  for (int k = 0; k < tb; ++k) {
    if (tid == 0) {
      const double d = s[k][k];
      if (!(d > 0.)) atomicOr(err, 4);
      s[k][k] = sqrt(d > 0. ? d : 1.);
    }
    __syncthreads();
    const double dk = s[k][k];
    for (int i = k + 1 + tid; i < tb; i += DT) s[i][k] /= dk;
    __syncthreads();
    for (int idx = tid; idx < (tb - k - 1) * (tb - k - 1); idx += DT) {
      const int i = k + 1 + idx / (tb - k - 1), j = k + 1 + idx % (tb - k - 1);
      if (j <= i) s[i][j] -= s[i][k] * s[j][k];
    }
    __syncthreads();
  }
  // L^-1 by forward substitution, one column per thread
  for (int c = tid; c < T; c += DT) {
    for (int i = 0; i < T; ++i) {
      double v = (i == c) ? 1. : 0.;
      for (int m = c; m < i; ++m) v -= s[i][m] * inv[m][c];
      inv[i][c] = (i >= c) ? v / s[i][i] : 0.;
    }
  }
  __syncthreads();
  for (int idx = tid; idx < T * T; idx += DT) {
    const int i = idx / T, j = idx % T;
    if (i < tb && j <= i) A[(size_t)(j0 + i) * n + j0 + j] = s[i][j];
    Linv[idx] = inv[i][j];
  }
}

// Tiles below the diagonal tile: A_ij <- A_ij L^-T.  One CTA per tile row
// (rows r0 .. r0 + T of the panel).
__global__ void __launch_bounds__(DT) k_trsm(double *A, int n, int j0, int tb, const double *Linv) {
  extern __shared__ double dyn[];
  double(*a)[T + 1] = reinterpret_cast<double(*)[T + 1]>(dyn);
  double(*li)[T + 1] = reinterpret_cast<double(*)[T + 1]>(dyn + T * (T + 1));
  const int r0 = j0 + tb + blockIdx.x * T;
  const int rb = min(T, n - r0);
  const int tid = threadIdx.x;
  for (int idx = tid; idx < T * T; idx += DT) {
    const int i = idx / T, j = idx % T;
    a[i][j] = (i < rb && j < tb) ? A[(size_t)(r0 + i) * n + j0 + j] : 0.;
    li[i][j] = Linv[idx];
  }
  __syncthreads();
  // out[i][j] = sum_m a[i][m] * li[j][m]  (L^-T), 4 x 4 outputs per thread
  const int ti = (tid / 16) * 4, tj = (tid % 16) * 4;
  double o[4][4] = {};
  for (int m = 0; m < tb; ++m) {
    double av[4], bv[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      av[u] = a[ti + u][m];
      bv[u] = li[tj + u][m];
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int v = 0; v < 4; ++v) o[u][v] += av[u] * bv[v];
  }
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v)
      if (ti + u < rb && tj + v < tb) A[(size_t)(r0 + ti + u) * n + j0 + tj + v] = o[u][v];
}

// Trailing update of the lower triangle: tile (bi, bk), bk <= bi, of the
// rows/columns after the panel: A_ik -= P_i P_k^T.
__global__ void __launch_bounds__(DT) k_syrk(double *A, int n, int j0, int tb, int m) {
  // blockIdx.x enumerates the m (m + 1) / 2 lower tiles
  const int t = blockIdx.x;
  int bi = (int)((sqrt(8. * t + 1.) - 1.) / 2.);
  while ((bi + 1) * (bi + 2) / 2 <= t) ++bi;
  while (bi * (bi + 1) / 2 > t) --bi;
  const int bk = t - bi * (bi + 1) / 2;
  const int base = j0 + tb;
  const int ri = base + bi * T, rk = base + bk * T;
  const int nbi = min(T, n - ri), nbk = min(T, n - rk);
  extern __shared__ double dyn[];
  double(*pi)[T + 1] = reinterpret_cast<double(*)[T + 1]>(dyn);
  double(*pk)[T + 1] = reinterpret_cast<double(*)[T + 1]>(dyn + T * (T + 1));
  const int tid = threadIdx.x;
  for (int idx = tid; idx < T * T; idx += DT) {
    const int i = idx / T, j = idx % T;
    pi[i][j] = (i < nbi && j < tb) ? A[(size_t)(ri + i) * n + j0 + j] : 0.;
    pk[i][j] = (i < nbk && j < tb) ? A[(size_t)(rk + i) * n + j0 + j] : 0.;
  }
  __syncthreads();
  const int ti = (tid / 16) * 4, tj = (tid % 16) * 4;
  double o[4][4] = {};
  for (int mm = 0; mm < tb; ++mm) {
    double av[4], bv[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      av[u] = pi[ti + u][mm];
      bv[u] = pk[tj + u][mm];
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int v = 0; v < 4; ++v) o[u][v] += av[u] * bv[v];
  }
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int gi = ri + ti + u, gk = rk + tj + v;
      if (ti + u < nbi && tj + v < nbk && gk <= gi) A[(size_t)gi * n + gk] -= o[u][v];
    }
}

// Forward substitution on a tile: y_j <- L_jj^-1 y_j (single CTA).
__global__ void k_tile_solve(const double *Linv, int tb, double *y, int j0, int transpose) {
  __shared__ double v[T];
  const int tid = threadIdx.x;
  if (tid < T) v[tid] = tid < tb ? y[j0 + tid] : 0.;
  __syncthreads();
  if (tid < tb) {
    double s = 0.;
    if (!transpose)
      for (int m = 0; m <= tid; ++m) s += Linv[tid * T + m] * v[m];
    else
      for (int m = tid; m < tb; ++m) s += Linv[m * T + tid] * v[m];
    y[j0 + tid] = s;
  }
}

// y[i] -= sum_{m in panel} L[i][j0 + m] y[j0 + m] for rows i >= j0 + tb
// (forward) ; y[i] -= sum_{m in panel} L[j0 + m][i] y[j0 + m] for i < j0
// (backward).  One warp per row.
__global__ void k_panel_update(const double *A, int n, int j0, int tb, double *y, int backward) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  const int i = backward ? warp : j0 + tb + warp;
  if ((backward && i >= j0) || (!backward && i >= n)) return;
  double s = 0.;
  for (int m = lane; m < tb; m += 32)
    s += (backward ? A[(size_t)(j0 + m) * n + i] : A[(size_t)i * n + j0 + m]) * y[j0 + m];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) y[i] -= s;
}


// Tile row it of X = L^-1: CTA j < it forms X_ij = -Linv_i sum_{j<=m<i}
// L_im X_mj (tile rows < it are complete); CTA j == it copies Linv_i.
__global__ void __launch_bounds__(DT) k_inv_row(const double *A, int n, const double *Linv, double *X, int it) {
  extern __shared__ double dyn[];
  double(*a)[T + 1] = reinterpret_cast<double(*)[T + 1]>(dyn);
  double(*b)[T + 1] = reinterpret_cast<double(*)[T + 1]>(dyn + T * (T + 1));
  const int jt = blockIdx.x, tid = threadIdx.x;
  const int i0 = it * T, ib = min(T, n - i0), j0 = jt * T, jb = min(T, n - j0);
  const double *Li = Linv + (size_t)it * T * T;
  if (jt == it) {
    for (int idx = tid; idx < T * T; idx += DT) {
      const int i = idx / T, j = idx % T;
      if (i < ib && j < jb) X[(size_t)(i0 + i) * n + j0 + j] = Li[idx];
    }
    return;
  }
  const int ti = (tid / 16) * 4, tj = (tid % 16) * 4;
  double o[4][4] = {};
  for (int mt = jt; mt < it; ++mt) {
    const int m0 = mt * T, mb = min(T, n - m0);
    __syncthreads();
    for (int idx = tid; idx < T * T; idx += DT) {
      const int i = idx / T, j = idx % T;
      a[i][j] = (i < ib && j < mb) ? A[(size_t)(i0 + i) * n + m0 + j] : 0.;    // L_im
      b[i][j] = (i < mb && j < jb) ? X[(size_t)(m0 + i) * n + j0 + j] : 0.;    // X_mj
    }
    __syncthreads();
    for (int m = 0; m < mb; ++m) {
      double av[4], bv[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        av[u] = a[ti + u][m];
        bv[u] = b[m][tj + u];
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) o[u][v] += av[u] * bv[v];
    }
  }
  __syncthreads();
  // Y -> shared b, then X_ij = -Linv_i Y
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v) b[ti + u][tj + v] = o[u][v];
  for (int idx = tid; idx < T * T; idx += DT) a[idx / T][idx % T] = Li[idx];
  __syncthreads();
  double y[4][4] = {};
  for (int m = 0; m < ib; ++m) {
    double av[4], bv[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      av[u] = a[ti + u][m];
      bv[u] = b[m][tj + u];
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int v = 0; v < 4; ++v) y[u][v] += av[u] * bv[v];
  }
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v)
      if (ti + u < ib && tj + v < jb) X[(size_t)(i0 + ti + u) * n + j0 + tj + v] = -y[u][v];
}

// A^-1 = X^T X for tile (bi, bk), bk <= bi: sum over tile rows m >= bi of
// X_m,bi^T X_m,bk; written to both triangles.
__global__ void __launch_bounds__(DT) k_xtx(const double *X, int n, double *Ainv) {
  const int t = blockIdx.x;
  int bi = (int)((sqrt(8. * t + 1.) - 1.) / 2.);
  while ((bi + 1) * (bi + 2) / 2 <= t) ++bi;
  while (bi * (bi + 1) / 2 > t) --bi;
  const int bk = t - bi * (bi + 1) / 2;
  const int ri = bi * T, rk = bk * T, nbi = min(T, n - ri), nbk = min(T, n - rk);
  extern __shared__ double dyn[];
  double(*pi)[T + 1] = reinterpret_cast<double(*)[T + 1]>(dyn);
  double(*pk)[T + 1] = reinterpret_cast<double(*)[T + 1]>(dyn + T * (T + 1));
  const int tid = threadIdx.x, ti = (tid / 16) * 4, tj = (tid % 16) * 4;
  const int ntiles = (n + T - 1) / T;
  double o[4][4] = {};
  for (int mt = bi; mt < ntiles; ++mt) {
    const int m0 = mt * T, mb = min(T, n - m0);
    __syncthreads();
    for (int idx = tid; idx < T * T; idx += DT) {
      const int m = idx / T, j = idx % T;
      pi[m][j] = (m < mb && j < nbi) ? X[(size_t)(m0 + m) * n + ri + j] : 0.;
      pk[m][j] = (m < mb && j < nbk) ? X[(size_t)(m0 + m) * n + rk + j] : 0.;
    }
    __syncthreads();
    for (int m = 0; m < mb; ++m) {
      double av[4], bv[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        av[u] = pi[m][ti + u];
        bv[u] = pk[m][tj + u];
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) o[u][v] += av[u] * bv[v];
    }
  }
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v)
      if (ti + u < nbi && tj + v < nbk) {
        Ainv[(size_t)(ri + ti + u) * n + rk + tj + v] = o[u][v];
        Ainv[(size_t)(rk + tj + v) * n + ri + ti + u] = o[u][v];
      }
}

}  // namespace

size_t direct_bytes(int n) { return (size_t)n * n * sizeof(double); }

// Factor a dense SPD matrix in place: the lower triangle of A (row major,
// n x n) becomes L with A = L L^T; Linv receives the inverses of L's
// diagonal T x T tiles.  A non-positive pivot sets bit 4 of *err.
void dense_cholesky(double *A, int n, double *Linv, int *err, cudaStream_t s) {
  if (n <= 0) return;
  RPBA_CUDA_CHECK(cudaFuncSetAttribute(k_potrf, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM2));
  RPBA_CUDA_CHECK(cudaFuncSetAttribute(k_trsm, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM2));
  RPBA_CUDA_CHECK(cudaFuncSetAttribute(k_syrk, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM2));
  const int ntiles = (n + T - 1) / T;
  for (int jt = 0; jt < ntiles; ++jt) {
    const int j0 = jt * T, tb = min(T, n - j0);
    k_potrf<<<1, DT, SMEM2, s>>>(A, n, j0, tb, Linv + (size_t)jt * T * T, err);
    const int rows_below = n - j0 - tb;
    if (rows_below > 0) {
      const int m = (rows_below + T - 1) / T;
      k_trsm<<<m, DT, SMEM2, s>>>(A, n, j0, tb, Linv + (size_t)jt * T * T);
      k_syrk<<<m * (m + 1) / 2, DT, SMEM2, s>>>(A, n, j0, tb, m);
    }
  }
}

// Explicit inverse from the factor: X = L^-1 tile row by tile row
// (X_ij = -L_ii^-1 sum_{j <= m < i} L_im X_mj), then A^-1 = X^T X, both
// triangles written.  X and Ainv are n x n row major.
void dense_spd_inverse(const double *A, int n, const double *Linv, double *X, double *Ainv, cudaStream_t s) {
  if (n <= 0) return;
  RPBA_CUDA_CHECK(cudaFuncSetAttribute(k_inv_row, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM2));
  RPBA_CUDA_CHECK(cudaFuncSetAttribute(k_xtx, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM2));
  const int ntiles = (n + T - 1) / T;
  for (int it = 0; it < ntiles; ++it) k_inv_row<<<it + 1, DT, SMEM2, s>>>(A, n, Linv, X, it);
  k_xtx<<<ntiles * (ntiles + 1) / 2, DT, SMEM2, s>>>(X, n, Ainv);
}

// Factor S = L L^T (kept in W.A / W.Linv) and solve S x = b for the
// reduced camera system; x in xsol (padded 9 per camera).  A non-positive
// pivot sets L.err bit 4.
void direct_factor(const DevLSA &L, const DirectWork &W, cudaStream_t s) {
  const int n = W.n;
  if (n <= 0) return;
  RPBA_CUDA_CHECK(cudaMemsetAsync(W.A, 0, (size_t)n * n * sizeof(double), s));
  const long long nd = (long long)(L.nimg - L.begini) * 81;
  if (nd > 0) {
    k_dense_fill<<<(int)((nd + 255) / 256), 256, 0, s>>>(L, W.coff, n, W.A);
    k_dense_fill_off<<<(int)((nd + 255) / 256), 256, 0, s>>>(L, W.coff, n, W.A);
  }
  dense_cholesky(W.A, n, W.Linv, L.err, s);
}

// x = S^-1 b with the factor from direct_factor; b and x padded 9 per camera
// (b == nullptr: the assembled right-hand side L.rhs).
void direct_resolve(const DevLSA &L, const DirectWork &W, const double *b, double *xsol, cudaStream_t s) {
  const int n = W.n;
  if (n <= 0) return;
  if (b)
    k_gather_vec<<<(L.nimg + 127) / 128, 128, 0, s>>>(L, W.coff, b, W.y);
  else
    k_gather_rhs<<<(L.nimg + 127) / 128, 128, 0, s>>>(L, W.coff, W.y);
  const int ntiles = (n + T - 1) / T;
  for (int jt = 0; jt < ntiles; ++jt) {
    const int j0 = jt * T, tb = min(T, n - j0);
    k_tile_solve<<<1, T, 0, s>>>(W.Linv + (size_t)jt * T * T, tb, W.y, j0, 0);
    const int rows = n - j0 - tb;
    if (rows > 0) k_panel_update<<<(rows * 32 + 255) / 256, 256, 0, s>>>(W.A, n, j0, tb, W.y, 0);
  }
  for (int jt = ntiles - 1; jt >= 0; --jt) {
    const int j0 = jt * T, tb = min(T, n - j0);
    k_tile_solve<<<1, T, 0, s>>>(W.Linv + (size_t)jt * T * T, tb, W.y, j0, 1);
    if (j0 > 0) k_panel_update<<<(j0 * 32 + 255) / 256, 256, 0, s>>>(W.A, n, j0, tb, W.y, 1);
  }
  k_scatter_solution<<<(L.nimg + 127) / 128, 128, 0, s>>>(L, W.coff, W.y, xsol);
}

void direct_solve(const DevLSA &L, const DirectWork &W, double *xsol, cudaStream_t s) {
  direct_factor(L, W, s);
  direct_resolve(L, W, nullptr, xsol, s);
}

}  // namespace rpba
