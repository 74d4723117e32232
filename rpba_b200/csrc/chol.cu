// chol.cu -- tiled FP64 Cholesky factorisation of symmetric positive definite
// matrices held as 64 x 64 tiles, in one cooperative launch, with the tile
// products on the FP64 tensor cores (mma.sync m8n8k4 f64; sm_100a has no
// FP64 kind of tcgen05.mma).
//
// Storage: the lower triangle in tiles, row by row; tile row I holds the
// tiles of columns fcol[I] .. I, with fcol nondecreasing (an envelope: a
// dense matrix has fcol = 0).  A Cholesky factor keeps the envelope of its
// matrix, so L overwrites A in place.  hrow[J] is the last tile row whose
// envelope reaches column J.
//
// Right-looking, per tile column J:
//   P  the diagonal tile is factored (one warp, shared memory) and inverted:
//      L_JJ and L_JJ^-1 (Linv[J]);
//   T  every tile below it: L_IJ = A_IJ L_JJ^-T, a tile product;
//   U  the trailing tiles: A_IK -= L_IJ L_KJ^T for J < K <= I <= hrow[J].
// Phases are separated by bounded grid barriers; the tiles of a phase are
// dealt to the CTAs round robin.  The factorisation of tile J + 1 is done by
// the CTA that applies its last update (in phase U of column J), so P costs
// no barrier of its own.  A non-positive pivot sets bit 4 of the error word.
//
// For a dense matrix the same launch can go on to the inverse:
//   X  = L^-1, right-looking by tile rows: X_Ij = Linv_I R_Ij (j <= I), then
//        R_Kj -= L_KI X_Ij for K > I;
//   A^-1 = X^T X, one output tile per work item, both triangles written.
#include "gridsync.cuh"
#include "internal.h"

namespace rpba {

namespace {

constexpr int CT = 64;                  // tile edge
constexpr int CLD = 68;                 // shared leading dimension: conflict-free fragment loads
constexpr int CTH = 256;                // threads per CTA (8 warps)
constexpr int TS = CT * CT;             // doubles per stored tile
constexpr size_t CSMEM = (2 * CT * CLD + 4 * CT) * sizeof(double);  // two tiles + partials

struct Tiles {
  double *L;               // tile storage (row major inside a tile, ld 64)
  const long long *toff;   // [nt] first tile of row I
  const int *fcol;         // [nt] first tile column of row I
  const int *hrow;         // [nt] last tile row reaching column J
  double *Linv;            // [nt][TS] inverses of the diagonal tiles
  double *X;               // dense inverse only: [nt(nt+1)/2][TS] L^-1, lower tiles
  double *Ainv;            // dense inverse only: [nt(nt+1)/2][TS] A^-1, lower tiles
  int nt;
  int want_inverse;
  unsigned *bar;
  int *err;
  unsigned long long bar_ns;
};

__device__ __forceinline__ double *tile_at(const Tiles &T, int I, int J) {
  return T.L + (size_t)(T.toff[I] + (J - T.fcol[I])) * TS;
}
__device__ __forceinline__ size_t tri(int I, int J) { return (size_t)I * (I + 1) / 2 + J; }

// D (8x8, two per thread) += A (8x4, one per thread) * B (4x8, one per thread)
__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// acc (warp w: rows 8w .. 8w + 7, all 64 columns, 8 fragments of 2) +=
// sA sB^T over k = 0 .. 63; sA, sB in shared memory with ld CLD.
__device__ __forceinline__ void gemm_nt(const double *sA, const double *sB, double (&acc)[8][2]) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const double *pa = sA + (8 * w + g) * CLD + t;
  const double *pb = sB + g * CLD + t;
#pragma unroll 4
  for (int kk = 0; kk < CT / 4; ++kk) {
    const double a = pa[4 * kk];
#pragma unroll
    for (int j = 0; j < 8; ++j) dmma(acc[j][0], acc[j][1], a, pb[8 * j * CLD + 4 * kk]);
  }
}

// Global tile (ld 64) -> shared (ld CLD), optionally transposed: every
// thread's sixteen loads are issued before its first store.
__device__ __forceinline__ void load_tile(double *s, const double *g, bool trans) {
  double v[TS / CTH];
#pragma unroll
  for (int q = 0; q < TS / CTH; ++q) v[q] = __ldcg(g + threadIdx.x + q * CTH);
#pragma unroll
  for (int q = 0; q < TS / CTH; ++q) {
    const int idx = threadIdx.x + q * CTH, i = idx >> 6, j = idx & 63;
    if (trans)
      s[j * CLD + i] = v[q];
    else
      s[i * CLD + j] = v[q];
  }
}

// Tile update gt -= acc (fragment positions): the sixteen old values are
// loaded before any is written back.
__device__ __forceinline__ void sub_frag(double *gt, const double (&acc)[8][2]) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int r = 8 * w + (lane >> 2), c0 = 2 * (lane & 3);
  double2 old[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) old[j] = __ldcg((const double2 *)(gt + r * CT + 8 * j + c0));
#pragma unroll
  for (int j = 0; j < 8; ++j)
    *(double2 *)(gt + r * CT + 8 * j + c0) = make_double2(old[j].x - acc[j][0], old[j].y - acc[j][1]);
}

// Fragment positions of acc[j][e]: row 8w + g, column 8j + 2t + e.
template <class F>
__device__ __forceinline__ void for_frag(F f) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int r = 8 * w + (lane >> 2), c0 = 2 * (lane & 3);
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    f(j, 0, r, 8 * j + c0);
    f(j, 1, r, 8 * j + c0 + 1);
  }
}

// Factor the diagonal tile in place and write L_JJ and L_JJ^-1, with all
// threads of the CTA.  Factor: panels of eight columns; warp 0 factors a
// panel (per column the pivot's square root, the column scaled by its
// reciprocal, the panel's later columns updated; warp barriers only), then
// all threads apply the panel to the trailing triangle, each entry's eight
// updates in column order, as in the unblocked column loop; two block
// barriers a panel.  Inverse:
// four lanes of one warp per column c, rows i in order (lane q takes the
// terms mm = c + q, c + q + 4, ... of entry (i, c), the partial sums added as
// (p0 + p1) + (p2 + p3), times the row's reciprocal pivot), warp barriers
// only.  s, si: two shared tiles (ld CT + 1); pp: CT doubles of scratch
// (the reciprocal pivots).
__device__ void potrf_tile(double *gtile, double *ginv, int *err, double *s, double *si, double *pp) {
  constexpr int LD = CT + 1, PW = 8;
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  __syncthreads();
  {
    double v[TS / CTH];
#pragma unroll
    for (int q = 0; q < TS / CTH; ++q) v[q] = __ldcg(gtile + t + q * CTH);
#pragma unroll
    for (int q = 0; q < TS / CTH; ++q) s[((t + q * CTH) >> 6) * LD + ((t + q * CTH) & 63)] = v[q];
  }
  __syncthreads();
  for (int k0 = 0; k0 < CT; k0 += PW) {
    if (w == 0) {
      for (int k = k0; k < k0 + PW; ++k) {
        const double d = s[k * LD + k];
        const double dk = sqrt(d > 0. ? d : 1.), rdk = 1. / dk;
        if (lane == 0 && !(d > 0.)) atomicOr(err, 4);
        for (int i = k + 1 + lane; i < CT; i += 32) s[i * LD + k] *= rdk;
        __syncwarp();
        if (lane == 0) s[k * LD + k] = dk;
        // the panel's later columns j (k < j < k0 + PW), rows i >= j
        for (int j = k + 1; j < k0 + PW; ++j) {
          const double ljk = s[j * LD + k];
          for (int i = j + lane; i < CT; i += 32) s[i * LD + j] -= s[i * LD + k] * ljk;
        }
        __syncwarp();
      }
    }
    __syncthreads();
    // trailing triangle (rows and columns >= k0 + PW): the panel's updates
    for (int i = k0 + PW + w; i < CT; i += CTH / 32)
      for (int j = k0 + PW + lane; j <= i; j += 32) {
        double v = s[i * LD + j];
#pragma unroll
        for (int k = k0; k < k0 + PW; ++k) v -= s[i * LD + k] * s[j * LD + k];
        s[i * LD + j] = v;
      }
    __syncthreads();
  }
  if (t < CT) pp[t] = 1. / s[t * LD + t];
  __syncthreads();
  {
    const int c = t >> 2, q = t & 3;  // column c (0..63), partial q
    for (int i = 0; i < CT; ++i) {
      double acc = 0.;
      if (c < i)
        for (int mm = c + q; mm < i; mm += 4) acc += s[i * LD + mm] * si[mm * LD + c];
      const double a1 = __shfl_down_sync(0xffffffffu, acc, 1);
      const double p01 = acc + a1;  // lanes q = 0 and 2: (p0 + p1), (p2 + p3)
      const double p23 = __shfl_down_sync(0xffffffffu, p01, 2);
      if (q == 0) {
        const double rdi = pp[i];
        si[i * LD + c] = c < i ? -(p01 + p23) * rdi : (c == i ? rdi : 0.);
      }
      __syncwarp();
    }
  }
  __syncthreads();
  for (int idx = t; idx < TS; idx += CTH) {
    const int i = idx >> 6, j = idx & 63;
    gtile[idx] = j <= i ? s[i * LD + j] : 0.;
    ginv[idx] = si[i * LD + j];
  }
  __syncthreads();
}

// k-th item of the lower triangle (bi >= bk) of an m x m tile triangle
__device__ __forceinline__ void tri_item(long long t, int &bi, int &bk) {
  int i = (int)((sqrt(8. * (double)t + 1.) - 1.) / 2.);
  while ((long long)(i + 1) * (i + 2) / 2 <= t) ++i;
  while ((long long)i * (i + 1) / 2 > t) --i;
  bi = i;
  bk = (int)(t - (long long)i * (i + 1) / 2);
}

__global__ void __launch_bounds__(CTH, 1) k_chol_tiles(Tiles T) {
  extern __shared__ __align__(16) double csm[];
  double *sA = csm, *sB = csm + CT * CLD, *sP = csm + 2 * CT * CLD;
  const int G = gridDim.x;
  const unsigned nb = (unsigned)G;
  // tile 0's diagonal block
  if (blockIdx.x == 0) potrf_tile(tile_at(T, 0, 0), T.Linv, T.err, sA, sB, sP);
  if (!grid_barrier(T.bar, nb, T.err, T.bar_ns)) return;
  // With the inverse, X = L^-1 is formed in the same loop: tile row J of X
  // in phase T of column J (X_Jj = Linv_J R_Jj, its R final after the
  // updates of the earlier columns), and its updates R_Kj -= L_KJ X_Jj in
  // phase U -- the same products in the same order as a separate pass over
  // the tile rows, without its barriers.
  const int nxj = T.want_inverse ? 1 : 0;
  for (int J = 0; J < T.nt; ++J) {
    const int h = T.hrow[J], m = h - J;
    // T: L_IJ = A_IJ L_JJ^-T (items 0 .. m - 1); X_Jj = Linv_J R_Jj (items
    // m .. m + J with the inverse)
    const int ntt = m + nxj * (J + 1);
    for (int t = blockIdx.x; t < ntt; t += G) {
      __syncthreads();
      double *gt;
      if (t < m) {
        gt = tile_at(T, J + 1 + t, J);
        load_tile(sA, gt, false);
        load_tile(sB, T.Linv + (size_t)J * TS, false);
      } else {
        gt = T.X + tri(J, t - m) * TS;
        load_tile(sA, T.Linv + (size_t)J * TS, false);
        load_tile(sB, gt, true);  // R^T: the product Linv R as Linv (R^T)^T
      }
      __syncthreads();
      double acc[8][2] = {};
      gemm_nt(sA, sB, acc);
      __syncthreads();
      for_frag([&](int j, int e, int r, int c) { gt[r * CT + c] = acc[j][e]; });
    }
    if (!grid_barrier(T.bar, nb, T.err, T.bar_ns)) return;
    // U: A_IK -= L_IJ L_KJ^T (items 0 .. nu - 1); the tile (J+1, J+1) is
    // then factored by the CTA of item 0, which takes no other item when
    // there are other CTAs.  With the inverse also R_Kj -= L_KJ X_Jj, K > J,
    // j <= J (items nu .. nu + m (J + 1) - 1).
    const long long nu = (long long)m * (m + 1) / 2;
    const long long ntu = nu + (long long)nxj * m * (J + 1);
    const long long t0 = (G > 1 && blockIdx.x > 0) ? blockIdx.x : 0, dt = (G > 1 && blockIdx.x > 0) ? G - 1 : G;
    for (long long t = (G > 1 && blockIdx.x == 0) ? 0 : t0; t < ntu; t += dt) {
      __syncthreads();
      double *gt;
      if (t < nu) {
        int bi, bk;
        tri_item(t, bi, bk);
        load_tile(sA, tile_at(T, J + 1 + bi, J), false);
        load_tile(sB, tile_at(T, J + 1 + bk, J), false);
        gt = tile_at(T, J + 1 + bi, J + 1 + bk);
      } else {
        const long long u = t - nu;
        const int K = J + 1 + (int)(u / (J + 1)), j = (int)(u % (J + 1));
        load_tile(sA, tile_at(T, K, J), false);
        load_tile(sB, T.X + tri(J, j) * TS, true);
        gt = T.X + tri(K, j) * TS;
      }
      __syncthreads();
      double acc[8][2] = {};
      gemm_nt(sA, sB, acc);
      sub_frag(gt, acc);
      if (t == 0) {
        __syncthreads();
        potrf_tile(gt, T.Linv + (size_t)(J + 1) * TS, T.err, sA, sB, sP);
      }
      if (G > 1 && blockIdx.x == 0) break;  // CTA 0: item 0 and the factor only
    }
    if (m == 0 && J + 1 < T.nt && blockIdx.x == (J + 1) % G)
      potrf_tile(tile_at(T, J + 1, J + 1), T.Linv + (size_t)(J + 1) * TS, T.err, sA, sB, sP);
    if (!grid_barrier(T.bar, nb, T.err, T.bar_ns)) return;
  }
  if (!T.want_inverse) return;
  const int nt = T.nt;
  // A^-1 tile (i, k), k <= i: sum over m >= i of X_mi^T X_mk
  const long long no = (long long)nt * (nt + 1) / 2;
  for (long long t = blockIdx.x; t < no; t += G) {
    int bi, bk;
    tri_item(t, bi, bk);
    double acc[8][2] = {};
    for (int mt = bi; mt < nt; ++mt) {
      __syncthreads();
      load_tile(sA, T.X + tri(mt, bi) * TS, true);
      load_tile(sB, T.X + tri(mt, bk) * TS, true);
      __syncthreads();
      gemm_nt(sA, sB, acc);
    }
    double *ga = T.Ainv + tri(bi, bk) * TS;
    for_frag([&](int j, int e, int r, int c) { ga[r * CT + c] = acc[j][e]; });
  }
}

// Dense n x n row-major (lower triangle used), scaled by d_i d_j (+ eps on
// the diagonal), into lower tiles; the padding of the last diagonal tile is
// the identity.  X starts as the identity (diagonal tiles), zero elsewhere.
__global__ void k_pack_dense(const double *A, const double *dsc, double eps, int n, int nt, double *Lt, double *X) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long ntile = (long long)nt * (nt + 1) / 2;
  if (idx >= ntile * TS) return;
  const long long t = idx / TS;
  const int e = (int)(idx % TS), a = e >> 6, b = e & 63;
  int I, J;
  tri_item(t, I, J);
  const int i = I * CT + a, j = J * CT + b;
  double v = 0.;
  if (i < n && j < n) {
    if (j <= i) {
      v = A[(size_t)i * n + j] * dsc[i] * dsc[j];
      if (i == j) v += eps;
    }
  } else if (i == j) {
    v = 1.;
  }
  Lt[idx] = v;
  X[idx] = (i == j) ? 1. : 0.;
}

// Lower inverse tiles back to the dense matrix (both triangles), scaled.
__global__ void k_unpack_dense(const double *At, const double *dsc, int n, int nt, double *Ainv) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long ntile = (long long)nt * (nt + 1) / 2;
  if (idx >= ntile * TS) return;
  const long long t = idx / TS;
  const int e = (int)(idx % TS), a = e >> 6, b = e & 63;
  int I, J;
  tri_item(t, I, J);
  const int i = I * CT + a, j = J * CT + b;
  if (i >= n || j >= n || (I == J && b > a)) return;
  const double v = At[idx] * dsc[i] * dsc[j];
  Ainv[(size_t)i * n + j] = v;
  Ainv[(size_t)j * n + i] = v;
}

__global__ void k_dense_meta(int nt, long long *toff, int *fcol, int *hrow) {
  const int I = blockIdx.x * blockDim.x + threadIdx.x;
  if (I >= nt) return;
  toff[I] = (long long)I * (I + 1) / 2;
  fcol[I] = 0;
  hrow[I] = nt - 1;
}

// one CTA per SM (fewer arrivals per grid barrier); 0 if none fits
int chol_grid() {
  int dev = 0, nsm = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  cudaFuncSetAttribute(k_chol_tiles, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CSMEM);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_chol_tiles, CTH, CSMEM);
  return per >= 1 ? nsm : 0;
}

}  // namespace

// Factor the envelope tiles in place (L over A) and write the inverses of
// the diagonal tiles; one cooperative launch.
void tile_cholesky(double *tiles, const long long *toff, const int *fcol, const int *hrow, double *Linv, int nt,
                   unsigned *bar, int *err, cudaStream_t s) {
  if (nt <= 0) return;
  Tiles T;
  T.L = tiles;
  T.toff = toff;
  T.fcol = fcol;
  T.hrow = hrow;
  T.Linv = Linv;
  T.X = nullptr;
  T.Ainv = nullptr;
  T.nt = nt;
  T.want_inverse = 0;
  T.bar = bar;
  T.err = err;
  T.bar_ns = BAR_TIMEOUT_NS;
  const int g = std::max(1, chol_grid());
  RPBA_CUDA_CHECK(cudaMemsetAsync(bar, 0, 2 * sizeof(unsigned), s));
  void *args[] = {&T};
  RPBA_CUDA_CHECK(cudaLaunchCooperativeKernel((const void *)k_chol_tiles, dim3(g), dim3(CTH), args, CSMEM, s));
}

size_t spd_inverse_bytes(int n) {
  const long long nt = (n + CT - 1) / CT;
  return (size_t)(3 * (nt * (nt + 1) / 2) + nt) * TS * sizeof(double) + nt * 16 + 64;
}

// A^-1 of the dense SPD matrix (D A D + eps I) scaled back by D, with D =
// diag(dsc): A (row major n x n, lower triangle used) -> Ainv (both
// triangles).  One cooperative launch for the factorisation and the inverse.
void spd_inverse_scaled(const double *A, const double *dsc, double eps, int n, double *Ainv, void *work,
                        unsigned *bar, int *err, cudaStream_t s) {
  if (n <= 0) return;
  const int nt = (n + CT - 1) / CT;
  const long long ntile = (long long)nt * (nt + 1) / 2;
  double *Lt = (double *)work;
  double *X = Lt + ntile * TS;
  double *At = X + ntile * TS;
  double *Linv = At + ntile * TS;
  long long *toff = (long long *)(Linv + (size_t)nt * TS);
  int *fcol = (int *)(toff + nt);
  int *hrow = fcol + nt;
  k_dense_meta<<<(nt + 127) / 128, 128, 0, s>>>(nt, toff, fcol, hrow);
  k_pack_dense<<<(int)((ntile * TS + 255) / 256), 256, 0, s>>>(A, dsc, eps, n, nt, Lt, X);
  Tiles T;
  T.L = Lt;
  T.toff = toff;
  T.fcol = fcol;
  T.hrow = hrow;
  T.Linv = Linv;
  T.X = X;
  T.Ainv = At;
  T.nt = nt;
  T.want_inverse = 1;
  T.bar = bar;
  T.err = err;
  T.bar_ns = BAR_TIMEOUT_NS;
  const int g = (int)std::max<long long>(1, std::min<long long>(chol_grid(), ntile));
  RPBA_CUDA_CHECK(cudaMemsetAsync(bar, 0, 2 * sizeof(unsigned), s));
  void *args[] = {&T};
  RPBA_CUDA_CHECK(cudaLaunchCooperativeKernel((const void *)k_chol_tiles, dim3(g), dim3(CTH), args, CSMEM, s));
  k_unpack_dense<<<(int)((ntile * TS + 255) / 256), 256, 0, s>>>(At, dsc, n, nt, Ainv);
  RPBA_CUDA_CHECK(cudaGetLastError());
}

}  // namespace rpba
