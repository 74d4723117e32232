// pcg.cu -- block-Jacobi preconditioned conjugate gradients on the reduced
// camera system, with the scalar logic of SparsePCG (rbacore.cpp:1807-1914):
// x0 = 0, best iterate kept (starting from the right-hand side), stop when
// the squared step increment drops by 1e5 or after msize iterations,
// beta = r1^T (h1 - h) / r^T h clamped at 0.
//
// One cooperative launch runs the whole solve.  Rows (cameras) are owned by
// warps; a 9x9 block product uses 27 lanes (3 blocks at a time).  Dot
// products are reduced per CTA and then, after a grid barrier, by every CTA
// in the same fixed order, so all CTAs take identical decisions.  The grid
// barrier's wait is bounded: after 2 s it sets an error bit and returns.
#include <cooperative_groups.h>

#include "gridsync.cuh"
#include "internal.h"

namespace rpba {

namespace {

constexpr int PCG_T = 256;
constexpr int PCG_W = PCG_T / 32;
struct PcgArgs {
  const double *blocks;
  const int *rowoff;
  const int2 *ent;
  const double *Cinv;
  double *r, *r1, *d, *q, *h, *h1, *x, *xbest;
  double *part1, *part2;
  unsigned *bar;
  int *err;
  int *iters;
  int row0, row1, msize;
};

// Deterministic CTA sum of two values; the result is valid in thread 0.
__device__ __forceinline__ void cta_sum2(double &a, double &b, double (*sh)[2]) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
    sh[warp][0] = a;
    sh[warp][1] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s0 = 0., s1 = 0.;
    for (int w = 0; w < PCG_W; ++w) {
      s0 += sh[w][0];
      s1 += sh[w][1];
    }
    a = s0;
    b = s1;
  }
  __syncthreads();
}

// Sum of the per-CTA partials in a fixed order; identical in every CTA.
__device__ __forceinline__ void grid_sum2(const double *part, int n, double &a, double &b,
                                          double *bc) {
  if (threadIdx.x < 32) {
    double s0 = 0., s1 = 0.;
    for (int i = threadIdx.x; i < n; i += 32) {
      s0 += __ldcg(part + 2 * i);
      s1 += __ldcg(part + 2 * i + 1);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      s0 += __shfl_xor_sync(0xffffffffu, s0, o);
      s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    }
    if (threadIdx.x == 0) {
      bc[0] = s0;
      bc[1] = s1;
    }
  }
  __syncthreads();
  a = bc[0];
  b = bc[1];
  __syncthreads();
}

__global__ void __launch_bounds__(PCG_T) k_pcg(PcgArgs A) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gwarp = blockIdx.x * PCG_W + warp, nwarps = gridDim.x * PCG_W;
  const int grp = lane / 9, rr = lane % 9;
  __shared__ double sh[PCG_W][2];
  __shared__ double bc[2];
  double meandrold = 1.e50, meandr0 = 1.e50;
  int k;
  for (k = 0; k < A.msize; ++k) {
    // q = A d ; r^T h ; d^T q
    double prh = 0., pdq = 0.;
    for (int row = A.row0 + gwarp; row < A.row1; row += nwarps) {
      double acc = 0.;
      if (lane < 27) {
        const int e1 = A.rowoff[row + 1];
        for (int e = A.rowoff[row] + grp; e < e1; e += 3) {
          const int2 en = A.ent[e];
          const double *B = A.blocks + (size_t)(en.y & 0x7fffffff) * 81;
          const double *xv = A.d + (size_t)en.x * 9;
          if (en.y >= 0) {
#pragma unroll
            for (int c = 0; c < 9; ++c) acc += B[rr * 9 + c] * __ldcg(xv + c);
          } else {
#pragma unroll
            for (int c = 0; c < 9; ++c) acc += B[c * 9 + rr] * __ldcg(xv + c);
          }
        }
      }
      const double a1 = __shfl_down_sync(0xffffffffu, acc, 9);
      const double a2 = __shfl_down_sync(0xffffffffu, acc, 18);
      if (lane < 9) {
        const size_t i = (size_t)row * 9 + lane;
        const double qv = acc + a1 + a2;
        A.q[i] = qv;
        prh += __ldcg(A.r + i) * __ldcg(A.h + i);
        pdq += __ldcg(A.d + i) * qv;
      }
    }
    cta_sum2(prh, pdq, sh);
    if (threadIdx.x == 0) {
      A.part1[2 * blockIdx.x] = prh;
      A.part1[2 * blockIdx.x + 1] = pdq;
    }
    if (!grid_barrier(A.bar, gridDim.x, A.err)) return;
    double erthk, edtAdk;
    grid_sum2(A.part1, gridDim.x, erthk, edtAdk, bc);
    double alpha;
    if (fabs(erthk) < 1.e-20 || fabs(erthk) > 1.e20)
      alpha = 0.;
    else
      alpha = erthk / edtAdk;
    // x += alpha d ; r1 = r - alpha q ; h1 = C r1
    double pmd = 0., pe1 = 0.;
    for (int row = A.row0 + gwarp; row < A.row1; row += nwarps) {
      const size_t i = (size_t)row * 9 + (lane < 9 ? lane : 0);
      double r1v = 0., hv = 0.;
      if (lane < 9) {
        const double dv = __ldcg(A.d + i);
        A.x[i] = __ldcg(A.x + i) + alpha * dv;
        const double dr = alpha * A.q[i];
        r1v = __ldcg(A.r + i) - dr;
        pmd += dr * dr;
        hv = __ldcg(A.h + i);
      }
      const double *C = A.Cinv + (size_t)row * 81;
      double h1v = 0.;
#pragma unroll
      for (int c = 0; c < 9; ++c) {
        const double rc = __shfl_sync(0xffffffffu, r1v, c);
        if (lane < 9) h1v += C[lane * 9 + c] * rc;
      }
      if (lane < 9) {
        A.r1[i] = r1v;
        A.h1[i] = h1v;
        pe1 += r1v * (h1v - hv);
      }
    }
    cta_sum2(pmd, pe1, sh);
    if (threadIdx.x == 0) {
      A.part2[2 * blockIdx.x] = pmd;
      A.part2[2 * blockIdx.x + 1] = pe1;
    }
    if (!grid_barrier(A.bar, gridDim.x, A.err)) return;
    double meandr, er1th1;
    grid_sum2(A.part2, gridDim.x, meandr, er1th1, bc);
    if (k == 0) meandr0 = meandr;
    const bool improved = meandr < meandrold;
    if (improved) meandrold = meandr;
    const bool stop = meandr * 1.e5 < meandr0;
    double beta = fabs(er1th1) < 1.e-10 ? 0. : er1th1 / erthk;
    if (beta < 0.) beta = 0.;
    for (int row = A.row0 + gwarp; row < A.row1; row += nwarps) {
      if (lane < 9) {
        const size_t i = (size_t)row * 9 + lane;
        if (improved) A.xbest[i] = A.x[i];
        if (!stop) {
          const double h1v = A.h1[i];
          A.d[i] = h1v + beta * __ldcg(A.d + i);
          A.r[i] = A.r1[i];
          A.h[i] = h1v;
        }
      }
    }
    if (stop) break;
    if (!grid_barrier(A.bar, gridDim.x, A.err)) return;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *A.iters = k < A.msize ? k + 1 : A.msize;
}

// Preconditioner C_k = S_kk^-1 (rbacore.cpp:1839-1846) and the start
// vectors: r = b, h = C r, d = h, x = 0, best = b.
__global__ void k_pcg_setup(DevLSA L, PcgWork W) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= L.nimg) return;
  double *C = W.Cinv + (size_t)k * 81;
  const size_t o = (size_t)k * 9;
  if (k < L.begini) {
    for (int a = 0; a < 9; ++a) W.r[o + a] = W.h[o + a] = W.d[o + a] = W.x[o + a] = W.xbest[o + a] = 0.;
    return;
  }
  const int np = L.camparv[k + 1] - L.camparv[k];
  lu_inverse9(np, L.blocks + (size_t)k * 81, C);
  double rv[9];
  for (int a = 0; a < 9; ++a) rv[a] = L.rhs[o + a];
  for (int a = 0; a < 9; ++a) {
    double s = 0.;
    for (int c = 0; c < 9; ++c) s += C[a * 9 + c] * rv[c];
    W.r[o + a] = rv[a];
    W.h[o + a] = s;
    W.d[o + a] = s;
    W.x[o + a] = 0.;
    W.xbest[o + a] = rv[a];
  }
}

}  // namespace

int pcg_max_grid(int device) {
  int nsm = 0, per = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_pcg, PCG_T, 0);
  if (per < 1) per = 1;
  return nsm * per;
}

// Returns the number of PCG iterations; throws CudaError on launch errors.
int pcg_solve(const DevLSA &L, const PcgWork &W, int msize, int grid, cudaStream_t s) {
  k_pcg_setup<<<(L.nimg + 127) / 128, 128, 0, s>>>(L, W);
  RPBA_CUDA_CHECK(cudaGetLastError());
  const int nrows = L.nimg - L.begini;
  if (nrows <= 0) return 0;
  int g = (nrows + PCG_W - 1) / PCG_W;
  if (g > grid) g = grid;
  if (g < 1) g = 1;
  PcgArgs A;
  A.blocks = L.blocks;
  A.rowoff = L.rowoff;
  A.ent = L.ent;
  A.Cinv = W.Cinv;
  A.r = W.r;
  A.r1 = W.r1;
  A.d = W.d;
  A.q = W.q;
  A.h = W.h;
  A.h1 = W.h1;
  A.x = W.x;
  A.xbest = W.xbest;
  A.part1 = W.partials;
  A.part2 = W.partials + 2 * (size_t)grid;
  A.bar = W.bar;
  A.err = L.err;
  A.iters = W.iters;
  A.row0 = L.begini;
  A.row1 = L.nimg;
  A.msize = msize;
  RPBA_CUDA_CHECK(cudaMemsetAsync(W.bar, 0, 2 * sizeof(unsigned), s));
  void *args[] = {&A};
  RPBA_CUDA_CHECK(cudaLaunchCooperativeKernel((const void *)k_pcg, dim3(g), dim3(PCG_T), args, 0, s));
  return 0;
}

}  // namespace rpba
