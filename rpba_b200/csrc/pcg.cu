// pcg.cu -- block-Jacobi preconditioned conjugate gradients on the reduced
// camera system, with the scalar logic of SparsePCG (rbacore.cpp:1807-1914):
// x0 = 0, best iterate kept (starting from the right-hand side), stop when
// the squared step increment drops by 1e5 or after msize iterations,
// beta = r1^T (h1 - h) / r^T h clamped at 0.
//
// One cooperative launch runs the whole solve.  FP64 form (k_pcg): rows
// (cameras) are owned by warps; a 9x9 block product uses 27 lanes (3 blocks
// at a time).  The FP32 form (k_pcg32) is described before it.  Dot
// products are reduced per CTA and then, after a grid barrier, by every CTA
// in the same fixed order, so all CTAs take identical decisions.  The grid
// barrier's wait is bounded: after 2 s it sets an error bit and returns.
#include <cooperative_groups.h>

#include <algorithm>

#include "gridsync.cuh"
#include "internal.h"

namespace rpba {

namespace {

// Threads per CTA of the FP64 form's persistent kernel: 32 warps, two work
// items in flight each through shared memory.  (The FP32 form is k_pcg32.)
template <class BT>
constexpr int pcg_threads() {
  return 1024;
}
template <class BT>
constexpr int pcg_warps() {
  return pcg_threads<BT>() / 32;
}


struct PcgArgs {
  const void *blocks;  // BT[(nimg + nboff) * 81]
  const int2 *ent;
  const int *rowoff;
  const int *row_item_off;
  const int4 *item_meta;  // (row, first entry, end entry, 0)
  const int2 *rowspan;    // (diagonal entry, end entry) of each row
  float *tpart;           // FP32 form: transposed products of the off-diagonal blocks
  // FP32 form (k_pcg32): (row, column) of every block in storage order, the
  // first off-diagonal block of every row, d^k in FP32 (12 floats a camera),
  // and the phase-1 row sums (diagonal, row head, warp-run head)
  const int4 *bidx;
  const int *firstN, *firstT;
  int nboff;
  float *d32;
  double *pdiag, *prow, *pw;  // pw: per chunk
  double *pdqc;               // per chunk: its share of d^T A d
  unsigned *ctr;              // next chunk of phase 1
  int chunk;                  // groups per phase-1 chunk
  const double *Cinv;
  double *r, *h, *x, *xbest, *D0, *D1;
  double *part;        // [nitems * 9] SpMV partial rows
  double *red1, *red2; // [gridDim * 4] per-CTA partial sums of phase 1 / phase 2
                       // (separate, so a fast CTA never overwrites a slot that
                       // a slow CTA is still reading)
  unsigned *bar;
  int *err;
  int *iters;
  // grid barriers wait for G + bar_extra arrivals, at most bar_ns each
  // (bar_extra 0 and the default limit outside the timeout test hook)
  unsigned bar_extra;
  unsigned long long bar_ns;
  int row0, row1, nitems, msize;
  int mode;     // 0: reference stop rule; 1: relative preconditioned residual
  double tol2;  // mode 1: stop when r^T M^-1 r <= tol2 * (r0^T M^-1 r0)
  // two-level preconditioner (coarse.cu): rows are owned per aggregate
  int nagg, nc;
  const int *agg_off, *agg_rows;
  const double *P, *Ainv;
  double *rc, *hj;
  double *rowc;  // FP32 form: per row its restriction P_k^T r1 (CO_M) and its share of dr^2, stride RC_S
};

// Deterministic CTA sum of up to three values; valid in every thread.
template <int N, int W>
__device__ __forceinline__ void cta_sum(double (&v)[N], double (*sh)[4]) {
#pragma unroll
  for (int j = 0; j < N; ++j)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[j] += __shfl_xor_sync(0xffffffffu, v[j], o);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0)
#pragma unroll
    for (int j = 0; j < N; ++j) sh[warp][j] = v[j];
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int j = 0; j < N; ++j) {
      double t = lane < W ? sh[lane][j] : 0.;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
      if (lane == 0) sh[W][j] = t;
    }
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < N; ++j) v[j] = sh[W][j];
  __syncthreads();
}

// Sum of the per-CTA partials (stride 4) in a fixed order; every CTA gets
// the same values.
template <int N, int W>
__device__ __forceinline__ void grid_sum(const double *red, int G, double (&v)[N], double (*sh)[4]) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp == 0) {
#pragma unroll
    for (int j = 0; j < N; ++j) {
      double t = 0.;
      for (int i = lane; i < G; i += 32) t += __ldcg(red + 4 * i + j);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
      if (lane == 0) sh[W][j] = t;
    }
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < N; ++j) v[j] = sh[W][j];
  __syncthreads();
}

// Asynchronous global -> shared copies of one element (the blocks are
// constant during the launch, so the L1-allocating form is safe).
template <class BT>
__device__ __forceinline__ void cp_async_elem(BT *dst, const BT *src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  if constexpr (sizeof(BT) == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src));
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// Phase-1 software pipeline: each warp has two work items in flight.  The
// next item's three blocks are copied to a shared-memory stage (cp.async),
// and its d^k values (column and row) are loaded into registers, while the
// current item is multiplied.
constexpr int P1_ELEMS = 3 * 81;
// Dynamic shared memory: the FP64 form's stages
template <class BT>
constexpr size_t pcg_smem_bytes() {
  return sizeof(BT) * (size_t)pcg_warps<BT>() * 2 * P1_ELEMS;
}
struct P1Item {
  int it, row, ne;  // item, its row, entries (0 past the end)
  int2 en;          // this lane's entry (group grp)
  double dc;        // d^k[col][rr] of this lane's entry
  double dk;        // d^k[row][lane] (lanes < 9)
};

template <class BT>
__device__ __forceinline__ void p1_issue(const PcgArgs &A, int it, BT *stage, const double *dprev, double beta,
                                         int lane, int grp, int rr, P1Item &I) {
  I.it = it;
  I.ne = 0;
  I.row = 0;
  I.en = make_int2(0, 0);
  I.dc = 0.;
  I.dk = 0.;
  if (it < A.nitems) {
    const int4 m = A.item_meta[it];
    I.row = m.x;
    I.ne = m.z - m.y;
    if (lane < 27 && grp < I.ne) {
      I.en = A.ent[m.y + grp];
      const size_t j = (size_t)I.en.x * 9 + rr;
      I.dc = __ldcg(A.h + j) + beta * __ldcg(dprev + j);
    }
    if (lane < 9) {
      const size_t i = (size_t)I.row * 9 + lane;
      I.dk = __ldcg(A.h + i) + beta * __ldcg(dprev + i);
    }
    const int b0 = __shfl_sync(0xffffffffu, I.en.y, 0) & 0x7fffffff;
    const int b1 = __shfl_sync(0xffffffffu, I.en.y, 9) & 0x7fffffff;
    const int b2 = __shfl_sync(0xffffffffu, I.en.y, 18) & 0x7fffffff;
    const BT *blocks = (const BT *)A.blocks;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int e = lane + 32 * q;
      if (e < P1_ELEMS) {
        const int g = e / 81, off = e - g * 81;
        if (g < I.ne) {
          const int b = g == 0 ? b0 : (g == 1 ? b1 : b2);
          cp_async_elem(stage + e, blocks + (size_t)b * 81 + off);
        }
      }
    }
  }
  cp_async_commit();
}

// q of one row (valid in lanes < 9) from the phase-1 partials of the FP64
// form: one partial per item, the three 9-lane groups taking every third
// item (four loads in flight), in a fixed order.
__device__ __forceinline__ double row_q(const PcgArgs &A, int row, int lane, int grp, int rr) {
  const int t0 = A.row_item_off[row], t1 = A.row_item_off[row + 1];
  double qg = 0.;
  if (lane < 27) {
    double q0 = 0., q1 = 0., q2 = 0., q3 = 0.;
    int t = t0 + grp;
    for (; t + 9 < t1; t += 12) {
      q0 += __ldcg(A.part + (size_t)t * 9 + rr);
      q1 += __ldcg(A.part + (size_t)(t + 3) * 9 + rr);
      q2 += __ldcg(A.part + (size_t)(t + 6) * 9 + rr);
      q3 += __ldcg(A.part + (size_t)(t + 9) * 9 + rr);
    }
    for (; t < t1; t += 3) q0 += __ldcg(A.part + (size_t)t * 9 + rr);
    qg = (q0 + q1) + (q2 + q3);
  }
  const double qa = __shfl_down_sync(0xffffffffu, qg, 9);
  const double qb = __shfl_down_sync(0xffffffffu, qg, 18);
  return qg + qa + qb;
}

// Iteration k (two grid barriers):
//  phase 1  q-partials of A d^k per work item (<= 3 blocks of one row), with
//           d^k = h^k + beta^(k-1) d^(k-1) formed on the fly; partial d^T q
//  phase 2  per row: q = sum of its items' partials, x += alpha d,
//           r1 = r - alpha q, h1 = C r1; partials of (alpha q)^2,
//           r1^T (h1 - h) and r1^T h1 (the next r^T h); d^k is stored
// With the coarse correction (CO) phase 2 is split by one more barrier:
//  phase 2a per aggregate (one CTA): as above but h1 is only the block part
//           (kept in hj), and the aggregate's restriction P^T r1 is formed
//  phase 2b per aggregate: z = A_c^-1[aggregate rows] (P^T r1), then
//           h1 = hj + P z and the two dot products
// BT: the storage type of the reduced camera system's blocks, double (the
// FP32 form has its own kernel, k_pcg32 below).
template <bool CO, class BT>
__global__ void __launch_bounds__(pcg_threads<BT>(), 1) k_pcg(PcgArgs A) {
  static_assert(sizeof(BT) == 8, "k_pcg is the FP64 form");
  constexpr int PCG_T = pcg_threads<BT>(), PCG_W = pcg_warps<BT>();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gwarp = blockIdx.x * PCG_W + warp, nwarps = gridDim.x * PCG_W;
  const int grp = lane / 9, rr = lane % 9, gbase = grp * 9;
  const int G = gridDim.x;
  __shared__ double sh[PCG_W + 1][4];
  extern __shared__ __align__(16) unsigned char pcg_dyn[];
  BT *stage0 = (BT *)pcg_dyn + (size_t)warp * 2 * P1_ELEMS;
  BT *stage1 = stage0 + P1_ELEMS;
  // r^T h of the start vectors
  {
    double v[1] = {0.};
    for (int row = A.row0 + gwarp; row < A.row1; row += nwarps)
      if (lane < 9) {
        const size_t i = (size_t)row * 9 + lane;
        v[0] += A.r[i] * A.h[i];
      }
    cta_sum<1, PCG_W>(v, sh);
    if (threadIdx.x == 0) A.red2[4 * blockIdx.x] = v[0];
  }
  if (!grid_barrier(A.bar, G + A.bar_extra, A.err, A.bar_ns)) return;
  double erthk;
  {
    double v[1];
    grid_sum<1, PCG_W>(A.red2, G, v, sh);
    erthk = v[0];
  }
  double meandrold = 1.e50, meandr0 = 1.e50, beta_prev = 0.;
  const double erthk0 = erthk;
  bool converged = false;
  int k;
  for (k = 0; k < A.msize; ++k) {
    const double *dprev = (k & 1) ? A.D0 : A.D1;
    double *dcur = (k & 1) ? A.D1 : A.D0;
    // ---- phase 1
    double pdq[1] = {0.};
      {
        P1Item cur, nxt;
        p1_issue<BT>(A, gwarp, stage0, dprev, beta_prev, lane, grp, rr, cur);
        p1_issue<BT>(A, gwarp + nwarps, stage1, dprev, beta_prev, lane, grp, rr, nxt);
        for (int t = 0; cur.it < A.nitems; ++t) {
          BT *st = (t & 1) ? stage1 : stage0;
          cp_async_wait<1>();
          __syncwarp();
          const bool act = lane < 27 && grp < cur.ne;
          const bool tr = cur.en.y < 0;
          const BT *B = st + grp * 81;
          double acc = 0.;
  #pragma unroll
          for (int c = 0; c < 9; ++c) {
            const double xc = __shfl_sync(0xffffffffu, cur.dc, (lane < 27 ? gbase : 0) + c);
            if (act) acc += (double)B[tr ? c * 9 + rr : rr * 9 + c] * xc;
          }
          const double a1 = __shfl_down_sync(0xffffffffu, acc, 9);
          const double a2 = __shfl_down_sync(0xffffffffu, acc, 18);
          if (lane < 9) {
            const double p = acc + a1 + a2;
            A.part[(size_t)cur.it * 9 + lane] = p;
            pdq[0] += cur.dk * p;
          }
          __syncwarp();
          cur = nxt;
          p1_issue<BT>(A, cur.it + nwarps, st, dprev, beta_prev, lane, grp, rr, nxt);
        }
        cp_async_wait<0>();
        __syncwarp();
      }
    cta_sum<1, PCG_W>(pdq, sh);
    if (threadIdx.x == 0) A.red1[4 * blockIdx.x] = pdq[0];
    if (!grid_barrier(A.bar, G + A.bar_extra, A.err, A.bar_ns)) return;
    double edtAdk;
    {
      double v[1];
      grid_sum<1, PCG_W>(A.red1, G, v, sh);
      edtAdk = v[0];
    }
    double alpha;
    if (fabs(erthk) < 1.e-20 || fabs(erthk) > 1.e20)
      alpha = 0.;
    else
      alpha = erthk / edtAdk;
    // ---- phase 2
    double p2[3] = {0., 0., 0.};
    if constexpr (!CO) {
      for (int row = A.row0 + gwarp; row < A.row1; row += nwarps) {
        const size_t i = (size_t)row * 9 + (lane < 9 ? lane : 0);
        double r1v = 0., hv = 0.;
        const double q = row_q(A, row, lane, grp, rr);
        if (lane < 9) {
          hv = __ldcg(A.h + i);
          const double dk = hv + beta_prev * __ldcg(dprev + i);
          dcur[i] = dk;
          A.x[i] = A.x[i] + alpha * dk;
          const double dr = alpha * q;
          r1v = A.r[i] - dr;
          p2[0] += dr * dr;
        }
        const double *C = A.Cinv + (size_t)row * 81;
        double h1v = 0.;
#pragma unroll
        for (int c = 0; c < 9; ++c) {
          const double rc = __shfl_sync(0xffffffffu, r1v, c);
          if (lane < 9) h1v += __ldg(C + lane * 9 + c) * rc;
        }
        if (lane < 9) {
          A.r[i] = r1v;
          A.h[i] = h1v;
          p2[1] += r1v * (h1v - hv);
          p2[2] += r1v * h1v;
        }
      }
    } else {
      __shared__ double shr[PCG_W][CO_M];
      __shared__ double shz[CO_M];
      for (int a = blockIdx.x; a < A.nagg; a += G) {
        const int t0 = A.agg_off[a], t1 = A.agg_off[a + 1];
        double rcw = 0.;
        for (int t = t0 + warp; t < t1; t += PCG_W) {
          const int row = A.agg_rows[t];
          const size_t i = (size_t)row * 9 + (lane < 9 ? lane : 0);
          double r1v = 0.;
          const double q = row_q(A, row, lane, grp, rr);
          if (lane < 9) {
            const double hv = __ldcg(A.h + i);
            const double dk = hv + beta_prev * __ldcg(dprev + i);
            dcur[i] = dk;
            A.x[i] = __ldcg(A.x + i) + alpha * dk;
            const double dr = alpha * q;
            r1v = __ldcg(A.r + i) - dr;
            p2[0] += dr * dr;
          }
          const double *C = A.Cinv + (size_t)row * 81;
          const double *Pk = A.P + (size_t)row * (9 * CO_M);
          double h1v = 0.;
#pragma unroll
          for (int c = 0; c < 9; ++c) {
            const double rc = __shfl_sync(0xffffffffu, r1v, c);
            if (lane < 9) h1v += __ldg(C + lane * 9 + c) * rc;
            if (lane < CO_M) rcw += __ldg(Pk + c * CO_M + lane) * rc;
          }
          if (lane < 9) {
            A.r[i] = r1v;
            A.hj[i] = h1v;
          }
        }
        if (lane < CO_M) shr[warp][lane] = rcw;
        __syncthreads();
        if (threadIdx.x < CO_M) {
          double sum = 0.;
          for (int w = 0; w < PCG_W; ++w) sum += shr[w][threadIdx.x];
          A.rc[a * CO_M + threadIdx.x] = sum;
        }
        __syncthreads();
      }
      if (!grid_barrier(A.bar, G + A.bar_extra, A.err, A.bar_ns)) return;
      for (int a = blockIdx.x; a < A.nagg; a += G) {
        double z[CO_M];
#pragma unroll
        for (int j = 0; j < CO_M; ++j) z[j] = 0.;
        for (int i = threadIdx.x; i < A.nc; i += PCG_T) {
          const double rv = __ldcg(A.rc + i);
#pragma unroll
          for (int j = 0; j < CO_M; ++j) z[j] += __ldg(A.Ainv + (size_t)(a * CO_M + j) * A.nc + i) * rv;
        }
#pragma unroll
        for (int j = 0; j < CO_M; ++j) {
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) z[j] += __shfl_xor_sync(0xffffffffu, z[j], o);
          if (lane == 0) shr[warp][j] = z[j];
        }
        __syncthreads();
        if (threadIdx.x < CO_M) {
          double sum = 0.;
          for (int w = 0; w < PCG_W; ++w) sum += shr[w][threadIdx.x];
          shz[threadIdx.x] = sum;
        }
        __syncthreads();
        const int t0 = A.agg_off[a], t1 = A.agg_off[a + 1];
        for (int t = t0 + warp; t < t1; t += PCG_W) {
          const int row = A.agg_rows[t];
          if (lane < 9) {
            const size_t i = (size_t)row * 9 + lane;
            const double *Pk = A.P + (size_t)row * (9 * CO_M) + lane * CO_M;
            double h1v = __ldcg(A.hj + i);
#pragma unroll
            for (int j = 0; j < CO_M; ++j) h1v += __ldg(Pk + j) * shz[j];
            const double hv = __ldcg(A.h + i), r1v = __ldcg(A.r + i);
            p2[1] += r1v * (h1v - hv);
            p2[2] += r1v * h1v;
            A.h[i] = h1v;
          }
        }
        __syncthreads();
      }
    }
    cta_sum<3, PCG_W>(p2, sh);
    if (threadIdx.x == 0) {
      A.red2[4 * blockIdx.x] = p2[0];
      A.red2[4 * blockIdx.x + 1] = p2[1];
      A.red2[4 * blockIdx.x + 2] = p2[2];
    }
    if (!grid_barrier(A.bar, G + A.bar_extra, A.err, A.bar_ns)) return;
    double g3[3];
    grid_sum<3, PCG_W>(A.red2, G, g3, sh);
    const double meandr = g3[0], er1th1 = g3[1];
    if (k == 0) meandr0 = meandr;
    // mode 0 keeps the iterate with the smallest increment (the reference's
    // exivold); mode 1 keeps the latest finite one and stops, unconverged,
    // at a breakdown (a non-finite residual or increment)
    const bool finite = isfinite(g3[0]) && isfinite(g3[2]);
    const bool improved = (A.mode == 1 && finite) || meandr < meandrold;
    if (improved) {
      meandrold = meandr;
      for (int row = A.row0 + gwarp; row < A.row1; row += nwarps)
        if (lane < 9) A.xbest[(size_t)row * 9 + lane] = __ldcg(A.x + (size_t)row * 9 + lane);
    }
    if (A.mode == 0 && meandr * 1.e5 < meandr0) break;
    if (A.mode == 1 && !finite) break;
    if (A.mode == 1 && g3[2] <= A.tol2 * erthk0) {
      converged = true;
      break;
    }
    double beta = fabs(er1th1) < 1.e-10 ? 0. : er1th1 / erthk;
    if (beta < 0.) beta = 0.;
    beta_prev = beta;
    erthk = g3[2];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    A.iters[0] = k < A.msize ? k + 1 : A.msize;
    A.iters[1] = converged ? 1 : 0;
  }
}

// ---------------------------------------------------------------------------
// The FP32 form's persistent PCG (mixed precision and the learned solver).
//
// Phase 1 streams the reduced camera system through shared memory with 1-D
// TMA bulk copies.  The blocks are read in storage order: the diagonal
// blocks of rows begini.. first, then every off-diagonal block once (upper
// triangle, row major).  The stream is cut into groups of 32 blocks and the
// groups into chunks of A.chunk groups (fixed boundaries); warps take chunks
// from a counter, the next one taken a chunk ahead, so a fast warp takes
// more of them.  One elected lane copies a group's blocks (32 x 324 B) and
// their (row, column, slot) triples into the warp's stage, completing on the
// stage's mbarrier; each lane then owns one block: it forms the block's row
// product B d_col (summed into its row) and, for an off-diagonal block, the
// transposed product B^T d_row, which goes to the block's slot of tpart.
// The slots are in column order (the blocks of column c, i.e. the
// transposed entries of row c, are consecutive), and a slot is 64 bytes (9
// values, zero padding: two whole sectors, so the scattered writes need no
// read of the rest of a sector), so that phase 2 reads each row's
// transposed products as one contiguous run.  Lane i reads its block at byte
// 324 i of the stage: 81 i is a distinct bank for every lane, so the reads
// are conflict-free.  The gathered vector is d^k rounded to FP32 (d32, 12
// floats per camera so that a camera is three aligned 16-byte loads),
// formed for all rows in phase D before phase 1.
//
// Row sums: a diagonal block's product is written to pdiag[row]; the
// off-diagonal products of a row are summed per group by a segmented warp
// scan in FP32 (a group inside the open row: per-lane FP64 running sums),
// carried across groups in FP64 and written once per (row, chunk): to
// prow[row] by the chunk that holds the row's first block, to pw[chunk] by a
// chunk that starts inside the row; each chunk's share of d^T A d goes to
// pdqc[chunk].  Everything a chunk writes depends on the chunk only, not on
// the warp that took it.  Phase 2 adds, per row and in a fixed order, pdiag,
// prow, the pw of the chunks that start inside the row, and the row's run of
// transposed products (the blocks stored by earlier rows in its column).
//
// Iteration k: phase D (d^k = h + beta d^(k-1), FP64 and FP32 copies),
// barrier, phase 1 (A d^k and d^T A d), barrier, phase 2 (as in the FP64
// form; with the coarse space: 2a, rows taken from a counter, barrier, 2a',
// the aggregates' restrictions, barrier, 2b, the coarse correction),
// barrier.
constexpr int P32_W = 16;  // warps per CTA
constexpr int P32_T = P32_W * 32;
constexpr int GB = 32;     // blocks per group: one per lane
constexpr int STG_BLK = GB * 324 + 16;
constexpr int STG_IDX = GB * 16;
constexpr int STG_BYTES = STG_BLK + STG_IDX + 16;  // + the mbarrier
constexpr size_t P32_SMEM = (size_t)P32_W * STG_BYTES;
static_assert(STG_BLK % 16 == 0 && STG_IDX % 16 == 0, "16-byte aligned stage parts");

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// global -> shared bulk copy completing on `bar` (one destination: this
// CTA's own shared memory; the source is this GPU's own memory)
__device__ __forceinline__ void bulk_load(void *dst, const void *src, unsigned bytes, unsigned long long *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// Group g of the stream: its first block (storage index), its block count
// and, for an off-diagonal group, the first block's off-diagonal index.
struct Grp32 {
  long long start;
  int n;
  bool diag;
  long long boff;
};
__device__ __forceinline__ Grp32 group_of(long long g, int gd, int row0, int row1, int nboff) {
  Grp32 q;
  if (g < gd) {
    q.start = row0 + GB * g;
    q.n = (int)min((long long)GB, row1 - q.start);
    q.diag = true;
    q.boff = -1;
  } else {
    const long long j = g - gd;
    q.boff = GB * j;
    q.start = row1 + q.boff;
    q.n = (int)min((long long)GB, nboff - q.boff);
    q.diag = false;
  }
  return q;
}
// Phase 1 is cut into chunks of A.chunk groups (fixed boundaries); the warps take
// chunks from a counter, so a fast warp takes more of them, and everything a
// chunk writes (its row sums, its share of d^T A d) depends only on the
// chunk: the result does not depend on which warp took it.

// Byte offsets of a group's data inside its 16-byte aligned copies.
__device__ __forceinline__ unsigned blk_misalign(const float *blocks, long long start) {
  return (unsigned)(((unsigned long long)(blocks + start * 81)) & 15ull);
}
constexpr int TP_STRIDE = 16;  // floats per transposed-product slot (64 B)
constexpr int RC_S = 12;       // doubles per row of rowc

// Issue the copies of group q into the warp's stage (one lane).
__device__ __forceinline__ void group_issue(const PcgArgs &A, const Grp32 &q, unsigned char *stg,
                                            unsigned long long *bar) {
  const float *blocks = (const float *)A.blocks;
  const unsigned mb = blk_misalign(blocks, q.start);
  const unsigned nb_bytes = (mb + (unsigned)q.n * 324u + 15u) & ~15u;
  const unsigned ni_bytes = (unsigned)q.n * 16u;
  mbar_expect_tx(bar, nb_bytes + ni_bytes);
  bulk_load(stg, (const unsigned char *)(blocks + q.start * 81) - mb, nb_bytes, bar);
  bulk_load(stg + STG_BLK, A.bidx + q.start, ni_bytes, bar);
}

// Bounded wait on the stage's mbarrier (the copies of this CTA's own
// memory end in microseconds; the limit only keeps a fault from hanging).
__device__ __forceinline__ bool stage_wait(const PcgArgs &A, unsigned long long *bar, unsigned parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = gtimer();
  while (!mbar_try_wait(bar, parity)) {
    if (gtimer() - t0 > A.bar_ns) return false;
  }
  return true;
}

// FP32 d^k of camera c (12-float stride) into v[0..8].  The loads may hit
// L1: d32 is written in phase D by all CTAs before a grid barrier, whose
// gpu-scope fence and block barrier order those writes before these loads,
// and the rows of a cluster keep gathering the same columns.
__device__ __forceinline__ void load_d32(const float *d32, int c, float (&v)[9]) {
  const float4 *p = (const float4 *)(d32 + (size_t)c * 12);
  const float4 a = __ldca(p), b = __ldca(p + 1), e = __ldca(p + 2);
  v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
  v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
  v[8] = e.x;
}

// q of one row in lanes < 9 (FP32 form).
__device__ __forceinline__ double row_q32(const PcgArgs &A, int row, long long gd, int lane) {
  // the row's run of transposed products (slots firstT[row] ..
  // firstT[row + 1]): one slot per lane (three 16-byte loads), and the sums
  // of the phase-1 chunks that start strictly inside the row's off-diagonal
  // blocks, one chunk per lane; nine FP64 partial sums, then a fixed butterfly
  double acc[9];
#pragma unroll
  for (int j = 0; j < 9; ++j) acc[j] = 0.;
  const int e0 = __ldg(A.firstT + row), e1 = __ldg(A.firstT + row + 1);
  const int f0 = __ldg(A.firstN + row), f1 = __ldg(A.firstN + row + 1);
#pragma unroll 4
  for (int e = e0 + lane; e < e1; e += 32) {
    const float4 *t = (const float4 *)(A.tpart + (size_t)e * TP_STRIDE);
    const float4 a = __ldcg(t), b = __ldcg(t + 1), c = __ldcg(t + 2);
    acc[0] += (double)a.x;
    acc[1] += (double)a.y;
    acc[2] += (double)a.z;
    acc[3] += (double)a.w;
    acc[4] += (double)b.x;
    acc[5] += (double)b.y;
    acc[6] += (double)b.z;
    acc[7] += (double)b.w;
    acc[8] += (double)c.x;
  }
  if (f1 > f0) {
    const long long ch = A.chunk, glo = gd + f0 / GB + 1, ghi = gd + (f1 - 1) / GB;
    for (long long c = (glo + ch - 1) / ch + lane; c * ch <= ghi; c += 32) {
      const double *w = A.pw + (size_t)c * 9;
#pragma unroll
      for (int j = 0; j < 9; ++j) acc[j] += __ldcg(w + j);
    }
  }
#pragma unroll
  for (int j = 0; j < 9; ++j)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc[j] += __shfl_xor_sync(0xffffffffu, acc[j], o);
  double q = 0.;
#pragma unroll
  for (int j = 0; j < 9; ++j)
    if (lane == j) q = acc[j];
  if (lane < 9) {
    const size_t i = (size_t)row * 9 + lane;
    q += __ldcg(A.pdiag + i);
    if (f1 > f0) q += __ldcg(A.prow + i);
  }
  return q;
}

template <bool CO>
__global__ void __launch_bounds__(P32_T, 1) k_pcg32(PcgArgs A) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gwarp = blockIdx.x * P32_W + warp, nwarps = gridDim.x * P32_W;
  const int G = gridDim.x;
  __shared__ double sh[P32_W + 1][4];
  extern __shared__ __align__(16) unsigned char pcg_dyn[];
  unsigned char *stg = pcg_dyn + (size_t)warp * STG_BYTES;
  unsigned long long *mbar = (unsigned long long *)(stg + STG_BLK + STG_IDX);
  unsigned parity = 0;
  if (lane == 0) mbar_init(mbar, 1);
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  __syncwarp();
  const float *blocks = (const float *)A.blocks;
  const long long gd = (A.row1 - A.row0 + GB - 1) / GB, go = ((long long)A.nboff + GB - 1) / GB;
  const long long ng = gd + go, ch = A.chunk, nch = (ng + ch - 1) / ch;
  // r^T h of the start vectors
  {
    double v[1] = {0.};
    for (int row = A.row0 + gwarp; row < A.row1; row += nwarps)
      if (lane < 9) {
        const size_t i = (size_t)row * 9 + lane;
        v[0] += A.r[i] * A.h[i];
      }
    cta_sum<1, P32_W>(v, sh);
    if (threadIdx.x == 0) A.red2[4 * blockIdx.x] = v[0];
  }
  if (!grid_barrier(A.bar, G + A.bar_extra, A.err, A.bar_ns)) return;
  double erthk;
  {
    double v[1];
    grid_sum<1, P32_W>(A.red2, G, v, sh);
    erthk = v[0];
  }
  double meandrold = 1.e50, meandr0 = 1.e50, beta_prev = 0.;
  const double erthk0 = erthk;
  bool converged = false;
  int k;
  for (k = 0; k < A.msize; ++k) {
    const double *dprev = (k & 1) ? A.D0 : A.D1;
    double *dcur = (k & 1) ? A.D1 : A.D0;
    // ---- phase D: d^k for every row, FP64 and FP32
    for (int row = A.row0 + gwarp; row < A.row1; row += nwarps)
      if (lane < 9) {
        const size_t i = (size_t)row * 9 + lane;
        const double dk = __ldcg(A.h + i) + beta_prev * __ldcg(dprev + i);
        dcur[i] = dk;
        A.d32[(size_t)row * 12 + lane] = (float)dk;
      }
    if (blockIdx.x == 0 && threadIdx.x < 2) A.ctr[threadIdx.x] = 0u;
    if (!grid_barrier(A.bar, G + A.bar_extra, A.err, A.bar_ns)) return;
    // ---- phase 1
    {
      auto grab = [&]() -> long long {
        unsigned c = 0;
        if (lane == 0) c = atomicAdd(A.ctr, 1u);
        return (long long)__shfl_sync(0xffffffffu, c, 0);
      };
      long long c = grab();
      long long cn = c < nch ? grab() : nch;  // the next chunk, taken one ahead
      int cur_row = -1;   // row of the running sum (-1: none yet in this chunk)
      bool cur_head = false;
      double racc = 0.;   // running sum of cur_row, component `lane` (lanes < 9)
      double pdq = 0.;    // this chunk's share of d^T A d (per lane)
      auto flush = [&]() {
        if (cur_row >= 0 && lane < 9) {
          double *dst = cur_head ? A.prow + (size_t)cur_row * 9 : A.pw + (size_t)c * 9;
          dst[lane] = racc;
        }
      };
      // per-lane running sums of the open row over the groups inside it,
      // folded into racc (lanes 0..8) at the row's end in a fixed butterfly
      double lacc[9];
#pragma unroll
      for (int j = 0; j < 9; ++j) lacc[j] = 0.;
      auto fold_lanes = [&]() {
        double v = 0.;
#pragma unroll
        for (int j = 0; j < 9; ++j) {
          double a = lacc[j];
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
          if (lane == j) v = a;
          lacc[j] = 0.;
        }
        racc += v;
      };
      if (c < nch && lane == 0) group_issue(A, group_of(c * ch, (int)gd, A.row0, A.row1, A.nboff), stg, mbar);
      bool ok = true;
      while (c < nch) {
      const long long g0 = c * ch, g1 = min(ng, g0 + ch);
      cur_row = -1;
      racc = 0.;
      pdq = 0.;
      for (long long g = g0; g < g1; ++g) {
        const Grp32 q = group_of(g, (int)gd, A.row0, A.row1, A.nboff);
        if (!stage_wait(A, mbar, parity)) {
          ok = false;
          break;
        }
        parity ^= 1u;
        const unsigned mb = blk_misalign(blocks, q.start);
        const bool act = lane < q.n;
        int4 rc = make_int4(-1 - lane, -1, 0, 0);
        float dc[9], dr[9], y[9], t[9];
#pragma unroll
        for (int j = 0; j < 9; ++j) {
          y[j] = 0.f;
          t[j] = 0.f;
        }
        if (act) {
          rc = *(const int4 *)(stg + STG_BLK + 16 * lane);
          load_d32(A.d32, rc.y, dc);
          load_d32(A.d32, rc.x, dr);
          const float *B = (const float *)(stg + mb + 324 * lane);
#pragma unroll
          for (int i = 0; i < 9; ++i) {
            float yi = 0.f;
#pragma unroll
            for (int j = 0; j < 9; ++j) {
              const float b = B[i * 9 + j];
              yi = fmaf(b, dc[j], yi);
              t[j] = fmaf(b, dr[i], t[j]);
            }
            y[i] = yi;
          }
          double s = 0.;
#pragma unroll
          for (int i = 0; i < 9; ++i) s += (double)dr[i] * (double)y[i];
          if (!q.diag)
#pragma unroll
            for (int j = 0; j < 9; ++j) s += (double)dc[j] * (double)t[j];
          pdq += s;
        }
        // the stage's blocks are read: the next group's copies may land
        // (the next group of this chunk, or the first of the next chunk)
        __syncwarp();
        const long long gn = g + 1 < g1 ? g + 1 : (cn < nch ? cn * ch : -1);
        if (lane == 0 && gn >= 0) {
          fence_proxy_async();
          group_issue(A, group_of(gn, (int)gd, A.row0, A.row1, A.nboff), stg, mbar);
        }
        if (q.diag) {
          if (act) {
            double *dst = A.pdiag + (size_t)rc.x * 9;
#pragma unroll
            for (int i = 0; i < 9; ++i) dst[i] = (double)y[i];
          }
          continue;
        }
        // the transposed product to the block's slot (column order)
        if (act) {
          float4 *dst = (float4 *)(A.tpart + (size_t)rc.z * TP_STRIDE);
          __stcg(dst, make_float4(t[0], t[1], t[2], t[3]));
          __stcg(dst + 1, make_float4(t[4], t[5], t[6], t[7]));
          __stcg(dst + 2, make_float4(t[8], 0.f, 0.f, 0.f));
          __stcg(dst + 3, make_float4(0.f, 0.f, 0.f, 0.f));
        }
        const int row = rc.x;
        // a group inside the open row (most groups: a row has hundreds of
        // blocks): every lane adds its product to its own FP64 running sum
        if (cur_row >= 0 && __all_sync(0xffffffffu, !act || row == cur_row)) {
          if (act)
#pragma unroll
            for (int j = 0; j < 9; ++j) lacc[j] += (double)y[j];
          continue;
        }
        // a row boundary: the lanes' running sums join the open row's sum,
        // then a segmented scan of the group's products (rows non-decreasing
        // in lane order; inactive lanes carry distinct negative rows)
        fold_lanes();
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int ru = __shfl_up_sync(0xffffffffu, row, o);
#pragma unroll
          for (int j = 0; j < 9; ++j) {
            const float vu = __shfl_up_sync(0xffffffffu, y[j], o);
            if (lane >= o && ru == row) y[j] += vu;
          }
        }
        const int rnext = __shfl_down_sync(0xffffffffu, row, 1);
        const bool end = act && (lane == q.n - 1 || rnext != row);
        unsigned ends = __ballot_sync(0xffffffffu, end);
        int seg_first = 0;  // first lane of the segment ending at e
        while (ends) {
          const int e = __ffs(ends) - 1;
          ends &= ends - 1;
          const int re = __shfl_sync(0xffffffffu, row, e);
          double sv = 0.;
#pragma unroll
          for (int j = 0; j < 9; ++j) {
            const float tv = __shfl_sync(0xffffffffu, y[j], e);
            if (lane == j) sv = (double)tv;
          }
          if (re == cur_row) {
            racc += sv;
          } else {
            flush();
            // a segment starts the row unless it is the chunk's first and
            // the row began before the chunk
            cur_head = cur_row >= 0 || seg_first > 0 || q.boff + seg_first == (long long)__ldg(A.firstN + re);
            cur_row = re;
            racc = sv;
          }
          seg_first = e + 1;
        }
      }
      if (!ok) break;
      fold_lanes();
      flush();
      // the chunk's share of d^T A d, summed over its lanes in a fixed order
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) pdq += __shfl_xor_sync(0xffffffffu, pdq, o);
      if (lane == 0) A.pdqc[c] = pdq;
      c = cn;
      cn = c < nch ? grab() : nch;
      }
      __syncwarp();
      if (!ok) {
        // a copy that never completed: record it, give it one more bounded
        // wait, and leave after the grid barrier below has failed as well
        if (lane == 0) atomicOr(A.err, 2);
        stage_wait(A, mbar, parity);
      }
    }

    if (!grid_barrier(A.bar, G + A.bar_extra, A.err, A.bar_ns)) return;
    double edtAdk;
    {
      // d^T A d: every CTA sums the chunks' shares in the same fixed order
      // (thread t takes chunks t, t + P32_T, ...; then a butterfly per warp
      // and the warps in order)
      double v = 0.;
      for (long long i = threadIdx.x; i < nch; i += P32_T) v += __ldcg(A.pdqc + i);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) sh[warp][0] = v;
      __syncthreads();
      if (threadIdx.x == 0) {
        double t = 0.;
        for (int w = 0; w < P32_W; ++w) t += sh[w][0];
        sh[P32_W][0] = t;
      }
      __syncthreads();
      edtAdk = sh[P32_W][0];
      __syncthreads();
    }
    double alpha;
    if (fabs(erthk) < 1.e-20 || fabs(erthk) > 1.e20)
      alpha = 0.;
    else
      alpha = erthk / edtAdk;
    // ---- phase 2
    double p2[3] = {0., 0., 0.};
    if constexpr (!CO) {
      for (int row = A.row0 + gwarp; row < A.row1; row += nwarps) {
        const size_t i = (size_t)row * 9 + (lane < 9 ? lane : 0);
        double r1v = 0., hv = 0.;
        const double q = row_q32(A, row, gd, lane);
        if (lane < 9) {
          hv = __ldcg(A.h + i);
          const double dk = __ldcg(dcur + i);
          A.x[i] = A.x[i] + alpha * dk;
          const double dr = alpha * q;
          r1v = A.r[i] - dr;
          p2[0] += dr * dr;
        }
        const double *C = A.Cinv + (size_t)row * 81;
        double h1v = 0.;
#pragma unroll
        for (int c = 0; c < 9; ++c) {
          const double rc = __shfl_sync(0xffffffffu, r1v, c);
          if (lane < 9) h1v += __ldg(C + lane * 9 + c) * rc;
        }
        if (lane < 9) {
          A.r[i] = r1v;
          A.h[i] = h1v;
          p2[1] += r1v * (h1v - hv);
          p2[2] += r1v * h1v;
        }
      }
    } else {
      __shared__ double shr[P32_W][CO_M + 1];
      __shared__ double shz[CO_M];
      // 2a: rows in any order, taken from a counter (the rows of high index,
      // with the longest runs of transposed products, first); each row's
      // results go to its own slots, so nothing depends on which warp took it
      // Every load of a row that does not depend on q is issued before the
      // row's walk: lanes 0..8 hold row `lane` of C_k, lanes 16..25 column
      // `lane - 16` of P_k (9 doubles a lane either way).
      const int nrows = A.row1 - A.row0;
      auto grab_row = [&]() -> int {
        unsigned t = 0;
        if (lane == 0) t = atomicAdd(A.ctr + 1, 1u);
        return (int)__shfl_sync(0xffffffffu, t, 0);
      };
      const bool cl = lane < 9, pl = lane >= 16 && lane < 16 + CO_M;
      for (int t = grab_row(); t < nrows;) {
        const int row = A.row1 - 1 - t;
        const int tn = grab_row();  // the next row, taken one ahead
        const size_t i = (size_t)row * 9 + (cl ? lane : 0);
        double cp[9];
        {
          const double *C = A.Cinv + (size_t)row * 81 + (cl ? lane * 9 : 0);
          const double *Pk = A.P + (size_t)row * (9 * CO_M) + (pl ? lane - 16 : 0);
#pragma unroll
          for (int c = 0; c < 9; ++c) cp[c] = cl ? __ldg(C + c) : (pl ? __ldg(Pk + c * CO_M) : 0.);
        }
        double dk = 0., xv = 0., rv = 0.;
        if (cl) {
          dk = __ldcg(dcur + i);
          xv = __ldcg(A.x + i);
          rv = __ldcg(A.r + i);
        }
        const double q = row_q32(A, row, gd, lane);
        double r1v = 0., d2 = 0.;
        if (cl) {
          A.x[i] = xv + alpha * dk;
          const double dr = alpha * q;
          r1v = rv - dr;
          d2 = dr * dr;
        }
        double acc = 0.;  // lanes 0..8: h_j; lanes 16..25: the restriction
#pragma unroll
        for (int c = 0; c < 9; ++c) {
          const double rc = __shfl_sync(0xffffffffu, r1v, c);
          acc += cp[c] * rc;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) d2 += __shfl_xor_sync(0xffffffffu, d2, o);
        if (cl) {
          A.r[i] = r1v;
          A.hj[i] = acc;
        }
        if (pl) A.rowc[(size_t)row * RC_S + lane - 16] = acc;
        if (lane == 31) A.rowc[(size_t)row * RC_S + CO_M] = d2;
        t = tn;
      }
      if (!grid_barrier(A.bar, G + A.bar_extra, A.err, A.bar_ns)) return;
      // 2a': per aggregate, its rows' restrictions and shares of dr^2 in a
      // fixed order (warp w: rows w, w + P32_W, ...; then the warps in order)
      for (int a = blockIdx.x; a < A.nagg; a += G) {
        const int t0 = A.agg_off[a], t1 = A.agg_off[a + 1];
        double v = 0.;
        if (lane <= CO_M)
          for (int t = t0 + warp; t < t1; t += P32_W) v += __ldcg(A.rowc + (size_t)A.agg_rows[t] * RC_S + lane);
        if (lane <= CO_M) shr[warp][lane] = v;
        __syncthreads();
        if (threadIdx.x <= CO_M) {
          double sum = 0.;
          for (int w = 0; w < P32_W; ++w) sum += shr[w][threadIdx.x];
          if (threadIdx.x < CO_M)
            A.rc[a * CO_M + threadIdx.x] = sum;
          else
            p2[0] += sum;
        }
        __syncthreads();
      }
      if (!grid_barrier(A.bar, G + A.bar_extra, A.err, A.bar_ns)) return;
      for (int a = blockIdx.x; a < A.nagg; a += G) {
        double z[CO_M];
#pragma unroll
        for (int j = 0; j < CO_M; ++j) z[j] = 0.;
        for (int i = threadIdx.x; i < A.nc; i += P32_T) {
          const double rv = __ldcg(A.rc + i);
#pragma unroll
          for (int j = 0; j < CO_M; ++j) z[j] += __ldg(A.Ainv + (size_t)(a * CO_M + j) * A.nc + i) * rv;
        }
#pragma unroll
        for (int j = 0; j < CO_M; ++j) {
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) z[j] += __shfl_xor_sync(0xffffffffu, z[j], o);
          if (lane == 0) shr[warp][j] = z[j];
        }
        __syncthreads();
        if (threadIdx.x < CO_M) {
          double sum = 0.;
          for (int w = 0; w < P32_W; ++w) sum += shr[w][threadIdx.x];
          shz[threadIdx.x] = sum;
        }
        __syncthreads();
        const int t0 = A.agg_off[a], t1 = A.agg_off[a + 1];
        for (int t = t0 + warp; t < t1; t += P32_W) {
          const int row = A.agg_rows[t];
          if (lane < 9) {
            const size_t i = (size_t)row * 9 + lane;
            const double *Pk = A.P + (size_t)row * (9 * CO_M) + lane * CO_M;
            double h1v = __ldcg(A.hj + i);
#pragma unroll
            for (int j = 0; j < CO_M; ++j) h1v += __ldg(Pk + j) * shz[j];
            const double hv = __ldcg(A.h + i), r1v = __ldcg(A.r + i);
            p2[1] += r1v * (h1v - hv);
            p2[2] += r1v * h1v;
            A.h[i] = h1v;
          }
        }
        __syncthreads();
      }
    }
    cta_sum<3, P32_W>(p2, sh);
    if (threadIdx.x == 0) {
      A.red2[4 * blockIdx.x] = p2[0];
      A.red2[4 * blockIdx.x + 1] = p2[1];
      A.red2[4 * blockIdx.x + 2] = p2[2];
    }
    if (!grid_barrier(A.bar, G + A.bar_extra, A.err, A.bar_ns)) return;
    double g3[3];
    grid_sum<3, P32_W>(A.red2, G, g3, sh);
    const double meandr = g3[0], er1th1 = g3[1];
    if (k == 0) meandr0 = meandr;
    const bool finite = isfinite(g3[0]) && isfinite(g3[2]);
    const bool improved = (A.mode == 1 && finite) || meandr < meandrold;
    if (improved) {
      meandrold = meandr;
      for (int row = A.row0 + gwarp; row < A.row1; row += nwarps)
        if (lane < 9) A.xbest[(size_t)row * 9 + lane] = __ldcg(A.x + (size_t)row * 9 + lane);
    }
    if (A.mode == 0 && meandr * 1.e5 < meandr0) break;
    if (A.mode == 1 && !finite) break;
    if (A.mode == 1 && g3[2] <= A.tol2 * erthk0) {
      converged = true;
      break;
    }
    double beta = fabs(er1th1) < 1.e-10 ? 0. : er1th1 / erthk;
    if (beta < 0.) beta = 0.;
    beta_prev = beta;
    erthk = g3[2];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    A.iters[0] = k < A.msize ? k + 1 : A.msize;
    A.iters[1] = converged ? 1 : 0;
  }
}

// Preconditioner C_k = S_kk^-1 (rbacore.cpp:1839-1846) and the start
// vectors: r = b, h = C r, d^(-1) = 0, x = 0, best = b.  One thread per
// camera with the serial lu_inverse9 (the drop-in form's numerics).
__global__ void k_pcg_setup(DevLSA L, PcgWork W) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= L.nimg) return;
  double *C = W.Cinv + (size_t)k * 81;
  const size_t o = (size_t)k * 9;
  for (int a = 0; a < 9; ++a) W.d[o + a] = 0.;
  if (k < L.begini) {
    for (int a = 0; a < 9; ++a) W.r[o + a] = W.h[o + a] = W.x[o + a] = W.xbest[o + a] = 0.;
    return;
  }
  const int np = L.camparv[k + 1] - L.camparv[k];
  load_block(L, (size_t)k, C);  // inverted in place below
  lu_inverse9(np, C, C);
  double rv[9];
  for (int a = 0; a < 9; ++a) rv[a] = L.rhs[o + a];
  for (int a = 0; a < 9; ++a) {
    double s = 0.;
    for (int c = 0; c < 9; ++c) s += C[a * 9 + c] * rv[c];
    W.r[o + a] = rv[a];
    W.h[o + a] = s;
    W.x[o + a] = 0.;
    W.xbest[o + a] = rv[a];
  }
}

}  // namespace

// the phase-1 stages of the FP64 form live in dynamic shared memory (124 KB)
void pcg_set_smem() {
  cudaFuncSetAttribute(k_pcg<false, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)pcg_smem_bytes<double>());
  cudaFuncSetAttribute(k_pcg<true, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)pcg_smem_bytes<double>());
  cudaFuncSetAttribute(k_pcg32<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)P32_SMEM);
  cudaFuncSetAttribute(k_pcg32<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)P32_SMEM);
}


// Groups of 32 blocks per phase-1 chunk of the FP32 PCG: small enough that
// the warps finish together, large enough that a chunk's fixed work (its
// first segmented scan, its sums) stays small (city workload, phase 1 with
// its barrier: 2 groups 377 us, 4 groups 365 us, 8 groups 379 us).
constexpr int PCG32_CHUNK = 4;

int pcg_max_grid(int device) {
  int nsm = 0, per = 0, per2 = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
  pcg_set_smem();
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_pcg<false, double>, pcg_threads<double>(),
                                                pcg_smem_bytes<double>());
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per2, k_pcg<true, double>, pcg_threads<double>(),
                                                pcg_smem_bytes<double>());
  per = std::min(per, per2);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per2, k_pcg32<false>, P32_T, P32_SMEM);
  per = std::min(per, per2);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per2, k_pcg32<true>, P32_T, P32_SMEM);
  per = std::min(per, per2);
  if (per < 1) per = 1;
  return nsm * per;
}

// Returns 0; throws CudaError on launch errors.  The iteration count is
// left in W.iters.
int pcg_prepare(const DevLSA &L, const PcgWork &W, int mode, const float *weights, const CoarseWork *coarse,
                cudaStream_t s) {
  const bool co = coarse && coarse->nagg > 0;
  if (mode == 1 || weights || co)
    learned_pcg_setup(L, W, weights, s);
  else
    k_pcg_setup<<<(L.nimg + 127) / 128, 128, 0, s>>>(L, W);
  if (co) coarse_apply(L, *coarse, W.r, W.h, s);
  RPBA_CUDA_CHECK(cudaGetLastError());
  return co ? 3 : 1;
}

int pcg_iterate(const DevLSA &L, const PcgWork &W, int msize, int grid, cudaStream_t s, int mode, double tol,
                const CoarseWork *coarse) {
  const bool co = coarse && coarse->nagg > 0;
  const int nrows = L.nimg - L.begini;
  if (nrows <= 0) return 0;
  int g;
  if (L.blocks32) {
    // FP32 form: groups of 32 blocks (the diagonal blocks of the system's
    // rows, then the off-diagonal blocks), at least one group per warp
    const long long ng = (nrows + GB - 1) / GB + ((long long)L.nboff + GB - 1) / GB;
    g = (int)std::min<long long>((ng + P32_W - 1) / P32_W, grid);
  } else {
    const int wpc = pcg_warps<double>();
    g = (L.nitems + wpc - 1) / wpc;
  }
  if (g > grid) g = grid;
  if (g < 1) g = 1;
  PcgArgs A;
  A.blocks = L.blocks32 ? (const void *)L.blocks32 : (const void *)L.blocks;
  A.ent = L.ent;
  A.rowoff = L.rowoff;
  A.row_item_off = L.row_item_off;
  A.item_meta = L.item_meta;
  A.rowspan = L.rowspan;
  A.tpart = L.tpart;
  A.bidx = L.bidx;
  A.firstN = L.firstN;
  A.firstT = L.firstT;
  A.nboff = L.nboff;
  A.d32 = W.d32;
  A.pdiag = W.pdiag;
  A.prow = W.prow;
  A.pw = W.pw;
  A.pdqc = W.pdqc;
  A.ctr = W.ctr;
  A.rowc = W.rowc;
  A.chunk = PCG32_CHUNK;
  A.Cinv = W.Cinv;
  A.r = W.r;
  A.h = W.h;
  A.x = W.x;
  A.xbest = W.xbest;
  A.D0 = W.q;
  A.D1 = W.d;
  A.part = W.part;
  A.red1 = W.partials;
  A.red2 = W.partials + 4 * (size_t)grid;
  A.bar = W.bar;
  A.err = L.err;
  A.iters = W.iters;
  A.bar_extra = L.bar_extra;
  A.bar_ns = L.bar_timeout_ns ? L.bar_timeout_ns : BAR_TIMEOUT_NS;
  A.row0 = L.begini;
  A.row1 = L.nimg;
  A.nitems = L.nitems;
  A.msize = msize;
  A.mode = mode;
  A.tol2 = tol * tol;
  A.nagg = co ? coarse->nagg : 0;
  A.nc = co ? coarse->nc : 0;
  A.agg_off = co ? coarse->agg_off : nullptr;
  A.agg_rows = co ? coarse->agg_rows : nullptr;
  A.P = co ? coarse->P : nullptr;
  A.Ainv = co ? coarse->Ainv : nullptr;
  A.rc = co ? coarse->rc : nullptr;
  A.hj = co ? coarse->hj : nullptr;
  RPBA_CUDA_CHECK(cudaMemsetAsync(W.bar, 0, 2 * sizeof(unsigned), s));
  void *args[] = {&A};
  const void *fn;
  size_t smem;
  int nthreads;
  if (L.blocks32) {
    fn = co ? (const void *)k_pcg32<true> : (const void *)k_pcg32<false>;
    smem = P32_SMEM;
    nthreads = P32_T;
  } else {
    fn = co ? (const void *)k_pcg<true, double> : (const void *)k_pcg<false, double>;
    smem = pcg_smem_bytes<double>();
    nthreads = pcg_threads<double>();
  }
  pcg_set_smem();
  RPBA_CUDA_CHECK(cudaLaunchCooperativeKernel(fn, dim3(g), dim3(nthreads), args, smem, s));
  return 0;
}

}  // namespace rpba
