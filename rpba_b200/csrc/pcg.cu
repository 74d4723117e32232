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

#include <algorithm>

#include "gridsync.cuh"
#include "internal.h"

namespace rpba {

namespace {

// Threads per CTA of the persistent kernel, per block storage type: 1024 in
// the FP64 form (32 warps, two work items in flight each through shared
// memory), 640 in the FP32 form (20 warps whose three-slot register pipeline
// and transposed products use 96 registers a thread; measured faster than
// 768 and 1024).
template <class BT>
constexpr int pcg_threads() {
  return sizeof(BT) == 8 ? 1024 : 640;
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
// Dynamic shared memory: the FP64 form's stages; the FP32 form keeps its
// pipeline in registers
template <class BT>
constexpr size_t pcg_smem_bytes() {
  return sizeof(BT) == 8 ? sizeof(BT) * (size_t)pcg_warps<BT>() * 2 * P1_ELEMS : 0;
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

// First item of warp w's chunk in the FP32 form's phase 1 (the items are
// split into nwarps contiguous chunks of near-equal size).
__device__ __forceinline__ int chunk_start(long long w, int nitems, int nwarps) {
  return (int)(w * nitems / nwarps);
}

// q of one row (valid in lanes < 9) from the phase-1 partials.  FP32 form:
// the transposed products of the row's transposed entries (in entry order,
// three interleaved groups), then one partial per (row, chunk) segment,
// stored at the segment's first item: the row's first item and every chunk
// start inside the row, summed in item order.  FP64 form: one partial per item, the three 9-lane groups taking
// every third item (four loads in flight), in a fixed order.
template <class BT>
__device__ __forceinline__ double row_q(const PcgArgs &A, int row, int nwarps, int lane, int grp, int rr) {
  const int t0 = A.row_item_off[row], t1 = A.row_item_off[row + 1];
  if constexpr (sizeof(BT) == 4) {
    // transposed products of the row's transposed entries (blocks stored by
    // the rows before it): the three 9-lane groups take every third entry
    double qt = 0.;
    if (lane < 27) {
      const int e1 = __ldg(&A.rowspan[row].x);
#pragma unroll 4
      for (int e = A.rowoff[row] + grp; e < e1; e += 3) {
        const int blk = (__ldg(&A.ent[e].y) & 0x7fffffff) - A.row1;
        qt += (double)__ldcg(A.tpart + (size_t)blk * 9 + rr);
      }
    }
    const double qa = __shfl_down_sync(0xffffffffu, qt, 9);
    const double qb = __shfl_down_sync(0xffffffffu, qt, 18);
    double q = qt + qa + qb;
    if (lane < 9 && t0 < t1) {
      q += __ldcg(A.part + (size_t)t0 * 9 + lane);
      // smallest w whose chunk starts after t0
      long long w = ((long long)(t0 + 1) * nwarps + A.nitems - 1) / A.nitems;
      int prev = t0;
      for (; w < nwarps; ++w) {
        const int st = chunk_start(w, A.nitems, nwarps);
        if (st >= t1) break;
        if (st != prev) {
          q += __ldcg(A.part + (size_t)st * 9 + lane);
          prev = st;
        }
      }
    }
    return q;
  } else {
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
// BT: the storage type of the reduced camera system's blocks (double, or
// float in the mixed-precision form); vectors and sums are FP64 either way.
template <bool CO, class BT>
__global__ void __launch_bounds__(pcg_threads<BT>(), 1) k_pcg(PcgArgs A) {
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
    if constexpr (sizeof(BT) == 8) {
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
    } else {
      // FP32 blocks, symmetric SpMV: the items cover each row's diagonal and
      // normal entries, so every off-diagonal block is read once and gives
      // both products: its row's (block row rr times the column camera's
      // d^k) and its column's (block column rr, re-read from L1, times the
      // row camera's d^k, stored in the block's slot of tpart; phase 2 adds
      // it to the column's row, and its share of d^T A d is summed here).
      // Each warp walks one contiguous chunk of the items (row order) with a
      // three-slot register pipeline: the blocks of item t + 2 (and the d^k
      // entries they multiply) are loaded while item t is multiplied, the
      // entries of item t + 3 one step earlier; entry positions follow from
      // the walk (row spans), so no load waits on another.  Products are
      // formed in FP32 (FP32 blocks times d^k rounded to FP32); the row sums
      // are carried in FP64, per (row, chunk) segment in registers, written
      // once at the segment's first item.
      const int c0 = chunk_start(gwarp, A.nitems, nwarps);
      const int c1 = chunk_start(gwarp + 1, A.nitems, nwarps);
      if (c0 < c1) {
        const BT *blocks = (const BT *)A.blocks;
        const int4 m0 = A.item_meta[c0];
        int wrow = m0.x, we = m0.y, wend = __ldg(&A.rowspan[m0.x].y);
        int rowN = 0;
        int2 enN = make_int2(-1, 0);
        // entries of the walk's next item (lanes < 27, col -1 past the row);
        // a row's items run from its diagonal entry to its end
        auto ent_next = [&]() {
          rowN = wrow;
          enN = make_int2(-1, 0);
          if (lane < 27 && we + grp < wend) enN = __ldg(A.ent + we + grp);
          we += 3;
          if (we >= wend && ++wrow < A.row1) {
            const int2 sp = __ldg(A.rowspan + wrow);
            we = sp.x;
            wend = sp.y;
          }
        };
        // loads of the item whose entries are in enN into a slot, then the
        // next entries (items past the chunk load nothing); ob: the lane's
        // off-diagonal block (-1: none or the diagonal)
        auto slot_load = [&](int t, float (&b)[9], float &dc, int &row, int &ob) {
          row = rowN;
          dc = 0.f;
          ob = -1;
          const int2 en = enN;
          if (t < c1 && en.x >= 0) {
            if (en.y >= A.row1) ob = en.y - A.row1;
            // row rr of the block, or column rr of a transposed one
            const bool tr = en.y < 0;
            const BT *B = blocks + (size_t)(en.y & 0x7fffffff) * BS32 + (tr ? rr : rr * 9);
            const int sc = tr ? 9 : 1;
#pragma unroll
            for (int c = 0; c < 9; ++c) b[c] = __ldg(B + c * sc);
            const size_t j = (size_t)en.x * 9 + rr;
            dc = (float)(__ldcg(A.h + j) + beta_prev * __ldcg(dprev + j));
          } else {
#pragma unroll
            for (int c = 0; c < 9; ++c) b[c] = 0.f;
          }
          if (t + 1 < c1) ent_next();
        };
        auto dk_of = [&](int row) {
          return lane < 9 ? __ldcg(A.h + (size_t)row * 9 + lane) + beta_prev * __ldcg(dprev + (size_t)row * 9 + lane)
                          : 0.;
        };
        float bA[9], bB[9], bC[9];
        float dA, dB, dC;
        int rA, rB, rC, oA, oB, oC;
        ent_next();
        slot_load(c0, bA, dA, rA, oA);
        slot_load(c0 + 1, bB, dB, rB, oB);
        int seg = c0, segrow = rA;
        double racc = 0., dseg = dk_of(segrow);
        // d^k of the segment's row in every lane (FP32), for the transposed
        // products
        float xr[9];
        auto row_x = [&]() {
          const float v = (float)dseg;
#pragma unroll
          for (int c = 0; c < 9; ++c) xr[c] = __shfl_sync(0xffffffffu, v, c);
        };
        row_x();
        // item t from slot (b, d, r, o); the slot `nb` receives item t + 2.
        // An off-diagonal block's transposed product (column rr of the block,
        // re-read from L1, times the row's d^k) goes to its slot of tpart.
        auto step = [&](int t, const float (&b)[9], float d, int r, int o, float (&nb)[9], float &nd, int &nr,
                        int &no) {
          slot_load(t + 2, nb, nd, nr, no);
          float acc = 0.f;
#pragma unroll
          for (int c = 0; c < 9; ++c) acc = fmaf(b[c], __shfl_sync(0xffffffffu, d, (lane < 27 ? gbase : 0) + c), acc);
          const float a1 = __shfl_down_sync(0xffffffffu, acc, 9);
          const float a2 = __shfl_down_sync(0xffffffffu, acc, 18);
          if (r != segrow) {
            if (lane < 9) {
              A.part[(size_t)seg * 9 + lane] = racc;
              pdq[0] += dseg * racc;
            }
            seg = t;
            segrow = r;
            racc = 0.;
            dseg = dk_of(r);
            row_x();
          }
          if (lane < 9) racc += (double)acc + (double)a1 + (double)a2;
          if (o >= 0) {
            const BT *Bc = blocks + (size_t)(o + A.row1) * BS32 + rr;
            float yt = 0.f;
#pragma unroll
            for (int c = 0; c < 9; ++c) yt = fmaf(__ldg(Bc + c * 9), xr[c], yt);
            A.tpart[(size_t)o * 9 + rr] = yt;
            // the transposed product's share of d^T A d: d_c^T (B^T d_r)
            pdq[0] += (double)d * (double)yt;
          }
        };
        for (int t = c0; t < c1; t += 3) {
          step(t, bA, dA, rA, oA, bC, dC, rC, oC);
          if (t + 1 >= c1) break;
          step(t + 1, bB, dB, rB, oB, bA, dA, rA, oA);
          if (t + 2 >= c1) break;
          step(t + 2, bC, dC, rC, oC, bB, dB, rB, oB);
        }
        if (lane < 9) {
          A.part[(size_t)seg * 9 + lane] = racc;
          pdq[0] += dseg * racc;
        }
      }
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
        const double q = row_q<BT>(A, row, nwarps, lane, grp, rr);
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
          const double q = row_q<BT>(A, row, nwarps, lane, grp, rr);
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

// Preconditioner C_k = S_kk^-1 (rbacore.cpp:1839-1846) and the start
// vectors: r = b, h = C r, d^(-1) = 0, x = 0, best = b.
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
  cudaFuncSetAttribute(k_pcg<false, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)pcg_smem_bytes<float>());
  cudaFuncSetAttribute(k_pcg<true, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)pcg_smem_bytes<float>());
}

int pcg_max_grid(int device) {
  int nsm = 0, per = 0, per2 = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
  pcg_set_smem();
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_pcg<false, double>, pcg_threads<double>(),
                                                pcg_smem_bytes<double>());
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per2, k_pcg<true, double>, pcg_threads<double>(),
                                                pcg_smem_bytes<double>());
  per = std::min(per, per2);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per2, k_pcg<false, float>, pcg_threads<float>(),
                                                pcg_smem_bytes<float>());
  per = std::min(per, per2);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per2, k_pcg<true, float>, pcg_threads<float>(),
                                                pcg_smem_bytes<float>());
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
  const int wpc = L.blocks32 ? pcg_warps<float>() : pcg_warps<double>();
  int g = (L.nitems + wpc - 1) / wpc;
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
  if (L.blocks32)
    fn = co ? (const void *)k_pcg<true, float> : (const void *)k_pcg<false, float>;
  else
    fn = co ? (const void *)k_pcg<true, double> : (const void *)k_pcg<false, double>;
  const size_t smem = L.blocks32 ? pcg_smem_bytes<float>() : pcg_smem_bytes<double>();
  pcg_set_smem();
  const int nthreads = L.blocks32 ? pcg_threads<float>() : pcg_threads<double>();
  RPBA_CUDA_CHECK(cudaLaunchCooperativeKernel(fn, dim3(g), dim3(nthreads), args, smem, s));
  return 0;
}

}  // namespace rpba
