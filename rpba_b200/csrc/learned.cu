// learned.cu -- learned correction of the block-Jacobi preconditioner of the
// reduced camera system (RCS), and its training.
//
// The reference preconditions its PCG with C_k = S_kk^-1 (rbacore.cpp:1841).
// Block-Jacobi ignores the coupling of camera k to its neighbours; the
// diagonal block of S^-1, which an ideal block-diagonal preconditioner would
// use, is larger wherever the coupling is strong.  A small network predicts,
// per camera block, a per-parameter scaling s (9 values, exp(ALPHA tanh o))
// and the preconditioner becomes
//     C_k = diag(s) S_kk^-1 diag(s)          (SPD for every output)
// from scale-free features of the assembled system:
//   f[0..8]   log S_kk[a][a] minus their mean over the block's parameters
//   f[9..17]  log(1 + sum_l sum_c |S_kl[a][c]| / sqrt(S_kk[a][a] S_ll[c][c]))
//   f[18]     log(1 + number of covisible cameras) / 4
// Network: h = tanh(W1 f + b1) (64), o = W2 h + b2 (9); weights are rounded
// to BF16 for inference and accumulated in FP32.
//
// Training: the systems the direct solver's own LM iterations assemble
// (with the exact steps x* for reporting) are recorded into one diagonally
// scaled block-diagonal training system.  The objective is the relative
// A-norm error left after one preconditioned step on right-hand sides b (the
// LM step's and random ones), a quantity CG's convergence rests on; see the
// training section below.  Forward/backward run one thread per block row;
// weight gradients are reduced over all rows in a fixed order (one thread
// per weight), then an Adam step.
#include <cuda_bf16.h>

#include <cmath>
#include <vector>

#include "internal.h"

namespace rpba {

namespace {

constexpr float ALPHA = 1.0f;

__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// 1 / sqrt of the diagonal entries of every camera block (0 past the
// camera's parameter count), for the normalised couplings of the features.
// The diagonal is damped (+1e-2), so the clamp never binds on a real entry.
__global__ void k_diag_rsqrt(DevLSA L, double *drs) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = i / 9, a = i % 9;
  if (k >= L.nimg) return;
  drs[i] = (k >= L.begini && a < L.camparv[k + 1] - L.camparv[k]) ? 1. / sqrt(fmax(blk_at(L, (size_t)k, a * 10), 1e-300))
                                                                   : 0.;
}

// Features of camera row k (>= begini) of the assembled system, computed by
// one warp.  Lane l owns the block elements e = l, l + 32, l + 64 of every
// off-diagonal block of the row (coalesced reads of the 81 values) and keeps
// their normalised magnitudes in two accumulators, for the block stored as
// (k, l) and as (l, k); the coupling sum of parameter a is then reduced over
// the lanes in a fixed butterfly order.  Every lane returns the same f.
// drs: 1 / sqrt of every camera block's diagonal entries (k_diag_rsqrt).
__device__ void block_features(const DevLSA &L, const double *__restrict__ drs, int k, int lane, float f[NN_F]) {
  const int np = L.camparv[k + 1] - L.camparv[k];
  {
    // f[0..8] first, so that only nine floats stay live through the walk
    double ld[9], mean = 0.;
#pragma unroll
    for (int a = 0; a < 9; ++a) {
      ld[a] = a < np ? log(fmax(blk_at(L, (size_t)k, a * 10), 1e-300)) : 0.;
      if (a < np) mean += ld[a];
    }
    mean /= (np > 0 ? np : 1);
#pragma unroll
    for (int a = 0; a < 9; ++a) f[a] = a < np ? (float)(ld[a] - mean) : 0.f;
  }
  // per owned slot: row i, column j of the stored block, and this row's
  // diagonal entry for either orientation
  int ei[3], ej[3];
  double rn[3], rt[3], an[3] = {0., 0., 0.}, at[3] = {0., 0., 0.};
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    const int e = lane + 32 * m;
    ei[m] = e < 81 ? e / 9 : 9;
    ej[m] = e < 81 ? e % 9 : 9;
    rn[m] = ei[m] < 9 ? drs[(size_t)k * 9 + ei[m]] : 0.;
    rt[m] = ej[m] < 9 ? drs[(size_t)k * 9 + ej[m]] : 0.;
  }
  // the row's entries eight at a time: their positions, block elements and
  // column scalings (as floats: features need no more) are all loaded
  // before any is used (independent loads in flight), then added in entry
  // order in FP64
  // (the next batch's entries are loaded one batch ahead, lane u entry u)
  constexpr int U = 8;
  const int t0 = L.rowoff[k], t1 = L.rowoff[k + 1];
  int2 enl = (lane < U && t0 + lane < t1) ? L.ent[t0 + lane] : make_int2(k, k);
  for (int tb = t0; tb < t1; tb += U) {
    int2 en[U];
    int nc[U];
    float v[U][3], rcv[U][3];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      en[u].x = __shfl_sync(0xffffffffu, enl.x, u);
      en[u].y = __shfl_sync(0xffffffffu, enl.y, u);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const bool tr = en[u].y < 0;
      const size_t B = (size_t)(en[u].y & 0x7fffffff);
      const double *rc = drs + (size_t)en[u].x * 9;
#pragma unroll
      for (int m = 0; m < 3; ++m) {
        const int i = ei[m], j = ej[m];
        v[u][m] = i < 9 ? (float)blk_at(L, B, i * 9 + j) : 0.f;
        rcv[u][m] = i < 9 ? (float)__ldg(rc + (tr ? i : j)) : 0.f;
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) nc[u] = L.camparv[en[u].x + 1] - L.camparv[en[u].x];
    {
      const int tn = tb + U + lane;
      enl = (lane < U && tn < t1) ? L.ent[tn] : make_int2(k, k);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (en[u].x == k) continue;  // the diagonal block (and the padding past the row)
      const bool tr = en[u].y < 0;
#pragma unroll
      for (int m = 0; m < 3; ++m) {
        const int i = ei[m], j = ej[m];
        if (i >= 9) continue;
        // stored (k, col): element (i, j) couples parameter i of k to j of
        // col; stored (col, k): it couples parameter j of k to i of col; both
        // normalised by the two diagonal entries, |S_ij| / sqrt(S_ii S_jj)
        if (!tr) {
          if (i < np && j < nc[u]) an[m] += fabs((double)v[u][m]) * rn[m] * (double)rcv[u][m];
        } else {
          if (j < np && i < nc[u]) at[m] += fabs((double)v[u][m]) * rt[m] * (double)rcv[u][m];
        }
      }
    }
  }
  double cpl[9];
#pragma unroll
  for (int a = 0; a < 9; ++a) {
    double v = 0.;
#pragma unroll
    for (int m = 0; m < 3; ++m) v += (ei[m] == a ? an[m] : 0.) + (ej[m] == a ? at[m] : 0.);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    cpl[a] = v;
  }
  const int deg = L.rowoff[k + 1] - L.rowoff[k] - 1;  // entries besides the diagonal block
#pragma unroll
  for (int a = 0; a < 9; ++a) f[9 + a] = a < np ? (float)log1p(cpl[a]) : 0.f;
  f[18] = (float)(log1p((double)deg) / 4.);
}

// Network forward: s (per-parameter scaling) and the tanh hidden layer.
__device__ __forceinline__ void mlp_forward(const float *W, const float f[NN_F], float h[NN_H], float o[NN_O],
                                            float s[NN_O]) {
  const float *W1 = W, *b1 = W + NN_H * NN_F, *W2 = b1 + NN_H, *b2 = W2 + NN_O * NN_H;
  for (int i = 0; i < NN_H; ++i) {
    float a = b1[i];
#pragma unroll
    for (int j = 0; j < NN_F; ++j) a += W1[i * NN_F + j] * f[j];
    h[i] = tanhf(a);
  }
  for (int i = 0; i < NN_O; ++i) {
    float a = b2[i];
    for (int j = 0; j < NN_H; ++j) a += W2[i * NN_H + j] * h[j];
    o[i] = a;
    s[i] = expf(ALPHA * tanhf(a));
  }
}

// The same forward pass by one warp (hidden units lane and lane + 32; the
// output sums run over the hidden units in order, as in mlp_forward); every
// lane returns the same s.
__device__ __forceinline__ void mlp_forward_warp(const float *W, const float f[NN_F], int lane, float s[NN_O]) {
  const float *W1 = W, *b1 = W + NN_H * NN_F, *W2 = b1 + NN_H, *b2 = W2 + NN_O * NN_H;
  float h2[2];
  for (int u = 0; u < 2; ++u) {
    const int i = lane + 32 * u;
    float a = b1[i];
#pragma unroll
    for (int j = 0; j < NN_F; ++j) a += W1[i * NN_F + j] * f[j];
    h2[u] = tanhf(a);
  }
  float o[NN_O];
#pragma unroll
  for (int i = 0; i < NN_O; ++i) o[i] = b2[i];
#pragma unroll
  for (int u = 0; u < 2; ++u)
    for (int jj = 0; jj < 32; ++jj) {
      const int j = 32 * u + jj;
      const float hj = __shfl_sync(0xffffffffu, h2[u], jj);
#pragma unroll
      for (int i = 0; i < NN_O; ++i) o[i] += W2[i * NN_H + j] * hj;
    }
#pragma unroll
  for (int i = 0; i < NN_O; ++i) s[i] = expf(ALPHA * tanhf(o[i]));
}

// Features of every camera row >= begini, one warp per row (block_features),
// to feat[k * NN_FS ..]: a kernel of its own, so that its loads run at the
// occupancy of a small register count.
constexpr int NN_FS = 20;  // floats per row of feat
__global__ void __launch_bounds__(128) k_learned_features(DevLSA L, const double *drs, float *feat) {
  const int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (k >= L.nimg || k < L.begini) return;
  float f[NN_F];
  block_features(L, drs, k, lane, f);
  float v = 0.f;
#pragma unroll
  for (int j = 0; j < NN_F; ++j)
    if (lane == j) v = f[j];
  if (lane < NN_F) feat[(size_t)k * NN_FS + lane] = v;
}

// PCG start with the learned preconditioner (replaces k_pcg_setup), one
// warp per camera row: C_k = diag(s) S_kk^-1 diag(s) with S_kk^-1 from
// lu_inverse9_warp and s from the network on the row's features
// (k_learned_features); W == nullptr gives plain block-Jacobi.
__global__ void k_learned_setup(DevLSA L, PcgWork Wk, const float *weights) {
  __shared__ float Ws[NN_WEIGHTS];
  for (int i = threadIdx.x; i < NN_WEIGHTS; i += blockDim.x) Ws[i] = weights ? bf16r(weights[i]) : 0.f;
  __syncthreads();
  const int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (k >= L.nimg) return;
  double *C = Wk.Cinv + (size_t)k * 81;
  const size_t o = (size_t)k * 9;
  if (lane < 9) Wk.d[o + lane] = 0.;
  if (k < L.begini) {
    if (lane < 9) Wk.r[o + lane] = Wk.h[o + lane] = Wk.x[o + lane] = Wk.xbest[o + lane] = 0.;
    return;
  }
  const int np = L.camparv[k + 1] - L.camparv[k];
  {
    double row[9];
#pragma unroll
    for (int c = 0; c < 9; ++c) row[c] = lane < 9 ? blk_at(L, (size_t)k, lane * 9 + c) : 0.;
    lu_inverse9_warp(np, row, C, lane);
  }
  float sc[NN_O];
#pragma unroll
  for (int a = 0; a < NN_O; ++a) sc[a] = 1.f;
  if (weights) {
    const float fl = lane < NN_F ? Wk.feat[(size_t)k * NN_FS + lane] : 0.f;
    float f[NN_F];
#pragma unroll
    for (int j = 0; j < NN_F; ++j) f[j] = __shfl_sync(0xffffffffu, fl, j);
    mlp_forward_warp(Ws, f, lane, sc);
  }
  __syncwarp();
  if (lane < 9) {
    const int a = lane;
    float sa = 1.f;
#pragma unroll
    for (int j = 0; j < NN_O; ++j)
      if (j == a) sa = sc[j];
    double sum = 0.;
#pragma unroll
    for (int c = 0; c < 9; ++c) {
      double cv = C[a * 9 + c];
      if (weights && a < np && c < np) {
        cv *= (double)sa * (double)sc[c];
        C[a * 9 + c] = cv;
      }
      sum += cv * L.rhs[o + c];
    }
    Wk.r[o + a] = L.rhs[o + a];
    Wk.h[o + a] = sum;
    Wk.x[o + a] = 0.;
    Wk.xbest[o + a] = L.rhs[o + a];
  }
}

__device__ __forceinline__ double hash_normal(unsigned long long seed, unsigned long long i) {
  // two rounds of splitmix64 -> Box-Muller
  auto mix = [](unsigned long long z) {
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
  };
  const unsigned long long a = mix(seed ^ (i * 2 + 1)), b = mix(seed ^ (i * 2 + 2) ^ 0x5bd1e995ull);
  const double u1 = ((a >> 11) + 0.5) * (1.0 / 9007199254740992.0);
  const double u2 = (b >> 11) * (1.0 / 9007199254740992.0);
  return sqrt(-2. * log(u1)) * cos(6.283185307179586 * u2);
}

// ---------------------------------------------------------------- training
// The training set is the disjoint union of recorded systems, diagonally
// scaled: S~ = D^-1/2 S D^-1/2 (unit diagonal), Sinv~_k = D^1/2 S_kk^-1 D^1/2,
// b~ = D^-1/2 b.  The objective is invariant under this scaling.  Per
// system and right-hand side b (the LM step's, and random ones), with
// u = C b, v = S u, p = b^T u, q = u^T v:
//     loss = ln q - 2 ln p   ( = ln(1 - e) + const, e = relative A-norm error
//                              left after one preconditioned steepest-descent
//                              step from x = 0)
//     dloss/du = 2 v / q - 2 b / p   (S symmetric: no second product)
// and, per block, with y = Sinv (s o b), u = s o y:
//     dloss/ds_j = g_j y_j + b_j (Sinv^T (s o g))_j.

__global__ void k_t_forward(TrainSet T, const float *W, float *sv, float *ov, float *hv) {
  __shared__ float Ws[NN_WEIGHTS];
  for (int i = threadIdx.x; i < NN_WEIGHTS; i += blockDim.x) Ws[i] = W[i];
  __syncthreads();
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= T.rows) return;
  float f[NN_F], h[NN_H], o[NN_O], sc[NN_O];
  for (int j = 0; j < NN_F; ++j) f[j] = T.f[(size_t)r * NN_F + j];
  mlp_forward(Ws, f, h, o, sc);
  const int np = T.np[r];
  for (int j = 0; j < NN_O; ++j) {
    sv[(size_t)r * NN_O + j] = j < np ? sc[j] : 1.f;
    ov[(size_t)r * NN_O + j] = o[j];
  }
  for (int j = 0; j < NN_H; ++j) hv[(size_t)r * NN_H + j] = h[j];
}

// u_p = s o (Sinv (s o b_p)) + uc_p for every row and right-hand side
__global__ void k_t_apply(TrainSet T, const float *sv, float *u) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = i % T.rows, pr = i / T.rows;
  if (pr >= T.probes) return;
  // right-hand sides are strided by the capacity, work vectors by the rows
  const float *Si = T.sinv + (size_t)r * 81, *b = T.b + ((size_t)pr * T.rows_cap + r) * 9, *sc = sv + (size_t)r * 9;
  float w[9];
  for (int a = 0; a < 9; ++a) w[a] = sc[a] * b[a];
  for (int a = 0; a < 9; ++a) {
    float t = 0.f;
    for (int c = 0; c < 9; ++c) t += Si[a * 9 + c] * w[c];
    const float cu = T.uc ? T.uc[((size_t)pr * T.rows_cap + r) * 9 + a] : 0.f;
    u[((size_t)pr * T.rows + r) * 9 + a] = sc[a] * t + cu;
  }
}

// v_p = S~ u_p (one warp per row and right-hand side, 27 lanes)
__global__ void k_t_spmv(TrainSet T, const float *u, float *v) {
  const long long wg = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31, grp = lane / 9, rr = lane % 9;
  const int r = (int)(wg % T.rows), pr = (int)(wg / T.rows);
  if (pr >= T.probes) return;
  const float *uu = u + (size_t)pr * T.rows * 9;
  float acc = 0.f;
  if (lane < 27)
    for (int e = T.rowoff[r] + grp; e < T.rowoff[r + 1]; e += 3) {
      const int2 en = T.ent[e];
      const float *B = T.blocks + (size_t)(en.y & 0x7fffffff) * 81;
      const float *x = uu + (size_t)en.x * 9;
      if (en.y >= 0)
        for (int c = 0; c < 9; ++c) acc += B[rr * 9 + c] * x[c];
      else
        for (int c = 0; c < 9; ++c) acc += B[c * 9 + rr] * x[c];
    }
  const float a1 = __shfl_down_sync(0xffffffffu, acc, 9);
  const float a2 = __shfl_down_sync(0xffffffffu, acc, 18);
  if (lane < 9) v[((size_t)pr * T.rows + r) * 9 + lane] = acc + a1 + a2;
}

// p = b^T u, q = u^T v and b^T x* per system and right-hand side (one CTA
// each, fixed-order reduction)
__global__ void k_t_dots(TrainSet T, const float *u, const float *v, double *pq) {
  const int sys = blockIdx.x % T.systems, pr = blockIdx.x / T.systems;
  __shared__ double sh[3][256];
  double a = 0., b2 = 0., c = 0.;
  const int r0 = T.sys_row[sys], r1 = T.sys_row[sys + 1];
  for (int r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
    const size_t o = ((size_t)pr * T.rows + r) * 9, ob = ((size_t)pr * T.rows_cap + r) * 9;
    for (int j = 0; j < 9; ++j) {
      a += (double)T.b[ob + j] * u[o + j];
      b2 += (double)u[o + j] * v[o + j];
      if (pr == 0) c += (double)T.b[ob + j] * T.xs[(size_t)r * 9 + j];
    }
  }
  sh[0][threadIdx.x] = a;
  sh[1][threadIdx.x] = b2;
  sh[2][threadIdx.x] = c;
  __syncthreads();
  for (int st = 128; st > 0; st >>= 1) {
    if (threadIdx.x < st)
      for (int j = 0; j < 3; ++j) sh[j][threadIdx.x] += sh[j][threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    pq[3 * blockIdx.x] = sh[0][0];
    pq[3 * blockIdx.x + 1] = sh[1][0];
    pq[3 * blockIdx.x + 2] = sh[2][0];
  }
}

// per row: dloss/ds summed over right-hand sides, back through the network
__global__ void k_t_backward(TrainSet T, const float *W, const float *sv, const float *ov, const float *hv,
                             const float *u, const float *v, const double *pq, float *d2, float *d1) {
  __shared__ float W2s[NN_O * NN_H];
  const float *W2 = W + NN_H * NN_F + NN_H;
  for (int i = threadIdx.x; i < NN_O * NN_H; i += blockDim.x) W2s[i] = W2[i];
  __syncthreads();
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= T.rows) return;
  const int sys = T.sys[r], np = T.np[r];
  const float *Si = T.sinv + (size_t)r * 81, *sc = sv + (size_t)r * 9;
  const float scale = 1.f / (float)(T.systems * T.probes);
  float ds[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int pr = 0; pr < T.probes; ++pr) {
    const size_t o = ((size_t)pr * T.rows + r) * 9, ob = ((size_t)pr * T.rows_cap + r) * 9;
    const double *P = pq + 3 * ((size_t)pr * T.systems + sys);
    const float ip = (float)(1. / P[0]), iq = (float)(1. / P[1]);
    float g[9], y[9], sg[9];
    for (int a = 0; a < 9; ++a) {
      g[a] = (2.f * v[o + a] * iq - 2.f * T.b[ob + a] * ip) * scale;
      const float cu = T.uc ? T.uc[ob + a] : 0.f;
      y[a] = sc[a] != 0.f ? (u[o + a] - cu) / sc[a] : 0.f;
      sg[a] = sc[a] * g[a];
    }
    for (int j = 0; j < np; ++j) {
      float t = 0.f;
      for (int a = 0; a < 9; ++a) t += Si[a * 9 + j] * sg[a];
      ds[j] += g[j] * y[j] + T.b[ob + j] * t;
    }
  }
  float dout[NN_O];
  for (int j = 0; j < NN_O; ++j) {
    const float th = tanhf(ov[(size_t)r * NN_O + j]);
    dout[j] = j < np ? ds[j] * ALPHA * sc[j] * (1.f - th * th) : 0.f;
    d2[(size_t)r * NN_O + j] = dout[j];
  }
  for (int i = 0; i < NN_H; ++i) {
    float t = 0.f;
    for (int j = 0; j < NN_O; ++j) t += W2s[j * NN_H + i] * dout[j];
    const float h = hv[(size_t)r * NN_H + i];
    d1[(size_t)r * NN_H + i] = t * (1.f - h * h);
  }
}

// One thread per weight: sum over the rows in a fixed order.
__global__ void k_grad_reduce(TrainSet T, const float *d2, const float *d1, const float *hv, float *grad) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= NN_WEIGHTS) return;
  float acc = 0.f;
  const int nW1 = NN_H * NN_F, nb1 = NN_H, nW2 = NN_O * NN_H;
  const int R = T.rows;
  if (w < nW1) {
    const int i = w / NN_F, j = w % NN_F;
    for (int r = 0; r < R; ++r) acc += d1[(size_t)r * NN_H + i] * T.f[(size_t)r * NN_F + j];
  } else if (w < nW1 + nb1) {
    const int i = w - nW1;
    for (int r = 0; r < R; ++r) acc += d1[(size_t)r * NN_H + i];
  } else if (w < nW1 + nb1 + nW2) {
    const int q = w - nW1 - nb1, i = q / NN_H, j = q % NN_H;
    for (int r = 0; r < R; ++r) acc += d2[(size_t)r * NN_O + i] * hv[(size_t)r * NN_H + j];
  } else {
    const int i = w - nW1 - nb1 - nW2;
    for (int r = 0; r < R; ++r) acc += d2[(size_t)r * NN_O + i];
  }
  grad[w] = acc;
}

__global__ void k_adam(float *W, float *m, float *v, const float *grad, float lr, float b1, float b2, float eps,
                       int t) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= NN_WEIGHTS) return;
  const float g = grad[i];
  m[i] = b1 * m[i] + (1.f - b1) * g;
  v[i] = b2 * v[i] + (1.f - b2) * g * g;
  const float mh = m[i] / (1.f - powf(b1, (float)t)), vh = v[i] / (1.f - powf(b2, (float)t));
  W[i] -= lr * mh / (sqrtf(vh) + eps);
}

// ---- recording a system into the training set
// One warp per row of the system being recorded (FP64 form): features, the
// scaled block inverse (LU by lane 0 into the FP64 scratch Si, then scaled
// by lanes 0..8), right-hand sides and the scaled solution.
__global__ void k_rec_rows(DevLSA L, TrainSet T, int row0, int sys, const double *xstar, unsigned long long seed,
                           double *Si, const double *drs) {
  const int k = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) + L.begini, lane = threadIdx.x & 31;
  if (k >= L.nimg) return;
  const int r = row0 + (k - L.begini);
  float f[NN_F];
  block_features(L, drs, k, lane, f);
  const int np = L.camparv[k + 1] - L.camparv[k];
  const double *D = L.blocks + (size_t)k * 81;
  double *Sk = Si + (size_t)k * 81;
  if (lane == 0) {
    for (int j = 0; j < NN_F; ++j) T.f[(size_t)r * NN_F + j] = f[j];
    T.np[r] = np;
    T.sys[r] = sys;
    lu_inverse9(np, D, Sk);
  }
  __syncwarp();
  if (lane >= 9) return;
  const int a = lane;
  const double sqa = a < np ? sqrt(D[a * 10]) : 1.;
  for (int c = 0; c < 9; ++c) {
    const double sqc = c < np ? sqrt(D[c * 10]) : 1.;
    T.sinv[(size_t)r * 81 + a * 9 + c] = (a < np && c < np) ? (float)(sqa * Sk[a * 9 + c] * sqc) : 0.f;
  }
  // right-hand side 0: the LM step's (b~ = D^-1/2 b, x~* = D^1/2 x*)
  T.b[(size_t)r * 9 + a] = a < np ? (float)(L.rhs[(size_t)k * 9 + a] / sqa) : 0.f;
  T.xs[(size_t)r * 9 + a] = a < np ? (float)(xstar[(size_t)k * 9 + a] * sqa) : 0.f;
  for (int pr = 1; pr < T.probes; ++pr)
    T.b[((size_t)pr * T.rows_cap + r) * 9 + a] =
        a < np ? (float)hash_normal(seed + 7919ull * pr, (unsigned long long)r * 9 + a) : 0.f;
}

// scaled blocks: diagonal blocks of rows >= begini, then the off-diagonal
// blocks (row, col) given by rc
__global__ void k_rec_blocks(DevLSA L, TrainSet T, int blk0, const int2 *rc, int nb) {
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int nd = L.nimg - L.begini;
  const long long b = gid / 81;
  const int e = (int)(gid % 81), i = e / 9, j = e % 9;
  if (b >= nd + nb) return;
  int r, c;
  size_t src;
  if (b < nd) {
    r = c = (int)b + L.begini;
    src = (size_t)r;
  } else {
    r = rc[b - nd].x;
    c = rc[b - nd].y;
    src = (size_t)(L.nimg + (b - nd));
  }
  const int nr = L.camparv[r + 1] - L.camparv[r], nc = L.camparv[c + 1] - L.camparv[c];
  float v = 0.f;
  if (i < nr && j < nc)
    v = (float)(blk_at(L, src, e) / sqrt(blk_at(L, (size_t)r, i * 10) * blk_at(L, (size_t)c, j * 10)));
  T.blocks[(size_t)(blk0 + b) * 81 + e] = v;
}

// unscaled right-hand side pr of the system being recorded: b = D^1/2 b~
__global__ void k_rec_bvec(DevLSA L, TrainSet T, int row0, int pr, double *vb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = i / 9, a = i % 9;
  if (k >= L.nimg) return;
  double v = 0.;
  if (k >= L.begini && a < L.camparv[k + 1] - L.camparv[k])
    v = (double)T.b[((size_t)pr * T.rows_cap + row0 + (k - L.begini)) * 9 + a] *
        sqrt(blk_at(L, (size_t)k, a * 10));
  vb[i] = v;
}

// uc~ = D^1/2 z for the rows of the system being recorded
__global__ void k_rec_uc(DevLSA L, TrainSet T, int row0, int pr, const double *vz) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + L.begini * 9;
  const int k = i / 9, a = i % 9;
  if (k >= L.nimg) return;
  const int np = L.camparv[k + 1] - L.camparv[k];
  T.uc[((size_t)pr * T.rows_cap + row0 + (k - L.begini)) * 9 + a] =
      a < np ? (float)(vz[i] * sqrt(blk_at(L, (size_t)k, a * 10))) : 0.f;
}

}  // namespace

void learned_pcg_setup(const DevLSA &L, const PcgWork &W, const float *weights, cudaStream_t s) {
  if (weights) {
    k_diag_rsqrt<<<(L.nimg * 9 + 255) / 256, 256, 0, s>>>(L, W.drs);
    k_learned_features<<<(L.nimg + 3) / 4, 128, 0, s>>>(L, W.drs, W.feat);
  }
  k_learned_setup<<<(L.nimg + 7) / 8, 256, 0, s>>>(L, W, weights);
}

void learned_record(const DevLSA &L, const CoarseWork *coarse, const double *xstar, double *scratch, double *drs,
                    unsigned long long seed, TrainSet &T, TrainHost &H, cudaStream_t s) {
  if (!L.blocks) return;  // systems are recorded in the FP64 form only
  const int nimg = L.nimg, nd = nimg - L.begini, nb = L.nboff;
  if (nd <= 0) return;
  const int nent = [&] {
    int v = 0;
    RPBA_CUDA_CHECK(cudaMemcpyAsync(&v, L.rowoff + nimg, sizeof(int), cudaMemcpyDeviceToHost, s));
    RPBA_CUDA_CHECK(cudaStreamSynchronize(s));
    return v;
  }();
  if (T.rows + nd > T.rows_cap || H.ents + nent > H.ents_cap || H.blocks + nd + nb > H.blocks_cap ||
      T.systems + 1 > H.sys_cap)
    return;  // training set full: later systems are not recorded
  std::vector<int> rowoff(nimg + 1);
  std::vector<int2> ent(nent);
  RPBA_CUDA_CHECK(cudaMemcpyAsync(rowoff.data(), L.rowoff, sizeof(int) * (nimg + 1), cudaMemcpyDeviceToHost, s));
  RPBA_CUDA_CHECK(cudaMemcpyAsync(ent.data(), L.ent, sizeof(int2) * nent, cudaMemcpyDeviceToHost, s));
  RPBA_CUDA_CHECK(cudaStreamSynchronize(s));
  const int row0 = T.rows, blk0 = H.blocks;
  // block (row, col) of each off-diagonal block from the normal entries
  std::vector<int2> rc(std::max(nb, 1));
  std::vector<int> new_off(nd + 1);
  std::vector<int2> new_ent;
  new_ent.reserve(nent);
  for (int k = L.begini; k < nimg; ++k) {
    new_off[k - L.begini] = H.ents + (int)new_ent.size();
    for (int t = rowoff[k]; t < rowoff[k + 1]; ++t) {
      const int2 e = ent[t];
      const int col = e.x;
      const int bi = e.y & 0x7fffffff;
      int nbi;
      if (bi < nimg) {
        nbi = blk0 + (bi - L.begini);
      } else {
        nbi = blk0 + nd + (bi - nimg);
        if (e.y >= 0) rc[bi - nimg] = make_int2(k, col);
      }
      new_ent.push_back(make_int2(row0 + (col - L.begini), (int)((unsigned)nbi | (e.y < 0 ? 0x80000000u : 0u))));
    }
  }
  new_off[nd] = H.ents + (int)new_ent.size();
  RPBA_CUDA_CHECK(cudaMemcpyAsync(T.rowoff + row0, new_off.data(), sizeof(int) * (nd + 1), cudaMemcpyHostToDevice, s));
  RPBA_CUDA_CHECK(cudaMemcpyAsync(T.ent + H.ents, new_ent.data(), sizeof(int2) * new_ent.size(), cudaMemcpyHostToDevice, s));
  RPBA_CUDA_CHECK(cudaMemcpyAsync(H.rc, rc.data(), sizeof(int2) * std::max(nb, 1), cudaMemcpyHostToDevice, s));
  k_diag_rsqrt<<<(nimg * 9 + 255) / 256, 256, 0, s>>>(L, drs);
  k_rec_rows<<<(nd + 7) / 8, 256, 0, s>>>(L, T, row0, T.systems, xstar, seed, scratch, drs);
  const long long nthreads = (long long)(nd + nb) * 81;
  k_rec_blocks<<<(int)((nthreads + 255) / 256), 256, 0, s>>>(L, T, blk0, H.rc, nb);
  if (T.uc) {
    // coarse part of each preconditioned right-hand side (zero without a
    // coarse space)
    const int nv = nimg * 9;
    for (int pr = 0; pr < T.probes; ++pr) {
      k_rec_bvec<<<(nv + 255) / 256, 256, 0, s>>>(L, T, row0, pr, H.vb);
      RPBA_CUDA_CHECK(cudaMemsetAsync(H.vz, 0, sizeof(double) * nv, s));
      if (coarse) coarse_apply(L, *coarse, H.vb, H.vz, s);
      k_rec_uc<<<(nd * 9 + 255) / 256, 256, 0, s>>>(L, T, row0, pr, H.vz);
    }
  }
  RPBA_CUDA_CHECK(cudaStreamSynchronize(s));
  T.rows += nd;
  H.ents += (int)new_ent.size();
  H.blocks += nd + nb;
  H.sys_row.push_back(T.rows);
  T.systems += 1;
}

// Loss (mean over systems and right-hand sides of ln q - 2 ln p), the
// relative A-norm error of the LM steps' first preconditioned step, and the
// gradient.
void learned_loss_grad(const TrainSet &T, const float *W, TrainBufs &B, float *loss, float *err, cudaStream_t s) {
  k_t_forward<<<(T.rows + 127) / 128, 128, 0, s>>>(T, W, B.sv, B.ov, B.hv);
  const long long np = (long long)T.rows * T.probes;
  k_t_apply<<<(int)((np + 255) / 256), 256, 0, s>>>(T, B.sv, B.u);
  k_t_spmv<<<(int)((np * 32 + 255) / 256), 256, 0, s>>>(T, B.u, B.v);
  k_t_dots<<<T.systems * T.probes, 256, 0, s>>>(T, B.u, B.v, B.pq);
  k_t_backward<<<(T.rows + 127) / 128, 128, 0, s>>>(T, W, B.sv, B.ov, B.hv, B.u, B.v, B.pq, B.d2, B.d1);
  k_grad_reduce<<<(NN_WEIGHTS + 127) / 128, 128, 0, s>>>(T, B.d2, B.d1, B.hv, B.grad);
  if (loss || err) {
    std::vector<double> pq(3 * (size_t)T.systems * T.probes);
    RPBA_CUDA_CHECK(cudaMemcpyAsync(pq.data(), B.pq, sizeof(double) * pq.size(), cudaMemcpyDeviceToHost, s));
    RPBA_CUDA_CHECK(cudaStreamSynchronize(s));
    double l = 0., e = 0.;
    for (int i = 0; i < T.systems * T.probes; ++i) l += std::log(pq[3 * i + 1]) - 2. * std::log(pq[3 * i]);
    for (int i = 0; i < T.systems; ++i) e += 1. - pq[3 * i] * pq[3 * i] / (pq[3 * i + 1] * pq[3 * i + 2]);
    if (loss) *loss = (float)(l / (T.systems * T.probes));
    if (err) *err = (float)(e / T.systems);
  }
}

void learned_adam(float *W, float *m, float *v, const float *grad, float lr, int t, cudaStream_t s) {
  k_adam<<<(NN_WEIGHTS + 127) / 128, 128, 0, s>>>(W, m, v, grad, lr, 0.9f, 0.999f, 1e-8f, t);
}

}  // namespace rpba
