// exactsum.cu -- the reference's float accumulations (sig0 += term in
// rbacore.cpp:1327, wsum += w in :727 and :881), computed in parallel with a
// result bitwise equal to the sequential float loop.
//
// Method.  Let s be the running float sum, s in [2^E, 2^(E+1)), u = ulp(s) =
// 2^(E-23), S = s/u (an integer in [2^23, 2^24)).  For v >= 0 with
// S + floor(v/u) < 2^24 the float addition is fl(s + v) = s + u*rne(v/u),
// and rne(v/u) does not depend on s unless v/u is exactly halfway between
// integers (a tie, where round-half-even looks at the parity of S).  So
// inside one binade a whole run of additions is an exact integer prefix sum
// of r_k = rne(v_k/u).  The run ends at the first element k with a tie or
// with S + R_(k-1) + floor(v_k/u) >= 2^24 (the sum leaves the binade); that
// single element is added with a real float addition, and a new run starts
// with the new binade.  Runs are few (the sum leaves a binade only when it
// doubles; ties have probability ~ v/s), so the loop takes a handful of grid
// passes instead of n dependent additions.
//
// The first HEAD elements and any stretch where s is zero or subnormal are
// added by one warp in plain sequence.  Inputs must be finite and >= 0.
#include <mutex>

#include "../../include/rpba_b200.h"
#include "gridsync.cuh"
#include "internal.h"

namespace rpba {

namespace {

constexpr int ES_T = 256;
constexpr int HEAD = 2048;
constexpr long long RCLAMP = 1ll << 30;  // n * RCLAMP < 2^61 for n < 2^31
constexpr int MAX_SEGMENTS = 512;

struct EsCtl {
  float s;    // running sum before element i
  int i;      // next element
};

struct EsArgs {
  const float *v;
  int n;
  float *out;
  long long *Rc, *Mc;  // per CTA: sum of r, max of (exclusive prefix + floor)
  int *Tc;             // per CTA: first tie index (INT_MAX if none)
  EsCtl *ctl;
  unsigned *bar;
  int *err;
};

__device__ __forceinline__ void classify(float v, double scale, long long &fl, long long &r, bool &tie) {
  const double f = (double)v * scale;
  if (f >= (double)RCLAMP) {
    fl = r = RCLAMP;
    tie = false;
    return;
  }
  const double ff = floor(f);
  const double fr = f - ff;
  fl = (long long)ff;
  tie = fr == 0.5;
  r = fl + (fr > 0.5 ? 1 : 0);
}

// Sequential float additions of v[i..i_end) onto s by one warp.
__device__ float warp_seq(const float *v, int i, int i_end, float s) {
  const int lane = threadIdx.x & 31;
  for (int base = i; base < i_end; base += 32) {
    const int idx = base + lane;
    const float x = idx < i_end ? v[idx] : 0.f;
#pragma unroll 8
    for (int l = 0; l < 32; ++l) {
      const float t = __shfl_sync(0xffffffffu, x, l);
      if (base + l < i_end) s = __fadd_rn(s, t);
    }
  }
  return s;
}

__global__ void __launch_bounds__(ES_T) k_exact_sum(EsArgs A) {
  const int G = gridDim.x, c = blockIdx.x, tid = threadIdx.x;
  const int n = A.n;
  const int chunk = (n + G - 1) / G;
  const int lo = min(n, c * chunk), hi = min(n, lo + chunk);
  const int per = (chunk + ES_T - 1) / ES_T;
  __shared__ long long s_off[ES_T];  // per-thread exclusive offsets within the chunk
  __shared__ long long s_tsum[ES_T];
  __shared__ long long s_tmax[ES_T];
  __shared__ int s_ttie[ES_T];
  __shared__ long long s_roff;       // exclusive prefix of r over earlier chunks
  __shared__ int s_cx, s_ct, s_tmin;
  __shared__ long long s_rtot;
  __shared__ int s_kx;

  if (c == 0 && tid < 32) {
    float s = warp_seq(A.v, 0, min(n, HEAD), 0.f);
    int i = min(n, HEAD);
    // leave the zero / subnormal range one element at a time
    while (i < n && !(s >= 1.17549435e-38f) && isfinite(s)) {
      s = __fadd_rn(s, A.v[i]);
      ++i;
    }
    if (tid == 0) {
      A.ctl->s = s;
      A.ctl->i = isfinite(s) ? i : n;
    }
  }
  if (!grid_barrier(A.bar, G, A.err)) return;

  for (int seg = 0;; ++seg) {
    const float s = __ldcg(&A.ctl->s);
    const int i0 = __ldcg(&A.ctl->i);
    if (i0 >= n) break;
    if (seg >= MAX_SEGMENTS) {
      // pathological input (a tie at nearly every element): finish in plain
      // sequence, still exact
      if (c == 0 && tid < 32) {
        const float sr = warp_seq(A.v, i0, n, s);
        if (tid == 0) A.ctl->s = sr;
      }
      break;
    }
    int E;
    frexpf(s, &E);
    E -= 1;  // s in [2^E, 2^(E+1))
    const double u = ldexp(1.0, E - 23);
    const double scale = ldexp(1.0, 23 - E);
    const long long S = (long long)((double)s * scale);
    const long long TOP = 1ll << 24;

    // phase A: per thread contiguous sub-range of this chunk, from max(lo, i0)
    const int a0 = max(lo, i0);
    const int t_lo = lo + tid * per, t_hi = min(hi, t_lo + per);
    long long tsum = 0, tmax = LLONG_MIN;
    int ttie = INT_MAX;
    for (int k = max(t_lo, a0); k < t_hi; ++k) {
      long long fl, r;
      bool tie;
      classify(A.v[k], scale, fl, r, tie);
      const long long m = tsum + fl;
      if (m > tmax) tmax = m;
      if (tie && k < ttie) ttie = k;
      tsum += r;
    }
    s_tsum[tid] = tsum;
    s_tmax[tid] = tmax;
    s_ttie[tid] = ttie;
    __syncthreads();
    if (tid == 0) {
      long long acc = 0, mx = LLONG_MIN;
      int tt = INT_MAX;
      for (int t = 0; t < ES_T; ++t) {
        s_off[t] = acc;
        if (s_tmax[t] != LLONG_MIN && acc + s_tmax[t] > mx) mx = acc + s_tmax[t];
        if (s_ttie[t] < tt) tt = s_ttie[t];
        acc += s_tsum[t];
      }
      A.Rc[c] = acc;
      A.Mc[c] = mx;
      A.Tc[c] = tt;
    }
    if (!grid_barrier(A.bar, G, A.err)) return;

    // phase B (every CTA, warp 0): chunk prefix, first crossing chunk, first tie
    if (tid < 32) {
      const int cper = (G + 31) / 32;
      const int c0 = tid * cper, c1 = min(G, c0 + cper);
      long long lsum = 0;
      for (int q = c0; q < c1; ++q) lsum += __ldcg(A.Rc + q);
      long long incl = lsum;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const long long y = __shfl_up_sync(0xffffffffu, incl, o);
        if (tid >= o) incl += y;
      }
      long long off = incl - lsum;
      int cx = INT_MAX, tmin = INT_MAX;
      for (int q = c0; q < c1; ++q) {
        const long long mq = __ldcg(A.Mc + q);
        if (cx == INT_MAX && mq != LLONG_MIN && S + off + mq >= TOP) cx = q;
        const int tq = __ldcg(A.Tc + q);
        if (tq < tmin) tmin = tq;
        if (q == c) s_roff = off;
        off += __ldcg(A.Rc + q);
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        cx = min(cx, __shfl_xor_sync(0xffffffffu, cx, o));
        tmin = min(tmin, __shfl_xor_sync(0xffffffffu, tmin, o));
      }
      const long long tot = __shfl_sync(0xffffffffu, incl, 31);
      if (tid == 0) {
        s_cx = cx;
        s_tmin = tmin;
        s_ct = tmin == INT_MAX ? INT_MAX : tmin / chunk;
        s_rtot = tot;
      }
    }
    __syncthreads();
    const int cx = s_cx, ct = s_ct, tmin = s_tmin;
    const int ev_cta = (cx == INT_MAX && ct == INT_MAX) ? 0 : (ct < cx ? ct : cx);
    if (c == ev_cta) {
      const long long roff = s_roff;
      if (cx == INT_MAX && ct == INT_MAX) {
        if (tid == 0) {
          A.ctl->s = (float)((double)(S + s_rtot) * u);
          A.ctl->i = n;
        }
      } else {
        // first crossing inside this chunk (when it is the crossing chunk)
        if (tid == 0) s_kx = INT_MAX;
        __syncthreads();
        if (c == cx) {
          long long run = roff + s_off[tid];
          for (int k = max(t_lo, a0); k < t_hi; ++k) {
            long long fl, r;
            bool tie;
            classify(A.v[k], scale, fl, r, tie);
            if (S + run + fl >= TOP) {
              atomicMin(&s_kx, k);
              break;
            }
            run += r;
          }
        }
        __syncthreads();
        const int kstar = min(s_kx, tmin);
        // the thread owning kstar adds it with a float addition
        if (kstar >= max(t_lo, a0) && kstar < t_hi) {
          long long run = roff + s_off[tid];
          for (int k = max(t_lo, a0); k < kstar; ++k) {
            long long fl, r;
            bool tie;
            classify(A.v[k], scale, fl, r, tie);
            run += r;
          }
          const float sb = (float)((double)(S + run) * u);
          const float sn = __fadd_rn(sb, A.v[kstar]);
          A.ctl->s = sn;
          A.ctl->i = isfinite(sn) ? kstar + 1 : n;
        }
      }
    }
    if (!grid_barrier(A.bar, G, A.err)) return;
    // a new run that starts in the zero/subnormal range is continued in sequence
    if (c == 0 && tid < 32) {
      float s2 = __ldcg(&A.ctl->s);
      int i2 = __ldcg(&A.ctl->i);
      bool moved = false;
      while (i2 < n && !(s2 >= 1.17549435e-38f)) {
        s2 = __fadd_rn(s2, A.v[i2]);
        ++i2;
        moved = true;
      }
      if (moved && tid == 0) {
        A.ctl->s = s2;
        A.ctl->i = i2;
      }
    }
    if (!grid_barrier(A.bar, G, A.err)) return;
  }
  if (c == 0 && tid == 0) *A.out = __ldcg(&A.ctl->s);
}

// Sequential float sum by one warp, for short arrays.
__global__ void k_warp_sum(const float *v, int n, float *out) {
  const float s = warp_seq(v, 0, n, 0.f);
  if (threadIdx.x == 0) *out = s;
}

}  // namespace

int exact_sum_max_grid(int device) {
  int nsm = 0, per = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_exact_sum, ES_T, 0);
  if (per < 1) per = 1;
  return nsm * (per < 2 ? per : 2);
}

void launch_exact_sum(const float *v, int n, float *out, const ExactSumWork &W, cudaStream_t s) {
  if (n <= 4 * HEAD) {
    k_warp_sum<<<1, 32, 0, s>>>(v, n, out);
    return;
  }
  int G = (n + 4095) / 4096;
  if (G > W.max_grid) G = W.max_grid;
  if (G < 1) G = 1;
  EsArgs A;
  A.v = v;
  A.n = n;
  A.out = out;
  A.Rc = W.Rc;
  A.Mc = W.Mc;
  A.Tc = W.Tc;
  A.ctl = (EsCtl *)W.ctl;
  A.bar = W.bar;
  A.err = W.err;
  RPBA_CUDA_CHECK(cudaMemsetAsync(W.bar, 0, 2 * sizeof(unsigned), s));
  void *args[] = {&A};
  RPBA_CUDA_CHECK(cudaLaunchCooperativeKernel((const void *)k_exact_sum, dim3(G), dim3(ES_T), args, 0, s));
}

}  // namespace rpba

// ---------------------------------------------------------------------------
// Allocation-free variant of the exact float sum.
//
// Some callers cannot let a library call cudaMalloc or cudaFree: a host
// application that hands all device memory out of its own fixed-budget pool
// (a stray cudaMalloc breaks its accounting or fails when the pool owns the
// whole device), or a latency-critical loop that cannot absorb the
// device-wide synchronisation cudaFree implies.  For them this entry point
// keeps its scratch -- the per-CTA run sums, the run control word and the
// grid-barrier counters of k_exact_sum -- in one statically sized device
// array that every GPU loading the library holds until the process exits
// (about 20 KB).  Its size caps the input at NA_MAX_CTAS CTAs of NA_CHUNK
// elements each.
using namespace rpba;

namespace {

constexpr int NA_MAX_CTAS = 1024;
constexpr int NA_CHUNK = 4096;
constexpr long long NA_MAX_N = (long long)NA_MAX_CTAS * NA_CHUNK;  // 4,194,304
constexpr size_t NA_OFF_RC = 0;
constexpr size_t NA_OFF_MC = NA_OFF_RC + sizeof(long long) * NA_MAX_CTAS;
constexpr size_t NA_OFF_TC = NA_OFF_MC + sizeof(long long) * NA_MAX_CTAS;
constexpr size_t NA_OFF_CTL = NA_OFF_TC + sizeof(int) * NA_MAX_CTAS;
constexpr size_t NA_OFF_BAR = NA_OFF_CTL + 16;
constexpr size_t NA_OFF_ERR = NA_OFF_BAR + 16;
constexpr size_t NA_BYTES = NA_OFF_ERR + 16;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_BYTES];

constexpr int NA_MAX_DEVICES = 64;
std::mutex g_na_mutex;
unsigned char *g_na_addr[NA_MAX_DEVICES];  // device address of the scratch, per device

}  // namespace

extern "C" int32_t rpba_float_sequential_sum_noalloc(const float *d_v, int64_t n, float *d_out, void *stream) {
  if (!d_out || n < 0 || (n > 0 && !d_v)) return RPBA_ERR_ARG;
  if (n > NA_MAX_N) return RPBA_ERR_TOO_LARGE;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return RPBA_ERR_NO_DEVICE;
  if (dev < 0 || dev >= NA_MAX_DEVICES) return RPBA_ERR_UNSUPPORTED;
  cudaStream_t s = (cudaStream_t)stream;
  unsigned char *base;
  {
    // set-up, once per device, with that device current: the array's name
    // is only a host-side stand-in, so its device address is looked up
    std::lock_guard<std::mutex> lock(g_na_mutex);
    if (!g_na_addr[dev]) {
      void *p = nullptr;
      if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return RPBA_ERR_CUDA;
      g_na_addr[dev] = (unsigned char *)p;
    }
    base = g_na_addr[dev];
  }
  const int ni = (int)n;
  if (ni <= 4 * HEAD) {
    k_warp_sum<<<1, 32, 0, s>>>(d_v, ni, d_out);
    return cudaGetLastError() == cudaSuccess ? RPBA_OK : RPBA_ERR_CUDA;
  }
  const int G = (ni + NA_CHUNK - 1) / NA_CHUNK;
  int nsm = 0, per = 0;
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_exact_sum, ES_T, 0) != cudaSuccess)
    return RPBA_ERR_CUDA;
  if (G > nsm * per) return RPBA_ERR_TOO_LARGE;  // the CTAs would not all be resident
  EsArgs A;
  A.v = d_v;
  A.n = ni;
  A.out = d_out;
  A.Rc = (long long *)(base + NA_OFF_RC);
  A.Mc = (long long *)(base + NA_OFF_MC);
  A.Tc = (int *)(base + NA_OFF_TC);
  A.ctl = (EsCtl *)(base + NA_OFF_CTL);
  A.bar = (unsigned *)(base + NA_OFF_BAR);
  A.err = (int *)(base + NA_OFF_ERR);
  // the array keeps the previous call's contents: the barrier counters and
  // the error word must start at zero; the rest is written before it is read
  if (cudaMemsetAsync(A.bar, 0, 2 * sizeof(unsigned), s) != cudaSuccess ||
      cudaMemsetAsync(A.err, 0, sizeof(int), s) != cudaSuccess)
    return RPBA_ERR_CUDA;
  void *args[] = {&A};
  if (cudaLaunchCooperativeKernel((const void *)k_exact_sum, dim3(G), dim3(ES_T), args, 0, s) != cudaSuccess)
    return RPBA_ERR_CUDA;
  return RPBA_OK;
}
