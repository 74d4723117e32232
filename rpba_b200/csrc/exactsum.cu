// exactsum.cu -- the reference's float accumulations (sig0 += term in
// rbacore.cpp:1327, wsum += w in :727 and :881), computed in parallel with a
// result bitwise equal to the sequential float loop.
//
// Method.  Let s be the running float sum, s in [2^E, 2^(E+1)), u = ulp(s) =
// 2^(E-23), S = s/u (an integer in [2^23, 2^24)).  For v >= 0 with
// S + floor(v/u) < 2^24 the float addition is fl(s + v) = s + u*rne(v/u)
// with rne(v/u) = floor(v/u) + [frac > 1/2], except when v/u is exactly
// halfway between integers (a tie): then round-half-even gives
// floor(v/u) + [S + floor(v/u) odd], and the new S is even.  So inside one
// binade each element acts on the parity p of the running integer sum as a
// two-state transform  p -> (increment r(p), new parity q(p)), and a run of
// elements is the composition of their transforms, an associative operation:
// a grid-wide scan of per-thread and per-CTA composites gives every prefix
// without a sequential pass, ties included.  A run ends only at the first
// element k with S + R_(k-1) + floor(v_k/u) >= 2^24 (the sum leaves the
// binade); that element is added with a real float addition and a new run
// starts in the new binade.  Runs are few: the sum leaves a binade only when
// it doubles.  Each step of the scan covers a window, the elements from the
// run's start on, as many again as the sum has taken so far: the sum doubles
// inside it unless the terms shrink (then the next step takes the next
// window in the same binade), so the steps together read the input about
// twice instead of once per binade.
//
// The first HEAD elements and any stretch where s is zero or subnormal are
// added by one warp in plain sequence.  Inputs must be finite and >= 0.
#include <cuda.h>

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
constexpr int ES_WMIN = 65536;  // smallest window of a run step
constexpr int ES_MAXG = 512;    // CTAs at most (their composites are staged in shared memory)

struct EsCtl {
  float s;    // running sum before element i
  int i;      // next element
};

// Composite transform of a run of elements for incoming parity 0 and 1:
// total increment R, outgoing parity q, and M = max over the run of
// (increment before the element + floor(v/u)), the crossing test.
struct Xf {
  long long R[2], M[2];
  int q[2];
};
__device__ __forceinline__ Xf xf_identity() {
  Xf x;
  for (int p = 0; p < 2; ++p) {
    x.R[p] = 0;
    x.M[p] = LLONG_MIN;
    x.q[p] = p;
  }
  return x;
}
// a then b
__device__ __forceinline__ Xf xf_then(const Xf &a, const Xf &b) {
  Xf x;
#pragma unroll
  for (int p = 0; p < 2; ++p) {
    const bool m = a.q[p] != 0;  // b's state entered with parity a.q[p] (selects: no indexing)
    const long long bR = m ? b.R[1] : b.R[0], bM = m ? b.M[1] : b.M[0];
    x.R[p] = a.R[p] + bR;
    x.q[p] = m ? b.q[1] : b.q[0];
    x.M[p] = bM == LLONG_MIN ? a.M[p] : max(a.M[p], a.R[p] + bM);
  }
  return x;
}

struct EsArgs {
  const float *v;
  int n;
  float *out;
  long long *Rc, *Mc;  // per CTA composite: R[2], M[2]
  int *Tc;             // per CTA composite: q[2]
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

// Apply one element to a composite (in place, both incoming parities).
__device__ __forceinline__ void xf_push(Xf &x, long long fl, long long r, bool tie) {
  for (int p = 0; p < 2; ++p) {
    const long long m = x.R[p] + fl;
    if (m > x.M[p]) x.M[p] = m;
    const long long rr = tie ? fl + ((x.q[p] + fl) & 1) : r;
    x.R[p] += rr;
    x.q[p] = (int)((x.q[p] + rr) & 1);
  }
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
  __shared__ Xf s_x[ES_T];  // per-thread composites of the current run
  __shared__ Xf s_w[ES_T / 32];  // per-warp composites
  __shared__ long long s_cR[2 * ES_MAXG], s_cM[2 * ES_MAXG];  // the chunks' composites
  __shared__ unsigned char s_cT[2 * ES_MAXG];
  __shared__ long long s_rtot, s_R;
  __shared__ int s_cx, s_qx, s_tcross, s_q;

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
      // far more steps (binade changes and windows) than sums of real data
      // take: finish in plain sequence, still exact
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
    const int p0 = (int)(S & 1);
    const long long TOP = 1ll << 24;

    // The step's window: the elements from i0 on, as many again as the sum
    // has taken so far (at least ES_WMIN).  The sum leaves its binade when it
    // doubles, so the crossing is inside the window unless the terms shrink;
    // a window without a crossing ends the step at its last element, the sum
    // still in the same binade, and the next step takes the next window.
    // The window is cut into G chunks (CTA c: chunk c).
    const int wend = (int)min((long long)n, (long long)i0 + max((long long)i0, (long long)ES_WMIN));
    const int chunk = (wend - i0 + G - 1) / G;
    const int lo = min(wend, i0 + c * chunk), hi = min(wend, lo + chunk);
    const int per = (chunk + ES_T - 1) / ES_T;
    // phase A: composite of each thread's contiguous sub-range of this
    // chunk, then of the chunk
    const int a0 = max(lo, i0);
    const int t_lo = lo + tid * per, t_hi = min(hi, t_lo + per);
    Xf tx = xf_identity();
    for (int k = max(t_lo, a0); k < t_hi; ++k) {
      long long fl, r;
      bool tie;
      classify(A.v[k], scale, fl, r, tie);
      xf_push(tx, fl, r, tie);
    }
    s_x[tid] = tx;  // kept for the crossing chunk's walk
    // the chunk's composite: each warp's thread composites combined in a
    // tree that keeps lane order ((x0 x1)(x2 x3))..., then the warps' in
    // order (the composition is exact integer arithmetic and associative)
    {
      const int lane = tid & 31;
      Xf wx = tx;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        Xf ot;
#pragma unroll
        for (int p = 0; p < 2; ++p) {
          ot.R[p] = __shfl_down_sync(0xffffffffu, wx.R[p], o);
          ot.M[p] = __shfl_down_sync(0xffffffffu, wx.M[p], o);
          ot.q[p] = __shfl_down_sync(0xffffffffu, wx.q[p], o);
        }
        if ((lane & (2 * o - 1)) == 0) wx = xf_then(wx, ot);
      }
      if (lane == 0) s_w[tid >> 5] = wx;
    }
    __syncthreads();
    if (tid == 0) {
      Xf cx = s_w[0];
      for (int w = 1; w < ES_T / 32; ++w) cx = xf_then(cx, s_w[w]);
      for (int p = 0; p < 2; ++p) {
        A.Rc[2 * c + p] = cx.R[p];
        A.Mc[2 * c + p] = cx.M[p];
        A.Tc[2 * c + p] = cx.q[p];
      }
    }
    if (!grid_barrier(A.bar, G, A.err)) return;

    // phase B (every CTA, one thread): walk the chunk composites in order
    // from the run's start state; find the first chunk that crosses, the
    // state at its start, and the state at the end
    // (the composites are first copied to shared memory by all threads,
    // independent loads, so the walk's dependent steps are shared loads)
    for (int j = tid; j < 2 * G; j += ES_T) {
      s_cR[j] = __ldcg(A.Rc + j);
      s_cM[j] = __ldcg(A.Mc + j);
      s_cT[j] = (unsigned char)__ldcg(A.Tc + j);
    }
    __syncthreads();
    if (tid == 0) {
      long long R = 0;
      int q = p0, cxq = INT_MAX;
      long long Rx = 0;
      int qx = 0;
      for (int cc = 0; cc < G; ++cc) {
        const long long Mq = s_cM[2 * cc + q];
        if (Mq != LLONG_MIN && S + R + Mq >= TOP) {
          cxq = cc;
          Rx = R;
          qx = q;
          break;
        }
        R += s_cR[2 * cc + q];
        q = s_cT[2 * cc + q];
      }
      s_cx = cxq;
      s_rtot = cxq == INT_MAX ? R : Rx;
      s_qx = qx;
    }
    __syncthreads();
    const int cxi = s_cx;
    if (cxi == INT_MAX) {
      if (c == 0 && tid == 0) {
        A.ctl->s = (float)((double)(S + s_rtot) * u);
        A.ctl->i = wend;
      }
    } else if (c == cxi) {
      // the crossing chunk: thread 0 finds the first crossing thread range,
      // whose thread then finds the element and adds it with a float addition
      if (tid == 0) {
        long long R = s_rtot;
        int q = s_qx;
        int tx_first = ES_T;
        for (int t = 0; t < ES_T; ++t) {
          const Xf &x = s_x[t];
          if (x.M[q] != LLONG_MIN && S + R + x.M[q] >= TOP) {
            tx_first = t;
            break;
          }
          R += x.R[q];
          q = x.q[q];
        }
        s_tcross = tx_first;
        s_R = R;
        s_q = q;
      }
      __syncthreads();
      if (tid == s_tcross) {
        long long R = s_R;
        int q = s_q;
        for (int k = max(t_lo, a0); k < t_hi; ++k) {
          long long fl, r;
          bool tie;
          classify(A.v[k], scale, fl, r, tie);
          if (S + R + fl >= TOP) {
            const float sb = (float)((double)(S + R) * u);
            const float sn = __fadd_rn(sb, A.v[k]);
            A.ctl->s = sn;
            A.ctl->i = isfinite(sn) ? k + 1 : n;
            break;
          }
          const long long rr = tie ? fl + ((q + fl) & 1) : r;
          R += rr;
          q = (int)((q + rr) & 1);
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
  const int g = nsm * (per < 2 ? per : 2);
  return g < ES_MAXG ? g : ES_MAXG;
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
// (about 20 KB).  Its size caps the grid at NA_MAX_CTAS CTAs; inputs up to
// NA_MAX_N elements are accepted on any device (with fewer resident CTAs,
// each CTA takes a longer chunk).
using namespace rpba;

namespace {

constexpr int NA_MAX_CTAS = 512;
static_assert(NA_MAX_CTAS <= ES_MAXG, "k_exact_sum stages at most ES_MAXG chunk composites");
constexpr int NA_CHUNK = 8192;  // elements per CTA when the grid allows it
constexpr long long NA_MAX_N = (long long)NA_MAX_CTAS * NA_CHUNK;  // 4,194,304
constexpr size_t NA_OFF_RC = 0;
// two entries per CTA (one per incoming parity)
constexpr size_t NA_OFF_MC = NA_OFF_RC + sizeof(long long) * 2 * NA_MAX_CTAS;
constexpr size_t NA_OFF_TC = NA_OFF_MC + sizeof(long long) * 2 * NA_MAX_CTAS;
constexpr size_t NA_OFF_CTL = NA_OFF_TC + sizeof(int) * 2 * NA_MAX_CTAS;
constexpr size_t NA_OFF_BAR = NA_OFF_CTL + 16;
constexpr size_t NA_OFF_ERR = NA_OFF_BAR + 16;
constexpr size_t NA_BYTES = NA_OFF_ERR + 16;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_BYTES];

// The array's device address belongs to the context the module was loaded
// in: after cudaDeviceReset (or when the caller makes another context
// current) it is looked up again.  Contexts are told apart by their
// process-unique id (cuCtxGetId); the two driver calls are fetched through
// the runtime, so the library does not link the driver library.
typedef CUresult (*PfnCtxGetCurrent)(CUcontext *);
typedef CUresult (*PfnCtxGetId)(CUcontext, unsigned long long *);

constexpr int NA_MAX_DEVICES = 64;
struct NaSlot {
  unsigned long long ctx_id;  // 0: not looked up yet
  unsigned char *addr;        // device address of the scratch in that context
};
std::mutex g_na_mutex;
NaSlot g_na[NA_MAX_DEVICES];
PfnCtxGetCurrent g_ctx_current = nullptr;
PfnCtxGetId g_ctx_id = nullptr;

// Id of the calling thread's current context; 0 when none is current.
// Call with g_na_mutex held.
bool current_ctx_id(unsigned long long *id) {
  if (!g_ctx_current || !g_ctx_id) {
    void *a = nullptr, *b = nullptr;
    cudaDriverEntryPointQueryResult qa, qb;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa) != cudaSuccess ||
        qa != cudaDriverEntryPointSuccess || !a ||
        cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb) != cudaSuccess ||
        qb != cudaDriverEntryPointSuccess || !b)
      return false;
    g_ctx_current = (PfnCtxGetCurrent)a;
    g_ctx_id = (PfnCtxGetId)b;
  }
  CUcontext ctx = nullptr;
  if (g_ctx_current(&ctx) != CUDA_SUCCESS) return false;
  *id = 0;
  return !ctx || g_ctx_id(ctx, id) == CUDA_SUCCESS;
}

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
    // set-up, once per device and context, with that device current: the
    // array's name is only a host-side stand-in, so its device address is
    // looked up (the lookup also makes the runtime's context current when
    // this thread has none yet)
    std::lock_guard<std::mutex> lock(g_na_mutex);
    unsigned long long id = 0;
    if (!current_ctx_id(&id)) return RPBA_ERR_CUDA;
    if (id == 0 || g_na[dev].ctx_id != id) {
      void *p = nullptr;
      if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return RPBA_ERR_CUDA;
      if (id == 0 && (!current_ctx_id(&id) || id == 0)) return RPBA_ERR_CUDA;
      g_na[dev].ctx_id = id;
      g_na[dev].addr = (unsigned char *)p;
    }
    base = g_na[dev].addr;
  }
  const int ni = (int)n;
  // until the sum is written, *d_out holds a NaN (all bits set): a grid
  // barrier that runs out leaves it there
  if (cudaMemsetAsync(d_out, 0xff, sizeof(float), s) != cudaSuccess) return RPBA_ERR_CUDA;
  if (ni <= 4 * HEAD) {
    void *wargs[] = {(void *)&d_v, (void *)&ni, (void *)&d_out};
    return cudaLaunchKernel((const void *)k_warp_sum, dim3(1), dim3(32), wargs, 0, s) == cudaSuccess ? RPBA_OK
                                                                                                      : RPBA_ERR_CUDA;
  }
  int nsm = 0, per = 0;
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_exact_sum, ES_T, 0) != cudaSuccess || nsm * per < 1)
    return RPBA_ERR_CUDA;
  // every CTA must be resident (cooperative launch) and own a slot of the
  // array: past either limit the CTAs take longer chunks
  int G = (ni + NA_CHUNK - 1) / NA_CHUNK;
  if (G > NA_MAX_CTAS) G = NA_MAX_CTAS;
  if (G > nsm * per) G = nsm * per;
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
