// kernels.cu -- per-observation, per-point and per-camera kernels of the
// global LSA (rbacore.cpp).  The linearisation kernels (point, camera,
// pair, back-substitution) are compiled for two forms: FP64 throughout (the
// drop-in form) and the mixed-precision form: FP32 records and blocks with
// FP32 arithmetic and compensated (Kahan) per-camera and per-pair sums, the
// point blocks factored in FP64 and the records whitened by the factor
// (k_point32).  Residuals and the cost stay FP64.
#include <cub/cub.cuh>

#include "internal.h"

namespace rpba {

namespace {

constexpr int GRP = 8;  // lanes per point in the point-major kernels

template <class T>
__device__ __forceinline__ T grp_sum(T v) {
#pragma unroll
  for (int o = GRP / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o, GRP);
  return v;
}

// Storage of the linearisation in either form.
template <class T>
struct Store;
template <>
struct Store<double> {
  static __device__ __forceinline__ double *rec(const DevLSA &L) { return L.rec; }
  static __device__ __forceinline__ double *ptV(const DevLSA &L) { return L.ptV; }
  static __device__ __forceinline__ double *blocks(const DevLSA &L) { return L.blocks; }
  static constexpr int BS = BS64;
};
template <>
struct Store<float> {
  static __device__ __forceinline__ float *rec(const DevLSA &L) { return L.rec32; }
  static __device__ __forceinline__ float *ptV(const DevLSA &L) { return L.ptV32; }
  static __device__ __forceinline__ float *blocks(const DevLSA &L) { return L.blocks32; }
  static constexpr int BS = BS32;
};

// Compensated (Kahan) accumulation for the FP32 form; plain in FP64.
template <class T>
struct Acc {
  T s = T(0), c = T(0);
  __device__ __forceinline__ void add(T x) {
    if constexpr (sizeof(T) == 4) {
      const T y = x - c;
      const T t = s + y;
      c = (t - s) - y;
      s = t;
    } else {
      s += x;
    }
  }
  __device__ __forceinline__ double value() const { return (double)s - (double)c; }
};

// In GCP mode camera 0 is free like the others and there is no scale
// camera (normcamera = -1; rbacore.cpp:697-698, 1005-1008).
__device__ __forceinline__ int role_of(const DevLSA &L, int k) {
  return (k == 0 && !L.ao) ? ROLE_ZERO : (k == L.normcamera ? ROLE_NORM : ROLE_FREE);
}

// ----------------------------------------------------------- cost pass
// CalcCorrections with derivflag = false (rbacore.cpp:1215-1331): per
// observation float cost term and the reweighting statistic sig0rmv.
__global__ void k_cost(DevLSA L, const double *__restrict__ XM, int srmv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= L.nobs) return;
  const int k = L.o_cam[i], p = L.o_pt[i];
  const double *X = XM + L.nrioff + 3 * p;
  const float2 xg = L.o_xg[i];
  ObsEval e;
  eval_obs(L.camn[k], X[0], X[1], X[2], xg.x, xg.y, L.defdiff, e);
  if (e.nan) {
    L.o_cost[i] = 0.f;
    L.o_s0rmv[i] = 1.e20f;
    return;
  }
  const float4 w = L.o_w[i];
  const float val = cost_term(e.d1, e.d2, w.x, w.y, w.z);
  L.o_cost[i] = val;
  if (srmv) {
    if (L.robust) {
      const float4 wo = L.o_wold[i];
      L.o_s0rmv[i] = cost_term(e.d1, e.d2, wo.x, wo.y, wo.z);
    } else {
      L.o_s0rmv[i] = val;
    }
  }
}

// GCP mode: the prior cost term of every point at the state XM, in the
// reference's float accumulation (sig0ao, rbacore.cpp:1677-1729): the double
// form d^T W d (d = gcp - X) in the reference's operation order, rounded to
// float; 0 for a point without a prior.
__global__ void k_gcp_cost(DevLSA L, const double *__restrict__ XM, float *out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= L.npts) return;
  float t = 0.f;
  const int gi = L.pt_gcp[p];
  if (gi > -1) {
    const float *w = L.W3 + 6 * (size_t)L.pt_w3row[p];
    const double *gx = L.gcpdata + 3 * (size_t)gi;
    const double *X = XM + L.nrioff + 3 * (size_t)p;
    const double d1 = __dsub_rn(gx[0], X[0]), d2 = __dsub_rn(gx[1], X[1]), d3 = __dsub_rn(gx[2], X[2]);
    const double a = __dadd_rn(__dadd_rn(__dmul_rn(__dmul_rn(d1, d1), (double)w[0]),
                                         __dmul_rn(__dmul_rn(d2, d2), (double)w[1])),
                               __dmul_rn(__dmul_rn(d3, d3), (double)w[2]));
    const double b = __dadd_rn(__dadd_rn(__dmul_rn(__dmul_rn(d1, d2), (double)w[3]),
                                         __dmul_rn(__dmul_rn(d1, d3), (double)w[4])),
                               __dmul_rn(__dmul_rn(d2, d3), (double)w[5]));
    t = __double2float_rn(__dadd_rn(a, __dmul_rn(2., b)));
  }
  out[p] = t;
}

// Sequential float sum in array order: the reference accumulates its cost
// and weight sums in float, one observation after the other
// (rbacore.cpp:1327, 727, 881).  One warp; every lane carries the same
// running sum, so the result is bitwise that of the sequential loop.
__global__ void k_seq_sum(const float *__restrict__ v, int n, float *out) {
  const int lane = threadIdx.x;
  constexpr int U = 8;
  float s = 0.f;
  float cur[U], nxt[U];
#pragma unroll
  for (int j = 0; j < U; ++j) {
    const int idx = j * 32 + lane;
    cur[j] = idx < n ? v[idx] : 0.f;
  }
  for (int base = 0; base < n; base += 32 * U) {
#pragma unroll
    for (int j = 0; j < U; ++j) {
      const int idx = base + 32 * U + j * 32 + lane;
      nxt[j] = idx < n ? v[idx] : 0.f;
    }
    const int lim = n - base;
#pragma unroll
    for (int j = 0; j < U; ++j) {
#pragma unroll 8
      for (int l = 0; l < 32; ++l) {
        const float t = __shfl_sync(0xffffffffu, cur[j], l);
        if (j * 32 + l < lim) s = __fadd_rn(s, t);
      }
    }
#pragma unroll
    for (int j = 0; j < U; ++j) cur[j] = nxt[j];
  }
  if (lane == 0) *out = s;
}

// ---------------------------------------------------------- point pass
// CalcCorrections/CalcDerivatives with derivflag = true, solveflag = false
// (rbacore.cpp:1215-1348, 1420-1616): Jacobians of every observation, the
// point block V = sum Jp^T W Jp and g = sum Jp^T W d, V damped and inverted;
// the per-observation record for the camera, pair and back-substitution
// kernels.  FP64 form (T = double); the FP32 form is k_point32.
template <class T>
__global__ void k_point(DevLSA L, double multfact1) {
  static_assert(sizeof(T) == 8, "the FP32 form is k_point32");
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int p = gt / GRP, ln = gt % GRP;
  // no early exit: the group reductions below shuffle over the full warp
  const bool valid = p < L.npts;
  const int t0 = valid ? L.pt_off[p] : 0, t1 = valid ? L.pt_off[p + 1] : 0;
  double X0 = 0., X1 = 0., X2 = 0.;
  if (valid) {
    const double *X = L.XPM + L.nrioff + 3 * p;
    X0 = X[0];
    X1 = X[1];
    X2 = X[2];
  }
  const int esvm[2] = {L.gauge[0], L.gauge[1]};
  T V[9], g[3];
#pragma unroll
  for (int j = 0; j < 9; ++j) V[j] = 0.;
  g[0] = g[1] = g[2] = 0.;
  for (int o = t0 + ln; o < t1; o += GRP) {
    const int k = L.o_cam[o];
    const CamState c = L.camn[k];
    const float2 xg = L.o_xg[o];
    ObsEval e;
    eval_obs(c, X0, X1, X2, xg.x, xg.y, L.defdiff, e);
    if (e.nan) L.o_s0rmv[o] = 1.e20f;
    T Bc[2][RPBA_P], Bp[2][3];
    jacobians<T>(c, e, role_of(L, k), esvm, L.addmask, Bc, Bp);
    const float4 w = L.o_w[o];
    const T W0 = w.x, W1 = w.y, W2 = w.z;
    const T d1 = (T)e.d1, d2 = (T)e.d2;
    T G[2][3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      G[0][j] = Bp[0][j] * W0 + Bp[1][j] * W2;
      G[1][j] = Bp[0][j] * W2 + Bp[1][j] * W1;
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
#pragma unroll
      for (int b = 0; b < 3; ++b) V[a * 3 + b] += G[0][a] * Bp[0][b] + G[1][a] * Bp[1][b];
      g[a] += G[0][a] * d1 + G[1][a] * d2;
    }
    T *r = Store<T>::rec(L) + (size_t)o * REC;
    const bool cam_active = k >= L.begini;
#pragma unroll
    for (int j = 0; j < RPBA_P; ++j) {
      r[j] = cam_active ? Bc[0][j] : T(0);
      r[9 + j] = cam_active ? Bc[1][j] : T(0);
    }
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      r[18 + j] = G[0][j];
      r[21 + j] = G[1][j];
    }
    r[24] = d1 * W0 + d2 * W2;
    r[25] = d1 * W2 + d2 * W1;
  }
#pragma unroll
  for (int j = 0; j < 9; ++j) V[j] = grp_sum(V[j]);
#pragma unroll
  for (int j = 0; j < 3; ++j) g[j] = grp_sum(g[j]);
  if (L.ao && valid && L.pt_gcp[p] > -1) {
    // CalcDerivatives3DGCP (rbacore.cpp:1677-1729): the 3-D prior of a
    // point shared with other partitions, residual gcp - X, B = -I
    const float *w = L.W3 + 6 * (size_t)L.pt_w3row[p];
    const double *gx = L.gcpdata + 3 * (size_t)L.pt_gcp[p];
    const double d1 = gx[0] - X0, d2 = gx[1] - X1, d3 = gx[2] - X2;
    const double Wm[9] = {w[0], w[3], w[4], w[3], w[1], w[5], w[4], w[5], w[2]};
#pragma unroll
    for (int j = 0; j < 9; ++j) V[j] += Wm[j];
#pragma unroll
    for (int r = 0; r < 3; ++r) g[r] += (-Wm[r * 3]) * d1 + (-Wm[r * 3 + 1]) * d2 + (-Wm[r * 3 + 2]) * d3;
  }
  V[0] = (T)(V[0] * multfact1);
  V[4] = (T)(V[4] * multfact1);
  V[8] = (T)(V[8] * multfact1);
  T Vi[9];
  inv3<T>(V, Vi);
  if (ln == 0 && valid) {
    T *pv = Store<T>::ptV(L) + (size_t)p * PREC;
#pragma unroll
    for (int j = 0; j < 9; ++j) pv[j] = Vi[j];
    pv[9] = g[0];
    pv[10] = g[1];
    pv[11] = g[2];
  }
  T vg[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) vg[a] = Vi[a * 3] * g[0] + Vi[a * 3 + 1] * g[1] + Vi[a * 3 + 2] * g[2];
  for (int o = t0 + ln; o < t1; o += GRP) {
    T *r = Store<T>::rec(L) + (size_t)o * REC;
    T G[2][3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      G[0][j] = r[18 + j];
      G[1][j] = r[21 + j];
    }
    const float4 w = L.o_w[o];
    T GV[2][3];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) GV[a][b] = G[a][0] * Vi[b] + G[a][1] * Vi[3 + b] + G[a][2] * Vi[6 + b];
    r[26] = (T)w.x - (GV[0][0] * G[0][0] + GV[0][1] * G[0][1] + GV[0][2] * G[0][2]);
    r[27] = (T)w.z - (GV[0][0] * G[1][0] + GV[0][1] * G[1][1] + GV[0][2] * G[1][2]);
    r[28] = (T)w.y - (GV[1][0] * G[1][0] + GV[1][1] * G[1][1] + GV[1][2] * G[1][2]);
    r[29] = r[24] - (G[0][0] * vg[0] + G[0][1] * vg[1] + G[0][2] * vg[2]);
    r[30] = r[25] - (G[1][0] * vg[0] + G[1][1] * vg[1] + G[1][2] * vg[2]);
  }
}

// FP32 form of the point pass, whitened.  V and g are summed in FP64 from
// the FP32-rounded point Jacobians, V = L L^T is factored in FP64, and the
// record carries H = G L^-T in place of G, so that every Schur product
// G V^-1 G^T = H H^T is formed from bounded factors (H H^T <= W for each
// observation) however ill-conditioned V is: the explicit V^-1 of a distant,
// down-weighted point overflows FP32, and products with it lose all digits.
// A pivot at or below 1e-13 of its diagonal entry (not resolvable in FP64
// arithmetic) or below 1e-60 drops its coordinate: the step leaves that
// coordinate of the point unchanged (the factor is that of V without its row
// and column), and the Schur contribution stays positive semidefinite.
// Point record: L^-1 (9, row major, zeros above the diagonal), q = L^-1 g.
__global__ void k_point32(DevLSA L, double multfact1) {
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int p = gt / GRP, ln = gt % GRP;
  const bool valid = p < L.npts;  // no early exit (full-warp shuffles below)
  const int t0 = valid ? L.pt_off[p] : 0, t1 = valid ? L.pt_off[p + 1] : 0;
  double X0 = 0., X1 = 0., X2 = 0.;
  if (valid) {
    const double *X = L.XPM + L.nrioff + 3 * p;
    X0 = X[0];
    X1 = X[1];
    X2 = X[2];
  }
  const int esvm[2] = {L.gauge[0], L.gauge[1]};
  double V[6] = {0., 0., 0., 0., 0., 0.};  // V00 V01 V02 V11 V12 V22
  double g[3] = {0., 0., 0.};
  for (int o = t0 + ln; o < t1; o += GRP) {
    const int k = L.o_cam[o];
    const CamState c = L.camn[k];
    const float2 xg = L.o_xg[o];
    ObsEval e;
    eval_obs(c, X0, X1, X2, xg.x, xg.y, L.defdiff, e);
    if (e.nan) L.o_s0rmv[o] = 1.e20f;
    float Bc[2][RPBA_P], Bp[2][3];
    jacobians<float>(c, e, role_of(L, k), esvm, L.addmask, Bc, Bp);
    const float4 w = L.o_w[o];
    const double W0 = w.x, W1 = w.y, W2 = w.z;
    double G[2][3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      G[0][j] = Bp[0][j] * W0 + Bp[1][j] * W2;
      G[1][j] = Bp[0][j] * W2 + Bp[1][j] * W1;
    }
    V[0] += G[0][0] * Bp[0][0] + G[1][0] * Bp[1][0];
    V[1] += G[0][0] * Bp[0][1] + G[1][0] * Bp[1][1];
    V[2] += G[0][0] * Bp[0][2] + G[1][0] * Bp[1][2];
    V[3] += G[0][1] * Bp[0][1] + G[1][1] * Bp[1][1];
    V[4] += G[0][1] * Bp[0][2] + G[1][1] * Bp[1][2];
    V[5] += G[0][2] * Bp[0][2] + G[1][2] * Bp[1][2];
#pragma unroll
    for (int a = 0; a < 3; ++a) g[a] += G[0][a] * e.d1 + G[1][a] * e.d2;
    // the record's floats 0..25 in 16-byte stores: Bc, then Jp until the
    // factor is known (replaced by H below), then W d
    const bool cam_active = k >= L.begini;
    float v[28];
#pragma unroll
    for (int j = 0; j < RPBA_P; ++j) {
      v[j] = cam_active ? Bc[0][j] : 0.f;
      v[9 + j] = cam_active ? Bc[1][j] : 0.f;
    }
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      v[18 + j] = Bp[0][j];
      v[21 + j] = Bp[1][j];
    }
    v[24] = (float)(e.d1 * W0 + e.d2 * W2);
    v[25] = (float)(e.d1 * W2 + e.d2 * W1);
    float4 *r4 = (float4 *)(L.rec32 + (size_t)o * REC);
#pragma unroll
    for (int j = 0; j < 6; ++j) r4[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
    *(float2 *)(r4 + 6) = make_float2(v[24], v[25]);
  }
#pragma unroll
  for (int j = 0; j < 6; ++j) V[j] = grp_sum(V[j]);
#pragma unroll
  for (int j = 0; j < 3; ++j) g[j] = grp_sum(g[j]);
  V[0] *= multfact1;
  V[3] *= multfact1;
  V[5] *= multfact1;
  // V = L L^T with guarded pivots; m = L^-1 (lower)
  auto root = [](double d, double diag) { return (d > 1.e-13 * diag && d > 1.e-60) ? sqrt(d) : 0.; };
  const double l00 = root(V[0], V[0]);
  const double i00 = l00 > 0. ? 1. / l00 : 0.;
  const double l10 = V[1] * i00, l20 = V[2] * i00;
  const double l11 = root(V[3] - l10 * l10, V[3]);
  const double i11 = l11 > 0. ? 1. / l11 : 0.;
  const double l21 = (V[4] - l20 * l10) * i11;
  const double l22 = root(V[5] - l20 * l20 - l21 * l21, V[5]);
  const double i22 = l22 > 0. ? 1. / l22 : 0.;
  double m[6] = {i00, -l10 * i00 * i11, i11, -(l20 * i00 - l21 * l10 * i00 * i11) * i22, -l21 * i11 * i22, i22};
  // m00 m10 m11 m20 m21 m22; a factor beyond the FP32 range drops the point
  bool inrange = true;
#pragma unroll
  for (int j = 0; j < 6; ++j) inrange = inrange && fabs(m[j]) < 1.e30;
  if (!inrange)
#pragma unroll
    for (int j = 0; j < 6; ++j) m[j] = 0.;
  const double q0 = m[0] * g[0], q1 = m[1] * g[0] + m[2] * g[1], q2 = m[3] * g[0] + m[4] * g[1] + m[5] * g[2];
  if (ln == 0 && valid) {
    float *pv = L.ptV32 + (size_t)p * PREC;
    pv[0] = (float)m[0];
    pv[1] = pv[2] = 0.f;
    pv[3] = (float)m[1];
    pv[4] = (float)m[2];
    pv[5] = 0.f;
    pv[6] = (float)m[3];
    pv[7] = (float)m[4];
    pv[8] = (float)m[5];
    pv[9] = (float)q0;
    pv[10] = (float)q1;
    pv[11] = (float)q2;
  }
  for (int o = t0 + ln; o < t1; o += GRP) {
    float *r = L.rec32 + (size_t)o * REC;
    const float4 w = L.o_w[o];
    const double W0 = w.x, W1 = w.y, W2 = w.z;
    // floats 16..27 of the record (Jp at 18..23, W d at 24, 25)
    const float4 ra = *(const float4 *)(r + 16), rb = *(const float4 *)(r + 20), rcv = *(const float4 *)(r + 24);
    double H[2][3];
    {
      const double p00 = ra.z, p01 = ra.w, p02 = rb.x, p10 = rb.y, p11 = rb.z, p12 = rb.w;
      const double G0[3] = {p00 * W0 + p10 * W2, p01 * W0 + p11 * W2, p02 * W0 + p12 * W2};
      const double G1[3] = {p00 * W2 + p10 * W1, p01 * W2 + p11 * W1, p02 * W2 + p12 * W1};
      H[0][0] = m[0] * G0[0];
      H[0][1] = m[1] * G0[0] + m[2] * G0[1];
      H[0][2] = m[3] * G0[0] + m[4] * G0[1] + m[5] * G0[2];
      H[1][0] = m[0] * G1[0];
      H[1][1] = m[1] * G1[0] + m[2] * G1[1];
      H[1][2] = m[3] * G1[0] + m[4] * G1[1] + m[5] * G1[2];
    }
    const double h00 = H[0][0] * H[0][0] + H[0][1] * H[0][1] + H[0][2] * H[0][2];
    const double h01 = H[0][0] * H[1][0] + H[0][1] * H[1][1] + H[0][2] * H[1][2];
    const double h11 = H[1][0] * H[1][0] + H[1][1] * H[1][1] + H[1][2] * H[1][2];
    // floats 16..31 in 16-byte stores: H at 18..23, W - H H^T at 26..28,
    // W d - H q at 29, 30 (16, 17, 24, 25 rewritten unchanged, 31 zero)
    float4 *r4 = (float4 *)(r + 16);
    r4[0] = make_float4(ra.x, ra.y, (float)H[0][0], (float)H[0][1]);
    r4[1] = make_float4((float)H[0][2], (float)H[1][0], (float)H[1][1], (float)H[1][2]);
    r4[2] = make_float4(rcv.x, rcv.y, (float)(W0 - h00), (float)(W2 - h01));
    r4[3] = make_float4((float)(W1 - h11), (float)((double)rcv.x - (H[0][0] * q0 + H[0][1] * q1 + H[0][2] * q2)),
                        (float)((double)rcv.y - (H[1][0] * q0 + H[1][1] * q1 + H[1][2] * q2)), 0.f);
  }
}

// --------------------------------------------------------- camera pass
// Diagonal blocks of the reduced camera system and its right-hand side:
// S_kk = sum_o Bc^T (W - G V^-1 G^T) Bc, b_k = sum_o Bc^T (W d - G V^-1 g)
// (the camera terms of rbacore.cpp:1552-1561 minus the Schur terms of
// :1358-1360), then the damping of rbacore.cpp:1164-1170.  One CTA per
// camera sums its observations in the reference's nro order.
constexpr int CAM_T = 64, CAM_B = 32, CAM_W = 24;

template <class T>
__global__ void __launch_bounds__(CAM_T) k_camera(DevLSA L, double multfact1) {
  const int k = blockIdx.x + L.begini;
  if (k >= L.nimg) return;
  __shared__ T s[CAM_B][CAM_W];
  const int tid = threadIdx.x;
  const int beg = L.coff[k], end = L.coff[k + 1];
  Acc<T> acc;
  int ei = 0, ej = 0;
  if (tid < 45) {
    int t = tid;
    while (t >= 9 - ei) {
      t -= 9 - ei;
      ++ei;
    }
    ej = ei + t;
  } else if (tid < 54) {
    ei = tid - 45;
  }
  // staging of a chunk: every warp reads the chunk's observation indices
  // once (lane j: observation j) and passes them by shuffle, so that the
  // CAM_SV record values a thread stages are independent loads in flight;
  // the next chunk's record values are loaded while this chunk is summed,
  // and the indices two chunks ahead
  constexpr int CAM_SV = (CAM_B * 23 + CAM_T - 1) / CAM_T;
  const int lane = tid & 31;
  auto idx_of = [&](int base) { return base + lane < end ? L.camlist[base + lane] : 0; };
  T vals[CAM_SV];
  auto fetch = [&](int base, int ol) {
    const int nb = min(CAM_B, end - base);
#pragma unroll
    for (int m = 0; m < CAM_SV; ++m) {
      const int idx = tid + CAM_T * m, ob = idx / 23, c = idx - 23 * (idx / 23);
      const int o = __shfl_sync(0xffffffffu, ol, ob & 31);
      const T *r = Store<T>::rec(L) + (size_t)o * REC;
      vals[m] = idx < nb * 23 ? (c < 18 ? r[c] : r[26 + (c - 18)]) : T(0);
    }
  };
  int ol_next = idx_of(beg + CAM_B);
  if (beg < end) fetch(beg, idx_of(beg));
  for (int base = beg; base < end; base += CAM_B) {
    const int nb = min(CAM_B, end - base);
#pragma unroll
    for (int m = 0; m < CAM_SV; ++m) {
      const int idx = tid + CAM_T * m, ob = idx / 23, c = idx - 23 * (idx / 23);
      if (idx < nb * 23) s[ob][c] = vals[m];
    }
    __syncthreads();
    if (base + CAM_B < end) {
      const int ol = ol_next;
      ol_next = idx_of(base + 2 * CAM_B);
      fetch(base + CAM_B, ol);
    }
    if (tid < 45) {
      for (int ob = 0; ob < nb; ++ob) {
        const T b0i = s[ob][ei], b1i = s[ob][9 + ei], b0j = s[ob][ej], b1j = s[ob][9 + ej];
        const T M00 = s[ob][18], M01 = s[ob][19], M11 = s[ob][20];
        acc.add(b0i * (M00 * b0j + M01 * b1j) + b1i * (M01 * b0j + M11 * b1j));
      }
    } else if (tid < 54) {
      for (int ob = 0; ob < nb; ++ob) acc.add(s[ob][ei] * s[ob][21] + s[ob][9 + ei] * s[ob][22]);
    }
    __syncthreads();
  }
  const int np = L.camparv[k + 1] - L.camparv[k];
  T *D = Store<T>::blocks(L) + (size_t)k * Store<T>::BS;
  if (tid < 45) {
    double v;
    if (ei < np && ej < np) {
      v = acc.value();
      if (ei == ej) v = __dadd_rn(__dmul_rn(v, multfact1), 1.e-2);
    } else {
      v = ei == ej ? 1. : 0.;
    }
    D[ei * 9 + ej] = (T)v;
    D[ej * 9 + ei] = (T)v;
  } else if (tid < 54) {
    L.rhs[k * 9 + ei] = ei < np ? (double)(T)acc.value() : 0.;
  }
}

// ----------------------------------------------------------- pair pass
// Off-diagonal blocks: S_kl = - sum_p W_pk V_p^-1 W_pl^T over the points
// seen by both cameras (rbacore.cpp:1362-1390), with W_po = Bc^T G.  One
// warp per block sums its contributions in a fixed order.  FP64 form; the
// FP32 form is k_pair32.
template <class T>
__global__ void k_pair(DevLSA L) {
  static_assert(sizeof(T) == 8, "the FP32 form is k_pair32");
  const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int wl = threadIdx.x >> 5;
  __shared__ T sm[8][64];
  if (wid >= L.nboff) return;
  T *s = sm[wl];
  Acc<T> acc[3];
  const T *rec = Store<T>::rec(L), *ptv = Store<T>::ptV(L);
  // values of one contribution: 24 of the row camera's observation (Bc 18,
  // G 6), 24 of the column camera's and V^-1 (9) of the point
  constexpr int NV = 57;
  auto fetch = [&](int ox, int oy, int p, T &v0, T &v1) {
    v0 = lane < 24 ? rec[(size_t)ox * REC + lane] : rec[(size_t)oy * REC + lane - 24];
    const int i1 = lane + 32;
    v1 = i1 < 48 ? rec[(size_t)oy * REC + i1 - 24] : (i1 < NV ? ptv[(size_t)p * PREC + i1 - 48] : T(0));
  };
  const int cb = L.boff[wid], ce = L.boff[wid + 1];
  for (int c0 = cb; c0 < ce; c0 += 32) {
    // the next (up to) 32 contributions' observation pairs and points, one
    // per lane; the record values of contribution j + 1 are fetched while j
    // is accumulated
    const int n = min(32, ce - c0);
    int2 pr = make_int2(0, 0);
    int pp = 0;
    if (lane < n) {
      pr = L.contrib[c0 + lane];
      pp = L.o_pt[pr.x];
    }
    T v0, v1;
    fetch(__shfl_sync(0xffffffffu, pr.x, 0), __shfl_sync(0xffffffffu, pr.y, 0), __shfl_sync(0xffffffffu, pp, 0),
          v0, v1);
    for (int j = 0; j < n; ++j) {
      s[lane] = v0;
      if (lane + 32 < NV) s[lane + 32] = v1;
      if (j + 1 < n)
        fetch(__shfl_sync(0xffffffffu, pr.x, j + 1), __shfl_sync(0xffffffffu, pr.y, j + 1),
              __shfl_sync(0xffffffffu, pp, j + 1), v0, v1);
      __syncwarp();
      // N = G_s V^-1 G_t^T (2 x 2)
      const T *Gs = s + 18, *Gt = s + 42, *Vi = s + 48;
      T GV[2][3], N[2][2];
#pragma unroll
      for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b)
          GV[a][b] = Gs[a * 3] * Vi[b] + Gs[a * 3 + 1] * Vi[3 + b] + Gs[a * 3 + 2] * Vi[6 + b];
#pragma unroll
      for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b)
          N[a][b] = GV[a][0] * Gt[b * 3] + GV[a][1] * Gt[b * 3 + 1] + GV[a][2] * Gt[b * 3 + 2];
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        const int e = lane + 32 * q;
        if (e < 81) {
          const int i = e / 9, jj = e % 9;
          const T bt0 = s[24 + jj], bt1 = s[24 + 9 + jj];
          const T t0 = N[0][0] * bt0 + N[0][1] * bt1;
          const T t1 = N[1][0] * bt0 + N[1][1] * bt1;
          acc[q].add(-(s[i] * t0 + s[9 + i] * t1));
        }
      }
      __syncwarp();
    }
  }
  T *B = Store<T>::blocks(L) + (size_t)(L.nimg + wid) * Store<T>::BS;
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const int e = lane + 32 * q;
    if (e < 81) __stcs(B + e, (T)acc[q].value());  // streaming: keep L2 for the records
  }
}

// FP32 form of the pair pass (whitened records): S_kl -= sum Bc_k^T (H_k
// H_l^T) Bc_l over the block's contributions.  One warp per block; per
// contribution the warp stages the row camera's and the column camera's
// record (Bc 18 and H 6 floats each, coalesced 4-byte loads, the next
// contribution's loads in flight) in shared memory in the order the lanes
// read them: lanes 0..26 own the three entries (i, 3 (lane % 3) .. + 2) of
// block row i = lane / 3, and each forms N = H_k H_l^T itself (two 16-byte
// and two 8-byte broadcast loads, 12 FMAs), U_i = (Bc_k[0][i], Bc_k[1][i]) N
// (one 8-byte load) and its three entries from the three (Bc_l[0][j],
// Bc_l[1][j]) pairs (one 16-byte and one 8-byte load): twelve shared-memory
// or global instructions per contribution.  Each lane sums a chunk of up to
// 32 contributions in FP32, in order, and adds the chunk into a compensated
// (Kahan) sum, so the entry is deterministic.
// Staging layout (floats): row record: pairs (Bc[0][j], Bc[1][j]) at 2 j,
// H at 20..25; column record: the pairs of j = 3 g .. 3 g + 2 at 28 + 8 g
// (16-byte aligned groups), H at 52..57.
constexpr int PS = 60;  // floats per warp
__device__ __forceinline__ int pair_slot_x(int e) {
  return e < 9 ? 2 * e : (e < 18 ? 2 * (e - 9) + 1 : e + 2);
}
__device__ __forceinline__ int pair_slot_y(int e) {
  if (e < 18) {
    const int r = e < 9 ? 0 : 1, j = e - 9 * r;
    return 28 + 8 * (j / 3) + 2 * (j % 3) + r;
  }
  return 52 + (e - 18);
}
__global__ void __launch_bounds__(256) k_pair32(DevLSA L) {
  const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int wl = threadIdx.x >> 5;
  __shared__ __align__(16) float sm[8][PS];
  __shared__ int2 spr[8][32];
  if (wid >= L.nboff) return;
  float *s = sm[wl];
  int2 *sp = spr[wl];
  const float *rec = L.rec32;
  const int i = lane < 27 ? lane / 3 : 0, g = lane < 27 ? lane - 3 * (lane / 3) : 0;
  // destinations of this lane's two record values: v0 = float `lane` of the
  // row record (lane < 24) or float lane - 24 of the column record; v1 =
  // float lane + 8 of the column record (lane < 16)
  const int d0 = lane < 24 ? pair_slot_x(lane) : pair_slot_y(lane - 24);
  const int d1 = pair_slot_y(lane < 16 ? lane + 8 : 8);
  float ks[3] = {0.f, 0.f, 0.f}, kc[3] = {0.f, 0.f, 0.f};
  auto fetch = [&](int ox, int oy, float &v0, float &v1) {
    v0 = lane < 24 ? rec[(size_t)ox * REC + lane] : rec[(size_t)oy * REC + lane - 24];
    v1 = lane < 16 ? rec[(size_t)oy * REC + lane + 8] : 0.f;
  };
  const int cb = L.boff[wid], ce = L.boff[wid + 1];
  for (int c0 = cb; c0 < ce; c0 += 32) {
    const int n = min(32, ce - c0);
    if (lane < n) sp[lane] = L.contrib[c0 + lane];
    __syncwarp();
    float v0, v1;
    {
      const int2 q = sp[0];
      fetch(q.x, q.y, v0, v1);
    }
    float part[3] = {0.f, 0.f, 0.f};
    for (int j = 0; j < n; ++j) {
      s[d0] = v0;
      if (lane < 16) s[d1] = v1;
      if (j + 1 < n) {
        const int2 q = sp[j + 1];
        fetch(q.x, q.y, v0, v1);
      }
      __syncwarp();
      const float4 hx = *(const float4 *)(s + 20), hy = *(const float4 *)(s + 52);
      const float2 hx2 = *(const float2 *)(s + 24), hy2 = *(const float2 *)(s + 56);
      const float n00 = hx.x * hy.x + hx.y * hy.y + hx.z * hy.z;
      const float n01 = hx.x * hy.w + hx.y * hy2.x + hx.z * hy2.y;
      const float n10 = hx.w * hy.x + hx2.x * hy.y + hx2.y * hy.z;
      const float n11 = hx.w * hy.w + hx2.x * hy2.x + hx2.y * hy2.y;
      const float2 bx = *(const float2 *)(s + 2 * i);
      const float4 ya = *(const float4 *)(s + 28 + 8 * g);
      const float2 yb = *(const float2 *)(s + 32 + 8 * g);
      const float u0 = bx.x * n00 + bx.y * n10, u1 = bx.x * n01 + bx.y * n11;
      part[0] -= u0 * ya.x + u1 * ya.y;
      part[1] -= u0 * ya.z + u1 * ya.w;
      part[2] -= u0 * yb.x + u1 * yb.y;
      __syncwarp();
    }
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const float y = part[q] - kc[q];
      const float t = ks[q] + y;
      kc[q] = (t - ks[q]) - y;
      ks[q] = t;
    }
    __syncwarp();  // sp is rewritten by the next chunk
  }
  if (lane < 27) {
    float *B = L.blocks32 + (size_t)(L.nimg + wid) * BS32 + i * 9 + 3 * g;
#pragma unroll
    for (int q = 0; q < 3; ++q) __stcs(B + q, (float)((double)ks[q] - (double)kc[q]));  // keep L2 for the records
  }
}

// ------------------------------------------------- back-substitution
// rbacore.cpp:1395-1410: dX_p = V^-1 (g - sum_o W_o^T dc_k), with
// W_o^T dc = G^T (Bc dc); in the FP32 form L^-T (q - sum_o H^T (Bc dc)).
template <class T>
__global__ void k_backsub(DevLSA L, const double *__restrict__ xsol) {
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int p = gt / GRP, ln = gt % GRP;
  const bool valid = p < L.npts;  // no early exit (full-warp shuffles below)
  const int t0 = valid ? L.pt_off[p] : 0, t1 = valid ? L.pt_off[p + 1] : 0;
  T a0 = 0., a1 = 0., a2 = 0.;
  for (int o = t0 + ln; o < t1; o += GRP) {
    const int k = L.o_cam[o];
    if (k < L.begini) continue;
    const T *rp = Store<T>::rec(L) + (size_t)o * REC;
    const double *dc = xsol + (size_t)k * 9;
    T r[24];
    if constexpr (sizeof(T) == 4) {
      // the FP32 record's first 24 floats in six 16-byte loads
#pragma unroll
      for (int v = 0; v < 6; ++v) {
        const float4 q = __ldg((const float4 *)rp + v);
        r[4 * v] = q.x;
        r[4 * v + 1] = q.y;
        r[4 * v + 2] = q.z;
        r[4 * v + 3] = q.w;
      }
    } else {
#pragma unroll
      for (int a = 0; a < 24; ++a) r[a] = rp[a];
    }
    T s0 = 0., s1 = 0.;
#pragma unroll
    for (int a = 0; a < 9; ++a) {
      s0 += r[a] * (T)dc[a];
      s1 += r[9 + a] * (T)dc[a];
    }
    a0 += r[18] * s0 + r[21] * s1;
    a1 += r[19] * s0 + r[22] * s1;
    a2 += r[20] * s0 + r[23] * s1;
  }
  a0 = grp_sum(a0);
  a1 = grp_sum(a1);
  a2 = grp_sum(a2);
  if (ln == 0 && valid) {
    const T *pv = Store<T>::ptV(L) + (size_t)p * PREC;
    double *xo = L.x + L.nrioff + 3 * p;
    if constexpr (sizeof(T) == 8) {
      const T r0 = pv[9] - a0, r1 = pv[10] - a1, r2 = pv[11] - a2;
      xo[0] = pv[0] * r0 + pv[1] * r1 + pv[2] * r2;
      xo[1] = pv[3] * r0 + pv[4] * r1 + pv[5] * r2;
      xo[2] = pv[6] * r0 + pv[7] * r1 + pv[8] * r2;
    } else {
      // whitened: a = L^-1 sum G^T Bc dc, dX = L^-T (q - a)
      const double y0 = (double)pv[9] - a0, y1 = (double)pv[10] - a1, y2 = (double)pv[11] - a2;
      xo[0] = (double)pv[0] * y0 + (double)pv[3] * y1 + (double)pv[6] * y2;
      xo[1] = (double)pv[4] * y1 + (double)pv[7] * y2;
      xo[2] = (double)pv[8] * y2;
    }
  }
}

// Camera entries of the step: x[k] = (float) exiv (rbacore.cpp:1181-1186).
__global__ void k_xcam(DevLSA L, const double *__restrict__ xsol) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = i / 9 + L.begini, a = i % 9;
  if (k >= L.nimg) return;
  const int cp = L.camparv[k], np = L.camparv[k + 1] - cp;
  if (a < np) L.x[cp + a] = (double)(float)xsol[(size_t)k * 9 + a];
}

// XPMatricesnew = XPMatrices - x with the NaN/Inf check (rbacore.cpp:541-548).
__global__ void k_update(DevLSA L, int nunk) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nunk) return;
  const double v = L.x[i];
  if (!isfinite(v)) atomicOr(L.err, 1);
  L.XPMn[i] = L.XPM[i] - v;
}

// ------------------------------------------------- camera (de)coding
// DecodeCameras, rbacore.cpp:1733-1800.
__global__ void k_decode(DevLSA L, const double *__restrict__ XM) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= L.nimg) return;
  // a NaN step returns before DecodeCameras (rbacore.cpp:541-550): keep the
  // previous trial cameras, which OutputLSAc reports
  if (*(volatile int *)L.err & 1) return;
  CamState &c = L.camn[k];
  if (k == 0 && !L.ao) {
    int a = -1;
    if (L.addmask & 1) c.d0 = XM[++a];
    if (L.addmask & 2) c.d1 = XM[++a];
    if (L.addmask & 4) c.K00 = c.K11 = XM[++a];
    return;
  }
  const int cp = L.camparv[k];
  double Ra[9];
  cayley(XM[cp], XM[cp + 1], XM[cp + 2], Ra);
  const double *B = L.Rb + (size_t)k * 9;
  double R[9];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) R[i * 3 + j] = Ra[i * 3] * B[j] + Ra[i * 3 + 1] * B[3 + j] + Ra[i * 3 + 2] * B[6 + j];
  rectify(R, 3);
#pragma unroll
  for (int i = 0; i < 9; ++i) c.R[i] = R[i];
  double e[3];
  if (k == L.normcamera) {
    e[L.gauge[0]] = XM[cp + 3];
    e[L.gauge[1]] = XM[cp + 4];
    e[L.gauge[2]] = 0.;
  } else {
    e[0] = XM[cp + 3];
    e[1] = XM[cp + 4];
    e[2] = XM[cp + 5];
  }
  const double *pb = L.PCb + (size_t)k * 3;
  c.PC[0] = e[0] + pb[0];
  c.PC[1] = e[1] + pb[1];
  c.PC[2] = e[2] + pb[2];
  int a = k == L.normcamera ? 4 : 5;
  if (L.addmask & 1) c.d0 = XM[++a + cp];
  if (L.addmask & 2) c.d1 = XM[++a + cp];
  if (L.addmask & 4) c.K00 = c.K11 = XM[++a + cp];
}

// EncodeCameras, rbacore.cpp:999-1087.
__global__ void k_encode(DevLSA L) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= L.nimg) return;
  if (k == 0 && !L.ao) {
    int a = -1;
    if (L.addmask & 1) L.XPM[++a] = L.dc[0];
    if (L.addmask & 2) L.XPM[++a] = L.dc[1];
    if (L.addmask & 4) L.XPM[++a] = L.Kc[0];
    return;
  }
  double *P = L.Pacc + (size_t)k * 12;
  rectify(P, 4);
  double *R = L.Rb + (size_t)k * 9;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) R[r * 3 + c] = P[r * 4 + c];
  double *pc = L.PCb + (size_t)k * 3;
  for (int i = 0; i < 3; ++i) pc[i] = R[i] * P[3] + R[3 + i] * P[7] + R[6 + i] * P[11];
  const int cp = L.camparv[k];
  L.XPM[cp] = L.XPM[cp + 1] = L.XPM[cp + 2] = 0.;
  int a;
  if (k == L.normcamera) {
    float maxv = 0.f;
    int maxi = 0;
    for (int i = 0; i < 3; ++i)
      if (fabs(pc[i]) > (double)maxv) {
        maxv = (float)fabs(pc[i]);
        maxi = i;
      }
    int ii = 0;
    for (int i = 0; i < 3; ++i)
      if (i != maxi) L.gauge[ii++] = i;
    L.gauge[2] = maxi;
    L.XPM[cp + 3] = L.XPM[cp + 4] = 0.;
    a = 4 + cp;
  } else {
    L.XPM[cp + 3] = L.XPM[cp + 4] = L.XPM[cp + 5] = 0.;
    a = 5 + cp;
  }
  if (L.addmask & 1) L.XPM[++a] = L.dc[2 * k];
  if (L.addmask & 2) L.XPM[++a] = L.dc[2 * k + 1];
  if (L.addmask & 4) L.XPM[++a] = L.Kc[9 * k];
}

// StoreResultsIteration, rbacore.cpp:891-918.
__global__ void k_store(DevLSA L, int xpmsize) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < xpmsize) L.XPM[i] = L.XPMn[i];
  if (i < L.nobs) L.o_flagnew[i] = L.o_flag[i];
  if (i < L.nimg) {
    const CamState &c = L.camn[i];
    double *P = L.Pacc + (size_t)i * 12;
    for (int r = 0; r < 3; ++r) {
      for (int cc = 0; cc < 3; ++cc) P[r * 4 + cc] = c.R[r * 3 + cc];
      P[r * 4 + 3] = c.R[r * 3] * c.PC[0] + c.R[r * 3 + 1] * c.PC[1] + c.R[r * 3 + 2] * c.PC[2];
    }
    double *K = L.Kc + (size_t)i * 9;
    K[0] = c.K00;
    K[1] = c.K01;
    K[2] = c.K02;
    K[4] = c.K11;
    K[5] = c.K12;
    K[8] = 1.;
    L.dc[2 * i] = c.d0;
    L.dc[2 * i + 1] = c.d1;
  }
}

// PrepareWeights2D (rbacore.cpp:704-783): Wij = Wijold and the terms of
// the float weight sum.
__global__ void k_prepare_weights(DevLSA L) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= L.nobs) return;
  const float4 w = L.o_wold[i];
  L.o_w[i] = w;
  L.o_wterm[i] = __fadd_rn(w.x, w.y);
  L.o_flag[i] = 0;
  L.o_flagnew[i] = 0;
}

// ----------------------------------------------------------- reweight
// Reweight2D, rbacore.cpp:823-887.
__global__ void k_rw_vals(DevLSA L, float *vals) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= L.nobs) return;
  const int o = L.camlist[i];
  const int p = L.o_pt[o];
  int pxs = (L.pt_off[p + 1] - L.pt_off[p]) * 2;
  if (pxs < 4) pxs = 4;
  const float rf = __fdiv_rn((float)pxs, (float)(pxs - 3));
  const float redfac = __fmul_rn(rf, rf);
  vals[i] = __fmul_rn(L.o_s0rmv[o], redfac);
}

// Per-image median by an exact radix select on the float bit patterns
// (values are >= 0, so the unsigned order is the numeric order).
__global__ void __launch_bounds__(256) k_median(DevLSA L, const float *vals, float *sig00v, int iflag) {
  const int k = blockIdx.x;
  if (k >= L.nimg) return;
  const int beg = L.coff[k], end = L.coff[k + 1], n = end - beg;
  __shared__ unsigned hist[256];
  __shared__ unsigned s_prefix, s_mask;
  __shared__ int s_rank;
  if (threadIdx.x == 0) {
    s_prefix = 0u;
    s_mask = 0u;
    s_rank = n / 2;
  }
  __syncthreads();
  for (int pass = 0; pass < 4; ++pass) {
    const int shift = 24 - 8 * pass;
    hist[threadIdx.x] = 0u;
    __syncthreads();
    const unsigned prefix = s_prefix, mask = s_mask;
    for (int i = beg + threadIdx.x; i < end; i += blockDim.x) {
      unsigned key = __float_as_uint(vals[i]);
      if (key == 0x80000000u) key = 0u;
      if ((key & mask) == prefix) atomicAdd(&hist[(key >> shift) & 255u], 1u);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      int r = s_rank;
      unsigned b = 0;
      for (; b < 256; ++b) {
        if ((int)hist[b] > r) break;
        r -= (int)hist[b];
      }
      if (b > 255) b = 255;
      s_rank = r;
      s_prefix = prefix | (b << shift);
      s_mask = mask | (255u << shift);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const float med = n > 0 ? __uint_as_float(s_prefix) : 0.f;
    float s = __fdiv_rn(1.f, __fmul_rn(med, 2.1981f));
    if (iflag > 1) s = __fmul_rn(s, 0.001f);
    sig00v[k] = s;
  }
}

__global__ void k_rw_apply(DevLSA L, const float *sig00v, int *nflag) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  int f = 0;
  if (i < L.nobs) {
    float ww = __fmul_rn(L.o_s0rmv[i], sig00v[L.o_cam[i]]);
    const bool fl = ww > 9.f;
    L.o_flag[i] = fl ? 1 : 0;
    if (fl) {
      ww = 1.e-4f;
      f = 1;
    } else {
      ww = 1.f;
    }
    const float4 wo = L.o_wold[i];
    float4 w;
    w.x = __fmul_rn(ww, wo.x);
    w.y = __fmul_rn(ww, wo.y);
    w.z = __fmul_rn(ww, wo.z);
    w.w = 0.f;
    if (__fadd_rn(w.x, w.y) < 2.e-8f) {
      w.x = w.y = 1.e-8f;
      w.z = 0.f;
    }
    L.o_w[i] = w;
    L.o_wterm[i] = __fadd_rn(w.x, w.y);
  }
  f = __syncthreads_count(f);
  if (threadIdx.x == 0 && f) atomicAdd(nflag, f);
}

// ------------------------------------------------------ final cost
// FP64 cost and squared residual sum of the accepted state with the
// Exteval projection (P X, distortion, f): the shared evaluator the oracle
// uses too.
__global__ void k_final_cost(DevLSA L, double *partials) {
  __shared__ double sc[256], sq[256];
  double c = 0., q = 0.;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < L.nobs; i += gridDim.x * blockDim.x) {
    const int k = L.o_cam[i], p = L.o_pt[i];
    const double *M = L.Pacc + (size_t)k * 12;
    const double *X = L.XPM + L.nrioff + 3 * p;
    double p1 = M[0] * X[0] + M[1] * X[1] + M[2] * X[2] + M[3];
    double p2 = M[4] * X[0] + M[5] * X[1] + M[6] * X[2] + M[7];
    double p3 = M[8] * X[0] + M[9] * X[1] + M[10] * X[2] + M[11];
    if (fabs(p3) < 1.e-3)
      p3 = p3 > 0. ? 1.e3 : -1.e3;
    else
      p3 = 1. / p3;
    p1 *= p3;
    p2 *= p3;
    const double dist = p1 * p1 + p2 * p2;
    const double z = 1. + (L.dc[2 * k] * dist + L.dc[2 * k + 1] * dist * dist);
    p1 *= z * L.Kc[9 * k];
    p2 *= z * L.Kc[9 * k];
    const float2 xg = L.o_xg[i];
    const double dx = (double)xg.x - p1, dy = (double)xg.y - p2;
    const float4 w = L.o_wold[i];
    c += dx * dx * w.x + dy * dy * w.y + 2. * dx * dy * w.z;
    q += dx * dx + dy * dy;
  }
  sc[threadIdx.x] = c;
  sq[threadIdx.x] = q;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      sc[threadIdx.x] += sc[threadIdx.x + s];
      sq[threadIdx.x] += sq[threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    partials[2 * blockIdx.x] = sc[0];
    partials[2 * blockIdx.x + 1] = sq[0];
  }
}

// ------------------------------------------------------------ Exteval
// EvalLSA + CalcCorrPointMulti (rpbacore.cpp:778-837, 882-941): one thread
// per point, float sums in the reference's order within the point.
__global__ void k_exteval(int n_points, const int *__restrict__ pt_off, const int *__restrict__ pt_img,
                          const int *__restrict__ pt_slot, const int *__restrict__ img_off,
                          const float *__restrict__ pmat, const float *__restrict__ Kf,
                          const float *__restrict__ dist, const float *__restrict__ XX,
                          const float *__restrict__ xg, const float *__restrict__ wx,
                          const float *__restrict__ wy, const float *__restrict__ wxy, double *resid,
                          float *ptterm, int *ptred) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n_points) return;
  const int s = pt_off[p], e = pt_off[p + 1];
  const int n = e - s;
  for (int j = s; j < e; ++j) resid[2 * j] = resid[2 * j + 1] = 0.;
  if (n <= 1) {
    ptterm[p] = 0.f;
    ptred[p] = 0;
    return;
  }
  float wsum = 0.f;
  for (int j = s; j < e; ++j) {
    const int sl = img_off[pt_img[j]] + pt_slot[j];
    wsum = __fadd_rn(wsum, __fadd_rn(wx[sl], wy[sl]));
  }
  wsum = __fdiv_rn(wsum, (float)(2 * n));
  const double X0 = XX[3 * p], X1 = XX[3 * p + 1], X2 = XX[3 * p + 2];
  float sig0 = 0.f;
  for (int j = s; j < e; ++j) {
    const int im = pt_img[j];
    const int sl = img_off[im] + pt_slot[j];
    const float *P = pmat + 12 * im;
    double p1 = add(add(add(mul((double)P[0], X0), mul((double)P[1], X1)), mul((double)P[2], X2)), (double)P[3]);
    double p2 = add(add(add(mul((double)P[4], X0), mul((double)P[5], X1)), mul((double)P[6], X2)), (double)P[7]);
    double p3 = add(add(add(mul((double)P[8], X0), mul((double)P[9], X1)), mul((double)P[10], X2)), (double)P[11]);
    if (fabs(p3) < 1.e-3)
      p3 = p3 > 0. ? 1.e3 : -1.e3;
    else
      p3 = __ddiv_rn(1., p3);
    p1 = mul(p1, p3);
    p2 = mul(p2, p3);
    const double dd = add(mul(p1, p1), mul(p2, p2));
    const double z = add(1., add(mul((double)dist[2 * im], dd), mul(mul((double)dist[2 * im + 1], dd), dd)));
    p1 = mul(p1, z);
    p2 = mul(p2, z);
    p1 = mul(p1, (double)Kf[9 * im]);
    p2 = mul(p2, (double)Kf[9 * im]);
    const double dx = sub((double)xg[2 * sl], p1), dy = sub((double)xg[2 * sl + 1], p2);
    resid[2 * j] = dx;
    resid[2 * j + 1] = dy;
    const double t = add(add(mul(mul(dx, dx), (double)wx[sl]), mul(mul(dy, dy), (double)wy[sl])),
                         mul(mul(mul(2., dx), dy), (double)wxy[sl]));
    sig0 = __fadd_rn(sig0, (float)t);
  }
  ptterm[p] = __fdiv_rn(sig0, wsum);
  ptred[p] = 2 * n - 3;
}

// ------------------------------------------------------ RobustDelete
// rbacore.cpp:922-995: observations flagged at the last accepted step are
// erased; a point left with fewer than minimagenrdel observations goes.
__global__ void k_delete_mark(DevLSA L, int *okeep, int *pkeep) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= L.npts) return;
  const int t0 = L.pt_off[p], t1 = L.pt_off[p + 1];
  int nf = 0;
  for (int o = t0; o < t1; ++o) nf += L.o_flagnew[o] ? 1 : 0;
  const bool erase = nf > 0 && (t1 - t0 - nf) < L.minimagenrdel;
  pkeep[p] = erase ? 0 : 1;
  for (int o = t0; o < t1; ++o) okeep[o] = (!erase && !L.o_flagnew[o]) ? 1 : 0;
}

__global__ void k_delete_obs(DevLSA L, const int *oidx, const int *pidx, const int *okeep, int *o_cam_n,
                             int *o_slot_n, int *o_pt_n, float2 *o_xg_n, float4 *o_wold_n) {
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= L.nobs || !okeep[o]) return;
  const int q = oidx[o];
  o_cam_n[q] = L.o_cam[o];
  o_slot_n[q] = L.o_slot[o];
  o_pt_n[q] = pidx[L.o_pt[o]];
  o_xg_n[q] = L.o_xg[o];
  o_wold_n[q] = L.o_wold[o];
}

__global__ void k_delete_pts(DevLSA L, const int *oidx, const int *pidx, const int *pkeep, int nobs_new,
                             int npts_new, int *pt_off_n, int *pt_id_n, double *X_n) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p == 0) pt_off_n[npts_new] = nobs_new;
  if (p >= L.npts || !pkeep[p]) return;
  const int q = pidx[p];
  pt_id_n[q] = L.pt_id[p];
  pt_off_n[q] = oidx[L.pt_off[p]];
  const double *X = L.XPM + L.nrioff + 3 * p;
  X_n[3 * q] = X[0];
  X_n[3 * q + 1] = X[1];
  X_n[3 * q + 2] = X[2];
}

inline int nblk(long long n, int t) { return (int)((n + t - 1) / t); }

}  // namespace

void launch_cost(const DevLSA &L, const double *XM, bool srmv, cudaStream_t s) {
  if (L.nobs > 0) k_cost<<<nblk(L.nobs, 256), 256, 0, s>>>(L, XM, srmv ? 1 : 0);
}

void launch_seq_sum(const float *v, int n, float *out, cudaStream_t s) {
  k_seq_sum<<<1, 32, 0, s>>>(v, n, out);
}

void launch_point_pass(const DevLSA &L, double multfact1, cudaStream_t s) {
  if (L.npts <= 0) return;
  if (L.rec32)
    k_point32<<<nblk((long long)L.npts * GRP, 128), 128, 0, s>>>(L, multfact1);
  else
    k_point<double><<<nblk((long long)L.npts * GRP, 128), 128, 0, s>>>(L, multfact1);
}

void launch_camera_pass(const DevLSA &L, double multfact1, cudaStream_t s) {
  const int nc = L.nimg - L.begini;
  if (nc <= 0) return;
  if (L.rec32)
    k_camera<float><<<nc, CAM_T, 0, s>>>(L, multfact1);
  else
    k_camera<double><<<nc, CAM_T, 0, s>>>(L, multfact1);
}

void launch_pair_pass(const DevLSA &L, cudaStream_t s) {
  if (L.nboff <= 0) return;
  if (L.rec32)
    k_pair32<<<nblk((long long)L.nboff * 32, 256), 256, 0, s>>>(L);
  else
    k_pair<double><<<nblk((long long)L.nboff * 32, 256), 256, 0, s>>>(L);
}

void launch_backsub(const DevLSA &L, const double *xsol, cudaStream_t s) {
  if (L.npts <= 0) return;
  if (L.rec32)
    k_backsub<float><<<nblk((long long)L.npts * GRP, 128), 128, 0, s>>>(L, xsol);
  else
    k_backsub<double><<<nblk((long long)L.npts * GRP, 128), 128, 0, s>>>(L, xsol);
}

void launch_xcam(const DevLSA &L, const double *xsol, cudaStream_t s) {
  const int n = (L.nimg - L.begini) * 9;
  if (n > 0) k_xcam<<<nblk(n, 256), 256, 0, s>>>(L, xsol);
}

void launch_update(const DevLSA &L, int nunk, cudaStream_t s) {
  if (nunk > 0) k_update<<<nblk(nunk, 256), 256, 0, s>>>(L, nunk);
}

void launch_decode(const DevLSA &L, const double *XM, cudaStream_t s) {
  k_decode<<<nblk(L.nimg, 128), 128, 0, s>>>(L, XM);
}

void launch_encode(const DevLSA &L, cudaStream_t s) { k_encode<<<nblk(L.nimg, 128), 128, 0, s>>>(L); }

void launch_store(const DevLSA &L, int xpmsize, cudaStream_t s) {
  long long n = xpmsize;
  if (L.nobs > n) n = L.nobs;
  if (L.nimg > n) n = L.nimg;
  k_store<<<nblk(n, 256), 256, 0, s>>>(L, xpmsize);
}

void launch_prepare_weights(const DevLSA &L, cudaStream_t s) {
  if (L.nobs > 0) k_prepare_weights<<<nblk(L.nobs, 256), 256, 0, s>>>(L);
}

void launch_reweight(const DevLSA &L, int iflag, float *vals, float *sig00v, int *nflag, cudaStream_t s) {
  cudaMemsetAsync(nflag, 0, sizeof(int), s);
  if (L.nobs > 0) k_rw_vals<<<nblk(L.nobs, 256), 256, 0, s>>>(L, vals);
  k_median<<<L.nimg, 256, 0, s>>>(L, vals, sig00v, iflag);
  if (L.nobs > 0) k_rw_apply<<<nblk(L.nobs, 256), 256, 0, s>>>(L, sig00v, nflag);
}

void launch_final_cost(const DevLSA &L, double *partials, int nparts, cudaStream_t s) {
  k_final_cost<<<nparts, 256, 0, s>>>(L, partials);
}

void launch_gcp_cost(const DevLSA &L, const double *XM, float *out, cudaStream_t s) {
  if (L.npts > 0) k_gcp_cost<<<nblk(L.npts, 256), 256, 0, s>>>(L, XM, out);
}

void launch_exteval(int n_points, const int *pt_off, const int *pt_img, const int *pt_slot, const int *img_off,
                    const float *pmat, const float *K, const float *dist, const float *XX, const float *xg,
                    const float *wx, const float *wy, const float *wxy, double *resid, float *ptterm,
                    int *ptred, cudaStream_t s) {
  if (n_points > 0)
    k_exteval<<<nblk(n_points, 128), 128, 0, s>>>(n_points, pt_off, pt_img, pt_slot, img_off, pmat, K, dist, XX,
                                                  xg, wx, wy, wxy, resid, ptterm, ptred);
}

void launch_delete_mark(const DevLSA &L, int *okeep, int *pkeep, cudaStream_t s) {
  if (L.npts > 0) k_delete_mark<<<nblk(L.npts, 256), 256, 0, s>>>(L, okeep, pkeep);
}

void launch_delete_compact(const DevLSA &L, const int *oidx, const int *pidx, const int *okeep, const int *pkeep,
                           int nobs_new, int npts_new, int *o_cam_n, int *o_slot_n, int *o_pt_n, float2 *o_xg_n,
                           float4 *o_wold_n, int *pt_off_n, int *pt_id_n, double *X_n, cudaStream_t s) {
  if (L.nobs > 0)
    k_delete_obs<<<nblk(L.nobs, 256), 256, 0, s>>>(L, oidx, pidx, okeep, o_cam_n, o_slot_n, o_pt_n, o_xg_n,
                                                   o_wold_n);
  k_delete_pts<<<nblk(L.npts > 0 ? L.npts : 1, 256), 256, 0, s>>>(L, oidx, pidx, pkeep, nobs_new, npts_new,
                                                                  pt_off_n, pt_id_n, X_n);
}

}  // namespace rpba
