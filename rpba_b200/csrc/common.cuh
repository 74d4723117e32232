// common.cuh -- device-side math shared by the bundle-adjustment kernels.
//
// Conventions (the reference's, rbacore.cpp):
//   camera frame   x = R (X + PC)                    rbacore.cpp:1238
//   projection     u = x/z, distortion (1 + d0 r^2 + d1 r^4), K   :1251-1267
//   residual       d = xg - K dist(u)                 :1270-1271
//   Jacobians      derivatives of d (so the step is x_new = x - dx)
//   camera params  in XPMatrices order: [rot(3) | PC(3, or 2 for the
//                  normcamera) | k1' k2' f] ; camera 0 has intrinsics only
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>
#include <utility>

#define RPBA_P 9  // padded camera block size (6 + 3 intrinsics)

namespace rpba {

// Trial camera state: eRMnew, ePCnew, camerasnew (rpba.h:626-666).
struct __align__(16) CamState {
  double R[9];
  double PC[3];
  double K00, K01, K02, K11, K12;
  double d0, d1;
  double pad;
};

// Exact IEEE operations: no FMA contraction, so that the residual of an
// observation is bitwise the value the C++ oracle computes.
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float fmulr(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float faddr(float a, float b) { return __fadd_rn(a, b); }

struct ObsEval {
  double u, v;    // normalised coordinates x/z, y/z (ex3(0), ex3(1))
  double uu, vv;  // distorted (ex3u)
  double xs3;     // 1/z or the guarded +-1e3
  double d1, d2;  // residual
  bool nan;
};

// Residual of one observation, CalcCorrections rbacore.cpp:1238-1307.
__device__ __forceinline__ void eval_obs(const CamState &c, double X0, double X1, double X2,
                                         float xgx, float xgy, double defdiff, ObsEval &e) {
  const double v0 = add(X0, c.PC[0]), v1 = add(X1, c.PC[1]), v2 = add(X2, c.PC[2]);
  const double ex0 = add(add(mul(c.R[0], v0), mul(c.R[1], v1)), mul(c.R[2], v2));
  const double ex1 = add(add(mul(c.R[3], v0), mul(c.R[4], v1)), mul(c.R[5], v2));
  const double ex2 = add(add(mul(c.R[6], v0), mul(c.R[7], v1)), mul(c.R[8], v2));
  double xs3 = ex2;
  if (fabs(xs3) < 1.e-3)
    xs3 = xs3 < 0. ? -1.e3 : 1.e3;
  else
    xs3 = __ddiv_rn(1., xs3);
  const double u = mul(ex0, xs3), v = mul(ex1, xs3);
  const double dist = add(mul(u, u), mul(v, v));
  const double z = add(1., add(mul(c.d0, dist), mul(mul(c.d1, dist), dist)));
  const double uu = mul(u, z), vv = mul(v, z);
  const double c0 = add(add(mul(uu, c.K00), mul(vv, c.K01)), c.K02);
  const double c1 = add(mul(vv, c.K11), c.K12);
  double d1 = sub((double)xgx, c0), d2 = sub((double)xgy, c1);
  if (d1 > defdiff) d1 = defdiff;
  if (d1 < -defdiff) d1 = -defdiff;
  if (d2 > defdiff) d2 = defdiff;
  if (d2 < -defdiff) d2 = -defdiff;
  e.nan = !isfinite(d1) || !isfinite(d2);
  if (e.nan) d1 = d2 = 0.;
  e.u = u;
  e.v = v;
  e.uu = uu;
  e.vv = vv;
  e.xs3 = xs3;
  e.d1 = d1;
  e.d2 = d2;
}

// Float cost terms of one observation (rbacore.cpp:1312-1324).
__device__ __forceinline__ float cost_term(double d1, double d2, float w0, float w1, float w2) {
  const float f1 = (float)d1, f2 = (float)d2;
  const float d11 = fmulr(f1, f1), d12 = fmulr(fmulr(2.f, f1), f2), d22 = fmulr(f2, f2);
  return faddr(faddr(fmulr(d11, w0), fmulr(d12, w2)), fmulr(d22, w1));
}

// Camera role of an image in the parameterisation.
enum CamRole : int { ROLE_ZERO = 0, ROLE_NORM = 1, ROLE_FREE = 2 };

// Jacobians of the residual (CalcDerivatives rbacore.cpp:1420-1616 with
// eCalcCalibratedDerivativesX/3 :1620-1673).  Bc: 2 x RPBA_P, columns in the
// camera's own parameter order, zero beyond its count; Bp: 2 x 3.
template <typename T>
__device__ __forceinline__ int jacobians(const CamState &c, const ObsEval &e, int role,
                                         const int esvm[2], int addmask, T Bc[2][RPBA_P],
                                         T Bp[2][3]) {
  const double u = e.u, v = e.v, xs3 = e.xs3;
  const double x1 = u * xs3, x2 = v * xs3;
  const double k2 = c.d0, k4 = c.d1;
  const double xy2 = u * u + v * v;
  const double xy4 = xy2 * xy2;
  const double xxpc = k4 * xy4 + u * (2 * k2 * u + 4 * k4 * u * xy2) + k2 * xy2 + 1.;
  const double xypc = u * (4 * k4 * xy2 * v + 2 * k2 * v);
  const double yxpc = (4 * k4 * u * xy2 + 2 * k2 * u) * v;
  const double yypc = v * (2 * k2 * v + 4 * k4 * xy2 * v) + k4 * xy4 + k2 * xy2 + 1.;
  auto calib = [&](double a0, double a1, T &o0, T &o1) {
    const double xp = xxpc * a0 + xypc * a1;
    const double yp = yypc * a1 + yxpc * a0;
    o0 = (T)(xp * c.K00 + yp * c.K01);
    o1 = (T)(yp * c.K11);
  };
  double pc0[3], pc1[3];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    pc0[j] = -c.R[j] * xs3 + c.R[6 + j] * x1;
    pc1[j] = -c.R[3 + j] * xs3 + c.R[6 + j] * x2;
    calib(pc0[j], pc1[j], Bp[0][j], Bp[1][j]);
  }
#pragma unroll
  for (int j = 0; j < RPBA_P; ++j) Bc[0][j] = Bc[1][j] = (T)0;
  const double xyp4 = xy2 * xy2;
  // the intrinsic columns (k2, k4, f) that addmask selects, in that order.
  // Every array index below is a compile-time constant (a runtime choice is
  // a select), so the camera, Bc and the columns stay in registers.
  const bool hk2 = (addmask & 1) != 0, hk4 = (addmask & 2) != 0, hf = (addmask & 4) != 0;
  const int ni = (int)hk2 + (int)hk4 + (int)hf;
  const double a0 = -u * xy2 * c.K00 - v * xy2 * c.K01, a1 = -v * xy2 * c.K11;
  const double b0 = -u * xyp4 * c.K00 - v * xyp4 * c.K01, b1 = -v * xyp4 * c.K11;
  const double f0 = -e.uu, f1 = -e.vv;
  const double ic0[3] = {hk2 ? a0 : (hk4 ? b0 : f0), (hk2 && hk4) ? b0 : f0, f0};
  const double ic1[3] = {hk2 ? a1 : (hk4 ? b1 : f1), (hk2 && hk4) ? b1 : f1, f1};
  auto put_intrinsics = [&](auto first) {
    constexpr int n0 = decltype(first)::value;
#pragma unroll
    for (int t = 0; t < 3; ++t)
      if (t < ni) {
        Bc[0][n0 + t] = (T)ic0[t];
        Bc[1][n0 + t] = (T)ic1[t];
      }
    return n0 + ni;
  };
  if (role == ROLE_ZERO) return put_intrinsics(std::integral_constant<int, 0>{});
  const double xs31 = 1. / xs3;
  const double xs32 = xs31 * xs31;
  calib(x2 * x1 * xs32, 1. + x2 * x2 * xs32, Bc[0][0], Bc[1][0]);
  calib(-1. - x1 * x1 * xs32, -x2 * x1 * xs32, Bc[0][1], Bc[1][1]);
  calib(x2 * xs31, -x1 * xs31, Bc[0][2], Bc[1][2]);
  if (role == ROLE_NORM) {
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int s = esvm[j];  // a column of R: 0, 1 or 2
      const double r0 = s == 0 ? c.R[0] : (s == 1 ? c.R[1] : c.R[2]);
      const double r3 = s == 0 ? c.R[3] : (s == 1 ? c.R[4] : c.R[5]);
      const double r6 = s == 0 ? c.R[6] : (s == 1 ? c.R[7] : c.R[8]);
      calib(-r0 * xs3 + r6 * x1, -r3 * xs3 + r6 * x2, Bc[0][3 + j], Bc[1][3 + j]);
    }
    return put_intrinsics(std::integral_constant<int, 5>{});
  }
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    Bc[0][3 + j] = Bp[0][j];
    Bc[1][3 + j] = Bp[1][j];
  }
  return put_intrinsics(std::integral_constant<int, 6>{});
}

// 3x3 inverse by cofactors; m, out row major.
template <typename T>
__device__ __forceinline__ T inv3(const T m[9], T out[9]) {
  T C[9];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const int i1 = (i + 1) % 3, i2 = (i + 2) % 3;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const int j1 = (j + 1) % 3, j2 = (j + 2) % 3;
      C[i * 3 + j] = m[i1 * 3 + j1] * m[i2 * 3 + j2] - m[i1 * 3 + j2] * m[i2 * 3 + j1];
    }
  }
  const T det = C[0] * m[0] + C[3] * m[3] + C[6] * m[6];
  const T id = (T)1 / det;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) out[i * 3 + j] = C[j * 3 + i] * id;
  return det;
}

// Cayley rotation, rbacore.cpp:2014-2043.
__device__ __forceinline__ void cayley(double a, double b, double c, double R[9]) {
  const double a2 = a * a, b2 = b * b, c2 = c * c;
  const double ab = a * b, ac = a * c, bc = b * c;
  double abc = 4 + a2 + b2 + c2;
  if (fabs(abc) < 1.e-20)
    abc = abc < 0. ? -1.e20 : 1.e20;
  else
    abc = 1. / abc;
  R[0] = abc * (4 + a2 - b2 - c2);
  R[1] = abc * (2 * ab - 4 * c);
  R[2] = abc * (2 * ac + 4 * b);
  R[3] = abc * (2 * ab + 4 * c);
  R[4] = abc * (4 - a2 + b2 - c2);
  R[5] = abc * (2 * bc - 4 * a);
  R[6] = abc * (2 * ac - 4 * b);
  R[7] = abc * (2 * bc + 4 * a);
  R[8] = abc * (4 - a2 - b2 + c2);
}

// Quaternion re-orthonormalisation, rpba.h:876-913; row stride rs.
__device__ __forceinline__ void rectify(double *R, int rs) {
  double a0 = R[2 * rs + 1] - R[1 * rs + 2];
  double a1 = R[0 * rs + 2] - R[2 * rs + 0];
  double a2 = R[1 * rs + 0] - R[0 * rs + 1];
  if (fabs(a0) < 1.e-20) a0 = 1.e-20;
  if (fabs(a1) < 1.e-20) a1 = 1.e-20;
  if (fabs(a2) < 1.e-20) a2 = 1.e-20;
  const double al = sqrt(a0 * a0 + a1 * a1 + a2 * a2);
  a0 /= al;
  a1 /= al;
  a2 /= al;
  const double phi = atan2(al, R[0] + R[rs + 1] + R[2 * rs + 2] - 1.);
  double s, q0;
  sincos(phi * 0.5, &s, &q0);
  const double q1 = a0 * s, q2 = a1 * s, q3 = a2 * s;
  R[0] = q0 * q0 + q1 * q1 - q2 * q2 - q3 * q3;
  R[1] = 2 * (q1 * q2 - q0 * q3);
  R[2] = 2 * (q1 * q3 + q0 * q2);
  R[rs + 0] = 2 * (q2 * q1 + q0 * q3);
  R[rs + 1] = q0 * q0 - q1 * q1 + q2 * q2 - q3 * q3;
  R[rs + 2] = 2 * (q2 * q3 - q0 * q1);
  R[2 * rs + 0] = 2 * (q3 * q1 - q0 * q2);
  R[2 * rs + 1] = 2 * (q3 * q2 + q0 * q1);
  R[2 * rs + 2] = q0 * q0 - q1 * q1 - q2 * q2 + q3 * q3;
}

// n x n (n <= 9) inverse by LU with partial pivoting; A, Ai row major with
// leading dimension 9.
__device__ __forceinline__ void lu_inverse9(int n, const double *A, double *Ai) {
  double LU[81];
  int perm[9];
  for (int i = 0; i < 81; ++i) LU[i] = A[i];
  for (int i = 0; i < 9; ++i) perm[i] = i;
  for (int k = 0; k < n; ++k) {
    int p = k;
    double best = fabs(LU[k * 9 + k]);
    for (int r = k + 1; r < n; ++r) {
      const double v = fabs(LU[r * 9 + k]);
      if (v > best) {
        best = v;
        p = r;
      }
    }
    if (p != k) {
      for (int c = 0; c < n; ++c) {
        const double t = LU[k * 9 + c];
        LU[k * 9 + c] = LU[p * 9 + c];
        LU[p * 9 + c] = t;
      }
      const int t = perm[k];
      perm[k] = perm[p];
      perm[p] = t;
    }
    const double piv = LU[k * 9 + k];
    for (int r = k + 1; r < n; ++r) {
      const double l = LU[r * 9 + k] / piv;
      LU[r * 9 + k] = l;
      for (int c = k + 1; c < n; ++c) LU[r * 9 + c] -= l * LU[k * 9 + c];
    }
  }
  for (int i = 0; i < 81; ++i) Ai[i] = 0.;
  for (int col = 0; col < n; ++col) {
    double y[9];
    for (int i = 0; i < n; ++i) {
      double s = perm[i] == col ? 1. : 0.;
      for (int j = 0; j < i; ++j) s -= LU[i * 9 + j] * y[j];
      y[i] = s;
    }
    for (int i = n - 1; i >= 0; --i) {
      double s = y[i];
      for (int j = i + 1; j < n; ++j) s -= LU[i * 9 + j] * y[j];
      y[i] = s / LU[i * 9 + i];
    }
    for (int i = 0; i < n; ++i) Ai[i * 9 + col] = y[i];
  }
  for (int i = n; i < 9; ++i) Ai[i * 9 + i] = 1.;
}

// lu_inverse9 by one warp: the same operations in the same order (the
// compiler may contract them into FMAs differently, so the last bits can
// differ), with row r of the factor in lane r's registers (r < 9) and
// column col of the inverse solved by lane col.  `row` holds row `lane` of
// the input (lanes < 9; anything in the other lanes); every lane of the warp
// calls it; lanes < n write their column of the inverse to Ai (Ai may be the
// input's storage: nothing is read from memory).
// Step k of lu_inverse9_warp's factorisation (k a compile-time constant, so
// that the rows stay in registers).
template <int k>
__device__ __forceinline__ void lu9_warp_step(int n, double (&row)[9], int &perm, int lane) {
  constexpr unsigned FULL = 0xffffffffu;
  if (k >= n) return;
  // pivot: the first row p >= k of the largest |LU[p][k]| (a strictly
  // larger value replaces, as the serial scan does)
  double best = __shfl_sync(FULL, fabs(row[k]), k);
  int p = k;
#pragma unroll
  for (int r = k + 1; r < 9; ++r) {
    const double v = __shfl_sync(FULL, fabs(row[k]), r);
    if (r < n && v > best) {
      best = v;
      p = r;
    }
  }
  if (p != k) {
    const int src = lane == k ? p : (lane == p ? k : lane);
#pragma unroll
    for (int c = 0; c < 9; ++c) row[c] = __shfl_sync(FULL, row[c], src);
    perm = __shfl_sync(FULL, perm, src);
  }
  const double piv = __shfl_sync(FULL, row[k], k);
  const bool below = lane > k && lane < n;
  const double l = below ? row[k] / piv : 0.;
  if (below) row[k] = l;
#pragma unroll
  for (int c = k + 1; c < 9; ++c) {
    const double pk = __shfl_sync(FULL, row[c], k);
    if (below && c < n) row[c] -= l * pk;
  }
}

template <int... K>
__device__ __forceinline__ void lu9_warp_factor(int n, double (&row)[9], int &perm, int lane,
                                                std::integer_sequence<int, K...>) {
  (lu9_warp_step<K>(n, row, perm, lane), ...);
}

// lu_inverse9 by one warp: the same operations in the same order (the
// compiler may contract them into FMAs differently, so the last bits can
// differ), with row r of the factor in lane r's registers (r < 9) and
// column col of the inverse solved by lane col.  `row` holds row `lane` of
// the input (lanes < 9; anything in the other lanes); every lane of the warp
// calls it; lanes < 9 write their column of the inverse to Ai (Ai may be the
// input's storage: nothing is read from memory).
__device__ __forceinline__ void lu_inverse9_warp(int n, double (&row)[9], double *Ai, int lane) {
  constexpr unsigned FULL = 0xffffffffu;
  int perm = lane;
  lu9_warp_factor(n, row, perm, lane, std::make_integer_sequence<int, 9>{});
  // column `lane` of the inverse: forward then back substitution
  double y[9];
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    y[i] = 0.;
    if (i < n) {
      double s = __shfl_sync(FULL, perm, i) == lane ? 1. : 0.;
#pragma unroll
      for (int j = 0; j < i; ++j) s -= __shfl_sync(FULL, row[j], i) * y[j];
      y[i] = s;
    }
  }
#pragma unroll
  for (int i = 8; i >= 0; --i) {
    if (i < n) {
      double s = y[i];
#pragma unroll
      for (int j = i + 1; j < 9; ++j) {
        const double u = __shfl_sync(FULL, row[j], i);
        if (j < n) s -= u * y[j];
      }
      y[i] = s / __shfl_sync(FULL, row[i], i);
    }
  }
  __syncwarp();
  if (lane < 9) {
#pragma unroll
    for (int i = 0; i < 9; ++i) Ai[i * 9 + lane] = (lane < n && i < n) ? y[i] : (i == lane && i >= n ? 1. : 0.);
  }
}

}  // namespace rpba
