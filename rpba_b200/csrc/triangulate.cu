// triangulate.cu -- per-point robust refinement against fixed cameras, the
// per-point bundle adjustment of the reference's parallel RPBA
// (CalcLSAXMulti, rpbacore.cpp:536-773, with CalcCorrPointMulti :778-837
// and CalcCalibratedDerivatives :841-877).
//
// Every point is independent: one thread per point runs its own damped
// Gauss-Newton loop (at most 100 steps, accept/stop on the float sigma0
// ratio), with the robust down-weighting of observations whose residual
// exceeds 16 x the image's threshold (mode 2) and the per-observation
// statistics collected for the thresholds (mode 1).  The per-observation
// temporaries of a point live in scratch arrays indexed by track entry.
// This file is compiled without FMA contraction and keeps the reference's
// operation order, so its results equal the CPU restatement's bit for bit.
// With a camera partition (rpba_triangulate_parts) the reference's
// per-partition weight blocks (wxyflag) are formed as well: for every
// partition that sees the point, the normal matrix of the point's
// observations in the other partitions (track order, one partition: all of
// them, undamped), taken at the start of the accepted iteration.
#include <cstring>
#include <vector>

#include "../../include/rpba_b200.h"
#include "internal.h"

namespace rpba {

namespace {

struct TriIn {
  const double *pmat;  // cameras in double precision (the reference's PMatricesd)
  const float *K, *dist, *XX, *xg, *wx, *wy, *wxy, *sig0w;
  const int *img_off, *pt_off, *pt_img, *pt_slot;
  const int *part;  // image -> partition (weight blocks), or null
  int np, robustmode, weight_only, nparts;
};
struct TriScratch {
  float *wx, *wy, *wxy, *p1, *p2, *p3;
  double *corr, *Bw;  // [2 x entry], [6 x entry]
  uint8_t *del;
  // weight blocks: the derivative rows [6 x entry]; the distinct partitions
  // of a point and their pending blocks, in the point's first entries
  double *Bxy;
  int *dpart;
  float *wt;  // [6 x entry]
};
struct TriOut {
  double *XX;
  uint8_t *keep, *conv;
  float *sig0v;
  double *s0;   // per point contribution to sig0io
  int *red;     // per point contribution to the redundancy
  float *w3d;   // [np x nparts x 6] (XX, YY, ZZ, XY, XZ, YZ), or null
};

__device__ void tri_corr(const TriIn &I, const TriScratch &S, int s, int e, double X0, double X1, double X2,
                         float &sig0, float *sig0v) {
  sig0 = 0.f;
  for (int t = s; t < e; ++t) {
    const int j = I.pt_img[t];
    const int sl = I.img_off[j] + I.pt_slot[t];
    const double *P = I.pmat + 12 * j;
    double p1 = (double)P[0] * X0 + (double)P[1] * X1 + (double)P[2] * X2 + (double)P[3];
    double p2 = (double)P[4] * X0 + (double)P[5] * X1 + (double)P[6] * X2 + (double)P[7];
    double p3 = (double)P[8] * X0 + (double)P[9] * X1 + (double)P[10] * X2 + (double)P[11];
    if (fabs(p3) < 1.e-3)
      p3 = p3 > 0. ? 1.e3 : -1.e3;
    else
      p3 = 1. / p3;
    p1 *= p3;
    p2 *= p3;
    S.p1[t] = (float)p1;
    S.p2[t] = (float)p2;
    S.p3[t] = (float)p3;
    const double dist = p1 * p1 + p2 * p2;
    const double z = 1. + (double)(I.dist[2 * j] * dist + I.dist[2 * j + 1] * dist * dist);
    p1 *= z;
    p2 *= z;
    p1 *= I.K[9 * j];
    p2 *= I.K[9 * j];
    const double dx = I.xg[2 * sl] - p1, dy = I.xg[2 * sl + 1] - p2;
    S.corr[2 * (size_t)t] = dx;
    S.corr[2 * (size_t)t + 1] = dy;
    sig0 += (float)(dx * dx * S.wx[t] + dy * dy * S.wy[t] + 2 * dx * dy * S.wxy[t]);
    sig0v[t] = (float)(dx * dx * I.wx[sl] + dy * dy * I.wy[sl] + 2 * dx * dy * I.wxy[sl]);
  }
}

__device__ __forceinline__ void tri_calibrated(double *xp, double *yp, double x, double y, double k2, double k4,
                                               double fx, double fy, double sk) {
  const double r2 = x * x + y * y, r4 = r2 * r2;
  const double axx = k4 * r4 + x * (2 * k2 * x + 4 * k4 * x * r2) + k2 * r2 + 1.;
  const double axy = x * (4 * k4 * r2 * y + 2 * k2 * y);
  const double ayx = y * (4 * k4 * x * r2 + 2 * k2 * x);
  const double ayy = y * (2 * k2 * y + 4 * k4 * r2 * y) + k4 * r4 + k2 * r2 + 1.;
  for (int c = 0; c < 3; ++c) {
    const double u = xp[c], v = yp[c];
    double nx = axx * u + axy * v;
    double ny = ayy * v + ayx * u;
    nx = nx * fx + ny * sk;
    ny *= fy;
    xp[c] = nx;
    yp[c] = ny;
  }
}

__global__ void k_triangulate(TriIn I, TriScratch S, TriOut O) {
  const int pi = blockIdx.x * blockDim.x + threadIdx.x;
  if (pi >= I.np) return;
  const int s = I.pt_off[pi], e = I.pt_off[pi + 1], pxs = e - s;
  const double Xin[3] = {(double)I.XX[3 * pi], (double)I.XX[3 * pi + 1], (double)I.XX[3 * pi + 2]};
  for (int q = 0; q < 3; ++q) O.XX[3 * (size_t)pi + q] = Xin[q];
  O.conv[pi] = 0;
  O.s0[pi] = 0.;
  O.red[pi] = 0;
  for (int t = s; t < e; ++t) O.keep[t] = 0;
  if (O.w3d)
    for (int q = 0; q < 6 * I.nparts; ++q) O.w3d[(size_t)pi * 6 * I.nparts + q] = 0.f;
  if (pxs <= 0) return;
  // the partitions that see the point, in order of first appearance
  int nd = 0;
  if (O.w3d && I.nparts > 1)
    for (int t = s; t < e; ++t) {
      const int q = I.part[I.pt_img[t]];
      bool seen = false;
      for (int u = 0; u < nd; ++u) seen = seen || S.dpart[s + u] == q;
      if (!seen) S.dpart[s + nd++] = q;
    }
  float wsum = 0.f;
  for (int t = s; t < e; ++t) {
    const int sl = I.img_off[I.pt_img[t]] + I.pt_slot[t];
    S.wx[t] = I.wx[sl];
    S.wy[t] = I.wy[sl];
    S.wxy[t] = I.wxy[sl];
    S.del[t] = 0;
    wsum += S.wx[t] + S.wy[t];
  }
  int pxs2 = 2 * pxs, pxsd = pxs;
  float X0 = (float)Xin[0], X1 = (float)Xin[1], X2 = (float)Xin[2];
  float Xo0 = X0, Xo1 = X1, Xo2 = X2, sig0 = 1.e20f, sig0opt = 1.e20f;
  int iflag = I.robustmode > 0 ? 2 : 1, iter = 1;
  bool cv = false;
  double s0 = 0.;
  int red = 0;
  tri_corr(I, S, s, e, X0, X1, X2, sig0opt, O.sig0v);
  if (I.weight_only) {
    wsum /= (float)pxs2;
    s0 += sig0opt / wsum;
    red += pxs2 - 3;
  }
  while (iflag > -1 && iter < 101) {
    double N[9] = {0., 0., 0., 0., 0., 0., 0., 0., 0.};
    for (int t = s; t < e; ++t) {
      const int j = I.pt_img[t];
      const double *P = I.pmat + 12 * j;
      const double x = S.p1[t], y = S.p2[t], P3 = S.p3[t], P1 = (double)S.p1[t] * S.p3[t],
                   P2 = (double)S.p2[t] * S.p3[t];
      double xp[3], yp[3];
      for (int c = 0; c < 3; ++c) {
        xp[c] = (double)P[c] * P3 - (double)P[8 + c] * P1;
        yp[c] = (double)P[4 + c] * P3 - (double)P[8 + c] * P2;
      }
      tri_calibrated(xp, yp, x, y, I.dist[2 * j], I.dist[2 * j + 1], I.K[9 * j], I.K[9 * j + 4], I.K[9 * j + 1]);
      double *W = S.Bw + 6 * (size_t)t;
      for (int c = 0; c < 3; ++c) {
        W[c] = xp[c] * S.wx[t] + yp[c] * S.wxy[t];
        W[3 + c] = yp[c] * S.wy[t] + xp[c] * S.wxy[t];
      }
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) N[r * 3 + c] += xp[r] * W[c] + yp[r] * W[3 + c];
      if (O.w3d)
        for (int c = 0; c < 3; ++c) {
          S.Bxy[6 * (size_t)t + c] = xp[c];
          S.Bxy[6 * (size_t)t + 3 + c] = yp[c];
        }
    }
    // pending weight blocks of this iteration (kept if it is accepted)
    if (O.w3d) {
      if (I.nparts == 1) {
        float *o = S.wt + 6 * (size_t)s;
        o[0] = (float)N[0];
        o[1] = (float)N[4];
        o[2] = (float)N[8];
        o[3] = (float)N[1];
        o[4] = (float)N[2];
        o[5] = (float)N[5];
      } else {
        for (int u = 0; u < nd; ++u) {
          const int q = S.dpart[s + u];
          double M[9] = {0., 0., 0., 0., 0., 0., 0., 0., 0.};
          for (int t = s; t < e; ++t) {
            if (I.part[I.pt_img[t]] == q) continue;
            const double *xp = S.Bxy + 6 * (size_t)t, *yp = xp + 3, *W = S.Bw + 6 * (size_t)t;
            for (int r = 0; r < 3; ++r)
              for (int c = 0; c < 3; ++c) M[r * 3 + c] += xp[r] * W[c] + yp[r] * W[3 + c];
          }
          float *o = S.wt + 6 * (size_t)(s + u);
          o[0] = (float)M[0];
          o[1] = (float)M[4];
          o[2] = (float)M[8];
          o[3] = (float)M[1];
          o[4] = (float)M[2];
          o[5] = (float)M[5];
        }
      }
    }
    N[0] *= 1.001;
    N[4] *= 1.001;
    N[8] *= 1.001;
    double Ni[9];
    inv3<double>(N, Ni);
    double dx[3] = {0., 0., 0.};
    for (int t = s; t < e; ++t) {
      const double *W = S.Bw + 6 * (size_t)t;
      const double c0 = S.corr[2 * (size_t)t], c1 = S.corr[2 * (size_t)t + 1];
      for (int r = 0; r < 3; ++r) {
        double v = 0.;
        for (int c = 0; c < 3; ++c) v += Ni[r * 3 + c] * (W[c] * c0 + W[3 + c] * c1);
        dx[r] += v;
      }
    }
    X0 = Xo0 + (float)dx[0];
    X1 = Xo1 + (float)dx[1];
    X2 = Xo2 + (float)dx[2];
    tri_corr(I, S, s, e, X0, X1, X2, sig0, O.sig0v);
    if (iflag == 1 && I.robustmode == 2) {
      for (int t = s; t < e; ++t)
        if (O.sig0v[t] * I.sig0w[I.pt_img[t]] > 16.f) {
          S.wx[t] *= 1.e-4f;
          S.wy[t] *= 1.e-4f;
          S.wxy[t] *= 1.e-4f;
          if (S.wx[t] + S.wy[t] < 2.e-8f) {
            S.wx[t] = S.wy[t] = 1.e-8f;
            S.wxy[t] = 0.f;
          }
          --pxsd;
          S.del[t] = 1;
        }
      if (pxsd < 2) break;
    }
    if (sig0 < sig0opt * 1.001) {
      if (sig0opt < sig0 * 1.05f) --iflag;
      if (!I.weight_only) {
        Xo0 = X0;
        Xo1 = X1;
        Xo2 = X2;
      }
      sig0opt = sig0;
      cv = true;
      if (O.w3d) {
        const int n = I.nparts == 1 ? 1 : nd;
        for (int u = 0; u < n; ++u) {
          const int q = I.nparts == 1 ? 0 : S.dpart[s + u];
          for (int k = 0; k < 6; ++k)
            O.w3d[((size_t)pi * I.nparts + q) * 6 + k] = S.wt[6 * (size_t)(s + u) + k];
        }
      }
    } else {
      --iflag;
    }
    if (I.weight_only) break;
    ++iter;
  }
  int kept = 0;
  for (int t = s; t < e; ++t) {
    const bool k = !(I.robustmode == 2 && S.del[t]);
    O.keep[t] = k ? 1 : 0;
    if (!k) pxs2 -= 2;
    kept += k;
  }
  if (kept < 2 || !cv) {
    for (int t = s; t < e; ++t) O.keep[t] = 0;
    O.s0[pi] = s0;  // the weight-only statistic is counted before the loop
    O.red[pi] = red;
    return;
  }
  O.conv[pi] = 1;
  if (!I.weight_only) {
    O.XX[3 * (size_t)pi] = Xo0;
    O.XX[3 * (size_t)pi + 1] = Xo1;
    O.XX[3 * (size_t)pi + 2] = Xo2;
    wsum /= (float)pxs2;
    s0 += sig0opt / wsum;
    red += pxs2 - 3;
  }
  O.s0[pi] = s0;
  O.red[pi] = red;
}

}  // namespace

}  // namespace rpba

using namespace rpba;

// CalcLSAXMulti over all points of b with the cameras Pd (12 doubles per
// image; null: b->pmat widened to double); s0_pt / red_pt (optional): every
// point's contribution to sig0io and to the redundancy.
int32_t rpba::triangulate_impl(const rpba_block *b, const double *Pd, const float *sig0w,
                               const rpba_tri_options *opt, const int32_t *part, int32_t nparts, double *XX_out,
                               uint8_t *keep, float *sig0v, uint8_t *conv, double *sig0io, int64_t *redundancy,
                               float *w3d, double *s0_pt, int32_t *red_pt) {
  if (!b || !opt || !XX_out || !keep || !sig0v || !conv || !sig0io || !redundancy) return RPBA_ERR_ARG;
  if (opt->robustmode < 0 || opt->robustmode > 2 || (opt->robustmode == 2 && !sig0w)) return RPBA_ERR_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= opt->device) return RPBA_ERR_NO_DEVICE;
  const int nc = b->n_images, np = b->n_points;
  if (nc < 1 || np < 0) return RPBA_ERR_ARG;
  const size_t nslot = (size_t)b->img_obs_off[nc], ntr = (size_t)b->pt_obs_off[np];
  for (size_t t = 0; t < ntr; ++t) {
    const int im = b->pt_obs_image[t];
    if (im < 0 || im >= nc || b->pt_obs_slot[t] < 0 || b->pt_obs_slot[t] >= b->img_obs_off[im + 1] - b->img_obs_off[im])
      return RPBA_ERR_ARG;
  }
  try {
    RPBA_CUDA_CHECK(cudaSetDevice(opt->device));
    cudaStream_t s;
    RPBA_CUDA_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    std::vector<void *> mem;
    struct Free {
      std::vector<void *> &m;
      cudaStream_t s;
      ~Free() {
        for (void *p : m) cudaFreeAsync(p, s);
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
      }
    } fr{mem, s};
    auto dev = [&](size_t bytes) {
      void *p = nullptr;
      RPBA_CUDA_CHECK(cudaMallocAsync(&p, bytes ? bytes : 16, s));
      mem.push_back(p);
      return p;
    };
    auto up = [&](const void *h, size_t bytes) {
      void *d = dev(bytes);
      if (bytes) RPBA_CUDA_CHECK(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, s));
      return d;
    };
    TriIn I;
    if (Pd) {
      I.pmat = (const double *)up(Pd, sizeof(double) * 12 * nc);
    } else {
      std::vector<double> P(12 * (size_t)nc);
      for (size_t i = 0; i < P.size(); ++i) P[i] = (double)b->pmat[i];
      I.pmat = (const double *)up(P.data(), sizeof(double) * P.size());
      RPBA_CUDA_CHECK(cudaStreamSynchronize(s));  // P is a local
    }
    I.K = (const float *)up(b->K, sizeof(float) * 9 * nc);
    I.dist = (const float *)up(b->distpara, sizeof(float) * 2 * nc);
    I.XX = (const float *)up(b->XX, sizeof(float) * 3 * np);
    I.xg = (const float *)up(b->xg, sizeof(float) * 2 * nslot);
    I.wx = (const float *)up(b->wx, sizeof(float) * nslot);
    I.wy = (const float *)up(b->wy, sizeof(float) * nslot);
    I.wxy = (const float *)up(b->wxy, sizeof(float) * nslot);
    I.sig0w = sig0w ? (const float *)up(sig0w, sizeof(float) * nc) : nullptr;
    I.img_off = (const int *)up(b->img_obs_off, sizeof(int) * (nc + 1));
    I.pt_off = (const int *)up(b->pt_obs_off, sizeof(int) * (np + 1));
    I.pt_img = (const int *)up(b->pt_obs_image, sizeof(int) * ntr);
    I.pt_slot = (const int *)up(b->pt_obs_slot, sizeof(int) * ntr);
    I.np = np;
    I.robustmode = opt->robustmode;
    I.weight_only = opt->weight_only != 0;
    I.part = w3d ? (const int *)up(part, sizeof(int) * nc) : nullptr;
    I.nparts = w3d ? nparts : 1;
    TriScratch S;
    S.wx = (float *)dev(sizeof(float) * ntr);
    S.wy = (float *)dev(sizeof(float) * ntr);
    S.wxy = (float *)dev(sizeof(float) * ntr);
    S.p1 = (float *)dev(sizeof(float) * ntr);
    S.p2 = (float *)dev(sizeof(float) * ntr);
    S.p3 = (float *)dev(sizeof(float) * ntr);
    S.corr = (double *)dev(sizeof(double) * 2 * ntr);
    S.Bw = (double *)dev(sizeof(double) * 6 * ntr);
    S.del = (uint8_t *)dev(ntr);
    S.Bxy = w3d ? (double *)dev(sizeof(double) * 6 * ntr) : nullptr;
    S.dpart = w3d ? (int *)dev(sizeof(int) * ntr) : nullptr;
    S.wt = w3d ? (float *)dev(sizeof(float) * 6 * ntr) : nullptr;
    TriOut O;
    O.XX = (double *)dev(sizeof(double) * 3 * np);
    O.keep = (uint8_t *)dev(ntr);
    O.conv = (uint8_t *)dev(np);
    O.sig0v = (float *)dev(sizeof(float) * ntr);
    O.s0 = (double *)dev(sizeof(double) * np);
    O.red = (int *)dev(sizeof(int) * np);
    O.w3d = w3d ? (float *)dev(sizeof(float) * 6 * (size_t)nparts * np) : nullptr;
    if (np > 0) k_triangulate<<<(np + 127) / 128, 128, 0, s>>>(I, S, O);
    RPBA_CUDA_CHECK(cudaGetLastError());
    std::vector<double> s0(np);
    std::vector<int> red(np);
    auto down = [&](void *h, const void *d, size_t bytes) {
      if (bytes) RPBA_CUDA_CHECK(cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, s));
    };
    down(XX_out, O.XX, sizeof(double) * 3 * np);
    down(keep, O.keep, ntr);
    down(conv, O.conv, np);
    down(sig0v, O.sig0v, sizeof(float) * ntr);
    down(s0.data(), O.s0, sizeof(double) * np);
    down(red.data(), O.red, sizeof(int) * np);
    if (w3d) down(w3d, O.w3d, sizeof(float) * 6 * (size_t)nparts * np);
    RPBA_CUDA_CHECK(cudaStreamSynchronize(s));
    // the reference accumulates these over the points in order
    double a = 0.;
    long long r = 0;
    for (int i = 0; i < np; ++i) {
      a += s0[i];
      r += red[i];
    }
    *sig0io = a;
    *redundancy = r;
    if (s0_pt) std::memcpy(s0_pt, s0.data(), sizeof(double) * np);
    if (red_pt) std::memcpy(red_pt, red.data(), sizeof(int32_t) * np);
  } catch (const CudaError &) {
    return RPBA_ERR_CUDA;
  }
  return RPBA_OK;
}

extern "C" int32_t rpba_triangulate(const rpba_block *b, const float *sig0w, const rpba_tri_options *opt,
                                    double *XX_out, uint8_t *keep, float *sig0v, uint8_t *conv, double *sig0io,
                                    int64_t *redundancy) {
  return triangulate_impl(b, nullptr, sig0w, opt, nullptr, 1, XX_out, keep, sig0v, conv, sig0io, redundancy, nullptr,
                          nullptr, nullptr);
}

extern "C" int32_t rpba_triangulate_parts(const rpba_block *b, const float *sig0w, const rpba_tri_options *opt,
                                          const int32_t *part, int32_t nparts, double *XX_out, uint8_t *keep,
                                          float *sig0v, uint8_t *conv, double *sig0io, int64_t *redundancy,
                                          float *w3d) {
  if (!b || !part || nparts < 1 || !w3d) return RPBA_ERR_ARG;
  for (int i = 0; i < b->n_images; ++i)
    if (part[i] < 0 || part[i] >= nparts) return RPBA_ERR_ARG;
  return triangulate_impl(b, nullptr, sig0w, opt, part, nparts, XX_out, keep, sig0v, conv, sig0io, redundancy, w3d,
                          nullptr, nullptr);
}
