/*
 * rpba_oracle.cpp -- CPU restatement of RPBA's global robust bundle
 * adjustment.  TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline leg use it as the checker and the CPU baseline.
 * The product (rpba_b200/) never links, loads or calls it.
 *
 * PARITY UNPINNED: the reference cannot be compiled in this environment
 * (it needs Eigen, Boost and METIS, none of which is installed) and it ships
 * no tests, golden vectors or datasets.  The restatement is pinned instead by
 * known-answer tests: rotation round trips, finite-difference checks of every
 * Jacobian column, the 3x3 / LU inverses, and a zero-noise scene.
 *
 * What it restates (reference file:line):
 *   InputBlock / OutputBlock            rpba.cpp:180-338
 *   angle-axis <-> R                    rpba.cpp:343-439
 *   CalcPLSA single-LSA + Exteval       rpbacore.cpp:28-98, 511-527
 *   EvalLSA / CalcCorrPointMulti        rpbacore.cpp:778-837, 882-941
 *   LSA ctor, PrepareIteration          rbacore.cpp:37-229
 *   Adjust                              rbacore.cpp:333-616
 *   OutputLSAc, PrepareCameras          rbacore.cpp:644-700
 *   PrepareWeights2D, Reweight2D        rbacore.cpp:704-783, 823-887
 *   StoreResultsIteration, RobustDelete rbacore.cpp:891-995
 *   EncodeCameras                       rbacore.cpp:999-1087
 *   CalcBundleSep                       rbacore.cpp:1094-1195
 *   CalcCorrections, CalcDerivatives    rbacore.cpp:1201-1616
 *   eCalcCalibratedDerivativesX/3       rbacore.cpp:1620-1673
 *   DecodeCameras                       rbacore.cpp:1733-1800
 *   SparsePCG, eAAdv, evvdv             rbacore.cpp:1807-1914, 2048-2084
 *   PointXXvIn / PointXXvOut            rbacore.cpp:1918-2010
 *   Cayley rotation                     rbacore.cpp:2014-2043
 *   RadialReconstructionImage           rpba.h:850-857
 *   RectifyRotationMatrix3/4            rpba.h:876-960
 * The float/double boundaries, loop orders and constants follow the
 * reference.  Eigen's 3x3 inverse (cofactors) and dynamic inverse (partial
 * pivot LU) are restated from their mathematical definition, so agreement
 * with an Eigen build is to roundoff, not bitwise.  Only the single global
 * LSA branch of CalcPLSA is restated (GCP/aoflag code paths are not).
 *
 * Build: oracle/Makefile (g++ -O2 -ffp-contract=off, so that no FMA
 * contraction changes the roundoff of the restated expressions).
 */
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <thread>
#include <map>
#include <random>
#include <sstream>
#include <string>
#include <vector>
#include <chrono>

#include "../include/rpba_b200.h"

namespace {

/* ------------------------------------------------------------------ math */

/* Cayley rotation, rbacore.cpp:2014-2043. */
void cayley(double a, double b, double c, double R[9]) {
  const double a2 = a * a, b2 = b * b, c2 = c * c;
  const double ab = a * b, ac = a * c, bc = b * c;
  double abc = 4 + a2 + b2 + c2;
  if (std::fabs(abc) < 1.e-20) {
    abc = abc < 0. ? -1.e20 : 1.e20;
  } else {
    abc = 1. / abc;
  }
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

/* Quaternion re-orthonormalisation, rpba.h:876-913 (the 3x3 part of
 * RectifyRotationMatrix4 is the same computation).  R row major with
 * row stride rs (3 for a 3x3, 4 for the left part of a 3x4). */
void rectify(double *R, int rs) {
  auto at = [&](int r, int c) -> double & { return R[r * rs + c]; };
  double a[3];
  a[0] = at(2, 1) - at(1, 2);
  a[1] = at(0, 2) - at(2, 0);
  a[2] = at(1, 0) - at(0, 1);
  for (int i = 0; i < 3; ++i)
    if (std::fabs(a[i]) < 1.e-20) a[i] = 1.e-20;
  const double al = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
  a[0] /= al;
  a[1] /= al;
  a[2] /= al;
  const double phi = std::atan2(al, at(0, 0) + at(1, 1) + at(2, 2) - 1.);
  double q[4];
  q[0] = std::cos(phi * 0.5);
  const double s = std::sin(phi * 0.5);
  for (int i = 1; i < 4; ++i) q[i] = a[i - 1] * s;
  at(0, 0) = q[0] * q[0] + q[1] * q[1] - q[2] * q[2] - q[3] * q[3];
  at(0, 1) = 2 * (q[1] * q[2] - q[0] * q[3]);
  at(0, 2) = 2 * (q[1] * q[3] + q[0] * q[2]);
  at(1, 0) = 2 * (q[2] * q[1] + q[0] * q[3]);
  at(1, 1) = q[0] * q[0] - q[1] * q[1] + q[2] * q[2] - q[3] * q[3];
  at(1, 2) = 2 * (q[2] * q[3] - q[0] * q[1]);
  at(2, 0) = 2 * (q[3] * q[1] - q[0] * q[2]);
  at(2, 1) = 2 * (q[3] * q[2] + q[0] * q[1]);
  at(2, 2) = q[0] * q[0] - q[1] * q[1] - q[2] * q[2] + q[3] * q[3];
}

/* ComputeRotationMatrixfromRodriguesAngle, rpba.cpp:343-366 (float out). */
void angleaxis_to_R(double a, double b, double c, float R[9]) {
  const double a2 = a * a, b2 = b * b, c2 = c * c;
  const double ab = a * b, ac = a * c, bc = b * c;
  const double aa = std::sqrt(a2 + b2 + c2);
  const double ct = aa == 0. ? 0.5 : (1. - std::cos(aa)) / (aa * aa);
  const double st = aa == 0. ? 1 : std::sin(aa) / aa;
  R[0] = (float)(1. - (b2 + c2) * ct);
  R[1] = (float)(ab * ct - c * st);
  R[2] = (float)(ac * ct + b * st);
  R[3] = (float)(ab * ct + c * st);
  R[4] = (float)(1. - (c2 + a2) * ct);
  R[5] = (float)(bc * ct - a * st);
  R[6] = (float)(ac * ct - b * st);
  R[7] = (float)(bc * ct + a * st);
  R[8] = (float)(1. - (a2 + b2) * ct);
}

/* ComputeRodriguesAnglefromRotationMatrix, rpba.cpp:371-439.  R is the
 * float 3x3 (row major). */
void R_to_angleaxis(const float *R, double *a, double *b, double *c) {
  /* the entries stay float as in the reference: a sum or difference of
   * two entries is rounded to float, anything with a double constant is
   * double */
  auto m = [&](int r, int cc) -> float { return R[r * 3 + cc]; };
  const double e0 = 0.01, e1 = 0.1, pi = 3.14159265358979323846;
  const double tr = (m(0, 0) + m(1, 1) + m(2, 2) - 1.) * 0.5;
  if (std::fabs(m(0, 1) - m(1, 0)) < e0 && std::fabs(m(1, 2) - m(2, 1)) < e0 &&
      std::fabs(m(0, 2) - m(2, 0)) < e0) {
    if (std::fabs(m(0, 1) + m(1, 0)) < e1 && std::fabs(m(1, 2) + m(2, 1)) < e1 &&
        std::fabs(m(0, 2) + m(2, 0)) < e1 && tr > 0.9) {
      *a = *b = *c = 0.;
      return;
    }
    const double xx = (m(0, 0) + 1.) * 0.5, yy = (m(1, 1) + 1.) * 0.5,
                 zz = (m(2, 2) + 1.) * 0.5;
    const double xy = (m(0, 1) + m(1, 0)) * 0.25, xz = (m(0, 2) + m(2, 0)) * 0.25,
                 yz = (m(1, 2) + m(2, 1)) * 0.25;
    if (xx > yy && xx > zz) {
      if (xx < e0) {
        *a = 0.;
        *b = *c = std::sqrt(0.5) * pi;
        return;
      }
      const double t = std::sqrt(xx);
      *a = t * pi;
      *b = xy / t * pi;
      *c = xz / t * pi;
      return;
    }
    if (yy > zz) {
      if (yy < e0) {
        *a = *c = std::sqrt(0.5) * pi;
        *b = 0.;
        return;
      }
      const double t = std::sqrt(yy);
      *a = xy / t * pi;
      *b = t * pi;
      *c = yz / t * pi;
      return;
    }
    if (zz < e0) {
      *a = *b = std::sqrt(0.5) * pi;
      *c = 0.;
      return;
    }
    const double t = std::sqrt(zz);
    *a = xz / t * pi;
    *b = yz / t * pi;
    *c = t * pi;
    return;
  }
  const double aa = std::acos(tr);
  const double bb = 0.5 * aa / std::sin(aa);
  *a = bb * (m(2, 1) - m(1, 2));
  *b = bb * (m(0, 2) - m(2, 0));
  *c = bb * (m(1, 0) - m(0, 1));
}

/* 3x3 inverse by cofactors (the closed form Eigen uses for fixed 3x3,
 * called at rbacore.cpp:1344).  Returns the determinant of the input. */
double inv3(const double *m, double *out) {
  auto M = [&](int r, int c) { return m[r * 3 + c]; };
  double C[9];
  for (int i = 0; i < 3; ++i) {
    const int i1 = (i + 1) % 3, i2 = (i + 2) % 3;
    for (int j = 0; j < 3; ++j) {
      const int j1 = (j + 1) % 3, j2 = (j + 2) % 3;
      C[i * 3 + j] = M(i1, j1) * M(i2, j2) - M(i1, j2) * M(i2, j1);
    }
  }
  const double det = C[0] * M(0, 0) + C[3] * M(1, 0) + C[6] * M(2, 0);
  const double id = 1. / det;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) out[i * 3 + j] = C[j * 3 + i] * id;
  return det;
}

/* n x n inverse by LU with partial pivoting (Eigen's dynamic-size
 * inverse(), called at rbacore.cpp:1841).  n <= 16. */
void lu_inverse(int n, const double *A, double *Ai) {
  double LU[16 * 16];
  int perm[16];
  std::memcpy(LU, A, sizeof(double) * n * n);
  for (int i = 0; i < n; ++i) perm[i] = i;
  for (int k = 0; k < n; ++k) {
    int p = k;
    double best = std::fabs(LU[k * n + k]);
    for (int r = k + 1; r < n; ++r) {
      const double v = std::fabs(LU[r * n + k]);
      if (v > best) {
        best = v;
        p = r;
      }
    }
    if (p != k) {
      for (int c = 0; c < n; ++c) std::swap(LU[k * n + c], LU[p * n + c]);
      std::swap(perm[k], perm[p]);
    }
    const double piv = LU[k * n + k];
    for (int r = k + 1; r < n; ++r) {
      const double l = LU[r * n + k] / piv;
      LU[r * n + k] = l;
      for (int c = k + 1; c < n; ++c) LU[r * n + c] -= l * LU[k * n + c];
    }
  }
  for (int col = 0; col < n; ++col) {
    double y[16];
    for (int i = 0; i < n; ++i) {
      double s = perm[i] == col ? 1. : 0.;
      for (int j = 0; j < i; ++j) s -= LU[i * n + j] * y[j];
      y[i] = s;
    }
    for (int i = n - 1; i >= 0; --i) {
      double s = y[i];
      for (int j = i + 1; j < n; ++j) s -= LU[i * n + j] * y[j];
      y[i] = s / LU[i * n + i];
    }
    for (int i = 0; i < n; ++i) Ai[i * n + col] = y[i];
  }
}

std::string fmt_g(double v) {
  char buf[64];
  std::snprintf(buf, sizeof buf, "%g", v);
  return buf;
}

/* ---------------------------------------------------------------- LSA */

/* Test hook: the order in which the off-diagonal blocks of a column are
 * visited in the SpMV.  0 the reference's (map order), 1 reversed, 2 rotated
 * by half, 3..19 a shuffle seeded by the variant; 20..39 the map order with
 * the PCG's sums over cameras blocked (dot_group); >= 40 the same sums as
 * pairwise trees (tree_leaf).  Used only to measure
 * how sensitive the reference's inexact PCG is to summation order. */
int g_order_variant = 0;

struct Opts {
  bool robust = true;
  bool addf[3] = {true, true, true};
  int solver = RPBA_SOLVER_PCG;
  int max_lm = -1;
};

/* GCP mode of the LSA (gcpflag / aoflag, rbacore.cpp:36-125, 233-329): the
 * per-partition LSA of the parallel RPBA.  Every camera of the block is
 * free (no gauge camera, nrioff = nrpari * nrimages); points shared with
 * other partitions carry a 3-D prior (CalcDerivatives3DGCP,
 * rbacore.cpp:1677-1729).  gcpinfo: per block point, its GCP index (into
 * gcpdata) or -1; W3: 6 weights (XX, YY, ZZ, XY, XZ, YZ) per GCP point of
 * this LSA, in the order the LSA keeps its points (the W3ijit of the
 * reference); ncam_total: the scene's camera count (the reference's
 * nrcameras, which enters the unknown count). */
struct GcpIn {
  const int32_t *gcpinfo;
  const float *W3;
  const double *gcpdata;
  int ncam_total;
  const double *Pd = nullptr;  /* the cameras in double precision (12 per image), or null */
};

class LSA {
 public:
  LSA(const rpba_block *blk, const Opts &o, std::string *os);
  LSA(const rpba_block *blk, const Opts &o, std::string *os, const GcpIn &g);
  /* Adjust(false, os, true, 0, W3, true, gcpdata), rbacore.cpp:333-616: one
   * damped step in GCP mode, stored unconditionally. */
  int adjust_gcp_step();
  /* rbacore.cpp:333-616; returns an rpba_status. */
  int adjust(rpba_report *rep);
  /* OutputLSAc, rbacore.cpp:644-666 + PointXXvOut rbacore.cpp:1978-2010. */
  void output(rpba_block *blk);

  /* test hooks */
  int xm_size() const { return (int)XPM.size(); }
  void setup_pass_for_tests();
  void residuals_at(const std::vector<double> &XM, std::vector<double> &res);
  void jacobian_of(int tobs, double *Bc, int *ncols, int *coff, double *Bp);
  double final_cost(double *rms);

  int status = RPBA_OK;
  int bad_setup = 0;

  /* problem */
  const rpba_block *b;
  int nimg, XXnr;
  Opts opt;
  int nadd;
  std::string *os;

  /* cameras: accepted (P, Kc, dc) and trial (eRMn, ePCn, Kn, dn) */
  std::vector<double> P;          /* 12 per image, PMatrices (double) */
  std::vector<double> Kc, dc;     /* cameras                          */
  std::vector<double> Kn, dn;     /* camerasnew                       */
  std::vector<double> Rb, PCb;    /* pass-start eRM / ePC per image   */
  std::vector<double> Rn, PCn;    /* eRMnew / ePCnew per image        */

  /* points and tracks (local indexing, PointXXvIn) */
  int nrpts = 0;
  std::vector<int> nrpv;
  std::vector<int> toff, timg, tslot; /* CSR tracks                   */
  std::vector<float> wold;            /* Wijoldv, 3 per track obs     */
  std::vector<float> W;               /* Wij, 3 per track obs         */
  std::vector<char> isflag, isflagnew;
  std::vector<float> sig0rmv;
  std::vector<double> XX, XXnew;

  /* parameterisation */
  int minimagenr = 2, minimagenrdel = 2;
  int normcamera = -1, esvm[3] = {0, 1, 2}, esvmaxm = 2;
  int nrpari = 0, nrparir = 0, nrioff = 0, nrioff3 = 0;
  std::vector<int> camparv;
  bool lflflag = false;
  float ihw2 = 1.f;
  double defdiff = 5000.;
  const float kf = 9.f;

  /* LM bookkeeping */
  std::vector<double> XPM, XPMn, x;
  int imagepointnr = 0, nrobs = 0, nrunknowns = 0, redundancy = 0;
  int nrobsnew = 0, nrunknownsnew = 0, redundancynew = 0;
  float sig0 = 0.f, sig0old = 0.f, sig0in = 0.f;
  float wsum = 0.f, wsumg = 0.f;
  std::vector<float> sig00v;
  bool iniflag = true;
  int begini = 1;
  int64_t pcg_iters = 0;

  /* reduced camera system: per camera diagonal block + rhs, off-diagonal
   * blocks per column keyed by row (descending row = ascending skyline
   * offset, the order eAAdv visits them in). */
  std::vector<int> nbv, nev;
  std::vector<std::vector<double>> Dg, rhs;
  std::vector<std::map<int, std::vector<double>, std::greater<int>>> Off;

  /* GCP mode */
  bool ao = false;
  int ncam_total = 0, nrgcp = 0, nrobsao = 0;
  std::vector<int> gcpi;       /* per kept point: GCP index or -1       */
  const float *W3 = nullptr;   /* 6 per GCP point in gcpnum order       */
  const double *gdata = nullptr;
  float sig0ao = 0.f, wsumao = 0.f, sig0aoi = 0.f, sig0aoiold = 0.f;

  /* per point scratch */
  double Vp[9], Vpi[9], gp[3];
  std::vector<std::vector<double>> Wl; /* eNlij per track obs (n x 3) */

  void prepare_cameras();
  void encode_cameras();
  void decode_cameras(const std::vector<double> &XM);
  void prepare_weights(int it);
  void reweight(int iflag);
  void store_results();
  void robust_delete();
  bool calc_bundle_sep(double multfact);
  void calc_corrections(bool solveflag, double multfact1, const std::vector<double> &XM,
                        bool srmvflag, bool derivflag);
  void sparse_pcg();
  void direct_solve();
  int cam_np(int k) const { return camparv[k + 1] - camparv[k]; }

  /* one observation: residual + (optionally) derivatives */
  struct ObsEval {
    double ex3[3], ex3u[2], xs3, d1, d2;
    bool nan;
  };
  void eval_obs(int k, int slot, const double *X, ObsEval &e) const;
  void derivs(const ObsEval &e, int k, const float *w, double *Bc, int *ncols,
              double *Bp) const;
};

LSA::LSA(const rpba_block *blk, const Opts &o, std::string *os_)
    : LSA(blk, o, os_, GcpIn{nullptr, nullptr, nullptr, 0}) {}

LSA::LSA(const rpba_block *blk, const Opts &o, std::string *os_, const GcpIn &g) : b(blk), opt(o), os(os_) {
  ao = g.gcpinfo != nullptr;
  W3 = g.W3;
  gdata = g.gcpdata;
  ncam_total = g.ncam_total;
  nimg = blk->n_images;
  XXnr = blk->n_points;
  nadd = (int)o.addf[0] + (int)o.addf[1] + (int)o.addf[2];
  /* CalcPLSA: ihw2 from iwidth=iheight=1 (rpba.cpp:264-265, rpbacore.cpp:87-90) */
  ihw2 = 0.f;
  for (int i = 0; i < nimg; ++i) ihw2 += (float)((1 + 1) * (1 + 1)) * 0.25f;
  ihw2 /= (float)nimg;
  defdiff = 5000. / (double)std::sqrt(ihw2); /* 5000./sqrtf(ihw2i), rbacore.cpp:48 */
  minimagenr = 2;
  minimagenrdel = nimg > 2 ? 3 : 2;

  P.resize(12 * nimg);
  for (int i = 0; i < 12 * nimg; ++i) P[i] = g.Pd ? g.Pd[i] : (double)blk->pmat[i];

  /* PointXXvIn, rbacore.cpp:1918-1974 (all images of the block selected);
   * in GCP mode a GCP point is kept with a single observation, if its GCP
   * index is above 0 (the reference's test is gcpinfoin[i] > 0) */
  toff.push_back(0);
  for (int i = 0; i < XXnr; ++i) {
    const int s = blk->pt_obs_off[i], e = blk->pt_obs_off[i + 1];
    int n = 0;
    for (int j = s; j < e; ++j)
      if (blk->pt_obs_image[j] > -1) ++n;
    const double Z = (double)blk->XX[3 * i + 2];
    if (std::fabs(Z) > 1.e-8 && (n >= minimagenr || (ao && g.gcpinfo[i] > 0 && n > 0))) {
      nrpv.push_back(i);
      if (ao) {
        gcpi.push_back(g.gcpinfo[i]);
        if (g.gcpinfo[i] > -1) ++nrgcp;
      }
      for (int j = s; j < e; ++j)
        if (blk->pt_obs_image[j] > -1) {
          timg.push_back(blk->pt_obs_image[j]);
          tslot.push_back(blk->pt_obs_slot[j]);
        }
      toff.push_back((int)timg.size());
      ++nrpts;
    }
  }
  XX.resize(3 * nrpts);
  for (int i = 0; i < nrpts; ++i)
    for (int j = 0; j < 3; ++j) XX[3 * i + j] = (double)blk->XX[3 * nrpv[i] + j];
  XXnew = XX;

  prepare_cameras();
  if (ao) normcamera = -1; /* rbacore.cpp:697-698 */

  /* PrepareIteration, rbacore.cpp:127-229 */
  camparv.assign(nimg + 2, 0);
  Rb.assign(9 * nimg, 0.);
  PCb.assign(3 * nimg, 0.);
  Rn.assign(9 * nimg, 0.);
  PCn.assign(3 * nimg, 0.);
  rectify(&P[0], 4);
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) Rn[r * 3 + c] = P[r * 4 + c];
  for (int i = 0; i < 3; ++i)
    PCn[i] = Rn[0 * 3 + i] * P[3] + Rn[1 * 3 + i] * P[7] + Rn[2 * 3 + i] * P[11];
  nrparir = 5 + nadd;
  nrpari = 6 + nadd;
  Kc.resize(9 * nimg);
  dc.resize(2 * nimg);
  for (int i = 0; i < nimg; ++i) {
    for (int j = 0; j < 9; ++j) Kc[9 * i + j] = (double)blk->K[9 * i + j];
    dc[2 * i] = (double)blk->distpara[2 * i];
    dc[2 * i + 1] = (double)blk->distpara[2 * i + 1];
  }
  Kn = Kc;
  dn = dc;
  lflflag = false;
  for (int i = 0; i < nimg; ++i)
    if (blk->K[9 * i] > 2.f || blk->K[9 * i + 4] > 2.f) {
      lflflag = true;
      break;
    }
  nrioff = ao ? nrpari * nimg : nadd + nrparir + nrpari * (nimg - 2);
  sig00v.assign(nimg, 0.f);
  /* xpmsize with nrcameras = the scene's camera count (rbacore.cpp:324) */
  const int xpmsize = nimg * 6 + 3 * XXnr + 7 * (ao ? std::max(ncam_total, nimg) : nimg);
  XPM.assign(xpmsize, 0.);
  XPMn.assign(xpmsize, 0.);
  if (nimg < 1 || (!ao && (nimg < 2 || normcamera < 1))) bad_setup = 1;
}

/* PrepareCameras, rbacore.cpp:670-700: normcamera = image whose R*t is
 * farthest from image 0's. */
void LSA::prepare_cameras() {
  std::vector<double> Tv(3 * nimg);
  for (int i = 0; i < nimg; ++i) {
    const double *p = &P[12 * i];
    for (int r = 0; r < 3; ++r) Tv[3 * i + r] = p[r * 4] * p[3] + p[r * 4 + 1] * p[7] + p[r * 4 + 2] * p[11];
  }
  double nd = 0.;
  normcamera = -1;
  for (int i = 1; i < nimg; ++i) {
    double d = 0;
    for (int j = 0; j < 3; ++j) d += (Tv[3 * i + j] - Tv[j]) * (Tv[3 * i + j] - Tv[j]);
    if (d > nd) {
      nd = d;
      normcamera = i;
    }
  }
}

/* EncodeCameras, rbacore.cpp:999-1087. */
void LSA::encode_cameras() {
  for (int k = 0; k < nimg + 1; ++k) camparv[k] = 0;
  if (ao) {
    /* every camera free, rotation, PC and the additional parameters */
    camparv[1] = nrpari;
    for (int k = 0; k < nimg; ++k) {
      const int cp = camparv[k];
      double *p = &P[12 * k];
      rectify(p, 4);
      double *R = &Rb[9 * k];
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) R[r * 3 + c] = p[r * 4 + c];
      for (int i = 0; i < 3; ++i)
        PCb[3 * k + i] = R[0 * 3 + i] * p[3] + R[1 * 3 + i] * p[7] + R[2 * 3 + i] * p[11];
      for (int i = 0; i < 6; ++i) XPM[cp + i] = 0.;
      int a = 5 + cp;
      if (opt.addf[0]) XPM[++a] = dc[2 * k];
      if (opt.addf[1]) XPM[++a] = dc[2 * k + 1];
      if (opt.addf[2]) XPM[++a] = Kc[9 * k];
      camparv[k + 2] = camparv[k + 1] + nrpari;
    }
    nrioff3 = nrioff + 3 * nrpts;
    return;
  }
  camparv[1] = nadd;
  int addp = -1;
  if (opt.addf[0]) XPM[++addp] = dc[0];
  if (opt.addf[1]) XPM[++addp] = dc[1];
  if (opt.addf[2]) XPM[++addp] = Kc[0];
  for (int k = 0; k < nimg - 1; ++k) {
    const int img = k + 1;
    const int cp = camparv[k + 1];
    double *p = &P[12 * img];
    rectify(p, 4);
    double *R = &Rb[9 * img];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) R[r * 3 + c] = p[r * 4 + c];
    for (int i = 0; i < 3; ++i)
      PCb[3 * img + i] = R[0 * 3 + i] * p[3] + R[1 * 3 + i] * p[7] + R[2 * 3 + i] * p[11];
    for (int i = 0; i < 3; ++i) XPM[cp + i] = 0.;
    if (k == normcamera - 1) {
      float maxv = 0.f;
      int maxi = 0;
      for (int i = 0; i < 3; ++i)
        if (std::fabs(PCb[3 * img + i]) > maxv) {
          maxv = (float)std::fabs(PCb[3 * img + i]);
          maxi = i;
        }
      int ii = -1;
      for (int i = 0; i < 3; ++i)
        if (i != maxi) esvm[++ii] = i;
      esvmaxm = maxi;
      XPM[cp + 3] = XPM[cp + 4] = 0.;
      int a = 4 + cp;
      if (opt.addf[0]) XPM[++a] = dc[2 * img];
      if (opt.addf[1]) XPM[++a] = dc[2 * img + 1];
      if (opt.addf[2]) XPM[++a] = Kc[9 * img];
      camparv[k + 2] = cp + nrparir;
    } else {
      for (int i = 0; i < 3; ++i) XPM[cp + 3 + i] = 0.;
      int a = 5 + cp;
      if (opt.addf[0]) XPM[++a] = dc[2 * img];
      if (opt.addf[1]) XPM[++a] = dc[2 * img + 1];
      if (opt.addf[2]) XPM[++a] = Kc[9 * img];
      camparv[k + 2] = camparv[k + 1] + nrpari;
    }
  }
  nrioff3 = nrioff + 3 * nrpts;
}

/* DecodeCameras, rbacore.cpp:1733-1800. */
void LSA::decode_cameras(const std::vector<double> &XM) {
  for (int k = ao ? 0 : 1; k < nimg; ++k) {
    const int cp = camparv[k];
    double Ra[9];
    cayley(XM[cp], XM[cp + 1], XM[cp + 2], Ra);
    const double *B = &Rb[9 * k];
    double *R = &Rn[9 * k];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j)
        R[i * 3 + j] = Ra[i * 3 + 0] * B[0 * 3 + j] + Ra[i * 3 + 1] * B[1 * 3 + j] + Ra[i * 3 + 2] * B[2 * 3 + j];
    rectify(R, 3);
    double e[3];
    if (k == normcamera) {
      e[esvm[0]] = XM[cp + 3];
      e[esvm[1]] = XM[cp + 4];
      e[esvmaxm] = 0.;
    } else {
      for (int i = 0; i < 3; ++i) e[i] = XM[cp + 3 + i];
    }
    for (int i = 0; i < 3; ++i) PCn[3 * k + i] = e[i] + PCb[3 * k + i];
    int a = k == normcamera ? 4 : 5;
    if (opt.addf[0]) dn[2 * k] = XM[++a + cp];
    if (opt.addf[1]) dn[2 * k + 1] = XM[++a + cp];
    if (opt.addf[2]) Kn[9 * k] = Kn[9 * k + 4] = XM[++a + cp];
    Kn[9 * k + 8] = 1.;
  }
  if (ao) return;
  int a = -1;
  if (opt.addf[0]) dn[0] = XM[++a];
  if (opt.addf[1]) dn[1] = XM[++a];
  if (opt.addf[2]) Kn[0] = Kn[4] = XM[++a];
  Kn[8] = 1.;
}

/* PrepareWeights2D, rbacore.cpp:704-783.  Pass 0 copies the caller's
 * weights into Wijoldv; pass 1 re-sums the (pruned) Wijoldv. */
void LSA::prepare_weights(int it) {
  const int n = toff[nrpts];
  wsum = 0.f;
  if (opt.robust) {
    if (it == 0) {
      wold.resize(3 * n);
      for (int o = 0; o < n; ++o) {
        const int img = timg[o], sl = b->img_obs_off[img] + tslot[o];
        wold[3 * o] = b->wx[sl];
        wold[3 * o + 1] = b->wy[sl];
        wold[3 * o + 2] = b->wxy[sl];
        wsum += wold[3 * o] + wold[3 * o + 1];
      }
    } else {
      for (int o = 0; o < n; ++o) wsum += (wold[3 * o] + wold[3 * o + 1]);
    }
    W = wold;
  } else {
    W.resize(3 * n);
    for (int o = 0; o < n; ++o) {
      const int img = timg[o], sl = b->img_obs_off[img] + tslot[o];
      W[3 * o] = b->wx[sl];
      W[3 * o + 1] = b->wy[sl];
      W[3 * o + 2] = b->wxy[sl];
      wsum += b->wx[sl] + b->wy[sl];
    }
  }
}

/* Reweight2D, rbacore.cpp:823-887. */
void LSA::reweight(int iflag) {
  std::vector<std::vector<float>> lists(nimg);
  for (int p = 0; p < nrpts; ++p) {
    int pxs = (toff[p + 1] - toff[p]) * 2;
    if (pxs < 4) pxs = 4;
    const float rf = (float)pxs / (float)(pxs - 3);
    const float redfac = rf * rf;
    for (int o = toff[p]; o < toff[p + 1]; ++o) lists[timg[o]].push_back(sig0rmv[o] * redfac);
  }
  for (int i = 0; i < nimg; ++i) {
    std::sort(lists[i].begin(), lists[i].end());
    sig00v[i] = 1.f / (lists[i][(int)lists[i].size() / 2] * 2.1981f);
    if (iflag > 1) sig00v[i] *= 0.001f;
  }
  wsum = 0.f;
  const int n = toff[nrpts];
  for (int o = 0; o < n; ++o) {
    float ww = sig0rmv[o] * sig00v[timg[o]];
    isflag[o] = ww > kf;
    if (isflag[o]) {
      ww = 1.e-4f;
      nrobs -= 2;
    } else {
      ww = 1.f;
    }
    W[3 * o] = ww * wold[3 * o];
    W[3 * o + 1] = ww * wold[3 * o + 1];
    W[3 * o + 2] = ww * wold[3 * o + 2];
    if (W[3 * o] + W[3 * o + 1] < 2.e-8f) {
      W[3 * o] = W[3 * o + 1] = 1.e-8f;
      W[3 * o + 2] = 0.f;
    }
    wsum += W[3 * o] + W[3 * o + 1];
  }
}

/* StoreResultsIteration, rbacore.cpp:891-918. */
void LSA::store_results() {
  XPM = XPMn;
  for (int k = 0; k < nimg; ++k) {
    double *p = &P[12 * k];
    const double *R = &Rn[9 * k], *c = &PCn[3 * k];
    for (int r = 0; r < 3; ++r) {
      for (int cc = 0; cc < 3; ++cc) p[r * 4 + cc] = R[r * 3 + cc];
      p[r * 4 + 3] = R[r * 3] * c[0] + R[r * 3 + 1] * c[1] + R[r * 3 + 2] * c[2];
    }
  }
  Kc = Kn;
  dc = dn;
  XX = XXnew;
  isflagnew = isflag;
  nrobsnew = nrobs;
  nrunknownsnew = nrunknowns;
  redundancynew = redundancy;
}

/* RobustDelete, rbacore.cpp:922-995 (no GCPs). */
void LSA::robust_delete() {
  std::vector<int> noff{0}, nimg_, nslot;
  std::vector<float> nw;
  std::vector<double> nX;
  std::vector<int> nnrpv;
  int kept = 0;
  for (int p = 0; p < nrpts; ++p) {
    int nflag = 0;
    for (int o = toff[p]; o < toff[p + 1]; ++o) nflag += isflagnew[o] ? 1 : 0;
    const int sz = toff[p + 1] - toff[p];
    if (nflag > 0 && sz - nflag < minimagenrdel) continue; /* point erased */
    for (int o = toff[p]; o < toff[p + 1]; ++o) {
      if (nflag > 0 && isflagnew[o]) continue;
      nimg_.push_back(timg[o]);
      nslot.push_back(tslot[o]);
      nw.push_back(wold[3 * o]);
      nw.push_back(wold[3 * o + 1]);
      nw.push_back(wold[3 * o + 2]);
    }
    noff.push_back((int)nimg_.size());
    nnrpv.push_back(nrpv[p]);
    for (int j = 0; j < 3; ++j) nX.push_back(XX[3 * p + j]);
    ++kept;
  }
  toff.swap(noff);
  timg.swap(nimg_);
  tslot.swap(nslot);
  wold.swap(nw);
  nrpv.swap(nnrpv);
  XX.swap(nX);
  nrpts = kept;
  XXnew = XX;
}

/* Projection of one observation: CalcCorrections rbacore.cpp:1238-1307. */
void LSA::eval_obs(int k, int slot, const double *X, ObsEval &e) const {
  const double *R = &Rn[9 * k], *c = &PCn[3 * k];
  const double v0 = X[0] + c[0], v1 = X[1] + c[1], v2 = X[2] + c[2];
  e.ex3[0] = R[0] * v0 + R[1] * v1 + R[2] * v2;
  e.ex3[1] = R[3] * v0 + R[4] * v1 + R[5] * v2;
  e.ex3[2] = R[6] * v0 + R[7] * v1 + R[8] * v2;
  double xs3 = e.ex3[2];
  if (std::fabs(xs3) < 1.e-3)
    xs3 = xs3 < 0. ? -1.e3 : 1.e3;
  else
    xs3 = 1. / xs3;
  e.ex3[0] *= xs3;
  e.ex3[1] *= xs3;
  e.ex3[2] = 1.;
  e.xs3 = xs3;
  double u = e.ex3[0], v = e.ex3[1];
  const double dist = u * u + v * v;
  const double z = 1. + (dn[2 * k] * dist + dn[2 * k + 1] * dist * dist);
  u *= z;
  v *= z;
  e.ex3u[0] = u;
  e.ex3u[1] = v;
  const double *K = &Kn[9 * k];
  const double c0 = u * K[0] + v * K[1] + K[2];
  const double c1 = v * K[4] + K[5];
  const int sl = b->img_obs_off[k] + slot;
  double d1 = (double)b->xg[2 * sl] - c0;
  double d2 = (double)b->xg[2 * sl + 1] - c1;
  if (d1 > defdiff) d1 = defdiff;
  if (d1 < -defdiff) d1 = -defdiff;
  if (d2 > defdiff) d2 = defdiff;
  if (d2 < -defdiff) d2 = -defdiff;
  e.nan = !std::isfinite(d1) || !std::isfinite(d2);
  if (e.nan) d1 = d2 = 0.;
  e.d1 = d1;
  e.d2 = d2;
}

/* CalcDerivatives + eCalcCalibratedDerivativesX/3, rbacore.cpp:1420-1673.
 * Bc: 2 x ncols camera block (row major, stride 9) in the camera's own
 * parameter order; Bp: 2 x 3 point block.  ncols = 0 for camera 0 when it
 * has no parameters (begini = 1). */
void LSA::derivs(const ObsEval &e, int k, const float *w, double *Bc, int *ncols,
                 double *Bp) const {
  (void)w;
  const double *R = &Rn[9 * k];
  const double u = e.ex3[0], v = e.ex3[1], xs3 = e.xs3;
  const double x1 = u * xs3, x2 = v * xs3;
  const double k2 = dn[2 * k], k4 = dn[2 * k + 1];
  const double *K = &Kn[9 * k];
  /* distortion Jacobian, eCalcCalibratedDerivativesX */
  const double xy2 = u * u + v * v;
  const double xy4 = xy2 * xy2;
  const double xxpc = k4 * xy4 + u * (2 * k2 * u + 4 * k4 * u * xy2) + k2 * xy2 + 1.;
  const double xypc = u * (4 * k4 * xy2 * v + 2 * k2 * v);
  const double yxpc = (4 * k4 * u * xy2 + 2 * k2 * u) * v;
  const double yypc = v * (2 * k2 * v + 4 * k4 * xy2 * v) + k4 * xy4 + k2 * xy2 + 1.;
  auto calib = [&](double &a0, double &a1) {
    const double xpo = a0, ypo = a1;
    const double xp = xxpc * xpo + xypc * ypo;
    const double yp = yypc * ypo + yxpc * xpo;
    a0 = xp * K[0] + yp * K[1];
    a1 = yp * K[4];
  };
  /* point columns (== PC columns) */
  for (int j = 0; j < 3; ++j) {
    Bp[j] = -R[0 * 3 + j] * xs3 + R[2 * 3 + j] * x1;
    Bp[3 + j] = -R[1 * 3 + j] * xs3 + R[2 * 3 + j] * x2;
    calib(Bp[j], Bp[3 + j]);
  }
  const double xp2 = u * u, yp2 = v * v;
  const double xyp2 = xp2 + yp2;
  const double xyp4 = xyp2 * xyp2;
  double ic0[3], ic1[3];
  int ni = 0;
  if (opt.addf[0]) {
    ic0[ni] = -u * xyp2 * K[0] - v * xyp2 * K[1];
    ic1[ni] = -v * xyp2 * K[4];
    ++ni;
  }
  if (opt.addf[1]) {
    ic0[ni] = -u * xyp4 * K[0] - v * xyp4 * K[1];
    ic1[ni] = -v * xyp4 * K[4];
    ++ni;
  }
  if (opt.addf[2]) {
    ic0[ni] = -e.ex3u[0];
    ic1[ni] = -e.ex3u[1];
    ++ni;
  }
  if (k == 0 && !ao) {
    for (int j = 0; j < ni; ++j) {
      Bc[j] = ic0[j];
      Bc[9 + j] = ic1[j];
    }
    *ncols = ni;
    return;
  }
  const double xs31 = 1. / xs3;
  const double xs32 = xs31 * xs31;
  double r0[3], r1[3];
  r0[0] = x2 * x1 * xs32;
  r1[0] = 1. + x2 * x2 * xs32;
  r0[1] = -1. - x1 * x1 * xs32;
  r1[1] = -x2 * x1 * xs32;
  r0[2] = x2 * xs31;
  r1[2] = -x1 * xs31;
  int n = 0;
  for (int j = 0; j < 3; ++j) {
    Bc[n] = r0[j];
    Bc[9 + n] = r1[j];
    calib(Bc[n], Bc[9 + n]);
    ++n;
  }
  if (k == normcamera) {
    for (int j = 0; j < 2; ++j) {
      const int s = esvm[j];
      Bc[n] = -R[0 * 3 + s] * xs3 + R[2 * 3 + s] * x1;
      Bc[9 + n] = -R[1 * 3 + s] * xs3 + R[2 * 3 + s] * x2;
      calib(Bc[n], Bc[9 + n]);
      ++n;
    }
  } else {
    for (int j = 0; j < 3; ++j) {
      Bc[n] = Bp[j];
      Bc[9 + n] = Bp[3 + j];
      ++n;
    }
  }
  for (int j = 0; j < ni; ++j) {
    Bc[n] = ic0[j];
    Bc[9 + n] = ic1[j];
    ++n;
  }
  *ncols = n;
}

/* CalcCorrections, rbacore.cpp:1201-1414 (no GCPs). */
void LSA::calc_corrections(bool solveflag, double multfact1, const std::vector<double> &XM,
                           bool srmvflag, bool derivflag) {
  sig0 = 0.f;
  int kkk = nrioff - 1;
  int gcpnum = 0;
  for (int i = 0; i < nrpts; ++i) {
    if (derivflag) {
      for (int j = 0; j < 9; ++j) Vp[j] = 0.;
      gp[0] = gp[1] = gp[2] = 0.;
    }
    const int base = nrioff + 3 * i;
    XXnew[3 * i] = XM[base];
    XXnew[3 * i + 1] = XM[base + 1];
    XXnew[3 * i + 2] = XM[base + 2];
    const int t0 = toff[i], t1 = toff[i + 1];
    for (int o = t0; o < t1; ++o) {
      const int k = timg[o];
      ObsEval e;
      eval_obs(k, tslot[o], &XXnew[3 * i], e);
      if (derivflag) {
        const float *w = &W[3 * o];
        double Bc[18], Bp[6];
        int nc = 0;
        derivs(e, k, w, Bc, &nc, Bp);
        const double W0 = w[0], W1 = w[1], W2 = w[2];
        const int ks = o - t0;
        std::vector<double> &wl = Wl[ks];
        if (k >= begini && nc > 0) {
          double Bt[9][2];
          for (int j = 0; j < nc; ++j) {
            const double xp = Bc[j], yp = Bc[9 + j];
            Bt[j][0] = xp * W0 + yp * W2;
            Bt[j][1] = xp * W2 + yp * W1;
          }
          if (!solveflag) {
            std::vector<double> &D = Dg[k];
            std::vector<double> &r = rhs[k];
            for (int a = 0; a < nc; ++a) {
              for (int c = 0; c < nc; ++c) D[a * nc + c] += Bt[a][0] * Bc[c] + Bt[a][1] * Bc[9 + c];
              r[a] += Bt[a][0] * e.d1 + Bt[a][1] * e.d2;
            }
          }
          wl.assign(3 * nc, 0.);
          for (int a = 0; a < nc; ++a)
            for (int c = 0; c < 3; ++c) wl[3 * a + c] = Bt[a][0] * Bp[c] + Bt[a][1] * Bp[3 + c];
        }
        double Bpt[3][2];
        for (int j = 0; j < 3; ++j) {
          const double xp = Bp[j], yp = Bp[3 + j];
          Bpt[j][0] = xp * W0 + yp * W2;
          Bpt[j][1] = xp * W2 + yp * W1;
        }
        for (int a = 0; a < 3; ++a) {
          for (int c = 0; c < 3; ++c) Vp[a * 3 + c] += Bpt[a][0] * Bp[c] + Bpt[a][1] * Bp[3 + c];
          gp[a] += Bpt[a][0] * e.d1 + Bpt[a][1] * e.d2;
        }
      }
      if (e.nan) {
        sig0rmv[o] = 1.e20f;
      } else {
        const float f1 = (float)e.d1, f2 = (float)e.d2;
        const float d11 = f1 * f1, d12 = 2.f * f1 * f2, d22 = f2 * f2;
        const float *w = &W[3 * o];
        const float val = (d11 * w[0] + d12 * w[2] + d22 * w[1]);
        float rval;
        if (opt.robust) {
          const float *wo = &wold[3 * o];
          rval = d11 * wo[0] + d12 * wo[2] + d22 * wo[1];
        } else {
          rval = val;
        }
        if (srmvflag) sig0rmv[o] = rval;
        sig0 += val;
      }
    }
    if (ao && gcpi[i] > -1) {
      /* CalcDerivatives3DGCP, rbacore.cpp:1677-1729: the 3-D prior of a
       * shared point, diff = gcp - X, B = -I */
      const float *w = &W3[6 * gcpnum];
      const double *gx = &gdata[3 * gcpi[i]];
      const double d1 = gx[0] - XXnew[3 * i], d2 = gx[1] - XXnew[3 * i + 1], d3 = gx[2] - XXnew[3 * i + 2];
      sig0ao += (float)(d1 * d1 * w[0] + d2 * d2 * w[1] + d3 * d3 * w[2] +
                        2 * (d1 * d2 * w[3] + d1 * d3 * w[4] + d2 * d3 * w[5]));
      if (derivflag) {
        const double Wm[9] = {w[0], w[3], w[4], w[3], w[1], w[5], w[4], w[5], w[2]};
        for (int r = 0; r < 3; ++r)
          for (int c = 0; c < 3; ++c) Vp[r * 3 + c] += Wm[r * 3 + c];
        for (int r = 0; r < 3; ++r) gp[r] += (-Wm[r * 3]) * d1 + (-Wm[r * 3 + 1]) * d2 + (-Wm[r * 3 + 2]) * d3;
      }
      ++gcpnum;
    }
    if (derivflag) {
      for (int j = 0; j < 3; ++j) Vp[j * 3 + j] *= multfact1;
      inv3(Vp, Vpi);
    }
    if (!solveflag && derivflag) {
      for (int s = t0; s < t1; ++s) {
        const int ij = timg[s];
        if (ij < begini) continue;
        const int ns = cam_np(ij);
        const std::vector<double> &Ws = Wl[s - t0];
        /* eNlijN = W_s * V^-1 (ns x 3) */
        double N[9][3];
        for (int a = 0; a < ns; ++a)
          for (int c = 0; c < 3; ++c)
            N[a][c] = Ws[3 * a] * Vpi[c] + Ws[3 * a + 1] * Vpi[3 + c] + Ws[3 * a + 2] * Vpi[6 + c];
        std::vector<double> &D = Dg[ij];
        for (int a = 0; a < ns; ++a) {
          for (int c = 0; c < ns; ++c)
            D[a * ns + c] -= N[a][0] * Ws[3 * c] + N[a][1] * Ws[3 * c + 1] + N[a][2] * Ws[3 * c + 2];
          rhs[ij][a] -= N[a][0] * gp[0] + N[a][1] * gp[1] + N[a][2] * gp[2];
        }
        for (int t = s + 1; t < t1; ++t) {
          const int ii = timg[t];
          if (ii < begini) continue;
          const int nt = cam_np(ii);
          const std::vector<double> &Wt = Wl[t - t0];
          if (ij < ii) {
            /* block (row ij, col ii) -= N * W_t^T */
            std::vector<double> &B = Off[ii][ij];
            if (B.empty()) B.assign(ns * nt, 0.);
            for (int a = 0; a < ns; ++a)
              for (int c = 0; c < nt; ++c)
                B[a * nt + c] -= N[a][0] * Wt[3 * c] + N[a][1] * Wt[3 * c + 1] + N[a][2] * Wt[3 * c + 2];
          } else if (ii < ij) {
            /* block (row ii, col ij) -= W_t * N^T */
            std::vector<double> &B = Off[ij][ii];
            if (B.empty()) B.assign(nt * ns, 0.);
            for (int a = 0; a < nt; ++a)
              for (int c = 0; c < ns; ++c)
                B[a * ns + c] -= Wt[3 * a] * N[c][0] + Wt[3 * a + 1] * N[c][1] + Wt[3 * a + 2] * N[c][2];
          } else {
            /* same image twice in one track: the reference adds W_t N^T to
             * the diagonal block (rbacore.cpp:1379-1388 with ii == ij) */
            std::vector<double> &Dd = Dg[ij];
            for (int a = 0; a < nt; ++a)
              for (int c = 0; c < ns; ++c)
                Dd[a * ns + c] -= Wt[3 * a] * N[c][0] + Wt[3 * a + 1] * N[c][1] + Wt[3 * a + 2] * N[c][2];
          }
        }
      }
    }
    if (solveflag) {
      double ex[3];
      for (int a = 0; a < 3; ++a) ex[a] = Vpi[a * 3] * gp[0] + Vpi[a * 3 + 1] * gp[1] + Vpi[a * 3 + 2] * gp[2];
      for (int s = t0; s < t1; ++s) {
        const int j = timg[s];
        if (j < begini) continue;
        const int ns = cam_np(j);
        const std::vector<double> &Ws = Wl[s - t0];
        /* (V^-1 * W_s^T) * dc_j */
        double tv[3] = {0., 0., 0.};
        for (int c = 0; c < 3; ++c) {
          double acc = 0.;
          for (int a = 0; a < ns; ++a) acc += Ws[3 * a + c] * rhs[j][a];
          tv[c] = acc;
        }
        for (int a = 0; a < 3; ++a) ex[a] -= Vpi[a * 3] * tv[0] + Vpi[a * 3 + 1] * tv[1] + Vpi[a * 3 + 2] * tv[2];
      }
      x[++kkk] = ex[0];
      x[++kkk] = ex[1];
      x[++kkk] = ex[2];
    }
  }
}

/* SparsePCG, rbacore.cpp:1807-1914, with eAAdv/evvdv (2048-2084).
 * On entry rhs holds exiv (the right-hand side); on exit the best
 * iterate. */
void LSA::sparse_pcg() {
  const int nb = nimg;
  std::vector<int> off(nb + 1, 0);
  for (int i = 0; i < nb; ++i) off[i + 1] = off[i] + (i >= begini ? cam_np(i) : 0);
  const int n = off[nb];
  std::vector<double> r(n), r1(n), d(n), Ad(n), h(n), h1(n), hd(n), xk(n, 0.), xbest(n, 0.);
  /* exivold starts as the right-hand side (rbacore.cpp:1834) */
  std::vector<std::vector<double>> C(nb);
  for (int i = begini; i < nb; ++i) {
    const int ni = cam_np(i);
    for (int a = 0; a < ni; ++a) r[off[i] + a] = xbest[off[i] + a] = rhs[i][a];
  }
  int msize = 0;
  for (int i = begini; i < nb; ++i) {
    const int ni = cam_np(i);
    C[i].assign(ni * ni, 0.);
    lu_inverse(ni, Dg[i].data(), C[i].data());
    msize += ni;
    for (int a = 0; a < ni; ++a) {
      double s = 0.;
      for (int c = 0; c < ni; ++c) s += C[i][a * ni + c] * r[off[i] + c];
      h[off[i] + a] = s;
    }
  }
  d = h;
  if (msize < 1000) msize = 1000;
  auto spmv = [&](const std::vector<double> &bv, std::vector<double> &cv) {
    for (int i = begini; i < nb; ++i)
      for (int a = 0; a < cam_np(i); ++a) cv[off[i] + a] = 0.;
    for (int i = begini; i < nb; ++i) {
      const int ni = cam_np(i);
      /* j = 0: diagonal */
      for (int a = 0; a < ni; ++a) {
        double s = 0.;
        for (int c = 0; c < ni; ++c) s += Dg[i][a * ni + c] * bv[off[i] + c];
        cv[off[i] + a] += s;
      }
      std::vector<const std::pair<const int, std::vector<double>> *> order;
      for (auto &kv : Off[i]) order.push_back(&kv);
      if (g_order_variant == 1) std::reverse(order.begin(), order.end());
      if (g_order_variant == 2) std::rotate(order.begin(), order.begin() + order.size() / 2, order.end());
      if (g_order_variant >= 3 && g_order_variant < 20) {
        std::mt19937 g((unsigned)g_order_variant * 7919u + (unsigned)i);
        std::shuffle(order.begin(), order.end(), g);
      }
      for (auto *kvp : order) {
        const auto &kv = *kvp;
        const int row = kv.first, nr = cam_np(row);
        const std::vector<double> &B = kv.second; /* nr x ni */
        for (int a = 0; a < nr; ++a) {
          double s = 0.;
          for (int c = 0; c < ni; ++c) s += B[a * ni + c] * bv[off[i] + c];
          cv[off[row] + a] += s;
        }
        for (int c = 0; c < ni; ++c) {
          double s = 0.;
          for (int a = 0; a < nr; ++a) s += B[a * ni + c] * bv[off[row] + a];
          cv[off[i] + c] += s;
        }
      }
    }
  };
  /* variants >= 20: the PCG's sums over cameras are blocked, per group of
   * (variant - 18) cameras, then the groups summed (a parallel reduction's
   * order) */
  const int dot_group = (g_order_variant >= 20 && g_order_variant < 40) ? g_order_variant - 18 : 0;
  /* variants >= 40: per-camera partials summed as a pairwise tree whose
   * leaves are groups of (variant - 39) cameras (a tree reduction's order) */
  const int tree_leaf = g_order_variant >= 40 ? g_order_variant - 39 : 0;
  std::function<double(const std::vector<double> &, int, int)> tree_sum =
      [&](const std::vector<double> &v, int lo, int hi) -> double {
    if (hi - lo <= tree_leaf) {
      double c = 0.;
      for (int i = lo; i < hi; ++i) c += v[i];
      return c;
    }
    const int mid = lo + (hi - lo) / 2;
    return tree_sum(v, lo, mid) + tree_sum(v, mid, hi);
  };
  std::vector<double> part_cam(nb > 0 ? nb : 1);
  auto dot = [&](const std::vector<double> &a, const std::vector<double> &bb) {
    double c = 0., g = 0.;
    if (tree_leaf) {
      for (int i = begini; i < nb; ++i) {
        double cc = 0.;
        for (int j = off[i]; j < off[i + 1]; ++j) cc += bb[j] * a[j];
        part_cam[i] = cc;
      }
      return tree_sum(part_cam, begini, nb);
    }
    for (int i = begini; i < nb; ++i) {
      double cc = 0.;
      for (int j = off[i]; j < off[i + 1]; ++j) cc += bb[j] * a[j];
      if (dot_group) {
        g += cc;
        if ((i - begini + 1) % dot_group == 0 || i + 1 == nb) {
          c += g;
          g = 0.;
        }
      } else {
        c += cc;
      }
    }
    return c;
  };
  double meandrold = 1.e50, meandr0 = 1.e50;
  int k;
  for (k = 0; k < msize; ++k) {
    spmv(d, Ad);
    const double erthk = dot(r, h);
    const double edtAdk = dot(d, Ad);
    double alpha;
    if (std::fabs(erthk) < 1.e-20 || std::fabs(erthk) > 1.e20)
      alpha = 0.;
    else
      alpha = erthk / edtAdk;
    double meandr = 0., mg = 0.;
    for (int i = begini; i < nb; ++i) {
      const int ni = cam_np(i);
      double mi = 0.;
      for (int j = off[i]; j < off[i + 1]; ++j) {
        xk[j] += alpha * d[j];
        const double dr = alpha * Ad[j];
        r1[j] = r[j] - dr;
        if (dot_group || tree_leaf)
          mi += dr * dr;
        else
          meandr += dr * dr;
      }
      if (tree_leaf) part_cam[i] = mi;
      if (dot_group) {
        mg += mi;
        if ((i - begini + 1) % dot_group == 0 || i + 1 == nb) {
          meandr += mg;
          mg = 0.;
        }
      }
      for (int a = 0; a < ni; ++a) {
        double s = 0.;
        for (int c = 0; c < ni; ++c) s += C[i][a * ni + c] * r1[off[i] + c];
        h1[off[i] + a] = s;
      }
    }
    if (tree_leaf) meandr = tree_sum(part_cam, begini, nb);
    if (k == 0) meandr0 = meandr;
    if (meandr < meandrold) {
      xbest = xk;
      meandrold = meandr;
    }
    if (meandr * 1.e5 < meandr0) break;
    for (int j = 0; j < n; ++j) hd[j] = h1[j] - h[j];
    const double er1th1 = dot(r1, hd);
    const double erth = dot(r, h);
    double beta = std::fabs(er1th1) < 1.e-10 ? 0. : er1th1 / erth;
    if (beta < 0.) beta = 0.;
    for (int j = 0; j < n; ++j) d[j] = h1[j] + beta * d[j];
    r = r1;
    h = h1;
  }
  pcg_iters += std::min(k + 1, msize);
  for (int i = begini; i < nb; ++i)
    for (int a = 0; a < cam_np(i); ++a) rhs[i][a] = xbest[off[i] + a];
}

/* Dense Cholesky of the reduced camera system (the --direct oracle mode
 * the GPU's direct form is compared with): the textbook row-by-row
 * Cholesky-Crout factorisation L L^T of the symmetrised matrix, then the
 * forward and back substitutions, every sum taken in increasing index order.
 * The matrix is held in its envelope (row r from the first column any of its
 * camera's blocks reaches): L has the same envelope, every entry left of it
 * is an exact zero, and the terms the dense loops would add for those
 * columns are exact zeros, so skipping them changes no value -- the result
 * is that of the dense loops at a fraction of the work on chain- and
 * grid-like scenes. */
void LSA::direct_solve() {
  const int nb = nimg;
  std::vector<int> off(nb + 1, 0);
  for (int i = 0; i < nb; ++i) off[i + 1] = off[i] + (i >= begini ? cam_np(i) : 0);
  const int n = off[nb];
  /* first column of every scalar row, and the row starts of the envelope */
  std::vector<int> fc(n);
  for (int i = begini; i < nb; ++i) {
    int f = off[i];
    for (auto &kv : Off[i]) f = std::min(f, off[kv.first]);
    for (int a = 0; a < cam_np(i); ++a) fc[off[i] + a] = f;
  }
  std::vector<size_t> rs(n + 1, 0);
  for (int r = 0; r < n; ++r) rs[r + 1] = rs[r] + (size_t)(r - fc[r] + 1);
  std::vector<double> L(rs[n], 0.), y(n);
  auto at = [&](int r, int c) -> double & { return L[rs[r] + (size_t)(c - fc[r])]; };
  for (int i = begini; i < nb; ++i) {
    const int ni = cam_np(i);
    /* symmetrised diagonal block (the assembled blocks are symmetric to
     * roundoff); the off-diagonal blocks enter both triangles with the same
     * value, whose symmetrised mean is itself */
    for (int a = 0; a < ni; ++a)
      for (int c = 0; c <= a; ++c)
        at(off[i] + a, off[i] + c) = c == a ? Dg[i][a * ni + a] : 0.5 * (Dg[i][a * ni + c] + Dg[i][c * ni + a]);
    for (auto &kv : Off[i]) {
      const int row = kv.first, nr = cam_np(row);
      for (int a = 0; a < nr; ++a)
        for (int c = 0; c < ni; ++c) {
          const double v = kv.second[a * ni + c];
          at(off[i] + c, off[row] + a) = 0.5 * (v + v);
        }
    }
    for (int a = 0; a < ni; ++a) y[off[i] + a] = rhs[i][a];
  }
  for (int j = 0; j < n; ++j) {
    double s = at(j, j);
    for (int k = fc[j]; k < j; ++k) s -= at(j, k) * at(j, k);
    if (!(s > 0.)) {
      status = RPBA_ERR_SOLVER;
      return;
    }
    const double l = std::sqrt(s);
    at(j, j) = l;
    for (int i = j + 1; i < n; ++i) {
      if (fc[i] > j) continue;  /* L(i, j) stays an exact zero */
      double t = at(i, j);
      for (int k = std::max(fc[i], fc[j]); k < j; ++k) t -= at(i, k) * at(j, k);
      at(i, j) = t / l;
    }
  }
  for (int i = 0; i < n; ++i) {
    double s = y[i];
    for (int k = fc[i]; k < i; ++k) s -= at(i, k) * y[k];
    y[i] = s / at(i, i);
  }
  for (int i = n - 1; i >= 0; --i) {
    double s = y[i];
    for (int k = i + 1; k < n; ++k)
      if (fc[k] <= i) s -= at(k, i) * y[k];
    y[i] = s / at(i, i);
  }
  for (int i = begini; i < nb; ++i)
    for (int a = 0; a < cam_np(i); ++a) rhs[i][a] = y[off[i] + a];
}

/* CalcBundleSep, rbacore.cpp:1094-1195. */
bool LSA::calc_bundle_sep(double multfact) {
  begini = (ao || nadd > 0) ? 0 : 1;
  sig0ao = 0.f;
  const double multfact1 = 1. + multfact;
  if (iniflag) {
    Dg.assign(nimg, {});
    rhs.assign(nimg, {});
    Off.assign(nimg, {});
  }
  for (int i = begini; i < nimg; ++i) {
    const int ni = cam_np(i);
    Dg[i].assign(ni * ni, 0.);
    rhs[i].assign(ni, 0.);
    for (auto &kv : Off[i]) std::fill(kv.second.begin(), kv.second.end(), 0.);
  }
  int maxt = 0;
  for (int p = 0; p < nrpts; ++p) maxt = std::max(maxt, toff[p + 1] - toff[p]);
  Wl.assign(maxt, {});
  calc_corrections(false, multfact1, XPM, false, true);
  for (int i = begini; i < nimg; ++i) {
    const int ni = cam_np(i);
    for (int j = 0; j < ni; ++j) Dg[i][j * ni + j] *= multfact1;
    for (int j = 0; j < ni; ++j) Dg[i][j * ni + j] += 1.e-2;
  }
  if (opt.solver == RPBA_SOLVER_DIRECT)
    direct_solve();
  else
    sparse_pcg();
  if (status != RPBA_OK) return true;
  for (int j = begini; j < nimg; ++j)
    for (int k = camparv[j]; k < camparv[j + 1]; ++k) x[k] = (float)rhs[j][k - camparv[j]];
  calc_corrections(true, multfact1, XPM, false, true);
  iniflag = false;
  return false;
}

/* Adjust, rbacore.cpp:333-616 (itbreakflag false, no GCPs). */
int LSA::adjust(rpba_report *rep) {
  if (bad_setup) return RPBA_ERR_ARG;
  int itt = 0;
  iniflag = true;
  bool ittflag = true;
  float sig0frac = 1.05f;
  if (lflflag) sig0frac = 1.01f;
  double multfact = 1.e-3;
  int solves = 0;
  bool cap_hit = false;
  for (int it = 0; it < 2; ++it) {
    if (cap_hit) break;
    sig0old = 1.e20f;
    if (it > 0) {
      iniflag = true;
      multfact = 1.e-6;
    }
    imagepointnr = toff[nrpts];
    nrobs = 2 * imagepointnr;
    std::vector<int> cnt(nimg, 0);
    for (int o = 0; o < imagepointnr; ++o) ++cnt[timg[o]];
    for (int i = 0; i < nimg; ++i)
      if (cnt[i] == 0) {
        if (nimg > 3) *os += "BA-Error: No observations in image " + std::to_string(i) + " (image index)\n";
        return RPBA_ERR_NO_OBS_IMAGE;
      }
    if (ittflag) {
      isflag.assign(imagepointnr, 0);
      isflagnew.assign(imagepointnr, 0);
      prepare_weights(it);
      ittflag = false;
    }
    wsum = (float)(2 * imagepointnr) / wsum;
    wsumg = wsum;
    for (int i = 0; i < nrpts; ++i)
      for (int j = 0; j < 3; ++j) XPM[nrioff + i * 3 + j] = XX[3 * i + j];
    encode_cameras();
    nrunknowns = nrioff3 + nadd * nimg;
    XXnew = XX;
    x.resize(nrunknowns, 0.);
    redundancy = nrobs - nrunknowns;
    if (redundancy < 0) {
      if (nimg > 3) *os += "BA-Error: Low redundancy\n";
      return RPBA_ERR_LOW_REDUNDANCY;
    }
    if (it == 0) {
      sig0rmv.assign(imagepointnr, 0.f);
      decode_cameras(XPM);
      calc_corrections(false, 1. + multfact, XPM, true, false);
      sig0 = sig0 * wsumg / (float)redundancy;
      sig0in = sig0old = sig0;
    } else {
      sig0in = sig0old;
    }
    int iflag = opt.robust ? 2 : 1;
    int iter = 1;
    const int nunk_given = nrunknowns, nobs_given = nrobs;
    while (iflag > 0) {
      if (it == 0 && opt.robust) {
        nrunknowns = nunk_given;
        nrobs = nobs_given;
        reweight(iflag);
        redundancy = nrobs - nrunknowns;
        wsum = (float)(2 * imagepointnr) / wsum;
        wsumg = wsum;
      }
      if (calc_bundle_sep(multfact)) return status;
      ++solves;
      for (int i = 0; i < nrunknowns; ++i) {
        if (!std::isfinite(x[i])) return RPBA_ERR_NAN_STEP;
        XPMn[i] = XPM[i] - x[i];
      }
      decode_cameras(XPMn);
      calc_corrections(false, 1. + multfact, XPMn, true, false);
      sig0 = sig0 * wsumg / (float)redundancy;
      if (sig0old < sig0 * sig0frac) --iflag;
      if (sig0 <= sig0old || iter == 1) {
        store_results();
        sig0old = sig0;
      }
      if (itt > 200) break;
      ++itt;
      ++iter;
      if (opt.max_lm >= 0 && solves >= opt.max_lm) {
        cap_hit = true;
        break;
      }
    }
    const float s_in = std::sqrt(sig0in * ihw2), s_out = std::sqrt(sig0old * ihw2);
    *os += "Sigma0: " + fmt_g(s_in) + ' ' + fmt_g(s_out) + "  ";
    int red, nob, nun;
    if (it == 0 && opt.robust) {
      red = redundancynew;
      nob = nrobsnew;
      nun = nrunknownsnew;
    } else {
      red = redundancy;
      nob = nrobs;
      nun = nrunknowns;
    }
    *os += std::to_string(red) + ' ' + std::to_string(nob) + ' ' + std::to_string(nun) + "  IT: " +
           std::to_string(it) + "  ITT: " + std::to_string(itt) + '\n';
    if (rep) {
      rep->sigma0_in[it] = s_in;
      rep->sigma0_out[it] = s_out;
      rep->redundancy[it] = red;
      rep->nrobs[it] = nob;
      rep->nrunknowns[it] = nun;
      rep->itt[it] = itt;
      rep->passes_done = it + 1;
    }
    if (opt.robust && it == 0) {
      const int before_obs = toff[nrpts], before_pts = nrpts;
      robust_delete();
      if (rep) {
        rep->obs_deleted += before_obs - toff[nrpts];
        rep->points_deleted += before_pts - nrpts;
      }
    }
    ittflag = true;
  }
  if (rep) {
    rep->linear_solves = solves;
    rep->pcg_iterations = pcg_iters;
  }
  return RPBA_OK;
}

/* Adjust(robust = false, itbreakflag = true, itmaxnum = 0, W3, gcp = true,
 * gcpdata), rbacore.cpp:333-616, the per-partition call of the parallel
 * RPBA (rpbacore.cpp:229): the GCP weights PrepareWeights3D sums
 * (rbacore.cpp:787-818), the cost with the priors, one damped step
 * (multfact 1e-4) stored unconditionally (iter == 1), the Sigma0 and
 * Sigma0AO lines.  As in the reference, sig0ao is reset only where
 * CalcBundleSep and the first cost evaluation reset it, so the printed
 * post-step value accumulates the three evaluations since the reset. */
int LSA::adjust_gcp_step() {
  if (bad_setup) return RPBA_ERR_ARG;
  iniflag = true;
  const double multfact = 1.e-4;
  sig0aoi = sig0aoiold = 1.e20f;
  float sig0aoin = 1.e20f;
  imagepointnr = toff[nrpts];
  nrobs = 2 * imagepointnr;
  nrobsao = 3 * nrgcp;
  nrobs += nrobsao;
  std::vector<int> cnt(nimg, 0);
  for (int o = 0; o < imagepointnr; ++o) ++cnt[timg[o]];
  for (int i = 0; i < nimg; ++i)
    if (cnt[i] == 0) {
      if (nimg > 3) *os += "BA-Error: No observations in image " + std::to_string(i) + " (image index)\n";
      return RPBA_ERR_NO_OBS_IMAGE;
    }
  isflag.assign(imagepointnr, 0);
  isflagnew.assign(imagepointnr, 0);
  prepare_weights(0);
  wsumao = 0.f;
  for (int i = 0; i < nrgcp; ++i) wsumao += W3[6 * i] + W3[6 * i + 1] + W3[6 * i + 2];
  wsumg = (float)(2 * imagepointnr + nrobsao) / (wsumao + wsum);
  wsumao = (float)nrobsao / wsumao;
  wsum = (float)(2 * imagepointnr) / wsum;
  for (int i = 0; i < nrpts; ++i)
    for (int j = 0; j < 3; ++j) XPM[nrioff + i * 3 + j] = XX[3 * i + j];
  encode_cameras();
  nrunknowns = nrioff3 + nadd * ncam_total;
  XXnew = XX;
  x.assign(nrunknowns, 0.);
  redundancy = nrobs - nrunknowns;
  if (redundancy < 0) {
    if (nimg > 3) *os += "BA-Error: Low redundancy\n";
    return RPBA_ERR_LOW_REDUNDANCY;
  }
  sig0rmv.assign(imagepointnr, 0.f);
  decode_cameras(XPM);
  sig0ao = 0.f;
  calc_corrections(false, 1. + multfact, XPM, true, false);
  sig0aoi = sig0 * wsumg / (float)redundancy;
  sig0aoin = sig0aoi;
  sig0 = (sig0 + sig0ao) * wsumg / (float)(redundancy + nrobsao - 7);
  sig0in = sig0old = sig0;
  if (calc_bundle_sep(multfact)) return status;
  for (int i = 0; i < nrunknowns; ++i) {
    if (!std::isfinite(x[i])) return RPBA_ERR_NAN_STEP;
    XPMn[i] = XPM[i] - x[i];
  }
  decode_cameras(XPMn);
  calc_corrections(false, 1. + multfact, XPMn, true, false);
  sig0aoi = sig0 * wsumg / (float)redundancy;
  sig0 = (sig0 + sig0ao) * wsumg / (float)(redundancy + nrobsao - 7);
  store_results();
  sig0old = sig0;
  sig0aoiold = sig0aoi;
  const float s_in = std::sqrt(sig0in * ihw2), s_out = std::sqrt(sig0old * ihw2);
  *os += "Sigma0: " + fmt_g(std::sqrt(sig0aoin * ihw2)) + ' ' + fmt_g(std::sqrt(sig0aoiold * ihw2)) + "  " +
         std::to_string(redundancy) + ' ' + std::to_string(nrobs) + ' ' + std::to_string(nrunknowns) +
         "  IT: 0  ITT: 0\n";
  *os += "Sigma0AO: " + fmt_g(std::sqrt(sig0ao * wsumao / (float)(nrobsao - 7))) + "  " + fmt_g(s_in) + ' ' +
         fmt_g(s_out) + "  " + std::to_string(nrobsao) + " " + fmt_g(wsumao) + '\n';
  return RPBA_OK;
}

void LSA::output(rpba_block *blk) {
  /* PointXXvOut: tracks of kept points, empty lists for the others */
  std::vector<int32_t> noff(XXnr + 1, 0), nimgv, nslot;
  int j = 0;
  for (int i = 0; i < XXnr; ++i) {
    if (j < nrpts && nrpv[j] == i) {
      for (int o = toff[j]; o < toff[j + 1]; ++o) {
        nimgv.push_back(timg[o]);
        nslot.push_back(tslot[o]);
      }
      for (int c = 0; c < 3; ++c) blk->XX[3 * i + c] = (float)XX[3 * j + c];
      ++j;
    }
    noff[i + 1] = (int32_t)nimgv.size();
  }
  std::memcpy(blk->pt_obs_off, noff.data(), sizeof(int32_t) * (XXnr + 1));
  if (!nimgv.empty()) {
    std::memcpy(blk->pt_obs_image, nimgv.data(), sizeof(int32_t) * nimgv.size());
    std::memcpy(blk->pt_obs_slot, nslot.data(), sizeof(int32_t) * nslot.size());
  }
  for (int i = 0; i < 12 * nimg; ++i) blk->pmat[i] = (float)P[i];
  /* cameraso from camerasnew (rbacore.cpp:658-663) */
  for (int i = 0; i < nimg; ++i) {
    for (int c = 0; c < 9; ++c) blk->K[9 * i + c] = (float)Kn[9 * i + c];
    blk->distpara[2 * i] = (float)dn[2 * i];
    blk->distpara[2 * i + 1] = (float)dn[2 * i + 1];
  }
}

/* FP64 cost and RMS of the accepted state, evaluated with the Exteval
 * projection (P * X, distortion, f) -- the shared final-state evaluator. */
double LSA::final_cost(double *rms) {
  double cost = 0., sq = 0.;
  const int n = toff[nrpts];
  for (int p = 0; p < nrpts; ++p) {
    const double X0 = XX[3 * p], X1 = XX[3 * p + 1], X2 = XX[3 * p + 2];
    for (int o = toff[p]; o < toff[p + 1]; ++o) {
      const int k = timg[o];
      const double *M = &P[12 * k];
      double p1 = M[0] * X0 + M[1] * X1 + M[2] * X2 + M[3];
      double p2 = M[4] * X0 + M[5] * X1 + M[6] * X2 + M[7];
      double p3 = M[8] * X0 + M[9] * X1 + M[10] * X2 + M[11];
      if (std::fabs(p3) < 1.e-3)
        p3 = p3 > 0. ? 1.e3 : -1.e3;
      else
        p3 = 1. / p3;
      p1 *= p3;
      p2 *= p3;
      const double dist = p1 * p1 + p2 * p2;
      const double z = 1. + (dc[2 * k] * dist + dc[2 * k + 1] * dist * dist);
      p1 *= z;
      p2 *= z;
      p1 *= Kc[9 * k];
      p2 *= Kc[9 * k];
      const int sl = b->img_obs_off[k] + tslot[o];
      const double dx = (double)b->xg[2 * sl] - p1, dy = (double)b->xg[2 * sl + 1] - p2;
      const double w0 = b->wx[sl], w1 = b->wy[sl], w2 = b->wxy[sl];
      cost += dx * dx * w0 + dy * dy * w1 + 2. * dx * dy * w2;
      sq += dx * dx + dy * dy;
    }
  }
  if (rms) *rms = n > 0 ? std::sqrt(sq / n) : 0.;
  return cost;
}

void LSA::setup_pass_for_tests() {
  imagepointnr = toff[nrpts];
  isflag.assign(imagepointnr, 0);
  isflagnew.assign(imagepointnr, 0);
  prepare_weights(0);
  for (int i = 0; i < nrpts; ++i)
    for (int j = 0; j < 3; ++j) XPM[nrioff + i * 3 + j] = XX[3 * i + j];
  encode_cameras();
  sig0rmv.assign(imagepointnr, 0.f);
  decode_cameras(XPM);
}

void LSA::residuals_at(const std::vector<double> &XM, std::vector<double> &res) {
  decode_cameras(XM);
  res.clear();
  for (int i = 0; i < nrpts; ++i) {
    const double X[3] = {XM[nrioff + 3 * i], XM[nrioff + 3 * i + 1], XM[nrioff + 3 * i + 2]};
    for (int o = toff[i]; o < toff[i + 1]; ++o) {
      ObsEval e;
      eval_obs(timg[o], tslot[o], X, e);
      res.push_back(e.d1);
      res.push_back(e.d2);
    }
  }
}

void LSA::jacobian_of(int tobs, double *Bc, int *ncols, int *coff, double *Bp) {
  int p = (int)(std::upper_bound(toff.begin(), toff.end(), tobs) - toff.begin()) - 1;
  const double X[3] = {XPM[nrioff + 3 * p], XPM[nrioff + 3 * p + 1], XPM[nrioff + 3 * p + 2]};
  ObsEval e;
  eval_obs(timg[tobs], tslot[tobs], X, e);
  derivs(e, timg[tobs], &W[3 * tobs], Bc, ncols, Bp);
  *coff = camparv[timg[tobs]];
}

/* ------------------------------------------------------------ EvalLSA */

/* EvalLSA + CalcCorrPointMulti, rpbacore.cpp:778-837, 882-941. */
void eval_lsa(const rpba_block *b, int nraddp, double *resid, rpba_report *rep, std::string *os) {
  const int nimg = b->n_images;
  float ihw2 = 0.f;
  for (int i = 0; i < nimg; ++i) ihw2 += (float)((1 + 1) * (1 + 1)) * 0.25f;
  ihw2 /= (float)nimg;
  long redundancy = 0, nrobs = 0;
  float sig0g = 0.f;
  for (int ii = 0; ii < b->n_points; ++ii) {
    const int s = b->pt_obs_off[ii], e = b->pt_obs_off[ii + 1];
    const int pxss = e - s, pxss2 = 2 * pxss;
    if (resid)
      for (int j = s; j < e; ++j) resid[2 * j] = resid[2 * j + 1] = 0.;
    if (pxss <= 1) continue;
    float wsum = 0.f;
    for (int j = s; j < e; ++j) {
      const int sl = b->img_obs_off[b->pt_obs_image[j]] + b->pt_obs_slot[j];
      wsum += b->wx[sl] + b->wy[sl];
    }
    wsum = wsum / (float)pxss2;
    const double X0 = b->XX[3 * ii], X1 = b->XX[3 * ii + 1], X2 = b->XX[3 * ii + 2];
    float sig0 = 0.f;
    for (int j = s; j < e; ++j) {
      const int im = b->pt_obs_image[j];
      const int sl = b->img_obs_off[im] + b->pt_obs_slot[j];
      const float *Pf = &b->pmat[12 * im];
      double M[12];
      for (int q = 0; q < 12; ++q) M[q] = (double)Pf[q];
      double p1 = M[0] * X0 + M[1] * X1 + M[2] * X2 + M[3];
      double p2 = M[4] * X0 + M[5] * X1 + M[6] * X2 + M[7];
      double p3 = M[8] * X0 + M[9] * X1 + M[10] * X2 + M[11];
      if (std::fabs(p3) < 1.e-3)
        p3 = p3 > 0. ? 1.e3 : -1.e3;
      else
        p3 = 1. / p3;
      p1 *= p3;
      p2 *= p3;
      const double dist = p1 * p1 + p2 * p2;
      const double z = 1. + (double)(b->distpara[2 * im] * dist + b->distpara[2 * im + 1] * dist * dist);
      p1 *= z;
      p2 *= z;
      p1 *= b->K[9 * im];
      p2 *= b->K[9 * im];
      const double dx = b->xg[2 * sl] - p1, dy = b->xg[2 * sl + 1] - p2;
      if (resid) {
        resid[2 * j] = dx;
        resid[2 * j + 1] = dy;
      }
      const float s0 = (float)(dx * dx * b->wx[sl] + dy * dy * b->wy[sl] + 2 * dx * dy * b->wxy[sl]);
      sig0 += s0;
    }
    sig0g += sig0 / wsum;
    redundancy += pxss2 - 3;
    nrobs += pxss2;
  }
  const long red = redundancy - (nimg - 2) * 6 - 5 - nimg * nraddp;
  sig0g *= 1.f / (float)red;
  const float v = std::sqrt(sig0g * ihw2);
  if (os) *os += "ITTTT: " + fmt_g(v) + ' ' + std::to_string(nrobs) + " " + std::to_string(red) + '\n';
  if (rep) {
    rep->exteval_sigma0 = v;
    rep->exteval_nrobs = nrobs;
    rep->exteval_redundancy = red;
  }
}

Opts make_opts(const rpba_options *o) {
  Opts r;
  r.robust = o->robust != 0;
  r.addf[0] = o->k2 != 0;
  r.addf[1] = o->k4 != 0;
  r.addf[2] = o->f != 0;
  r.solver = o->solver;
  r.max_lm = o->max_lm_iterations;
  return r;
}

void copy_log(const std::string &s, char *log, size_t cap) {
  if (!log || cap == 0) return;
  const size_t n = std::min(cap - 1, s.size());
  std::memcpy(log, s.data(), n);
  log[n] = 0;
}

} // namespace

/* ------------------------------------------- per-point triangulation
 * CalcLSAXMulti (rpbacore.cpp:536-773) with CalcCorrPointMulti (:778-837)
 * and CalcCalibratedDerivatives (:841-877): robust Gauss-Newton of one
 * point against fixed cameras.  With a camera partition (part, nparts) the
 * per-partition weight blocks (wxyflag, rpbacore.cpp:579-590, 612-622,
 * 663-672) are formed too: for every partition i that sees the point, the
 * normal matrix (B^T W B, undamped) of the point's observations in the
 * other partitions (one partition: all of them), from the iteration last
 * accepted, as floats; zero for partitions that do not see the point and
 * for points without an accepted iteration. */
namespace {

struct TriObs {
  int im, sl;
};

// residuals and projections of one point (CalcCorrPointMulti)
void tri_corr(const rpba_block *b, const double *Pd, const std::vector<TriObs> &ob, double X0, double X1, double X2,
              const std::vector<float> &wx, const std::vector<float> &wy, const std::vector<float> &wxy,
              const std::vector<float> &wxo, const std::vector<float> &wyo, const std::vector<float> &wxyo,
              std::vector<double> &corr, float &sig0, std::vector<float> &sig0v, std::vector<float> &p1v,
              std::vector<float> &p2v, std::vector<float> &p3v) {
  sig0 = 0.f;
  for (size_t js = 0; js < ob.size(); ++js) {
    const int j = ob[js].im;
    const double *P = &Pd[12 * j];
    double p1 = P[0] * X0 + P[1] * X1 + P[2] * X2 + P[3];
    double p2 = P[4] * X0 + P[5] * X1 + P[6] * X2 + P[7];
    double p3 = P[8] * X0 + P[9] * X1 + P[10] * X2 + P[11];
    if (std::fabs(p3) < 1.e-3)
      p3 = p3 > 0. ? 1.e3 : -1.e3;
    else
      p3 = 1. / p3;
    p1 *= p3;
    p2 *= p3;
    p1v[js] = (float)p1;
    p2v[js] = (float)p2;
    p3v[js] = (float)p3;
    const double dist = p1 * p1 + p2 * p2;
    const double z = 1. + (double)(b->distpara[2 * j] * dist + b->distpara[2 * j + 1] * dist * dist);
    p1 *= z;
    p2 *= z;
    p1 *= b->K[9 * j];
    p2 *= b->K[9 * j];
    const double dx = b->xg[2 * ob[js].sl] - p1, dy = b->xg[2 * ob[js].sl + 1] - p2;
    corr[2 * js] = dx;
    corr[2 * js + 1] = dy;
    sig0 += (float)(dx * dx * wx[js] + dy * dy * wy[js] + 2 * dx * dy * wxy[js]);
    sig0v[js] = (float)(dx * dx * wxo[js] + dy * dy * wyo[js] + 2 * dx * dy * wxyo[js]);
  }
}

// d(projection)/dX chained through the distortion and the calibration
void tri_calibrated(double *xp, double *yp, double x, double y, double k2, double k4, double fx, double fy,
                    double sk) {
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

}  // namespace

/* Points p0 .. p1 - 1; Pd: the cameras in double precision (12 per image;
 * null: the block's). */
static int32_t tri_impl(const rpba_block *b, const double *Pd_in, int p0, int p1, const float *sig0w,
                        int32_t robustmode, int32_t weight_only, const int32_t *part, int32_t nparts, double *XXo,
                        uint8_t *keep, float *sig0v_out, uint8_t *conv, double *sig0io, int64_t *redundancy,
                        float *w3d) {
  std::vector<double> Pown;
  if (!Pd_in) {
    Pown.resize(12 * (size_t)b->n_images);
    for (size_t i = 0; i < Pown.size(); ++i) Pown[i] = (double)b->pmat[i];
  }
  const double *Pd = Pd_in ? Pd_in : Pown.data();
  double s0io = 0.;
  long long red = 0;
  for (int pi = p0; pi < p1; ++pi) {
    const int s = b->pt_obs_off[pi], e = b->pt_obs_off[pi + 1], pxs = e - s;
    for (int j = s; j < e; ++j) keep[j] = 0;
    conv[pi] = 0;
    const double Xin[3] = {(double)b->XX[3 * pi], (double)b->XX[3 * pi + 1], (double)b->XX[3 * pi + 2]};
    for (int q = 0; q < 3; ++q) XXo[3 * pi + q] = Xin[q];
    if (w3d)
      for (int q = 0; q < 6 * nparts; ++q) w3d[(size_t)pi * 6 * nparts + q] = 0.f;
    if (pxs <= 0) continue;
    // partitions that see the point (pitflags)
    std::vector<char> pit(w3d ? nparts : 0, 0);
    if (w3d)
      for (int j = s; j < e; ++j) pit[part[b->pt_obs_image[j]]] = 1;
    std::vector<TriObs> ob(pxs);
    std::vector<float> wx(pxs), wy(pxs), wxy(pxs), wxo(pxs), wyo(pxs), wxyo(pxs), sv(pxs), p1v(pxs), p2v(pxs),
        p3v(pxs);
    std::vector<double> corr(2 * pxs), Bw(6 * pxs);
    std::vector<bool> del(pxs, false);
    float wsum = 0.f;
    for (int js = 0; js < pxs; ++js) {
      ob[js].im = b->pt_obs_image[s + js];
      ob[js].sl = b->img_obs_off[ob[js].im] + b->pt_obs_slot[s + js];
      wx[js] = wxo[js] = b->wx[ob[js].sl];
      wy[js] = wyo[js] = b->wy[ob[js].sl];
      wxy[js] = wxyo[js] = b->wxy[ob[js].sl];
      wsum += wx[js] + wy[js];
    }
    int pxs2 = 2 * pxs, pxsd = pxs;
    float X0 = (float)Xin[0], X1 = (float)Xin[1], X2 = (float)Xin[2];
    float Xo0 = X0, Xo1 = X1, Xo2 = X2, sig0 = 1.e20f, sig0opt = 1.e20f;
    int iflag = robustmode > 0 ? 2 : 1, iter = 1;
    bool cv = false;
    tri_corr(b, Pd, ob, X0, X1, X2, wx, wy, wxy, wxo, wyo, wxyo, corr, sig0opt, sv, p1v, p2v, p3v);
    if (weight_only) {
      wsum /= (float)pxs2;
      s0io += sig0opt / wsum;
      red += pxs2 - 3;
    }
    std::vector<double> Nv(w3d ? 9 * nparts : 0);
    while (iflag > -1 && iter < 101) {
      double N[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      std::fill(Nv.begin(), Nv.end(), 0.);
      for (int js = 0; js < pxs; ++js) {
        const int j = ob[js].im;
        const double *P = &Pd[12 * j];
        const double x = p1v[js], y = p2v[js], P3 = p3v[js], P1 = (double)p1v[js] * p3v[js],
                     P2 = (double)p2v[js] * p3v[js];
        double xp[3], yp[3];
        for (int c = 0; c < 3; ++c) {
          xp[c] = P[c] * P3 - P[8 + c] * P1;
          yp[c] = P[4 + c] * P3 - P[8 + c] * P2;
        }
        tri_calibrated(xp, yp, x, y, b->distpara[2 * j], b->distpara[2 * j + 1], b->K[9 * j], b->K[9 * j + 4],
                       b->K[9 * j + 1]);
        double *W = &Bw[6 * js];  // row 0: x, row 1: y; weighted
        for (int c = 0; c < 3; ++c) {
          W[c] = xp[c] * wx[js] + yp[c] * wxy[js];
          W[3 + c] = yp[c] * wy[js] + xp[c] * wxy[js];
        }
        for (int r = 0; r < 3; ++r)
          for (int c = 0; c < 3; ++c) N[r * 3 + c] += xp[r] * W[c] + yp[r] * W[3 + c];
        if (w3d && nparts > 1) {
          const int ij = part[j];
          for (int i = 0; i < nparts; ++i)
            if (pit[i] && i != ij)
              for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) Nv[9 * i + r * 3 + c] += xp[r] * W[c] + yp[r] * W[3 + c];
        }
      }
      if (w3d && nparts == 1) std::copy(N, N + 9, Nv.begin());
      N[0] *= 1.001;
      N[4] *= 1.001;
      N[8] *= 1.001;
      double Ni[9];
      inv3(N, Ni);
      double dx[3] = {0., 0., 0.};
      for (int js = 0; js < pxs; ++js) {
        const double *W = &Bw[6 * js];
        for (int r = 0; r < 3; ++r) {
          double t = 0.;
          for (int c = 0; c < 3; ++c) t += Ni[r * 3 + c] * (W[c] * corr[2 * js] + W[3 + c] * corr[2 * js + 1]);
          dx[r] += t;
        }
      }
      X0 = Xo0 + (float)dx[0];
      X1 = Xo1 + (float)dx[1];
      X2 = Xo2 + (float)dx[2];
      tri_corr(b, Pd, ob, X0, X1, X2, wx, wy, wxy, wxo, wyo, wxyo, corr, sig0, sv, p1v, p2v, p3v);
      if (iflag == 1 && robustmode == 2) {
        for (int js = 0; js < pxs; ++js)
          if (sv[js] * sig0w[ob[js].im] > 16.f) {
            wx[js] *= 1.e-4f;
            wy[js] *= 1.e-4f;
            wxy[js] *= 1.e-4f;
            if (wx[js] + wy[js] < 2.e-8f) {
              wx[js] = wy[js] = 1.e-8f;
              wxy[js] = 0.f;
            }
            --pxsd;
            del[js] = true;
          }
        if (pxsd < 2) break;
      }
      if (sig0 < sig0opt * 1.001) {
        if (sig0opt < sig0 * 1.05f) --iflag;
        if (!weight_only) {
          Xo0 = X0;
          Xo1 = X1;
          Xo2 = X2;
        }
        sig0opt = sig0;
        cv = true;
        if (w3d)
          for (int i = 0; i < nparts; ++i) {
            float *o = &w3d[((size_t)pi * nparts + i) * 6];
            const double *M = &Nv[9 * i];
            o[0] = (float)M[0];  // XX
            o[1] = (float)M[4];  // YY
            o[2] = (float)M[8];  // ZZ
            o[3] = (float)M[1];  // XY
            o[4] = (float)M[2];  // XZ
            o[5] = (float)M[5];  // YZ
          }
      } else {
        --iflag;
      }
      if (weight_only) break;
      ++iter;
    }
    int kept = 0;
    for (int js = 0; js < pxs; ++js) {
      sig0v_out[s + js] = sv[js];
      const bool k = !(robustmode == 2 && del[js]);
      keep[s + js] = k ? 1 : 0;
      if (!k) pxs2 -= 2;
      kept += k;
    }
    if (kept < 2 || !cv) {
      for (int js = 0; js < pxs; ++js) keep[s + js] = 0;
      for (int q = 0; q < 3; ++q) XXo[3 * pi + q] = Xin[q];
      continue;
    }
    conv[pi] = 1;
    if (!weight_only) {
      XXo[3 * pi] = Xo0;
      XXo[3 * pi + 1] = Xo1;
      XXo[3 * pi + 2] = Xo2;
      wsum /= (float)pxs2;
      s0io += sig0opt / wsum;
      red += pxs2 - 3;
    }
  }
  *sig0io = s0io;
  *redundancy = red;
  return RPBA_OK;
}

extern "C" int32_t oracle_triangulate(const rpba_block *b, const float *sig0w, int32_t robustmode,
                                      int32_t weight_only, double *XXo, uint8_t *keep, float *sig0v_out,
                                      uint8_t *conv, double *sig0io, int64_t *redundancy) {
  return tri_impl(b, nullptr, 0, b->n_points, sig0w, robustmode, weight_only, nullptr, 1, XXo, keep, sig0v_out,
                  conv, sig0io, redundancy, nullptr);
}

/* One GCP-mode step of the LSA on a block (the parallel RPBA's
 * per-partition call; the block holds the partition's images and the
 * observations in them): gcpinfo per point (GCP index or -1), W3 (6 per GCP
 * point the LSA keeps, in point order), gcpdata (3 per GCP index), the
 * scene's camera count.  The cameras (pmat, K, distpara), the points and the
 * point lists of the block are replaced by the LSA's output.  Robust is off,
 * as in the reference's call. */
extern "C" int32_t oracle_lsa_gcp_step(rpba_block *blk, const rpba_options *o, const int32_t *gcpinfo,
                                       const float *W3, const double *gcpdata, int32_t ncam_total, char *log,
                                       size_t cap) {
  if (!blk || !o || !gcpinfo || !gcpdata || ncam_total < blk->n_images) return RPBA_ERR_ARG;
  std::string os;
  Opts op = make_opts(o);
  op.robust = false;
  LSA lsa(blk, op, &os, GcpIn{gcpinfo, W3, gcpdata, ncam_total});
  const int st = lsa.adjust_gcp_step();
  if (st == RPBA_OK) lsa.output(blk);
  copy_log(os, log, cap);
  return st;
}

/* The parallel RPBA's two steps with the signatures of the library's
 * rpba_gcp_step_fn and rpba_merge_fn (checker side of the host-side test of
 * the library's loop):
 *   the partition step: oracle_lsa_gcp_step with the cameras in double
 *   precision in and out and the points PointXXvIn took; the block gets
 *   cameras, points and tracks whatever the step's status (OutputLSAP runs
 *   after Adjust either way, rpbacore.cpp:229-231);
 *   the merge pass: CalcLSAXMulti over every point (tri_impl), with every
 *   point's contribution to the sum and to the redundancy. */
extern "C" int32_t oracle_lsa_gcp_step_full(rpba_block *blk, const rpba_options *o, const int32_t *gcpinfo,
                                            const float *W3, int32_t n_w3, const double *gcpdata, int32_t n_gcp,
                                            int32_t ncam_total, const double *pmat_d, double *pmat_d_out,
                                            uint8_t *point_used, rpba_report *rep, char *log, size_t cap) {
  if (!blk || !o || !gcpinfo || (n_gcp > 0 && !gcpdata) || ncam_total < blk->n_images) return RPBA_ERR_ARG;
  (void)n_w3;
  (void)rep;
  std::string os;
  Opts op = make_opts(o);
  op.robust = false;
  GcpIn g{gcpinfo, W3, gcpdata, ncam_total};
  g.Pd = pmat_d;
  LSA lsa(blk, op, &os, g);
  const int st = lsa.adjust_gcp_step();
  lsa.output(blk);
  if (pmat_d_out) std::memcpy(pmat_d_out, lsa.P.data(), sizeof(double) * lsa.P.size());
  if (point_used) {
    std::memset(point_used, 0, (size_t)blk->n_points);
    for (int q : lsa.nrpv) point_used[q] = 1;
  }
  copy_log(os, log, cap);
  return st;
}

extern "C" int32_t oracle_merge(const rpba_block *b, const double *Pd, const float *sig0w, int32_t robustmode,
                                int32_t weight_only, const int32_t *part, int32_t nparts, int32_t device,
                                double *XX_out, uint8_t *keep, float *sig0v, uint8_t *conv, float *w3d,
                                double *s0_pt, int32_t *red_pt) {
  (void)device;
  for (int p = 0; p < b->n_points; ++p) {
    double s0 = 0.;
    int64_t red = 0;
    tri_impl(b, Pd, p, p + 1, sig0w, robustmode, weight_only, part, nparts, XX_out, keep, sig0v, conv, &s0, &red,
             w3d);
    if (s0_pt) s0_pt[p] = s0;
    if (red_pt) red_pt[p] = (int32_t)red;
  }
  return RPBA_OK;
}

/* ---------------------------------------------------------------------
 * Parallel RPBA: the partitioned branch of CalcPLSA, rpbacore.cpp:100-510.
 * The images are cut into nthreads partitions (part[image]; the reference
 * partitions with METIS, rpba_partition_images replaces it).  Outer
 * iteration `iter`:
 *   iter > 1: every partition's LSA takes one GCP-mode step (its images,
 *     the observations in them, the points it shares with other partitions
 *     held by 3-D priors with the weight blocks of the last merge; the
 *     additional parameters stay fixed at iter 2) and its cameras replace
 *     the scene's;
 *   the merge: every point is refined against the new cameras by
 *   CalcLSAXMulti (first a robust pass that gives the per-image thresholds
 *   when the robust stage starts, then the main pass: robust deletion,
 *   weight-only at iter 1, the per-partition weight blocks), in nthreads
 *   chunks of points whose sums are added in chunk order;
 *   sigma0 = sum / (redundancy - unknowns); the best state is kept, and the
 *   points seen by more than one partition become the next GCPs at their
 *   refined positions;
 * until iflag runs out (sig0frac rule) or 50 iterations.  The partition
 * LSAs and the point chunks run on host threads; results do not depend on
 * the scheduling. */
namespace {

struct PObs {
  int image, slot;
};
struct PCam {
  float K[9], d[2];
};

template <class F>
void par_for(int n, F &&f) {
  std::vector<std::thread> th;
  for (int k = 1; k < n; ++k) th.emplace_back(f, k);
  if (n > 0) f(0);
  for (auto &t : th) t.join();
}

// a block over the scene's cameras and slots with the given point lists
struct TmpBlock {
  rpba_block b{};
  std::vector<int32_t> off, img, slot;
  std::vector<float> XX, pmat, K, dist;
};

}  // namespace

extern "C" int32_t oracle_calc_plsa_parallel(rpba_block *blk, const rpba_options *o, int32_t nthreads,
                                             const int32_t *part, char *log, size_t cap, double *stats) {
  const int nrimages = blk->n_images, pxs = blk->n_points, T = nthreads;
  if (T < 2 || !part) return RPBA_ERR_ARG;
  for (int i = 0; i < nrimages; ++i)
    if (part[i] < 0 || part[i] >= T) return RPBA_ERR_ARG;
  std::string os;
  const Opts op = make_opts(o);
  const bool robustflag = op.robust;
  const int nraddp = (int)op.addf[0] + (int)op.addf[1] + (int)op.addf[2];
  // partitions: images in index order
  std::vector<std::vector<int>> imgindv(T);
  std::vector<int> imgindbv(nrimages);
  for (int i = 0; i < nrimages; ++i) {
    imgindv[part[i]].push_back(i);
    imgindbv[i] = part[i];
  }
  for (int it = 0; it < T; ++it)
    if (imgindv[it].empty()) return RPBA_ERR_ARG;
  // state
  std::vector<double> XXd(3 * (size_t)pxs), XXdold, PMd(12 * (size_t)nrimages), PMdold;
  for (size_t i = 0; i < XXd.size(); ++i) XXd[i] = (double)blk->XX[i];
  for (size_t i = 0; i < PMd.size(); ++i) PMd[i] = (double)blk->pmat[i];
  PMdold = PMd;
  XXdold = XXd;
  std::vector<PCam> cameras(nrimages), cameraps, camerasnew(nrimages), camerasold(nrimages);
  for (int i = 0; i < nrimages; ++i) {
    for (int c = 0; c < 9; ++c) cameras[i].K[c] = blk->K[9 * i + c];
    cameras[i].d[0] = blk->distpara[2 * i];
    cameras[i].d[1] = blk->distpara[2 * i + 1];
  }
  cameraps = cameras;
  std::vector<std::vector<PObs>> pointXXv(pxs), pointXXvold;
  for (int p = 0; p < pxs; ++p)
    for (int t = blk->pt_obs_off[p]; t < blk->pt_obs_off[p + 1]; ++t)
      pointXXv[p].push_back({blk->pt_obs_image[t], blk->pt_obs_slot[t]});
  pointXXvold = pointXXv;
  std::vector<std::vector<char>> pitflagsv(pxs);
  std::vector<int> gcpinfo(pxs, -1);
  std::vector<std::vector<PCam>> camerasoit(T, cameras);
  std::vector<std::vector<double>> PMdd(T, PMd);
  std::vector<std::vector<std::vector<PObs>>> pointXXvv(T);
  std::vector<std::vector<int>> pindv(T), gcpinfov(T);
  std::vector<std::vector<float>> W3ijiv(T);
  std::vector<double> gcpdatav;
  std::vector<float> sig0wv(nrimages, 0.f);
  const int nrparimages = (nrimages - 2) * 6 + 5 + nrimages * nraddp;
  const int nrppt = pxs / T;
  std::vector<int> beginv(T), endv(T);
  for (int c = 0; c < T; ++c) {
    beginv[c] = nrppt * c;
    endv[c] = c == T - 1 ? pxs : nrppt * (c + 1);
  }
  double sig0opt = 1.e20, sig0g = 0.;
  int iflag = robustflag ? 2 : 1, iter = 1;
  float sig0frac = 1.01f;
  std::vector<float> w3d((size_t)pxs * T * 6, 0.f);

  // a block of the whole scene with the current point lists and points
  auto scene_block = [&](TmpBlock &tb) {
    tb.b = *blk;
    tb.off.assign(pxs + 1, 0);
    tb.img.clear();
    tb.slot.clear();
    for (int p = 0; p < pxs; ++p) {
      for (const PObs &q : pointXXv[p]) {
        tb.img.push_back(q.image);
        tb.slot.push_back(q.slot);
      }
      tb.off[p + 1] = (int32_t)tb.img.size();
    }
    tb.XX.resize(3 * (size_t)pxs);
    for (size_t i = 0; i < tb.XX.size(); ++i) tb.XX[i] = (float)XXd[i];
    tb.K.resize(9 * (size_t)nrimages);
    tb.dist.resize(2 * (size_t)nrimages);
    for (int i = 0; i < nrimages; ++i) {
      for (int c = 0; c < 9; ++c) tb.K[9 * i + c] = cameraps[i].K[c];
      tb.dist[2 * i] = cameraps[i].d[0];
      tb.dist[2 * i + 1] = cameraps[i].d[1];
    }
    tb.b.pt_obs_off = tb.off.data();
    tb.b.pt_obs_image = tb.img.data();
    tb.b.pt_obs_slot = tb.slot.data();
    tb.b.XX = tb.XX.data();
    tb.b.K = tb.K.data();
    tb.b.distpara = tb.dist.data();
  };
  // one CalcLSAXMulti sweep over all points in chunks; applies the point
  // updates and the deletions; returns the chunk sums in chunk order
  auto sweep = [&](int robustmode, bool weightonly, bool wxy, std::vector<std::vector<float>> *sig0vv) {
    TmpBlock tb;
    scene_block(tb);
    const size_t nt = tb.img.size();
    std::vector<double> XXo(3 * (size_t)pxs);
    std::vector<uint8_t> keep(nt), conv(pxs);
    std::vector<float> sv(nt);
    std::vector<double> s0(T, 0.);
    std::vector<int64_t> red(T, 0);
    par_for(T, [&](int c) {
      tri_impl(&tb.b, PMd.data(), beginv[c], endv[c], sig0wv.data(), robustmode, weightonly ? 1 : 0,
               wxy ? imgindbv.data() : nullptr, wxy ? T : 1, XXo.data(), keep.data(), sv.data(), conv.data(), &s0[c],
               &red[c], wxy ? w3d.data() : nullptr);
    });
    if (sig0vv)
      for (int p = 0; p < pxs; ++p)
        if (!pointXXv[p].empty())
          for (int t = tb.off[p]; t < tb.off[p + 1]; ++t) (*sig0vv)[tb.img[t]].push_back(sv[t]);
    for (int p = 0; p < pxs; ++p) {
      if (pointXXv[p].empty()) continue;
      for (int q = 0; q < 3; ++q) XXd[3 * (size_t)p + q] = XXo[3 * (size_t)p + q];
      std::vector<PObs> kept;
      for (int t = tb.off[p]; t < tb.off[p + 1]; ++t)
        if (keep[t]) kept.push_back(pointXXv[p][t - tb.off[p]]);
      pointXXv[p] = kept;
    }
    double a = 0.;
    long long r = 0;
    for (int c = 0; c < T; ++c) {
      a += s0[c];
      r += red[c];
    }
    return std::make_pair(a, r);
  };

  while (iflag > 0 && iter < 51) {
    bool robustflagit = false;
    if (iter > 1) {
      Opts ol = op;
      ol.robust = false;
      if (iter < 3) ol.addf[0] = ol.addf[1] = ol.addf[2] = false;
      std::vector<std::string> osv(T);
      par_for(T, [&](int it) {
        const std::vector<int> &imgs = imgindv[it];
        const int m = (int)imgs.size();
        TmpBlock tb;
        std::vector<float> xg, wx, wy, wxy;
        std::vector<int32_t> ioff(m + 1, 0);
        std::vector<int> loc(nrimages, -1);
        std::vector<double> Pd(12 * (size_t)m);
        tb.pmat.resize(12 * (size_t)m);
        tb.K.resize(9 * (size_t)m);
        tb.dist.resize(2 * (size_t)m);
        for (int li = 0; li < m; ++li) {
          const int g = imgs[li];
          loc[g] = li;
          for (int c = 0; c < 12; ++c) {
            Pd[12 * li + c] = PMdd[it][12 * (size_t)g + c];
            tb.pmat[12 * li + c] = (float)Pd[12 * li + c];
          }
          for (int c = 0; c < 9; ++c) tb.K[9 * li + c] = camerasoit[it][g].K[c];
          tb.dist[2 * li] = camerasoit[it][g].d[0];
          tb.dist[2 * li + 1] = camerasoit[it][g].d[1];
          for (int sl = blk->img_obs_off[g]; sl < blk->img_obs_off[g + 1]; ++sl) {
            xg.push_back(blk->xg[2 * sl]);
            xg.push_back(blk->xg[2 * sl + 1]);
            wx.push_back(blk->wx[sl]);
            wy.push_back(blk->wy[sl]);
            wxy.push_back(blk->wxy[sl]);
          }
          ioff[li + 1] = (int32_t)wx.size();
        }
        const int np = (int)pindv[it].size();
        tb.off.assign(np + 1, 0);
        tb.XX.resize(3 * (size_t)np);
        for (int j = 0; j < np; ++j) {
          for (const PObs &q : pointXXvv[it][j]) {
            tb.img.push_back(loc[q.image]);
            tb.slot.push_back(q.slot);
          }
          tb.off[j + 1] = (int32_t)tb.img.size();
          for (int c = 0; c < 3; ++c) tb.XX[3 * j + c] = (float)XXd[3 * (size_t)pindv[it][j] + c];
        }
        rpba_block &b = tb.b;
        b.n_images = m;
        b.n_points = np;
        b.pmat = tb.pmat.data();
        b.K = tb.K.data();
        b.distpara = tb.dist.data();
        b.XX = tb.XX.data();
        b.img_obs_off = ioff.data();
        b.xg = xg.data();
        b.wx = wx.data();
        b.wy = wy.data();
        b.wxy = wxy.data();
        b.pt_obs_off = tb.off.data();
        b.pt_obs_image = tb.img.data();
        b.pt_obs_slot = tb.slot.data();
        GcpIn g{gcpinfov[it].data(), W3ijiv[it].data(), gcpdatav.data(), nrimages};
        g.Pd = Pd.data();
        LSA lsa(&b, ol, &osv[it], g);
        lsa.adjust_gcp_step();
        // OutputLSAP: PointXXvOut clears the lists of the points that
        // PointXXvIn did not take; the stored cameras (rectified by the
        // encoding even when the step did not run) and camerasnew
        for (int j = 0, k = 0; j < np; ++j) {
          if (k < lsa.nrpts && lsa.nrpv[k] == j)
            ++k;
          else
            pointXXvv[it][j].clear();
        }
        for (int li = 0; li < m; ++li) {
          const int gi = imgs[li];
          for (int c = 0; c < 12; ++c) PMdd[it][12 * (size_t)gi + c] = lsa.P[12 * li + c];
          for (int c = 0; c < 9; ++c) camerasoit[it][gi].K[c] = (float)lsa.Kn[9 * li + c];
          camerasoit[it][gi].d[0] = (float)lsa.dn[2 * li];
          camerasoit[it][gi].d[1] = (float)lsa.dn[2 * li + 1];
        }
      });
      for (int it = 0; it < T; ++it) {
        os += osv[it];
        for (int gi : imgindv[it]) {
          for (int c = 0; c < 12; ++c) PMd[12 * (size_t)gi + c] = PMdd[it][12 * (size_t)gi + c];
          cameraps[gi] = camerasoit[it][gi];
          camerasnew[gi] = camerasoit[it][gi];
        }
      }
    }
    if (iflag == 1) {
      robustflagit = robustflag;
      if (robustflag) sig0frac = 1.02f;
    }
    if (iter > 1) {
      for (int p = 0; p < pxs; ++p) pointXXv[p].clear();
      for (int it = 0; it < T; ++it)
        for (size_t j = 0; j < pindv[it].size(); ++j)
          for (const PObs &q : pointXXvv[it][j]) pointXXv[pindv[it][j]].push_back(q);
      for (int p = 0; p < pxs; ++p)
        if (pointXXv[p].size() < 2) pointXXv[p].clear();
    } else {
      for (int i = 0; i < nrimages; ++i) cameraps[i] = camerasnew[i] = cameras[i];
    }
    for (int p = 0; p < pxs; ++p)
      if (!pointXXv[p].empty()) {
        pitflagsv[p].assign(T, 0);
        for (const PObs &q : pointXXv[p]) pitflagsv[p][imgindbv[q.image]] = 1;
      }
    if (robustflagit) {
      std::vector<std::vector<float>> sig0vvs(nrimages);
      sweep(1, false, false, &sig0vvs);
      for (int i = 0; i < nrimages; ++i) {
        if (sig0vvs[i].empty()) {
          sig0wv[i] = 0.f;
        } else {
          std::sort(sig0vvs[i].begin(), sig0vvs[i].end());
          sig0wv[i] = 1.f / (sig0vvs[i][(int)sig0vvs[i].size() / 2] * 2.1981f);
        }
      }
    }
    const auto sr = sweep(robustflagit ? 2 : 0, iter == 1, true, nullptr);
    sig0g = sr.first / (double)(sr.second - nrparimages);
    {
      // the progress line (rpbacore.cpp:377-389; ihw2 = 1 for unit image sizes)
      long long nrobs = 0;
      for (int p = 0; p < pxs; ++p) nrobs += (long long)pointXXv[p].size();
      nrobs *= 2;
      const float ihw2 = 1.f;
      os += "IT: " + std::to_string(iter) + " " + std::to_string(iflag) + "  " + fmt_g(std::sqrt(sig0g * ihw2)) + ' ' +
            fmt_g(sig0opt / sig0g) + "  " + fmt_g(sig0g) + " " + std::to_string(sr.second) + " " +
            std::to_string(nrobs) + " " + std::to_string(nrparimages) + " " + std::to_string(nraddp) + "  " +
            std::to_string(sr.second - nrparimages) + "\n";
    }
    if (sig0g <= sig0opt) {
      XXdold = XXd;
      PMdold = PMd;
      pointXXvold = pointXXv;
      camerasold = camerasnew;
    }
    for (int it = 0; it < T; ++it) {
      camerasoit[it] = camerasnew;
      for (int gi : imgindv[it])
        for (int c = 0; c < 12; ++c) PMdd[it][12 * (size_t)gi + c] = PMd[12 * (size_t)gi + c];
      pointXXvv[it].clear();
      pindv[it].clear();
      W3ijiv[it].clear();
    }
    // the next GCPs: points (tracks of 2 or more) seen by more than one partition
    int nrgcpnew = 0;
    gcpdatav.clear();
    for (int c = 0; c < T; ++c)
      for (int p = beginv[c]; p < endv[c]; ++p) {
        if (pointXXv[p].size() < 2) continue;
        int gnum = 0;
        for (int it = 0; it < T && gnum < 2; ++it) gnum += pitflagsv[p][it];
        if (gnum > 1) {
          gcpinfo[p] = nrgcpnew;
          for (int q = 0; q < 3; ++q) gcpdatav.push_back(XXd[3 * (size_t)p + q]);
          for (int it = 0; it < T; ++it)
            if (pitflagsv[p][it])
              for (int q = 0; q < 6; ++q) W3ijiv[it].push_back(w3d[((size_t)p * T + it) * 6 + q]);
          ++nrgcpnew;
        } else {
          gcpinfo[p] = -1;
        }
      }
    for (int p = 0; p < pxs; ++p) {
      std::vector<std::vector<PObs>> per(T);
      for (const PObs &q : pointXXv[p]) per[imgindbv[q.image]].push_back(q);
      for (int it = 0; it < T; ++it)
        if (!per[it].empty()) {
          pointXXvv[it].push_back(per[it]);
          pindv[it].push_back(p);
        }
    }
    for (int it = 0; it < T; ++it) {
      gcpinfov[it].resize(pindv[it].size());
      for (size_t j = 0; j < pindv[it].size(); ++j) gcpinfov[it][j] = gcpinfo[pindv[it][j]];
    }
    if (iter > 1) {
      if (sig0g <= sig0opt) {
        if (sig0opt < sig0g * sig0frac && iter > 3)
          --iflag;
        else
          sig0opt = sig0g;
      } else if (iter > 3) {
        --iflag;
      }
    }
    ++iter;
  }
  // pointXXvio = pointXXvold, PMatrices, XX, cameras (rpbacore.cpp:498-507)
  int32_t t = 0;
  for (int p = 0; p < pxs; ++p) {
    blk->pt_obs_off[p] = t;
    for (const PObs &q : pointXXvold[p]) {
      blk->pt_obs_image[t] = q.image;
      blk->pt_obs_slot[t] = q.slot;
      ++t;
    }
  }
  blk->pt_obs_off[pxs] = t;
  for (size_t i = 0; i < PMdold.size(); ++i) blk->pmat[i] = (float)PMdold[i];
  for (size_t i = 0; i < XXdold.size(); ++i) blk->XX[i] = (float)XXdold[i];
  for (int i = 0; i < nrimages; ++i) {
    for (int c = 0; c < 9; ++c) blk->K[9 * i + c] = camerasold[i].K[c];
    blk->distpara[2 * i] = camerasold[i].d[0];
    blk->distpara[2 * i + 1] = camerasold[i].d[1];
  }
  if (stats) {
    stats[0] = sig0opt;
    stats[1] = iter - 1;
  }
  copy_log(os, log, cap);
  return RPBA_OK;
}

/* The same with the camera partition part[image] in 0 .. nparts - 1 and
 * the per-partition weight blocks w3d[n_points][nparts][6] (XX, YY, ZZ,
 * XY, XZ, YZ). */
extern "C" int32_t oracle_triangulate_parts(const rpba_block *b, const float *sig0w, int32_t robustmode,
                                            int32_t weight_only, const int32_t *part, int32_t nparts,
                                            double *XXo, uint8_t *keep, float *sig0v_out, uint8_t *conv,
                                            double *sig0io, int64_t *redundancy, float *w3d) {
  if (!part || nparts < 1 || !w3d) return RPBA_ERR_ARG;
  for (int i = 0; i < b->n_images; ++i)
    if (part[i] < 0 || part[i] >= nparts) return RPBA_ERR_ARG;
  return tri_impl(b, nullptr, 0, b->n_points, sig0w, robustmode, weight_only, part, nparts, XXo, keep, sig0v_out,
                  conv, sig0io, redundancy, w3d);
}

extern "C" {

/* CalcPLSA single-LSA / Exteval branches (rpbacore.cpp:28-98, 511-527). */
int32_t oracle_calc_plsa(rpba_block *blk, const rpba_options *o, char *log, size_t cap,
                         rpba_report *rep) {
  std::string os;
  if (rep) std::memset(rep, 0, sizeof *rep);
  const Opts op = make_opts(o);
  const int nraddp = (int)op.addf[0] + (int)op.addf[1] + (int)op.addf[2];
  auto t0 = std::chrono::steady_clock::now();
  if (o->exteval) {
    eval_lsa(blk, nraddp, nullptr, rep, &os);
    copy_log(os, log, cap);
    return RPBA_OK;
  }
  LSA lsa(blk, op, &os);
  if (rep) rep->points_used = lsa.nrpts;
  int st = lsa.adjust(rep);
  if (st == RPBA_OK || st == RPBA_ERR_NO_OBS_IMAGE || st == RPBA_ERR_LOW_REDUNDANCY ||
      st == RPBA_ERR_NAN_STEP) {
    /* the reference outputs its last stored state on every return path */
    if (!lsa.bad_setup) lsa.output(blk);
  }
  if (rep) {
    double rms = 0.;
    rep->cost = lsa.final_cost(&rms);
    rep->rms = rms;
    rep->status = st;
    rep->solve_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
  copy_log(os, log, cap);
  return st;
}

/* CalcPLSA with a summation-order variant of the SpMV (see g_order_variant). */
int32_t oracle_calc_plsa_variant(rpba_block *blk, const rpba_options *o, char *log, size_t cap,
                                 rpba_report *rep, int32_t variant) {
  g_order_variant = variant;
  const int32_t st = oracle_calc_plsa(blk, o, log, cap, rep);
  g_order_variant = 0;
  return st;
}

/* Per-observation Exteval residuals (dx, dy) in track order. */
int32_t oracle_exteval(const rpba_block *blk, const rpba_options *o, double *resid, rpba_report *rep) {
  const Opts op = make_opts(o);
  const int nraddp = (int)op.addf[0] + (int)op.addf[1] + (int)op.addf[2];
  if (rep) std::memset(rep, 0, sizeof *rep);
  eval_lsa(blk, nraddp, resid, rep, nullptr);
  return RPBA_OK;
}

/* -------- known-answer-test hooks -------- */
void oracle_cayley(double a, double b, double c, double *R) { cayley(a, b, c, R); }
void oracle_rectify3(double *R) { rectify(R, 3); }
void oracle_angleaxis_to_R(double a, double b, double c, float *R) { angleaxis_to_R(a, b, c, R); }
void oracle_R_to_angleaxis(const float *R, double *abc) { R_to_angleaxis(R, abc, abc + 1, abc + 2); }
double oracle_inv3(const double *m, double *out) { return inv3(m, out); }
void oracle_lu_inverse(int n, const double *A, double *Ai) { lu_inverse(n, A, Ai); }

void *oracle_lsa_create(const rpba_block *blk, const rpba_options *o) {
  static std::string sink;
  LSA *l = new LSA(blk, make_opts(o), &sink);
  if (l->bad_setup) {
    delete l;
    return nullptr;
  }
  l->setup_pass_for_tests();
  return l;
}
/* The same in GCP mode (every camera free, 3-D priors). */
void *oracle_lsa_create_gcp(const rpba_block *blk, const rpba_options *o, const int32_t *gcpinfo, const float *W3,
                            const double *gcpdata, int32_t ncam_total) {
  static std::string sink;
  Opts op = make_opts(o);
  op.robust = false;
  LSA *l = new LSA(blk, op, &sink, GcpIn{gcpinfo, W3, gcpdata, ncam_total});
  if (l->bad_setup) {
    delete l;
    return nullptr;
  }
  l->setup_pass_for_tests();
  return l;
}
int32_t oracle_lsa_n_points(void *h) { return ((LSA *)h)->nrpts; }
/* PointXXvIn's result: track offsets, images and slots (local order) and,
 * in GCP mode, every kept point's GCP index. */
void oracle_lsa_tracks(void *h, int32_t *toff, int32_t *timg, int32_t *tslot, int32_t *gcpi) {
  LSA *l = (LSA *)h;
  std::copy(l->toff.begin(), l->toff.end(), toff);
  std::copy(l->timg.begin(), l->timg.end(), timg);
  std::copy(l->tslot.begin(), l->tslot.end(), tslot);
  if (gcpi && l->ao) std::copy(l->gcpi.begin(), l->gcpi.end(), gcpi);
}
/* Reweight2D on a test handle (robust options): the cost pass at the state
 * vector gives sig0rmv (track order), then the reweighting with iflag.
 * Outputs: sig0rmv, the per-image thresholds sig00v, the weights W (3 per
 * observation), the flags and the float weight sum. */
void oracle_lsa_reweight(void *h, int32_t iflag, float *sig0rmv, float *sig00v, float *W, uint8_t *flags,
                         float *wsum) {
  LSA *l = (LSA *)h;
  l->calc_corrections(false, 1., l->XPM, true, false);
  l->reweight(iflag);
  const int n = l->toff[l->nrpts];
  std::copy(l->sig0rmv.begin(), l->sig0rmv.begin() + n, sig0rmv);
  std::copy(l->sig00v.begin(), l->sig00v.end(), sig00v);
  std::copy(l->W.begin(), l->W.begin() + 3 * n, W);
  for (int o = 0; o < n; ++o) flags[o] = l->isflag[o] ? 1 : 0;
  *wsum = l->wsum;
}
/* RobustDelete on a test handle, with the flags of a Reweight2D(iflag)
 * taken as the stored state's (ISflagnew); the handle's tracks, points and
 * weights are replaced (read them with oracle_lsa_tracks and
 * oracle_lsa_points). */
void oracle_lsa_robust_delete(void *h, int32_t iflag) {
  LSA *l = (LSA *)h;
  l->calc_corrections(false, 1., l->XPM, true, false);
  l->reweight(iflag);
  l->isflagnew = l->isflag;
  l->robust_delete();
}
/* The kept points: their indices in the caller's block and coordinates. */
void oracle_lsa_points(void *h, int32_t *nrpv, double *XX) {
  LSA *l = (LSA *)h;
  std::copy(l->nrpv.begin(), l->nrpv.end(), nrpv);
  std::copy(l->XX.begin(), l->XX.end(), XX);
}
/* The trial cameras the last decoding produced (eRMnew, ePCnew, camerasnew:
 * 9, 3, 9 and 2 doubles per image) and defdiff. */
double oracle_lsa_cameras(void *h, double *R, double *PC, double *K, double *d) {
  LSA *l = (LSA *)h;
  std::copy(l->Rn.begin(), l->Rn.end(), R);
  std::copy(l->PCn.begin(), l->PCn.end(), PC);
  std::copy(l->Kn.begin(), l->Kn.end(), K);
  std::copy(l->dn.begin(), l->dn.end(), d);
  return l->defdiff;
}
/* The float cost sum of the cost pass at the state vector. */
float oracle_lsa_sig0(void *h) {
  LSA *l = (LSA *)h;
  l->calc_corrections(false, 1., l->XPM, true, false);
  return l->sig0;
}
/* The LSA's primitives one at a time, for a restatement of Adjust's
 * control flow driven from outside (rbacore.cpp:333-616).  A raw handle
 * (after the constructor only) and one operation per call:
 *   0 PrepareWeights2D(pass = arg), flags cleared; out: wsum
 *   1 points into XPMatrices, EncodeCameras; out: nrioff3, nraddpi *
 *     nrcameras, observations, lflflag, 1 if an image has no observation
 *   2 DecodeCameras(XPMatrices) and the cost pass; out: sig0
 *   3 Reweight2D(iflag = arg); out: wsum, flagged observations
 *   4 CalcBundleSep(multfact = arg), XPMatricesnew = XPMatrices - x; out:
 *     1 if x holds a NaN or an infinity
 *   5 DecodeCameras(XPMatricesnew) and the cost pass; out: sig0
 *   6 StoreResultsIteration
 *   7 RobustDelete (flags of the stored state); out: observations, points
 *   8 iniflag = true (a new pass) */
void *oracle_lsa_create_raw(const rpba_block *blk, const rpba_options *o) {
  static std::string sink;
  LSA *l = new LSA(blk, make_opts(o), &sink);
  if (l->bad_setup) {
    delete l;
    return nullptr;
  }
  return l;
}
void oracle_lsa_op(void *h, int32_t op, double arg, double *out) {
  LSA *l = (LSA *)h;
  switch (op) {
    case 0:
      l->imagepointnr = l->toff[l->nrpts];
      l->isflag.assign(l->imagepointnr, 0);
      l->isflagnew.assign(l->imagepointnr, 0);
      l->sig0rmv.assign(l->imagepointnr, 0.f);
      l->prepare_weights((int)arg);
      out[0] = l->wsum;
      break;
    case 1: {
      for (int i = 0; i < l->nrpts; ++i)
        for (int j = 0; j < 3; ++j) l->XPM[l->nrioff + i * 3 + j] = l->XX[3 * i + j];
      l->encode_cameras();
      std::vector<int> cnt(l->nimg, 0);
      for (int o = 0; o < l->toff[l->nrpts]; ++o) ++cnt[l->timg[o]];
      out[0] = l->nrioff3;
      out[1] = l->nadd * l->nimg;
      out[2] = l->toff[l->nrpts];
      out[3] = l->lflflag ? 1 : 0;
      out[4] = std::count(cnt.begin(), cnt.end(), 0) > 0 ? 1 : 0;
      l->x.assign(l->nrioff3 + l->nadd * l->nimg, 0.);
      break;
    }
    case 2:
      l->decode_cameras(l->XPM);
      l->calc_corrections(false, 1., l->XPM, true, false);
      out[0] = l->sig0;
      break;
    case 3: {
      l->reweight((int)arg);
      int nf = 0;
      for (char f : l->isflag) nf += f ? 1 : 0;
      out[0] = l->wsum;
      out[1] = nf;
      break;
    }
    case 4: {
      out[0] = l->calc_bundle_sep(arg) ? 2 : 0;
      for (int i = 0; i < (int)l->x.size(); ++i) {
        if (!std::isfinite(l->x[i])) out[0] = 1;
        l->XPMn[i] = l->XPM[i] - l->x[i];
      }
      break;
    }
    case 5:
      l->decode_cameras(l->XPMn);
      l->calc_corrections(false, 1., l->XPMn, true, false);
      out[0] = l->sig0;
      break;
    case 6:
      l->store_results();
      break;
    case 7:
      l->robust_delete();
      out[0] = l->toff[l->nrpts];
      out[1] = l->nrpts;
      break;
    case 8:
      l->iniflag = true;
      break;
  }
}
void oracle_lsa_output(void *h, rpba_block *blk) { ((LSA *)h)->output(blk); }
/* DecodeCameras of a given state vector (nrioff3 entries); read the result
 * with oracle_lsa_cameras. */
void oracle_lsa_decode(void *h, const double *xm) {
  LSA *l = (LSA *)h;
  std::vector<double> XM(l->XPM);
  std::memcpy(XM.data(), xm, sizeof(double) * l->nrioff3);
  l->decode_cameras(XM);
}
/* One damped solve (CalcBundleSep with multfact) on a test handle: the
 * trial state vector XPMatricesnew = XPMatrices - x (nrioff3 entries). */
int32_t oracle_lsa_step_xm(void *h, double multfact, double *xm_new) {
  LSA *l = (LSA *)h;
  l->iniflag = true;
  l->x.assign(l->nrioff3 + l->nadd * l->nimg, 0.);
  if (l->calc_bundle_sep(multfact)) return l->status != RPBA_OK ? l->status : RPBA_ERR_SOLVER;
  for (int i = 0; i < l->nrioff3; ++i) xm_new[i] = l->XPM[i] - l->x[i];
  return RPBA_OK;
}
/* One GCP-mode step on a fresh LSA: the state vector after it (the
 * stored XPMatrices, nrioff3 entries). */
int32_t oracle_lsa_gcp_step_xm(const rpba_block *blk, const rpba_options *o, const int32_t *gcpinfo,
                               const float *W3, const double *gcpdata, int32_t ncam_total, double *xm_after) {
  std::string os;
  Opts op = make_opts(o);
  op.robust = false;
  LSA l(blk, op, &os, GcpIn{gcpinfo, W3, gcpdata, ncam_total});
  const int st = l.adjust_gcp_step();
  std::memcpy(xm_after, l.XPM.data(), sizeof(double) * l.nrioff3);
  return st;
}
void oracle_lsa_destroy(void *h) { delete (LSA *)h; }
int32_t oracle_lsa_xm_size(void *h) { return ((LSA *)h)->nrioff3; }
int32_t oracle_lsa_n_track_obs(void *h) { return ((LSA *)h)->toff[((LSA *)h)->nrpts]; }
int32_t oracle_lsa_nrioff(void *h) { return ((LSA *)h)->nrioff; }
int32_t oracle_lsa_normcamera(void *h) { return ((LSA *)h)->normcamera; }
void oracle_lsa_get_xm(void *h, double *xm) {
  LSA *l = (LSA *)h;
  std::memcpy(xm, l->XPM.data(), sizeof(double) * l->nrioff3);
}
void oracle_lsa_residuals(void *h, const double *xm, double *res) {
  LSA *l = (LSA *)h;
  std::vector<double> XM(l->XPM);
  std::memcpy(XM.data(), xm, sizeof(double) * l->nrioff3);
  std::vector<double> r;
  l->residuals_at(XM, r);
  std::memcpy(res, r.data(), sizeof(double) * r.size());
  l->decode_cameras(l->XPM);
}
void oracle_lsa_jacobian(void *h, int tobs, double *Bc, int *ncols, int *coff, double *Bp) {
  ((LSA *)h)->jacobian_of(tobs, Bc, ncols, coff, Bp);
}

/* ------------------------------------------------ BAL I/O (rpba.cpp) */

/* InputBlock, rpba.cpp:180-284. */
int32_t oracle_input_block(const char *path, int32_t nraddpar, int32_t k24out, rpba_block *out) {
  (void)nraddpar;
  std::ifstream fin(path);
  if (!fin) return RPBA_ERR_IO;
  int nc = 0, np = 0, no = 0;
  fin >> nc >> np >> no;
  if (!fin || nc <= 0 || np < 0 || no < 0) return RPBA_ERR_IO;
  std::vector<std::vector<float>> xin(nc), yin(nc);
  std::vector<std::vector<int32_t>> pimg(np), pslot(np);
  for (int i = 0; i < no; ++i) {
    int c, p;
    float x, y;
    fin >> c >> p >> x >> y;
    if (!fin || c < 0 || c >= nc || p < 0 || p >= np) return RPBA_ERR_IO;
    xin[c].push_back(x);
    yin[c].push_back(y);
    pimg[p].push_back(c);
    pslot[p].push_back((int32_t)xin[c].size() - 1);
  }
  rpba_block b;
  std::memset(&b, 0, sizeof b);
  b.n_images = nc;
  b.n_points = np;
  auto A = [](size_t n) {
    void *p = std::calloc(n ? n : 1, 1);
    return p;
  };
  b.pmat = (float *)A(sizeof(float) * 12 * nc);
  b.K = (float *)A(sizeof(float) * 9 * nc);
  b.distpara = (float *)A(sizeof(float) * 2 * nc);
  b.XX = (float *)A(sizeof(float) * 3 * np);
  b.img_obs_off = (int32_t *)A(sizeof(int32_t) * (nc + 1));
  b.xg = (float *)A(sizeof(float) * 2 * no);
  b.wx = (float *)A(sizeof(float) * no);
  b.wy = (float *)A(sizeof(float) * no);
  b.wxy = (float *)A(sizeof(float) * no);
  b.pt_obs_off = (int32_t *)A(sizeof(int32_t) * (np + 1));
  b.pt_obs_image = (int32_t *)A(sizeof(int32_t) * no);
  b.pt_obs_slot = (int32_t *)A(sizeof(int32_t) * no);
  for (int i = 0; i < nc; ++i) {
    double a, bb, c;
    float t0, t1, t2, f, k2, k4;
    fin >> a >> bb >> c >> t0 >> t1 >> t2 >> f >> k2 >> k4;
    float R[9];
    angleaxis_to_R(a, bb, c, R);
    float *P = &b.pmat[12 * i];
    for (int r = 0; r < 3; ++r)
      for (int cc = 0; cc < 3; ++cc) P[r * 4 + cc] = R[r * 3 + cc];
    P[3] = t0;
    P[7] = t1;
    P[11] = t2;
    float *K = &b.K[9 * i];
    K[0] = K[4] = f;
    K[8] = 1.f;
    if (k24out) {
      b.distpara[2 * i] = k2;
      b.distpara[2 * i + 1] = k4;
    } else {
      b.distpara[2 * i] = k2 * f * f;
      b.distpara[2 * i + 1] = k4 * f * f * f * f;
    }
    b.img_obs_off[i + 1] = b.img_obs_off[i] + (int32_t)xin[i].size();
    for (size_t j = 0; j < xin[i].size(); ++j) {
      const int sl = b.img_obs_off[i] + (int)j;
      b.xg[2 * sl] = -xin[i][j];
      b.xg[2 * sl + 1] = -yin[i][j];
      b.wx[sl] = 1.f;
      b.wy[sl] = 1.f;
      b.wxy[sl] = 0.f;
    }
  }
  for (int i = 0; i < np; ++i) fin >> b.XX[3 * i] >> b.XX[3 * i + 1] >> b.XX[3 * i + 2];
  int o = 0;
  for (int i = 0; i < np; ++i) {
    for (size_t j = 0; j < pimg[i].size(); ++j, ++o) {
      b.pt_obs_image[o] = pimg[i][j];
      b.pt_obs_slot[o] = pslot[i][j];
    }
    b.pt_obs_off[i + 1] = o;
  }
  if (!fin) return RPBA_ERR_IO;
  *out = b;
  return RPBA_OK;
}

void oracle_block_free(rpba_block *b) {
  std::free(b->pmat);
  std::free(b->K);
  std::free(b->distpara);
  std::free(b->XX);
  std::free(b->img_obs_off);
  std::free(b->xg);
  std::free(b->wx);
  std::free(b->wy);
  std::free(b->wxy);
  std::free(b->pt_obs_off);
  std::free(b->pt_obs_image);
  std::free(b->pt_obs_slot);
  std::memset(b, 0, sizeof *b);
}

/* OutputBlock, rpba.cpp:288-338. */
int32_t oracle_output_block(const char *path, rpba_block *b, int32_t k24out) {
  std::ofstream fout(path);
  if (!fout) return RPBA_ERR_IO;
  const int nc = b->n_images, np = b->n_points;
  const int nobs = b->pt_obs_off[np];
  fout << nc << ' ' << np << ' ' << nobs << '\n';
  fout.precision(8);
  for (int i = 0; i < np; ++i) {
    const int s = b->pt_obs_off[i], e = b->pt_obs_off[i + 1];
    std::vector<std::pair<int, int>> v;
    for (int j = s; j < e; ++j) v.emplace_back(b->pt_obs_image[j], b->pt_obs_slot[j]);
    std::stable_sort(v.begin(), v.end(), [](auto &l, auto &r) { return l.first < r.first; });
    for (int j = s; j < e; ++j) {
      b->pt_obs_image[j] = v[j - s].first;
      b->pt_obs_slot[j] = v[j - s].second;
      const int sl = b->img_obs_off[v[j - s].first] + v[j - s].second;
      fout << v[j - s].first << ' ' << i << ' ' << -b->xg[2 * sl] << ' ' << -b->xg[2 * sl + 1] << '\n';
    }
  }
  for (int i = 0; i < nc; ++i) {
    double a, bb, c;
    float R[9];
    const float *P = &b->pmat[12 * i];
    for (int r = 0; r < 3; ++r)
      for (int cc = 0; cc < 3; ++cc) R[r * 3 + cc] = P[r * 4 + cc];
    R_to_angleaxis(R, &a, &bb, &c);
    fout << a << ' ' << bb << ' ' << c << ' ' << P[3] << ' ' << P[7] << ' ' << P[11] << ' ';
    fout << b->K[9 * i] << ' ';
    if (k24out) {
      fout << b->distpara[2 * i] << ' ' << b->distpara[2 * i + 1] << '\n';
    } else {
      const double f = b->K[9 * i];
      const double f2 = 1. / (f * f);
      fout << b->distpara[2 * i] * f2 << ' ' << b->distpara[2 * i + 1] * f2 * f2 << '\n';
    }
  }
  for (int i = 0; i < np; ++i) fout << b->XX[3 * i] << ' ' << b->XX[3 * i + 1] << ' ' << b->XX[3 * i + 2] << '\n';
  return fout ? RPBA_OK : RPBA_ERR_IO;
}

} // extern "C"
