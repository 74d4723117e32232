// bal_io.cpp -- BAL text I/O of a block: InputBlock / OutputBlock
// (rpba.cpp:180-338) with the angle-axis conversions (rpba.cpp:343-439).
// The parse keeps the reference's quantisation: the angle-axis is read as
// double and the rotation stored as float; translation, focal length,
// distortion, points and observations are floats; observations are negated
// into xg; every slot gets unit weights; with k24out = 0 the distortion is
// scaled by f^2 / f^4.
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <algorithm>

#include "../../include/rpba_b200.h"

namespace {

// Whitespace-separated number reader over a whole file in memory.
struct Reader {
  std::vector<char> buf;
  const char *p = nullptr, *e = nullptr;
  bool ok = true;
  bool open(const char *path) {
    FILE *f = std::fopen(path, "rb");
    if (!f) return false;
    std::fseek(f, 0, SEEK_END);
    const long n = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    buf.resize((size_t)n + 1);
    const size_t got = std::fread(buf.data(), 1, (size_t)n, f);
    std::fclose(f);
    buf[got] = 0;
    p = buf.data();
    e = p + got;
    return true;
  }
  void skip() {
    while (p < e && (*p == ' ' || *p == '\n' || *p == '\r' || *p == '\t')) ++p;
  }
  long long integer() {
    skip();
    char *end = nullptr;
    const long long v = std::strtoll(p, &end, 10);
    if (end == p) ok = false;
    p = end;
    return v;
  }
  double dbl() {
    skip();
    char *end = nullptr;
    const double v = std::strtod(p, &end);
    if (end == p) ok = false;
    p = end;
    return v;
  }
  float flt() {
    skip();
    char *end = nullptr;
    const float v = std::strtof(p, &end);
    if (end == p) ok = false;
    p = end;
    return v;
  }
};

// rpba.cpp:343-366
void angleaxis_to_R(double a, double b, double c, float *R) {
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

// rpba.cpp:371-439
void R_to_angleaxis(const float *R, double &a, double &b, double &c) {
  auto m = [&](int r, int cc) { return (double)R[r * 3 + cc]; };
  const double e0 = 0.01, e1 = 0.1, pi = 3.14159265358979323846;
  const double tr = (m(0, 0) + m(1, 1) + m(2, 2) - 1.) * 0.5;
  if (std::fabs(m(0, 1) - m(1, 0)) < e0 && std::fabs(m(1, 2) - m(2, 1)) < e0 && std::fabs(m(0, 2) - m(2, 0)) < e0) {
    if (std::fabs(m(0, 1) + m(1, 0)) < e1 && std::fabs(m(1, 2) + m(2, 1)) < e1 &&
        std::fabs(m(0, 2) + m(2, 0)) < e1 && tr > 0.9) {
      a = b = c = 0.;
      return;
    }
    const double xx = (m(0, 0) + 1.) * 0.5, yy = (m(1, 1) + 1.) * 0.5, zz = (m(2, 2) + 1.) * 0.5;
    const double xy = (m(0, 1) + m(1, 0)) * 0.25, xz = (m(0, 2) + m(2, 0)) * 0.25, yz = (m(1, 2) + m(2, 1)) * 0.25;
    if (xx > yy && xx > zz) {
      if (xx < e0) {
        a = 0.;
        b = c = std::sqrt(0.5) * pi;
        return;
      }
      const double t = std::sqrt(xx);
      a = t * pi;
      b = xy / t * pi;
      c = xz / t * pi;
      return;
    }
    if (yy > zz) {
      if (yy < e0) {
        a = c = std::sqrt(0.5) * pi;
        b = 0.;
        return;
      }
      const double t = std::sqrt(yy);
      a = xy / t * pi;
      b = t * pi;
      c = yz / t * pi;
      return;
    }
    if (zz < e0) {
      a = b = std::sqrt(0.5) * pi;
      c = 0.;
      return;
    }
    const double t = std::sqrt(zz);
    a = xz / t * pi;
    b = yz / t * pi;
    c = t * pi;
    return;
  }
  const double aa = std::acos(tr);
  const double bb = 0.5 * aa / std::sin(aa);
  a = bb * (m(2, 1) - m(1, 2));
  b = bb * (m(0, 2) - m(2, 0));
  c = bb * (m(1, 0) - m(0, 1));
}

template <typename T>
T *cal(size_t n) {
  return (T *)std::calloc(n ? n : 1, sizeof(T));
}

}  // namespace

extern "C" {

int32_t rpba_input_block(const char *path, int32_t nraddpar, int32_t k24out, rpba_block *out) {
  (void)nraddpar;
  if (!path || !out) return RPBA_ERR_ARG;
  Reader r;
  if (!r.open(path)) return RPBA_ERR_IO;
  const long long nc = r.integer(), np = r.integer(), no = r.integer();
  if (!r.ok || nc <= 0 || np < 0 || no < 0 || nc > 0x7fffffff || np > 0x7fffffff || no > 0x7fffffff)
    return RPBA_ERR_IO;
  std::vector<int32_t> ocam(no), opt(no);
  std::vector<float> ox(no), oy(no);
  std::vector<int32_t> cnt(nc + 1, 0), pcnt(np + 1, 0);
  for (long long i = 0; i < no; ++i) {
    const long long c = r.integer(), p = r.integer();
    const float x = r.flt(), y = r.flt();
    if (!r.ok || c < 0 || c >= nc || p < 0 || p >= np) return RPBA_ERR_IO;
    ocam[i] = (int32_t)c;
    opt[i] = (int32_t)p;
    ox[i] = x;
    oy[i] = y;
    ++cnt[c + 1];
    ++pcnt[p + 1];
  }
  rpba_block b;
  std::memset(&b, 0, sizeof b);
  b.n_images = (int32_t)nc;
  b.n_points = (int32_t)np;
  b.pmat = cal<float>(12 * nc);
  b.K = cal<float>(9 * nc);
  b.distpara = cal<float>(2 * nc);
  b.XX = cal<float>(3 * np);
  b.img_obs_off = cal<int32_t>(nc + 1);
  b.xg = cal<float>(2 * no);
  b.wx = cal<float>(no);
  b.wy = cal<float>(no);
  b.wxy = cal<float>(no);
  b.pt_obs_off = cal<int32_t>(np + 1);
  b.pt_obs_image = cal<int32_t>(no);
  b.pt_obs_slot = cal<int32_t>(no);
  for (long long i = 0; i < nc; ++i) b.img_obs_off[i + 1] = b.img_obs_off[i] + cnt[i + 1];
  for (long long i = 0; i < np; ++i) b.pt_obs_off[i + 1] = b.pt_obs_off[i] + pcnt[i + 1];
  std::vector<int32_t> ifill(nc, 0), pfill(np, 0);
  for (long long i = 0; i < no; ++i) {
    const int c = ocam[i], p = opt[i];
    const int slot = ifill[c]++;
    const int sl = b.img_obs_off[c] + slot;
    b.xg[2 * sl] = -ox[i];
    b.xg[2 * sl + 1] = -oy[i];
    b.wx[sl] = 1.f;
    b.wy[sl] = 1.f;
    b.wxy[sl] = 0.f;
    const int w = b.pt_obs_off[p] + pfill[p]++;
    b.pt_obs_image[w] = c;
    b.pt_obs_slot[w] = slot;
  }
  for (long long i = 0; i < nc; ++i) {
    const double a = r.dbl(), bb = r.dbl(), c = r.dbl();
    float *P = b.pmat + 12 * i;
    P[3] = r.flt();
    P[7] = r.flt();
    P[11] = r.flt();
    const float f = r.flt(), k2 = r.flt(), k4 = r.flt();
    float R[9];
    angleaxis_to_R(a, bb, c, R);
    for (int rr = 0; rr < 3; ++rr)
      for (int cc = 0; cc < 3; ++cc) P[rr * 4 + cc] = R[rr * 3 + cc];
    float *K = b.K + 9 * i;
    K[0] = K[4] = f;
    K[8] = 1.f;
    if (k24out) {
      b.distpara[2 * i] = k2;
      b.distpara[2 * i + 1] = k4;
    } else {
      b.distpara[2 * i] = k2 * f * f;
      b.distpara[2 * i + 1] = k4 * f * f * f * f;
    }
  }
  for (long long i = 0; i < 3 * np; ++i) b.XX[i] = r.flt();
  if (!r.ok) {
    rpba_block_free(&b);
    return RPBA_ERR_IO;
  }
  *out = b;
  return RPBA_OK;
}

void rpba_block_free(rpba_block *b) {
  if (!b) return;
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

int32_t rpba_output_block(const char *path, rpba_block *b, int32_t k24out) {
  if (!path || !b) return RPBA_ERR_ARG;
  FILE *f = std::fopen(path, "w");
  if (!f) return RPBA_ERR_IO;
  const int nc = b->n_images, np = b->n_points;
  std::fprintf(f, "%d %d %d\n", nc, np, b->pt_obs_off[np]);
  std::vector<std::pair<int, int>> v;
  for (int i = 0; i < np; ++i) {
    const int s = b->pt_obs_off[i], e = b->pt_obs_off[i + 1];
    v.clear();
    for (int j = s; j < e; ++j) v.emplace_back(b->pt_obs_image[j], b->pt_obs_slot[j]);
    std::stable_sort(v.begin(), v.end(), [](const std::pair<int, int> &l, const std::pair<int, int> &r) {
      return l.first < r.first;
    });
    for (int j = s; j < e; ++j) {
      b->pt_obs_image[j] = v[j - s].first;
      b->pt_obs_slot[j] = v[j - s].second;
      const int sl = b->img_obs_off[v[j - s].first] + v[j - s].second;
      std::fprintf(f, "%d %d %.8g %.8g\n", v[j - s].first, i, -b->xg[2 * sl], -b->xg[2 * sl + 1]);
    }
  }
  for (int i = 0; i < nc; ++i) {
    float R[9];
    const float *P = b->pmat + 12 * i;
    for (int rr = 0; rr < 3; ++rr)
      for (int cc = 0; cc < 3; ++cc) R[rr * 3 + cc] = P[rr * 4 + cc];
    double a, bb, c;
    R_to_angleaxis(R, a, bb, c);
    std::fprintf(f, "%.8g %.8g %.8g %.8g %.8g %.8g %.8g ", a, bb, c, P[3], P[7], P[11], b->K[9 * i]);
    if (k24out) {
      std::fprintf(f, "%.8g %.8g\n", b->distpara[2 * i], b->distpara[2 * i + 1]);
    } else {
      const double fl = b->K[9 * i];
      const double f2 = 1. / (fl * fl);
      std::fprintf(f, "%.8g %.8g\n", b->distpara[2 * i] * f2, b->distpara[2 * i + 1] * f2 * f2);
    }
  }
  for (int i = 0; i < np; ++i) std::fprintf(f, "%.8g %.8g %.8g\n", b->XX[3 * i], b->XX[3 * i + 1], b->XX[3 * i + 2]);
  const bool ok = std::ferror(f) == 0;
  std::fclose(f);
  return ok ? RPBA_OK : RPBA_ERR_IO;
}

}  // extern "C"
