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
#include <algorithm>
#include <atomic>
#include <charconv>
#include <memory>
#include <string>
#include <system_error>
#include <thread>
#include <vector>

#include "../../include/rpba_b200.h"

namespace {

// Whitespace-separated number reader over a whole file in memory.
struct Reader {
  std::unique_ptr<char[]> buf;  // the whole file (not zero-filled first)
  const char *p = nullptr, *e = nullptr;
  bool ok = true;
  bool open(const char *path) {
    FILE *f = std::fopen(path, "rb");
    if (!f) return false;
    std::fseek(f, 0, SEEK_END);
    const long n = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    buf.reset(new char[(size_t)n + 1]);
    const size_t got = std::fread(buf.get(), 1, (size_t)n, f);
    std::fclose(f);
    buf[got] = 0;
    p = buf.get();
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
  // the entries stay float as in the reference: a sum or difference of two
  // entries is rounded to float, anything with a double constant is double
  auto m = [&](int r, int cc) -> float { return R[r * 3 + cc]; };
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

// ---- parallel parse and format of large files
// The body of a BAL file (after the three counts) is a whitespace-separated
// token stream: 4 per observation (image, point, x, y), 9 per camera, 3 per
// point, whatever the line layout.  A token's global index fixes its field
// and type, so the stream is cut into byte ranges at token boundaries,
// tokens are counted per range (pass 1), and every range parses its tokens
// knowing their global index (pass 2).  std::from_chars rounds correctly,
// like the strtof/strtod of the serial path, so both give the same bits.

int io_threads() {
  const char *e = std::getenv("RPBA_IO_THREADS");
  if (e && *e) return std::max(1, std::atoi(e));
  return (int)std::min(32u, std::max(1u, std::thread::hardware_concurrency()));
}
size_t io_parallel_min_bytes() {
  const char *e = std::getenv("RPBA_IO_PARALLEL_MIN_BYTES");
  return e && *e ? (size_t)std::atoll(e) : (size_t)(8u << 20);
}

inline bool is_ws(char c) { return c == ' ' || c == '\n' || c == '\r' || c == '\t'; }

// f(k) for k < T, one thread each (a k whose thread cannot be created runs
// on the calling thread: the ranges are independent)
template <class F>
void parallel_for(int T, F &&f) {
  std::vector<std::thread> th;
  int k = 1;
  try {
    for (; k < T; ++k) th.emplace_back(f, k);
  } catch (const std::system_error &) {
  }
  for (int j = k; j < T; ++j) f(j);
  f(0);
  for (auto &t : th) t.join();
}

template <class V>
bool parse_num(const char *b, const char *e, V &v) {
  if (b < e && *b == '+') ++b;
  const auto r = std::from_chars(b, e, v);
  return r.ec == std::errc() && r.ptr == e;
}

struct BodyOut {
  long long nc, np, no;
  int32_t *ocam, *opt;
  float *ox, *oy;
  double *cam_d;  // [nc][3] angle-axis
  float *cam_f;   // [nc][6] t, f, k2, k4
  float *XX;      // [np][3]
};

// Parse the body [b, e) in parallel; false on a malformed or short body.
bool parse_body_parallel(const char *b, const char *e, BodyOut &O, int T) {
  const long long need = 4 * O.no + 9 * O.nc + 3 * O.np;
  const size_t L = (size_t)(e - b) / T + 1;
  std::vector<const char *> st(T + 1);
  for (int k = 0; k <= T; ++k) {
    const char *q = std::min(e, b + L * k);
    if (k > 0 && k < T)
      while (q < e && q > b && !is_ws(q[-1])) ++q;  // to the start of the next token
    st[k] = k == T ? e : q;
  }
  std::vector<long long> cnt(T, 0);
  parallel_for(T, [&](int k) {
    long long c = 0;
    const char *q = st[k], *z = st[k + 1];
    while (q < z) {
      while (q < z && is_ws(*q)) ++q;
      if (q >= z) break;
      ++c;
      while (q < z && !is_ws(*q)) ++q;
    }
    cnt[k] = c;
  });
  std::vector<long long> first(T + 1, 0);
  for (int k = 0; k < T; ++k) first[k + 1] = first[k] + cnt[k];
  if (first[T] < need) return false;
  std::atomic<bool> ok{true};
  const long long o1 = 4 * O.no, c1 = o1 + 9 * O.nc;
  parallel_for(T, [&](int k) {
    long long t = first[k];
    const char *q = st[k], *z = st[k + 1];
    bool good = true;
    while (q < z && t < need && good) {
      while (q < z && is_ws(*q)) ++q;
      if (q >= z) break;
      const char *s0 = q;
      while (q < z && !is_ws(*q)) ++q;
      if (t < o1) {
        const long long i = t >> 2;
        switch (t & 3) {
          case 0: { long long v; good = parse_num(s0, q, v) && v >= 0 && v < O.nc; O.ocam[i] = (int32_t)v; break; }
          case 1: { long long v; good = parse_num(s0, q, v) && v >= 0 && v < O.np; O.opt[i] = (int32_t)v; break; }
          case 2: good = parse_num(s0, q, O.ox[i]); break;
          default: good = parse_num(s0, q, O.oy[i]); break;
        }
      } else if (t < c1) {
        const long long u = t - o1, i = u / 9, f = u % 9;
        if (f < 3)
          good = parse_num(s0, q, O.cam_d[3 * i + f]);
        else
          good = parse_num(s0, q, O.cam_f[6 * i + f - 3]);
      } else {
        good = parse_num(s0, q, O.XX[t - c1]);
      }
      ++t;
    }
    if (!good) ok = false;
  });
  return ok;
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
  // large files: the whole body in parallel (same values as the serial path)
  const int T = io_threads();
  const bool par = T > 1 && (size_t)(r.e - r.p) >= io_parallel_min_bytes();
  std::vector<double> cam_d(par ? 3 * nc : 0);
  std::vector<float> cam_f(par ? 6 * nc : 0), xx(par ? 3 * np : 0);
  if (par) {
    BodyOut O{nc, np, no, ocam.data(), opt.data(), ox.data(), oy.data(), cam_d.data(), cam_f.data(), xx.data()};
    if (!parse_body_parallel(r.p, r.e, O, T)) return RPBA_ERR_IO;
    // the counts per image and per point (threads own ranges of images,
    // then of points, each scanning every observation)
    parallel_for(T, [&](int k) {
      const long long c0 = nc * k / T, c1 = nc * (k + 1) / T, p0 = np * k / T, p1 = np * (k + 1) / T;
      for (long long i = 0; i < no; ++i) {
        if (ocam[i] >= c0 && ocam[i] < c1) ++cnt[ocam[i] + 1];
        if (opt[i] >= p0 && opt[i] < p1) ++pcnt[opt[i] + 1];
      }
    });
  } else {
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
  // every observation's slot in its image and entry in its point's track,
  // in file order (with threads: each owns a range of images, then of
  // points, and scans every observation; the same slots and entries)
  std::vector<int32_t> ifill(nc, 0), pfill(np, 0), oslot(no);
  const int TS = par ? T : 1;
  auto fill_images = [&](int k) {
    const long long c0 = nc * k / TS, c1 = nc * (k + 1) / TS;
    for (long long i = 0; i < no; ++i) {
      const int c = ocam[i];
      if (c < c0 || c >= c1) continue;
      const int slot = ifill[c]++;
      const int sl = b.img_obs_off[c] + slot;
      oslot[i] = slot;
      b.xg[2 * (size_t)sl] = -ox[i];
      b.xg[2 * (size_t)sl + 1] = -oy[i];
      b.wx[sl] = 1.f;
      b.wy[sl] = 1.f;
      b.wxy[sl] = 0.f;
    }
  };
  auto fill_points = [&](int k) {
    const long long p0 = np * k / TS, p1 = np * (k + 1) / TS;
    for (long long i = 0; i < no; ++i) {
      const int p = opt[i];
      if (p < p0 || p >= p1) continue;
      const int w = b.pt_obs_off[p] + pfill[p]++;
      b.pt_obs_image[w] = ocam[i];
      b.pt_obs_slot[w] = oslot[i];
    }
  };
  parallel_for(TS, fill_images);
  parallel_for(TS, fill_points);
  for (long long i = 0; i < nc; ++i) {
    const double a = par ? cam_d[3 * i] : r.dbl(), bb = par ? cam_d[3 * i + 1] : r.dbl(),
                 c = par ? cam_d[3 * i + 2] : r.dbl();
    float *P = b.pmat + 12 * i;
    P[3] = par ? cam_f[6 * i] : r.flt();
    P[7] = par ? cam_f[6 * i + 1] : r.flt();
    P[11] = par ? cam_f[6 * i + 2] : r.flt();
    const float f = par ? cam_f[6 * i + 3] : r.flt(), k2 = par ? cam_f[6 * i + 4] : r.flt(),
                k4 = par ? cam_f[6 * i + 5] : r.flt();
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
  if (par)
    std::memcpy(b.XX, xx.data(), sizeof(float) * 3 * np);
  else
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

// printf's "%.8g" and "%d" (std::to_chars in the general format with a
// precision gives printf's characters for that conversion in the "C" locale;
// the value is taken as a double, as printf's varargs promote it)
namespace {
inline char *put_g8(char *p, double v) { return std::to_chars(p, p + 40, v, std::chars_format::general, 8).ptr; }
inline char *put_d(char *p, int v) { return std::to_chars(p, p + 16, v).ptr; }
}  // namespace

int32_t rpba_output_block(const char *path, rpba_block *b, int32_t k24out) {
  if (!path || !b) return RPBA_ERR_ARG;
  FILE *f = std::fopen(path, "w");
  if (!f) return RPBA_ERR_IO;
  const int nc = b->n_images, np = b->n_points;
  std::fprintf(f, "%d %d %d\n", nc, np, b->pt_obs_off[np]);
  // observation lines of points [p0, p1): each point's observations sorted
  // by image (stable), written back in that order
  auto obs_lines = [&](int p0, int p1, std::string &out) {
    std::vector<std::pair<int, int>> v;
    char line[96];
    for (int i = p0; i < p1; ++i) {
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
        char *q = put_d(line, v[j - s].first);
        *q++ = ' ';
        q = put_d(q, i);
        *q++ = ' ';
        q = put_g8(q, -b->xg[2 * sl]);
        *q++ = ' ';
        q = put_g8(q, -b->xg[2 * sl + 1]);
        *q++ = '\n';
        out.append(line, (size_t)(q - line));
      }
    }
  };
  auto pt_lines = [&](int p0, int p1, std::string &out) {
    char line[96];
    for (int i = p0; i < p1; ++i) {
      char *q = put_g8(line, b->XX[3 * i]);
      *q++ = ' ';
      q = put_g8(q, b->XX[3 * i + 1]);
      *q++ = ' ';
      q = put_g8(q, b->XX[3 * i + 2]);
      *q++ = '\n';
      out.append(line, (size_t)(q - line));
    }
  };
  // large blocks: per-thread buffers over point ranges, written in order
  const int T = (size_t)b->pt_obs_off[np] * 40 >= io_parallel_min_bytes() ? io_threads() : 1;
  std::vector<std::string> bufs(T);
  parallel_for(T, [&](int k) { obs_lines((int)((long long)np * k / T), (int)((long long)np * (k + 1) / T), bufs[k]); });
  for (auto &x : bufs) std::fwrite(x.data(), 1, x.size(), f);
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
  for (auto &x : bufs) x.clear();
  parallel_for(T, [&](int k) { pt_lines((int)((long long)np * k / T), (int)((long long)np * (k + 1) / T), bufs[k]); });
  for (auto &x : bufs) std::fwrite(x.data(), 1, x.size(), f);
  const bool ok = std::ferror(f) == 0;
  std::fclose(f);
  return ok ? RPBA_OK : RPBA_ERR_IO;
}

}  // extern "C"
