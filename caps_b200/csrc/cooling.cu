// The glass-transition fits of a cooling scan (core/src/mechanics.cpp:1218-1378): host code of the engine library, used
// by the batched cooling driver (caps_b200/cooling.py) on the points its replicas measure. Both fits keep the
// reference's arithmetic and its bootstrap (std::mt19937_64 seeded 12345, uniform picks by rejection as
// core/include/caps/rng.hpp:54-67), so a fit of the same points gives the same Tg and error.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <numeric>
#include <random>
#include <string>
#include <vector>

#include "caps_gpu.h"

namespace {

thread_local std::string g_fit_err;

// A uniform index in [0, n - 1] by rejection from 64-bit draws (no modulo bias), as the reference's UniformInt.
struct PickIndex {
  uint64_t n;
  explicit PickIndex(size_t count) : n(uint64_t(count)) {}
  size_t operator()(std::mt19937_64& g) const {
    const uint64_t limit = std::numeric_limits<uint64_t>::max() - std::numeric_limits<uint64_t>::max() % n;
    uint64_t x;
    do x = uint64_t(g() - std::mt19937_64::min()); while (x >= limit);
    return size_t(x % n);
  }
};

std::string fmt4(double v) {
  char b[64];
  std::snprintf(b, sizeof b, "%.4g", v);
  return b;
}

// y = c0 + c1 min(T - h, 0) + c2 max(T - h, 0), least squares for a fixed hinge h (Gauss-Jordan with partial pivoting);
// returns the residual sum of squares (max double when singular)
double hinge_solve(const std::vector<double>& T, const std::vector<double>& y, double h, double c[3]) {
  const size_t n = T.size();
  double A[3][4] = {};
  for (size_t i = 0; i < n; ++i) {
    const double u[3] = {1, std::min(T[i] - h, 0.0), std::max(T[i] - h, 0.0)};
    for (int a = 0; a < 3; ++a) {
      for (int b = 0; b < 3; ++b) A[a][b] += u[a] * u[b];
      A[a][3] += u[a] * y[i];
    }
  }
  for (int k = 0; k < 3; ++k) {
    int p = k;
    for (int i = k + 1; i < 3; ++i)
      if (std::fabs(A[i][k]) > std::fabs(A[p][k])) p = i;
    for (int j = 0; j < 4; ++j) std::swap(A[k][j], A[p][j]);
    if (std::fabs(A[k][k]) < 1e-300) return std::numeric_limits<double>::max();
    for (int i = 0; i < 3; ++i)
      if (i != k) {
        const double m = A[i][k] / A[k][k];
        for (int j = 0; j < 4; ++j) A[i][j] -= m * A[k][j];
      }
  }
  for (int k = 0; k < 3; ++k) c[k] = A[k][3] / A[k][k];
  double rss = 0;
  for (size_t i = 0; i < n; ++i) {
    const double r = y[i] - (c[0] + c[1] * std::min(T[i] - h, 0.0) + c[2] * std::max(T[i] - h, 0.0));
    rss += r * r;
  }
  return rss;
}

// The hinge between the second and the second-to-last temperature: a scan of `scan` + 1 points, then 60 golden-section
// steps around the best; the refined hinge unless it fits worse than the scanned one.
double best_hinge(const std::vector<double>& T, const std::vector<double>& y, int scan) {
  const size_t n = T.size();
  const double lo = T[1], hi = T[n - 2];
  double c[3], bh = lo, br = std::numeric_limits<double>::max();
  for (int k = 0; k <= scan; ++k) {
    const double h = lo + (hi - lo) * k / scan, r = hinge_solve(T, y, h, c);
    if (r < br) br = r, bh = h;
  }
  double a = std::max(lo, bh - (hi - lo) / scan), b = std::min(hi, bh + (hi - lo) / scan);
  const double g = 0.5 * (std::sqrt(5.0) - 1);
  double x1 = b - g * (b - a), x2 = a + g * (b - a), f1 = hinge_solve(T, y, x1, c), f2 = hinge_solve(T, y, x2, c);
  for (int it = 0; it < 60; ++it) {
    if (f1 < f2) {
      b = x2, x2 = x1, f2 = f1, x1 = b - g * (b - a), f1 = hinge_solve(T, y, x1, c);
    } else {
      a = x1, x1 = x2, f1 = f2, x2 = a + g * (b - a), f2 = hinge_solve(T, y, x2, c);
    }
  }
  const double h = 0.5 * (a + b);
  return hinge_solve(T, y, h, c) <= br ? h : bh;
}

void set_note(caps_gpu_tg_fit* f, const std::string& s) {
  std::strncpy(f->note, s.c_str(), sizeof f->note - 1);
  f->note[sizeof f->note - 1] = 0;
}

// Continuous two-line fit with the hinge free (mechanics.cpp:1218-1308).
void fit_bilinear(const double* T0, const double* y0, size_t n, caps_gpu_tg_fit* fit) {
  if (n < 5) return set_note(fit, "a two-line fit needs at least five temperatures");
  std::vector<size_t> ord(n);
  std::iota(ord.begin(), ord.end(), 0);
  std::sort(ord.begin(), ord.end(), [&](size_t a, size_t b) { return T0[a] < T0[b]; });
  std::vector<double> T(n), Y(n);
  for (size_t i = 0; i < n; ++i) T[i] = T0[ord[i]], Y[i] = y0[ord[i]];
  const double h = best_hinge(T, Y, 400);
  double c[3];
  fit->rss = hinge_solve(T, Y, h, c);
  fit->tg = h;
  fit->value_at_tg = c[0];
  fit->slope_low = c[1];
  fit->slope_high = c[2];
  fit->alpha_low = c[1] / c[0];
  fit->alpha_high = c[2] / c[0];
  fit->ok = 1;
  // bootstrap of residuals: 200 resamples, each refitted with a coarser scan
  std::vector<double> fitted(n), res(n);
  for (size_t i = 0; i < n; ++i) {
    fitted[i] = c[0] + c[1] * std::min(T[i] - h, 0.0) + c[2] * std::max(T[i] - h, 0.0);
    res[i] = Y[i] - fitted[i];
  }
  std::mt19937_64 rng(12345);
  const PickIndex pick(n);
  std::vector<double> hs;
  for (int b = 0; b < 200; ++b) {
    std::vector<double> yb(n);
    for (size_t i = 0; i < n; ++i) yb[i] = fitted[i] + res[pick(rng)];
    hs.push_back(best_hinge(T, yb, 100));
  }
  double m = 0, v = 0;
  for (double x : hs) m += x / double(hs.size());
  for (double x : hs) v += (x - m) * (x - m) / double(hs.size() - 1);
  fit->tg_err = std::sqrt(v);
  if (std::fabs(c[2] - c[1]) < 0.1 * std::max(std::fabs(c[1]), std::fabs(c[2])))
    set_note(fit, "the two slopes differ by less than 10 %: no clear transition in this range");
  else if (h - T[0] < 1.5 * (T[1] - T[0]) || T[n - 1] - h < 1.5 * (T[n - 1] - T[n - 2]))
    set_note(fit, "the hinge sits at the edge of the range: extend the temperatures");
}

// Two straight lines through a glassy range (T <= glassy_max) and a rubbery one (T >= rubbery_min) and Tg where they
// cross, the error by a bootstrap of the ranges' residuals (mechanics.cpp:1310-1378).
void fit_two_ranges(const double* T, const double* y, size_t n, double glassy_max, double rubbery_min, caps_gpu_tg_fit* fit) {
  if (n < 4) return set_note(fit, "a two-range fit needs at least four temperatures");
  const auto mm = std::minmax_element(T, T + n);
  const double tmin = *mm.first, tmax = *mm.second;
  if (glassy_max <= 0) glassy_max = tmin + (tmax - tmin) / 3.0;
  if (rubbery_min <= 0) rubbery_min = tmax - (tmax - tmin) / 3.0;
  if (glassy_max >= rubbery_min) return set_note(fit, "the glassy range must end below where the rubbery range starts");
  std::vector<size_t> lo, hi;
  for (size_t i = 0; i < n; ++i) {
    if (T[i] <= glassy_max + 1e-9) lo.push_back(i);
    if (T[i] >= rubbery_min - 1e-9) hi.push_back(i);
  }
  if (lo.size() < 2 || hi.size() < 2) return set_note(fit, "each range needs at least two temperatures");
  auto line = [&](const std::vector<size_t>& idx, const std::vector<double>& Y, double& a, double& b) {
    double st = 0, sy = 0, stt = 0, sty = 0;
    for (size_t i : idx) st += T[i], sy += Y[i], stt += T[i] * T[i], sty += T[i] * Y[i];
    const double m = double(idx.size()), den = m * stt - st * st;
    b = den != 0 ? (m * sty - st * sy) / den : 0;
    a = (sy - b * st) / m;
  };
  auto cross_at = [&](const std::vector<double>& Y, double& tg, double& bl, double& bh, double& al, double& ah) {
    line(lo, Y, al, bl);
    line(hi, Y, ah, bh);
    tg = bl != bh ? (ah - al) / (bl - bh) : 0;
  };
  const std::vector<double> yv(y, y + n);
  double al, bl, ah, bh, tg;
  cross_at(yv, tg, bl, bh, al, ah);
  if (bl == bh) return set_note(fit, "the two lines are parallel: no crossing");
  fit->ok = 1;
  fit->tg = tg;
  fit->slope_low = bl;
  fit->slope_high = bh;
  fit->value_at_tg = al + bl * tg;
  if (fit->value_at_tg != 0) fit->alpha_low = bl / fit->value_at_tg, fit->alpha_high = bh / fit->value_at_tg;
  std::vector<double> res(n, 0), fitted(n, 0);
  for (size_t i : lo) fitted[i] = al + bl * T[i], res[i] = y[i] - fitted[i];
  for (size_t i : hi) fitted[i] = ah + bh * T[i], res[i] = y[i] - fitted[i];
  for (size_t i : lo) fit->rss += res[i] * res[i];
  for (size_t i : hi) fit->rss += res[i] * res[i];
  std::vector<size_t> used(lo);
  used.insert(used.end(), hi.begin(), hi.end());
  std::mt19937_64 rng(12345);
  const PickIndex pick(used.size());
  std::vector<double> tgs;
  for (int b = 0; b < 400; ++b) {
    std::vector<double> yb = yv;
    for (size_t i : used) yb[i] = fitted[i] + res[used[pick(rng)]];
    double t2, b1, b2, a1, a2;
    cross_at(yb, t2, b1, b2, a1, a2);
    if (b1 != b2 && std::isfinite(t2)) tgs.push_back(t2);
  }
  if (tgs.size() > 10) {
    const double m = std::accumulate(tgs.begin(), tgs.end(), 0.0) / double(tgs.size());
    double v = 0;
    for (double x : tgs) v += (x - m) * (x - m);
    fit->tg_err = std::sqrt(v / double(tgs.size() - 1));
  }
  if (lo.size() < 3 || hi.size() < 3) {   // two points fix a line exactly: nothing for the bootstrap to resample
    fit->tg_err = std::numeric_limits<double>::quiet_NaN();
    set_note(fit, "a range with two temperatures fixes its line exactly: no error estimate — use at least three per range");
  }
  if (tg < glassy_max || tg > rubbery_min) {
    fit->ok = 0;
    set_note(fit, "the lines cross at " + fmt4(tg) + " K, outside the gap between the ranges (" + fmt4(glassy_max) + "–" + fmt4(rubbery_min) +
                      " K): no Tg — longer holds, a wider scan or other ranges");
  }
}

}  // namespace

extern "C" int32_t caps_gpu_fit_tg(const double* T, const double* y, int32_t n, int32_t method, double glassy_max, double rubbery_min,
                                   caps_gpu_tg_fit* out) {
  if (!out) return CAPS_GPU_EINVAL;
  std::memset(out, 0, sizeof *out);
  if (n < 0 || (n > 0 && (!T || !y)) || (method != 0 && method != 1)) {
    g_fit_err = "caps_gpu_fit_tg: bad arguments";
    return CAPS_GPU_EINVAL;
  }
  if (method == 0) fit_bilinear(T, y, size_t(n), out);
  else fit_two_ranges(T, y, size_t(n), glassy_max, rubbery_min, out);
  return CAPS_GPU_OK;
}
