// ORACLE / TEST INFRASTRUCTURE — not part of the product path.
//
// A C++ restatement of CAPS's Fortran k-space module (core/fortran/caps_kspace.f90), which cannot be compiled in this
// environment (no Fortran compiler). It provides the 14 bind(C) entry points that core/src/kspace.cpp declares
// (kspace.cpp:11-31), so the reference's own C++ core links and runs unmodified on top of it. Each routine follows the
// Fortran one step by step, keeping its column-major layouts:
//   x(3,n) -> x[3*i + d];  th(p,3,n) -> th[a + p*(d + 3*i)];  g(0:k1-1,0:k2-1,0:k3-1) -> g[i + k1*(j + k2*k)];
//   h(3,3) built from cell[9] (C rows a, b, c) so that column c of h is edge vector c.
// Pinned against the reference's own tests (tests/test_kspace.cpp: FFT vs direct DFT, good_size known answers, Madelung
// constant of rock salt, PME vs plain Ewald, threaded half-spectrum PME vs serial PME), run by oracle/Makefile's
// `pin` target and by tests/test_oracle.py.
#include <cmath>
#include <complex>
#include <cstdlib>
#include <vector>

namespace {

constexpr double kPi = 3.14159265358979323846;

struct C {   // complex(c_double_complex) with plain arithmetic
  double re, im;
};
inline C operator+(C a, C b) { return {a.re + b.re, a.im + b.im}; }
inline C operator-(C a, C b) { return {a.re - b.re, a.im - b.im}; }
inline C operator*(C a, C b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline C operator*(C a, double s) { return {a.re * s, a.im * s}; }
inline C operator*(double s, C a) { return {a.re * s, a.im * s}; }
inline C conj(C a) { return {a.re, -a.im}; }

// caps_kspace.f90:23-36
int good_size(int n) {
  int m = n > 1 ? n : 1;
  for (;;) {
    int k = m;
    while (k % 2 == 0) k /= 2;
    while (k % 3 == 0) k /= 3;
    while (k % 5 == 0) k /= 5;
    while (k % 7 == 0) k /= 7;
    if (k == 1) return m;
    ++m;
  }
}

// Butterflies of the mixed-radix decimation-in-time transform (caps_kspace.f90:78-245). f is the output buffer, o
// the offset of this sub-transform, fs the twiddle stride, m the length of each of the p sub-transforms.
void bfly2(C* f, int o, int fs, const C* tw, int m) {   // f90:78-89
  for (int k = 0; k < m; ++k) {
    const C t = f[o + k + m] * tw[k * fs];
    f[o + k + m] = f[o + k] - t;
    f[o + k] = f[o + k] + t;
  }
}

void bfly4(C* f, int o, int fs, const C* tw, int m, int sign) {   // f90:91-116
  for (int k = 0; k < m; ++k) {
    const C s0 = f[o + k + m] * tw[k * fs];
    const C s1 = f[o + k + 2 * m] * tw[2 * k * fs];
    const C s2 = f[o + k + 3 * m] * tw[3 * k * fs];
    const C s5 = f[o + k] - s1;
    f[o + k] = f[o + k] + s1;
    const C s3 = s0 + s2;
    const C s4 = s0 - s2;
    f[o + k + 2 * m] = f[o + k] - s3;
    f[o + k] = f[o + k] + s3;
    const C is4{-s4.im, s4.re};
    if (sign > 0) {
      f[o + k + m] = s5 + is4;
      f[o + k + 3 * m] = s5 - is4;
    } else {
      f[o + k + m] = s5 - is4;
      f[o + k + 3 * m] = s5 + is4;
    }
  }
}

void bfly3(C* f, int o, int fs, const C* tw, int m) {   // f90:118-140
  const C w3 = tw[fs * m];
  const double epi3 = w3.im;
  for (int k = 0; k < m; ++k) {
    const C s1 = f[o + k + m] * tw[k * fs];
    const C s2 = f[o + k + 2 * m] * tw[2 * k * fs];
    const C s3 = s1 + s2;
    C s0 = s1 - s2;
    f[o + k + m] = f[o + k] - 0.5 * s3;
    s0 = s0 * epi3;
    f[o + k] = f[o + k] + s3;
    f[o + k + 2 * m] = f[o + k + m] + C{s0.im, -s0.re};
    f[o + k + m] = f[o + k + m] + C{-s0.im, s0.re};
  }
}

void bfly5(C* f, int o, int fs, const C* tw, int m) {   // f90:142-172
  const C ya = tw[fs * m], yb = tw[2 * fs * m];
  for (int u = 0; u < m; ++u) {
    const C s0 = f[o + u];
    const C s1 = f[o + u + m] * tw[u * fs];
    const C s2 = f[o + u + 2 * m] * tw[2 * u * fs];
    const C s3 = f[o + u + 3 * m] * tw[3 * u * fs];
    const C s4 = f[o + u + 4 * m] * tw[4 * u * fs];
    const C s7 = s1 + s4, s10 = s1 - s4, s8 = s2 + s3, s9 = s2 - s3;
    f[o + u] = s0 + s7 + s8;
    const C s5 = s0 + C{s7.re * ya.re + s8.re * yb.re, s7.im * ya.re + s8.im * yb.re};
    const C s6{s10.im * ya.im + s9.im * yb.im, -(s10.re * ya.im) - s9.re * yb.im};
    f[o + u + m] = s5 - s6;
    f[o + u + 4 * m] = s5 + s6;
    const C s11 = s0 + C{s7.re * yb.re + s8.re * ya.re, s7.im * yb.re + s8.im * ya.re};
    const C s12{-(s10.im * yb.im) + s9.im * ya.im, s10.re * yb.im - s9.re * ya.im};
    f[o + u + 2 * m] = s11 + s12;
    f[o + u + 3 * m] = s11 - s12;
  }
}

void bfly7(C* f, int o, int fs, const C* tw, int m) {   // f90:176-212
  const double c1 = tw[fs * m].re, q1 = tw[fs * m].im;
  const double c2 = tw[2 * fs * m].re, q2 = tw[2 * fs * m].im;
  const double c3 = tw[3 * fs * m].re, q3 = tw[3 * fs * m].im;
  auto rot = [](C t) { return C{-t.im, t.re}; };
  for (int u = 0; u < m; ++u) {
    const C s0 = f[o + u];
    const C s1 = f[o + u + m] * tw[u * fs];
    const C s2 = f[o + u + 2 * m] * tw[2 * u * fs];
    const C s3 = f[o + u + 3 * m] * tw[3 * u * fs];
    const C s4 = f[o + u + 4 * m] * tw[4 * u * fs];
    const C s5 = f[o + u + 5 * m] * tw[5 * u * fs];
    const C s6 = f[o + u + 6 * m] * tw[6 * u * fs];
    const C a1 = s1 + s6, b1 = s1 - s6, a2 = s2 + s5, b2 = s2 - s5, a3 = s3 + s4, b3 = s3 - s4;
    f[o + u] = s0 + a1 + a2 + a3;
    C r = s0 + a1 * c1 + a2 * c2 + a3 * c3;
    C t = b1 * q1 + b2 * q2 + b3 * q3;
    f[o + u + m] = r + rot(t);
    f[o + u + 6 * m] = r - rot(t);
    r = s0 + a1 * c2 + a2 * c3 + a3 * c1;
    t = b1 * q2 - b2 * q3 - b3 * q1;
    f[o + u + 2 * m] = r + rot(t);
    f[o + u + 5 * m] = r - rot(t);
    r = s0 + a1 * c3 + a2 * c1 + a3 * c2;
    t = b1 * q3 - b2 * q1 + b3 * q2;
    f[o + u + 3 * m] = r + rot(t);
    f[o + u + 4 * m] = r - rot(t);
  }
}

void bfly_generic(C* f, int o, int fs, const C* tw, int m, int p, int n) {   // f90:214-245
  std::vector<C> sc(size_t(p > 16 ? p : 16));
  for (int u = 0; u < m; ++u) {
    for (int q1 = 0; q1 < p; ++q1) sc[size_t(q1)] = f[o + u + q1 * m];
    for (int q1 = 0; q1 < p; ++q1) {
      const int k = u + q1 * m;
      C acc = sc[0];
      int idx = 0;
      const int step = fs * k;
      for (int q = 1; q < p; ++q) {
        idx += step;
        if (idx >= n) idx -= n;
        acc = acc + sc[size_t(q)] * tw[idx];
      }
      f[o + k] = acc;
    }
  }
}

// kf_work (f90:45-76): out-of-place recursive transform; pf/mm are 0-based here (lev from 0)
void kf_work(C* out, int ofs, const C* x, int ifs, int fstride, const int* pf, const int* mm, int lev, const C* tw, int n, int sign) {
  const int p = pf[lev], m = mm[lev];
  if (m == 1) {
    for (int j = 0; j < p; ++j) out[ofs + j] = x[ifs + j * fstride];
  } else {
    for (int j = 0; j < p; ++j) kf_work(out, ofs + j * m, x, ifs + j * fstride, fstride * p, pf, mm, lev + 1, tw, n, sign);
  }
  switch (p) {
    case 2: bfly2(out, ofs, fstride, tw, m); break;
    case 4: bfly4(out, ofs, fstride, tw, m, sign); break;
    case 3: bfly3(out, ofs, fstride, tw, m); break;
    case 5: bfly5(out, ofs, fstride, tw, m); break;
    case 7: bfly7(out, ofs, fstride, tw, m); break;
    default: bfly_generic(out, ofs, fstride, tw, m, p, n); break;
  }
}

// factorize (f90:248-270): radices 4 first, then 2, 3, 5, 7, ...
void factorize(int n, int* pf, int* mm, int& nf) {
  int r = n, p = 4;
  nf = 0;
  while (r > 1) {
    while (r % p != 0) {
      if (p == 4) p = 2;
      else if (p == 2) p = 3;
      else p += 2;
      if (p * p > r) p = r;
    }
    r /= p;
    pf[nf] = p;
    mm[nf] = r;
    ++nf;
  }
}

// twiddles (f90:272-279)
void twiddles(int n, int sign, std::vector<C>& tab) {
  tab.resize(size_t(n));
  for (int j = 0; j < n; ++j) tab[size_t(j)] = C{std::cos(2 * kPi * j / n), sign * std::sin(2 * kPi * j / n)};
}

struct Plan {
  int n = 0, nf = 0;
  int pf[32], mm[32];
  std::vector<C> tw;
  Plan(int n_, int sign) : n(n_) {
    twiddles(n, sign, tw);
    factorize(n, pf, mm, nf);
  }
  void run(C* res, const C* line, int sign) const { kf_work(res, 0, line, 0, 1, pf, mm, 0, tw.data(), n, sign); }
};

// fft3d (f90:306-344): in place, one axis at a time
void fft3d(C* g, int k1, int k2, int k3, int sign) {
  const int kmax = std::max(k1, std::max(k2, k3));
  std::vector<C> line(static_cast<size_t>(kmax)), res(static_cast<size_t>(kmax));
  auto at = [&](int i, int j, int k) -> C& { return g[size_t(i) + size_t(k1) * (size_t(j) + size_t(k2) * size_t(k))]; };
  if (k1 > 1) {
    Plan P(k1, sign);
    for (int k = 0; k < k3; ++k)
      for (int j = 0; j < k2; ++j) {
        for (int i = 0; i < k1; ++i) line[size_t(i)] = at(i, j, k);
        P.run(res.data(), line.data(), sign);
        for (int i = 0; i < k1; ++i) at(i, j, k) = res[size_t(i)];
      }
  }
  if (k2 > 1) {
    Plan P(k2, sign);
    for (int k = 0; k < k3; ++k)
      for (int i = 0; i < k1; ++i) {
        for (int j = 0; j < k2; ++j) line[size_t(j)] = at(i, j, k);
        P.run(res.data(), line.data(), sign);
        for (int j = 0; j < k2; ++j) at(i, j, k) = res[size_t(j)];
      }
  }
  if (k3 > 1) {
    Plan P(k3, sign);
    for (int j = 0; j < k2; ++j)
      for (int i = 0; i < k1; ++i) {
        for (int k = 0; k < k3; ++k) line[size_t(k)] = at(i, j, k);
        P.run(res.data(), line.data(), sign);
        for (int k = 0; k < k3; ++k) at(i, j, k) = res[size_t(k)];
      }
  }
}

// cell_inverse (f90:495-511): h(:,c) = edge vector c; hi = h^-1 (rows are the reciprocal vectors, no 2 pi)
struct Cell3 {
  double h[3][3], hi[3][3], vol;
};
Cell3 cell_inverse(const double* cell) {
  Cell3 o;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) o.h[r][c] = cell[r + 3 * c];   // Fortran cell(r+1, c+1) = cell[r + 3c]
  const auto& h = o.h;
  double vol = h[0][0] * (h[1][1] * h[2][2] - h[2][1] * h[1][2]) - h[0][1] * (h[1][0] * h[2][2] - h[2][0] * h[1][2]) +
               h[0][2] * (h[1][0] * h[2][1] - h[2][0] * h[1][1]);
  o.hi[0][0] = (h[1][1] * h[2][2] - h[1][2] * h[2][1]) / vol;
  o.hi[0][1] = (h[0][2] * h[2][1] - h[0][1] * h[2][2]) / vol;
  o.hi[0][2] = (h[0][1] * h[1][2] - h[0][2] * h[1][1]) / vol;
  o.hi[1][0] = (h[1][2] * h[2][0] - h[1][0] * h[2][2]) / vol;
  o.hi[1][1] = (h[0][0] * h[2][2] - h[0][2] * h[2][0]) / vol;
  o.hi[1][2] = (h[0][2] * h[1][0] - h[0][0] * h[1][2]) / vol;
  o.hi[2][0] = (h[1][0] * h[2][1] - h[1][1] * h[2][0]) / vol;
  o.hi[2][1] = (h[0][1] * h[2][0] - h[0][0] * h[2][1]) / vol;
  o.hi[2][2] = (h[0][0] * h[1][1] - h[0][1] * h[1][0]) / vol;
  o.vol = std::fabs(vol);
  return o;
}

// green (f90:518-564): influence function and virial weights at index (a, b, c), Nyquist planes averaged over both signs
void green(int a, int b, int c, const int* k, const double hi[3][3], double vol, double fac, double kcoul, const double* b1, const double* b2,
           const double* b3, double& g, double w[6]) {
  const int idx[3] = {a, b, c};
  int m[3];
  bool nyq[3];
  int nn = 0;
  for (int d = 0; d < 3; ++d) {
    m[d] = idx[d];
    if (m[d] >= (k[d] + 1) / 2) m[d] -= k[d];
    nyq[d] = k[d] % 2 == 0 && 2 * idx[d] == k[d];
    nn += nyq[d];
  }
  const double bm = b1[a] * b2[b] * b3[c];
  const int ns = 1 << nn;
  g = 0;
  for (int q = 0; q < 6; ++q) w[q] = 0;
  for (int s = 0; s < ns; ++s) {
    int sel = 0;
    double mv[3] = {0, 0, 0};
    for (int d = 0; d < 3; ++d) {
      if (nyq[d]) {
        if ((s >> sel) & 1)
          for (int q = 0; q < 3; ++q) mv[q] = mv[q] - m[d] * hi[d][q];
        else
          for (int q = 0; q < 3; ++q) mv[q] = mv[q] + m[d] * hi[d][q];
        ++sel;
      } else {
        for (int q = 0; q < 3; ++q) mv[q] = mv[q] + m[d] * hi[d][q];
      }
    }
    const double m2len = mv[0] * mv[0] + mv[1] * mv[1] + mv[2] * mv[2];
    const double e = kcoul * std::exp(-fac * m2len) / (kPi * vol * m2len * bm);
    const double ss = 2 * (1 + fac * m2len) / m2len;
    g += e;
    w[0] += e * (1 - ss * mv[0] * mv[0]);
    w[1] += e * (1 - ss * mv[1] * mv[1]);
    w[2] += e * (1 - ss * mv[2] * mv[2]);
    w[3] -= e * ss * mv[0] * mv[1];
    w[4] -= e * ss * mv[0] * mv[2];
    w[5] -= e * ss * mv[1] * mv[2];
  }
  g /= ns;
  for (int q = 0; q < 6; ++q) w[q] /= ns;
}

// bspline (f90:568-598): theta(j) = M_p(w + p - j), j = 1..p (0-based here), and its derivative
void bspline(double w, int p, double* theta, double* dtheta) {
  for (int j = 0; j < p; ++j) theta[j] = 0;
  theta[p - 1] = 0;
  theta[1] = w;
  theta[0] = 1 - w;
  for (int k = 3; k <= p - 1; ++k) {
    const double div = 1.0 / (k - 1);
    theta[k - 1] = div * w * theta[k - 2];
    for (int j = 1; j <= k - 2; ++j) theta[k - j - 1] = div * ((w + j) * theta[k - j - 2] + (k - j - w) * theta[k - j - 1]);
    theta[0] = div * (1 - w) * theta[0];
  }
  dtheta[0] = -theta[0];
  for (int j = 2; j <= p; ++j) dtheta[j - 1] = theta[j - 2] - theta[j - 1];
  const double div = 1.0 / (p - 1);
  theta[p - 1] = div * w * theta[p - 2];
  for (int j = 1; j <= p - 2; ++j) theta[p - j - 1] = div * ((w + j) * theta[p - j - 2] + (p - j - w) * theta[p - j - 1]);
  theta[0] = div * (1 - w) * theta[0];
}

// bspline_moduli (f90:601-620)
void bspline_moduli(int k, int p, double* bsp) {
  std::vector<double> arr(static_cast<size_t>(p)), darr(static_cast<size_t>(p));
  bspline(0.0, p, arr.data(), darr.data());
  for (int m = 0; m < k; ++m) {
    double sr = 0, si = 0;
    for (int j = 0; j <= p - 2; ++j) {
      const double arg = 2 * kPi * m * j / double(k);
      sr += arr[size_t(j)] * std::cos(arg);
      si += arr[size_t(j)] * std::sin(arg);
    }
    bsp[m] = sr * sr + si * si;
  }
  for (int m = 0; m < k; ++m)
    if (bsp[m] < 1e-7) bsp[m] = 0.5 * (bsp[((m - 1) % k + k) % k] + bsp[(m + 1) % k]);
}

inline int fmodulo(int a, int p) { return ((a % p) + p) % p; }

// splines of one atom (f90:631-643, 785-795): s = h^-1 x, u = frac(s) K, w = frac(u); idx(a) = modulo(floor(u) - p + a, K)
void atom_splines(const double* xi, const Cell3& cc, const int* grid, int p, double* th, double* dth, int* idx) {
  double s[3];
  for (int r = 0; r < 3; ++r) s[r] = cc.hi[r][0] * xi[0] + cc.hi[r][1] * xi[1] + cc.hi[r][2] * xi[2];
  for (int d = 0; d < 3; ++d) {
    const double u = (s[d] - std::floor(s[d])) * grid[d];
    const double w = u - std::floor(u);
    bspline(w, p, th + p * d, dth + p * d);
    for (int a = 1; a <= p; ++a) idx[p * d + a - 1] = fmodulo(int(std::floor(u)) - p + a, grid[d]);
  }
}

}  // namespace

extern "C" {

int caps_f_good_size(int n) { return good_size(n); }

// caps_f_fft3d (f90:484-493)
void caps_f_fft3d(double* re, double* im, int k1, int k2, int k3, int sign) {
  const size_t n = size_t(k1) * size_t(k2) * size_t(k3);
  std::vector<C> g(n);
  for (size_t i = 0; i < n; ++i) g[i] = C{re[i], im[i]};
  fft3d(g.data(), k1, k2, k3, sign);
  for (size_t i = 0; i < n; ++i) re[i] = g[i].re, im[i] = g[i].im;
}

void caps_f_bspline_moduli(int k, int p, double* bsp) { bspline_moduli(k, p, bsp); }

// caps_f_pme (f90:624-715): serial whole-grid smooth PME
void caps_f_pme(int n, const double* x, const double* q, const double* cell, const int* grid, int p, double beta, double kcoul, double* energy,
                double* f, double* vir) {
  const int k1 = grid[0], k2 = grid[1], k3 = grid[2];
  const Cell3 cc = cell_inverse(cell);
  std::vector<double> th(size_t(p) * 3 * size_t(n)), dth(th.size());
  std::vector<int> idx(th.size());
  for (int i = 0; i < n; ++i) atom_splines(x + 3 * i, cc, grid, p, &th[size_t(3 * p) * i], &dth[size_t(3 * p) * i], &idx[size_t(3 * p) * i]);
  const size_t G = size_t(k1) * size_t(k2) * size_t(k3);
  std::vector<C> g(G, C{0, 0});
  auto gi = [&](int a, int b, int c) { return size_t(a) + size_t(k1) * (size_t(b) + size_t(k2) * size_t(c)); };
  for (int i = 0; i < n; ++i) {
    const double* T = &th[size_t(3 * p) * i];
    const int* I = &idx[size_t(3 * p) * i];
    for (int c = 0; c < p; ++c) {
      const int ic = I[2 * p + c];
      for (int b = 0; b < p; ++b) {
        const int ib = I[p + b];
        const double st = q[i] * T[p + b] * T[2 * p + c];
        for (int a = 0; a < p; ++a) {
          const int ia = I[a];
          g[gi(ia, ib, ic)].re += st * T[a];
        }
      }
    }
  }
  fft3d(g.data(), k1, k2, k3, +1);
  std::vector<double> b1(static_cast<size_t>(k1)), b2(static_cast<size_t>(k2)), b3(static_cast<size_t>(k3));
  bspline_moduli(k1, p, b1.data());
  bspline_moduli(k2, p, b2.data());
  bspline_moduli(k3, p, b3.data());
  double e = 0, wsum[6] = {0, 0, 0, 0, 0, 0};
  const double fac = kPi * kPi / (beta * beta);
  for (int c = 0; c < k3; ++c)
    for (int b = 0; b < k2; ++b)
      for (int a = 0; a < k1; ++a) {
        C& v = g[gi(a, b, c)];
        if (a == 0 && b == 0 && c == 0) {
          v = C{0, 0};
          continue;
        }
        double eterm, wv[6];
        green(a, b, c, grid, cc.hi, cc.vol, fac, kcoul, b1.data(), b2.data(), b3.data(), eterm, wv);
        const double e_m = 0.5 * (v.re * v.re + v.im * v.im);
        e += e_m * eterm;
        for (int q6 = 0; q6 < 6; ++q6) wsum[q6] += e_m * wv[q6];
        v = v * eterm;
      }
  fft3d(g.data(), k1, k2, k3, -1);
  for (int i = 0; i < n; ++i) {
    const double* T = &th[size_t(3 * p) * i];
    const double* D = &dth[size_t(3 * p) * i];
    const int* I = &idx[size_t(3 * p) * i];
    double gs[3] = {0, 0, 0};
    for (int c = 0; c < p; ++c) {
      const int ic = I[2 * p + c];
      for (int b = 0; b < p; ++b) {
        const int ib = I[p + b];
        for (int a = 0; a < p; ++a) {
          const int ia = I[a];
          const double st = g[gi(ia, ib, ic)].re;
          gs[0] += D[a] * T[p + b] * T[2 * p + c] * st;
          gs[1] += T[a] * D[p + b] * T[2 * p + c] * st;
          gs[2] += T[a] * T[p + b] * D[2 * p + c] * st;
        }
      }
    }
    for (int r = 0; r < 3; ++r) {
      const double grad = grid[0] * gs[0] * cc.hi[0][r] + grid[1] * gs[1] * cc.hi[1][r] + grid[2] * gs[2] * cc.hi[2][r];
      f[3 * i + r] -= q[i] * grad;
    }
  }
  *energy = e;
  for (int q6 = 0; q6 < 6; ++q6) vir[q6] = wsum[q6];
}

// caps_f_ewald (f90:718-764): the plain Ewald reciprocal sum over |m_d| <= kmax(d)
void caps_f_ewald(int n, const double* x, const double* q, const double* cell, const int* kmax, double beta, double kcoul, double* energy,
                  double* f, double* vir) {
  const Cell3 cc = cell_inverse(cell);
  double e = 0, w[6] = {0, 0, 0, 0, 0, 0};
  const double fac = kPi * kPi / (beta * beta);
  for (int m1 = -kmax[0]; m1 <= kmax[0]; ++m1)
    for (int m2 = -kmax[1]; m2 <= kmax[1]; ++m2)
      for (int m3 = -kmax[2]; m3 <= kmax[2]; ++m3) {
        if (m1 == 0 && m2 == 0 && m3 == 0) continue;
        double mv[3];
        for (int r = 0; r < 3; ++r) mv[r] = m1 * cc.hi[0][r] + m2 * cc.hi[1][r] + m3 * cc.hi[2][r];
        const double m2len = mv[0] * mv[0] + mv[1] * mv[1] + mv[2] * mv[2];
        const double a = kcoul * std::exp(-fac * m2len) / (2 * kPi * cc.vol * m2len);
        double sr = 0, si = 0;
        for (int i = 0; i < n; ++i) {
          const double arg = 2 * kPi * (mv[0] * x[3 * i] + mv[1] * x[3 * i + 1] + mv[2] * x[3 * i + 2]);
          sr += q[i] * std::cos(arg);
          si += q[i] * std::sin(arg);
        }
        const double e_m = a * (sr * sr + si * si);
        e += e_m;
        const double ss = 2 * (1 + fac * m2len) / m2len;
        w[0] += e_m * (1 - ss * mv[0] * mv[0]);
        w[1] += e_m * (1 - ss * mv[1] * mv[1]);
        w[2] += e_m * (1 - ss * mv[2] * mv[2]);
        w[3] -= e_m * ss * mv[0] * mv[1];
        w[4] -= e_m * ss * mv[0] * mv[2];
        w[5] -= e_m * ss * mv[1] * mv[2];
        for (int i = 0; i < n; ++i) {
          const double arg = 2 * kPi * (mv[0] * x[3 * i] + mv[1] * x[3 * i + 1] + mv[2] * x[3 * i + 2]);
          const double cs = std::cos(arg), sn = std::sin(arg);
          for (int r = 0; r < 3; ++r) f[3 * i + r] += 4 * kPi * a * q[i] * mv[r] * (sr * sn - si * cs);
        }
      }
  *energy = e;
  for (int q6 = 0; q6 < 6; ++q6) vir[q6] = w[q6];
}

// caps_f_pme_splines (f90:776-796): atoms [first, last)
void caps_f_pme_splines(int n, const double* x, const double* cell, const int* grid, int p, double* th, double* dth, int* idx, int first, int last) {
  (void)n;
  const Cell3 cc = cell_inverse(cell);
  for (int i = first; i < last; ++i) atom_splines(x + 3 * i, cc, grid, p, th + size_t(3 * p) * i, dth + size_t(3 * p) * i, idx + size_t(3 * p) * i);
}

// caps_f_pme_spread_planes (f90:800-822): planes [first, last) of the third axis, zeroed first, atoms in index order
void caps_f_pme_spread_planes(int n, const double* q, const int* grid, int p, double* g, const double* th, const int* idx, int first, int last) {
  const size_t k1 = size_t(grid[0]), k2 = size_t(grid[1]);
  for (int c = first; c < last; ++c)
    for (size_t t = 0; t < k1 * k2; ++t) g[t + k1 * k2 * size_t(c)] = 0.0;
  for (int i = 0; i < n; ++i) {
    const double* T = th + size_t(3 * p) * i;
    const int* I = idx + size_t(3 * p) * i;
    for (int c = 0; c < p; ++c) {
      const int ic = I[2 * p + c];
      if (ic < first || ic >= last) continue;
      for (int b = 0; b < p; ++b) {
        const double st = q[i] * T[p + b] * T[2 * p + c];
        for (int a = 0; a < p; ++a) {
          const size_t at = size_t(I[a]) + k1 * (size_t(I[p + b]) + k2 * size_t(ic));
          g[at] = g[at] + st * T[a];
        }
      }
    }
  }
}

// caps_f_r2c_lines / r2c_lines (f90:392-423, 859-864): pairs of real lines [first, last) through one complex FFT
void caps_f_r2c_lines(const double* r, std::complex<double>* hout, int k1, int k2, int k3, int first, int last) {
  C* h = reinterpret_cast<C*>(hout);
  const int nl = k2 * k3, h1 = k1 / 2 + 1;
  Plan P(k1, 1);
  std::vector<C> z(static_cast<size_t>(k1)), zz(static_cast<size_t>(k1));
  for (int l = first; l < last; ++l) {
    const int la = 2 * l, lb = std::min(2 * l + 1, nl - 1);
    for (int i = 0; i < k1; ++i) z[size_t(i)] = C{r[size_t(i) + size_t(k1) * la], lb == la ? 0.0 : r[size_t(i) + size_t(k1) * lb]};
    if (k1 > 1) P.run(zz.data(), z.data(), 1);
    else zz = z;
    for (int m = 0; m <= k1 / 2; ++m) {
      const C zm = zz[size_t(m)];
      const C zc = conj(zz[size_t(fmodulo(k1 - m, k1))]);
      h[size_t(m) + size_t(h1) * la] = 0.5 * (zm + zc);
      if (lb != la) {
        const C dz = zm - zc;
        h[size_t(m) + size_t(h1) * lb] = 0.5 * C{dz.im, -dz.re};
      }
    }
  }
}

// caps_f_c2r_lines / c2r_lines (f90:427-461, 866-871)
void caps_f_c2r_lines(const std::complex<double>* hin, double* r, int k1, int k2, int k3, int first, int last) {
  const C* h = reinterpret_cast<const C*>(hin);
  const int nl = k2 * k3, h1 = k1 / 2 + 1;
  Plan P(k1, -1);
  std::vector<C> z(static_cast<size_t>(k1)), zz(static_cast<size_t>(k1));
  for (int l = first; l < last; ++l) {
    const int la = 2 * l, lb = std::min(2 * l + 1, nl - 1);
    for (int m = 0; m < k1; ++m) {
      int mh = m;
      if (m > k1 / 2) mh = k1 - m;
      C a = h[size_t(mh) + size_t(h1) * la];
      C b{0, 0};
      if (lb != la) b = h[size_t(mh) + size_t(h1) * lb];
      if (m > k1 / 2) {
        a = conj(a);
        b = conj(b);
      }
      z[size_t(m)] = a + C{-b.im, b.re};
    }
    if (k1 > 1) P.run(zz.data(), z.data(), -1);
    else zz = z;
    for (int i = 0; i < k1; ++i) {
      r[size_t(i) + size_t(k1) * la] = zz[size_t(i)].re;
      if (lb != la) r[size_t(i) + size_t(k1) * lb] = zz[size_t(i)].im;
    }
  }
}

// caps_f_fft_lines / fft_lines (f90:348-387, 873-877)
void caps_f_fft_lines(std::complex<double>* gin, int k1, int k2, int k3, int axis, int sign, int first, int last) {
  C* g = reinterpret_cast<C*>(gin);
  const int n = axis == 1 ? k1 : axis == 2 ? k2 : k3;
  if (n <= 1) return;
  Plan P(n, sign);
  std::vector<C> line(static_cast<size_t>(n)), res(static_cast<size_t>(n));
  auto at = [&](int i, int j, int k) -> C& { return g[size_t(i) + size_t(k1) * (size_t(j) + size_t(k2) * size_t(k))]; };
  for (int l = first; l < last; ++l) {
    int i = 0, j = 0, k = 0;
    if (axis == 1) { j = l % k2; k = l / k2; for (int t = 0; t < n; ++t) line[size_t(t)] = at(t, j, k); }
    else if (axis == 2) { i = l % k1; k = l / k1; for (int t = 0; t < n; ++t) line[size_t(t)] = at(i, t, k); }
    else { i = l % k1; j = l / k1; for (int t = 0; t < n; ++t) line[size_t(t)] = at(i, j, t); }
    P.run(res.data(), line.data(), sign);
    if (axis == 1) for (int t = 0; t < n; ++t) at(t, j, k) = res[size_t(t)];
    else if (axis == 2) for (int t = 0; t < n; ++t) at(i, t, k) = res[size_t(t)];
    else for (int t = 0; t < n; ++t) at(i, j, t) = res[size_t(t)];
  }
}

// caps_f_pme_influence (f90:882-912): half spectrum, G applied in place, energy and virial of planes [first, last)
void caps_f_pme_influence(std::complex<double>* gin, const int* grid, const double* cell, const double* b1, const double* b2, const double* b3,
                          double beta, double kcoul, int first, int last, double* energy, double* vir) {
  C* g = reinterpret_cast<C*>(gin);
  const int k1 = grid[0], h1 = k1 / 2 + 1;
  const Cell3 cc = cell_inverse(cell);
  const double fac = kPi * kPi / (beta * beta);
  for (int c = first; c < last; ++c)
    for (int b = 0; b < grid[1]; ++b)
      for (int a = 0; a <= k1 / 2; ++a) {
        C& v = g[size_t(a) + size_t(h1) * (size_t(b) + size_t(grid[1]) * size_t(c))];
        if (a == 0 && b == 0 && c == 0) {
          v = C{0, 0};
          continue;
        }
        double eterm, wv[6];
        green(a, b, c, grid, cc.hi, cc.vol, fac, kcoul, b1, b2, b3, eterm, wv);
        double e_m = 0.5 * (v.re * v.re + v.im * v.im);
        if (a > 0 && 2 * a != k1) e_m = 2 * e_m;
        *energy += e_m * eterm;
        for (int q6 = 0; q6 < 6; ++q6) vir[q6] += e_m * wv[q6];
        v = v * eterm;
      }
}

// caps_f_pme_green (f90:916-940)
void caps_f_pme_green(const int* grid, const double* cell, const double* b1, const double* b2, const double* b3, double beta, double kcoul, int first,
                      int last, double* gt, double* wt) {
  const int k1 = grid[0], h1 = k1 / 2 + 1;
  const Cell3 cc = cell_inverse(cell);
  const double fac = kPi * kPi / (beta * beta);
  for (int c = first; c < last; ++c)
    for (int b = 0; b < grid[1]; ++b)
      for (int a = 0; a <= k1 / 2; ++a) {
        const size_t t = size_t(a) + size_t(h1) * (size_t(b) + size_t(grid[1]) * size_t(c));
        if (a == 0 && b == 0 && c == 0) {
          gt[t] = 0;
          for (int q6 = 0; q6 < 6; ++q6) wt[6 * t + q6] = 0;
          continue;
        }
        green(a, b, c, grid, cc.hi, cc.vol, fac, kcoul, b1, b2, b3, gt[t], &wt[6 * t]);
      }
}

// caps_f_pme_apply (f90:943-962)
void caps_f_pme_apply(std::complex<double>* gin, const int* grid, const double* gt, const double* wt, int first, int last, double* energy, double* vir) {
  C* g = reinterpret_cast<C*>(gin);
  const int k1 = grid[0], h1 = k1 / 2 + 1;
  for (int c = first; c < last; ++c)
    for (int b = 0; b < grid[1]; ++b)
      for (int a = 0; a <= k1 / 2; ++a) {
        const size_t t = size_t(a) + size_t(h1) * (size_t(b) + size_t(grid[1]) * size_t(c));
        C& v = g[t];
        double e_m = 0.5 * (v.re * v.re + v.im * v.im);
        if (a > 0 && 2 * a != k1) e_m = 2 * e_m;
        *energy += e_m * gt[t];
        for (int q6 = 0; q6 < 6; ++q6) vir[q6] += e_m * wt[6 * t + q6];
        v = v * gt[t];
      }
}

// caps_f_pme_gather (f90:965-992): atoms [first, last)
void caps_f_pme_gather(int n, const double* q, const double* cell, const int* grid, int p, const double* g, const double* th, const double* dth,
                       const int* idx, int first, int last, double* f) {
  (void)n;
  const Cell3 cc = cell_inverse(cell);
  const size_t k1 = size_t(grid[0]), k2 = size_t(grid[1]);
  for (int i = first; i < last; ++i) {
    const double* T = th + size_t(3 * p) * i;
    const double* D = dth + size_t(3 * p) * i;
    const int* I = idx + size_t(3 * p) * i;
    double gs[3] = {0, 0, 0};
    for (int c = 0; c < p; ++c) {
      const double tc = T[2 * p + c], dc = D[2 * p + c];
      for (int b = 0; b < p; ++b) {
        const double tb = T[p + b], db = D[p + b];
        for (int a = 0; a < p; ++a) {
          const double st = g[size_t(I[a]) + k1 * (size_t(I[p + b]) + k2 * size_t(I[2 * p + c]))];
          gs[0] += D[a] * tb * tc * st;
          gs[1] += T[a] * db * tc * st;
          gs[2] += T[a] * tb * dc * st;
        }
      }
    }
    for (int r = 0; r < 3; ++r) {
      const double grad = grid[0] * gs[0] * cc.hi[0][r] + grid[1] * gs[1] * cc.hi[1][r] + grid[2] * gs[2] * cc.hi[2][r];
      f[3 * i + r] -= q[i] * grad;
    }
  }
}

}  // extern "C"
