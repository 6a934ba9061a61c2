// PME on the device: order-p cardinal B-spline spreading, the 3-D FFT of the real charge grid (half spectrum along
// the first axis), the influence function with energy and virial, the inverse transform and the force gather.
// Reference: core/src/kspace.cpp:80-175 (the stage pipeline) over core/fortran/caps_kspace.f90: bspline :568-598,
// splines and grid indices :776-796, spreading :800-822, the half-spectrum influence function with Nyquist averaging
// (green :518-564, applied with e_m doubled for interior m1 at :943-962), gather :965-992. The grid layout and index
// convention are the reference's: g(a, b, c) at a + K1 (b + K2 c), and theta(a) weighs grid point floor(u) - p + a.
//
// Precision: the FP64 path is double throughout. The mixed path spreads in FP32 arithmetic into an exact fixed-point
// grid, runs the transforms and the influence function in FP64 (a 70^3 grid is a few MB: the FFT is a small share of the
// step, and FP32 transforms measured 1.3e-5 RMS relative force error on a relaxed cell against the 5e-6 target), and
// gathers in FP32 arithmetic.
//
// Kernels: K-SPREAD (thread per atom, fixed-point atomics on the FP32 path: deterministic), K-FFT-X (real lines to half
// spectra), K-FFT-Y, K-FFT-Z+SOLVE (forward z transform, G multiply with energy/virial, inverse z transform, fused in one
// pass over the grid), K-FFT-Y inverse, K-FFT-X inverse (half spectra to real lines), K-GATHER. Each line transform is a
// Stockham autosort FFT in shared memory (radix 2, 3, 4, 5, 7 butterflies unrolled in registers), twiddles staged from
// host-computed tables into shared memory.
#pragma once
#include "pme_types.cuh"

namespace capsb {

// One radix-RAD Stockham pass over `nl` lines of length n, line-major, from `in` to `out`; Ns = product of the radices
// before this pass. tw is the plan's twiddle table staged in shared memory. Every index stays below n: r k stride <=
// (RAD-1)(Ns-1) n / (Ns RAD) < n. Butterflies are unrolled in registers; the small-radix DFT constants W_RAD^e = tw[e n/RAD].
template <class T, int RAD>
__device__ __forceinline__ void stockham_pass(const T* __restrict__ in, T* __restrict__ out, const T* __restrict__ tw, int n, int Ns, int nl,
                                              int sign) {
  using R = decltype(T::x);
  const int nb = n / RAD, stride = n / (Ns * RAD);
  T w[RAD];
#pragma unroll
  for (int e = 0; e < RAD; ++e) w[e] = tw[e * nb];
  for (int t = threadIdx.x; t < nl * nb; t += blockDim.x) {
    const int l = t / nb, j = t - l * nb;
    const int k = j % Ns;
    const T* src = in + l * n;
    T v[RAD];
    v[0] = src[j];
#pragma unroll
    for (int r = 1; r < RAD; ++r) v[r] = cmul(src[j + r * nb], tw[r * k * stride]);
    T o[RAD];
    if constexpr (RAD == 2) {
      o[0] = cadd(v[0], v[1]);
      o[1] = csub(v[0], v[1]);
    } else if constexpr (RAD == 4) {
      const T s0 = cadd(v[0], v[2]), s1 = csub(v[0], v[2]), s2 = cadd(v[1], v[3]), s3 = csub(v[1], v[3]);
      const T is3 = {R(-sign) * s3.y, R(sign) * s3.x};   // sign * i * s3
      o[0] = cadd(s0, s2);
      o[2] = csub(s0, s2);
      o[1] = cadd(s1, is3);
      o[3] = csub(s1, is3);
    } else {
#pragma unroll
      for (int m = 0; m < RAD; ++m) {
        T acc = v[0];
#pragma unroll
        for (int r = 1; r < RAD; ++r) acc = cadd(acc, cmul(v[r], w[(m * r) % RAD]));
        o[m] = acc;
      }
    }
    T* dst = out + l * n + (j - k) * RAD + k;   // (j / Ns) Ns RAD + k
#pragma unroll
    for (int r = 0; r < RAD; ++r) dst[r * Ns] = o[r];
  }
}

// All passes of a plan over `nl` lines held line-major in a (scratch b; tw in shared memory). Returns the buffer holding
// the result (a or b). The plans hold radices 2, 3, 4, 5 and 7 only (grid lengths are 2^a 3^b 5^c 7^d).
template <class R>
__device__ typename Cpx<R>::T* fft_lines_smem(typename Cpx<R>::T* a, typename Cpx<R>::T* b, const typename Cpx<R>::T* tw, int nl,
                                              const FftPlan<R>& P) {
  using T = typename Cpx<R>::T;
  int Ns = 1;
  T* in = a;
  T* out = b;
  for (int s = 0; s < P.nst; ++s) {
    const int Rr = P.rad[s];
    switch (Rr) {
      case 2: stockham_pass<T, 2>(in, out, tw, P.n, Ns, nl, P.sign); break;
      case 3: stockham_pass<T, 3>(in, out, tw, P.n, Ns, nl, P.sign); break;
      case 4: stockham_pass<T, 4>(in, out, tw, P.n, Ns, nl, P.sign); break;
      case 5: stockham_pass<T, 5>(in, out, tw, P.n, Ns, nl, P.sign); break;
      default: stockham_pass<T, 7>(in, out, tw, P.n, Ns, nl, P.sign); break;
    }
    __syncthreads();
    T* tmp = in;
    in = out;
    out = tmp;
    Ns *= Rr;
  }
  return in;
}

template <class T>
__device__ __forceinline__ void stage_twiddles(T* dst, const T* __restrict__ src, int n) {
  for (int t = threadIdx.x; t < n; t += blockDim.x) dst[t] = src[t];
}

// Cardinal B-spline weights of order P at fractional offset w (caps_kspace.f90:568-598), 0-based: th[j] weighs grid
// point floor(u) - P + 1 + j.
template <class R, int P>
__device__ __forceinline__ void bspline(R w, R th[P], R dth[P]) {
#pragma unroll
  for (int j = 0; j < P; ++j) th[j] = 0;
  th[1] = w;
  th[0] = 1 - w;
#pragma unroll
  for (int k = 3; k <= P - 1; ++k) {
    const R div = R(1) / R(k - 1);
    th[k - 1] = div * w * th[k - 2];
#pragma unroll
    for (int j = 1; j <= k - 2; ++j) th[k - j - 1] = div * ((w + R(j)) * th[k - j - 2] + (R(k - j) - w) * th[k - j - 1]);
    th[0] = div * (1 - w) * th[0];
  }
  dth[0] = -th[0];
#pragma unroll
  for (int j = 2; j <= P; ++j) dth[j - 1] = th[j - 2] - th[j - 1];
  const R div = R(1) / R(P - 1);
  th[P - 1] = div * w * th[P - 2];
#pragma unroll
  for (int j = 1; j <= P - 2; ++j) th[P - j - 1] = div * ((w + R(j)) * th[P - j - 2] + (R(P - j) - w) * th[P - j - 1]);
  th[0] = div * (1 - w) * th[0];
}

struct PmeArgs {
  int k1, k2, k3, h1;
  DevCell cell;
  const double* x;
  const double* q;
  int n;
};

// fractional coordinates as the Fortran takes them: s = h^-1 x (no origin), u = frac(s) K, w = frac(u)
template <class R, int P>
__device__ __forceinline__ void atom_splines(const PmeArgs& A, int i, R th[3][P], R dth[3][P], int base[3]) {
  const double xi[3] = {A.x[3 * i], A.x[3 * i + 1], A.x[3 * i + 2]};
  const int K[3] = {A.k1, A.k2, A.k3};
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double s = A.cell.hi[d][0] * xi[0] + A.cell.hi[d][1] * xi[1] + A.cell.hi[d][2] * xi[2];
    const double u = (s - floor(s)) * K[d];
    const double fu = floor(u);
    bspline<R, P>(R(u - fu), th[d], dth[d]);
    base[d] = int(fu) - P + 1;
  }
}

__device__ __forceinline__ int wrapk(int v, int K) {
  v %= K;
  return v < 0 ? v + K : v;
}

// K-SPREAD. FP64: double atomics into g. FP32: fixed point (2^40 per e) into gq, exact and order-free.
template <class R, int P>
static __global__ void k_spread(PmeArgs A, double* __restrict__ g, long long* __restrict__ gq) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.n) return;
  const double qi = A.q[i];
  if (qi == 0) return;
  R th[3][P], dth[3][P];
  int base[3];
  atom_splines<R, P>(A, i, th, dth, base);
  int ia[P], ib[P];
#pragma unroll
  for (int a = 0; a < P; ++a) ia[a] = wrapk(base[0] + a, A.k1), ib[a] = wrapk(base[1] + a, A.k2);
  for (int c = 0; c < P; ++c) {
    const int ic = wrapk(base[2] + c, A.k3);
#pragma unroll
    for (int b = 0; b < P; ++b) {
      const R st = R(qi) * th[1][b] * th[2][c];
      const size_t row = size_t(A.k1) * (size_t(ib[b]) + size_t(A.k2) * size_t(ic));
#pragma unroll
      for (int a = 0; a < P; ++a) {
        const R v = st * th[0][a];
        if (sizeof(R) == 8) atomicAdd(g + row + ia[a], double(v));
        else atomic_add_fix(gq + row + ia[a], to_fix(double(v), kFixQ));
      }
    }
  }
}

// Shared memory of the line-transform kernels: the twiddle table(s), then two buffers of `lines` lines of length n.
// K-FFT-X forward: real lines (b, c) of length K1 to half spectra h(a, b, c), a <= K1/2. Input: g (double) or gq (fixed).
template <class R>
static __global__ void __launch_bounds__(128) k_fft_x_fwd(PmeArgs A, const double* __restrict__ g, const long long* __restrict__ gq,
                                                          typename Cpx<R>::T* __restrict__ h, FftPlan<R> P, int lines_per_block) {
  using T = typename Cpx<R>::T;
  extern __shared__ unsigned char smem_raw[];
  T* tw = reinterpret_cast<T*>(smem_raw);
  T* s0 = tw + A.k1;
  T* s1 = s0 + lines_per_block * A.k1;
  const int nlines = A.k2 * A.k3;
  stage_twiddles(tw, P.tw, A.k1);
  // groups of lines_per_block lines, strided over the grid (the grid may be smaller than the group count)
  for (int l0 = blockIdx.x * lines_per_block; l0 < nlines; l0 += gridDim.x * lines_per_block) {
    const int nl = min(lines_per_block, nlines - l0);
    for (int t = threadIdx.x; t < nl * A.k1; t += blockDim.x) {
      const size_t gidx = size_t(l0) * A.k1 + t;   // lines are contiguous in the real grid
      const R v = gq ? R(double(gq[gidx]) * kInvFixQ) : R(g[gidx]);
      s0[t] = {v, R(0)};
    }
    __syncthreads();
    const T* res = fft_lines_smem<R>(s0, s1, tw, nl, P);
    for (int t = threadIdx.x; t < nl * A.h1; t += blockDim.x) {
      const int l = t / A.h1, a = t - l * A.h1;
      h[size_t(l0 + l) * A.h1 + a] = res[l * A.k1 + a];
    }
    __syncthreads();
  }
}

// K-FFT-X inverse: half spectra back to real lines (the missing half by Hermitian symmetry), real part kept.
template <class R>
static __global__ void __launch_bounds__(128) k_fft_x_inv(PmeArgs A, const typename Cpx<R>::T* __restrict__ h, R* __restrict__ gr, FftPlan<R> P,
                                                          int lines_per_block) {
  using T = typename Cpx<R>::T;
  extern __shared__ unsigned char smem_raw[];
  T* tw = reinterpret_cast<T*>(smem_raw);
  T* s0 = tw + A.k1;
  T* s1 = s0 + lines_per_block * A.k1;
  const int nlines = A.k2 * A.k3;
  stage_twiddles(tw, P.tw, A.k1);
  for (int l0 = blockIdx.x * lines_per_block; l0 < nlines; l0 += gridDim.x * lines_per_block) {
    const int nl = min(lines_per_block, nlines - l0);
    for (int t = threadIdx.x; t < nl * A.k1; t += blockDim.x) {
      const int l = t / A.k1, m = t - l * A.k1;
      const size_t lb = size_t(l0 + l) * A.h1;
      T v;
      if (m <= A.k1 / 2) v = h[lb + m];
      else {
        const T c = h[lb + (A.k1 - m)];
        v = {c.x, -c.y};
      }
      s0[t] = v;
    }
    __syncthreads();
    const T* res = fft_lines_smem<R>(s0, s1, tw, nl, P);
    for (int t = threadIdx.x; t < nl * A.k1; t += blockDim.x) gr[size_t(l0) * A.k1 + t] = res[t].x;
    __syncthreads();
  }
}

// K-FFT-Y: lines along b for fixed (a, c); a block takes `la` consecutive a (coalesced rows) of one c.
template <class R>
static __global__ void __launch_bounds__(128) k_fft_y(PmeArgs A, typename Cpx<R>::T* __restrict__ h, FftPlan<R> P, int la) {
  using T = typename Cpx<R>::T;
  extern __shared__ unsigned char smem_raw[];
  T* tw = reinterpret_cast<T*>(smem_raw);
  T* s0 = tw + A.k2;
  T* s1 = s0 + la * A.k2;
  const int ngrp = (A.h1 + la - 1) / la;
  stage_twiddles(tw, P.tw, A.k2);
  for (int grp = blockIdx.x; grp < ngrp * A.k3; grp += gridDim.x) {
    const int c = grp / ngrp, a0 = (grp % ngrp) * la;
    const int nl = min(la, A.h1 - a0);
    for (int t = threadIdx.x; t < nl * A.k2; t += blockDim.x) {
      const int b = t / nl, al = t - b * nl;
      s0[al * A.k2 + b] = h[size_t(a0 + al) + size_t(A.h1) * (size_t(b) + size_t(A.k2) * c)];
    }
    __syncthreads();
    const T* res = fft_lines_smem<R>(s0, s1, tw, nl, P);
    for (int t = threadIdx.x; t < nl * A.k2; t += blockDim.x) {
      const int b = t / nl, al = t - b * nl;
      h[size_t(a0 + al) + size_t(A.h1) * (size_t(b) + size_t(A.k2) * c)] = res[al * A.k2 + b];
    }
    __syncthreads();
  }
}

// K-FFT-Z+SOLVE: lines along c for fixed (a, b): forward transform, energy and virial of the half spectrum (e_m doubled
// for 0 < a < K1/2), multiply by G, inverse transform, in one pass.
template <class R, bool ENER, bool VIR>
static __global__ void __launch_bounds__(128) k_fft_z_solve(PmeArgs A, typename Cpx<R>::T* __restrict__ h, const R* __restrict__ gt,
                                                            const R* __restrict__ wt, FftPlan<R> Pf, FftPlan<R> Pi, int la, EnergySink en,
                                                            int fixed) {
  using T = typename Cpx<R>::T;
  extern __shared__ unsigned char smem_raw[];
  T* twf = reinterpret_cast<T*>(smem_raw);
  T* twi = twf + A.k3;
  T* s0 = twi + A.k3;
  T* s1 = s0 + la * A.k3;
  const int ngrp = (A.h1 + la - 1) / la;
  const size_t plane = size_t(A.h1) * A.k2;
  stage_twiddles(twf, Pf.tw, A.k3);
  stage_twiddles(twi, Pi.tw, A.k3);
  double e = 0, w[6] = {0, 0, 0, 0, 0, 0};
  long long ef = 0, wf[6] = {0, 0, 0, 0, 0, 0};
  for (int grp = blockIdx.x; grp < ngrp * A.k2; grp += gridDim.x) {
    const int b = grp / ngrp, a0 = (grp % ngrp) * la;
    const int nl = min(la, A.h1 - a0);
    for (int t = threadIdx.x; t < nl * A.k3; t += blockDim.x) {
      const int c = t / nl, al = t - c * nl;
      s0[al * A.k3 + c] = h[size_t(a0 + al) + size_t(A.h1) * b + plane * c];
    }
    __syncthreads();
    T* res = fft_lines_smem<R>(s0, s1, twf, nl, Pf);
    T* other = res == s0 ? s1 : s0;
    for (int t = threadIdx.x; t < nl * A.k3; t += blockDim.x) {
      const int al = t / A.k3, c = t - al * A.k3;
      const int a = a0 + al;
      const size_t gi = size_t(a) + size_t(A.h1) * b + plane * c;
      T v = res[t];
      const R G = gt[gi];
      if (ENER || VIR) {
        double em = 0.5 * (double(v.x) * v.x + double(v.y) * v.y);
        if (a > 0 && 2 * a != A.k1) em *= 2;
        // mixed path: every term rounded to fixed point on its own, so the sum does not depend on which block took
        // which line group
        if (ENER) {
          if (fixed) ef += to_fix(em * double(G), kFixE);
          else e += em * double(G);
        }
        if (VIR)
          for (int k = 0; k < 6; ++k) {
            if (fixed) wf[k] += to_fix(em * double(wt[6 * gi + k]), kFixE);
            else w[k] += em * double(wt[6 * gi + k]);
          }
      }
      v.x *= G;
      v.y *= G;
      res[t] = v;
    }
    __syncthreads();
    const T* back = fft_lines_smem<R>(res, other, twi, nl, Pi);
    for (int t = threadIdx.x; t < nl * A.k3; t += blockDim.x) {
      const int c = t / nl, al = t - c * nl;
      h[size_t(a0 + al) + size_t(A.h1) * b + plane * c] = back[al * A.k3 + c];
    }
    __syncthreads();
  }
  if ((ENER || VIR) && fixed) {
    __shared__ long long scratch_q[32];
    if (ENER) {
      const long long s = block_sum(ef, scratch_q);
      if (threadIdx.x == 0) atomic_add_fix(en.fix + kECoul, s), atomic_add_fix(en.fix + kEPmeRecip, s);
    }
    if (VIR)
      for (int k = 0; k < 6; ++k) {
        const long long s = block_sum(wf[k], scratch_q);
        if (threadIdx.x == 0) atomic_add_fix(en.fix + kEW0 + k, s);
      }
  } else if (ENER || VIR) {
    __shared__ double scratch[32];
    if (ENER) {
      const double s = block_sum(e, scratch);
      if (threadIdx.x == 0) en.add(kECoul, s, false);
      if (threadIdx.x == 0) en.add(kEPmeRecip, s, false);
    }
    if (VIR)
      for (int k = 0; k < 6; ++k) {
        const double s = block_sum(w[k], scratch);
        if (threadIdx.x == 0) en.add(kEW0 + k, s, false);
      }
  }
}

// The influence function and its virial weights on the half spectrum (caps_kspace.f90:518-564, 916-940), in double,
// stored as R. Rebuilt when the cell, grid, order or beta change.
template <class R>
static __global__ void k_pme_green(PmeArgs A, const double* __restrict__ b1, const double* __restrict__ b2, const double* __restrict__ b3, double beta,
                            double kcoul, R* __restrict__ gt, R* __restrict__ wt) {
  const size_t total = size_t(A.h1) * A.k2 * A.k3;
  const double fac = kPi * kPi / (beta * beta);
  const int K[3] = {A.k1, A.k2, A.k3};
  for (size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += size_t(gridDim.x) * blockDim.x) {
    const int a = int(t % A.h1), b = int((t / A.h1) % A.k2), c = int(t / (size_t(A.h1) * A.k2));
    if (a == 0 && b == 0 && c == 0) {
      gt[t] = 0;
      for (int k = 0; k < 6; ++k) wt[6 * t + k] = 0;
      continue;
    }
    const int idx[3] = {a, b, c};
    int m[3];
    bool nyq[3];
    int nn = 0;
    for (int d = 0; d < 3; ++d) {
      m[d] = idx[d];
      if (m[d] >= (K[d] + 1) / 2) m[d] -= K[d];
      nyq[d] = K[d] % 2 == 0 && 2 * idx[d] == K[d];
      nn += nyq[d];
    }
    const double bm = b1[a] * b2[b] * b3[c];
    const int ns = 1 << nn;
    double g = 0, w[6] = {0, 0, 0, 0, 0, 0};
    for (int s = 0; s < ns; ++s) {
      int sel = 0;
      double mv[3] = {0, 0, 0};
      for (int d = 0; d < 3; ++d) {
        double sg = 1;
        if (nyq[d]) {
          if ((s >> sel) & 1) sg = -1;
          ++sel;
        }
        for (int r = 0; r < 3; ++r) mv[r] += sg * m[d] * A.cell.hi[d][r];
      }
      const double m2 = mv[0] * mv[0] + mv[1] * mv[1] + mv[2] * mv[2];
      const double e = kcoul * exp(-fac * m2) / (kPi * A.cell.vol * m2 * bm);
      const double ss = 2 * (1 + fac * m2) / m2;
      g += e;
      w[0] += e * (1 - ss * mv[0] * mv[0]);
      w[1] += e * (1 - ss * mv[1] * mv[1]);
      w[2] += e * (1 - ss * mv[2] * mv[2]);
      w[3] -= e * ss * mv[0] * mv[1];
      w[4] -= e * ss * mv[0] * mv[2];
      w[5] -= e * ss * mv[1] * mv[2];
    }
    gt[t] = R(g / ns);
    for (int k = 0; k < 6; ++k) wt[6 * t + k] = R(w[k] / ns);
  }
}

// K-GATHER: F_i -= q_i sum_d K_d (row d of h^-1) dE/du_d (caps_kspace.f90:965-992).
template <class R, class G, int P>
static __global__ void k_gather(PmeArgs A, const G* __restrict__ gr, ForceSink<R> F) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.n) return;
  const double qi = A.q[i];
  if (qi == 0) return;
  R th[3][P], dth[3][P];
  int base[3];
  atom_splines<R, P>(A, i, th, dth, base);
  int ia[P], ib[P];
#pragma unroll
  for (int a = 0; a < P; ++a) ia[a] = wrapk(base[0] + a, A.k1), ib[a] = wrapk(base[1] + a, A.k2);
  R gs0 = 0, gs1 = 0, gs2 = 0;
  for (int c = 0; c < P; ++c) {
    const int ic = wrapk(base[2] + c, A.k3);
    const R tc = th[2][c], dc = dth[2][c];
#pragma unroll
    for (int b = 0; b < P; ++b) {
      const R tb = th[1][b], db = dth[1][b];
      const size_t row = size_t(A.k1) * (size_t(ib[b]) + size_t(A.k2) * size_t(ic));
#pragma unroll
      for (int a = 0; a < P; ++a) {
        const R st = R(gr[row + ia[a]]);
        gs0 += dth[0][a] * tb * tc * st;
        gs1 += th[0][a] * db * tc * st;
        gs2 += th[0][a] * tb * dc * st;
      }
    }
  }
  R f[3];
  for (int r = 0; r < 3; ++r)
    f[r] = -R(qi) * (R(A.k1) * gs0 * R(A.cell.hi[0][r]) + R(A.k2) * gs1 * R(A.cell.hi[1][r]) + R(A.k3) * gs2 * R(A.cell.hi[2][r]));
  F.add(i, f[0], f[1], f[2]);
}

}  // namespace capsb
