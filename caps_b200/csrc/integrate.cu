// run_dynamics on the device (core/src/dynamics.cpp:71-815): velocity Verlet with the Bussi, Langevin (BAOAB) and
// Nose-Hoover-chain thermostats, stochastic cell rescaling, SHAKE / RATTLE for bonds to hydrogen and rigid waters.
//
// The state (x, v, forces, thermostat chain) stays in HBM for the whole run. One MD step is a fixed kernel sequence,
// captured once as a CUDA graph and replayed: the list check and the gated list build, the force kernels, the kicks,
// drifts, constraint solves and thermostat updates all read their scalars (target temperature, step number, chain
// variables) from device memory, so the graph is the same every step. Steps that report a thermo row, record a frame or
// scale the cell run the same sequence uncaptured with energies and virial on and synchronise with the host.
//
// Random numbers. Initial Maxwell-Boltzmann velocities and the Bussi thermostat's per-step draws come from a host
// stream built exactly as the reference's (std::mt19937_64 seeded with DynamicsOptions::seed, 53-bit uniforms,
// Marsaglia's polar normals, Marsaglia-Tsang gamma; core/include/caps/rng.hpp), uploaded ahead in chunks, so a Bussi or
// NVE or Nose-Hoover run starts from the reference's velocities and draws the reference's numbers. Langevin noise, 3N
// normals a step, comes from a counter-based Philox stream on the device (a pure function of seed, step and atom).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "engine.h"

namespace capsb {

// Whether a captured graph node is a kernel node.
static bool is_kernel_node(cudaGraphNode_t nd) {
  cudaGraphNodeType ty;
  CK(cudaGraphNodeGetType(nd, &ty));
  return ty == cudaGraphNodeTypeKernel;
}


namespace {

constexpr double kB = 0.0019872041;    // kcal/(mol K), as core/src/dynamics.cpp:22
constexpr double kAcc = 4.184e-4;      // (kcal/mol/Å)/(g/mol) -> Å/fs^2
constexpr double kAtm = 68568.415;     // kcal/(mol Å^3) -> atm
constexpr double kNA = 6.02214076e23;
constexpr int kMaxClAtoms = 8, kMaxClCons = 8;
constexpr int kShakeIter = 1000;
constexpr double kShakeTol = 1e-8;

// device scalars
enum Sc { kScKE = 0, kScKE0, kScBath, kScFactor, kScTnow, kScKtarget, kScStep, kScCW0, kScKin0 = kScCW0 + 6, kScNum = kScKin0 + 6 };
struct Chain {
  double eta[3], eta_dot[4], eta_dotdot[3], eta_mass[3];
};

int blocks(size_t n, int t) { return int(std::max<size_t>(1, (n + size_t(t) - 1) / size_t(t))); }

// --- the reference's random stream (core/include/caps/rng.hpp): 53-bit uniforms, polar normals, Marsaglia-Tsang ---
struct HostRng {
  std::mt19937_64 g;
  bool have = false;
  double spare = 0;
  explicit HostRng(uint64_t seed) : g(seed) {}
  double u01() { return double(uint64_t(g() - std::mt19937_64::min()) >> 11) * 0x1.0p-53; }
  double normal(bool& hv, double& sp) {
    if (hv) {
      hv = false;
      return sp;
    }
    double u, v, q;
    do {
      u = 2 * u01() - 1, v = 2 * u01() - 1, q = u * u + v * v;
    } while (q >= 1 || q == 0);
    const double f = std::sqrt(-2 * std::log(q) / q);
    sp = v * f;
    hv = true;
    return u * f;
  }
  double gauss() { return normal(have, spare); }
  double gamma(double k, double th) {   // shape k >= 1 (a fresh normal generator per call, as a fresh Gamma object)
    bool hv = false;
    double sp = 0;
    if (k <= 0) return 0;
    if (k < 1) {
      double u;
      do u = u01(); while (u == 0);
      const double up = gamma(k + 1, th);
      return up * std::pow(u, 1.0 / k);
    }
    const double d = k - 1.0 / 3.0, c = 1.0 / std::sqrt(9 * d);
    for (;;) {
      double x, v;
      do {
        x = normal(hv, sp);
        v = 1 + c * x;
      } while (v <= 0);
      v = v * v * v;
      double u;
      do u = u01(); while (u == 0);
      if (u < 1 - 0.0331 * x * x * x * x || std::log(u) < 0.5 * x * x + d * (1 - v + std::log(v))) return d * v * th;
    }
  }
};

// --- kernels --------------------------------------------------------------------------------------------------
// Kick then drift, per atom: v = s v + (hk f + hk2 f2) kAcc / m (s = sc[kScFactor] when `scale`, the thermostat's
// pending velocity factor, else 1; f2 may be null), x0 = x (the constraint reference), x += hd v. Non-finite positions
// raise the error word. With `zero_cw` the constraint-virial sums of this step start at zero. With fq (FP32 path) or fd
// (FP64 path) set, the atom's rows of the force evaluation's atom-order sums are cleared for the evaluation that follows
// (its own clearing is then skipped).
struct KickArgs {
  int n;
  double* x;
  double* v;
  double* x0;
  const double* f;
  const double* invm;
  double hk;
  const double* f2;
  double hk2;
  double hd;
  double* sc;
  int scale, zero_cw;
  int* counters;
  long long* fq;
  double* fd;
  double* info;   // the engine's error details (the step of the first non-finite position)
  int step_ahead; // 1 when this step's counter is advanced after this kick (the Langevin step's first kick)
};
__device__ __forceinline__ void kick_drift_atom(const KickArgs& K, int i, double s) {
  const double a = K.hk * kAcc * K.invm[i], a2 = K.hk2 * kAcc * K.invm[i];
  bool bad = false;
  for (int r = 0; r < 3; ++r) {
    double vr = K.v[3 * i + r];
    if (K.scale) vr *= s;
    vr += a * K.f[3 * i + r];
    if (K.f2) vr += a2 * K.f2[3 * i + r];   // r-RESPA: the slow and the fast forces in one kick
    K.v[3 * i + r] = vr;
    const double xo = K.x[3 * i + r];
    K.x0[3 * i + r] = xo;
    const double xn = xo + K.hd * vr;
    K.x[3 * i + r] = xn;
    bad |= !isfinite(xn);
    if (K.fq) K.fq[size_t(r) * K.n + i] = 0;
    if (K.fd) K.fd[size_t(r) * K.n + i] = 0;
  }
  if (bad) {
    atomicOr(reinterpret_cast<unsigned*>(K.counters + kCntErr), kErrNonFinite);
    if (K.info && atomicCAS(K.counters + kCntNanClaim, 0, 1) == 0) K.info[kInfoNonFiniteStep] = K.sc[kScStep] + K.step_ahead;
  }
}
// With L.xb set (a run without constraints), the displacement check of the drifted positions.
__global__ void k_kick_drift(KickArgs K, ListCheck L) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (K.zero_cw && i < 6) K.sc[kScCW0 + i] = 0;
  bool mb = false, mp = false;
  if (i < K.n) {
    kick_drift_atom(K, i, K.scale ? K.sc[kScFactor] : 1.0);
    if (L.xb) list_check_atom(L, i, K.x, mb, mp);
  }
  if (L.xb) list_check_flags(L, mb, mp);
}

// Constraint clusters. Star clusters (one centre bonded to 1-3 atoms, every constraint through the centre: CH, CH2, CH3)
// come first, ordered by size (ends e1, e2, e3), each as {centre, a1, a2, a3} and the squared lengths of (centre, a_k) in
// the reference's constraint order; then rigid waters (O-H1, O-H2, H1-H2 with equal O-H lengths and equal H masses),
// solved by SETTLE; the other clusters follow in the general layout.
struct ConsArgs {
  int ncl;                 // all clusters: e3 star clusters, then e4 - e3 rigid waters, then ncl - e4 general ones
  int e1, e2, e3, e4;
  const int4* star;        // e3: centre, then up to three partners (-1 unused)
  const double4* star_d2;  // e3: squared lengths of (centre, partner k)
  const int4* water;       // e4 - e3: O, H1, H2
  const double2* water_geo;   // e4 - e3: d(O-H), d(H-H)
  const int* cl_start;     // general clusters + 1: constraints of each cluster
  const int* cl_atom0;     // general clusters + 1: atoms of each cluster in cl_atoms
  const int* cl_atoms;     // atom indices
  const int4* cons;        // x, y: local atom indices, z: global i, w: global j
  const double* d2;        // squared lengths
  const double* invm;      // per atom
  DevCell cell;
  // LINCS (every cluster in the general layout): the constraints' lengths, and per cluster its couplings, pairs of its
  // constraints (local indices) that share an atom with the coefficient -S_k S_l s_ka s_la / m_a, in the reference's
  // order (atoms ascending, then the constraints on each)
  int lincs;
  const double* dlen;
  const int* cp_start;     // general clusters + 1
  const int2* cp;
  const double* cpc;
};
constexpr int kMaxCouple = 56;   // couplings of a cluster of 8 constraints

// SHAKE on a star cluster with NK constraints, in registers. The same Gauss-Seidel sweep as the general kernel, with each
// constraint taken as (centre, partner).
template <int NK>
__device__ void shake_star(const ConsArgs& C, int s, double* __restrict__ x, const double* __restrict__ x0, double* __restrict__ v, double h,
                           int* counters) {
  const int4 at = C.star[s];
  const double4 d4 = C.star_d2[s];
  const int ids[4] = {at.x, at.y, at.z, at.w};
  const double dd[3] = {d4.x, d4.y, d4.z};
  double p[NK + 1][3], o[NK + 1][3], im[NK + 1];
#pragma unroll
  for (int a = 0; a <= NK; ++a) {
    const int g = ids[a];
    for (int r = 0; r < 3; ++r) p[a][r] = x[3 * g + r], o[a][r] = x0[3 * g + r];
    im[a] = C.invm[g];
  }
  double ref[NK][3];
#pragma unroll
  for (int k = 0; k < NK; ++k) {
    double d0 = o[0][0] - o[k + 1][0], d1 = o[0][1] - o[k + 1][1], d2v = o[0][2] - o[k + 1][2];
    min_image(C.cell, d0, d1, d2v);
    ref[k][0] = d0, ref[k][1] = d1, ref[k][2] = d2v;
  }
  bool done = false;
  for (int it = 0; it < kShakeIter && !done; ++it) {
    done = true;
#pragma unroll
    for (int k = 0; k < NK; ++k) {
      double sv[3];
      for (int r = 0; r < 3; ++r) sv[r] = ref[k][r] + (p[0][r] - o[0][r]) - (p[k + 1][r] - o[k + 1][r]);
      const double diff = dd[k] - (sv[0] * sv[0] + sv[1] * sv[1] + sv[2] * sv[2]);
      if (fabs(diff) <= 2 * kShakeTol * dd[k]) continue;
      done = false;
      const double sr = sv[0] * ref[k][0] + sv[1] * ref[k][1] + sv[2] * ref[k][2];
      if (sr < 1e-6 * dd[k]) {
        atomicOr(reinterpret_cast<unsigned*>(counters + kCntErr), kErrShakeTurn);
        return;
      }
      const double g = diff / (2 * (im[0] + im[k + 1]) * sr);
      for (int r = 0; r < 3; ++r) {
        p[0][r] += g * im[0] * ref[k][r];
        p[k + 1][r] -= g * im[k + 1] * ref[k][r];
      }
    }
  }
  if (!done) atomicOr(reinterpret_cast<unsigned*>(counters + kCntErr), kErrShake);
#pragma unroll
  for (int a = 0; a <= NK; ++a) {
    const int g = ids[a];
    for (int r = 0; r < 3; ++r) {
      const double xb = x[3 * g + r];
      x[3 * g + r] = p[a][r];
      if (h > 0) v[3 * g + r] += (p[a][r] - xb) / h;
    }
  }
}


__device__ __forceinline__ void cross3d(const double a[3], const double b[3], double o[3]) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}
__device__ __forceinline__ double dot3d(const double a[3], const double b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
__device__ __forceinline__ void unit3d(double a[3]) {
  const double s = rsqrt(dot3d(a, a));
  for (int r = 0; r < 3; ++r) a[r] *= s;
}

// SETTLE (Miyamoto & Kollman, J. Comput. Chem. 13, 952 (1992)): the positions of a rigid water that satisfy its three
// distances exactly, found analytically from the unconstrained positions and the previous (constrained) ones. The
// molecule's centre of mass is kept; the canonical triangle (O at (0, ra, 0), H at (-+rc, -rb, 0) about the centre of
// mass) is rotated by the angles phi, psi, theta the paper derives, in a frame with z normal to the previous plane and x
// normal to the new O direction. The reference solves waters with SHAKE (constraints.cpp:196-230); SETTLE meets the
// same distances exactly instead of to SHAKE's 1e-8 tolerance. Displacements are added to each atom's own image.
__device__ void settle_water(const ConsArgs& C, int w, double* __restrict__ x, const double* __restrict__ x0, double* __restrict__ v, double h,
                             int* counters) {
  const int4 at = C.water[w];
  const int ia = at.x, ib = at.y, ic = at.z;
  const double2 geo = C.water_geo[w];
  const double mo = 1.0 / C.invm[ia], mh = 1.0 / C.invm[ib];
  const double mt = mo + 2 * mh;
  const double rc = 0.5 * geo.y;
  const double hgt = sqrt(geo.x * geo.x - rc * rc);
  const double ra = 2 * mh * hgt / mt, rb = hgt - ra;
  // previous and present positions of the hydrogens relative to their oxygen (nearest images)
  double b0[3], c0[3], b1[3], c1[3];
  for (int r = 0; r < 3; ++r) {
    b0[r] = x0[3 * ib + r] - x0[3 * ia + r], c0[r] = x0[3 * ic + r] - x0[3 * ia + r];
    b1[r] = x[3 * ib + r] - x[3 * ia + r], c1[r] = x[3 * ic + r] - x[3 * ia + r];
  }
  min_image(C.cell, b0[0], b0[1], b0[2]);
  min_image(C.cell, c0[0], c0[1], c0[2]);
  min_image(C.cell, b1[0], b1[1], b1[2]);
  min_image(C.cell, c1[0], c1[1], c1[2]);
  // present positions relative to their centre of mass
  double A1[3], B1[3], C1[3];
  for (int r = 0; r < 3; ++r) {
    const double com = mh * (b1[r] + c1[r]) / mt;
    A1[r] = -com, B1[r] = b1[r] - com, C1[r] = c1[r] - com;
  }
  double ez[3], ex[3], ey[3];
  cross3d(b0, c0, ez);
  cross3d(A1, ez, ex);
  cross3d(ez, ex, ey);
  unit3d(ex);
  unit3d(ey);
  unit3d(ez);
  const double xb0 = dot3d(b0, ex), yb0 = dot3d(b0, ey), xc0 = dot3d(c0, ex), yc0 = dot3d(c0, ey);
  const double za1 = dot3d(A1, ez);
  const double xb1 = dot3d(B1, ex), yb1 = dot3d(B1, ey), zb1 = dot3d(B1, ez);
  const double xc1 = dot3d(C1, ex), yc1 = dot3d(C1, ey), zc1 = dot3d(C1, ez);
  const double sinphi = za1 / ra;
  const double cphi2 = 1 - sinphi * sinphi;
  const double cosphi = sqrt(fmax(cphi2, 0.0));
  const double sinpsi = (zb1 - zc1) / (2 * rc * cosphi);
  const double cpsi2 = 1 - sinpsi * sinpsi;
  const double cospsi = sqrt(fmax(cpsi2, 0.0));
  const double ya2 = ra * cosphi, xb2 = -rc * cospsi;
  const double t1 = -rb * cosphi, t2 = rc * sinpsi * sinphi;
  const double yb2 = t1 - t2, yc2 = t1 + t2;
  const double alpha = xb2 * (xb0 - xc0) + yb0 * yb2 + yc0 * yc2;
  const double beta = xb2 * (yc0 - yb0) + xb0 * yb2 + xc0 * yc2;
  const double gamma = xb0 * yb1 - xb1 * yb0 + xc0 * yc1 - xc1 * yc0;
  const double ab2 = alpha * alpha + beta * beta;
  const double disc = ab2 - gamma * gamma;
  if (!(cphi2 > 0) || !(cpsi2 >= 0) || !(disc >= 0) || !(ab2 > 0)) {   // moved too far in one step for a rigid water
    atomicOr(reinterpret_cast<unsigned*>(counters + kCntErr), kErrShake);
    return;
  }
  const double sinth = (alpha * gamma - beta * sqrt(disc)) / ab2;
  const double costh = sqrt(fmax(1 - sinth * sinth, 0.0));
  const double a3[3] = {-ya2 * sinth, ya2 * costh, za1};
  const double b3[3] = {xb2 * costh - yb2 * sinth, xb2 * sinth + yb2 * costh, zb1};
  const double c3[3] = {-xb2 * costh - yc2 * sinth, -xb2 * sinth + yc2 * costh, zc1};
  for (int r = 0; r < 3; ++r) {
    const double da = a3[0] * ex[r] + a3[1] * ey[r] + a3[2] * ez[r] - A1[r];
    const double db = b3[0] * ex[r] + b3[1] * ey[r] + b3[2] * ez[r] - B1[r];
    const double dc = c3[0] * ex[r] + c3[1] * ey[r] + c3[2] * ez[r] - C1[r];
    x[3 * ia + r] += da, x[3 * ib + r] += db, x[3 * ic + r] += dc;
    if (h > 0) v[3 * ia + r] += da / h, v[3 * ib + r] += db / h, v[3 * ic + r] += dc / h;
  }
}

// LINCS on general cluster c (core/src/constraints.cpp:125-185, Hess 1997, order 4): from the old directions B_k, one
// projection of the separations onto the constraint lengths through the expansion (I - A)^-1 = sum_{n<=4} A^n, then the
// rotational corrections (the projection along B_k aimed at sqrt(d^2 - perp^2)) until every length holds to tol; then
// v += (x - x_before) / h when h > 0. The reference couples all constraints that share an atom; those of different
// clusters share none, so each cluster is solved alone (its iterations stop when its own lengths hold).
__device__ void lincs_cluster(const ConsArgs& C, int c, double* __restrict__ x, const double* __restrict__ x0, double* __restrict__ v, double h,
                              int* counters) {
  const int k0 = C.cl_start[c], k1 = C.cl_start[c + 1], a0 = C.cl_atom0[c], a1 = C.cl_atom0[c + 1];
  const int q0 = C.cp_start[c], nq = C.cp_start[c + 1] - q0;
  const int na = a1 - a0, nk = k1 - k0;
  double px[kMaxClAtoms][3], ox[kMaxClAtoms][3], bx[kMaxClAtoms][3], im[kMaxClAtoms];
  for (int a = 0; a < na; ++a) {
    const int g = C.cl_atoms[a0 + a];
    for (int r = 0; r < 3; ++r) px[a][r] = x[3 * g + r], ox[a][r] = x0[3 * g + r], bx[a][r] = px[a][r];
    im[a] = C.invm[g];
  }
  double ref[kMaxClCons][3], B[kMaxClCons][3], S[kMaxClCons], dl[kMaxClCons];
  int li[kMaxClCons], lj[kMaxClCons];
  for (int k = 0; k < nk; ++k) {
    const int4 q = C.cons[k0 + k];
    li[k] = q.x, lj[k] = q.y;
    dl[k] = C.dlen[k0 + k];
    double d0 = ox[q.x][0] - ox[q.y][0], d1 = ox[q.x][1] - ox[q.y][1], d2v = ox[q.x][2] - ox[q.y][2];
    min_image(C.cell, d0, d1, d2v);
    ref[k][0] = d0, ref[k][1] = d1, ref[k][2] = d2v;
    const double l = sqrt(d0 * d0 + d1 * d1 + d2v * d2v);
    if (l < 1e-12) {
      atomicOr(reinterpret_cast<unsigned*>(counters + kCntErr), kErrConsOverlap);
      return;
    }
    const double il = 1 / l;
    for (int r = 0; r < 3; ++r) B[k][r] = ref[k][r] * il;
    S[k] = 1.0 / sqrt(im[q.x] + im[q.y]);
  }
  double akl[kMaxCouple];
  int ck[kMaxCouple], cl[kMaxCouple];
  for (int q = 0; q < nq; ++q) {
    const int2 p = C.cp[q0 + q];
    ck[q] = p.x, cl[q] = p.y;
    akl[q] = C.cpc[q0 + q] * (B[p.x][0] * B[p.y][0] + B[p.x][1] * B[p.y][1] + B[p.x][2] * B[p.y][2]);
  }
  auto sep = [&](int k, double s[3]) {
    for (int r = 0; r < 3; ++r) s[r] = ref[k][r] + (px[li[k]][r] - ox[li[k]][r]) - (px[lj[k]][r] - ox[lj[k]][r]);
  };
  double rhs[kMaxClCons], sol[kMaxClCons], t[kMaxClCons], t2[kMaxClCons];
  auto solve_apply = [&]() {
    for (int k = 0; k < nk; ++k) sol[k] = rhs[k], t[k] = rhs[k];
    for (int order = 0; order < 4; ++order) {
      for (int k = 0; k < nk; ++k) t2[k] = 0.0;
      for (int q = 0; q < nq; ++q) t2[ck[q]] += akl[q] * t[cl[q]];
      for (int k = 0; k < nk; ++k) sol[k] += t2[k], t[k] = t2[k];
    }
    for (int k = 0; k < nk; ++k) {
      const double g = S[k] * sol[k];
      for (int r = 0; r < 3; ++r) {
        px[li[k]][r] -= im[li[k]] * g * B[k][r];
        px[lj[k]][r] += im[lj[k]] * g * B[k][r];
      }
    }
  };
  for (int k = 0; k < nk; ++k) {
    double s[3];
    sep(k, s);
    rhs[k] = S[k] * ((B[k][0] * s[0] + B[k][1] * s[1] + B[k][2] * s[2]) - dl[k]);
  }
  solve_apply();
  bool done = false;
  for (int it = 0; it < kShakeIter && !done; ++it) {
    done = true;
    for (int k = 0; k < nk; ++k) {
      double s[3];
      sep(k, s);
      const double d = dl[k], l2 = s[0] * s[0] + s[1] * s[1] + s[2] * s[2], along = B[k][0] * s[0] + B[k][1] * s[1] + B[k][2] * s[2];
      if (fabs(d * d - l2) > 2 * kShakeTol * d * d) done = false;
      if (along < 0) {
        atomicOr(reinterpret_cast<unsigned*>(counters + kCntErr), kErrShakeTurn);
        return;
      }
      const double perp2 = fmax(0.0, l2 - along * along);
      rhs[k] = S[k] * (along - sqrt(fmax(0.0, d * d - perp2)));
    }
    if (!done) solve_apply();
  }
  if (!done) atomicOr(reinterpret_cast<unsigned*>(counters + kCntErr), kErrLincs);
  for (int a = 0; a < na; ++a) {
    const int g = C.cl_atoms[a0 + a];
    for (int r = 0; r < 3; ++r) {
      x[3 * g + r] = px[a][r];
      if (h > 0) v[3 * g + r] += (px[a][r] - bx[a][r]) / h;
    }
  }
}

// SHAKE on each cluster (Gauss-Seidel along the reference vectors, tol 1e-8 relative; core/src/constraints.cpp:196-230),
// then v += (x - x_before) / h when h > 0.
__device__ void shake_cluster(const ConsArgs& C, int cc, double* __restrict__ x, const double* __restrict__ x0, double* __restrict__ v, double h,
                              int* counters) {
  if (cc < C.e1) return shake_star<1>(C, cc, x, x0, v, h, counters);
  if (cc < C.e2) return shake_star<2>(C, cc, x, x0, v, h, counters);
  if (cc < C.e3) return shake_star<3>(C, cc, x, x0, v, h, counters);
  if (cc < C.e4) return settle_water(C, cc - C.e3, x, x0, v, h, counters);
  const int c = cc - C.e4;
  const int k0 = C.cl_start[c], k1 = C.cl_start[c + 1], a0 = C.cl_atom0[c], a1 = C.cl_atom0[c + 1];
  const int na = a1 - a0, nk = k1 - k0;
  double px[kMaxClAtoms][3], ox[kMaxClAtoms][3], bx[kMaxClAtoms][3], im[kMaxClAtoms];
  for (int a = 0; a < na; ++a) {
    const int g = C.cl_atoms[a0 + a];
    for (int r = 0; r < 3; ++r) px[a][r] = x[3 * g + r], ox[a][r] = x0[3 * g + r], bx[a][r] = px[a][r];
    im[a] = C.invm[g];
  }
  double ref[kMaxClCons][3];
  int li[kMaxClCons], lj[kMaxClCons];
  double dd[kMaxClCons];
  for (int k = 0; k < nk; ++k) {
    const int4 q = C.cons[k0 + k];
    li[k] = q.x, lj[k] = q.y;
    dd[k] = C.d2[k0 + k];
    double d0 = ox[q.x][0] - ox[q.y][0], d1 = ox[q.x][1] - ox[q.y][1], d2v = ox[q.x][2] - ox[q.y][2];
    min_image(C.cell, d0, d1, d2v);
    ref[k][0] = d0, ref[k][1] = d1, ref[k][2] = d2v;
  }
  bool done = false;
  for (int it = 0; it < kShakeIter && !done; ++it) {
    done = true;
    for (int k = 0; k < nk; ++k) {
      const int i = li[k], j = lj[k];
      double s[3];
      for (int r = 0; r < 3; ++r) s[r] = ref[k][r] + (px[i][r] - ox[i][r]) - (px[j][r] - ox[j][r]);
      const double diff = dd[k] - (s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
      if (fabs(diff) <= 2 * kShakeTol * dd[k]) continue;
      done = false;
      const double sr = s[0] * ref[k][0] + s[1] * ref[k][1] + s[2] * ref[k][2];
      if (sr < 1e-6 * dd[k]) {
        atomicOr(reinterpret_cast<unsigned*>(counters + kCntErr), kErrShakeTurn);
        return;
      }
      const double g = diff / (2 * (im[i] + im[j]) * sr);
      for (int r = 0; r < 3; ++r) {
        px[i][r] += g * im[i] * ref[k][r];
        px[j][r] -= g * im[j] * ref[k][r];
      }
    }
  }
  if (!done) atomicOr(reinterpret_cast<unsigned*>(counters + kCntErr), kErrShake);
  for (int a = 0; a < na; ++a) {
    const int g = C.cl_atoms[a0 + a];
    for (int r = 0; r < 3; ++r) {
      x[3 * g + r] = px[a][r];
      if (h > 0) v[3 * g + r] += (px[a][r] - bx[a][r]) / h;
    }
  }
}

// The atoms of cluster cc through the displacement check.
__device__ void check_cluster(const ConsArgs& C, const ListCheck& L, int cc, const double* x, bool& mb, bool& mp) {
  if (cc < C.e3) {
    const int4 at = C.star[cc];
    const int ids[4] = {at.x, at.y, at.z, at.w};
    for (int a = 0; a < 4; ++a)
      if (ids[a] >= 0) list_check_atom(L, ids[a], x, mb, mp);
  } else if (cc < C.e4) {
    const int4 w = C.water[cc - C.e3];
    list_check_atom(L, w.x, x, mb, mp);
    list_check_atom(L, w.y, x, mb, mp);
    list_check_atom(L, w.z, x, mb, mp);
  } else {
    const int c = cc - C.e4;
    for (int a = C.cl_atom0[c]; a < C.cl_atom0[c + 1]; ++a) list_check_atom(L, C.cl_atoms[a], x, mb, mp);
  }
}

// LINCS, a thread per cluster (every cluster in the general layout), with the displacement check as k_shake has it.
__global__ void k_lincs(ConsArgs C, double* __restrict__ x, const double* __restrict__ x0, double* __restrict__ v, double h, int* counters,
                        ListCheck L) {
  const int cc = blockIdx.x * blockDim.x + threadIdx.x;
  bool mb = false, mp = false;
  if (cc < C.ncl) {
    lincs_cluster(C, cc, x, x0, v, h, counters);
    if (L.xb) check_cluster(C, L, cc, x, mb, mp);
  } else if (L.xb && cc < C.ncl + L.nfree) {
    list_check_atom(L, L.free_atoms[cc - C.ncl], x, mb, mp);
  }
  if (L.xb) list_check_flags(L, mb, mp);
}

// SHAKE, a thread per cluster; with L.xb set, the displacement check of the step's final positions on the clusters'
// atoms and, after the clusters, on the L.nfree atoms in none.
__global__ void k_shake(ConsArgs C, double* __restrict__ x, const double* __restrict__ x0, double* __restrict__ v, double h, int* counters,
                        ListCheck L) {
  const int cc = blockIdx.x * blockDim.x + threadIdx.x;
  bool mb = false, mp = false;
  if (cc < C.ncl) {
    shake_cluster(C, cc, x, x0, v, h, counters);
    if (L.xb) check_cluster(C, L, cc, x, mb, mp);
  } else if (L.xb && cc < C.ncl + L.nfree) {
    list_check_atom(L, L.free_atoms[cc - C.ncl], x, mb, mp);
  }
  if (L.xb) list_check_flags(L, mb, mp);
}

// The velocity update of one atom before RATTLE: a kick (v += hk kAcc f / m) or the Langevin O step
// (v = c1 v + c2 sqrt(kB T kAcc / m) N(0, 1), Philox normals keyed by (seed, step, atom)).
struct VelOp {
  int kind;                  // 0 none, 1 kick (f, and f2 when not null), 2 Langevin O
  const double* f;
  double hk;
  double c1, c2;
  uint64_t seed;
  const double* f2;
  double hk2;
  // kick from the force evaluation's own sums instead of f (when fq or fd is set): atom-order sums plus the pair
  // kernel's slot-order sums at iperm (the reduction Engine::forces otherwise runs as a kernel of its own); the total is
  // stored to fout for the next step's first kick
  const long long* fq;       // FP32 path: fixed point, 3 x nat then 3 x nslots
  const long long* fsq;
  const double* fd;          // FP64 path
  const double* fsd;
  const int* iperm;
  int nat, nslots;
  double* fout;
};
// The force on atom g for a kick: f, or the evaluation's sums (stored to fout).
__device__ __forceinline__ void kick_force(const VelOp& op, int g, double f[3]) {
  if (!op.fq && !op.fd) {
    for (int r = 0; r < 3; ++r) f[r] = op.f[3 * g + r];
    return;
  }
  const int s = op.iperm ? op.iperm[g] : -1;
  const bool ok = s >= 0 && s < op.nslots;   // as the reduction: a build that overflowed can leave iperm stale (reported)
  for (int r = 0; r < 3; ++r) {
    if (op.fq) {
      long long q = op.fq[size_t(r) * op.nat + g];
      if (ok) q += op.fsq[size_t(r) * op.nslots + s];
      f[r] = double(q) * kInvFixF;
    } else {
      double q = op.fd[size_t(r) * op.nat + g];
      if (ok) q += op.fsd[size_t(r) * op.nslots + s];
      f[r] = q;
    }
    op.fout[3 * g + r] = f[r];
  }
}
__device__ __forceinline__ void vel_op(const VelOp& op, int g, double* vv, const double* __restrict__ invm, const double* sc) {
  if (op.kind == 1) {
    const double a = op.hk * kAcc * invm[g];
    double f[3];
    kick_force(op, g, f);
    for (int r = 0; r < 3; ++r) vv[r] += a * f[r];
    if (op.f2) {
      const double a2 = op.hk2 * kAcc * invm[g];
      for (int r = 0; r < 3; ++r) vv[r] += a2 * op.f2[3 * g + r];
    }
  } else if (op.kind == 2) {
    double z[4];
    normals4(op.seed, (uint64_t)sc[kScStep], uint32_t(g), 0x4C414E47u, z);
    const double sd = sqrt(kB * sc[kScTnow] * kAcc * invm[g]);
    for (int r = 0; r < 3; ++r) vv[r] = op.c1 * vv[r] + op.c2 * sd * z[r];
  }
}

// The velocity update alone, one thread per atom (runs without constraints).
__global__ void k_vel(int n, double* __restrict__ v, const double* __restrict__ invm, const double* sc, VelOp op) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double vv[3] = {v[3 * i], v[3 * i + 1], v[3 * i + 2]};
  vel_op(op, i, vv, invm, sc);
  for (int r = 0; r < 3; ++r) v[3 * i + r] = vv[r];
}

// RATTLE on a star cluster with NK constraints, in registers (the general kernel's sweep, constraints as (centre, partner)).
template <int NK>
__device__ void rattle_star(const ConsArgs& C, int s, const double* __restrict__ x, double* __restrict__ v, const VelOp& op, const double* sc,
                            double h, double w[6], int* counters) {
  const int4 at = C.star[s];
  const double4 d4 = C.star_d2[s];
  const int ids[4] = {at.x, at.y, at.z, at.w};
  const double dd[3] = {d4.x, d4.y, d4.z};
  double pv[NK + 1][3], im[NK + 1];
#pragma unroll
  for (int a = 0; a <= NK; ++a) {
    const int g = ids[a];
    for (int r = 0; r < 3; ++r) pv[a][r] = v[3 * g + r];
    vel_op(op, g, pv[a], C.invm, sc);
    im[a] = C.invm[g];
  }
  double rr[NK][3], lam[NK];
#pragma unroll
  for (int k = 0; k < NK; ++k) {
    const int gi = ids[0], gj = ids[k + 1];
    double d0 = x[3 * gi] - x[3 * gj], d1 = x[3 * gi + 1] - x[3 * gj + 1], d2v = x[3 * gi + 2] - x[3 * gj + 2];
    min_image(C.cell, d0, d1, d2v);
    rr[k][0] = d0, rr[k][1] = d1, rr[k][2] = d2v;
    lam[k] = 0;
  }
  bool done = false;
  for (int it = 0; it < kShakeIter && !done; ++it) {
    done = true;
#pragma unroll
    for (int k = 0; k < NK; ++k) {
      const double rv = rr[k][0] * (pv[0][0] - pv[k + 1][0]) + rr[k][1] * (pv[0][1] - pv[k + 1][1]) + rr[k][2] * (pv[0][2] - pv[k + 1][2]);
      if (fabs(rv) <= kShakeTol * dd[k]) continue;
      done = false;
      const double g = -rv / ((im[0] + im[k + 1]) * dd[k]);
      lam[k] += g;
      for (int r = 0; r < 3; ++r) {
        pv[0][r] += g * im[0] * rr[k][r];
        pv[k + 1][r] -= g * im[k + 1] * rr[k][r];
      }
    }
  }
  if (!done) atomicOr(reinterpret_cast<unsigned*>(counters + kCntErr), kErrRattle);
#pragma unroll
  for (int a = 0; a <= NK; ++a)
    for (int r = 0; r < 3; ++r) v[3 * ids[a] + r] = pv[a][r];
  if (h > 0)
#pragma unroll
    for (int k = 0; k < NK; ++k) {
      const double sk = 2 * lam[k] / (h * kAcc);
      w[0] += sk * rr[k][0] * rr[k][0];
      w[1] += sk * rr[k][1] * rr[k][1];
      w[2] += sk * rr[k][2] * rr[k][2];
      w[3] += sk * rr[k][0] * rr[k][1];
      w[4] += sk * rr[k][0] * rr[k][2];
      w[5] += sk * rr[k][1] * rr[k][2];
    }
}

// RATTLE on a rigid water in registers: Gauss-Seidel over (O, H1), (O, H2), (H1, H2).
__device__ void rattle_water(const ConsArgs& C, int wi, const double* __restrict__ x, double* __restrict__ v, const VelOp& op, const double* sc,
                             double h, double w[6], int* counters) {
  const int4 at = C.water[wi];
  const double2 geo = C.water_geo[wi];
  const int ids[3] = {at.x, at.y, at.z};
  const int pi[3] = {0, 0, 1}, pj[3] = {1, 2, 2};
  const double dd[3] = {geo.x * geo.x, geo.x * geo.x, geo.y * geo.y};
  double pv[3][3], im[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int g = ids[a];
    for (int r = 0; r < 3; ++r) pv[a][r] = v[3 * g + r];
    vel_op(op, g, pv[a], C.invm, sc);
    im[a] = C.invm[g];
  }
  double rr[3][3], lam[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int gi = ids[pi[k]], gj = ids[pj[k]];
    double d0 = x[3 * gi] - x[3 * gj], d1 = x[3 * gi + 1] - x[3 * gj + 1], d2v = x[3 * gi + 2] - x[3 * gj + 2];
    min_image(C.cell, d0, d1, d2v);
    rr[k][0] = d0, rr[k][1] = d1, rr[k][2] = d2v;
    lam[k] = 0;
  }
  bool done = false;
  for (int it = 0; it < kShakeIter && !done; ++it) {
    done = true;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const int i = pi[k], j = pj[k];
      const double rv = rr[k][0] * (pv[i][0] - pv[j][0]) + rr[k][1] * (pv[i][1] - pv[j][1]) + rr[k][2] * (pv[i][2] - pv[j][2]);
      if (fabs(rv) <= kShakeTol * dd[k]) continue;
      done = false;
      const double g = -rv / ((im[i] + im[j]) * dd[k]);
      lam[k] += g;
      for (int r = 0; r < 3; ++r) {
        pv[i][r] += g * im[i] * rr[k][r];
        pv[j][r] -= g * im[j] * rr[k][r];
      }
    }
  }
  if (!done) atomicOr(reinterpret_cast<unsigned*>(counters + kCntErr), kErrRattle);
#pragma unroll
  for (int a = 0; a < 3; ++a)
    for (int r = 0; r < 3; ++r) v[3 * ids[a] + r] = pv[a][r];
  if (h > 0)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double sk = 2 * lam[k] / (h * kAcc);
      w[0] += sk * rr[k][0] * rr[k][0];
      w[1] += sk * rr[k][1] * rr[k][1];
      w[2] += sk * rr[k][2] * rr[k][2];
      w[3] += sk * rr[k][0] * rr[k][1];
      w[4] += sk * rr[k][0] * rr[k][2];
      w[5] += sk * rr[k][1] * rr[k][2];
    }
}

__global__ void k_scale_v(int n, double* __restrict__ v, const double* __restrict__ sc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 3 * n) return;
  v[i] *= sc[kScFactor];
}
// v *= f (the MTK step's factors, made on the host)
__global__ void k_scale_by(int n, double* __restrict__ v, double f) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < 3 * n) v[i] *= f;
}
// The MTK remap (dynamics.cpp:560-570): x = c0 + mu (x - c0) about the cell's centre c0.
__global__ void k_remap(int n, double* __restrict__ x, double c0x, double c0y, double c0z, double mu) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  x[3 * i] = c0x + mu * (x[3 * i] - c0x);
  x[3 * i + 1] = c0y + mu * (x[3 * i + 1] - c0y);
  x[3 * i + 2] = c0z + mu * (x[3 * i + 2] - c0z);
}

// The step counter and the thermostat target: T ramps linearly from t0 to t1 over `steps` when t1 >= 0.
__device__ void step_begin_body(double* sc, double t0, double t1, long long steps, double ndof) {
  const double step = sc[kScStep] + 1;
  sc[kScStep] = step;
  const double t = (t1 >= 0 && steps > 0) ? t0 + (t1 - t0) * step / double(steps) : t0;
  sc[kScTnow] = t;
  sc[kScKtarget] = 0.5 * ndof * kB * t;
}
__global__ void k_step_begin(double* sc, double t0, double t1, long long steps, double ndof) {
  step_begin_body(sc, t0, t1, steps, ndof);
}

// Nose-Hoover chain over half a step (LAMMPS FixNH::nhc_temp_integrate, as dynamics.cpp:479-508): sets the velocity
// factor in sc[kScFactor]; the caller scales v by it.
__device__ void nhc_body(Chain* ch, double* sc, double ndof, double t_freq, double dt) {
  const double dthalf = 0.5 * dt, dt4 = 0.25 * dt, dt8 = 0.125 * dt;
  const double tt = sc[kScTnow], kt = kB * tt, ke_target = ndof * kt;
  Chain& c = *ch;
  c.eta_mass[0] = ndof * kt / (t_freq * t_freq);
  for (int q = 1; q < 3; ++q) c.eta_mass[q] = kt / (t_freq * t_freq);
  double kecur = 2 * sc[kScKE];
  c.eta_dotdot[0] = (kecur - ke_target) / c.eta_mass[0];
  for (int q = 2; q > 0; --q) {
    const double ex = exp(-dt8 * c.eta_dot[q + 1]);
    c.eta_dot[q] = (c.eta_dot[q] * ex + c.eta_dotdot[q] * dt4) * ex;
  }
  double ex = exp(-dt8 * c.eta_dot[1]);
  c.eta_dot[0] = (c.eta_dot[0] * ex + c.eta_dotdot[0] * dt4) * ex;
  const double factor = exp(-dthalf * c.eta_dot[0]);
  kecur *= factor * factor;
  c.eta_dotdot[0] = (kecur - ke_target) / c.eta_mass[0];
  for (int q = 0; q < 3; ++q) c.eta[q] += dthalf * c.eta_dot[q];
  c.eta_dot[0] = (c.eta_dot[0] * ex + c.eta_dotdot[0] * dt4) * ex;
  for (int q = 1; q < 3; ++q) {
    ex = exp(-dt8 * c.eta_dot[q + 1]);
    c.eta_dot[q] *= ex;
    c.eta_dotdot[q] = (c.eta_mass[q - 1] * c.eta_dot[q - 1] * c.eta_dot[q - 1] - kt) / c.eta_mass[q];
    c.eta_dot[q] = (c.eta_dot[q] + c.eta_dotdot[q] * dt4) * ex;
  }
  sc[kScFactor] = factor;
  sc[kScKE] = 0.5 * kecur;
}

// Bussi velocity rescaling (Bussi, Donadio & Parrinello 2007, appendix; dynamics.cpp:466-477) from this step's draws
// (r1, sum of ndof - 1 squared normals) read from the host-made table.
__device__ void bussi_body(double* sc, const double2* __restrict__ draws, long long first_step, double h, double tau, double ndof) {
  const double k = sc[kScKE];
  const long long step = (long long)sc[kScStep];
  if (k <= 0) {
    sc[kScFactor] = 1;
    return;
  }
  const double2 d = draws[step - first_step];
  const double c = exp(-h / tau), kt = sc[kScKtarget];
  const double r1 = d.x, sum = d.y;
  const double knew = k + (1 - c) * (kt * (r1 * r1 + sum) / ndof - k) + 2 * r1 * sqrt(c * (1 - c) * kt * k / ndof);
  sc[kScFactor] = sqrt(fmax(knew, 0.0) / k);
  sc[kScBath] -= knew - k;
}

// What the last block of k_ke does with the fresh kinetic energy.
enum KeThen { kThenNone = 0, kThenNhc, kThenBussi, kThenBath };
struct KeArgs {
  int n;
  const double* v;
  const double* m;
  double* part;          // 7 per block
  unsigned* done;        // blocks finished; the last block resets it
  double* sc;
  int slot;              // sc slot receiving 0.5 sum m v^2 / kAcc
  int tensor;            // also the kinetic tensor into kScKin0..
  int begin;             // run the step-begin update first
  int then;              // KeThen
  double t0, t1, ndof;
  long long steps;
  Chain* chain;
  double t_freq, dt;
  const double2* draws;
  long long draws_first;
  double tau;
};

// One atom's share: m v^2, and the tensor terms on request.
__device__ __forceinline__ void ke_atom(const KeArgs& A, int i, double& e, double t[6]) {
  const double vx = A.v[3 * i], vy = A.v[3 * i + 1], vz = A.v[3 * i + 2], mi = A.m[i];
  e += mi * (vx * vx + vy * vy + vz * vz);
  if (A.tensor) t[0] += mi * vx * vx, t[1] += mi * vy * vy, t[2] += mi * vz * vz, t[3] += mi * vx * vy, t[4] += mi * vx * vz, t[5] += mi * vy * vz;
}

// The block sums of every thread's share into A.part (7 per block), then in the last block to finish: the partials in
// block order and the scalar update. Every thread of every block calls it.
__device__ void ke_blocks(const KeArgs& A, double e, double t[6]) {
  __shared__ double scratch[32];
  __shared__ bool last;
  const double s = block_sum(e, scratch);
  if (threadIdx.x == 0) A.part[blockIdx.x * 7] = s;
  if (A.tensor)
    for (int q = 0; q < 6; ++q) {
      const double st = block_sum(t[q], scratch);
      if (threadIdx.x == 0) A.part[blockIdx.x * 7 + 1 + q] = st;
    }
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(A.done, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  e = 0;
  for (int q = 0; q < 6; ++q) t[q] = 0;
  for (int b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
    e += __ldcg(A.part + 7 * b);
    if (A.tensor)
      for (int q = 0; q < 6; ++q) t[q] += __ldcg(A.part + 7 * b + 1 + q);
  }
  const double tot = block_sum(e, scratch);
  double tt[6];
  if (A.tensor)
    for (int q = 0; q < 6; ++q) tt[q] = block_sum(t[q], scratch);
  if (threadIdx.x != 0) return;
  *A.done = 0;
  double* sc = A.sc;
  sc[A.slot] = 0.5 * tot / kAcc;
  if (A.tensor)
    for (int q = 0; q < 6; ++q) sc[kScKin0 + q] = tt[q] / kAcc;
  if (A.begin) step_begin_body(sc, A.t0, A.t1, A.steps, A.ndof);
  if (A.then == kThenNhc) nhc_body(A.chain, sc, A.ndof, A.t_freq, A.dt);
  else if (A.then == kThenBussi) bussi_body(sc, A.draws, A.draws_first, A.dt, A.tau, A.ndof);
  else if (A.then == kThenBath) sc[kScBath] -= sc[kScKE] - sc[kScKE0];
}

// The first Nose-Hoover half step of a step, on the kinetic energy the previous step left in sc[kScKE]: its second half
// set it to the scaled velocities' value, and the velocities have not changed since.
__global__ void k_nhc_begin(Chain* ch, double* sc, double t0, double t1, long long steps, double ndof, double t_freq, double dt) {
  step_begin_body(sc, t0, t1, steps, ndof);
  nhc_body(ch, sc, ndof, t_freq, dt);
}

// Velocity update then RATTLE in one launch: threads [0, ncl) take one constraint cluster each (its atoms' update, then
// the relative velocity along each constraint removed, core/src/constraints.cpp:232-269; star clusters in registers);
// threads [ncl, ncl + nfree) update one unconstrained atom each. With h > 0 the impulses are read as forces over a half kick and their virial
// (xx yy zz xy xz yz) is added to sc[kScCW0..]. With K.n > 0 the launch also takes the kinetic energy of the new
// velocities and runs K's thermostat update in its last block (what k_ke does in a launch of its own).
__global__ void k_vel_rattle(ConsArgs C, int nfree, const int* __restrict__ free_atoms, const double* __restrict__ x, double* __restrict__ v, VelOp op,
                             double h, double* sc, int* counters, KeArgs K) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  double w[6] = {0, 0, 0, 0, 0, 0};
  if (c >= C.ncl && c < C.ncl + nfree) {
    const int g = free_atoms[c - C.ncl];
    double vv[3] = {v[3 * g], v[3 * g + 1], v[3 * g + 2]};
    vel_op(op, g, vv, C.invm, sc);
    for (int r = 0; r < 3; ++r) v[3 * g + r] = vv[r];
  }
  if (c < C.e1) rattle_star<1>(C, c, x, v, op, sc, h, w, counters);
  else if (c < C.e2) rattle_star<2>(C, c, x, v, op, sc, h, w, counters);
  else if (c < C.e3) rattle_star<3>(C, c, x, v, op, sc, h, w, counters);
  else if (c < C.e4) rattle_water(C, c - C.e3, x, v, op, sc, h, w, counters);
  else if (c < C.ncl) {
    const int cg = c - C.e4;
    const int k0 = C.cl_start[cg], k1 = C.cl_start[cg + 1], a0 = C.cl_atom0[cg], a1 = C.cl_atom0[cg + 1];
    const int na = a1 - a0, nk = k1 - k0;
    double pv[kMaxClAtoms][3], im[kMaxClAtoms];
    for (int a = 0; a < na; ++a) {
      const int g = C.cl_atoms[a0 + a];
      for (int r = 0; r < 3; ++r) pv[a][r] = v[3 * g + r];
      vel_op(op, g, pv[a], C.invm, sc);
      im[a] = C.invm[g];
    }
    double rr[kMaxClCons][3], lam[kMaxClCons], dd[kMaxClCons];
    int li[kMaxClCons], lj[kMaxClCons];
    for (int k = 0; k < nk; ++k) {
      const int4 q = C.cons[k0 + k];
      li[k] = q.x, lj[k] = q.y;
      dd[k] = C.d2[k0 + k];
      lam[k] = 0;
      double d0 = x[3 * q.z] - x[3 * q.w], d1 = x[3 * q.z + 1] - x[3 * q.w + 1], d2v = x[3 * q.z + 2] - x[3 * q.w + 2];
      min_image(C.cell, d0, d1, d2v);
      rr[k][0] = d0, rr[k][1] = d1, rr[k][2] = d2v;
    }
    bool done = false;
    for (int it = 0; it < kShakeIter && !done; ++it) {
      done = true;
      for (int k = 0; k < nk; ++k) {
        const int i = li[k], j = lj[k];
        const double rv = rr[k][0] * (pv[i][0] - pv[j][0]) + rr[k][1] * (pv[i][1] - pv[j][1]) + rr[k][2] * (pv[i][2] - pv[j][2]);
        if (fabs(rv) <= kShakeTol * dd[k]) continue;
        done = false;
        const double g = -rv / ((im[i] + im[j]) * dd[k]);
        lam[k] += g;
        for (int r = 0; r < 3; ++r) {
          pv[i][r] += g * im[i] * rr[k][r];
          pv[j][r] -= g * im[j] * rr[k][r];
        }
      }
    }
    if (!done) atomicOr(reinterpret_cast<unsigned*>(counters + kCntErr), kErrRattle);
    for (int a = 0; a < na; ++a) {
      const int g = C.cl_atoms[a0 + a];
      for (int r = 0; r < 3; ++r) v[3 * g + r] = pv[a][r];
    }
    if (h > 0)
      for (int k = 0; k < nk; ++k) {
        const double s = 2 * lam[k] / (h * kAcc);
        w[0] += s * rr[k][0] * rr[k][0];
        w[1] += s * rr[k][1] * rr[k][1];
        w[2] += s * rr[k][2] * rr[k][2];
        w[3] += s * rr[k][0] * rr[k][1];
        w[4] += s * rr[k][0] * rr[k][2];
        w[5] += s * rr[k][1] * rr[k][2];
      }
  }
  if (h > 0) {
    __shared__ double scratch[32];
    for (int q = 0; q < 6; ++q) {
      const double s = block_sum(w[q], scratch);
      if (threadIdx.x == 0 && s != 0) atomicAdd(sc + kScCW0 + q, s);
    }
  }
  // the kinetic energy of the updated velocities (this thread's atoms, read back) and the thermostat update, as k_ke
  if (K.n > 0) {
    double e = 0, t[6] = {0, 0, 0, 0, 0, 0};
    if (c >= C.ncl && c < C.ncl + nfree) {
      ke_atom(K, free_atoms[c - C.ncl], e, t);
    } else if (c < C.e3) {
      const int4 at = C.star[c];
      const int ids[4] = {at.x, at.y, at.z, at.w};
      for (int a = 0; a < 4; ++a)
        if (ids[a] >= 0) ke_atom(K, ids[a], e, t);
    } else if (c < C.e4) {
      const int4 at = C.water[c - C.e3];
      ke_atom(K, at.x, e, t);
      ke_atom(K, at.y, e, t);
      ke_atom(K, at.z, e, t);
    } else if (c < C.ncl) {
      const int cg = c - C.e4;
      for (int a = C.cl_atom0[cg]; a < C.cl_atom0[cg + 1]; ++a) ke_atom(K, C.cl_atoms[a], e, t);
    }
    ke_blocks(K, e, t);
  }
}


// Kinetic energy (and the kinetic tensor sum m v_a v_b / kAcc on request), then a thermostat update, in one launch:
// each block writes its partial sums; the last block to finish adds the partials in block order (deterministic) and
// runs the scalar update. No block waits on another.
__global__ void k_ke(KeArgs A) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double e = 0, t[6] = {0, 0, 0, 0, 0, 0};
  if (i < A.n) ke_atom(A, i, e, t);
  ke_blocks(A, e, t);
}

}  // namespace

// ---------------------------------------------------------------------------------------------------------------
// The MD state of one engine. It is kept by the engine between runs (Engine::stepper_), so that a run pays the set-up of
// its buffers, pinned scalars, constraint clusters and step graphs only when something they depend on has changed.
struct Stepper {
  Engine& E;
  caps_gpu_md_opts o{};   // the current run's options
  int n;
  DevBuf<double> x, v, x0, invm, m, sc, part;
  DevBuf<unsigned> done;       // k_ke's finished-block counter
  DevBuf<int> free_atoms;      // atoms in no constraint cluster
  int nfree = 0;
  DevBuf<Chain> chain;
  DevBuf<int> cl_start, cl_atom0, cl_atoms;
  DevBuf<int4> cons, star, water;
  DevBuf<double4> star_d2;
  DevBuf<double2> water_g;
  DevBuf<double> d2, dlen, cpc;   // LINCS: lengths, coupling coefficients
  DevBuf<int> cp_start;
  DevBuf<int2> cp;
  int cons_alg = -1;
  DevBuf<double2> draws;
  long long draws_first = 0, draws_count = 0;
  ConsArgs C{};
  int ncons = 0;
  double ndof = 0;
  bool nhc = false, bussi = false, langevin = false;
  double t_freq = 0;
  std::unique_ptr<HostRng> rng;
  double* h_sc = nullptr;
  Chain* h_chain = nullptr;
  double* h_xv = nullptr;   // pinned staging for a run's positions and velocities in and out (2 x 3N)
  size_t h_xv_n = 0;
  double* pinned_xv(size_t n3) {
    if (h_xv_n < n3) {
      if (h_xv) CK(cudaFreeHost(h_xv));
      h_xv = nullptr;
      CK(cudaMallocHost(&h_xv, 2 * n3 * sizeof(double)));
      h_xv_n = n3;
    }
    return h_xv;
  }
  // the captured plain step, thermo step (energies and virial on) and a block of kBlockSteps plain steps
  static constexpr int kBlockSteps = 8;
  cudaGraphExec_t graph[3] = {nullptr, nullptr, nullptr};
  std::string graph_key[3];                          // what each was captured with (capture_key)
  bool graph_valid[3] = {false, false, false};
  int graph_kernels[3] = {0, 0, 0};
  int nparts = 0;
  // kept between runs: host velocities, the copies for step 0's trial step, the masses, the constraint set and what it
  // was built from, the run's timing events
  std::vector<double> hv;
  DevBuf<double> xs, vs;
  bool masses_ready = false;
  // the run's masses: the force field's, or with hydrogen mass repartitioning (what they were made with: hmr, flags)
  std::vector<double> hm;
  double hm_hmr = -1;
  std::vector<int8_t> hm_h;
  long long hmr_moved = 0;
  bool hmr_kept = false;
  bool cons_built = false, cons_from_positions = false;
  int cons_flag = -1;
  std::vector<int8_t> cons_h, cons_o;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;

  explicit Stepper(Engine& e) : E(e), n(e.n_) {}
  ~Stepper() {
    for (auto& g : graph)
      if (g) cudaGraphExecDestroy(g);
    if (h_sc) cudaFreeHost(h_sc);
    if (h_xv) cudaFreeHost(h_xv);
    if (h_chain) cudaFreeHost(h_chain);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
  }

  // The constraint set of ConstraintMode::HBonds (core/src/constraints.cpp:40-103): every bond to a hydrogen at its r0
  // (or its present length without one), and rigid waters (an oxygen bonded to exactly two hydrogens: their H-H
  // distance from r0 and theta0). Connected constraints form a cluster, solved by one thread.
  void build_constraints(const double* hx) {
    std::vector<int8_t> hflags, oflags;
    if (o.constraints && o.is_hydrogen) hflags.assign(o.is_hydrogen, o.is_hydrogen + n);
    if (o.constraints && o.is_oxygen) oflags.assign(o.is_oxygen, o.is_oxygen + n);
    // the set depends on the options, the element flags and the force field; on the positions only where a bond has no
    // usable r0 or a water no angle
    if (cons_built && !cons_from_positions && cons_flag == o.constraints && cons_alg == o.constraint_algorithm && hflags == cons_h &&
        oflags == cons_o)
      return;
    cons_built = false;
    cons_alg = o.constraint_algorithm;
    const bool lincs = o.constraint_algorithm == 1;   // every cluster in the general layout, solved by LINCS
    cons_from_positions = false;
    ncons = 0;
    nfree = 0;
    C = ConsArgs{};
    C.invm = invm.p;
    cons_flag = o.constraints;
    cons_h = hflags;
    cons_o = oflags;
    if (!o.constraints) {
      cons_built = true;
      return;
    }
    const auto& hm = E.h_mass_;
    auto is_h = [&](int a) { return o.is_hydrogen ? o.is_hydrogen[a] != 0 : hm[size_t(a)] < 1.6; };
    auto is_o = [&](int a) { return o.is_oxygen ? o.is_oxygen[a] != 0 : false; };
    std::vector<std::array<uint32_t, 2>> bonds;
    std::vector<double> r0;
    for (size_t k = 0; k < E.hb_.size(); ++k) bonds.push_back(E.hb_[k]), r0.push_back(E.hr0_[k]);
    std::vector<std::vector<int>> nb(static_cast<size_t>(n));
    for (auto& b : bonds) nb[b[0]].push_back(int(b[1])), nb[b[1]].push_back(int(b[0]));
    auto dist = [&](int i, int j) {
      cons_from_positions = true;
      double d[3] = {hx[3 * j] - hx[3 * i], hx[3 * j + 1] - hx[3 * i + 1], hx[3 * j + 2] - hx[3 * i + 2]};
      min_image_host(d);
      return std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    };
    auto length = [&](int i, int j) {
      for (size_t k = 0; k < bonds.size(); ++k)
        if ((int(bonds[k][0]) == i && int(bonds[k][1]) == j) || (int(bonds[k][0]) == j && int(bonds[k][1]) == i))
          if (r0[k] > 0.3) return r0[k];
      return dist(i, j);
    };
    struct Cn { int i, j; double d; };
    std::vector<Cn> cs;
    for (size_t k = 0; k < bonds.size(); ++k) {
      const int i = int(bonds[k][0]), j = int(bonds[k][1]);
      if (!(is_h(i) || is_h(j))) continue;
      cs.push_back({i, j, r0[k] > 0.3 ? r0[k] : dist(i, j)});
    }
    for (int ox = 0; ox < n; ++ox) {
      if (!is_o(ox) || nb[size_t(ox)].size() != 2) continue;
      const int a = nb[size_t(ox)][0], b = nb[size_t(ox)][1];
      if (!is_h(a) || !is_h(b)) continue;
      const double da = length(ox, a), db = length(ox, b);
      double th = -1;
      for (size_t k = 0; k < E.ha_.size(); ++k) {
        const auto& t = E.ha_[k];
        if (int(t[1]) == ox && ((int(t[0]) == a && int(t[2]) == b) || (int(t[0]) == b && int(t[2]) == a))) th = E.hth0_[k];
      }
      if (th < 0) {
        cons_from_positions = true;
        double u[3] = {hx[3 * a] - hx[3 * ox], hx[3 * a + 1] - hx[3 * ox + 1], hx[3 * a + 2] - hx[3 * ox + 2]};
        double w[3] = {hx[3 * b] - hx[3 * ox], hx[3 * b + 1] - hx[3 * ox + 1], hx[3 * b + 2] - hx[3 * ox + 2]};
        min_image_host(u);
        min_image_host(w);
        const double c = (u[0] * w[0] + u[1] * w[1] + u[2] * w[2]) /
                         (std::sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]) * std::sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]));
        th = std::acos(std::max(-1.0, std::min(1.0, c)));
      }
      cs.push_back({a, b, std::sqrt(da * da + db * db - 2 * da * db * std::cos(th))});
    }
    ncons = int(cs.size());
    if (!ncons) {
      cons_built = true;
      return;
    }
    // clusters: connected components of the constraint graph
    std::vector<int> root(static_cast<size_t>(n));
    for (int i = 0; i < n; ++i) root[size_t(i)] = i;
    std::function<int(int)> find = [&](int a) { return root[size_t(a)] == a ? a : root[size_t(a)] = find(root[size_t(a)]); };
    for (auto& c : cs) root[size_t(find(c.i))] = find(c.j);
    std::map<int, std::vector<int>> comp_cons;
    for (int k = 0; k < ncons; ++k) comp_cons[find(cs[size_t(k)].i)].push_back(k);
    std::vector<int> st{0}, a0{0}, atoms, gen_atoms;   // atoms: every constrained atom; gen_atoms: the general clusters
    std::vector<int4> cv;
    std::vector<double> dv, dlv, cpcv;
    std::vector<int> cps{0};
    std::vector<int2> cpv;
    std::vector<int4> star_at[3], water_at;
    std::vector<double4> star_dd[3];
    std::vector<double2> water_geo;
    for (auto& comp : comp_cons) {
      const std::vector<int>& ks = comp.second;
      if (int(ks.size()) > kMaxClCons) throw ModelError(CAPS_GPU_EINVAL, "a constraint cluster has more than 8 atoms or constraints (the device SHAKE takes bonds to hydrogen and rigid waters)");
      // a star: 1-3 constraints that all share one atom, each with a distinct partner
      int centre = -1;
      if (!lincs && ks.size() <= 3) {
        const Cn& c0 = cs[size_t(ks[0])];
        for (int cand : {c0.i, c0.j}) {
          bool all = true;
          std::vector<int> partners;
          for (int k : ks) {
            const Cn& c = cs[size_t(k)];
            if (c.i != cand && c.j != cand) all = false;
            else partners.push_back(c.i == cand ? c.j : c.i);
          }
          std::vector<int> u = partners;
          std::sort(u.begin(), u.end());
          if (all && std::unique(u.begin(), u.end()) == u.end()) {
            centre = cand;
            break;
          }
        }
      }
      if (centre >= 0) {
        int4 a = make_int4(centre, -1, -1, -1);
        double dd[3] = {0, 0, 0};
        int q = 0;
        for (int k : ks) {
          const Cn& c = cs[size_t(k)];
          const int partner = c.i == centre ? c.j : c.i;
          (q == 0 ? a.y : q == 1 ? a.z : a.w) = partner;
          dd[q++] = c.d * c.d;
          atoms.push_back(partner);
        }
        atoms.push_back(centre);
        star_at[ks.size() - 1].push_back(a);
        star_dd[ks.size() - 1].push_back(make_double4(dd[0], dd[1], dd[2], 0.0));
        continue;
      }
      if (!lincs && ks.size() == 3) {
        // a rigid water: the atom shared by two equal constraints (O) and two partners of equal mass joined by the third
        const Cn& k0 = cs[size_t(ks[0])];
        const Cn& k1 = cs[size_t(ks[1])];
        const Cn& k2 = cs[size_t(ks[2])];
        int ox = -1;
        for (int cand : {k0.i, k0.j})
          if ((k1.i == cand || k1.j == cand) && !(k2.i == cand || k2.j == cand)) ox = cand;
        if (ox >= 0) {
          const int h1 = k0.i == ox ? k0.j : k0.i, h2 = k1.i == ox ? k1.j : k1.i;
          const bool tri = ((k2.i == h1 && k2.j == h2) || (k2.i == h2 && k2.j == h1)) && h1 != h2;
          const bool eq_len = std::fabs(k0.d - k1.d) <= 1e-12 * k0.d;
          const bool eq_mass = E.h_mass_[size_t(h1)] == E.h_mass_[size_t(h2)];
          if (tri && eq_len && eq_mass) {
            water_at.push_back(make_int4(ox, h1, h2, -1));
            water_geo.push_back(make_double2(k0.d, k2.d));
            atoms.push_back(ox), atoms.push_back(h1), atoms.push_back(h2);
            continue;
          }
        }
      }
      std::vector<int> loc;
      auto local = [&](int a) {
        for (size_t q = 0; q < loc.size(); ++q)
          if (loc[q] == a) return int(q);
        loc.push_back(a);
        return int(loc.size() - 1);
      };
      for (int k : ks) {
        const Cn& c = cs[size_t(k)];
        const int li = local(c.i), lj = local(c.j);
        cv.push_back(make_int4(li, lj, c.i, c.j));
        dv.push_back(c.d * c.d);
        dlv.push_back(c.d);
      }
      if (lincs) {
        // the couplings in the reference's order (constraints.cpp:110-119): atoms ascending, then each pair (k, l), k != l,
        // of the constraints on the atom in constraint order; S_k = 1 / sqrt(1/m_i + 1/m_j)
        auto inv = [&](int a) { return hm[size_t(a)] > 0 ? 1.0 / hm[size_t(a)] : 0.0; };
        auto S = [&](int k) {
          const Cn& c = cs[size_t(ks[size_t(k)])];
          return 1.0 / std::sqrt(inv(c.i) + inv(c.j));
        };
        std::vector<int> sorted = loc;
        std::sort(sorted.begin(), sorted.end());
        for (int a : sorted) {
          std::vector<int> on;
          for (int k = 0; k < int(ks.size()); ++k) {
            const Cn& c = cs[size_t(ks[size_t(k)])];
            if (c.i == a || c.j == a) on.push_back(k);
          }
          for (int k : on)
            for (int l : on) {
              if (k == l) continue;
              const double sk = cs[size_t(ks[size_t(k)])].i == a ? 1.0 : -1.0, sl = cs[size_t(ks[size_t(l)])].i == a ? 1.0 : -1.0;
              cpv.push_back(make_int2(k, l));
              cpcv.push_back(-S(k) * S(l) * sk * sl * inv(a));
            }
        }
        if (int(cpv.size()) - cps.back() > kMaxCouple) throw ModelError(CAPS_GPU_EINVAL, "a constraint cluster couples more than 56 constraint pairs (LINCS)");
        cps.push_back(int(cpv.size()));
      }
      if (int(loc.size()) > kMaxClAtoms)
        throw ModelError(CAPS_GPU_EINVAL, "a constraint cluster has more than 8 atoms or constraints (the device SHAKE takes bonds to hydrogen and rigid waters)");
      gen_atoms.insert(gen_atoms.end(), loc.begin(), loc.end());
      atoms.insert(atoms.end(), loc.begin(), loc.end());
      st.push_back(int(cv.size()));
      a0.push_back(int(gen_atoms.size()));
    }
    std::vector<int4> sa;
    std::vector<double4> sd;
    for (int k = 0; k < 3; ++k) {
      sa.insert(sa.end(), star_at[k].begin(), star_at[k].end());
      sd.insert(sd.end(), star_dd[k].begin(), star_dd[k].end());
    }
    C.e1 = int(star_at[0].size());
    C.e2 = C.e1 + int(star_at[1].size());
    C.e3 = C.e2 + int(star_at[2].size());
    if (!sa.empty()) {
      star.upload(sa, E.stream_);
      star_d2.upload(sd, E.stream_);
    }
    C.star = star.p;
    C.star_d2 = star_d2.p;
    C.e4 = C.e3 + int(water_at.size());
    if (!water_at.empty()) {
      water.upload(water_at, E.stream_);
      water_g.upload(water_geo, E.stream_);
    }
    C.water = water.p;
    C.water_geo = water_g.p;
    std::vector<char> in_cluster(static_cast<size_t>(n), 0);
    for (int a : atoms) in_cluster[size_t(a)] = 1;
    std::vector<int> fa;
    for (int a = 0; a < n; ++a)
      if (!in_cluster[size_t(a)]) fa.push_back(a);
    nfree = int(fa.size());
    if (nfree) free_atoms.upload(fa, E.stream_);
    cl_start.upload(st, E.stream_);
    cl_atom0.upload(a0, E.stream_);
    if (!gen_atoms.empty()) {
      cl_atoms.upload(gen_atoms, E.stream_);
      cons.upload(cv, E.stream_);
      d2.upload(dv, E.stream_);
    }
    C.lincs = lincs ? 1 : 0;
    if (lincs) {
      dlen.upload(dlv, E.stream_);
      cp_start.upload(cps, E.stream_);
      if (!cpv.empty()) {
        cp.upload(cpv, E.stream_);
        cpc.upload(cpcv, E.stream_);
      }
      C.dlen = dlen.p;
      C.cp_start = cp_start.p;
      C.cp = cp.p;
      C.cpc = cpc.p;
    }
    C.ncl = C.e4 + int(st.size()) - 1;
    C.cl_start = cl_start.p;
    C.cl_atom0 = cl_atom0.p;
    C.cl_atoms = cl_atoms.p;
    C.cons = cons.p;
    C.d2 = d2.p;
    C.invm = invm.p;
    CK(cudaStreamSynchronize(E.stream_));
    cons_built = true;
  }

  void min_image_host(double* d) const {
    const DevCell& c = E.dcell_;
    double f[3];
    for (int r = 0; r < 3; ++r) {
      f[r] = c.hi[r][0] * d[0] + c.hi[r][1] * d[1] + c.hi[r][2] * d[2];
      f[r] -= std::nearbyint(f[r]);
    }
    for (int r = 0; r < 3; ++r) d[r] = c.h[r][0] * f[0] + c.h[r][1] * f[1] + c.h[r][2] * f[2];
  }

  // The captured steps no longer match the run (new thermostat draws, a rescaled cell): the next launch captures again
  // and updates the instantiated graph in place.
  void drop_graphs() { graph_valid[0] = graph_valid[1] = graph_valid[2] = false; }

  // Everything a capture of step() records besides the kernels themselves: the engine's capture state and this run's
  // scalars and buffers. Equal keys give equal graphs.
  std::string capture_key(bool thermo) const {
    std::string k = E.capture_state();
    auto put = [&k](const void* p, size_t bytes) { k.append(static_cast<const char*>(p), bytes); };
    const double dv[] = {o.dt, o.temperature, o.temperature_end, o.tau_t, ndof, t_freq};
    put(dv, sizeof dv);
    const long long iv[] = {(long long)o.steps, (long long)o.seed, o.thermostat, o.respa, o.respa_split, o.constraints, draws_first,
                            ncons, nfree, nparts, respa, slow_parts, fast_parts, thermo ? 1 : 0};
    put(iv, sizeof iv);
    put(&C, sizeof C);
    const void* ptrs[] = {x.p, v.p, x0.p, invm.p, m.p, sc.p, part.p, done.p, chain.p, draws.p, free_atoms.p, f_slow.p, f_fast.p};
    put(ptrs, sizeof ptrs);
    return k;
  }

  // Replays the step graph. It is captured when the run's key differs from the one it was made with; an instantiated
  // graph is then updated in place (cudaGraphExecUpdate), and instantiated anew only if the update is refused.
  // Returns its kernel count.
  int launch_step(bool thermo) {
    const int k = thermo ? 1 : 0;
    ensure_graph(thermo);
    if (k == 0) E.graph_kernels_ = graph_kernels[k];
    CK(cudaGraphLaunch(graph[k], E.stream_));
    return graph_kernels[k];
  }
  // Replays kBlockSteps plain steps as one graph (no launch gap between them); returns its kernel count.
  int launch_block() {
    ensure_graph(false, true);
    CK(cudaGraphLaunch(graph[2], E.stream_));
    return graph_kernels[2];
  }
  // Captures (or updates) the plain or thermo step graph, or the block of plain steps, when the run's key differs from
  // the one it was made with.
  void ensure_graph(bool thermo, bool block = false) {
    const int k = block ? 2 : thermo ? 1 : 0;
    std::string key = capture_key(thermo) + (block ? "B" : "");
    if (!graph[k] || !graph_valid[k] || key != graph_key[k]) {
      cudaGraph_t g;
      CK(cudaStreamBeginCapture(E.stream_, cudaStreamCaptureModeThreadLocal));
      try {
        for (int i = 0; i < (block ? kBlockSteps : 1); ++i) step(thermo, thermo);
      } catch (...) {   // leave no capture open behind an error
        cudaGraph_t junk = nullptr;
        (void)cudaStreamEndCapture(E.stream_, &junk);
        if (junk) cudaGraphDestroy(junk);
        (void)cudaGetLastError();
        throw;
      }
      CK(cudaStreamEndCapture(E.stream_, &g));
      size_t nn = 0;
      CK(cudaGraphGetNodes(g, nullptr, &nn));
      std::vector<cudaGraphNode_t> nodes(nn);
      CK(cudaGraphGetNodes(g, nodes.data(), &nn));
      int kernels = 0;
      for (auto nd : nodes) kernels += is_kernel_node(nd);
      graph_kernels[k] = kernels;
      bool updated = false;
      if (graph[k]) {
        cudaGraphExecUpdateResultInfo info{};
        updated = cudaGraphExecUpdate(graph[k], g, &info) == cudaSuccess;
        if (!updated) {
          (void)cudaGetLastError();   // the refusal is not an error of the run
          CK(cudaGraphExecDestroy(graph[k]));
          graph[k] = nullptr;
        }
      }
      if (!updated) CK(cudaGraphInstantiate(&graph[k], g, cudaGraphInstantiateFlagUseNodePriority));
      CK(cudaGraphDestroy(g));
      // the capture state is read after the capture: step() may have changed host flags it holds
      graph_key[k] = capture_key(thermo) + (block ? "B" : "");
      graph_valid[k] = graph_key[k] == key;
    }
  }

  // --- step pieces (all asynchronous on E.stream_) ---
  KeArgs ke_args(int slot, bool tensor) const {
    KeArgs A{};
    A.n = n;
    A.v = v.p;
    A.m = m.p;
    A.part = part.p;
    A.done = done.p;
    A.sc = sc.p;
    A.slot = slot;
    A.tensor = tensor ? 1 : 0;
    A.t0 = o.temperature;
    A.t1 = o.temperature_end;
    A.steps = (long long)o.steps;
    A.ndof = ndof;
    A.chain = chain.p;
    A.t_freq = t_freq;
    A.dt = o.dt;
    A.draws = draws.p;
    A.draws_first = draws_first;
    A.tau = o.tau_t;
    return A;
  }
  void ke_launch(const KeArgs& A) { launch_k(k_ke, nparts, 256, 0, E.stream_, A); }
  void ke(int slot, bool tensor) { ke_launch(ke_args(slot, tensor)); }
  // half kick, then drift with SHAKE; `scale` applies the thermostat's pending factor first
  // kick + drift, then SHAKE; the kick also clears the force evaluation's atom-order sums for the evaluation that
  // follows (Engine::forces then skips its own clearing)
  // check: the list's displacement check runs in the drift (no constraints) or in SHAKE, and the force evaluation that
  // follows skips its own
  void kick_drift(double hk, double hd, bool scale, bool zero_cw, const double* f = nullptr, const double* f2 = nullptr, double hk2 = 0,
                  int step_ahead = 0, bool check = false) {
    KickArgs K{n, x.p, v.p, x0.p, f ? f : E.d_f_.p, invm.p, hk, f2, hk2, hd, sc.p, scale ? 1 : 0, zero_cw ? 1 : 0, E.d_counters_.p,
               E.mixed_ ? E.d_F_.p : nullptr, E.mixed_ ? nullptr : E.d_Fd_.p, E.d_errinfo_.p, step_ahead};
    const ListCheck L = check ? E.list_check(nfree, free_atoms.p) : ListCheck{};
    launch_k(k_kick_drift, blocks(size_t(n), 256), 256, 0, E.stream_, K, ncons ? ListCheck{} : L);
    if (ncons) launch_k(C.lincs ? k_lincs : k_shake, blocks(size_t(C.ncl) + (check ? size_t(nfree) : 0), 128), 128, 0, E.stream_, C, x.p, x0.p, v.p, hd, E.d_counters_.p, L);
    E.sums_cleared_ = true;
  }
  // whether this step's drift may take the list's displacement check (a plain step: not r-RESPA)
  bool fuse_check() const { return respa <= 1 && E.list_check_fusable(); }
  // a velocity update, then RATTLE (constraint virial summed when h > 0); with ke, also the kinetic energy and ke's
  // thermostat update (constraints only: the caller launches k_ke otherwise)
  void vel_rattle(const VelOp& op, double h, const KeArgs* ke = nullptr) {
    if (!ncons) {
      if (op.kind != 0) launch_k(k_vel, blocks(size_t(n), 256), 256, 0, E.stream_, n, v.p, invm.p, sc.p, op);
      return;
    }
    KeArgs K{};
    if (ke) K = *ke;
    launch_k(k_vel_rattle, blocks(size_t(C.ncl + nfree), 128), 128, 0, E.stream_, C, nfree, free_atoms.p, x.p, v.p, op, h, sc.p, E.d_counters_.p, K);
  }
  VelOp kick_op(double hk) const { return VelOp{1, E.d_f_.p, hk, 0, 0, 0, nullptr, 0}; }
  // the kick from the force evaluation's sums (its reduction skipped), storing the forces to E.d_f_
  VelOp kick_op_sums(double hk) const {
    VelOp op = kick_op(hk);
    op.f = nullptr;
    const bool pairs = (E.opt_.parts & 2) != 0;
    if (E.mixed_) op.fq = E.d_F_.p, op.fsq = pairs ? E.d_Fs_.p : nullptr;
    else op.fd = E.d_Fd_.p, op.fsd = pairs ? E.d_Fsd_.p : nullptr;
    op.iperm = pairs ? E.d_iperm_.p : nullptr;
    op.nat = n;
    op.nslots = int(size_t(E.nsc_cap_) * kScAtoms);
    op.fout = E.d_f_.p;
    return op;
  }
  // the kick + RATTLE + kinetic energy + thermostat tail in one launch (constraints, no r-RESPA)
  bool fused_tail() const { return ncons > 0 && respa == 1; }
  void rattle(double h) {   // RATTLE alone (initial velocities)
    if (ncons) vel_rattle(VelOp{0, nullptr, 0, 0, 0, 0, nullptr, 0}, h);
  }
  void scale_v() { launch_k(k_scale_v, blocks(size_t(3) * n, 256), 256, 0, E.stream_, n, v.p, sc.p); }
  // r-RESPA force sets (dynamics.cpp:113-122, 318-326): the non-bonded (slow) and bonded (fast) parts in their own
  // arrays; the evaluation at the end of a step computes both, with energies and virial summed over the two.
  // The PME split puts the reciprocal sum (and its exclusion corrections) in the slow set and every other term in the
  // fast one. Part masks as Engine::forces takes them.
  DevBuf<double> f_slow, f_fast;
  int respa = 1, slow_parts = 6, fast_parts = 1;
  // checked: the drift before ran the list's displacement check
  void forces(bool ener, bool vir, bool reduce = true, bool checked = false) {
    if (respa > 1) {
      E.forces(x.p, ener, vir, true, slow_parts, f_slow.p, true);
      E.forces(x.p, ener, vir, true, fast_parts, f_fast.p, false);
      return;
    }
    E.forces(x.p, ener, vir, !checked, -1, nullptr, true, reduce);
  }
  void fast_forces() { E.forces(x.p, false, false, true, fast_parts, f_fast.p, true); }

  // One MD step (dynamics.cpp:606-666), energies and virial on request. Kernel sequence per step: NVT Nose-Hoover
  // chain (on the kinetic energy the last step left), kick+drift, SHAKE, forces, kick+RATTLE+KE+chain (with constraints
  // the kick reads the force sums and the kinetic energy and chain update run in the RATTLE launch's last block), scale;
  // Bussi step-begin, kick+drift, SHAKE, forces, kick+RATTLE+KE+Bussi, scale; Langevin (BAOAB) kick+drift, SHAKE, KE,
  // O+RATTLE, KE+bath, drift, SHAKE, forces, kick+RATTLE.
  void step(bool ener, bool vir) {
    const double dt = o.dt;
    const double hw = vir ? dt : 0.0;   // the constraint virial only on steps that report it
    if (respa > 1) {
      // r-RESPA (dynamics.cpp:643-657): outer half kick with the slow forces; `respa` velocity-Verlet steps of dt/respa
      // with the fast ones; outer half kick. Adjacent kicks with the same forces are merged.
      const double h = dt / respa;
      launch_k(k_step_begin, 1, 1, 0, E.stream_, sc.p, o.temperature, o.temperature_end, (long long)o.steps, ndof);
      kick_drift(0.5 * dt, h, false, true, f_slow.p, f_fast.p, 0.5 * h);
      for (int j = 0; j + 1 < respa; ++j) {
        fast_forces();
        kick_drift(h, h, false, false, f_fast.p);
      }
      forces(ener, vir);
      vel_rattle(VelOp{1, f_fast.p, 0.5 * h, 0, 0, 0, f_slow.p, 0.5 * dt}, hw);
      if (bussi) {
        KeArgs A = ke_args(kScKE, false);
        A.then = kThenBussi;
        ke_launch(A);
        scale_v();
      }
      return;
    }
    if (langevin) {
      const double c1 = std::exp(-dt / std::max(o.tau_t, 1e-9)), c2 = std::sqrt(1 - c1 * c1);
      kick_drift(0.5 * dt, 0.5 * dt, false, true, nullptr, nullptr, 0, 1);
      KeArgs A = ke_args(kScKE0, false);
      A.begin = 1;
      ke_launch(A);
      vel_rattle(VelOp{2, nullptr, 0, c1, c2, o.seed, nullptr, 0}, 0);
      A = ke_args(kScKE, false);
      A.then = kThenBath;
      ke_launch(A);
      const bool chk = fuse_check();
      kick_drift(0, 0.5 * dt, false, false, nullptr, nullptr, 0, 0, chk);
      forces(ener, vir, true, chk);
      vel_rattle(kick_op(0.5 * dt), hw);
    } else if (nhc) {
      launch_k(k_nhc_begin, 1, 1, 0, E.stream_, chain.p, sc.p, o.temperature, o.temperature_end, (long long)o.steps, ndof, t_freq, dt);
      const bool chk = fuse_check();
      kick_drift(0.5 * dt, dt, true, true, nullptr, nullptr, 0, 0, chk);
      KeArgs A = ke_args(kScKE, false);
      A.then = kThenNhc;
      if (fused_tail()) {
        forces(ener, vir, false, chk);
        vel_rattle(kick_op_sums(0.5 * dt), hw, &A);
      } else {
        forces(ener, vir, true, chk);
        vel_rattle(kick_op(0.5 * dt), hw);
        ke_launch(A);
      }
      scale_v();
    } else {
      launch_k(k_step_begin, 1, 1, 0, E.stream_, sc.p, o.temperature, o.temperature_end, (long long)o.steps, ndof);
      const bool chk = fuse_check();
      kick_drift(0.5 * dt, dt, false, true, nullptr, nullptr, 0, 0, chk);
      KeArgs A = ke_args(kScKE, false);
      A.then = kThenBussi;
      if (fused_tail()) {
        forces(ener, vir, false, chk);
        vel_rattle(kick_op_sums(0.5 * dt), hw, bussi ? &A : nullptr);
      } else {
        forces(ener, vir, true, chk);
        vel_rattle(kick_op(0.5 * dt), hw);
        if (bussi) ke_launch(A);
      }
      if (bussi) scale_v();
    }
  }

  // Bussi draws for steps [first, first + count): r1 = gauss, then the chi-squared of ndof - 1 by a fresh Gamma
  static constexpr long long kDrawChunk = 4096;   // draws made ahead at most (the buffer holds one chunk and one more)
  void make_draws(long long first, long long count) {
    std::vector<double2> d(static_cast<size_t>(count));
    for (long long s = 0; s < count; ++s) {
      const double r1 = rng->gauss();
      const double sum = ndof > 1 ? rng->gamma((ndof - 1) / 2, 2.0) : 0.0;
      d[size_t(s)] = make_double2(r1, sum);
    }
    draws.upload(d, E.stream_);
    draws_first = first;
    draws_count = count;
  }
};

void StepperDeleter::operator()(Stepper* s) const { delete s; }

void Engine::drop_run_state() {
  if (stream_) CK(cudaStreamSynchronize(stream_));
  stepper_.reset();
}

void Engine::validate_md(const caps_gpu_md_opts& o) const {
  if (n_ < 2) throw ModelError(CAPS_GPU_EFIELD, "dynamics needs at least two atoms");
  if (frozen_) throw ModelError(CAPS_GPU_EINVAL, "the pair list is frozen (freeze_pairs): unfreeze it before dynamics");
  if (o.dt <= 0 || o.dt > 50) throw ModelError(CAPS_GPU_EINVAL, "time step must be in (0, 50] fs");
  if (o.steps < 0) throw ModelError(CAPS_GPU_EINVAL, "the number of steps must be 0 or more");
  if (o.respa < 0 || o.respa > 16) throw ModelError(CAPS_GPU_EINVAL, "r-RESPA inner steps must be 1 … 16");
  if (o.respa > 1 && (o.thermostat == 2 || o.thermostat == 3)) throw ModelError(CAPS_GPU_EINVAL, "r-RESPA runs with the Bussi thermostat or none");
  if (o.respa > 1 && o.constraints) throw ModelError(CAPS_GPU_EINVAL, "r-RESPA and bond constraints are alternatives: choose one");
  if (o.respa_split != 0 && o.respa_split != 1) throw ModelError(CAPS_GPU_EINVAL, "unknown r-RESPA split");
  if (o.thermostat < 0 || o.thermostat > 3) throw ModelError(CAPS_GPU_EINVAL, "unknown thermostat");
  if (o.barostat < 0 || o.barostat > 3) throw ModelError(CAPS_GPU_EINVAL, "unknown barostat (none, crescale, berendsen, mtk)");
  // the reference's checks for MTK (dynamics.cpp:93-94, 103-106)
  if (o.barostat == 3 && o.respa > 1) throw ModelError(CAPS_GPU_EINVAL, "r-RESPA runs with the Bussi thermostat or none");
  if (o.barostat == 3 && o.anisotropic)
    throw ModelError(CAPS_GPU_EINVAL, "the MTK barostat couples the volume isotropically; per-axis coupling and deformation use Berendsen");
  if (o.barostat == 3 && o.constraints)
    throw ModelError(CAPS_GPU_EINVAL, "the MTK barostat runs without bond constraints; use the stochastic cell rescaling barostat with constraints");
  if (o.barostat == 3 && !(o.thermostat == 3 || o.thermostat == 0))
    throw ModelError(CAPS_GPU_EINVAL, "the MTK barostat pairs with the Nosé–Hoover thermostat (NPT) or none (NPH)");
  if (o.barostat == 1 && o.thermostat == 0) throw ModelError(CAPS_GPU_EINVAL, "stochastic cell rescaling needs a thermostat");
  if (o.anisotropic && o.barostat == 1) throw ModelError(CAPS_GPU_EINVAL, "per-axis pressure coupling is available with the Berendsen barostat");
  if (o.hmr < 0 || !std::isfinite(o.hmr)) throw ModelError(CAPS_GPU_EINVAL, "the repartitioned hydrogen mass must be 0 (off) or positive");
  if (o.constraint_algorithm != 0 && o.constraint_algorithm != 1) throw ModelError(CAPS_GPU_EINVAL, "unknown constraint algorithm (shake | lincs)");
}

// A stop asked for from outside (caps_gpu_request_stop): read once per step by the run loops.
std::atomic<int> g_stop{0};

// Frames and checkpoints leave the device through a ring of snapshot slots. At a recorded step the run's stream copies x
// (and v, for a checkpoint) into a slot's device buffers, which takes a microsecond, and a copy stream moves them into
// the slot's pinned host buffers while the next steps run. The callbacks get the slots in step order at the next step
// that reports or records, once the device has queued that step's work, or when the ring is full, or at the end of the
// run: the host writes a frame while the device integrates the steps after it.
struct SnapRing {
  static constexpr int kSlots = 4;
  struct Slot {
    DevBuf<double> dx, dv;
    double* hx = nullptr;
    double* hv = nullptr;
    double cell[12];
    long long step = 0;
    bool frame = false;
    int checkpoints = 0;   // 2: a regular checkpoint and the one a stop takes, both of this step (dynamics.cpp:759-770)
    cudaEvent_t copied = nullptr;
  };
  Slot slot[kSlots];
  int head = 0, count = 0;
  cudaStream_t cs = nullptr;
  cudaEvent_t taken = nullptr;
  size_t n3 = 0;
  ~SnapRing() {
    if (cs) cudaStreamSynchronize(cs);
    for (auto& q : slot) {
      if (q.hx) cudaFreeHost(q.hx);
      if (q.hv) cudaFreeHost(q.hv);
      if (q.copied) cudaEventDestroy(q.copied);
    }
    if (taken) cudaEventDestroy(taken);
    if (cs) cudaStreamDestroy(cs);
  }
  void init(size_t n) {
    if (cs) return;
    n3 = n;
    CK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&taken, cudaEventDisableTiming));
    for (auto& q : slot) CK(cudaEventCreateWithFlags(&q.copied, cudaEventDisableTiming));
  }
  // copies of x (and v) of the stream's current step into the next slot; the ring must have room
  void take(cudaStream_t st, const double* x, const double* v, const double* cell, long long step, bool frame, int checkpoints) {
    Slot& q = slot[(head + count) % kSlots];
    q.dx.alloc(n3);
    if (!q.hx) CK(cudaMallocHost(&q.hx, n3 * sizeof(double)));
    CK(cudaMemcpyAsync(q.dx.p, x, n3 * sizeof(double), cudaMemcpyDeviceToDevice, st));
    if (checkpoints > 0) {
      q.dv.alloc(n3);
      if (!q.hv) CK(cudaMallocHost(&q.hv, n3 * sizeof(double)));
      CK(cudaMemcpyAsync(q.dv.p, v, n3 * sizeof(double), cudaMemcpyDeviceToDevice, st));
    }
    CK(cudaEventRecord(taken, st));
    CK(cudaStreamWaitEvent(cs, taken, 0));
    CK(cudaMemcpyAsync(q.hx, q.dx.p, n3 * sizeof(double), cudaMemcpyDeviceToHost, cs));
    if (checkpoints > 0) CK(cudaMemcpyAsync(q.hv, q.dv.p, n3 * sizeof(double), cudaMemcpyDeviceToHost, cs));
    CK(cudaEventRecord(q.copied, cs));
    std::memcpy(q.cell, cell, sizeof q.cell);
    q.step = step;
    q.frame = frame;
    q.checkpoints = checkpoints;
    ++count;
  }
};

// One replica's run_dynamics on the device: set-up to step 0 (start), one step (advance), the state back (finish).
// Engine::run drives one; caps_gpu_run_batch drives several in lock step, their plain steps in one graph.
struct MdRun {
  Engine& E;
  const caps_gpu_md_opts& o;
  caps_gpu_state* st;
  caps_gpu_progress_fn progress;
  caps_gpu_frame_fn frame;
  void* user;
  Stepper& S;
  size_t n3;
  std::vector<double>& hv;
  int thermo_every = 1, baro_every = 1;
  long long kernels = 0, emits = 0, baro_steps = 0;
  int generation = 0;   // bumped whenever this replica's captured step changes (its graphs are dropped)
  SnapRing snaps;
  long long stopped_at = -1;   // the step a stop ended the run at
  bool completed = false;      // the run reached its end (or its stop) without an error

  // The engine's kept MD state, made on its first run.
  static Stepper& kept_state(Engine& e) {
    if (!e.stepper_) e.stepper_.reset(new Stepper(e));
    return *e.stepper_;
  }
  MdRun(Engine& e, caps_gpu_state* state, const caps_gpu_md_opts* md, caps_gpu_progress_fn prog, caps_gpu_frame_fn fr, void* u)
      : E(e), o(*md), st(state), progress(prog), frame(fr), user(u), S(kept_state(e)), n3(size_t(3) * e.n_), hv(S.hv) {
    S.o = *md;
  }
  // a run that ended in an error may have left its captured steps half-way: the next run captures them again
  ~MdRun() {
    if (!completed) S.drop_graphs();
  }

  double host_ke(const std::vector<double>& vv) const {
    double k = 0;
    for (int i = 0; i < E.n_; ++i)
      k += S.hm[size_t(i)] * (vv[3 * i] * vv[3 * i] + vv[3 * i + 1] * vv[3 * i + 1] + vv[3 * i + 2] * vv[3 * i + 2]);
    return 0.5 * k / kAcc;
  }

  void row(long long step, caps_gpu_thermo& r) {
    caps_gpu_terms t{};
    E.read_terms(&t, true, true);
    const double* sc = S.h_sc;
    for (int c = 0; c < 6; ++c) t.w[c] += sc[kScCW0 + c];
    t.virial = t.w[0] + t.w[1] + t.w[2];
    std::memset(&r, 0, sizeof r);
    r.step = step + o.step_offset;
    r.time_ps = double(step + o.step_offset) * o.dt * 1e-3;
    r.target_temperature = (o.temperature_end >= 0 && o.steps > 0) ? o.temperature + (o.temperature_end - o.temperature) * double(step) / double(o.steps)
                                                                  : o.temperature;
    r.kinetic = sc[kScKE];
    r.temperature = 2 * r.kinetic / (S.ndof * kB);
    r.potential = t.bond + t.angle + t.dihedral + t.improper + t.vdw + t.coulomb;
    r.total = r.potential + r.kinetic;
    r.volume = E.dcell_.vol;
    double mtot = 0;
    for (double mm : E.h_mass_) mtot += mm;
    r.density = mtot / kNA / (r.volume * 1e-24);
    r.pressure = (2 * r.kinetic + t.virial) / (3 * r.volume) * kAtm;
    for (int c = 0; c < 6; ++c) r.p[c] = (sc[kScKin0 + c] + t.w[c]) / r.volume * kAtm;
    if (S.nhc || mtk()) {
      // the extended system's energy (LAMMPS fix nh compute_scalar, dynamics.cpp:369-381)
      const double kt = kB * r.target_temperature;
      double e = 0;
      if (S.nhc) {
        const Chain& ch = *S.h_chain;
        e += S.ndof * kt * ch.eta[0] + 0.5 * ch.eta_mass[0] * ch.eta_dot[0] * ch.eta_dot[0];
        for (int c = 1; c < 3; ++c) e += kt * ch.eta[c] + 0.5 * ch.eta_mass[c] * ch.eta_dot[c] * ch.eta_dot[c];
      }
      if (mtk()) {
        e += 3 * 0.5 * omega_mass * omega_dot * omega_dot + o.pressure * (r.volume - vol0) / kAtm;
        e += 3 * kt * etap[0] + 0.5 * etap_mass[0] * etap_dot[0] * etap_dot[0];
        for (int c = 1; c < 3; ++c) e += kt * etap[c] + 0.5 * etap_mass[c] * etap_dot[c] * etap_dot[c];
      }
      r.conserved = r.total + e;
    } else {
      r.conserved = r.total + sc[kScBath] + (o.barostat ? o.pressure * r.volume / kAtm : 0.0);
    }
    r.terms = t;
  }
  void sync_scalars() {
    cudaStream_t stream_ = E.stream_;
    CK(cudaMemcpyAsync(S.h_sc, S.sc.p, sizeof(double) * kScNum, cudaMemcpyDeviceToHost, stream_));
    CK(cudaMemcpyAsync(S.h_chain, S.chain.p, sizeof(Chain), cudaMemcpyDeviceToHost, stream_));
    CK(cudaMemcpyAsync(E.h_counters_, E.d_counters_.p, sizeof(int) * kCntNum, cudaMemcpyDeviceToHost, stream_));
    CK(cudaMemcpyAsync(E.h_efix_, E.d_efix_.p, sizeof(long long) * kENumSlots, cudaMemcpyDeviceToHost, stream_));
    CK(cudaMemcpyAsync(E.h_edbl_, E.d_edbl_.p, sizeof(double) * kENumSlots, cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
    E.check_errors();
  }
  void emit(long long step) {
    S.ke(kScKE, true);
    sync_scalars();
    caps_gpu_thermo r;
    row(step, r);
    if (progress && progress(&r, user) != 0) throw ModelError(CAPS_GPU_ECANCEL, "dynamics cancelled");
  }
  bool frame_due(long long s) const { return frame && o.frame_every > 0 && (s % o.frame_every == 0 || s == o.steps); }
  bool checkpoint_due(long long s) const { return o.checkpoint && o.checkpoint_every > 0 && s % o.checkpoint_every == 0 && s < o.steps; }
  // a snapshot of step s for its frame and checkpoints
  void take(long long s, bool fr, int checkpoints) {
    if (!fr && checkpoints == 0) return;
    snaps.init(n3);
    if (snaps.count == SnapRing::kSlots) deliver_one();
    snaps.take(E.stream_, S.x.p, S.v.p, E.cell_h_, s, fr, checkpoints);
  }
  // the oldest snapshot to its callbacks, once its copy is in host memory; a checkpoint only of a state whose coordinates
  // and velocities are all finite (dynamics.cpp:758-760)
  void deliver_one() {
    SnapRing::Slot& q = snaps.slot[snaps.head];
    CK(cudaEventSynchronize(q.copied));
    snaps.head = (snaps.head + 1) % SnapRing::kSlots;
    --snaps.count;
    const long long step = q.step + o.step_offset;
    if (q.frame) frame(q.hx, q.cell, step, user);
    if (q.checkpoints > 0) {
      bool finite = true;
      for (size_t k = 0; k < n3 && finite; ++k) finite = std::isfinite(q.hx[k]) && std::isfinite(q.hv[k]);
      if (finite)
        for (int c = 0; c < q.checkpoints; ++c) o.checkpoint(q.hx, q.hv, q.cell, step, o.checkpoint_user);
    }
  }
  // every snapshot of a step before `before`
  void deliver(long long before) {
    while (snaps.count > 0 && snaps.slot[snaps.head].step < before) deliver_one();
  }
  // a stop after step s, whose regular frame and checkpoint have been taken: the stop's own checkpoint, every callback
  void stop_here(long long s) {
    take(s, false, o.checkpoint ? 1 : 0);
    deliver(s + 1);
    stopped_at = s;
  }
  bool refill_due(long long s) const { return S.bussi && s - S.draws_first >= S.draws_count; }
  // Bussi draws are made ahead for steps [s, s + chunk). With the barostat on, a chunk ends at the next barostat step:
  // the reference draws each step's thermostat numbers and then, on a barostat step, the barostat's normal from the
  // same stream (dynamics.cpp:665, 709-711), so the host stream is consumed in that order.
  long long draw_chunk(long long s) const {
    long long c = std::min<long long>(std::max<long long>(o.steps - s + 1, 1), Stepper::kDrawChunk);
    if (o.barostat) {
      const long long be = std::max(1, o.barostat_every);
      const long long next = (s + be - 1) / be * be;
      c = std::min(c, next - s + 1);
    }
    return c;
  }
  bool baro_due(long long s) const { return (o.barostat == 1 || o.barostat == 2) && s % baro_every == 0; }
  // The MTK barostat (Barostat::MTK, LAMMPS fix npt / nph as dynamics.cpp:479-570, 628-642): every step on the host's
  // schedule, outside the graphs (the cell moves twice a step); the barostat's chain, the volume's momentum and, with the
  // Nose-Hoover thermostat, the particles' chain as the reference orders them.
  bool mtk() const { return o.barostat == 3; }
  double etap[3] = {0, 0, 0}, etap_dot[4] = {0, 0, 0, 0}, etap_dotdot[3] = {0, 0, 0}, etap_mass[3] = {0, 0, 0};
  double omega_dot = 0, omega_mass = 0, mtk_term2 = 0, vol0 = 0, mtk_virial = 0;
  double target_t(long long step) const {
    return (o.temperature_end >= 0 && o.steps > 0) ? o.temperature + (o.temperature_end - o.temperature) * double(step) / double(o.steps) : o.temperature;
  }
  double ke_now() {
    S.ke(kScKE, false);
    CK(cudaMemcpyAsync(S.h_sc + kScKE, S.sc.p + kScKE, sizeof(double), cudaMemcpyDeviceToHost, E.stream_));
    CK(cudaStreamSynchronize(E.stream_));
    return S.h_sc[kScKE];
  }
  void scale_by(double f) { launch_k(k_scale_by, blocks(size_t(3) * S.n, 256), 256, 0, E.stream_, S.n, S.v.p, f); }
  // the virial of the last force evaluation (energies and virial on), as the rows take it
  void read_virial() {
    sync_scalars();
    caps_gpu_terms t{};
    E.read_terms(&t, true, true);
    mtk_virial = t.w[0] + t.w[1] + t.w[2];
  }
  void mtk_nhc_temp(double tt);
  void mtk_nhc_press(double tt);
  void mtk_omega_step(double tt);
  void mtk_remap();
  void mtk_step(long long s);
  // a step that reports, records, rescales the cell or refills the thermostat's draws
  // (every MTK step is one: it runs on the host's schedule, in a batch too)
  bool special(long long s) const {
    return mtk() || s % thermo_every == 0 || s == o.steps || frame_due(s) || checkpoint_due(s) || baro_due(s) || refill_due(s);
  }

  void start();
  // step s; stop: a stop was asked for before it (and s < steps), so the run ends after it
  void advance(long long s, bool stop = false);
  // steps s .. s + kBlockSteps - 1 are plain steps (no row, frame, checkpoint, cell rescaling or thermostat refill)
  bool block_due(long long s) const {
    if (mtk() || s + Stepper::kBlockSteps - 1 >= o.steps) return false;
    for (long long t = s; t < s + Stepper::kBlockSteps; ++t)
      if (special(t)) return false;
    return true;
  }
  void baro_step(long long s);
};

void MdRun::start() {
  cudaStream_t stream_ = E.stream_;
  Engine& e = E;
  const int n_ = E.n_;
  e.set_cell(st->cell);
  {   // through pinned staging: the copy runs at the link's rate and returns at once
    double* px = S.pinned_xv(n3);
    std::memcpy(px, st->x, n3 * sizeof(double));
    S.x.alloc(n3);
    CK(cudaMemcpyAsync(S.x.p, px, n3 * sizeof(double), cudaMemcpyHostToDevice, stream_));
  }
  S.x0.alloc(n3);
  S.v.alloc(n3);
  {
    std::vector<int8_t> hflags;
    if (o.hmr > 0 && o.is_hydrogen) hflags.assign(o.is_hydrogen, o.is_hydrogen + n_);
    if (!S.masses_ready || S.hm_hmr != o.hmr || S.hm_h != hflags) {   // set again only when what they depend on changed
      S.hm = E.h_mass_;
      S.hmr_moved = 0;
      S.hmr_kept = false;
      if (o.hmr > 0) {
        // hydrogen mass repartitioning (dynamics.cpp:125-147): a hydrogen with exactly one bonded neighbour heavier
        // than itself takes mass from that neighbour up to o.hmr; a neighbour that would be left lighter than 1 u keeps
        // its mass. Hydrogens: the element flags, or a mass below 1.6 u without them.
        std::vector<std::vector<int>> nb(static_cast<size_t>(n_));
        for (const auto& b : E.hb_) nb[b[0]].push_back(int(b[1])), nb[b[1]].push_back(int(b[0]));
        auto hydrogen = [&](int i) { return o.is_hydrogen ? o.is_hydrogen[i] != 0 : E.h_mass_[size_t(i)] < 1.6; };
        for (int i = 0; i < n_; ++i) {
          if (!hydrogen(i) || nb[size_t(i)].size() != 1 || S.hm[size_t(i)] >= o.hmr) continue;
          const int h = nb[size_t(i)][0];
          const double dm = o.hmr - S.hm[size_t(i)];
          if (hydrogen(h) || S.hm[size_t(h)] - dm < 1.0) {
            S.hmr_kept = true;
            continue;
          }
          S.hm[size_t(h)] -= dm;
          S.hm[size_t(i)] = o.hmr;
          ++S.hmr_moved;
        }
      }
      S.m.upload(S.hm, stream_);
      std::vector<double> im(static_cast<size_t>(n_));
      for (int i = 0; i < n_; ++i) im[size_t(i)] = S.hm[size_t(i)] > 0 ? 1.0 / S.hm[size_t(i)] : 0.0;
      S.invm.upload(im, stream_);
      CK(cudaStreamSynchronize(stream_));
      S.masses_ready = true;
      S.hm_hmr = o.hmr;
      S.hm_h = hflags;
      S.cons_built = false;   // the constraint clusters are set up again with the masses
    }
  }
  S.sc.alloc(kScNum);
  S.sc.zero(stream_);
  S.chain.alloc(1);
  CK(cudaMemsetAsync(S.chain.p, 0, sizeof(Chain), stream_));
  S.nparts = blocks(size_t(n_), 256);
  S.part.alloc(size_t(7) * std::max(S.nparts, blocks(size_t(n_), 128)));   // k_ke's blocks, or k_vel_rattle's
  S.done.alloc(1);
  S.done.zero(stream_);
  S.draws.alloc(size_t(Stepper::kDrawChunk) + 1);
  S.respa = std::max(1, o.respa);
  S.slow_parts = 6, S.fast_parts = 1;
  if (o.respa_split == 1) {
    if (!E.pme_) throw ModelError(CAPS_GPU_EINVAL, "the PME r-RESPA split needs PME electrostatics");
    S.slow_parts = 4, S.fast_parts = 3;
  }
  if (S.respa > 1) {
    S.f_slow.alloc(n3);
    S.f_fast.alloc(n3);
  }
  if (!S.h_sc) CK(cudaMallocHost(&S.h_sc, sizeof(double) * kScNum));
  if (!S.h_chain) CK(cudaMallocHost(&S.h_chain, sizeof(Chain)));
  S.nhc = o.thermostat == 3;
  S.bussi = o.thermostat == 1;
  S.langevin = o.thermostat == 2;
  S.t_freq = 1.0 / std::max(o.tau_t, 1e-9);
  S.C.cell = E.dcell_;
  S.build_constraints(st->x);
  S.C.cell = E.dcell_;
  S.ndof = 3.0 * double(n_) - 3.0 - double(S.ncons);
  if (S.ndof < 1) throw ModelError(CAPS_GPU_EINVAL, "the constraints leave no degree of freedom");
  S.rng = std::make_unique<HostRng>(o.seed);
  if (S.ncons) {   // the constrained lengths hold from the start (dynamics.cpp:198-203)
    CK(cudaMemcpyAsync(S.x0.p, S.x.p, n3 * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    launch_k(S.C.lincs ? k_lincs : k_shake, blocks(size_t(S.C.ncl), 128), 128, 0, stream_, S.C, S.x.p, S.x0.p, S.v.p, 0.0, E.d_counters_.p, ListCheck{});
  }

  // velocities: given, or Maxwell-Boltzmann from the reference's stream, no centre-of-mass motion, rescaled to T
  hv.resize(n3);
  const bool drawn = !(st->has_velocities && st->v && !o.new_velocities);
  if (!drawn) {
    std::memcpy(hv.data(), st->v, n3 * sizeof(double));
  } else {
    std::fill(hv.begin(), hv.end(), 0.0);
    for (int i = 0; i < n_; ++i) {
      const double sd = std::sqrt(kB * o.temperature * kAcc / S.hm[size_t(i)]);
      for (int k = 0; k < 3; ++k) hv[3 * size_t(i) + k] = sd * S.rng->gauss();
    }
    double p[3] = {0, 0, 0}, mf = 0;
    for (int i = 0; i < n_; ++i) {
      mf += S.hm[size_t(i)];
      for (int k = 0; k < 3; ++k) p[k] += S.hm[size_t(i)] * hv[3 * size_t(i) + k];
    }
    for (int i = 0; i < n_; ++i)
      for (int k = 0; k < 3; ++k) hv[3 * size_t(i) + k] -= p[k] / mf;
  }
  auto upload_v = [&] {   // through the pinned staging (the copy before it has completed: the stream was synchronised)
    double* pv = S.pinned_xv(n3) + n3;
    std::memcpy(pv, hv.data(), n3 * sizeof(double));
    S.v.alloc(n3);
    CK(cudaMemcpyAsync(S.v.p, pv, n3 * sizeof(double), cudaMemcpyHostToDevice, stream_));
  };
  upload_v();
  if (drawn) {
    if (S.ncons) S.rattle(0);
    CK(cudaMemcpyAsync(hv.data(), S.v.p, n3 * sizeof(double), cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
    const double t0 = 2 * host_ke(hv) / (S.ndof * kB);
    if (t0 > 0)
      for (auto& q : hv) q *= std::sqrt(o.temperature / t0);
    upload_v();
  }
  if (S.ncons) S.rattle(0);
  if (S.bussi) S.make_draws(1, draw_chunk(1));

  // the first force, energies and virial; a list without room enough for the run is grown and built again
  for (int attempt = 0;; ++attempt) {
    S.forces(true, true);
    if (attempt >= 3 || !E.grow_list_for_run()) break;
  }
  if (S.ncons) {
    // step 0's constraint virial from one trial step on copies (dynamics.cpp:582-600)
    DevBuf<double>& xs = S.xs;
    DevBuf<double>& vs = S.vs;
    xs.alloc(n3);
    vs.alloc(n3);
    CK(cudaMemcpyAsync(xs.p, S.x.p, n3 * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    CK(cudaMemcpyAsync(vs.p, S.v.p, n3 * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    S.kick_drift(0.5 * o.dt, o.dt, false, true);
    S.vel_rattle(S.kick_op(0.5 * o.dt), o.dt);
    CK(cudaMemcpyAsync(S.x.p, xs.p, n3 * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    CK(cudaMemcpyAsync(S.v.p, vs.p, n3 * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    CK(cudaStreamSynchronize(stream_));
  }
  if (mtk()) {   // the MTK state starts at rest (dynamics.cpp:331-337)
    for (int c = 0; c < 3; ++c) etap[c] = etap_dotdot[c] = etap_mass[c] = 0;
    for (int c = 0; c < 4; ++c) etap_dot[c] = 0;
    omega_dot = omega_mass = mtk_term2 = 0;
    vol0 = E.dcell_.vol;
  }
  emit(0);
  take(0, frame_due(0), 0);
  if (mtk()) read_virial();   // the first evaluation's virial, for the first step's volume momentum

  thermo_every = std::max(1, o.thermo_every);
  baro_every = std::max(1, o.barostat_every);
}

// One step s: the captured plain step, or a special one (thermo row, frame, cell rescaling, new thermostat draws).
void MdRun::advance(long long s, bool stop) {
  if (refill_due(s)) {
    CK(cudaStreamSynchronize(E.stream_));
    S.make_draws(s, draw_chunk(s));
    S.drop_graphs();   // the draw table's first step is a parameter of the captured thermostat kernel
    ++generation;
  }
  if (mtk()) {
    mtk_step(s);
    ++baro_steps;
  } else if (baro_due(s)) {
    baro_step(s);
  } else {
    // energies and virial only for a thermo row: a step that only records, refills or stops runs the plain graph
    kernels += S.launch_step(s % thermo_every == 0 || s == o.steps);
    if (!special(s) && !stop) return;
  }
  // the order of dynamics.cpp:754-770: the thermo row, the frame, the checkpoint, and on a stop one more checkpoint;
  // the snapshots of earlier steps reach their callbacks before this step's row
  take(s, frame_due(s), (checkpoint_due(s) ? 1 : 0) + (stop && o.checkpoint ? 1 : 0));
  deliver(s);
  if (s % thermo_every == 0 || s == o.steps) {
    emit(s);
    ++emits;
  }
  if (stop) {
    deliver(s + 1);
    stopped_at = s;
  } else if (s < o.steps && g_stop.load(std::memory_order_relaxed) != 0) {
    stop_here(s);   // asked for during this step's callbacks: the reference's check comes after them (dynamics.cpp:765)
  }
}

// The particles' chain over half a step (dynamics.cpp:479-504) on the host copy of the chain, the velocities scaled on
// the device; the chain goes back to the device for the rows.
void MdRun::mtk_nhc_temp(double tt) {
  const double dt = o.dt, dthalf = 0.5 * dt, dt4 = 0.25 * dt, dt8 = 0.125 * dt, t_freq = S.t_freq, ndof = S.ndof;
  Chain& c = *S.h_chain;
  const double kt = kB * tt, ke_target = ndof * kt;
  c.eta_mass[0] = ndof * kt / (t_freq * t_freq);
  for (int q = 1; q < 3; ++q) c.eta_mass[q] = kt / (t_freq * t_freq);
  double kecur = 2 * ke_now();
  c.eta_dotdot[0] = (kecur - ke_target) / c.eta_mass[0];
  for (int q = 2; q > 0; --q) {
    const double ex = std::exp(-dt8 * c.eta_dot[q + 1]);
    c.eta_dot[q] = (c.eta_dot[q] * ex + c.eta_dotdot[q] * dt4) * ex;
  }
  double ex = std::exp(-dt8 * c.eta_dot[1]);
  c.eta_dot[0] = (c.eta_dot[0] * ex + c.eta_dotdot[0] * dt4) * ex;
  const double factor = std::exp(-dthalf * c.eta_dot[0]);
  scale_by(factor);
  kecur *= factor * factor;
  c.eta_dotdot[0] = (kecur - ke_target) / c.eta_mass[0];
  for (int q = 0; q < 3; ++q) c.eta[q] += dthalf * c.eta_dot[q];
  c.eta_dot[0] = (c.eta_dot[0] * ex + c.eta_dotdot[0] * dt4) * ex;
  for (int q = 1; q < 3; ++q) {
    ex = std::exp(-dt8 * c.eta_dot[q + 1]);
    c.eta_dot[q] *= ex;
    c.eta_dotdot[q] = (c.eta_mass[q - 1] * c.eta_dot[q - 1] * c.eta_dot[q - 1] - kt) / c.eta_mass[q];
    c.eta_dot[q] = (c.eta_dot[q] + c.eta_dotdot[q] * dt4) * ex;
  }
  CK(cudaMemcpy(S.chain.p, S.h_chain, sizeof(Chain), cudaMemcpyHostToDevice));
}

// The barostat's chain over half a step (FixNH::nhc_press_integrate, iso; dynamics.cpp:506-531).
void MdRun::mtk_nhc_press(double tt) {
  const double dt = o.dt, dthalf = 0.5 * dt, dt4 = 0.25 * dt, dt8 = 0.125 * dt;
  const double p_freq = 1.0 / std::max(o.tau_p, 1e-9), natoms = double(S.n);
  const double kt = kB * tt;
  omega_mass = (natoms + 1) * kt / (p_freq * p_freq);
  for (int c = 0; c < 3; ++c) etap_mass[c] = kt / (p_freq * p_freq);
  for (int c = 1; c < 3; ++c) etap_dotdot[c] = (etap_mass[c - 1] * etap_dot[c - 1] * etap_dot[c - 1] - kt) / etap_mass[c];
  double kecur = 3 * omega_mass * omega_dot * omega_dot;
  etap_dotdot[0] = (kecur - kt) / etap_mass[0];
  for (int c = 2; c > 0; --c) {
    const double ex = std::exp(-dt8 * etap_dot[c + 1]);
    etap_dot[c] = (etap_dot[c] * ex + etap_dotdot[c] * dt4) * ex;
  }
  double ex = std::exp(-dt8 * etap_dot[1]);
  etap_dot[0] = (etap_dot[0] * ex + etap_dotdot[0] * dt4) * ex;
  for (int c = 0; c < 3; ++c) etap[c] += dthalf * etap_dot[c];
  omega_dot *= std::exp(-dthalf * etap_dot[0]);
  kecur = 3 * omega_mass * omega_dot * omega_dot;
  etap_dotdot[0] = (kecur - kt) / etap_mass[0];
  etap_dot[0] = (etap_dot[0] * ex + etap_dotdot[0] * dt4) * ex;
  for (int c = 1; c < 3; ++c) {
    ex = std::exp(-dt8 * etap_dot[c + 1]);
    etap_dot[c] *= ex;
    etap_dotdot[c] = (etap_mass[c - 1] * etap_dot[c - 1] * etap_dot[c - 1] - kt) / etap_mass[c];
    etap_dot[c] = (etap_dot[c] + etap_dotdot[c] * dt4) * ex;
  }
}

// The volume's momentum over half a step (FixNH::nh_omega_dot, iso, with the MTK terms; dynamics.cpp:533-541), from the
// kinetic energy now and the virial of the last force evaluation.
void MdRun::mtk_omega_step(double tt) {
  const double dthalf = 0.5 * o.dt, p_freq = 1.0 / std::max(o.tau_p, 1e-9), natoms = double(S.n);
  const double kt = kB * tt;
  omega_mass = (natoms + 1) * kt / (p_freq * p_freq);
  const double vol = E.dcell_.vol;
  const double ke2 = 2 * ke_now();
  const double p = (ke2 + mtk_virial) / (3 * vol) * kAtm;
  const double mtk_term1 = ke2 / (3 * natoms);
  omega_dot += ((p - o.pressure) * vol / (omega_mass * kAtm) + mtk_term1 / omega_mass) * dthalf;
  mtk_term2 = 3 * omega_dot / (3 * natoms);
}

// The cell and the positions scaled by exp(dt/2 omega_dot) about the cell's centre (dynamics.cpp:560-570).
void MdRun::mtk_remap() {
  const double mu = std::exp(0.5 * o.dt * omega_dot);
  double c[12];
  std::memcpy(c, E.cell_h_, sizeof c);
  double c0[3];
  for (int k = 0; k < 3; ++k) c0[k] = c[k] + (c[3 + k] + c[6 + k] + c[9 + k]) * 0.5;
  launch_k(k_remap, blocks(size_t(S.n), 256), 256, 0, E.stream_, S.n, S.x.p, c0[0], c0[1], c0[2], mu);
  for (int k = 3; k < 12; ++k) c[k] = c[k] * mu;
  for (int k = 0; k < 3; ++k) c[k] = c0[k] - (c[3 + k] + c[6 + k] + c[9 + k]) * 0.5;
  E.set_cell(c);
  S.C.cell = E.dcell_;
  S.drop_graphs();
}

// One MTK step in the reference's order (dynamics.cpp:628-642): the barostat's chain, the particles' chain, the volume's
// momentum and its velocity factor, half kick, remap, drift, remap, forces (energies and virial), half kick, velocity
// factor, the volume's momentum, the particles' chain, the barostat's chain.
void MdRun::mtk_step(long long s) {
  cudaStream_t stream_ = E.stream_;
  const double dt = o.dt, dthalf = 0.5 * dt;
  launch_k(k_step_begin, 1, 1, 0, stream_, S.sc.p, o.temperature, o.temperature_end, (long long)o.steps, S.ndof);
  const double tt = target_t(s);
  mtk_nhc_press(tt);
  if (S.nhc) mtk_nhc_temp(tt);
  mtk_omega_step(tt);
  scale_by(std::exp(-dthalf * (omega_dot + mtk_term2)));
  S.vel_rattle(S.kick_op(0.5 * dt), 0);
  mtk_remap();
  S.kick_drift(0.0, dt, false, true);
  mtk_remap();
  S.forces(true, true);
  read_virial();
  S.vel_rattle(S.kick_op(0.5 * dt), 0);
  scale_by(std::exp(-dthalf * (omega_dot + mtk_term2)));
  mtk_omega_step(tt);
  if (S.nhc) mtk_nhc_temp(tt);
  mtk_nhc_press(tt);
}

// A step with stochastic cell rescaling (Bernetti & Bussi 2020, dynamics.cpp:684-723), isotropic.
void MdRun::baro_step(long long s) {
  (void)s;
  cudaStream_t stream_ = E.stream_;
  S.step(true, true);
  ++baro_steps;
  S.ke(kScKE, true);
  sync_scalars();
  caps_gpu_terms t{};
  E.read_terms(&t, true, true);
  for (int c = 0; c < 6; ++c) t.w[c] += S.h_sc[kScCW0 + c];
  t.virial = t.w[0] + t.w[1] + t.w[2];
  const double k = S.h_sc[kScKE], vol = E.dcell_.vol;
  const double p = (2 * k + t.virial) / (3 * vol) * kAtm;
  const double hp = o.dt * baro_every;
  const double tnow = S.h_sc[kScTnow];
  // per-axis factors (the isotropic update scales all three by the same mu)
  double mu[3] = {1, 1, 1};
  if (o.barostat == 2 && o.anisotropic) {
    // Berendsen per axis (dynamics.cpp:668-687): mu_k = exp(-beta hp (P0 - P_kk) / (3 tau)), the step at most 0.33 %
    const int axes = o.couple_axes ? o.couple_axes : 7;
    for (int ax = 0; ax < 3; ++ax) {
      if (!((axes >> ax) & 1)) continue;
      const double target = ((o.axis_pressure_set >> ax) & 1) ? o.axis_pressure[ax] : o.pressure;
      const double pk = (S.h_sc[kScKin0 + ax] + t.w[ax]) / vol * kAtm;
      const double deps = std::max(-0.0033, std::min(0.0033, -o.compressibility / o.tau_p * (target - pk) * hp / 3));
      mu[ax] = std::exp(deps);
    }
  } else {
    double deps = -o.compressibility / o.tau_p * (o.pressure - p) * hp;
    if (o.barostat == 1) {
      // stochastic cell rescaling (Bernetti & Bussi 2020, eq. 5): the drift's k_B T / V term and the noise
      const double ktv = kB * tnow / vol * kAtm;
      deps += o.compressibility / o.tau_p * ktv * hp + std::sqrt(2 * ktv * o.compressibility * hp / o.tau_p) * S.rng->gauss();
    }
    deps = std::max(-0.01, std::min(0.01, deps));   // at most 1 % in volume per update
    mu[0] = mu[1] = mu[2] = std::exp(deps / 3);
  }
  std::vector<double> hx(n3);
  CK(cudaMemcpyAsync(hx.data(), S.x.p, n3 * sizeof(double), cudaMemcpyDeviceToHost, stream_));
  CK(cudaMemcpyAsync(hv.data(), S.v.p, n3 * sizeof(double), cudaMemcpyDeviceToHost, stream_));
  CK(cudaStreamSynchronize(stream_));
  double cell[12];
  std::memcpy(cell, E.cell_h_, sizeof cell);
  // positions about the cell origin, and every cell vector's component c, by mu[c]
  for (int i = 0; i < E.n_; ++i)
    for (int c = 0; c < 3; ++c) hx[3 * size_t(i) + c] = cell[c] + mu[c] * (hx[3 * size_t(i) + c] - cell[c]);
  for (int q = 3; q < 12; ++q) cell[q] *= mu[q % 3];
  if (o.barostat == 1) {   // the velocities follow the cell, and the bath takes the kinetic energy's change
    for (auto& q : hv) q /= mu[0];
    const double k2 = host_ke(hv);
    S.h_sc[kScBath] -= k2 - k;
    CK(cudaMemcpyAsync(S.sc.p + kScBath, S.h_sc + kScBath, sizeof(double), cudaMemcpyHostToDevice, stream_));
  }
  // the step's constraint virial, each component r_a F_b scaled with the cell (dynamics.cpp:448-456)
  {
    static const int ia[6] = {0, 1, 2, 0, 0, 1}, ib[6] = {0, 1, 2, 1, 2, 2};
    for (int c = 0; c < 6; ++c) S.h_sc[kScCW0 + c] *= std::sqrt(mu[ia[c]] * mu[ib[c]]);
    CK(cudaMemcpyAsync(S.sc.p + kScCW0, S.h_sc + kScCW0, 6 * sizeof(double), cudaMemcpyHostToDevice, stream_));
  }
  S.x.upload(hx, stream_);
  S.v.upload(hv, stream_);
  E.set_cell(cell);
  S.C.cell = E.dcell_;
  if (S.ncons) {
    CK(cudaMemcpyAsync(S.x0.p, S.x.p, n3 * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    launch_k(S.C.lincs ? k_lincs : k_shake, blocks(size_t(S.C.ncl), 128), 128, 0, stream_, S.C, S.x.p, S.x0.p, S.v.p, 0.0, E.d_counters_.p, ListCheck{});
    S.rattle(0);
  }
  S.forces(true, true);
  S.ke(kScKE, false);   // the rescaled velocities' kinetic energy, which the next Nose-Hoover step starts from
  S.drop_graphs();   // the cell is a parameter of the captured kernels
  ++generation;
}

void Engine::run(caps_gpu_state* st, const caps_gpu_md_opts* md, caps_gpu_progress_fn progress, caps_gpu_frame_fn frame, void* user, std::string* report) {
  const auto t_enter = std::chrono::steady_clock::now();
  validate_md(*md);
  MdRun R(*this, st, md, progress, frame, user);
  R.start();
  const caps_gpu_md_opts& o = *md;
  Stepper& S = R.S;
  const size_t n3 = R.n3;
  if (!S.ev0) CK(cudaEventCreate(&S.ev0));
  if (!S.ev1) CK(cudaEventCreate(&S.ev1));
  cudaEvent_t ev0 = S.ev0, ev1 = S.ev1;
  // measurement mode (include/caps_gpu_diag.h): an event pair around every step and an L2 flush between steps
  const bool timed = timing_flush_ >= 0;
  std::vector<cudaEvent_t> tev;
  if (timed) {
    tev.resize(size_t(2 * std::max<long long>(o.steps, 0)));
    for (auto& e : tev) CK(cudaEventCreate(&e));
    if (timing_flush_ > 0) d_flush_.alloc(size_t(timing_flush_));
  }
  // the step graphs are captured before the step loop, as set-up (like the first force evaluation), so that no step's
  // time holds a capture
  if (o.steps > 0 && !R.mtk() && !R.baro_due(1) && !R.refill_due(1)) {
    S.ensure_graph(false);
    S.ensure_graph(true);
    if (!timed && o.steps > Stepper::kBlockSteps) S.ensure_graph(false, true);
  }
  const auto w0 = std::chrono::steady_clock::now();
  CK(cudaEventRecord(ev0, stream_));
  for (long long s = 1; s <= o.steps; ++s) {
    // outside measurement mode, runs of plain steps go as blocks of kBlockSteps (a stop asked for from another thread
    // takes effect at the end of a block)
    if (!timed && g_stop.load(std::memory_order_relaxed) == 0 && R.block_due(s)) {
      R.kernels += S.launch_block();
      s += Stepper::kBlockSteps - 1;
      continue;
    }
    if (timed) {
      if (timing_flush_ > 0) CK(cudaMemsetAsync(d_flush_.p, int(s & 255), size_t(timing_flush_), stream_));
      CK(cudaEventRecord(tev[size_t(2 * (s - 1))], stream_));
    }
    struct EndEvent {
      bool on;
      cudaEvent_t e;
      cudaStream_t st;
      ~EndEvent() {
        if (on) cudaEventRecord(e, st);
      }
    } end_ev{timed, timed ? tev[size_t(2 * (s - 1) + 1)] : nullptr, stream_};
    R.advance(s, g_stop.load(std::memory_order_relaxed) != 0 && s < o.steps);
    if (R.stopped_at >= 0) break;
  }
  CK(cudaEventRecord(ev1, stream_));
  CK(cudaEventSynchronize(ev1));
  R.deliver(o.steps + 1);
  kernels_run_ = R.kernels + R.emits + R.baro_steps * S.graph_kernels[1];
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, ev0, ev1));
  const long long done = R.stopped_at >= 0 ? R.stopped_at : o.steps;   // steps run
  if (timed && done > 0) {
    double sum = 0;
    for (long long k = 0; k < done; ++k) {
      float t = 0;
      CK(cudaEventElapsedTime(&t, tev[size_t(2 * k)], tev[size_t(2 * k + 1)]));
      sum += t;
    }
    for (auto& e : tev) cudaEventDestroy(e);
    ms = float(sum);
  }
  last_step_ms_ = done > 0 ? double(ms) / double(done) : 0.0;
  const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - w0).count();
  R.sync_scalars();
  last_sps_ = done > 0 && ms > 0 ? double(done) / (ms * 1e-3) : 0.0;
  // state back to the caller, through the pinned staging
  double* px = S.pinned_xv(n3);
  CK(cudaMemcpyAsync(px, S.x.p, n3 * sizeof(double), cudaMemcpyDeviceToHost, stream_));
  if (st->v) CK(cudaMemcpyAsync(px + n3, S.v.p, n3 * sizeof(double), cudaMemcpyDeviceToHost, stream_));
  CK(cudaStreamSynchronize(stream_));
  std::memcpy(st->x, px, n3 * sizeof(double));
  if (st->v) std::memcpy(st->v, px + n3, n3 * sizeof(double));
  std::memcpy(st->cell, cell_h_, sizeof cell_h_);
  if (report) {
    char b[512];
    const double nsday = wall > 0 ? double(done) * o.dt * 1e-6 / wall * 86400 : 0.0;
    const double setup = std::chrono::duration<double>(w0 - t_enter).count();
    std::snprintf(b, sizeof b,
                  "%lld steps of %.2f fs in %.3f s (device %.3f s, set-up %.3f s) · %.2f ns/day · %d constraints · %.0f degrees of freedom · %s"
                  " · tuned: %d entries per work item, pair grid %d block(s) per SM short of full, PME line blocks %d/%d/%d, PME grid cap %d, bonded cap %d",
                  (long long)done, o.dt, wall, ms * 1e-3, setup, nsday, S.ncons, S.ndof, mixed_ ? "mixed FP32/fixed-point" : "FP64", batch_,
                  pair_cut_, pme_lines()[0], pme_lines()[1], pme_lines()[2], pme_cap_, bonded_cap_);
    *report = b;
    if (o.hmr > 0) {   // the reference's note (dynamics.cpp:143-145)
      std::snprintf(b, sizeof b, " · hydrogen mass repartitioning: %lld hydrogens at %.3f u, the difference taken from their bonded atoms%s",
                    S.hmr_moved, o.hmr, S.hmr_kept ? " (some left as they were: their neighbour would have been too light)" : "");
      *report += b;
    }
    if (S.ncons && o.constraint_algorithm == 1)   // the reference's note (dynamics.cpp:176)
      *report += " · constraint solver: LINCS (order 4) for positions, RATTLE for velocities";
  }
  R.completed = true;
  if (R.stopped_at >= 0) throw ModelError(CAPS_GPU_ESTOPPED, "stopped at step " + std::to_string(R.stopped_at + o.step_offset) + " (a stop was asked for)");
}

// Replicas in lock step (caps_gpu_run_batch). A step on which no replica reports, records, rescales or refills is one
// CUDA graph holding every replica's step as a parallel branch (each on its own engine's streams); other steps run
// replica by replica. The graph is captured again whenever a replica's captured step changes.
void run_batch(const std::vector<Engine*>& es, caps_gpu_state* const* states, const caps_gpu_md_opts* const* mds, caps_gpu_progress_fn progress,
               caps_gpu_frame_fn frame, void* const* users) {
  const size_t R = es.size();
  if (R == 0) return;
  const long long steps = mds[0]->steps;
  for (size_t r = 0; r < R; ++r) {
    es[r]->validate_md(*mds[r]);
    if (mds[r]->steps != steps) throw ModelError(CAPS_GPU_EINVAL, "the replicas of a batch run the same number of steps");
    for (size_t q = 0; q < r; ++q)
      if (es[q] == es[r]) throw ModelError(CAPS_GPU_EINVAL, "each replica of a batch needs its own engine");
  }
  std::vector<std::unique_ptr<MdRun>> runs;
  for (size_t r = 0; r < R; ++r) {
    runs.emplace_back(new MdRun(*es[r], states[r], mds[r], progress, frame, users ? users[r] : nullptr));
    runs.back()->start();
  }
  struct Res {
    cudaStream_t bs = nullptr;
    cudaEvent_t fork = nullptr, t0 = nullptr, t1 = nullptr;
    std::vector<cudaEvent_t> ev;
    cudaGraphExec_t g = nullptr;
    ~Res() {
      if (g) cudaGraphExecDestroy(g);
      for (auto e : ev)
        if (e) cudaEventDestroy(e);
      if (fork) cudaEventDestroy(fork);
      if (t0) cudaEventDestroy(t0);
      if (t1) cudaEventDestroy(t1);
      if (bs) cudaStreamDestroy(bs);
    }
  } res;
  CK(cudaStreamCreateWithFlags(&res.bs, cudaStreamNonBlocking));
  CK(cudaEventCreateWithFlags(&res.fork, cudaEventDisableTiming));
  CK(cudaEventCreate(&res.t0));
  CK(cudaEventCreate(&res.t1));
  res.ev.assign(R, nullptr);
  for (auto& e : res.ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  std::vector<int> seen(R, -1);
  long long batch_kernels = 0, graph_nodes = 0;
  bool on_replicas = true;   // the replicas' own streams hold the latest work
  // orders the batch stream after every replica stream, or every replica stream after the batch stream
  auto join_to_batch = [&] {
    for (size_t r = 0; r < R; ++r) {
      CK(cudaEventRecord(res.ev[r], es[r]->stream_));
      CK(cudaStreamWaitEvent(res.bs, res.ev[r], 0));
    }
  };
  auto fork_to_replicas = [&] {
    CK(cudaEventRecord(res.fork, res.bs));
    for (size_t r = 0; r < R; ++r) CK(cudaStreamWaitEvent(es[r]->stream_, res.fork, 0));
  };
  join_to_batch();
  CK(cudaEventRecord(res.t0, res.bs));
  const auto w0 = std::chrono::steady_clock::now();
  long long stopped_at = -1;
  for (long long s = 1; s <= steps; ++s) {
    const bool stop = g_stop.load(std::memory_order_relaxed) != 0 && s < steps;
    bool plain = !stop;
    for (size_t r = 0; r < R; ++r) plain = plain && !runs[r]->special(s);
    if (!plain) {
      if (!on_replicas) fork_to_replicas(), on_replicas = true;
      bool any = false;
      for (size_t r = 0; r < R; ++r) {
        runs[r]->advance(s, stop);
        any = any || runs[r]->stopped_at >= 0;
      }
      if (any) {   // a stop seen by one replica (asked for in its callbacks) ends every replica at this step
        for (size_t r = 0; r < R; ++r)
          if (runs[r]->stopped_at < 0) runs[r]->stop_here(s);
        stopped_at = s;
        break;
      }
      continue;
    }
    if (on_replicas) join_to_batch(), on_replicas = false;
    bool stale = res.g == nullptr;
    for (size_t r = 0; r < R; ++r) stale = stale || seen[r] != runs[r]->generation;
    if (stale) {
      if (res.g) {
        CK(cudaGraphExecDestroy(res.g));
        res.g = nullptr;
      }
      cudaGraph_t graph;
      CK(cudaStreamBeginCapture(res.bs, cudaStreamCaptureModeThreadLocal));
      try {
        CK(cudaEventRecord(res.fork, res.bs));
        for (size_t r = 0; r < R; ++r) {
          CK(cudaStreamWaitEvent(es[r]->stream_, res.fork, 0));
          runs[r]->S.step(false, false);
          CK(cudaEventRecord(res.ev[r], es[r]->stream_));
          CK(cudaStreamWaitEvent(res.bs, res.ev[r], 0));
        }
      } catch (...) {   // leave no capture open behind an error
        cudaGraph_t junk = nullptr;
        (void)cudaStreamEndCapture(res.bs, &junk);
        if (junk) cudaGraphDestroy(junk);
        (void)cudaGetLastError();
        throw;
      }
      CK(cudaStreamEndCapture(res.bs, &graph));
      size_t nn = 0;
      CK(cudaGraphGetNodes(graph, nullptr, &nn));
      std::vector<cudaGraphNode_t> nodes(nn);
      CK(cudaGraphGetNodes(graph, nodes.data(), &nn));
      graph_nodes = 0;
      for (auto nd : nodes) graph_nodes += is_kernel_node(nd);
      CK(cudaGraphInstantiate(&res.g, graph, cudaGraphInstantiateFlagUseNodePriority));
      CK(cudaGraphDestroy(graph));
      for (size_t r = 0; r < R; ++r) seen[r] = runs[r]->generation;
    }
    CK(cudaGraphLaunch(res.g, res.bs));
    batch_kernels += graph_nodes;
  }
  if (on_replicas) join_to_batch();
  CK(cudaEventRecord(res.t1, res.bs));
  CK(cudaEventSynchronize(res.t1));
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, res.t0, res.t1));
  const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - w0).count();
  (void)wall;
  for (size_t r = 0; r < R; ++r) runs[r]->deliver(steps + 1);
  const long long done = stopped_at >= 0 ? stopped_at : steps;
  for (size_t r = 0; r < R; ++r) {
    MdRun& M = *runs[r];
    Engine& E = M.E;
    M.sync_scalars();
    E.last_step_ms_ = done > 0 ? double(ms) / double(done) : 0.0;
    E.last_sps_ = done > 0 && ms > 0 ? double(done) / (ms * 1e-3) : 0.0;
    E.kernels_run_ = M.kernels + M.emits + (r == 0 ? batch_kernels : 0);
    CK(cudaMemcpyAsync(M.st->x, M.S.x.p, M.n3 * sizeof(double), cudaMemcpyDeviceToHost, E.stream_));
    if (M.st->v) CK(cudaMemcpyAsync(M.st->v, M.S.v.p, M.n3 * sizeof(double), cudaMemcpyDeviceToHost, E.stream_));
    CK(cudaStreamSynchronize(E.stream_));
    std::memcpy(M.st->cell, E.cell_h_, sizeof E.cell_h_);
    M.completed = true;
  }
  if (stopped_at >= 0)
    throw ModelError(CAPS_GPU_ESTOPPED, "stopped at step " + std::to_string(stopped_at + mds[0]->step_offset) + " (a stop was asked for)");
}

}  // namespace capsb

extern "C" {
void caps_gpu_request_stop(int32_t on) { capsb::g_stop.store(on != 0 ? 1 : 0); }
int32_t caps_gpu_stop_requested(void) { return capsb::g_stop.load() != 0 ? 1 : 0; }
}
