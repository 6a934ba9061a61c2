// K-BOND: bonded terms, 1-4 pairs, the Coulomb corrections of excluded pairs and FENE bonds, one thread per term, all
// kinds in one launch (k_bonded).
// Reference: Evaluator::compute's bonded phase (core/src/field.cpp:1863-2283): harmonic bonds (:1986-1995), harmonic
// angles (:1996-2010), Fourier torsion groups for dihedrals and impropers (:1875-1920, 2011-2018), 1-4 pairs (:2019-2043),
// excluded-pair electrostatics (:2206-2266), FENE + WCA (:2152-2166). These run in double arithmetic on both paths (the
// reference keeps them double in its mixed mode too: r - r0 of a stiff bond loses most of a float's digits, which
// measured 1.4e-4 RMS relative force error on a relaxed cell against the 5e-6 target); the mixed path adds the forces
// as 64-bit fixed point (order-free, bit-reproducible), the FP64 path as doubles. The sink type S picks which.
#pragma once
#include "common.cuh"

namespace capsb {

struct BondedArgs {
  const double* x;
  DevCell cell;
  EnergySink en;
  int fixed;   // 1: mixed path (fixed-point sinks)
};

// Per-thread energy and virial, summed over the block and added once. On the mixed path (fixed) every term is rounded
// to fixed point on its own, so that the sums do not depend on how the terms are spread over threads and blocks.
template <bool VIR>
struct Tally {
  bool fixed;
  double e = 0;
  double w[6] = {0, 0, 0, 0, 0, 0};
  long long eq = 0;
  long long wq[6] = {0, 0, 0, 0, 0, 0};
  __device__ explicit Tally(bool f) : fixed(f) {}
  __device__ __forceinline__ void energy(double v) {
    if (fixed) eq += to_fix(v, kFixE);
    else e += v;
  }
  __device__ __forceinline__ void wadd(int k, double v) {
    if (fixed) wq[k] += to_fix(v, kFixE);
    else w[k] += v;
  }
  template <class R>
  __device__ __forceinline__ void vir(R dx, R dy, R dz, R fx, R fy, R fz) {
    if (!VIR) return;
    wadd(0, double(dx * fx));
    wadd(1, double(dy * fy));
    wadd(2, double(dz * fz));
    wadd(3, 0.5 * double(dx * fy + dy * fx));
    wadd(4, 0.5 * double(dx * fz + dz * fx));
    wadd(5, 0.5 * double(dy * fz + dz * fy));
  }
  __device__ void flush(const BondedArgs& A, int slot, bool ener) {
    if (fixed) {
      __shared__ long long scratch_q[32];
      if (ener) {
        const long long s = block_sum(eq, scratch_q);
        if (threadIdx.x == 0 && s != 0) atomic_add_fix(A.en.fix + slot, s);
      }
      if (VIR)
        for (int k = 0; k < 6; ++k) {
          const long long s = block_sum(wq[k], scratch_q);
          if (threadIdx.x == 0 && s != 0) atomic_add_fix(A.en.fix + kEW0 + k, s);
        }
      return;
    }
    __shared__ double scratch[32];
    if (ener) {
      const double s = block_sum(e, scratch);
      if (threadIdx.x == 0 && s != 0) A.en.add(slot, s, false);
    }
    if (VIR)
      for (int k = 0; k < 6; ++k) {
        const double s = block_sum(w[k], scratch);
        if (threadIdx.x == 0 && s != 0) A.en.add(kEW0 + k, s, false);
      }
  }
};

template <class R>
__device__ __forceinline__ void sep(const BondedArgs& A, int i, int j, R& dx, R& dy, R& dz) {
  double ex = A.x[3 * j] - A.x[3 * i], ey = A.x[3 * j + 1] - A.x[3 * i + 1], ez = A.x[3 * j + 2] - A.x[3 * i + 2];
  min_image(A.cell, ex, ey, ez);
  dx = R(ex), dy = R(ey), dz = R(ez);
}

template <class R> __device__ __forceinline__ R rsq(R v) { return sqrt(v); }
template <> __device__ __forceinline__ float rsq<float>(float v) { return sqrtf(v); }

// harmonic bonds: k (r - r0)^2
template <class R, class S, bool ENER, bool VIR>
__device__ __forceinline__ void bonds_body(int blk, int nblk, int nb, const uint32_t* __restrict__ ij, const double* __restrict__ kr, BondedArgs A, S F) {
  Tally<VIR> T(A.fixed != 0);
  for (int t = blk * blockDim.x + threadIdx.x; t < nb; t += nblk * blockDim.x) {
    const int i = int(ij[2 * t]), j = int(ij[2 * t + 1]);
    R dx, dy, dz;
    sep(A, i, j, dx, dy, dz);
    const R k = R(kr[2 * t]), r0 = R(kr[2 * t + 1]);
    const R r = rsq(dx * dx + dy * dy + dz * dz), dr = r - r0;
    if (ENER) T.energy(double(k * dr * dr));
    const R s = r > R(1e-12) ? -2 * k * dr / r : R(0);
    const R fx = dx * s, fy = dy * s, fz = dz * s;
    F.add(j, fx, fy, fz);
    F.add(i, -fx, -fy, -fz);
    T.vir(dx, dy, dz, fx, fy, fz);
  }
  T.flush(A, kEBond, ENER);
}

// harmonic angles: kt (theta - theta0)^2, j the vertex
template <class R, class S, bool ENER, bool VIR>
__device__ __forceinline__ void angles_body(int blk, int nblk, int na, const uint32_t* __restrict__ ijk, const double* __restrict__ kt0, BondedArgs A, S F) {
  Tally<VIR> T(A.fixed != 0);
  for (int t = blk * blockDim.x + threadIdx.x; t < na; t += nblk * blockDim.x) {
    const int i = int(ijk[3 * t]), j = int(ijk[3 * t + 1]), k = int(ijk[3 * t + 2]);
    R ux, uy, uz, vx, vy, vz;
    sep(A, j, i, ux, uy, uz);   // u = x_i - x_j
    sep(A, j, k, vx, vy, vz);   // v = x_k - x_j
    const R lu = rsq(ux * ux + uy * uy + uz * uz), lv = rsq(vx * vx + vy * vy + vz * vz);
    R c = (ux * vx + uy * vy + uz * vz) / (lu * lv);
    c = c > R(1) ? R(1) : (c < R(-1) ? R(-1) : c);
    const R th = acos(c);
    R sn = rsq(R(1) - c * c);
    sn = sn > R(1e-8) ? sn : R(1e-8);
    const R dth = th - R(kt0[2 * t + 1]);
    const R kk = R(kt0[2 * t]);
    if (ENER) T.energy(double(kk * dth * dth));
    const R g = 2 * kk * dth / sn;
    const R iuv = R(1) / (lu * lv), cu = c / (lu * lu), cv = c / (lv * lv);
    const R fix = (vx * iuv - ux * cu) * g, fiy = (vy * iuv - uy * cu) * g, fiz = (vz * iuv - uz * cu) * g;
    const R fkx = (ux * iuv - vx * cv) * g, fky = (uy * iuv - vy * cv) * g, fkz = (uz * iuv - vz * cv) * g;
    F.add(i, fix, fiy, fiz);
    F.add(k, fkx, fky, fkz);
    F.add(j, -(fix + fkx), -(fiy + fky), -(fiz + fkz));
    T.vir(ux, uy, uz, fix, fiy, fiz);
    T.vir(vx, vy, vz, fkx, fky, fkz);
  }
  T.flush(A, kEAngle, ENER);
}

// Fourier torsion groups: terms [gs[g], gs[g+1]) share one quadruple; v [1 + cos(n phi - delta)], phi IUPAC, cos/sin of
// n phi by recurrence (field.cpp:1875-1920).
template <class R, class S, bool ENER, bool VIR>
__device__ __forceinline__ void torsions_body(int blk, int nblk, int ngroups, const int* __restrict__ gs, const uint32_t* __restrict__ ijkl, const double* __restrict__ vd,
                           const int* __restrict__ nn, BondedArgs A, S F, int slot) {
  Tally<VIR> T(A.fixed != 0);
  for (int g = blk * blockDim.x + threadIdx.x; g < ngroups; g += nblk * blockDim.x) {
    const int t0 = gs[g], t1 = gs[g + 1];
    const int i = int(ijkl[4 * t0]), j = int(ijkl[4 * t0 + 1]), k = int(ijkl[4 * t0 + 2]), l = int(ijkl[4 * t0 + 3]);
    R b1x, b1y, b1z, b2x, b2y, b2z, b3x, b3y, b3z;
    sep(A, i, j, b1x, b1y, b1z);
    sep(A, j, k, b2x, b2y, b2z);
    sep(A, k, l, b3x, b3y, b3z);
    const R mx = b1y * b2z - b1z * b2y, my = b1z * b2x - b1x * b2z, mz = b1x * b2y - b1y * b2x;
    const R nx = b2y * b3z - b2z * b3y, ny = b2z * b3x - b2x * b3z, nz = b2x * b3y - b2y * b3x;
    const R m2 = mx * mx + my * my + mz * mz, n2 = nx * nx + ny * ny + nz * nz;
    const R lb2 = rsq(b2x * b2x + b2y * b2y + b2z * b2z);
    if (m2 < R(1e-12) || n2 < R(1e-12) || lb2 < R(1e-9)) continue;
    const R xc = mx * nx + my * ny + mz * nz, yc = lb2 * (b1x * nx + b1y * ny + b1z * nz);
    const R rc_ = rsq(xc * xc + yc * yc);
    const R c1 = xc / rc_, s1 = yc / rc_;
    R dEdphi = 0, e = 0;
    for (int t = t0; t < t1; ++t) {
      const int n = nn[t];
      R cn = 1, sn = 0;
      if (n >= 0 && n <= 12) {
        for (int r = 0; r < n; ++r) {
          const R c = cn * c1 - sn * s1;
          sn = sn * c1 + cn * s1;
          cn = c;
        }
      } else {
        const R phi = atan2(yc, xc);
        cn = cos(R(n) * phi), sn = sin(R(n) * phi);
      }
      const double delta = vd[2 * t + 1];
      R cd = 1, sd = 0;
      if (delta != 0) {
        if (fabs(delta - kPi) < 1e-12) cd = -1;
        else cd = R(cos(delta)), sd = R(sin(delta));
      }
      const R v = R(vd[2 * t]);
      e += v * (1 + cn * cd + sn * sd);
      dEdphi -= v * R(n) * (sn * cd - cn * sd);
    }
    if (ENER) T.energy(double(e));
    const R g1x = mx * (-lb2 / m2), g1y = my * (-lb2 / m2), g1z = mz * (-lb2 / m2);
    const R g4x = nx * (lb2 / n2), g4y = ny * (lb2 / n2), g4z = nz * (lb2 / n2);
    const R p = (b1x * b2x + b1y * b2y + b1z * b2z) / (lb2 * lb2), qd = (b3x * b2x + b3y * b2y + b3z * b2z) / (lb2 * lb2);
    const R g2x = g4x * qd - g1x * (1 + p), g2y = g4y * qd - g1y * (1 + p), g2z = g4z * qd - g1z * (1 + p);
    const R g3x = g1x * p - g4x * (1 + qd), g3y = g1y * p - g4y * (1 + qd), g3z = g1z * p - g4z * (1 + qd);
    const R s = -dEdphi;
    F.add(i, g1x * s, g1y * s, g1z * s);
    F.add(j, g2x * s, g2y * s, g2z * s);
    F.add(k, g3x * s, g3y * s, g3z * s);
    F.add(l, g4x * s, g4y * s, g4z * s);
    T.vir(b1x, b1y, b1z, g2x * s, g2y * s, g2z * s);
    T.vir(b1x + b2x, b1y + b2y, b1z + b2z, g3x * s, g3y * s, g3z * s);
    T.vir(b1x + b2x + b3x, b1y + b2y + b3y, b1z + b2z + b3z, g4x * s, g4y * s, g4z * s);
  }
  T.flush(A, slot, ENER);
}

// 1-4 pairs: LJ times the 1-4 scale (and the same cut-off shift as the pairs), at the nearest image (field.cpp:2019-2043).
// lj: per type pair (eps, sigma^6, the pairs' energy shift or 0, 0); capped: (rcap^2, ecap, fcap, 0). lj96: the class II
// form eps (2 q^(3/2) - 3 q), q = (s/r)^6 (field.cpp:1471-1475), else 4 eps (q^2 - q).
template <class R, class S, bool ENER, bool VIR>
__device__ __forceinline__ void pairs14_body(int blk, int nblk, int np, const uint32_t* __restrict__ ij, const double* __restrict__ scale, double lj14, const int* __restrict__ type, int nt,
                          const double4* __restrict__ lj, const double4* __restrict__ cap, const double4* __restrict__ gen, const double4* __restrict__ gen2,
                          double r1, PairTables tabs, BondedArgs A, S F, int lj96, int fsw, double rc) {
  Tally<VIR> T(A.fixed != 0);
  for (int t = blk * blockDim.x + threadIdx.x; t < np; t += nblk * blockDim.x) {
    const int i = int(ij[2 * t]), j = int(ij[2 * t + 1]);
    R dx, dy, dz;
    sep(A, i, j, dx, dy, dz);
    const double4 c = lj[type[i] * nt + type[j]];
    if (c.x <= 0) continue;
    const R sc = R(scale ? scale[t] : lj14);
    const R r2 = dx * dx + dy * dy + dz * dz;
    R fr, ev;
    if (c.w != 0) {
      // a generic form (field.cpp:2033-2034, FP64 only): nothing beyond the pair's own cut-off
      const double4 g = gen[type[i] * nt + type[j]];
      const double r2d = double(r2);
      if (g.w > 0 && r2d > g.w) continue;
      double e = 0;
      const double f = generic_pair(int(c.w), g, gen2[type[i] * nt + type[j]], r1, tabs, r2d, e);
      ev = R(double(sc) * e);
      fr = R(double(sc) * f);
    } else if (cap && r2 < R(cap[type[i] * nt + type[j]].x)) {
      const double4 cp = cap[type[i] * nt + type[j]];
      const R r = rsq(r2), rcp = rsq(R(cp.x));
      ev = sc * (R(cp.y) + R(cp.z) * (rcp - r));
      fr = sc * R(cp.z) / r;
    } else if (fsw) {   // CHARMM's force switch (the 1-4 pairs take it as the others, field.cpp:2033)
      double e = 0;
      const double f = charmm_fsw(4 * c.x * c.y * c.y, 4 * c.x * c.y, r1, rc, double(r2), e, true);
      ev = R(double(sc) * e);
      fr = R(double(sc) * f);
    } else {
      const R q = R(c.y) / (r2 * r2 * r2);
      if (lj96) {
        const R q9 = q * sqrt(q);
        ev = sc * R(c.x) * (2 * q9 - 3 * q);
        fr = sc * 18 * R(c.x) * (q9 - q) / r2;
      } else {
        ev = sc * 4 * R(c.x) * (q * q - q);
        fr = sc * 24 * R(c.x) * (2 * q * q - q) / r2;
      }
    }
    if (ENER) T.energy(double(ev - sc * R(c.z)));
    const R fx = dx * fr, fy = dy * fr, fz = dz * fr;
    F.add(j, fx, fy, fz);
    F.add(i, -fx, -fy, -fz);
    T.vir(dx, dy, dz, fx, fy, fz);
  }
  T.flush(A, kEVdw, ENER);
}

// Coulomb of excluded pairs (1-2, 1-3 factor 0; 1-4 the Coulomb fraction they keep): the damped / Ewald real-space sum
// includes them and the bare 1/r is removed in proportion (1 - factor) (field.cpp:2206-2266). FP64: the reference's
// branches (the Hermite table inside the cut-off, its erf form below 0.5 Å, Abramowitz-Stegun erfc beyond the cut-off
// under PME). FP32: E = qq (f/r - erf(kr)/r) in closed form (no cancellation), the same terms beyond.
struct ExclArgs {
  const uint32_t* ij;
  const double* factor;
  const double* q;
  const double* gtab;
  double ghi, rc, rc2, kappa, dsf_e0, dsf_f0;
  int pme;
};

__device__ __forceinline__ double erfc_as(double x, double& ex2) {   // Abramowitz & Stegun 7.1.26, as field.cpp:585-591
  const double P = 0.3275911, A1 = 0.254829592, A2 = -0.284496736, A3 = 1.421413741, A4 = -1.453152027, A5 = 1.061405429;
  ex2 = exp(-x * x);
  const double t = 1.0 / (1.0 + P * x);
  return t * (A1 + t * (A2 + t * (A3 + t * (A4 + t * A5)))) * ex2;
}

template <class S, bool ENER, bool VIR>
__device__ __forceinline__ void excl_body(int blk, int nblk, int nx, ExclArgs E, BondedArgs A, S F) {
  Tally<VIR> T(A.fixed != 0);
  const double sp = 2 / sqrt(kPi), kap = E.kappa;
  for (int t = blk * blockDim.x + threadIdx.x; t < nx; t += nblk * blockDim.x) {
    const int i = int(E.ij[2 * t]), j = int(E.ij[2 * t + 1]);
    if (E.q[i] == 0 || E.q[j] == 0) continue;
    double dx, dy, dz;
    sep(A, i, j, dx, dy, dz);
    const double r2 = dx * dx + dy * dy + dz * dz;
    if (r2 >= E.rc2 && !E.pme) continue;
    const double r = sqrt(r2), qq = kCoulomb * E.q[i] * E.q[j], f = E.factor[t];
    double e, fr;
    if (r < 0.5) {
      const double xk = kap * r;
      const double g = r > 1e-8 ? erf(xk) / r : sp * kap;
      const double gr = r > 1e-4 ? (sp * kap * exp(-xk * xk) * r - erf(xk)) / (r2 * r) : -2 * sp * kap * kap * kap / 3;
      const double shift = E.pme ? 0.0 : -E.dsf_e0 + E.dsf_f0 * (r - E.rc);
      const double inv = r > 1e-8 ? 1 / r : 0.0;
      e = qq * (-g + f * inv + shift);
      fr = qq * (gr + f * inv * inv * inv - (E.pme ? 0.0 : E.dsf_f0) * inv);
    } else if (r2 < E.rc2) {
      const double u = r2 * E.ghi;
      const int k = int(u);
      const double tt = u - k, t2 = tt * tt;
      const double* g = E.gtab + 2 * k;
      const double G = g[0] + t2 * (3 - 2 * tt) * (g[2] - g[0]) + tt * (1 - tt) * ((1 - tt) * g[1] - tt * g[3]);
      const double dG = (6 * tt * (1 - tt) * (g[2] - g[0]) * E.ghi) + (1 - tt) * (1 - 3 * tt) * g[1] * E.ghi + tt * (3 * tt - 2) * g[3] * E.ghi;
      const double rinv = 1 / r, Ee = rinv - G, Fc = rinv * rinv * rinv + 2 * dG;
      if (E.pme) {
        e = qq * Ee - (1 - f) * qq / r;
        fr = qq * (Fc - (1 - f) / (r2 * r));
      } else {
        e = qq * (Ee - E.dsf_e0 + E.dsf_f0 * (r - E.rc)) - (1 - f) * qq / r;
        fr = qq * (Fc - E.dsf_f0 / r - (1 - f) / (r2 * r));
      }
    } else {
      double ex2;
      const double er = erfc_as(kap * r, ex2);
      e = qq * er / r - (1 - f) * qq / r;
      fr = qq * ((er / r2 + sp * kap * ex2 / r) - (1 - f) / r2) / r;
    }
    if (ENER) T.energy(e);
    const double fx = dx * fr, fy = dy * fr, fz = dz * fr;
    F.add(j, fx, fy, fz);
    F.add(i, -fx, -fy, -fz);
    T.vir(dx, dy, dz, fx, fy, fz);
  }
  T.flush(A, kECoul, ENER);
}

// FENE (-1/2 K R0^2 ln(1 - (r/R0)^2)) plus WCA below 2^(1/6) sigma (LAMMPS bond fene; field.cpp:2152-2166). A bond
// stretched to R0 or past raises kErrFene (the reference throws FieldError there).
template <class R, class S, bool ENER, bool VIR>
__device__ __forceinline__ void fene_body(int blk, int nblk, int nf, const uint32_t* __restrict__ ij, const double* __restrict__ p, BondedArgs A, S F, int* counters,
                                          double* info) {
  Tally<VIR> T(A.fixed != 0);
  for (int t = blk * blockDim.x + threadIdx.x; t < nf; t += nblk * blockDim.x) {
    const int i = int(ij[2 * t]), j = int(ij[2 * t + 1]);
    R dx, dy, dz;
    sep(A, i, j, dx, dy, dz);
    const R K = R(p[4 * t]), R0 = R(p[4 * t + 1]), eps = R(p[4 * t + 2]), sg = R(p[4 * t + 3]);
    const R r = rsq(dx * dx + dy * dy + dz * dz);
    const R q = r / R0;
    if (!(q < R(1))) {
      atomicOr(reinterpret_cast<unsigned*>(counters + kCntErr), kErrFene);
      if (info && atomicCAS(counters + kCntFeneClaim, 0, 1) == 0) {   // the first one found: its bond and length
        double ex = A.x[3 * j] - A.x[3 * i], ey = A.x[3 * j + 1] - A.x[3 * i + 1], ez = A.x[3 * j + 2] - A.x[3 * i + 2];
        min_image(A.cell, ex, ey, ez);
        info[kInfoFeneBond] = double(t);
        info[kInfoFeneR] = sqrt(ex * ex + ey * ey + ez * ez);
      }
      continue;
    }
    R e = -R(0.5) * K * R0 * R0 * log(R(1) - q * q);
    R dEdr = K * r / (R(1) - q * q);
    if (eps > 0 && r < R(1.122462048309373) * sg) {
      const R s2 = sg * sg / (r * r), s6 = s2 * s2 * s2;
      e += 4 * eps * (s6 * s6 - s6) + eps;
      dEdr += -24 * eps * (2 * s6 * s6 - s6) / r;
    }
    if (ENER) T.energy(double(e));
    const R s = r > R(1e-12) ? -dEdr / r : R(0);
    const R fx = dx * s, fy = dy * s, fz = dz * s;
    F.add(j, fx, fy, fz);
    F.add(i, -fx, -fy, -fz);
    T.vir(dx, dy, dz, fx, fy, fz);
  }
  T.flush(A, kEBond, ENER);
}

// All bonded work of one force evaluation in one launch: the grid is cut into segments of blocks, one per term kind, each
// segment sized to its term count; a block runs the body of its segment's kind over that segment's terms. One launch
// instead of one per kind keeps the short bonded branch from queuing kernel after kernel beside the pair kernel.
enum BondedKind { kBkBonds = 0, kBkAngles, kBkDihedrals, kBkImpropers, kBkFene, kBkPairs14, kBkExcl, kBkKinds };

struct BondedWork {
  int nseg;
  int kind[kBkKinds];
  int first[kBkKinds + 1];   // first block of each segment; first[nseg] is the grid size
  int nb, na, ndg, nig, nf, np14, nx;
  const uint32_t *bond_ij, *angle_ijk, *dih_ijkl, *imp_ijkl, *fene_ij, *p14_ij;
  const double *bond_kr, *angle_kt, *dih_vd, *imp_vd, *fene_p, *p14_scale;
  const int *dih_grp, *dih_n, *imp_grp, *imp_n;
  int* counters;
  double* info;
  double lj14;
  const int* type;
  int nt, lj96;
  const double4 *lj14_tab, *cap14_tab, *lj14g_tab, *lj14g2_tab;
  double lj_inner, rc;
  int lj_fsw;
  PairTables tables;
  ExclArgs X;
};

template <class R, class S, bool ENER, bool VIR>
static __global__ void __launch_bounds__(256) k_bonded(BondedWork W, BondedArgs A, S F) {
  int sgm = 0;
  while (sgm + 1 < W.nseg && int(blockIdx.x) >= W.first[sgm + 1]) ++sgm;
  const int blk = int(blockIdx.x) - W.first[sgm], nblk = W.first[sgm + 1] - W.first[sgm];
  switch (W.kind[sgm]) {
    case kBkBonds: bonds_body<R, S, ENER, VIR>(blk, nblk, W.nb, W.bond_ij, W.bond_kr, A, F); break;
    case kBkAngles: angles_body<R, S, ENER, VIR>(blk, nblk, W.na, W.angle_ijk, W.angle_kt, A, F); break;
    case kBkDihedrals:
      torsions_body<R, S, ENER, VIR>(blk, nblk, W.ndg, W.dih_grp, W.dih_ijkl, W.dih_vd, W.dih_n, A, F, int(kEDihedral));
      break;
    case kBkImpropers:
      torsions_body<R, S, ENER, VIR>(blk, nblk, W.nig, W.imp_grp, W.imp_ijkl, W.imp_vd, W.imp_n, A, F, int(kEImproper));
      break;
    case kBkFene: fene_body<R, S, ENER, VIR>(blk, nblk, W.nf, W.fene_ij, W.fene_p, A, F, W.counters, W.info); break;
    case kBkPairs14:
      pairs14_body<R, S, ENER, VIR>(blk, nblk, W.np14, W.p14_ij, W.p14_scale, W.lj14, W.type, W.nt, W.lj14_tab, W.cap14_tab, W.lj14g_tab, W.lj14g2_tab, W.lj_inner, W.tables, A, F, W.lj96, W.lj_fsw, W.rc);
      break;
    default: excl_body<S, ENER, VIR>(blk, nblk, W.nx, W.X, A, F); break;
  }
}

}  // namespace capsb
