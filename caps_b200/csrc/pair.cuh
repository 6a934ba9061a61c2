// K-PACK and K-PAIR: the LJ 12-6 plus real-space Coulomb pair kernels over the cluster pair list.
//
// Reference: the FP64 atom-pair loop (core/src/field.cpp:1604-1686: 12-6 LJ with the cut-off shift, Ewald real space
// from the cubic-Hermite table of erf(kappa sqrt s)/sqrt s, field.cpp:1126-1157 and 1593-1602, DSF) and the FP32
// cluster kernel (core/src/nbnxm.cpp:408-567). Excluded pairs are left out of the list (their Ewald / DSF corrections
// are the bonded-phase kernel's, as the reference's FP64 path does at field.cpp:2206-2266).
//
// One warp per work item: a super-cluster of 64 i atoms (8 clusters, kept in shared memory) against up to 32 j
// clusters. Lane l takes i atom l & 7 of every i cluster and j atoms (l >> 3) and (l >> 3) + 4 of each j cluster, so a
// j cluster costs one 128-byte line and its forces are reduced over 8 lanes once per entry, after all 8 i clusters.
// FP32 path: float arithmetic, positions relative to super-cluster origins (the shift of an entry carries the origins'
// difference, so single precision keeps its digits), forces and energies summed as 64-bit fixed point.
// FP64 path: double arithmetic on wrapped absolute positions, the reference's Hermite table for the Ewald term.
#pragma once
#include "common.cuh"
#include "nblist.cuh"
#include "ewald_fit.cuh"

namespace capsb {

constexpr float kPadFar = 1.0e5f;   // padding slots sit this far from their super-cluster's origin (never within reach)

// K-PACK (FP32): per slot, float4 (position relative to the super-cluster origin, charge) and the type index.
static __global__ void k_pack_f32(int nslots, const int* __restrict__ perm, const double* __restrict__ x, const int* __restrict__ ioff, DevCell cell,
                           const double* __restrict__ sc_org, const double* __restrict__ q, const int* __restrict__ type, int pad_type,
                           float4* __restrict__ xq, int* __restrict__ tslot, int* counters, double* __restrict__ x0,
                           long long* __restrict__ fs) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < nslots)   // the pair kernel's slot-order sums (3 x nslots) start at zero
    for (int r = 0; r < 3; ++r) fs[size_t(r) * nslots + s] = 0;
  const bool built = counters[kCntRebuild] != 0;   // a build ran this step: the list was built at these positions
  if (s == 0) {
    counters[kCntPairNext] = 0;   // the pair kernel's work-item counter
    if (built) {
      counters[kCntPrune] = 1;    // a fresh list is pruned at once
      counters[kCntBuilds] += 1;
    }
  }
  const int nsc = counters[kCntNsc];
  if (s >= nslots || s >= 64 * nsc) return;
  const int a = perm[s];
  if (a < 0) {
    xq[s] = make_float4(0.f, 0.f, kPadFar, 0.f);
    tslot[s] = pad_type;
    return;
  }
  if (built)
    for (int r = 0; r < 3; ++r) x0[3 * a + r] = x[3 * a + r];
  const int sc = s >> 6;
  const int o0 = ioff[3 * a], o1 = ioff[3 * a + 1], o2 = ioff[3 * a + 2];
  float p[3];
  for (int r = 0; r < 3; ++r)
    p[r] = float(x[3 * a + r] + (cell.h[r][0] * o0 + cell.h[r][1] * o1 + cell.h[r][2] * o2) - sc_org[3 * sc + r]);
  xq[s] = make_float4(p[0], p[1], p[2], float(q[a]));
  tslot[s] = type[a];
}

// K-PACK (FP64): per slot, double4 (wrapped absolute position, charge) and the type index.
static __global__ void k_pack_f64(int nslots, const int* __restrict__ perm, const double* __restrict__ x, const int* __restrict__ ioff, DevCell cell,
                           const double* __restrict__ q, const int* __restrict__ type, int pad_type, double4* __restrict__ xq, int* __restrict__ tslot,
                           int* counters, double* __restrict__ x0, double* __restrict__ fs) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < nslots)   // the pair kernel's slot-order sums (3 x nslots) start at zero
    for (int r = 0; r < 3; ++r) fs[size_t(r) * nslots + s] = 0;
  const bool built = counters[kCntRebuild] != 0;
  if (s == 0) {
    counters[kCntPairNext] = 0;
    if (built) {
      counters[kCntPrune] = 1;
      counters[kCntBuilds] += 1;
    }
  }
  const int nsc = counters[kCntNsc];
  if (s >= nslots || s >= 64 * nsc) return;
  const int a = perm[s];
  if (a < 0) {
    xq[s] = make_double4(1e7, 1e7, 1e7 + 16.0 * (s & 63), 0.0);
    tslot[s] = pad_type;
    return;
  }
  if (built)
    for (int r = 0; r < 3; ++r) x0[3 * a + r] = x[3 * a + r];
  const int o0 = ioff[3 * a], o1 = ioff[3 * a + 1], o2 = ioff[3 * a + 2];
  double p[3];
  for (int r = 0; r < 3; ++r) p[r] = x[3 * a + r] + (cell.h[r][0] * o0 + cell.h[r][1] * o1 + cell.h[r][2] * o2);
  xq[s] = make_double4(p[0], p[1], p[2], q[a]);
  tslot[s] = type[a];
}

struct PairArgs {
  const int4* work;
  const uint4* ent;
  const float4* ent_shift;
  const unsigned long long* masks;
  const unsigned long long* frozen;   // a frozen pair set: 8 per entry (one per i cluster), the pairs that interact
  const int* counters;
  const int* tslot;
  const float4* xq;      // FP32 path
  const double4* xqd;    // FP64 path
  const float4* tab;     // FP32: per type pair (c6, c12, energy shift, 0)
  const float2* ljf;     // FP32 with geometric mixing: per type (sqrt c6, sqrt c12)
  int batch;             // entries per work item of the list (<= kBatch): the FP32 kernel's staging per warp
  const double4* tabd;   // FP64: per type pair (c6, c12, energy shift, 0)
  const double4* tabcap; // FP64 with a force cap: per type pair (r_cap^2, E at r_cap, |F| at r_cap, 0)
  const double4* tabg;   // FP64 generic forms (tabd.w the form): per type pair (a, b, c, the pair's own cut-off^2)
  const double4* tabg2;  // and the lj/gromacs switch coefficients
  double lj_inner;
  int lj_fsw;            // FP64: CHARMM's force switch on the 12-6 pairs
  PairTables tables;
  const double* gtab;    // FP64 Ewald table: 2 per node (G, h dG/ds)
  int ntab;              // types incl. the padding type
  int gnodes;            // table nodes
  double ghi;            // 1 / node spacing
  DevCell cell;
  double rc2, rc, beta, kc, kcoul, dsf_e0, dsf_f0;
  long long* fsx;        // slot-order force sums (FP32 path: fixed point)
  long long* fsy;
  long long* fsz;
  double* fdx;           // slot-order force sums (FP64 path)
  double* fdy;
  double* fdz;
  EnergySink en;
  int work_cap;
  int* err;              // the error word (range errors of the fixed-point sums)
};

// Work items are taken dynamically: each warp fetches the next unclaimed item from a device counter (reset by the pack
// kernel before every force evaluation). Items differ in size, so a static split leaves SMs idle at the end of the launch.
__device__ __forceinline__ int next_work_item(const int* counters, int lane) {
  int w = 0;
  if (lane == 0) w = atomicAdd(const_cast<int*>(counters) + kCntPairNext, 1);
  return __shfl_sync(0xffffffffu, w, 0);
}

// Sums the j forces (a: j atom q, b: j atom q + 4) over the 8 lanes of an i8 group (lanes xor 1, 2, 4): the first level
// swaps halves so that each lane keeps one j atom's three components, the other two are a butterfly. 9 shuffles; lanes
// with i8 < 4 end with a's sums, lanes with i8 >= 4 with b's.
template <class T>
__device__ __forceinline__ void reduce_j(int i8, T ax, T ay, T az, T bx, T by, T bz, T& kx, T& ky, T& kz) {
  const bool hi = (i8 & 4) != 0;
  kx = hi ? bx : ax, ky = hi ? by : ay, kz = hi ? bz : az;
  const T sx = hi ? ax : bx, sy = hi ? ay : by, sz = hi ? az : bz;
  kx += __shfl_xor_sync(0xffffffffu, sx, 4);
  ky += __shfl_xor_sync(0xffffffffu, sy, 4);
  kz += __shfl_xor_sync(0xffffffffu, sz, 4);
#pragma unroll
  for (int o = 1; o < 4; o <<= 1) {
    kx += __shfl_xor_sync(0xffffffffu, kx, o);
    ky += __shfl_xor_sync(0xffffffffu, ky, o);
    kz += __shfl_xor_sync(0xffffffffu, kz, o);
  }
}

// Sums the i forces of the 8 clusters over the 4 lanes of each i atom (lanes xor 8, 16) by halving: 18 shuffles. Lane
// jq ends with clusters jq and jq + 4: out[0..2] = cluster jq (x, y, z), out[3..5] = cluster jq + 4.
template <class T>
__device__ __forceinline__ void reduce_i(int jq, const T fx[8], const T fy[8], const T fz[8], T out[6]) {
  // level xor 16: keep the clusters c with (c & 2) == (jq & 2): c0 in {0, 1, 4, 5} or c0 ^ 2
  const bool b1 = (jq & 2) != 0, b0 = (jq & 1) != 0;
  T h[4][3];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int c0 = (k & 1) | ((k & 2) << 1);   // 0, 1, 4, 5
    const int c2 = c0 ^ 2;
    const T kx = b1 ? fx[c2] : fx[c0], ky = b1 ? fy[c2] : fy[c0], kz = b1 ? fz[c2] : fz[c0];
    const T sx = b1 ? fx[c0] : fx[c2], sy = b1 ? fy[c0] : fy[c2], sz = b1 ? fz[c0] : fz[c2];
    h[k][0] = kx + __shfl_xor_sync(0xffffffffu, sx, 16);
    h[k][1] = ky + __shfl_xor_sync(0xffffffffu, sy, 16);
    h[k][2] = kz + __shfl_xor_sync(0xffffffffu, sz, 16);
  }
  // level xor 8: of h[k] (k = 0, 1: clusters (jq & 2) + 0/1; k = 2, 3: the same + 4) keep (c & 1) == (jq & 1)
#pragma unroll
  for (int m = 0; m < 2; ++m) {
    const int k0 = 2 * m, k1 = 2 * m + 1;
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      const T kv = b0 ? h[k1][r] : h[k0][r];
      const T sv = b0 ? h[k0][r] : h[k1][r];
      out[3 * m + r] = kv + __shfl_xor_sync(0xffffffffu, sv, 8);
    }
  }
}

// --- FP32 path ---------------------------------------------------------------------------------------------------
// Packed FP32 arithmetic (sm_100 f32x2): a lane's two j atoms of an entry (quarters jq and jq + 4) are the two lanes of
// every add, multiply and multiply-add, so one instruction evaluates both of its pairs with an i atom.
__device__ __forceinline__ float2 p_add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 p_mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 p_fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 p_dup(float v) { return make_float2(v, v); }
// the SFU's approximate 1/sqrt with denormals flushed (squared distances of listed pairs are > 0.01, or 1 for a pair
// left out)
__device__ __forceinline__ float rsqrt_ftz(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// COUL: 0 none; 1 Ewald real space (PME) and 2 damped shifted force through the rational fits of ewald_fit.cuh
// (kappa r_c <= 4); 3 and 4 the same through erfcf and expf (any kappa). COMB: the LJ coefficients of a type pair are
// products of per-type factors (geometric mixing: c6_ab = sqrt(c6_aa c6_bb), the same for c12), taken from a
// per-type table instead of the per-pair one. Force-only evaluations only: the products of rounded factors carry a
// bias of a few 1e-7 per type pair, which the cancelling sums of LJ energies would magnify, so energy steps take the
// per-pair table.
template <int COUL, bool ENER, bool VIR, bool LJ96 = false, bool COMB = false>
static __global__ void __launch_bounds__(128, (ENER || VIR) ? 4 : 5) k_pair_f32(PairArgs A) {
  static_assert(!(COMB && ENER), "energy evaluations use the per-pair table");
  extern __shared__ float4 smem_f4[];
  float4* tab = smem_f4;                                  // ntab * ntab (per-pair table; COMB: ntab float2 factors)
  float2* ljf = reinterpret_cast<float2*>(smem_f4);
  // per warp and i atom: (-x, -x, -y, -y), (-z, -z, q, q) and, COMB, (-6 f6, -6 f6, 12 f12, 12 f12); else the type
  float4* s_xi = smem_f4 + A.ntab * A.ntab;               // 4 warps x 64 x 3
  int* s_ti = reinterpret_cast<int*>(s_xi + 4 * 64 * 3);  // 4 warps x 64
  // a work item's entries, their j atoms and their exclusion masks, staged per warp in one batch of independent loads
  // (sized for the list's entries per work item, A.batch <= kBatch)
  const int nb = A.batch;
  uint4* s_en_all = reinterpret_cast<uint4*>(s_ti + 4 * 64);   // 4 warps x nb entries
  float4* s_sh_all = reinterpret_cast<float4*>(s_en_all + 4 * nb);
  // the j atoms of an entry, shifted by its image and packed per lane quarter jq as the lane's operands:
  // (x_jq, x_jq+4, y_jq, y_jq+4), (z_jq, z_jq+4, q_jq, q_jq+4)
  float4* s_xj_all = s_sh_all + 4 * nb;                         // 4 warps x nb entries x 8 float4
  // COMB: the j atoms' LJ factors per quarter, (f6_jq, f6_jq+4, f12_jq, f12_jq+4); else the j atoms' types
  float4* s_gj_all = s_xj_all + 4 * nb * 8;                     // 4 warps x nb entries x 4 float4 (or 8 int)
  unsigned long long* s_mk_all = reinterpret_cast<unsigned long long*>(s_gj_all + 4 * nb * 4);
  if (COMB) {
    for (int t = threadIdx.x; t < A.ntab; t += blockDim.x) ljf[t] = A.ljf[t];
  } else {
    for (int t = threadIdx.x; t < A.ntab * A.ntab; t += blockDim.x) tab[t] = A.tab[t];
  }
  __syncthreads();
  const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i8 = lane & 7, jq = lane >> 3;
  float4* xi_s = s_xi + 3 * 64 * wib;
  int* ti_s = s_ti + 64 * wib;
  if (blockIdx.x == 0 && threadIdx.x == 0) {   // the step's list work is done: lower the rebuild and prune flags
    int* c = const_cast<int*>(A.counters);
    c[kCntRebuild] = 0;
    c[kCntPrune] = 0;
  }
  // a list build that ran out of room leaves stale work items: skip the pass, the host reports the error
  if (A.counters[kCntErr] & (kErrListOverflow | kErrMaskOverflow | kErrScOverflow | kErrColumnTooBig | kErrExclOverflow)) return;
  const int nwork = min(A.counters[kCntWork], A.work_cap);
  const int pad = A.ntab - 1;
  const float rc2 = float(A.rc2), beta = float(A.beta), kc = float(A.kc), kcoul = float(A.kcoul);
  const float2 ku = p_dup(float(A.beta * A.beta / kEwUMax)), nkap3 = p_dup(-float(A.beta * A.beta * A.beta));
  const float e0 = float(A.dsf_e0), f0 = float(A.dsf_f0), rcf = float(A.rc);
  // energy and virial: every pair's terms rounded to fixed point on their own (2^24 per kcal/mol), so that the totals do
  // not depend on the list's grouping of pairs into entries and work items
  long long acc_v = 0, acc_c = 0, acc_w[6] = {0, 0, 0, 0, 0, 0};
  double acc_np = 0, acc_nl = 0;
  constexpr float kq = 16777216.f;
  for (int w = next_work_item(A.counters, lane); w < nwork; w = next_work_item(A.counters, lane)) {
    const int4 wk = A.work[w];
    const int sc = wk.x;
    for (int t = lane; t < 64; t += 32) {
      const float4 v = A.xq[64 * sc + t];
      const int ty = A.tslot[64 * sc + t];
      const float q = v.w * kcoul;
      xi_s[3 * t] = make_float4(-v.x, -v.x, -v.y, -v.y);
      xi_s[3 * t + 1] = make_float4(-v.z, -v.z, q, q);
      if (COMB) {
        const float2 g = ljf[ty];
        xi_s[3 * t + 2] = make_float4(-6.f * g.x, -6.f * g.x, 12.f * g.y, 12.f * g.y);
      }
      ti_s[t] = ty;
    }
    __syncwarp();
    // real i atoms of the lane, per i cluster c, in the layout of an entry's prune mask (bit c: the pair with j atom
    // jq, bit c + 8: with jq + 4)
    unsigned ireal = 0;
#pragma unroll
    for (int c = 0; c < 8; ++c) ireal |= unsigned(ti_s[8 * c + i8] != pad) << c;
    ireal |= ireal << 8;
    float fix[8], fiy[8], fiz[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) fix[c] = fiy[c] = fiz[c] = 0.f;
    float npair = 0.f, nlist = 0.f;
    uint4* s_en = s_en_all + nb * wib;
    float4* s_sh = s_sh_all + nb * wib;
    float4* s_xj = s_xj_all + nb * 8 * wib;
    float4* s_gj = s_gj_all + nb * 4 * wib;
    int* s_tj = reinterpret_cast<int*>(s_gj);
    unsigned long long* s_mk = s_mk_all + nb * 8 * wib;
    const int ne = min(wk.z, nb);
    if (lane < ne) {
      s_en[lane] = A.ent[wk.y + lane];
      s_sh[lane] = A.ent_shift[wk.y + lane];
    }
    __syncwarp();
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int t = lane + 32 * k;   // entry t / 8, j atom t % 8
      if (t < 8 * ne) {
        const int e = t >> 3, j = t & 7, q4 = j & 3, h = j >> 2;
        const uint4 e4 = s_en[e];
        const float4 sh = s_sh[e];
        const int ja = 8 * int(e4.x) + j;
        const float4 v = A.xq[ja];
        float* px = reinterpret_cast<float*>(s_xj + 8 * e + 2 * q4);
        px[h] = v.x + sh.x;
        px[2 + h] = v.y + sh.y;
        px[4 + h] = v.z + sh.z;
        px[6 + h] = v.w;
        const int ty = A.tslot[ja];
        if (COMB) {
          const float2 g = ljf[ty];
          float* pg = reinterpret_cast<float*>(s_gj + 4 * e + q4);
          pg[h] = g.x;
          pg[2 + h] = g.y;
        } else {
          s_tj[t] = ty;
        }
        s_mk[t] = e4.z ? A.masks[8 * size_t(e4.z - 1) + j] : ~0ull;   // entry t / 8, i cluster t % 8
      }
    }
    __syncwarp();
    for (int el = 0; el < ne; ++el) {
      const uint4 en = s_en[el];
      const unsigned hmask = en.w & 0xffffu;
      if (!hmask) continue;
      const int cj = int(en.x);
      const unsigned imask = (hmask | (hmask >> 8)) & 255u;
      // the lane's listed pairs of the entry: a j half within the prune radius, a real i atom and, where the entry
      // has exclusion masks, bits jq and jq + 4 of the i atom's row of its cluster's mask
      unsigned lv = hmask & ireal;
      if (en.z) {
        unsigned xm = 0;
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          const unsigned b = unsigned(s_mk[8 * el + c] >> (8 * i8 + jq));
          xm |= ((b & 1u) << c) | (((b >> 4) & 1u) << (c + 8));
        }
        lv &= xm;
      }
      const int j0 = 8 * cj + jq, j1 = j0 + 4;
      const float4 xa = s_xj[8 * el + 2 * jq], xb = s_xj[8 * el + 2 * jq + 1];
      const float2 xj = make_float2(xa.x, xa.y), yj = make_float2(xa.z, xa.w), zj = make_float2(xb.x, xb.y), qj = make_float2(xb.z, xb.w);
      float2 g6j = p_dup(0.f), g12j = p_dup(0.f);
      int t0 = 0, t1 = 0;
      if (COMB) {
        const float4 gg = s_gj[4 * el + jq];
        g6j = make_float2(gg.x, gg.y);
        g12j = make_float2(gg.z, gg.w);
      } else {
        t0 = s_tj[8 * el + jq];
        t1 = s_tj[8 * el + jq + 4];
      }
      float2 fjx = p_dup(0.f), fjy = p_dup(0.f), fjz = p_dup(0.f);
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        if (!((imask >> c) & 1u)) continue;
        const float4 pa = xi_s[3 * (8 * c + i8)], pb = xi_s[3 * (8 * c + i8) + 1];
        const bool l0 = (lv >> c) & 1u, l1 = (lv >> (c + 8)) & 1u;
        const float2 dx = p_add(xj, make_float2(pa.x, pa.y)), dy = p_add(yj, make_float2(pa.z, pa.w)), dz = p_add(zj, make_float2(pb.x, pb.y));
        const float2 r2 = p_fma(dx, dx, p_fma(dy, dy, p_mul(dz, dz)));
        const bool ok0 = l0 && (r2.x < rc2), ok1 = l1 && (r2.y < rc2);
        if (ENER) {
          npair += float(ok0) + float(ok1);
          nlist += float(l0) + float(l1);
        }
        const float2 r2s = make_float2(ok0 ? r2.x : 1.f, ok1 ? r2.y : 1.f);
        const float2 rinv = make_float2(rsqrt_ftz(r2s.x), rsqrt_ftz(r2s.y));
        const float2 r2i = p_mul(rinv, rinv);
        const float2 r6i = p_mul(p_mul(r2i, r2i), r2i);
        float2 fr, elj;
        if (COMB) {
          const float4 pl = xi_s[3 * (8 * c + i8) + 2];
          const float2 nC6 = p_mul(make_float2(pl.x, pl.y), g6j), C12 = p_mul(make_float2(pl.z, pl.w), g12j);
          fr = p_mul(p_mul(r6i, p_fma(C12, r6i, nC6)), r2i);   // (12 c12 r^-12 - 6 c6 r^-6) / r^2
        } else {
          const int ti = ti_s[8 * c + i8];
          const float4 cc0 = tab[ti * A.ntab + t0], cc1 = tab[ti * A.ntab + t1];
          const float2 c6 = make_float2(cc0.x, cc1.x), c12 = make_float2(cc0.y, cc1.y);
          // 12-6: a = c12 r^-6; 9-6: a = c9 r^-3 (the table's second slot holds c12 or c9): E = r^-6 (a - c6) - shift
          const float2 a12 = p_mul(c12, LJ96 ? p_mul(r2i, rinv) : r6i);
          fr = p_mul(p_mul(r6i, p_fma(p_dup(LJ96 ? 9.f : 12.f), a12, p_mul(p_dup(-6.f), c6))), r2i);
          if (ENER) elj = p_fma(r6i, p_add(a12, p_mul(p_dup(-1.f), c6)), make_float2(-cc0.z, -cc1.z));
        }
        if (ENER) acc_v += (ok0 ? __float2ll_rn(elj.x * kq) : 0ll) + (ok1 ? __float2ll_rn(elj.y * kq) : 0ll);
        if (COUL == 1 || COUL == 2) {
          // E = qq (1/r - kappa g(u)), F = qq (1/r^3 - kappa^3 h(u)), u = (kappa r)^2: FMAs and one division per pair
          const float2 qq = p_mul(make_float2(pb.z, pb.w), qj);
          const float2 t = p_mul(r2s, ku);
          float2 fc = p_mul(qq, p_fma(nkap3, ew_h2(t), p_mul(rinv, r2i)));
          if (COUL == 2) fc = p_fma(p_mul(qq, p_dup(-f0)), rinv, fc);
          fr = p_add(fr, fc);
          if (ENER) {
            float2 ecp = p_mul(qq, p_fma(p_dup(-beta), ew_g2(t), rinv));
            if (COUL == 2) ecp = p_fma(qq, p_fma(p_dup(f0), p_add(p_mul(r2s, rinv), p_dup(-rcf)), p_dup(-e0)), ecp);
            acc_c += (ok0 ? __float2ll_rn(ecp.x * kq) : 0ll) + (ok1 ? __float2ll_rn(ecp.y * kq) : 0ll);
          }
        }
        if (COUL == 3 || COUL == 4) {
          const float2 qq = p_mul(make_float2(pb.z, pb.w), qj);
          const float2 r = p_mul(r2s, rinv);
          float fcs[2], ecs[2];
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const float rh = h ? r.y : r.x, ih = h ? rinv.y : rinv.x, qh = h ? qq.y : qq.x;
            const float br = beta * rh;
            const float erfcv = erfcf(br);
            const float ex = __expf(-br * br);
            fcs[h] = qh * fmaf(erfcv, ih, kc * ex) * (ih * ih);
            if (COUL == 4) fcs[h] -= qh * f0 * ih;
            ecs[h] = qh * erfcv * ih;
            if (COUL == 4) ecs[h] += qh * (f0 * (rh - rcf) - e0);
          }
          fr = p_add(fr, make_float2(fcs[0], fcs[1]));
          if (ENER) acc_c += (ok0 ? __float2ll_rn(ecs[0] * kq) : 0ll) + (ok1 ? __float2ll_rn(ecs[1] * kq) : 0ll);
        }
        fr = make_float2(ok0 ? fr.x : 0.f, ok1 ? fr.y : 0.f);
        const float2 fx = p_mul(fr, dx), fy = p_mul(fr, dy), fz = p_mul(fr, dz);
        fjx = p_add(fjx, fx);
        fjy = p_add(fjy, fy);
        fjz = p_add(fjz, fz);
        fix[c] -= fx.x + fx.y;
        fiy[c] -= fy.x + fy.y;
        fiz[c] -= fz.x + fz.y;
        if (VIR) {   // fr is 0 for the pairs left out
          const float2 w6[6] = {p_mul(fx, dx), p_mul(fy, dy), p_mul(fz, dz), p_mul(fx, dy), p_mul(fx, dz), p_mul(fy, dz)};
#pragma unroll
          for (int k = 0; k < 6; ++k) acc_w[k] += __float2ll_rn(w6[k].x * kq) + __float2ll_rn(w6[k].y * kq);
        }
      }
      // j forces: summed over the 8 lanes holding the same j atoms, then one fixed-point add per component
      {
        float kx, ky, kz;
        reduce_j(i8, fjx.x, fjy.x, fjz.x, fjx.y, fjy.y, fjz.y, kx, ky, kz);
        const int comp = i8 & 3;
        if (comp < 3) {
          const float v = comp == 0 ? kx : comp == 1 ? ky : kz;
          long long* dst = comp == 0 ? A.fsx : comp == 1 ? A.fsy : A.fsz;
          if (v != 0.f) fix_add_f(dst + ((i8 & 4) ? j1 : j0), v, A.err);
        }
      }
    }
    // i forces: summed over the 4 lanes of each i atom; lane jq adds clusters jq and jq + 4
    {
      float fo[6];
      reduce_i(jq, fix, fiy, fiz, fo);
#pragma unroll
      for (int m = 0; m < 2; ++m) {
        const int c = jq + 4 * m;
        if (!((ireal >> c) & 1u)) continue;
        const int s = 64 * sc + 8 * c + i8;
        if (fo[3 * m] != 0.f) fix_add_f(A.fsx + s, fo[3 * m], A.err);
        if (fo[3 * m + 1] != 0.f) fix_add_f(A.fsy + s, fo[3 * m + 1], A.err);
        if (fo[3 * m + 2] != 0.f) fix_add_f(A.fsz + s, fo[3 * m + 2], A.err);
      }
    }
    if (ENER) {
      acc_np += double(warp_sum(npair));   // whole numbers: exact in any order
      acc_nl += double(warp_sum(nlist));
    }
    __syncwarp();
  }
  if (ENER) {
    acc_v = warp_sum(acc_v);
    acc_c = warp_sum(acc_c);
  }
  if (VIR)
    for (int k = 0; k < 6; ++k) acc_w[k] = warp_sum(acc_w[k]);
  if (lane == 0) {
    if (ENER) {
      atomic_add_fix(A.en.fix + kEVdw, acc_v);
      atomic_add_fix(A.en.fix + kECoul, acc_c);
      A.en.add(kEPairs, acc_np, true);
      A.en.add(kEListed, acc_nl, true);
    }
    if (VIR)
      for (int k = 0; k < 6; ++k) atomic_add_fix(A.en.fix + kEW0 + k, acc_w[k]);
  }
}

// --- FP64 path ---------------------------------------------------------------------------------------------------

// The reference's ewald_ef (field.cpp:1593-1602): E = 1/r - G(s), F = 1/r^3 + 2 dG/ds by cubic Hermite interpolation.
__device__ __forceinline__ void ewald_ef(const double* __restrict__ gt, double ghi, double s, double rinv, double& E, double& F) {
  const double u = s * ghi;
  const int k = int(u);
  const double t = u - double(k), t2 = t * t;
  const double g0 = gt[2 * k], g1 = gt[2 * k + 1], g2 = gt[2 * k + 2], g3 = gt[2 * k + 3];
  const double G = g0 + t2 * (3 - 2 * t) * (g2 - g0) + t * (1 - t) * ((1 - t) * g1 - t * g3);
  const double dG = (6 * t * (1 - t) * (g2 - g0) * ghi) + (1 - t) * (1 - 3 * t) * g1 * ghi + t * (3 * t - 2) * g3 * ghi;
  E = rinv - G;
  F = rinv * rinv * rinv + 2 * dG;
}

// erfc(x) and exp(-x^2) by Abramowitz & Stegun 7.1.26, the reference's erfc_exp (field.cpp:585-590): the closed form a
// frozen pair takes beyond the cut-off, where the Ewald table ends.
__device__ __forceinline__ double erfc_exp_as(double x, double& ex2) {
  const double P = 0.3275911, A1 = 0.254829592, A2 = -0.284496736, A3 = 1.421413741, A4 = -1.453152027, A5 = 1.061405429;
  ex2 = exp(-x * x);
  const double t = 1.0 / (1.0 + P * x);
  return t * (A1 + t * (A2 + t * (A3 + t * (A4 + t * A5)))) * ex2;
}

// FROZEN: the pairs are those of the frozen set (A.frozen), whatever their distance now (field.cpp:1700); one beyond
// the cut-off takes the closed-form Coulomb term (field.cpp:1759-1768).
// CAP: the rare forms' variant (the push-off force cap, the generic pair forms, CHARMM's force switch), taken with energies
// and virial on; the plain variants carry none of their branches.
template <int COUL, bool ENER, bool VIR, bool CAP = false, bool LJ96 = false, bool FROZEN = false>
static __global__ void __launch_bounds__(128, 2) k_pair_f64(PairArgs A) {
  extern __shared__ double4 smem_d4[];
  double4* tab = smem_d4;                                   // ntab * ntab
  double* gt = reinterpret_cast<double*>(tab + A.ntab * A.ntab);   // 2 * gnodes with Coulomb, none without (as the launch sizes it)
  double4* s_xi = reinterpret_cast<double4*>(gt + (COUL != 0 ? 2 * A.gnodes : 0));   // 4 x 64
  int* s_ti = reinterpret_cast<int*>(s_xi + 4 * 64);
  for (int t = threadIdx.x; t < A.ntab * A.ntab; t += blockDim.x) tab[t] = A.tabd[t];
  if (COUL != 0)
    for (int t = threadIdx.x; t < 2 * A.gnodes; t += blockDim.x) gt[t] = A.gtab[t];
  __syncthreads();
  const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i8 = lane & 7, jq = lane >> 3;
  double4* xi_s = s_xi + 64 * wib;
  int* ti_s = s_ti + 64 * wib;
  if (blockIdx.x == 0 && threadIdx.x == 0) {   // the step's list work is done: lower the rebuild and prune flags
    int* c = const_cast<int*>(A.counters);
    c[kCntRebuild] = 0;
    c[kCntPrune] = 0;
  }
  if (A.counters[kCntErr] & (kErrListOverflow | kErrMaskOverflow | kErrScOverflow | kErrColumnTooBig | kErrExclOverflow)) return;
  const int nwork = min(A.counters[kCntWork], A.work_cap);
  const int pad = A.ntab - 1;
  double acc_v = 0, acc_c = 0, acc_w[6] = {0, 0, 0, 0, 0, 0};
  for (int w = next_work_item(A.counters, lane); w < nwork; w = next_work_item(A.counters, lane)) {
    const int4 wk = A.work[w];
    const int sc = wk.x;
    for (int t = lane; t < 64; t += 32) {
      double4 v = A.xqd[64 * sc + t];
      v.w *= A.kcoul;
      xi_s[t] = v;
      ti_s[t] = A.tslot[64 * sc + t];
    }
    __syncwarp();
    unsigned ireal = 0;
#pragma unroll
    for (int c = 0; c < 8; ++c) ireal |= unsigned(ti_s[8 * c + i8] != pad) << c;
    double fix[8], fiy[8], fiz[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) fix[c] = fiy[c] = fiz[c] = 0.0;
    double ev = 0, ec = 0, vw[6] = {0, 0, 0, 0, 0, 0};
    for (int e = wk.y; e < wk.y + wk.z; ++e) {
      const uint4 en = A.ent[e];
      const int cj = int(en.x);
      const unsigned hmask = en.w & 0xffffu;
      if (!hmask) continue;
      const unsigned imask = (hmask | (hmask >> 8)) & 255u;
      int qa, qb, qc;
      unpack_image(en.y >> 8, qa, qb, qc);
      const double Sx = A.cell.h[0][0] * qa + A.cell.h[0][1] * qb + A.cell.h[0][2] * qc;
      const double Sy = A.cell.h[1][0] * qa + A.cell.h[1][1] * qb + A.cell.h[1][2] * qc;
      const double Sz = A.cell.h[2][0] * qa + A.cell.h[2][1] * qb + A.cell.h[2][2] * qc;
      const int j0 = 8 * cj + jq, j1 = j0 + 4;
      const double4 a0 = A.xqd[j0], a1 = A.xqd[j1];
      const int t0 = A.tslot[j0], t1 = A.tslot[j1];
      double f0x = 0, f0y = 0, f0z = 0, f1x = 0, f1y = 0, f1z = 0;
#pragma unroll 2
      for (int c = 0; c < 8; ++c) {
        if (!((imask >> c) & 1u)) continue;
        const unsigned long long mm = FROZEN ? A.frozen[8 * size_t(e) + c] : en.z ? A.masks[8 * size_t(en.z - 1) + c] : ~0ull;
        const double4 xi = xi_s[8 * c + i8];
        const int ti = ti_s[8 * c + i8];
        const bool oki = (ireal >> c) & 1u;
        // d = xs_j - (xs_i - S), as field.cpp:1628-1636
        const double xs = xi.x - Sx, ys = xi.y - Sy, zs = xi.z - Sz;
#pragma unroll
        for (int jj = 0; jj < 2; ++jj) {
          if (!((hmask >> (c + 8 * jj)) & 1u)) continue;
          const double4 aj = jj ? a1 : a0;
          const int tj = jj ? t1 : t0;
          const int bit = 8 * i8 + jq + 4 * jj;
          const double dx = aj.x - xs, dy = aj.y - ys, dz = aj.z - zs;
          const double r2 = dx * dx + dy * dy + dz * dz;
          const bool ok = oki && ((mm >> bit) & 1ull) && (FROZEN || r2 < A.rc2);
          if (!ok) continue;
          const double r2i = 1 / r2, r6i = r2i * r2i * r2i, rinv = sqrt(r2i);
          const double4 cc = tab[ti * A.ntab + tj];
          double fr;
          const double4 cp = CAP ? A.tabcap[ti * A.ntab + tj] : make_double4(0, 0, 0, 0);
          if (CAP && r2 < cp.x) {
            // the push-off cap (field.cpp:1534-1538): LJ continued linearly inside the radius where |F| reaches the cap
            const double r = r2 * rinv, rcp = sqrt(cp.x);
            fr = cp.z * rinv;   // F / r with |F| = the cap
            if (ENER) ev += cp.y + cp.z * (rcp - r) - cc.z;
          } else if ((CAP || FROZEN) && cc.w != 0) {
            // a generic form (field.cpp:1381-1396), nothing beyond the pair's own cut-off (and no shift there)
            const double4 g = A.tabg[ti * A.ntab + tj];
            double e = 0;
            fr = (g.w > 0 && r2 > g.w) ? 0.0 : generic_pair(int(cc.w), g, A.tabg2[ti * A.ntab + tj], A.lj_inner, A.tables, r2, e);
            if (ENER && !(g.w > 0 && r2 > g.w)) ev += e - cc.z;
          } else {
            if (LJ96) {   // field.cpp:1658-1661
              const double r9i = r6i * r2i * rinv;
              fr = (9 * cc.y * r9i - 6 * cc.x * r6i) * r2i;
              if (ENER) ev += cc.y * r9i - cc.x * r6i - cc.z;
            } else if ((CAP || FROZEN) && A.lj_fsw) {
              fr = charmm_fsw(cc.y, cc.x, A.lj_inner, A.rc, r2, ev, ENER);
            } else {
              fr = r6i * (12 * cc.y * r6i - 6 * cc.x) * r2i;
              if (ENER) ev += r6i * (cc.y * r6i - cc.x) - cc.z;
            }
          }
          if (COUL != 0 && FROZEN && !(r2 < A.rc2)) {
            const double qq = xi.w * aj.w;
            const double r = sqrt(r2);
            double ex2;
            const double er = erfc_exp_as(A.beta * r, ex2);   // beta: the Ewald or DSF coefficient; kc = 2 beta / sqrt(pi)
            if (COUL == 1) {
              if (ENER) ec += qq * er / r;
              fr += qq * (er / r2 + A.kc * ex2 / r) / r;
            } else {
              if (ENER) ec += qq * (er / r - A.dsf_e0 + A.dsf_f0 * (r - A.rc));
              fr += qq * (er / r2 + A.kc * ex2 / r - A.dsf_f0) / r;
            }
          } else if (COUL != 0) {
            const double qq = xi.w * aj.w;
            double E, Fc;
            ewald_ef(gt, A.ghi, r2, rinv, E, Fc);
            if (COUL == 1) {
              if (ENER) ec += qq * E;
              fr += qq * Fc;
            } else {
              if (ENER) ec += qq * (E - A.dsf_e0 + A.dsf_f0 * (r2 * rinv - A.rc));
              fr += qq * (Fc - A.dsf_f0 * rinv);
            }
          }
          const double fx = fr * dx, fy = fr * dy, fz = fr * dz;
          if (jj) f1x += fx, f1y += fy, f1z += fz;
          else f0x += fx, f0y += fy, f0z += fz;
          fix[c] -= fx;
          fiy[c] -= fy;
          fiz[c] -= fz;
          if (VIR) {
            vw[0] += fx * dx;
            vw[1] += fy * dy;
            vw[2] += fz * dz;
            vw[3] += fx * dy;
            vw[4] += fx * dz;
            vw[5] += fy * dz;
          }
        }
      }
      {
        double kx, ky, kz;
        reduce_j(i8, f0x, f0y, f0z, f1x, f1y, f1z, kx, ky, kz);
        const int comp = i8 & 3;
        if (comp < 3) {
          const double v = comp == 0 ? kx : comp == 1 ? ky : kz;
          double* dst = comp == 0 ? A.fdx : comp == 1 ? A.fdy : A.fdz;
          if (v != 0.0) atomicAdd(dst + ((i8 & 4) ? j1 : j0), v);
        }
      }
    }
    {
      double fo[6];
      reduce_i(jq, fix, fiy, fiz, fo);
#pragma unroll
      for (int m = 0; m < 2; ++m) {
        const int c = jq + 4 * m;
        if (!((ireal >> c) & 1u)) continue;
        const int s = 64 * sc + 8 * c + i8;
        if (fo[3 * m] != 0.0) atomicAdd(A.fdx + s, fo[3 * m]);
        if (fo[3 * m + 1] != 0.0) atomicAdd(A.fdy + s, fo[3 * m + 1]);
        if (fo[3 * m + 2] != 0.0) atomicAdd(A.fdz + s, fo[3 * m + 2]);
      }
    }
    if (ENER) {
      acc_v += warp_sum(ev);
      acc_c += warp_sum(ec);
    }
    if (VIR)
      for (int k = 0; k < 6; ++k) acc_w[k] += warp_sum(vw[k]);
    __syncwarp();
  }
  if (lane == 0) {
    if (ENER) {
      A.en.add(kEVdw, acc_v, false);
      A.en.add(kECoul, acc_c, false);
    }
    if (VIR)
      for (int k = 0; k < 6; ++k) A.en.add(kEW0 + k, acc_w[k], false);
  }
}

// K-FREEZE: the frozen pair set of Evaluator::freeze_pairs (field.cpp:2541-2559) on the FP64 path: per entry and i
// cluster the 64 atom pairs that are listed, real, not excluded and inside r_c at the packed positions; the entry's
// half mask becomes their union, so that the pair kernel visits exactly those halves. One thread per entry.
static __global__ void __launch_bounds__(128) k_freeze(PairArgs A, uint4* __restrict__ ent, unsigned long long* __restrict__ frozen) {
  if (A.counters[kCntErr] & (kErrListOverflow | kErrMaskOverflow | kErrScOverflow | kErrColumnTooBig | kErrExclOverflow)) return;
  const int nwork = min(A.counters[kCntWork], A.work_cap);
  const int pad = A.ntab - 1;
  const int lane = threadIdx.x & 31;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < nwork; w += nwarps) {
    const int4 wk = A.work[w];
    for (int e = wk.y + lane; e < wk.y + wk.z; e += 32) {
      uint4 en = ent[e];
      int qa, qb, qc;
      unpack_image(en.y >> 8, qa, qb, qc);
      const double Sx = A.cell.h[0][0] * qa + A.cell.h[0][1] * qb + A.cell.h[0][2] * qc;
      const double Sy = A.cell.h[1][0] * qa + A.cell.h[1][1] * qb + A.cell.h[1][2] * qc;
      const double Sz = A.cell.h[2][0] * qa + A.cell.h[2][1] * qb + A.cell.h[2][2] * qc;
      const unsigned built = en.y & 255u;
      unsigned keep = 0;
      for (int c = 0; c < 8; ++c) {
        unsigned long long m = 0;
        if ((built >> c) & 1u) {
          const unsigned long long mm = en.z ? A.masks[8 * size_t(en.z - 1) + c] : ~0ull;
          for (int i8 = 0; i8 < 8; ++i8) {
            const int si = 64 * wk.x + 8 * c + i8;
            if (A.tslot[si] == pad) continue;
            const double4 xi = A.xqd[si];
            const double xs = xi.x - Sx, ys = xi.y - Sy, zs = xi.z - Sz;
            for (int jl = 0; jl < 8; ++jl) {
              const int bit = 8 * i8 + jl;
              const int sj = 8 * int(en.x) + jl;
              if (!((mm >> bit) & 1ull) || A.tslot[sj] == pad) continue;
              const double4 aj = A.xqd[sj];
              const double dx = aj.x - xs, dy = aj.y - ys, dz = aj.z - zs;
              if (dx * dx + dy * dy + dz * dz < A.rc2) m |= 1ull << bit;
            }
          }
        }
        frozen[8 * size_t(e) + c] = m;
        if (m & 0x0f0f0f0f0f0f0f0full) keep |= 1u << c;         // j atoms 0-3: the lower half
        if (m & 0xf0f0f0f0f0f0f0f0ull) keep |= 1u << (c + 8);   // j atoms 4-7: the upper half
      }
      en.w = keep;
      ent[e] = en;
    }
  }
}

// K-COUNT-PAIRS: the atom pairs of the list within r_list = r_c + skin at the positions of its build (x0), real and not
// excluded, each unordered pair once: Evaluator::pairs() of the reference's FP64 atom-pair list (field.cpp:1030-1049).
static __global__ void __launch_bounds__(128) k_count_pairs(PairArgs A, const uint4* __restrict__ ent, const int* __restrict__ perm,
                                                           const double* __restrict__ x0, const int* __restrict__ ioff, double rl2,
                                                           unsigned long long* __restrict__ out) {
  if (A.counters[kCntErr] & (kErrListOverflow | kErrMaskOverflow | kErrScOverflow | kErrColumnTooBig | kErrExclOverflow)) return;
  const int nwork = min(A.counters[kCntWork], A.work_cap);
  const int lane = threadIdx.x & 31;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  unsigned long long cnt = 0;
  auto pos = [&](int a, double p[3]) {
    const int o0 = ioff[3 * a], o1 = ioff[3 * a + 1], o2 = ioff[3 * a + 2];
    for (int r = 0; r < 3; ++r) p[r] = x0[3 * a + r] + (A.cell.h[r][0] * o0 + A.cell.h[r][1] * o1 + A.cell.h[r][2] * o2);
  };
  for (int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < nwork; w += nwarps) {
    const int4 wk = A.work[w];
    for (int e = wk.y + lane; e < wk.y + wk.z; e += 32) {
      const uint4 en = ent[e];
      int qa, qb, qc;
      unpack_image(en.y >> 8, qa, qb, qc);
      const double S[3] = {A.cell.h[0][0] * qa + A.cell.h[0][1] * qb + A.cell.h[0][2] * qc, A.cell.h[1][0] * qa + A.cell.h[1][1] * qb + A.cell.h[1][2] * qc,
                           A.cell.h[2][0] * qa + A.cell.h[2][1] * qb + A.cell.h[2][2] * qc};
      const unsigned built = en.y & 255u;
      for (int c = 0; c < 8; ++c) {
        if (!((built >> c) & 1u)) continue;
        const unsigned long long mm = en.z ? A.masks[8 * size_t(en.z - 1) + c] : ~0ull;
        for (int i8 = 0; i8 < 8; ++i8) {
          const int ai = perm[64 * wk.x + 8 * c + i8];
          if (ai < 0) continue;
          double pi[3];
          pos(ai, pi);
          for (int jl = 0; jl < 8; ++jl) {
            const int aj = perm[8 * int(en.x) + jl];
            if (aj < 0 || !((mm >> (8 * i8 + jl)) & 1ull)) continue;
            double pj[3];
            pos(aj, pj);
            const double dx = pj[0] - (pi[0] - S[0]), dy = pj[1] - (pi[1] - S[1]), dz = pj[2] - (pi[2] - S[2]);
            cnt += dx * dx + dy * dy + dz * dz < rl2 ? 1 : 0;
          }
        }
      }
    }
  }
  if (cnt) atomicAdd(out, cnt);
}

// K-PRUNE (dynamic pruning, as core/src/nbnxm.cpp:328-363 does on the CPU): each entry's mask is rewritten to the
// (i cluster, j half) pairs with at least one atom pair inside r_prune = r_c + b at the present positions; the pair
// kernels read that mask. The j halves are the cluster's lower-x and upper-x four atoms (the cluster split orders its
// atoms along x), so a half mask drops the far half of a j cluster that reaches an i cluster with its near half only. Pruned again once an atom has moved b/2 since the last prune, so no pair inside r_c is lost. Gated by
// the prune flag, set by the displacement check and by every list build. FP32 path: packed float positions; FP64 path:
// packed double positions.
template <bool DBL>
static __global__ void __launch_bounds__(128) k_prune(PairArgs A, double rprune2, uint4* __restrict__ ent, int n, const double* __restrict__ x,
                                                     double* __restrict__ xp) {
  if (*(volatile const int*)(A.counters + kCntPrune) == 0) return;
  // the positions of this prune, for the next displacement check; and the prune count
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 3 * n; i += gridDim.x * blockDim.x) xp[i] = x[i];
  if (blockIdx.x == 0 && threadIdx.x == 0) const_cast<int*>(A.counters)[kCntPrunes] += 1;
  if (A.counters[kCntErr] & (kErrListOverflow | kErrMaskOverflow | kErrScOverflow | kErrColumnTooBig | kErrExclOverflow)) return;
  // per warp: the work item's i atoms, its entries' j atoms (w: 1 real, 0 padding) and the new half masks
  __shared__ float4 s_xi[4][64];
  __shared__ float4 s_xj[4][kBatch * 8];
  __shared__ unsigned s_keep[4][kBatch];
  const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i8 = lane & 7, jq = lane >> 3;
  const int nwork = min(A.counters[kCntWork], A.work_cap);
  const int pad = A.ntab - 1;
  const float rp2 = float(rprune2);
  for (int w = blockIdx.x * 4 + wib; w < nwork; w += gridDim.x * 4) {
    const int4 wk = A.work[w];
    const int sc = wk.x;
    const int ne = min(wk.z, kBatch);
    // one batch of independent loads: i atoms, the entries, then every entry's 8 j atoms with the entry's image shift
    uint4 en = make_uint4(0u, 0u, 0u, 0u);
    float sx = 0.f, sy = 0.f, sz = 0.f;
    if (lane < ne) {
      en = ent[wk.y + lane];
      if (DBL) {
        int qa, qb, qc;
        unpack_image(en.y >> 8, qa, qb, qc);
        sx = float(A.cell.h[0][0] * qa + A.cell.h[0][1] * qb + A.cell.h[0][2] * qc);
        sy = float(A.cell.h[1][0] * qa + A.cell.h[1][1] * qb + A.cell.h[1][2] * qc);
        sz = float(A.cell.h[2][0] * qa + A.cell.h[2][1] * qb + A.cell.h[2][2] * qc);
      } else {
        const float4 sh = A.ent_shift[wk.y + lane];
        sx = sh.x, sy = sh.y, sz = sh.z;
      }
    }
    for (int t = lane; t < 64; t += 32) {
      float4 v;
      if (DBL) {
        const double4 d = A.xqd[64 * sc + t];
        v = make_float4(float(d.x), float(d.y), float(d.z), 0.f);
      } else {
        v = A.xq[64 * sc + t];
      }
      v.w = A.tslot[64 * sc + t] != pad ? 1.f : 0.f;
      s_xi[wib][t] = v;
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int t = lane + 32 * k;   // entry t / 8, j atom t % 8
      const int e = t >> 3;
      const unsigned cj = __shfl_sync(0xffffffffu, en.x, e & 31);
      const float ex = __shfl_sync(0xffffffffu, sx, e & 31), ey = __shfl_sync(0xffffffffu, sy, e & 31),
                  ez = __shfl_sync(0xffffffffu, sz, e & 31);
      if (e < ne) {
        const int ja = 8 * int(cj) + (t & 7);
        float4 v;
        // FP64 path: absolute positions rounded to float (1e-5 Å at 100 Å), far inside the 0.8 Å prune margin
        if (DBL) {
          const double4 d = A.xqd[ja];
          v = make_float4(float(d.x), float(d.y), float(d.z), 0.f);
        } else {
          v = A.xq[ja];
        }
        v.x += ex, v.y += ey, v.z += ez;
        v.w = A.tslot[ja] != pad ? 1.f : 0.f;
        s_xj[wib][t] = v;
      }
    }
    __syncwarp();
    for (int el = 0; el < ne; ++el) {
      const unsigned built = __shfl_sync(0xffffffffu, en.y, el) & 255u;
      const float4 a0 = s_xj[wib][8 * el + jq], a1 = s_xj[wib][8 * el + jq + 4];
      unsigned keep = 0;
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        if (!((built >> c) & 1u)) continue;
        const float4 xi = s_xi[wib][8 * c + i8];
#pragma unroll
        for (int jj = 0; jj < 2; ++jj) {
          const float4 xj = jj ? a1 : a0;
          const float dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
          const float r2 = dx * dx + dy * dy + dz * dz;
          const bool in = xi.w != 0.f && xj.w != 0.f && r2 < rp2;
          if (__any_sync(0xffffffffu, in)) keep |= 1u << (c + 8 * jj);
        }
      }
      if (lane == 0) s_keep[wib][el] = keep;
    }
    __syncwarp();
    if (lane < ne) {
      en.w = s_keep[wib][lane];
      ent[wk.y + lane] = en;
    }
    __syncwarp();
  }
}


}  // namespace capsb
