// Shared device helpers for the B200 MD engine: cell algebra, fixed-point accumulation, warp reductions, error words.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace capsb {

constexpr double kPi = 3.14159265358979323846;
constexpr double kCoulomb = 332.06371;   // kcal*Å/(mol*e^2), as the reference (core/src/field.cpp:29)

// Fixed-point scales. Forces: 2^32 units per kcal/mol/Å: resolution 2.3e-10, range +-2.1e9. PME grid charges: 2^40 per e (resolution 9e-13 e). Integer sums are exact, so every reduction that goes
// through these is independent of the order the GPU runs it in: bit-reproducible forces and energies.
constexpr double kFixF = 4294967296.0;
constexpr double kInvFixF = 1.0 / 4294967296.0;
// Energies and virials: 2^24 per kcal/mol (resolution 6e-8, range +-5.5e11).
constexpr double kFixE = 16777216.0;
constexpr double kInvFixE = 1.0 / 16777216.0;
// A force component past this cannot be held in the fixed-point sums: the kernel raises kErrFixRange instead.
constexpr float kFixFMax = 2.0e9f;
constexpr double kFixQ = 1099511627776.0;
constexpr double kInvFixQ = 1.0 / 1099511627776.0;

// Error bits raised by kernels (never a trap): the host reads the word and throws the reference's message.
enum ErrorBits : unsigned {
  kErrListOverflow = 1u << 0,     // cluster-pair entries past capacity
  kErrExclOverflow = 1u << 1,     // exclusion records of a super-cluster past the per-warp table
  kErrColumnTooBig = 1u << 2,     // a grid column holds more atoms than the column sort takes
  kErrScOverflow = 1u << 3,       // more super-clusters than allocated
  kErrFene = 1u << 4,             // a FENE bond stretched past R0
  kErrShake = 1u << 5,            // SHAKE / RATTLE did not converge
  kErrShakeTurn = 1u << 6,        // a constrained bond turned past 90 degrees
  kErrNonFinite = 1u << 7,        // a coordinate became NaN / inf
  kErrMaskOverflow = 1u << 8,     // exclusion masks past capacity
  kErrImageRange = 1u << 9,       // an image shift outside +-63 cells
  kErrFixRange = 1u << 10,        // a force or energy outside the fixed-point range (overlapping atoms: push off first)
  kErrRattle = 1u << 11,          // RATTLE (the velocity constraints) did not converge
  kErrLincs = 1u << 12,           // LINCS's rotational corrections did not converge
  kErrConsOverlap = 1u << 13,     // two constrained atoms on each other (LINCS takes their direction)
};

// What the first failure of a kind leaves for the host's message (the engine's error-detail array, doubles): the
// stretched FENE bond and its length, and the step whose positions stopped being finite.
enum ErrInfo { kInfoFeneBond = 0, kInfoFeneR, kInfoNonFiniteStep, kInfoNum = 4 };

// The generic pair forms (field.cpp:1381-1455): returns -(dE/dr)/r, E in e. p = (a, b, c, the pair's cut-off^2), g the
// lj/gromacs switch coefficients (its constant is the caller's shift), r1 = lj_inner, T the tabulated pairs.
// 1 Buckingham A e^(-r/rho) - C/r^6 (a A, b rho, c C); 2 Morse D (e^(-2 alpha (r - r0)) - 2 e^(-alpha (r - r0))) (a D,
// b alpha, c r0); 3 Rydberg (A + C r) e^(-r/rho) (a A, b rho, c C); 11-14 SDK C eps ((s/r)^m - (s/r)^n) (a eps, b
// sigma); 20 lj/gromacs (a eps, b sigma); 31 / 32 cosine-squared, 32 with WCA (a eps, b sigma, c cut-off); 40 a table.
// CHARMM's force switch on a 12-6 pair (field.cpp:1455-1469; A = 4 eps s^12, B = 4 eps s^6): below r_in the plain 12-6
// plus a constant, between r_in and r_c E = A k12 (r^-6 - r_c^-6)^2 - B k6 (r^-3 - r_c^-3)^2; returns -(dE/dr)/r, adds
// E to e when ener.
__device__ __forceinline__ double charmm_fsw(double A, double B, double ri, double rc, double r2, double& e, bool ener) {
  const double ri3 = ri * ri * ri, rc2 = rc * rc, rc3 = rc2 * rc, ri6 = ri3 * ri3, rc6 = rc3 * rc3, r6i = 1 / (r2 * r2 * r2);
  if (r2 <= ri * ri) {
    if (ener) e += A * (r6i * r6i - 1 / (ri6 * rc6)) - B * (r6i - 1 / (ri3 * rc3));
    return (12 * A * r6i * r6i - 6 * B * r6i) / r2;
  }
  const double r3i = 1 / (r2 * sqrt(r2)), k12 = rc6 / (rc6 - ri6), k6 = rc3 / (rc3 - ri3);
  const double u = r6i - 1 / rc6, w = r3i - 1 / rc3;
  if (ener) e += A * k12 * u * u - B * k6 * w * w;
  return (12 * A * k12 * u * r6i - 6 * B * k6 * w * r3i) / r2;
}

struct PairTables {
  const int* off;        // [ntables + 1] first point of each table
  const double* r0dr;    // [2 ntables]
  const double* e;
  const double* f;
};
__device__ __forceinline__ double generic_pair(int form, const double4& p, const double4& g, double r1, const PairTables& T, double r2, double& e) {
  const double pa = p.x, pb = p.y, pc = p.z;
  e = 0;
  if (form == 1) {
    const double r = sqrt(r2), ex = pa * exp(-r / pb), c6 = pc / (r2 * r2 * r2);
    e = ex - c6;
    return (ex / pb - 6 * c6 / r) / r;
  }
  if (form == 3) {
    const double r = sqrt(r2), ex = exp(-r / pb), u = pa + pc * r;
    e = u * ex;
    return (u / pb - pc) * ex / r;
  }
  if (form == 2) {
    const double r = sqrt(r2), e1 = exp(-pb * (r - pc));
    e = pa * (e1 * e1 - 2 * e1);
    return 2 * pa * pb * (e1 * e1 - e1) / r;
  }
  if (form == 31 || form == 32) {
    const double r = sqrt(r2), ep = pa, sg = pb, rcp = pc;
    if (r >= rcp && !(form == 32 && r < sg)) return 0.0;
    double ev = 0, dEdr = 0;
    if (r < sg) {
      if (rcp > sg) ev = -ep;
      if (form == 32) {
        const double s6 = pow(sg / r, 6.0);
        ev += ep * (s6 * s6 - 2 * s6 + 1);
        dEdr += -12 * ep * (s6 * s6 - s6) / r;
      }
    } else {
      const double w = 3.14159265358979323846 * (r - sg) / (2 * (rcp - sg)), c = cos(w);
      ev = -ep * c * c;
      dEdr = ep * 2 * c * sin(w) * 3.14159265358979323846 / (2 * (rcp - sg));
    }
    e = ev;
    return -dEdr / r;
  }
  if (form == 40) {
    const int t = int(pa), k0 = T.off[t], m = T.off[t + 1] - k0;
    const double r = sqrt(r2), t0 = T.r0dr[2 * t], dr = T.r0dr[2 * t + 1];
    if (m < 2 || r >= t0 + dr * double(m - 1)) return 0.0;
    if (r < t0) {   // below the table: a straight wall at the first force
      e = T.e[k0] + T.f[k0] * (t0 - r);
      return T.f[k0] / r;
    }
    const double u = (r - t0) / dr;
    const int k = min(m - 2, int(u));
    const double w = u - double(k);
    e = T.e[k0 + k] * (1 - w) + T.e[k0 + k + 1] * w;
    return (T.f[k0 + k] * (1 - w) + T.f[k0 + k + 1] * w) / r;
  }
  if (form == 20) {
    const double s6 = pow(pb, 6.0), r2i = 1 / r2, r6i = r2i * r2i * r2i;
    double ev = r6i * (4 * pa * s6 * s6 * r6i - 4 * pa * s6), fr = r6i * (48 * pa * s6 * s6 * r6i - 24 * pa * s6);
    if (r2 > r1 * r1) {
      const double r = sqrt(r2), tl = r - r1;
      ev += tl * tl * tl * (g.z + g.w * tl);
      fr += r * tl * tl * (g.x + g.y * tl);
    }
    e = ev;
    return fr * r2i;
  }
  // SDK (11-14)
  const double pw1 = form == 11 ? 9.0 : 12.0, pw2 = form == 11 ? 6.0 : form == 12 ? 4.0 : form == 13 ? 6.0 : 5.0;
  const double pre = form == 11 ? 6.75 : form == 12 ? 2.59807621135332 : form == 13 ? 4.0 : 3.20377984125109;
  const double sr2 = pb * pb / r2, sm = pow(sr2, pw1 / 2), sn = pow(sr2, pw2 / 2), c = pre * pa;
  e = c * (sm - sn);
  return c * (pw1 * sm - pw2 * sn) / r2;
}

// Periodic cell: origin o, edge vectors a, b, c (columns of h) and h^-1 (rows: reciprocal vectors without 2 pi).
struct DevCell {
  double o[3];
  double h[3][3];    // h[r][c]: component r of edge vector c
  double hi[3][3];   // inverse
  double vol;
};

__host__ __device__ inline void frac_of(const DevCell& c, const double x[3], double f[3]) {
  const double d0 = x[0] - c.o[0], d1 = x[1] - c.o[1], d2 = x[2] - c.o[2];
  for (int r = 0; r < 3; ++r) f[r] = c.hi[r][0] * d0 + c.hi[r][1] * d1 + c.hi[r][2] * d2;
}

// Separation d brought to its nearest periodic image (fractional rounding; bonded partners sit well inside half a cell).
template <class R>
__device__ __forceinline__ void min_image(const DevCell& c, R& dx, R& dy, R& dz) {
  double f[3];
  for (int r = 0; r < 3; ++r) {
    f[r] = c.hi[r][0] * double(dx) + c.hi[r][1] * double(dy) + c.hi[r][2] * double(dz);
    f[r] -= rint(f[r]);
  }
  dx = R(c.h[0][0] * f[0] + c.h[0][1] * f[1] + c.h[0][2] * f[2]);
  dy = R(c.h[1][0] * f[0] + c.h[1][1] * f[1] + c.h[1][2] * f[2]);
  dz = R(c.h[2][0] * f[0] + c.h[2][1] * f[1] + c.h[2][2] * f[2]);
}

__device__ __forceinline__ long long to_fix(double v, double scale) { return __double2ll_rn(v * scale); }
__device__ __forceinline__ long long to_fixf(float v) { return __float2ll_rn(v * 4294967296.0f); }

__device__ __forceinline__ void atomic_add_fix(long long* p, long long v) {
  atomicAdd(reinterpret_cast<unsigned long long*>(p), static_cast<unsigned long long>(v));
}

// A float force component into fixed point, or the range error (bit 10 of the error word) when it cannot be held.
__device__ __forceinline__ void fix_add_f(long long* p, float v, int* err) {
  if (fabsf(v) < kFixFMax) atomic_add_fix(p, to_fixf(v));
  else atomicOr(reinterpret_cast<unsigned*>(err), 1u << 10);
}

// Force accumulation into either fixed-point (mixed precision) or double (FP64) SoA arrays.
template <class R> struct ForceSink;
template <> struct ForceSink<float> {
  long long* fx;
  long long* fy;
  long long* fz;
  int* err;
  __device__ __forceinline__ void one(long long* p, double v) const {
    if (fabs(v) < double(kFixFMax)) atomic_add_fix(p, to_fix(v, kFixF));
    else atomicOr(reinterpret_cast<unsigned*>(err), 1u << 10);
  }
  __device__ __forceinline__ void add(int i, double x, double y, double z) const {
    one(fx + i, x);
    one(fy + i, y);
    one(fz + i, z);
  }
  __device__ __forceinline__ void add1(int comp, int i, double v) const { one(comp == 0 ? fx : comp == 1 ? fy : fz, v); }
};
template <> struct ForceSink<double> {
  double* fx;
  double* fy;
  double* fz;
  __device__ __forceinline__ void add(int i, double x, double y, double z) const {
    atomicAdd(fx + i, x);
    atomicAdd(fy + i, y);
    atomicAdd(fz + i, z);
  }
  __device__ __forceinline__ void add1(int comp, int i, double v) const {
    double* p = comp == 0 ? fx : comp == 1 ? fy : fz;
    atomicAdd(p + i, v);
  }
};

// Energy / virial accumulators: index into a small array; fixed point for the mixed path (deterministic), double for
// the FP64 path.
enum EnergySlot { kEBond = 0, kEAngle, kEDihedral, kEImproper, kEVdw, kECoul, kEW0, kEW1, kEW2, kEW3, kEW4, kEW5, kEPmeRecip, kEPairs, kEListed,
                  kENumSlots = 16 };

struct EnergySink {
  long long* fix;    // [kENumSlots] mixed path
  double* dbl;       // [kENumSlots] FP64 path
  __device__ __forceinline__ void add(int slot, double v, bool fixed) const {
    if (fixed) atomic_add_fix(fix + slot, to_fix(v, kFixE));
    else atomicAdd(dbl + slot, v);
  }
};

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum (any blockDim that is a multiple of 32, up to 1024); result valid in thread 0.
template <class T>
__device__ T block_sum(T v, T* scratch /* >= 32 */) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) scratch[w] = v;
  __syncthreads();
  T s = 0;
  if (w == 0) {
    s = lane < int(blockDim.x >> 5) ? scratch[lane] : T(0);
    s = warp_sum(s);
  }
  return s;
}

// Philox4x32-10 (Salmon, Moraes, Dror & Shaw, SC'11): counter-based random numbers, so every atom's noise at every
// step is a pure function of (seed, step, atom) whatever the launch shape.
struct Philox {
  __device__ __forceinline__ static void round(uint32_t& c0, uint32_t& c1, uint32_t& c2, uint32_t& c3, uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t hi0 = __umulhi(M0, c0), lo0 = M0 * c0;
    const uint32_t hi1 = __umulhi(M1, c2), lo1 = M1 * c2;
    const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
  }
  __device__ static uint4 gen(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1) {
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
      round(c0, c1, c2, c3, k0, k1);
      k0 += W0;
      k1 += W1;
    }
    return make_uint4(c0, c1, c2, c3);
  }
};

// Four standard normals from one Philox block (Box-Muller on 24-bit uniforms in (0, 1]).
__device__ inline void normals4(uint64_t seed, uint64_t step, uint32_t idx, uint32_t stream, double out[4]) {
  const uint4 r = Philox::gen(idx, stream, uint32_t(step), uint32_t(step >> 32), uint32_t(seed), uint32_t(seed >> 32));
  const double s = 1.0 / 4294967296.0;
  const double u0 = (double(r.x) + 1.0) * s, u1 = (double(r.y) + 0.5) * s, u2 = (double(r.z) + 1.0) * s, u3 = (double(r.w) + 0.5) * s;
  const double ra = sqrt(-2.0 * log(u0)), rb = sqrt(-2.0 * log(u2));
  double sa, ca, sb, cb;
  sincospi(2.0 * u1, &sa, &ca);
  sincospi(2.0 * u3, &sb, &cb);
  out[0] = ra * ca;
  out[1] = ra * sa;
  out[2] = rb * cb;
  out[3] = rb * sb;
}

}  // namespace capsb
