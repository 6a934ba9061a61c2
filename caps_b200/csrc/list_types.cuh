// Types and constants of the device pair list (layout: nblist.cuh), shared by the host engine and the list kernels.
#pragma once
#include "common.cuh"

namespace capsb {

constexpr int kScAtoms = 64;
constexpr int kClAtoms = 8;
constexpr int kSortMax = 4096;         // largest column the in-block sort takes
constexpr int kExclRecMax = 2048;      // exclusion records per super-cluster (64 atoms x 32 partners)
constexpr int kExclHash = 256;         // distinct (cluster, image) keys of one super-cluster's exclusions
constexpr int kBatch = 32;             // entries per work item

struct ListGeom {
  int nu, nv, ncol;
  int ru, rv, rq;
  double w[3];        // perpendicular widths of the cell
  double rlist, rlist2;
  double dw;          // rlist / w[2]
  int batch;          // entries per work item (the pair kernels' j-tile depth), at most kBatch; chosen by timing
};

struct ListBufs {
  // per atom
  int* col;
  double* frac;       // 3 per atom: wrapped fractional coordinates
  int* ioff;          // 3 per atom: lattice offset from x to the wrapped position
  int* order;         // atoms by column, sorted along c
  int* iperm;         // atom -> slot
  // per column
  int* col_count;
  int* col_fill;
  int* col_start;     // ncol + 1
  int* col_sc;        // ncol + 1: first super-cluster of each column
  // per super-cluster
  int* sc_col;
  double* sc_z;       // 2 per sc: fractional c range
  double* sc_org;     // 3 per sc: origin (centre of its bounding box)
  // per cluster
  double* cl_box;     // 6 per cluster: lo xyz, hi xyz (wrapped Cartesian)
  unsigned char* cl_real;   // 8-bit mask of real atoms
  // per slot
  int* perm;
  // list
  // x cj, y imask | image << 8, z mask index + 1, w the pruned masks the pair kernels read: bit c when j atoms 0-3
  // (the cluster's lower-x half) come within the prune radius of i cluster c, bit 8 + c for j atoms 4-7
  uint4* ent;
  float4* ent_shift;  // org(sc_j) + S - org(sc_i), for the FP32 kernel
  unsigned long long* masks;   // 8 rows (i clusters) per (super-cluster, j cluster, image) with exclusions
  int4* work;         // x sc, y first entry, z count
  // capacities
  int nsc_cap, ent_cap, mask_cap, work_cap;
  // device counters: [0] entries, [1] work items, [2] masks, [3] error bits, [4] rebuild flag, [5] nsc, [6] max column
  int* counters;
};

// Device counters: list sizes, the error word, the rebuild and prune flags, and running counts of builds and prunes.
enum Counter { kCntEnt = 0, kCntWork, kCntMask, kCntErr, kCntRebuild, kCntNsc, kCntMaxCol, kCntPrune, kCntBuilds, kCntPrunes, kCntPairNext,
               kCntFeneClaim, kCntNanClaim, kCntBinDone, kCntNum = 14 };   // *Claim: 1 once the first failure of that kind left its details

__device__ __forceinline__ void raise_error(int* counters, unsigned bit) { atomicOr(reinterpret_cast<unsigned*>(counters + kCntErr), bit); }

// Image (qa, qb, qc) packed into 21 bits, 7 per component offset by 64.
__host__ __device__ __forceinline__ unsigned pack_image(int qa, int qb, int qc) {
  return unsigned(qa + 64) | (unsigned(qb + 64) << 7) | (unsigned(qc + 64) << 14);
}
__host__ __device__ __forceinline__ void unpack_image(unsigned p, int& qa, int& qb, int& qc) {
  qa = int(p & 127u) - 64;
  qb = int((p >> 7) & 127u) - 64;
  qc = int((p >> 14) & 127u) - 64;
}

// Gate for the build kernels in a captured step: they all return at once unless the rebuild flag is set.
__device__ __forceinline__ bool build_off(const int* counters) { return *(volatile const int*)(counters + kCntRebuild) == 0; }

// The displacement check (core/src/field.cpp:800-838, the constant-cell branch): has an atom moved more than half the
// skin since the last build (x against xb, lim_b2), or half the prune margin since the last prune (x against xp,
// lim_p2)? Sets the rebuild and prune flags. It runs in the kernel that writes a step's final positions (the drift, or
// SHAKE and the atoms in no constraint cluster), or as a kernel of its own; xb null: no check.
struct ListCheck {
  const double* xb;
  const double* xp;
  double lim_b2, lim_p2;
  int* counters;
  int nfree;              // SHAKE's launch: the atoms in no cluster, after the clusters
  const int* free_atoms;
};
__device__ __forceinline__ void list_check_atom(const ListCheck& L, int g, const double* x, bool& mb, bool& mp) {
  const double x_ = x[3 * g], y_ = x[3 * g + 1], z_ = x[3 * g + 2];
  const double bx = x_ - L.xb[3 * g], by = y_ - L.xb[3 * g + 1], bz = z_ - L.xb[3 * g + 2];
  const double px = x_ - L.xp[3 * g], py = y_ - L.xp[3 * g + 1], pz = z_ - L.xp[3 * g + 2];
  mb |= !(bx * bx + by * by + bz * bz <= L.lim_b2);   // NaN counts as moved
  mp |= !(px * px + py * py + pz * pz <= L.lim_p2);
}
// Raises the flags a warp's atoms call for (every lane of the warp calls it).
__device__ __forceinline__ void list_check_flags(const ListCheck& L, bool mb, bool mp) {
  const bool lane0 = (threadIdx.x & 31) == 0;
  if (__any_sync(0xffffffffu, mb) && lane0) atomicOr(L.counters + kCntRebuild, 1);
  if (__any_sync(0xffffffffu, mp) && lane0) atomicOr(L.counters + kCntPrune, 1);
}

}  // namespace capsb
