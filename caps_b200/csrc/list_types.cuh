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
               kCntFeneClaim, kCntNanClaim, kCntNum = 13 };   // *Claim: 1 once the first failure of that kind left its details

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

}  // namespace capsb
