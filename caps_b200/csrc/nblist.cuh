// The cluster pair list on the device (the reference builds it on the CPU: core/src/nbnxm.cpp:22-326, and its FP64
// atom-pair list, core/src/field.cpp:892-1101).
//
// Layout. Atoms are binned into columns over the (a, b) fractional plane, sorted along c inside each column and cut
// into super-clusters of 64 consecutive atoms; each super-cluster is split 2 x 2 x 2 (z halves, then y, then x) into
// eight clusters of 8 atoms. Slot s = 64 sc + 8 k + l holds atom perm[s] (-1 padding). A list entry pairs one
// super-cluster (the i side, 64 atoms, held by one warp) with one j cluster (8 atoms) under one periodic image, with an
// 8-bit mask of the super-cluster's clusters whose bounding boxes come within the list radius, and an optional index to
// eight 64-bit atom masks (exclusions at their nearest image, each pair of one cluster once). The half list keeps each
// cluster pair from one side, chosen by the parity of ci + cj as the reference does (nbnxm.cpp:201-206), and a cluster
// with its own images once per +- shift. Entries are produced in batches of up to 32 per super-cluster: each batch is
// one work item of the pair kernel.
#pragma once
#include "list_types.cuh"

namespace capsb {

// ---------------------------------------------------------------------------------------------------------------
// K-CHECK: the displacement check as a kernel of its own, for force evaluations outside a step that folds it in.
static __global__ void k_check_step(int n, const double* __restrict__ x, ListCheck L) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  bool mb = false, mp = false;
  if (i < n) list_check_atom(L, i, x, mb, mp);
  list_check_flags(L, mb, mp);
}

// K-SCAN (one block, NT threads): column starts, super-cluster starts (64 atoms each, the last one of a column
// partial), and the column of every super-cluster. Also resets the list counters for the search. The column counts are
// read through L2 (the other blocks of the binning made them with atomics).
template <int NT>
__device__ void scan_columns(const ListGeom& g, const ListBufs& b) {
  __shared__ int s_a[NT], s_s[NT];
  __shared__ int carry_a, carry_s, s_max;
  if (threadIdx.x == 0) carry_a = carry_s = s_max = 0;
  __syncthreads();
  for (int base = 0; base < g.ncol; base += NT) {
    const int c = base + threadIdx.x;
    const int cnt = c < g.ncol ? __ldcg(b.col_count + c) : 0;
    if (c < g.ncol) b.col_count[c] = 0;   // cleared for the next build's binning
    if (c < g.ncol) atomicMax(&s_max, cnt);
    s_a[threadIdx.x] = cnt;
    s_s[threadIdx.x] = (cnt + kScAtoms - 1) / kScAtoms;
    __syncthreads();
    for (int off = 1; off < NT; off <<= 1) {   // inclusive Hillis-Steele scan
      const int ta = threadIdx.x >= unsigned(off) ? s_a[threadIdx.x - off] : 0;
      const int ts = threadIdx.x >= unsigned(off) ? s_s[threadIdx.x - off] : 0;
      __syncthreads();
      s_a[threadIdx.x] += ta;
      s_s[threadIdx.x] += ts;
      __syncthreads();
    }
    if (c < g.ncol) {
      b.col_start[c + 1] = carry_a + s_a[threadIdx.x];
      b.col_sc[c + 1] = carry_s + s_s[threadIdx.x];
      b.col_fill[c] = 0;
    }
    __syncthreads();
    if (threadIdx.x == NT - 1) {
      carry_a += s_a[threadIdx.x];
      carry_s += s_s[threadIdx.x];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    b.col_start[0] = 0;
    b.col_sc[0] = 0;
    b.counters[kCntNsc] = carry_s;
    b.counters[kCntMaxCol] = s_max;
    b.counters[kCntEnt] = 0;
    b.counters[kCntWork] = 0;
    b.counters[kCntMask] = 0;
    if (carry_s > b.nsc_cap) raise_error(b.counters, kErrScOverflow);
    if (s_max > kSortMax) raise_error(b.counters, kErrColumnTooBig);
  }
  __syncthreads();
  const int nsc = min(carry_s, b.nsc_cap);
  for (int c = threadIdx.x; c < g.ncol; c += NT)
    for (int s = b.col_sc[c]; s < b.col_sc[c + 1] && s < nsc; ++s) b.sc_col[s] = c;
}

// K-BIN: wrapped fractional coordinates, lattice offsets and the column of every atom; column counts. The last block
// to finish (a ticket taken after a fence) runs the column scan, so the build has no launch of its own for it.
constexpr int kBinThreads = 256;
static __global__ void __launch_bounds__(kBinThreads) k_bin(int n, const double* __restrict__ x, DevCell cell, ListGeom g, ListBufs b) {
  if (build_off(b.counters)) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    const double xi[3] = {x[3 * i], x[3 * i + 1], x[3 * i + 2]};
    double f[3];
    frac_of(cell, xi, f);
    for (int k = 0; k < 3; ++k) {
      const double fl = floor(f[k]);
      double w = f[k] - fl;
      w = fmin(fmax(w, 0.0), 1.0 - 1e-12);
      b.frac[3 * i + k] = w;
      b.ioff[3 * i + k] = -int(fl);
    }
    const int cu = min(g.nu - 1, int(b.frac[3 * i] * g.nu)), cv = min(g.nv - 1, int(b.frac[3 * i + 1] * g.nv));
    const int c = cu * g.nv + cv;
    b.col[i] = c;
    // one atomic per distinct column in the warp (a column holds hundreds of atoms: the adds would contend)
    const unsigned act = __activemask();
    const unsigned same = __match_any_sync(act, c);
    if ((threadIdx.x & 31) == __ffs(same) - 1) atomicAdd(b.col_count + c, __popc(same));
  }
  __shared__ bool s_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = atomicAdd(b.counters + kCntBinDone, 1) == int(gridDim.x) - 1;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  scan_columns<kBinThreads>(g, b);
  if (threadIdx.x == 0) b.counters[kCntBinDone] = 0;
}

// K-SCATTER: atoms into their column's range (unordered; the sort that follows fixes the order).
static __global__ void k_scatter(int n, ListBufs b) {
  if (build_off(b.counters)) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int c = b.col[i];
  // warp-aggregated: the lowest lane of each column group reserves the group's places
  const unsigned act = __activemask();
  const unsigned same = __match_any_sync(act, c);
  const int lane = threadIdx.x & 31, leader = __ffs(same) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(b.col_fill + c, __popc(same));
  base = __shfl_sync(same, base, leader);
  b.order[b.col_start[c] + base + __popc(same & ((1u << lane) - 1))] = i;
}

// K-SUPER (a warp per super-cluster, inside the sort of its column): the 2 x 2 x 2 split into clusters, perm / iperm,
// cluster boxes and real-atom masks, the super-cluster's origin and its c range. Lane l holds atoms l (lower c half) and
// l + 32 (upper c half): the ranks along y and x come from shuffles, the boxes from butterfly reductions over the 8 lanes
// of a cluster. s_w and s_a: the warp's world positions and atoms by local slot (-1 padding).
__device__ void form_supercluster(const DevCell& cell, const ListBufs& b, int sc, int c, int lane, double (*s_w)[3], int* s_a) {
  const unsigned full = 0xffffffffu;
  {
    const int k = sc - b.col_sc[c];
    const int s0 = b.col_start[c] + kScAtoms * k;
    const int m = min(kScAtoms, b.col_start[c + 1] - s0);
    if (m <= 0) {   // not made by the scan (every super-cluster holds at least one atom); kept empty
      b.perm[64 * sc + lane] = b.perm[64 * sc + lane + 32] = -1;
      return;
    }
    int id[2];
    double fx[2], fy[2], w[2][3];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int t = lane + 32 * h;
      id[h] = -1;
      fx[h] = fy[h] = 0;
      w[h][0] = w[h][1] = w[h][2] = 0;
      if (t < m) {
        const int a = b.order[s0 + t];
        id[h] = a;
        const double f0 = b.frac[3 * a], f1 = b.frac[3 * a + 1], f2 = b.frac[3 * a + 2];
        fx[h] = f0, fy[h] = f1;
        for (int r = 0; r < 3; ++r) w[h][r] = cell.o[r] + cell.h[r][0] * f0 + cell.h[r][1] * f1 + cell.h[r][2] * f2;
      }
      s_a[t] = -1;
    }
    // rank along y within the c half, then along x within the y half of the c half (ties by atom index)
    int ry[2] = {0, 0}, rx[2] = {0, 0};
    for (int u = 0; u < 32; ++u) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const double yu = __shfl_sync(full, fy[h], u);
        const int iu = __shfl_sync(full, id[h], u);
        ry[h] += (u + 32 * h < m) && (yu < fy[h] || (yu == fy[h] && iu < id[h]));
      }
    }
    for (int u = 0; u < 32; ++u) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const double xu = __shfl_sync(full, fx[h], u);
        const int iu = __shfl_sync(full, id[h], u);
        const int qu = __shfl_sync(full, ry[h] >> 4, u);
        rx[h] += (u + 32 * h < m) && qu == (ry[h] >> 4) && (xu < fx[h] || (xu == fx[h] && iu < id[h]));
      }
    }
    __syncwarp();
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      if (lane + 32 * h >= m) continue;
      const int slot = 8 * (4 * h + 2 * (ry[h] >> 4) + (rx[h] >> 3)) + (rx[h] & 7);
      s_a[slot] = id[h];
      for (int r = 0; r < 3; ++r) s_w[slot][r] = w[h][r];
      b.iperm[id[h]] = 64 * sc + slot;
    }
    __syncwarp();
    // cluster boxes and real masks: slot lane + 32 h belongs to cluster (lane >> 3) + 4 h
    double slo[3] = {1e300, 1e300, 1e300}, shi[3] = {-1e300, -1e300, -1e300};
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int t = lane + 32 * h;
      const int a = s_a[t];
      b.perm[64 * sc + t] = a;
      double lo[3], hi[3];
      for (int r = 0; r < 3; ++r) {
        lo[r] = a >= 0 ? s_w[t][r] : 1e300;
        hi[r] = a >= 0 ? s_w[t][r] : -1e300;
      }
#pragma unroll
      for (int o = 1; o < 8; o <<= 1)
        for (int r = 0; r < 3; ++r) {
          lo[r] = fmin(lo[r], __shfl_xor_sync(full, lo[r], o));
          hi[r] = fmax(hi[r], __shfl_xor_sync(full, hi[r], o));
        }
      const unsigned real = __ballot_sync(full, a >= 0);
      if ((lane & 7) == 0) {
        const int cg = 8 * sc + (lane >> 3) + 4 * h;
        for (int r = 0; r < 3; ++r) b.cl_box[6 * cg + r] = lo[r], b.cl_box[6 * cg + 3 + r] = hi[r];
        b.cl_real[cg] = (unsigned char)((real >> (lane & 24)) & 255u);
      }
      for (int r = 0; r < 3; ++r) slo[r] = fmin(slo[r], lo[r]), shi[r] = fmax(shi[r], hi[r]);
    }
#pragma unroll
    for (int o = 8; o < 32; o <<= 1)
      for (int r = 0; r < 3; ++r) {
        slo[r] = fmin(slo[r], __shfl_xor_sync(full, slo[r], o));
        shi[r] = fmax(shi[r], __shfl_xor_sync(full, shi[r], o));
      }
    const int last = m - 1;
    const int id_first = __shfl_sync(full, id[0], 0);
    const int id_last = __shfl_sync(full, (last >> 5) ? id[1] : id[0], last & 31);
    if (lane == 0) {
      for (int r = 0; r < 3; ++r) b.sc_org[3 * sc + r] = 0.5 * (slo[r] + shi[r]);
      b.sc_z[2 * sc] = b.frac[3 * id_first + 2];
      b.sc_z[2 * sc + 1] = b.frac[3 * id_last + 2];
    }
    __syncwarp();
  }
}

// K-SORT (block per column): atoms by fractional c, ties by index, then the column's super-clusters (K-SUPER). A
// bitonic sorting network in shared memory over the column padded to a power of two (pad keys sort last):
// log2(n)(log2(n)+1)/2 compare-exchange rounds, one barrier each.
constexpr int kSortThreads = 1024;
constexpr int kScWarps = 16;   // warps of the sort block that form the column's super-clusters
static_assert(sizeof(double) * 3 * 64 * kScWarps + sizeof(int) * 64 * kScWarps <= size_t(kSortMax) * (sizeof(double) + sizeof(int)),
              "the super-cluster stage fits the sort's shared memory");
static __global__ void __launch_bounds__(kSortThreads) k_sort_columns(DevCell cell, ListGeom g, ListBufs b) {
  if (build_off(b.counters)) return;
  extern __shared__ unsigned char smem_raw[];
  const int nsc = min(b.counters[kCntNsc], b.nsc_cap);
  double* key = reinterpret_cast<double*>(smem_raw);
  int* id = reinterpret_cast<int*>(key + kSortMax);
  for (int c = blockIdx.x; c < g.ncol; c += gridDim.x) {
    const int s0 = b.col_start[c], n = min(b.col_start[c + 1] - s0, kSortMax);
    int np = 1;
    while (np < n) np <<= 1;
    for (int k = threadIdx.x; k < np; k += blockDim.x) {
      if (k < n) {
        const int a = b.order[s0 + k];
        id[k] = a;
        key[k] = b.frac[3 * a + 2];
      } else {
        id[k] = 0x7fffffff;
        key[k] = 2.0;   // fractional coordinates are below 1
      }
    }
    __syncthreads();
    for (int kk = 2; kk <= np; kk <<= 1)
      for (int j = kk >> 1; j > 0; j >>= 1) {
        for (int t = threadIdx.x; t < (np >> 1); t += blockDim.x) {
          const int lo = 2 * j * (t / j) + (t & (j - 1)), hi = lo + j;
          const double ka = key[lo], kb = key[hi];
          const int ia = id[lo], ib = id[hi];
          const bool gt = ka > kb || (ka == kb && ia > ib);
          if (gt == ((lo & kk) == 0)) {
            key[lo] = kb, key[hi] = ka;
            id[lo] = ib, id[hi] = ia;
          }
        }
        __syncthreads();
      }
    for (int k = threadIdx.x; k < n; k += blockDim.x) b.order[s0 + k] = id[k];
    __syncthreads();
    // the column's super-clusters, a warp each, in the shared memory the sort is done with
    const int w = threadIdx.x >> 5;
    if (w < kScWarps) {
      double(*s_w)[3] = reinterpret_cast<double(*)[3]>(smem_raw) + 64 * w;
      int* s_a = reinterpret_cast<int*>(smem_raw + sizeof(double) * 3 * 64 * kScWarps) + 64 * w;
      const int sc1 = min(b.col_sc[c + 1], nsc);
      for (int sc = b.col_sc[c] + w; sc < sc1; sc += kScWarps) form_supercluster(cell, b, sc, c, threadIdx.x & 31, s_w, s_a);
    }
    __syncthreads();
  }
}


// ---------------------------------------------------------------------------------------------------------------
constexpr int kSearchWarps = 8;       // warps per super-cluster in the search

// One warp's batch of entries in the making.
struct SearchBatch {
  uint4 ent[2 * kBatch];
  float4 sh[2 * kBatch];
  int nent;
};

struct SearchShared {
  uint2 rec[kExclRecMax];                 // x: j cluster, y: i local (6 bits) | j in cluster (3) << 6 | image << 9
  unsigned long long key[kExclHash];      // distinct (j cluster, image) of the records; ~0 empty
  unsigned short krank[kExclHash];        // rank of each occupied key slot: its masks are number mbase + rank
  int mbase;
  double ibox[8][6];
  double org_i[3];
  int nrec;
  SearchBatch batch[kSearchWarps];
};

__device__ __forceinline__ unsigned long long excl_key(unsigned cj, unsigned img) { return (unsigned long long)cj | ((unsigned long long)img << 32); }

// The slot of a key in the open-addressing table, or -1.
static __device__ int key_slot(const SearchShared& S, unsigned long long key) {
  unsigned h = (unsigned)(key * 0x9E3779B97F4A7C15ull >> 56) & (kExclHash - 1);
  for (int p = 0; p < kExclHash; ++p) {
    const unsigned long long v = S.key[h];
    if (v == key) return int(h);
    if (v == ~0ull) return -1;
    h = (h + 1) & (kExclHash - 1);
  }
  return -1;
}

static __device__ int key_insert(SearchShared& S, unsigned long long key, int* counters) {
  unsigned h = (unsigned)(key * 0x9E3779B97F4A7C15ull >> 56) & (kExclHash - 1);
  for (int p = 0; p < kExclHash; ++p) {
    const unsigned long long old = atomicCAS(&S.key[h], ~0ull, key);
    if (old == ~0ull || old == key) return int(h);
    h = (h + 1) & (kExclHash - 1);
  }
  raise_error(counters, kErrExclOverflow);
  return -1;
}
// Writes the batch [0, cnt) of B as one work item. One atomic reserves the entries and the work item: the entry and work
// counters are the two halves of one 64-bit word (entries low, work items high), shared by every warp of the build.
static __device__ void flush_batch(SearchBatch& B, int sc, int cnt, int lane, const ListBufs& b) {
  if (cnt <= 0) return;
  static_assert(kCntEnt == 0 && kCntWork == 1, "entry and work counters form one 64-bit word");
  int base = 0, wi = 0;
  if (lane == 0) {
    const unsigned long long old = atomicAdd(reinterpret_cast<unsigned long long*>(b.counters + kCntEnt), (1ull << 32) | unsigned(cnt));
    base = int(unsigned(old & 0xffffffffull));
    wi = int(unsigned(old >> 32));
  }
  base = __shfl_sync(0xffffffffu, base, 0);
  wi = __shfl_sync(0xffffffffu, wi, 0);
  if (base + cnt > b.ent_cap || wi >= b.work_cap) {
    if (lane == 0) raise_error(b.counters, kErrListOverflow);
    return;
  }
  for (int e = lane; e < cnt; e += 32) {
    uint4 en = B.ent[e];
    en.w = (en.y & 255u) * 0x101u;   // unpruned until the first prune: both halves of every listed i cluster
    b.ent[base + e] = en;
    b.ent_shift[base + e] = B.sh[e];
  }
  if (lane == 0) b.work[wi] = make_int4(sc, base, cnt, 0);
}

// K-SEARCH: one block of kSearchWarps warps per super-cluster. The block records the super-cluster's excluded pairs and
// builds the atom masks of every (j cluster, image) they touch; then each warp takes a contiguous share of the
// neighbouring columns (with their images) and batches its own entries. Exclusions (ForceField::excluded) hold at their
// nearest image only (core/src/nbnxm.cpp:229-252): each of the super-cluster's excluded atom pairs is recorded with the
// image that is nearest at the build, and the entry for that j cluster under that image carries masks with those pairs
// cleared. The super-cluster's own clusters under the zero image always carry masks (each pair of a cluster with
// itself once).
static __global__ void __launch_bounds__(32 * kSearchWarps, 4) k_search(DevCell cell, ListGeom g, const uint32_t* __restrict__ excl_off,
                                                                     const uint32_t* __restrict__ excl_list, ListBufs b) {
  if (build_off(b.counters)) return;
  extern __shared__ unsigned char smem_raw[];
  SearchShared& S = *reinterpret_cast<SearchShared*>(smem_raw);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  SearchBatch& B = S.batch[warp];
  const int nsc = min(b.counters[kCntNsc], b.nsc_cap);
  for (int sc = blockIdx.x; sc < nsc; sc += gridDim.x) {
    // --- the super-cluster's boxes and exclusion records (the whole block)
    for (int t = threadIdx.x; t < kExclHash; t += blockDim.x) S.key[t] = ~0ull;
    if (threadIdx.x < 8)
      for (int r = 0; r < 6; ++r) S.ibox[threadIdx.x][r] = b.cl_box[6 * (8 * sc + threadIdx.x) + r];
    if (threadIdx.x < 3) S.org_i[threadIdx.x] = b.sc_org[3 * sc + threadIdx.x];
    if (threadIdx.x == 0) S.nrec = 0;
    if (lane == 0) B.nent = 0;
    __syncthreads();
    if (threadIdx.x < 8) key_insert(S, excl_key(unsigned(8 * sc + threadIdx.x), pack_image(0, 0, 0)), b.counters);
    // kSearchWarps / 2 threads per atom, each taking every (kSearchWarps / 2)-th of the atom's excluded partners
    for (int u = threadIdx.x; u < 64 * (kSearchWarps / 2); u += blockDim.x) {
      const int t = u & 63;
      const int a = b.perm[64 * sc + t];
      if (a < 0) continue;
      const double* fa = b.frac + 3 * a;
      for (uint32_t p = excl_off[a] + uint32_t(u >> 6); p < excl_off[a + 1]; p += kSearchWarps / 2) {
        const int bb = int(excl_list[p]);
        const int sb = b.iperm[bb];
        const double* fb = b.frac + 3 * bb;
        // nearest image of bb seen from a: bb + q, q = -round(fb - fa)
        const int qa = -int(rint(fb[0] - fa[0])), qb = -int(rint(fb[1] - fa[1])), qc = -int(rint(fb[2] - fa[2]));
        if (qa < -63 || qa > 63 || qb < -63 || qb > 63 || qc < -63 || qc > 63) { raise_error(b.counters, kErrImageRange); continue; }
        const unsigned img = pack_image(qa, qb, qc);
        const int r = atomicAdd(&S.nrec, 1);
        if (r >= kExclRecMax) { raise_error(b.counters, kErrExclOverflow); continue; }
        S.rec[r] = make_uint2(unsigned(sb >> 3), unsigned(t) | (unsigned(sb & 7) << 6) | (img << 9));
        key_insert(S, excl_key(unsigned(sb >> 3), img), b.counters);
      }
    }
    __syncthreads();
    if (threadIdx.x == 0 && S.nrec > kExclRecMax) S.nrec = kExclRecMax;
    // masks: one set of 8 rows (i cluster r against the key's j cluster) per occupied key slot, numbered by the slot's
    // rank from a base reserved with one atomic; rows start as all pairs (each pair once for a cluster with itself under
    // the zero image), then every record clears its pair
    if (warp == 0) {
      constexpr int per = kExclHash / 32;
      unsigned occ = 0;
#pragma unroll
      for (int q = 0; q < per; ++q) occ |= unsigned(S.key[lane * per + q] != ~0ull) << q;
      const unsigned tot = __popc(occ);
      unsigned run = tot;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(0xffffffffu, run, o);
        if (lane >= o) run += y;
      }
      unsigned start = run - tot;
#pragma unroll
      for (int q = 0; q < per; ++q) {
        S.krank[lane * per + q] = (unsigned short)start;
        start += (occ >> q) & 1u;
      }
      const unsigned nkeys = __shfl_sync(0xffffffffu, run, 31);
      if (lane == 0) {
        const int m0 = atomicAdd(b.counters + kCntMask, int(nkeys));
        if (m0 + int(nkeys) > b.mask_cap) raise_error(b.counters, kErrMaskOverflow);
        S.mbase = m0;
      }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < 8 * kExclHash; t += blockDim.x) {
      const int h = t >> 3, r = t & 7;
      const unsigned long long key = S.key[h];
      if (key == ~0ull) continue;
      const int mi = S.mbase + S.krank[h];
      if (mi >= b.mask_cap) continue;
      unsigned long long mm = ~0ull;
      if (key == excl_key(unsigned(8 * sc + r), pack_image(0, 0, 0))) {
        mm = 0;
        for (int i = 0; i < 8; ++i)
          for (int j = i + 1; j < 8; ++j) mm |= 1ull << (8 * i + j);
      }
      b.masks[8 * size_t(mi) + r] = mm;
    }
    __syncthreads();   // the rows are written before any record clears a bit of them
    for (int r = threadIdx.x; r < S.nrec; r += blockDim.x) {
      const uint2 rc = S.rec[r];
      const int h = key_slot(S, excl_key(rc.x, rc.y >> 9));
      if (h < 0) continue;
      const int mi = S.mbase + S.krank[h];
      if (mi >= b.mask_cap) continue;
      const unsigned il = rc.y & 63u, jl = (rc.y >> 6) & 7u;
      atomicAnd(b.masks + 8 * size_t(mi) + (il >> 3), ~(1ull << (8 * (il & 7) + jl)));
    }
    // --- candidates: neighbouring columns (with their images), super-clusters in c range, their 8 clusters. Each warp
    // takes a contiguous block of the columns: its entries (and the pair kernel's work items made of them) stay spatially
    // together, which measured faster in the pair kernel than an interleaved split. The split is fixed, so every build
    // groups the same entries into the same work items (the pair kernel's float partial sums, and so the forces, do not
    // depend on timing).
    const int col = b.sc_col[sc];
    const int cu = col / g.nv, cv = col % g.nv;
    const double zlo = b.sc_z[2 * sc], zhi = b.sc_z[2 * sc + 1];
    const int ci0 = 8 * sc;
    const int nvw = 2 * g.rv + 1, ncols = (2 * g.ru + 1) * nvw;
    const int kper = (ncols + kSearchWarps - 1) / kSearchWarps;
    for (int k = warp * kper; k < min(ncols, (warp + 1) * kper); ++k) {
      const int du = k / nvw - g.ru, dv = k % nvw - g.rv;
      int U = cu + du;
      const int qa = (int)floor(double(U) / g.nu);
      U -= qa * g.nu;
      int V = cv + dv;
      const int qb = (int)floor(double(V) / g.nv);
      V -= qb * g.nv;
      const int cc = U * g.nv + V;
      const int qc0 = max(-g.rq, (int)floor(zlo - g.dw)), qc1 = min(g.rq, (int)floor(zhi + g.dw));
      for (int qc = qc0; qc <= qc1; ++qc) {
        const double S0 = cell.h[0][0] * qa + cell.h[0][1] * qb + cell.h[0][2] * qc;
        const double S1 = cell.h[1][0] * qa + cell.h[1][1] * qb + cell.h[1][2] * qc;
        const double S2 = cell.h[2][0] * qa + cell.h[2][1] * qb + cell.h[2][2] * qc;
        const bool zero = qa == 0 && qb == 0 && qc == 0;
        const bool positive = qa > 0 || (qa == 0 && (qb > 0 || (qb == 0 && qc > 0)));
        const unsigned img = pack_image(qa, qb, qc);
        const double lo = zlo - g.dw - qc, hi = zhi + g.dw - qc;
        // super-clusters of column cc whose c range meets [lo, hi]: their ranges rise along the column
        int sj = b.col_sc[cc];
        const int sje = min(b.col_sc[cc + 1], nsc);
        {
          int lo_i = sj, hi_i = sje;   // first with z_hi >= lo
          while (lo_i < hi_i) {
            const int mid = (lo_i + hi_i) >> 1;
            if (b.sc_z[2 * mid + 1] < lo) lo_i = mid + 1;
            else hi_i = mid;
          }
          sj = lo_i;
        }
        for (; sj < sje && b.sc_z[2 * sj] <= hi; sj += 4) {
          // four candidate super-clusters per pass: lane = 8 * which + j cluster
          const int sjl = sj + (lane >> 3);
          bool have = false;
          unsigned imask = 0;
          int cj = -1;
          if (sjl < sje && b.sc_z[2 * sjl] <= hi) {
            cj = 8 * sjl + (lane & 7);
            const double* bj = b.cl_box + 6 * cj;
            const double jlo[3] = {bj[0] + S0, bj[1] + S1, bj[2] + S2}, jhi[3] = {bj[3] + S0, bj[4] + S1, bj[5] + S2};
            for (int c = 0; c < 8; ++c) {
              const int ci = ci0 + c;
              // half list: one side of each cluster pair by parity; a cluster with itself under zero or + images
              bool keep;
              if (cj != ci) keep = (cj > ci) == (((ci + cj) & 1) == 0);
              else keep = zero || positive;
              if (!keep) continue;
              double d2 = 0;
              for (int r = 0; r < 3; ++r) {
                const double g1 = jlo[r] - S.ibox[c][3 + r], g2 = S.ibox[c][r] - jhi[r];
                const double gg = g1 > 0 ? g1 : (g2 > 0 ? g2 : 0.0);
                d2 += gg * gg;
              }
              if (d2 < g.rlist2) imask |= 1u << c;
            }
            have = imask != 0;
          }
          const unsigned ball = __ballot_sync(0xffffffffu, have);
          if (have) {
            const int pos = B.nent + __popc(ball & ((1u << lane) - 1));   // < batch + 32 <= 2 kBatch (flushed below)
            const int sjc = cj >> 3;
            const int h = key_slot(S, excl_key(unsigned(cj), img));
            const int mi = h >= 0 ? S.mbase + S.krank[h] : -1;
            B.ent[pos] = make_uint4(unsigned(cj), imask | (img << 8), mi >= 0 && mi < b.mask_cap ? unsigned(mi + 1) : 0u, 0u);
            B.sh[pos] = make_float4(float(b.sc_org[3 * sjc] + S0 - S.org_i[0]), float(b.sc_org[3 * sjc + 1] + S1 - S.org_i[1]),
                                    float(b.sc_org[3 * sjc + 2] + S2 - S.org_i[2]), 0.f);
          }
          __syncwarp();
          if (lane == 0) B.nent += __popc(ball);
          __syncwarp();
          while (B.nent >= g.batch) {   // a pass adds up to 32 entries: with a depth below 32 more than one batch fills
            flush_batch(B, sc, g.batch, lane, b);
            __syncwarp();
            // the rest (< 2 kBatch - batch entries) moves down: read all, then write (the ranges can overlap)
            const int rest = B.nent - g.batch;
            uint4 te[2];
            float4 ts[2];
#pragma unroll
            for (int k = 0; k < 2; ++k) {
              const int e = lane + 32 * k;
              if (e < rest) te[k] = B.ent[g.batch + e], ts[k] = B.sh[g.batch + e];
            }
            __syncwarp();
#pragma unroll
            for (int k = 0; k < 2; ++k) {
              const int e = lane + 32 * k;
              if (e < rest) B.ent[e] = te[k], B.sh[e] = ts[k];
            }
            __syncwarp();
            if (lane == 0) B.nent = rest;
            __syncwarp();
          }
        }
      }
    }
    flush_batch(B, sc, B.nent, lane, b);
    __syncthreads();   // S is rewritten for the next super-cluster
  }
}

}  // namespace capsb
