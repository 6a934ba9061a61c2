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
// K-CHECK: has any atom moved more than half the skin since the last build (x against x0, lim_b2; core/src/field.cpp:
// 800-838, the constant-cell branch), or half the prune margin since the last prune (x against xp, lim_p2)? Sets the
// rebuild and prune flags; the pair kernel lowers both once the step's list work is done.
static __global__ void k_check_step(int n, const double* __restrict__ x, const double* __restrict__ x0, double lim_b2, const double* __restrict__ xp,
                                    double lim_p2, int* counters) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  bool mb = false, mp = false;
  if (i < n) {
    const double x_ = x[3 * i], y_ = x[3 * i + 1], z_ = x[3 * i + 2];
    const double bx = x_ - x0[3 * i], by = y_ - x0[3 * i + 1], bz = z_ - x0[3 * i + 2];
    const double px = x_ - xp[3 * i], py = y_ - xp[3 * i + 1], pz = z_ - xp[3 * i + 2];
    mb = !(bx * bx + by * by + bz * bz <= lim_b2);   // NaN counts as moved
    mp = !(px * px + py * py + pz * pz <= lim_p2);
  }
  const bool lane0 = (threadIdx.x & 31) == 0;
  if (__any_sync(0xffffffffu, mb) && lane0) atomicOr(counters + kCntRebuild, 1);
  if (__any_sync(0xffffffffu, mp) && lane0) atomicOr(counters + kCntPrune, 1);
}


// K-BIN: wrapped fractional coordinates, lattice offsets and the column of every atom; column counts.
static __global__ void k_bin(int n, const double* __restrict__ x, DevCell cell, ListGeom g, ListBufs b) {
  if (build_off(b.counters)) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
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

// K-SCAN (one block): column starts, super-cluster starts (64 atoms each, the last one of a column partial), and the
// column of every super-cluster. Also resets the list counters for the search.
static __global__ void k_scan_columns(ListGeom g, ListBufs b) {
  if (build_off(b.counters)) return;
  __shared__ int s_a[1024], s_s[1024];
  __shared__ int carry_a, carry_s, s_max;
  if (threadIdx.x == 0) carry_a = carry_s = s_max = 0;
  __syncthreads();
  for (int base = 0; base < g.ncol; base += blockDim.x) {
    const int c = base + threadIdx.x;
    const int cnt = c < g.ncol ? b.col_count[c] : 0;
    if (c < g.ncol) b.col_count[c] = 0;   // cleared for the next build's binning
    if (c < g.ncol) atomicMax(&s_max, cnt);
    s_a[threadIdx.x] = cnt;
    s_s[threadIdx.x] = (cnt + kScAtoms - 1) / kScAtoms;
    __syncthreads();
    for (int off = 1; off < int(blockDim.x); off <<= 1) {   // inclusive Hillis-Steele scan
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
    if (threadIdx.x == blockDim.x - 1) {
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
  for (int c = threadIdx.x; c < g.ncol; c += blockDim.x)
    for (int s = b.col_sc[c]; s < b.col_sc[c + 1] && s < nsc; ++s) b.sc_col[s] = c;
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

// K-SORT (block per column): atoms by fractional c, ties by index (a rank sort in shared memory).
static __global__ void k_sort_columns(ListGeom g, ListBufs b) {
  if (build_off(b.counters)) return;
  extern __shared__ unsigned char smem_raw[];
  double* key = reinterpret_cast<double*>(smem_raw);
  int* id = reinterpret_cast<int*>(key + kSortMax);
  for (int c = blockIdx.x; c < g.ncol; c += gridDim.x) {
    const int s0 = b.col_start[c], n = min(b.col_start[c + 1] - s0, kSortMax);
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
      const int a = b.order[s0 + k];
      id[k] = a;
      key[k] = b.frac[3 * a + 2];
    }
    __syncthreads();
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
      const double kk = key[k];
      const int ik = id[k];
      int r0 = 0, r1 = 0, r2 = 0, r3 = 0;   // four independent counts: the loop is latency-bound otherwise
      int u = 0;
      for (; u + 4 <= n; u += 4) {
        r0 += (key[u] < kk) || (key[u] == kk && id[u] < ik);
        r1 += (key[u + 1] < kk) || (key[u + 1] == kk && id[u + 1] < ik);
        r2 += (key[u + 2] < kk) || (key[u + 2] == kk && id[u + 2] < ik);
        r3 += (key[u + 3] < kk) || (key[u + 3] == kk && id[u + 3] < ik);
      }
      for (; u < n; ++u) r0 += (key[u] < kk) || (key[u] == kk && id[u] < ik);
      b.order[s0 + r0 + r1 + r2 + r3] = ik;
    }
    __syncthreads();
  }
}

// K-SUPER (warp per super-cluster): the 2 x 2 x 2 split into clusters, perm / iperm, cluster boxes and real-atom
// masks, the super-cluster's origin and its c range.
static __global__ void k_superclusters(DevCell cell, ListBufs b) {
  if (build_off(b.counters)) return;
  __shared__ double s_y[4][64], s_x[4][64], s_w[4][64][3];
  __shared__ int s_id[4][64], s_slot[4][64], s_ry[4][64];
  const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nsc = min(b.counters[kCntNsc], b.nsc_cap);
  for (int sc = blockIdx.x * 4 + wib; sc < nsc; sc += gridDim.x * 4) {
    const int c = b.sc_col[sc];
    const int k = sc - b.col_sc[c];
    const int s0 = b.col_start[c] + kScAtoms * k;
    const int m = min(kScAtoms, b.col_start[c + 1] - s0);
    for (int t = lane; t < 64; t += 32) {
      b.perm[64 * sc + t] = -1;
      if (t < m) {
        const int a = b.order[s0 + t];
        s_id[wib][t] = a;
        const double f0 = b.frac[3 * a], f1 = b.frac[3 * a + 1], f2 = b.frac[3 * a + 2];
        s_x[wib][t] = f0;
        s_y[wib][t] = f1;
        for (int r = 0; r < 3; ++r) s_w[wib][t][r] = cell.o[r] + cell.h[r][0] * f0 + cell.h[r][1] * f1 + cell.h[r][2] * f2;
      }
    }
    __syncwarp();
    for (int t = lane; t < m; t += 32) {
      const int h = t >> 5;                // z half (positions are sorted along c)
      const int hb = h * 32, he = min(m, hb + 32);
      int ry = 0;
      for (int u = hb; u < he; ++u) ry += (s_y[wib][u] < s_y[wib][t]) || (s_y[wib][u] == s_y[wib][t] && s_id[wib][u] < s_id[wib][t]);
      s_ry[wib][t] = ry;   // the rank along y within the z half
    }
    __syncwarp();
    for (int t = lane; t < m; t += 32) {
      const int h = t >> 5, hb = h * 32, he = min(m, hb + 32);
      const int q = s_ry[wib][t] >> 4;   // y half within the z half
      int rx = 0;
      for (int u = hb; u < he; ++u) {
        if ((s_ry[wib][u] >> 4) != q) continue;
        rx += (s_x[wib][u] < s_x[wib][t]) || (s_x[wib][u] == s_x[wib][t] && s_id[wib][u] < s_id[wib][t]);
      }
      const int cl = 4 * h + 2 * q + (rx >> 3);
      s_slot[wib][t] = 64 * sc + 8 * cl + (rx & 7);
    }
    __syncwarp();
    for (int t = lane; t < m; t += 32) {
      const int slot = s_slot[wib][t], a = s_id[wib][t];
      b.perm[slot] = a;
      b.iperm[a] = slot;
    }
    __syncwarp();
    // cluster boxes: lane l < 8 takes cluster l
    if (lane < 8) {
      double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
      unsigned real = 0;
      for (int t = 0; t < m; ++t) {
        const int slot = s_slot[wib][t] - 64 * sc;
        if ((slot >> 3) != lane) continue;
        real |= 1u << (slot & 7);
        for (int r = 0; r < 3; ++r) lo[r] = fmin(lo[r], s_w[wib][t][r]), hi[r] = fmax(hi[r], s_w[wib][t][r]);
      }
      const int cg = 8 * sc + lane;
      for (int r = 0; r < 3; ++r) b.cl_box[6 * cg + r] = lo[r], b.cl_box[6 * cg + 3 + r] = hi[r];
      b.cl_real[cg] = (unsigned char)real;
    }
    if (lane == 0) {
      double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
      for (int t = 0; t < m; ++t)
        for (int r = 0; r < 3; ++r) lo[r] = fmin(lo[r], s_w[wib][t][r]), hi[r] = fmax(hi[r], s_w[wib][t][r]);
      for (int r = 0; r < 3; ++r) b.sc_org[3 * sc + r] = 0.5 * (lo[r] + hi[r]);
      b.sc_z[2 * sc] = b.frac[3 * s_id[wib][0] + 2];
      b.sc_z[2 * sc + 1] = b.frac[3 * s_id[wib][m - 1] + 2];
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------------------------------------------
constexpr int kSearchWarps = 4;       // warps per super-cluster in the search

// One warp's batch of entries in the making.
struct SearchBatch {
  uint4 ent[2 * kBatch];
  float4 sh[2 * kBatch];
  unsigned char needs_mask[2 * kBatch];
  unsigned long long m[kBatch][8];
  int nent;
};

struct SearchShared {
  uint2 rec[kExclRecMax];                 // x: j cluster, y: i local (6 bits) | j in cluster (3) << 6 | image << 9
  unsigned long long key[kExclHash];      // distinct (j cluster, image) of the records; ~0 empty
  double ibox[8][6];
  double org_i[3];
  int nrec;
  SearchBatch batch[kSearchWarps];
};

__device__ __forceinline__ unsigned long long excl_key(unsigned cj, unsigned img) { return (unsigned long long)cj | ((unsigned long long)img << 32); }

static __device__ bool key_find(const SearchShared& S, unsigned long long key) {
  unsigned h = (unsigned)(key * 0x9E3779B97F4A7C15ull >> 56) & (kExclHash - 1);
  for (int p = 0; p < kExclHash; ++p) {
    const unsigned long long v = S.key[h];
    if (v == key) return true;
    if (v == ~0ull) return false;
    h = (h + 1) & (kExclHash - 1);
  }
  return false;
}

static __device__ void key_insert(SearchShared& S, unsigned long long key, int* counters) {
  unsigned h = (unsigned)(key * 0x9E3779B97F4A7C15ull >> 56) & (kExclHash - 1);
  for (int p = 0; p < kExclHash; ++p) {
    const unsigned long long old = atomicCAS(&S.key[h], ~0ull, key);
    if (old == ~0ull || old == key) return;
    h = (h + 1) & (kExclHash - 1);
  }
  raise_error(counters, kErrExclOverflow);
}

// Writes the batch [0, cnt) of B as one work item (the masks of entries that need them first).
static __device__ void flush_batch(const SearchShared& S, SearchBatch& B, int sc, int cnt, int lane, const ListBufs& b) {
  if (cnt <= 0) return;
  // masks for the entries that need them: start from all pairs, drop exclusions and the lower triangle of a cluster
  // with itself under the zero image
  for (int e = 0; e < cnt; ++e) {
    if (!B.needs_mask[e]) continue;
    const unsigned cj = B.ent[e].x;
    const unsigned img = (B.ent[e].y >> 8) & 0x1FFFFFu;
    if (lane < 8) {
      unsigned long long mm = ~0ull;
      if (cj == unsigned(8 * sc + lane) && img == pack_image(0, 0, 0)) {
        // a cluster with itself: each pair once (j > i): bit 8 i + j
        mm = 0;
        for (int i = 0; i < 8; ++i)
          for (int j = i + 1; j < 8; ++j) mm |= 1ull << (8 * i + j);
      }
      B.m[e][lane] = mm;
    }
    __syncwarp();
    for (int r = lane; r < S.nrec; r += 32) {
      const uint2 rc = S.rec[r];
      if (rc.x != cj || (rc.y >> 9) != img) continue;
      const unsigned il = rc.y & 63u, jl = (rc.y >> 6) & 7u;
      atomicAnd(&B.m[e][il >> 3], ~(1ull << (8 * (il & 7) + jl)));
    }
    __syncwarp();
  }
  int base = 0, wi = 0;
  if (lane == 0) {
    base = atomicAdd(b.counters + kCntEnt, cnt);
    wi = atomicAdd(b.counters + kCntWork, 1);
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
    if (B.needs_mask[e]) {
      const int mi = atomicAdd(b.counters + kCntMask, 1);
      if (mi < b.mask_cap) {
        for (int k = 0; k < 8; ++k) b.masks[8 * size_t(mi) + k] = B.m[e][k];
        en.z = unsigned(mi + 1);
      } else {
        raise_error(b.counters, kErrMaskOverflow);
      }
    }
    b.ent[base + e] = en;
    b.ent_shift[base + e] = B.sh[e];
  }
  if (lane == 0) b.work[wi] = make_int4(sc, base, cnt, 0);
}

// K-SEARCH: one block of kSearchWarps warps per super-cluster. The block records the super-cluster's excluded pairs;
// then each warp takes a quarter of the neighbouring columns (with their images) and batches its own entries.
// Exclusions (ForceField::excluded) hold at their nearest image only (core/src/nbnxm.cpp:229-252): each of the
// super-cluster's excluded atom pairs is recorded with the image that is nearest at the build, and an entry for that j
// cluster under that image carries masks with those pairs cleared.
static __global__ void __launch_bounds__(32 * kSearchWarps) k_search(DevCell cell, ListGeom g, const uint32_t* __restrict__ excl_off,
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
    for (int t = threadIdx.x; t < 64; t += blockDim.x) {
      const int a = b.perm[64 * sc + t];
      if (a < 0) continue;
      const double* fa = b.frac + 3 * a;
      for (uint32_t p = excl_off[a]; p < excl_off[a + 1]; ++p) {
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
    __syncthreads();
    // --- candidates: neighbouring columns (with their images), super-clusters in c range, their 8 clusters. Each warp
    // takes a contiguous block of the columns, so that its entries (and the pair kernel's work items made of them) stay
    // spatially together.
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
            B.ent[pos] = make_uint4(unsigned(cj), imask | (img << 8), 0u, 0u);
            B.sh[pos] = make_float4(float(b.sc_org[3 * sjc] + S0 - S.org_i[0]), float(b.sc_org[3 * sjc + 1] + S1 - S.org_i[1]),
                                    float(b.sc_org[3 * sjc + 2] + S2 - S.org_i[2]), 0.f);
            B.needs_mask[pos] = (unsigned char)((zero && sjc == sc) || key_find(S, excl_key(unsigned(cj), img)));
          }
          __syncwarp();
          if (lane == 0) B.nent += __popc(ball);
          __syncwarp();
          while (B.nent >= g.batch) {   // a pass adds up to 32 entries: with a depth below 32 more than one batch fills
            flush_batch(S, B, sc, g.batch, lane, b);
            __syncwarp();
            // the rest (< 2 kBatch - batch entries) moves down: read all, then write (the ranges can overlap)
            const int rest = B.nent - g.batch;
            uint4 te[2];
            float4 ts[2];
            unsigned char tm[2];
#pragma unroll
            for (int k = 0; k < 2; ++k) {
              const int e = lane + 32 * k;
              if (e < rest) te[k] = B.ent[g.batch + e], ts[k] = B.sh[g.batch + e], tm[k] = B.needs_mask[g.batch + e];
            }
            __syncwarp();
#pragma unroll
            for (int k = 0; k < 2; ++k) {
              const int e = lane + 32 * k;
              if (e < rest) B.ent[e] = te[k], B.sh[e] = ts[k], B.needs_mask[e] = tm[k];
            }
            __syncwarp();
            if (lane == 0) B.nent = rest;
            __syncwarp();
          }
        }
      }
    }
    flush_batch(S, B, sc, B.nent, lane, b);
    __syncthreads();   // S is rewritten for the next super-cluster
  }
}

}  // namespace capsb
