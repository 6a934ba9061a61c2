// Host side of the non-bonded forces: the list build sequence, dynamic pruning, the pair-kernel launch, and the
// per-evaluation orchestration of every force term into the caller's AoS doubles.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <vector>

#include "engine.h"
#include "pair.cuh"

namespace capsb {

namespace {

__global__ void k_set_flag(int* counters, int slot, int v) {
  counters[slot] = v;
}

// Forces to the caller's AoS doubles: atom-order sums plus the pair kernel's slot-order sums.
__global__ void k_reduce_f32(int n, const long long* __restrict__ F, const long long* __restrict__ Fs, int nslots, const int* __restrict__ iperm,
                             double* __restrict__ f, int with_pairs) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int s = with_pairs ? iperm[i] : -1;
  const bool ok = s >= 0 && s < nslots;   // a build that overflowed can leave iperm stale: the host reports it
  for (int k = 0; k < 3; ++k) {
    long long v = F[size_t(k) * n + i];
    if (ok) v += Fs[size_t(k) * nslots + s];
    f[3 * i + k] = double(v) * kInvFixF;
  }
}
__global__ void k_reduce_f64(int n, const double* __restrict__ F, const double* __restrict__ Fs, int nslots, const int* __restrict__ iperm,
                             double* __restrict__ f, int with_pairs) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int s = with_pairs ? iperm[i] : -1;
  const bool ok = s >= 0 && s < nslots;
  for (int k = 0; k < 3; ++k) {
    double v = F[size_t(k) * n + i];
    if (ok) v += Fs[size_t(k) * nslots + s];
    f[3 * i + k] = v;
  }
}

}  // namespace

void Engine::fork(int k, const std::function<void()>& launch) {
  CK(cudaEventRecord(ev_fork_, stream_));
  CK(cudaStreamWaitEvent(side_[k], ev_fork_, 0));
  struct Swap {
    cudaStream_t& s;
    cudaStream_t saved;
    ~Swap() { s = saved; }
  } swap{stream_, stream_};
  stream_ = side_[k];
  launch();
  CK(cudaEventRecord(ev_join_[k], side_[k]));
}

void Engine::join(int k) { CK(cudaStreamWaitEvent(stream_, ev_join_[k], 0)); }

// Autotuner for the j-tile depth: the list is built with 32, 24 and 16 entries per work item and the pair kernel timed
// on each (fewer entries per item balance small systems better, more amortise the per-item work); the fastest is kept
// for this engine. Runs once, at the first non-bonded evaluation (never inside a stream capture).
void Engine::tune_batch(const double* d_x) {
  batch_tuned_ = true;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  float best = 1e30f;
  int pick = batch_;
  const size_t ns = size_t(nsc_cap_) * kScAtoms;
  for (int bsz : {32, 24, 16}) {
    geom_.batch = bsz;
    launch_k(k_set_flag, 1, 1, 0, stream_, d_counters_.p, kCntRebuild, 1);
    launch_build(d_x);
    if (mixed_)
      launch_k(k_pack_f32, blocks_for(ns, 256), 256, 0, stream_, int(ns), d_perm_.p, d_x, d_ioff_.p, dcell_, d_sc_org_.p, d_q_.p, d_type_.p, nt_,
                                                           d_xq_.p, d_tslot_.p, d_counters_.p, d_x0_.p, d_Fs_.p);
    else
      launch_k(k_pack_f64, blocks_for(ns, 256), 256, 0, stream_, int(ns), d_perm_.p, d_x, d_ioff_.p, dcell_, d_q_.p, d_type_.p, nt_, d_xqd_.p, d_tslot_.p,
                                                           d_counters_.p, d_x0_.p, d_Fsd_.p);
    prune(d_x);
    float ms = 0;
    for (int rep = 0; rep < 4; ++rep) {
      CK(cudaMemsetAsync(d_counters_.p + kCntPairNext, 0, sizeof(int), stream_));
      if (rep == 1) CK(cudaEventRecord(e0, stream_));
      pair_forces(false, false);
    }
    CK(cudaEventRecord(e1, stream_));
    CK(cudaEventSynchronize(e1));
    CK(cudaEventElapsedTime(&ms, e0, e1));
    if (ms < best) best = ms, pick = bsz;
  }
  batch_ = pick;
  geom_.batch = pick;
  list_valid_ = false;   // the evaluation that follows builds the list with the chosen depth
  // The pair kernel's persistent grid holds every SM slot while it runs, so the bonded and PME branches of the same
  // evaluation wait for it to end unless it leaves room; PME's line transforms, on the other hand, run in fewer waves
  // on the slots left when their grid is capped. Time whole force-only evaluations for each pair (pair grid full or one
  // block per SM fewer; PME grid uncapped, one or two blocks per SM), in alternating rounds, and keep the fastest.
  // The bonded kernel's blocks, launched at the same time on a side stream, are capped likewise (four per SM, or half
  // a block per SM per term kind), so that they do not take every slot ahead of the list and pair kernels.
  const int caps[3] = {0, dev_sms_, 2 * dev_sms_};
  const int bcaps[2] = {0, std::max(1, dev_sms_ / 2)};
  float bestc[2][3][2];
  for (auto& r : bestc)
    for (auto& q : r)
      for (float& v : q) v = 1e30f;
  for (int round = 0; round < 3; ++round)
    for (int cut = 0; cut < 2; ++cut)
      for (int ci = 0; ci < (pme_ ? 3 : 1); ++ci)
        for (int bi = 0; bi < 2; ++bi) {
          pair_cut_ = cut;
          pme_cap_ = caps[ci];
          bonded_cap_ = bcaps[bi];
          for (int rep = 0; rep < 4; ++rep) {
            if (rep == 1) CK(cudaEventRecord(e0, stream_));
            forces(d_x, false, false, false);
          }
          CK(cudaEventRecord(e1, stream_));
          CK(cudaEventSynchronize(e1));
          float ms = 0;
          CK(cudaEventElapsedTime(&ms, e0, e1));
          bestc[cut][ci][bi] = std::min(bestc[cut][ci][bi], ms);
        }
  int bc = 0, pc = 0, bb = 0;
  for (int cut = 0; cut < 2; ++cut)
    for (int ci = 0; ci < 3; ++ci)
      for (int bi = 0; bi < 2; ++bi)
        if (bestc[cut][ci][bi] < bestc[bc][pc][bb]) bc = cut, pc = ci, bb = bi;
  pair_cut_ = bc;
  pme_cap_ = caps[pc];
  bonded_cap_ = bcaps[bb];
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
}

int Engine::list_builds() { return counter(kCntBuilds); }
void Engine::list_counts(int64_t* v) {
  v[0] = counter(kCntBuilds);
  v[1] = counter(kCntPrunes);
}

int Engine::counter(int slot) {
  int v = 0;
  CK(cudaMemcpyAsync(&v, d_counters_.p + slot, sizeof(int), cudaMemcpyDeviceToHost, stream_));
  CK(cudaStreamSynchronize(stream_));
  return v;
}

// ---------------------------------------------------------------------------------------------------------------
void Engine::launch_build(const double* d_x) {
  const ListGeom& g = geom_;
  // binning (its last block scans the columns), the scatter into columns, and the sort of each column (its block then
  // forms the column's super-clusters): three launches before the search
  launch_k(k_bin, blocks_for(size_t(n_), kBinThreads), kBinThreads, 0, stream_, n_, d_x, dcell_, g, lb_);
  launch_k(k_scatter, blocks_for(size_t(n_), 256), 256, 0, stream_, n_, lb_);
  const size_t sort_smem = size_t(kSortMax) * (sizeof(double) + sizeof(int));
  launch_k(k_sort_columns, std::min(g.ncol, dev_sms_ * 8), kSortThreads, sort_smem, stream_, dcell_, g, lb_);
  if (sizeof(SearchShared) > 48 * 1024) CK(cudaFuncSetAttribute(k_search, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sizeof(SearchShared))));
  launch_k(k_search, std::max(1, std::min(nsc_cap_, dev_sms_ * 8)), 32 * kSearchWarps, sizeof(SearchShared), stream_, dcell_, g, d_excl_off_.p,
                                                                                                          d_excl_list_.p, lb_);
  CK(cudaGetLastError());
}

PairArgs Engine::pair_args() {
  PairArgs A{};
  A.work = d_work_.p;
  A.ent = d_ent_.p;
  A.ent_shift = d_ent_shift_.p;
  A.masks = d_masks_.p;
  A.frozen = d_frozen_.p;
  A.counters = d_counters_.p;
  A.tslot = d_tslot_.p;
  A.xq = d_xq_.p;
  A.xqd = d_xqd_.p;
  A.tab = d_tab_.p;
  A.ljf = d_ljf_.p;
  A.batch = std::max(1, std::min(geom_.batch, kBatch));
  A.tabd = d_tabd_.p;
  A.tabcap = d_tabcap_.p;
  A.tabg = d_tabg_.p;
  A.tabg2 = d_tabg2_.p;
  A.lj_inner = lj_inner_;
  A.lj_fsw = lj_fsw_ && !lj96_ ? 1 : 0;
  A.tables = pair_tables();
  A.gtab = d_gtab_.p;
  A.ntab = nt_ + 1;
  A.gnodes = coul_ ? gnodes_ : 0;   // a table only with Coulomb: the FP64 kernel's shared memory holds it then
  A.ghi = ghi_;
  A.cell = dcell_;
  A.rc2 = rc_ * rc_;
  A.rc = rc_;
  A.beta = kappa_;
  A.kc = 2 * kappa_ / std::sqrt(kPi);
  A.kcoul = kCoulomb;
  A.dsf_e0 = dsf_e0_;
  A.dsf_f0 = dsf_f0_;
  A.fsx = d_Fs_.p;
  A.fsy = d_Fs_.p + d_Fs_.n / 3;
  A.fsz = d_Fs_.p + 2 * (d_Fs_.n / 3);
  if (!mixed_) {
    A.fdx = d_Fsd_.p;
    A.fdy = d_Fsd_.p + d_Fsd_.n / 3;
    A.fdz = d_Fsd_.p + 2 * (d_Fsd_.n / 3);
  }
  A.en.fix = d_efix_.p;
  A.en.dbl = d_edbl_.p;
  A.work_cap = int(d_work_.n);
  A.err = d_counters_.p + kCntErr;
  return A;
}

ListCheck Engine::list_check(int nfree, const int* free_atoms) const {
  const double b = std::min(0.8, skin_);   // the prune margin (see prune())
  return ListCheck{d_x0_.p, d_xp_.p, 0.25 * skin_ * skin_, 0.25 * b * b, d_counters_.p, nfree, free_atoms};
}

bool Engine::list_check_fusable() const { return (opt_.parts & 2) != 0 && list_valid_ && !frozen_; }

// Dynamic pruning: when an atom has moved b/2 since the last prune (b = min(0.8 Å, skin), as field.cpp:1306-1312; the
// step's displacement check tests it), or a build set the flag, every entry's masks are rewritten for r_c + b.
void Engine::prune(const double* d_x) {
  const double b = std::min(0.8, skin_);
  const PairArgs A = pair_args();
  const double rp = rc_ + b;
  if (mixed_) launch_k(k_prune<false>, dev_sms_ * 8, 128, 0, stream_, A, rp * rp, d_ent_.p, n_, d_x, d_xp_.p);
  else launch_k(k_prune<true>, dev_sms_ * 8, 128, 0, stream_, A, rp * rp, d_ent_.p, n_, d_x, d_xp_.p);
}

void Engine::pair_forces(bool ener, bool vir) {
  PairArgs A = pair_args();
  const int coul = coul_ ? (pme_ ? 1 : 2) : 0;
  // persistent grids: as many blocks as fit on the SMs at once (less pair_cut_ per SM, the tuner's choice); their warps
  // fetch work items until none are left
  const int ntab = nt_ + 1;
  if (mixed_) {
    // LJ table, the 4 warps' i atoms (three float4 each) and types, and their staged entries with the entries' j atoms
    // and exclusion masks
    const size_t smem = sizeof(float4) * (size_t(ntab) * ntab + 4 * 64 * 3) + sizeof(int) * 4 * 64 +
                        4 * size_t(A.batch) * (sizeof(uint4) + sizeof(float4) + 8 * sizeof(float4) + 4 * sizeof(float4) + 8 * sizeof(unsigned long long));
    // the rational fits hold for (kappa r_c)^2 <= 16; past that the library erfc form
    const int c32 = coul == 0 ? 0 : (kappa_ * kappa_ * rc_ * rc_ <= double(kEwUMax) ? coul : coul + 2);
#define PAIR32L(C, E, V, L, M)                                                                                       \
  do {                                                                                                               \
    if (smem > 48 * 1024) CK(cudaFuncSetAttribute(k_pair_f32<C, E, V, L, M>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem))); \
    int per_sm = 0;                                                                                                  \
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pair_f32<C, E, V, L, M>, 128, smem));                \
    launch_k(k_pair_f32<C, E, V, L, M>, dev_sms_ * std::max(1, per_sm - pair_cut_), 128, smem, stream_, A);          \
  } while (0)
#define PAIR32(C, E, V)                                                                                              \
  do {                                                                                                               \
    if (lj96_) PAIR32L(C, E, V, true, false);                                                                        \
    else if (comb_ && !(E)) PAIR32L(C, E, V, false, !(E));                                                           \
    else PAIR32L(C, E, V, false, false);                                                                             \
  } while (0)
#define PAIR32C(C) { if (ener) { if (vir) PAIR32(C, true, true); else PAIR32(C, true, false); } else { if (vir) PAIR32(C, false, true); else PAIR32(C, false, false); } }
    switch (c32) {
      case 1: PAIR32C(1) break;
      case 2: PAIR32C(2) break;
      case 3: PAIR32C(3) break;
      case 4: PAIR32C(4) break;
      default: PAIR32C(0) break;
    }
#undef PAIR32C
#undef PAIR32
#undef PAIR32L
  } else {
    const size_t smem = sizeof(double4) * (size_t(ntab) * ntab + 4 * 64) + sizeof(double) * 2 * size_t(coul ? gnodes_ : 0) + sizeof(int) * 4 * 64;
#define PAIR64LF(C, E, V, CAP, L, F)                                                                                 \
  do {                                                                                                               \
    if (smem > 48 * 1024) CK(cudaFuncSetAttribute(k_pair_f64<C, E, V, CAP, L, F>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem))); \
    int per_sm = 0;                                                                                                  \
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pair_f64<C, E, V, CAP, L, F>, 128, smem));           \
    launch_k(k_pair_f64<C, E, V, CAP, L, F>, dev_sms_ * std::max(1, per_sm - pair_cut_), 128, smem, stream_, A);                       \
  } while (0)
#define PAIR64L(C, E, V, CAP, L) PAIR64LF(C, E, V, CAP, L, false)
#define PAIR64(C, E, V, CAP)                                                                                         \
  do {                                                                                                               \
    if (lj96_) PAIR64L(C, E, V, CAP, true);                                                                          \
    else PAIR64L(C, E, V, CAP, false);                                                                               \
  } while (0)
#define PAIR64FROZEN(C)                                                                                              \
  do {                                                                                                               \
    if (lj96_) PAIR64LF(C, true, true, false, true, true);                                                           \
    else PAIR64LF(C, true, true, false, false, true);                                                                \
  } while (0)
    if (frozen_) {
      // a frozen pair set: energies and virial always on (finite-difference second derivatives read them)
      if (coul == 1) PAIR64FROZEN(1);
      else if (coul == 2) PAIR64FROZEN(2);
      else PAIR64FROZEN(0);
    } else if (opt_.force_cap > 0 || generic_ || lj_fsw_) {
      // the push-off cap, the generic pair forms and CHARMM's force switch: energies and virial always on (rare paths,
      // kept to one instantiation per Coulomb form, so the plain kernels carry none of their branches)
      if (coul == 1) PAIR64(1, true, true, true);
      else if (coul == 2) PAIR64(2, true, true, true);
      else PAIR64(0, true, true, true);
    } else if (coul == 1) { if (ener) { if (vir) PAIR64(1, true, true, false); else PAIR64(1, true, false, false); } else { if (vir) PAIR64(1, false, true, false); else PAIR64(1, false, false, false); } }
    else if (coul == 2) { if (ener) { if (vir) PAIR64(2, true, true, false); else PAIR64(2, true, false, false); } else { if (vir) PAIR64(2, false, true, false); else PAIR64(2, false, false, false); } }
    else { if (ener) { if (vir) PAIR64(0, true, true, false); else PAIR64(0, true, false, false); } else { if (vir) PAIR64(0, false, true, false); else PAIR64(0, false, false, false); } }
#undef PAIR64FROZEN
#undef PAIR64
#undef PAIR64L
#undef PAIR64LF
  }
  CK(cudaGetLastError());
}

long long Engine::count_pairs() {
  if (!list_valid_ || mixed_) return 0;
  DevBuf<unsigned long long> cnt;
  cnt.alloc(1);
  cnt.zero(stream_);
  launch_k(k_count_pairs, dev_sms_ * 4, 128, 0, stream_, pair_args(), d_ent_.p, d_perm_.p, d_x0_.p, d_ioff_.p, (rc_ + skin_) * (rc_ + skin_), cnt.p);
  CK(cudaGetLastError());
  unsigned long long v = 0;
  CK(cudaMemcpyAsync(&v, cnt.p, sizeof v, cudaMemcpyDeviceToHost, stream_));
  CK(cudaStreamSynchronize(stream_));
  return static_cast<long long>(v);
}

// The reference's pairs() is the size of its FP64 atom-pair list; on its cluster (mixed) path that list is only built by
// freeze_pairs, so a mixed evaluator reports the list of its last freeze, or none.
long long Engine::pairs() {
  if (frozen_) return frozen_pairs_;
  return mixed_ ? frozen_pairs_ : count_pairs();
}

void Engine::freeze_pairs(const double* x, const double* cell) {
  if (opt_.force_cap > 0) throw ModelError(CAPS_GPU_EINVAL, "freeze_pairs: the device path freezes no list under a force cap");
  unfreeze();
  if (mixed_) {   // a frozen list runs on the reference's FP64 atom-pair path (field.cpp:845), so on this engine's FP64 path
    frozen_saved_precision_ = opt_.precision;
    opt_.precision = 1;
    setup_options();
  }
  // the list built at (x, cell), then the pairs inside r_c there
  list_valid_ = false;
  std::vector<double> f(3 * size_t(n_));
  caps_gpu_terms t{};
  compute_host(x, cell, f.data(), &t);
  frozen_pairs_ = count_pairs();
  d_frozen_.alloc(size_t(8) * d_ent_.n);
  launch_k(k_freeze, dev_sms_ * 4, 128, 0, stream_, pair_args(), d_ent_.p, d_frozen_.p);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(stream_));
  frozen_ = true;
}

void Engine::unfreeze() {
  if (!frozen_) return;
  frozen_ = false;
  if (frozen_saved_precision_ >= 0) {
    opt_.precision = frozen_saved_precision_;
    frozen_saved_precision_ = -1;
  }
  setup_options();   // the cell may have changed while frozen: geometry, capacity and list from scratch
}

// One force evaluation on device positions d_x (AoS, 3 n): accumulators cleared, list checked / rebuilt, every term,
// forces reduced into d_f_ (AoS doubles). Asynchronous on stream_.
void Engine::forces(const double* d_x, bool ener, bool vir, bool check_rebuild, int parts, double* d_out, bool clear_energies, bool reduce) {
  // internal part mask: 1 bonded, 2 short-range non-bonded (list, pair kernel, 1-4 pairs), 4 long-range (PME and its
  // excluded-pair corrections); the options' non-bonded bit means both 2 and 4
  const int pm = parts >= 0 ? parts : ((opt_.parts & 1) | ((opt_.parts & 2) ? 6 : 0));
  const bool nonb = (pm & 2) != 0;
  double* out = d_out ? d_out : d_f_.p;
  if (nonb && !batch_tuned_) tune_batch(d_x);
  // the atom-order sums start at zero (the integrator's kick may have cleared them already); the pack kernel clears the
  // pair kernel's slot-order sums
  if (!sums_cleared_) {
    if (mixed_) CK(cudaMemsetAsync(d_F_.p, 0, d_F_.n * sizeof(long long), stream_));
    else CK(cudaMemsetAsync(d_Fd_.p, 0, d_Fd_.n * sizeof(double), stream_));
  }
  sums_cleared_ = false;
  if ((ener || vir) && clear_energies) {
    CK(cudaMemsetAsync(d_efix_.p, 0, d_efix_.n * sizeof(long long), stream_));
    CK(cudaMemsetAsync(d_edbl_.p, 0, d_edbl_.n * sizeof(double), stream_));
  }
  // Three branches: bonded terms and PME beside the list and pair kernels. All add into order-free fixed-point (or
  // atomic FP64) sums, so how the branches interleave does not change the mixed path's result.
  fork(0, [&] { bonded_forces(d_x, ener, vir, pm); });
  const bool pme = (pm & 4) != 0 && pme_;
  if (pme) fork(1, [&] { pme_forces(d_x, ener, vir); });
  if (nonb) {
    if (frozen_) {
      // a frozen pair set: no displacement check, build or prune; the pack and the pair kernel run on the frozen list
    } else if (!list_valid_) {
      launch_k(k_set_flag, 1, 1, 0, stream_, d_counters_.p, kCntRebuild, 1);
      list_valid_ = true;
    } else if (check_rebuild) {
      launch_k(k_check_step, blocks_for(size_t(n_), 256), 256, 0, stream_, n_, d_x, list_check(0, nullptr));
    }
    if (!frozen_) launch_build(d_x);
    const size_t ns = size_t(nsc_cap_) * kScAtoms;
    if (mixed_)
      launch_k(k_pack_f32, blocks_for(ns, 256), 256, 0, stream_, int(ns), d_perm_.p, d_x, d_ioff_.p, dcell_, d_sc_org_.p, d_q_.p, d_type_.p, nt_,
                                                           d_xq_.p, d_tslot_.p, d_counters_.p, d_x0_.p, d_Fs_.p);
    else
      launch_k(k_pack_f64, blocks_for(ns, 256), 256, 0, stream_, int(ns), d_perm_.p, d_x, d_ioff_.p, dcell_, d_q_.p, d_type_.p, nt_, d_xqd_.p, d_tslot_.p,
                                                           d_counters_.p, d_x0_.p, d_Fsd_.p);
    if (!frozen_) prune(d_x);
    pair_forces(ener, vir);
  }
  join(0);
  if (pme) join(1);
  if (!reduce) return;   // the caller's kick reads the sums (with iperm) itself
  const size_t ns = size_t(nsc_cap_) * kScAtoms;
  if (mixed_) launch_k(k_reduce_f32, blocks_for(size_t(n_), 256), 256, 0, stream_, n_, d_F_.p, d_Fs_.p, int(ns), d_iperm_.p, out, nonb ? 1 : 0);
  else launch_k(k_reduce_f64, blocks_for(size_t(n_), 256), 256, 0, stream_, n_, d_Fd_.p, d_Fsd_.p, int(ns), d_iperm_.p, out, nonb ? 1 : 0);
  CK(cudaGetLastError());
}

}  // namespace capsb
