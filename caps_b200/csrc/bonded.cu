// Host side of the bonded terms, 1-4 pairs and excluded-pair corrections: every kind in one launch (k_bonded).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <vector>

#include "engine.h"
#include "bonded.cuh"

namespace capsb {

void Engine::bonded_forces(const double* d_x, bool ener, bool vir, int parts) {
  BondedArgs A{d_x, dcell_, EnergySink{d_efix_.p, d_edbl_.p}, mixed_ ? 1 : 0};
  const int T = 256;
  // parts: 1 bonded terms, 2 short-range non-bonded (1-4 pairs; DSF exclusion corrections), 4 long-range (the PME
  // exclusion corrections)
  const bool bonded = (parts & 1) != 0, nonb = (parts & 2) != 0, excl = (parts & (pme_ ? 4 : 2)) != 0;
  BondedWork W{};
  int blocks = 0;
  auto segment = [&](int kind, int cnt) {
    if (cnt <= 0) return;
    W.kind[W.nseg] = kind;
    W.first[W.nseg] = blocks;
    blocks += std::min(blocks_for(size_t(cnt), T), bonded_cap_ > 0 ? bonded_cap_ : dev_sms_ * 4);
    ++W.nseg;
  };
  if (bonded) {
    segment(kBkDihedrals, ndg_);   // the costliest terms first, so that their blocks start first
    segment(kBkImpropers, nig_);
    segment(kBkAngles, na_);
    segment(kBkBonds, nb_);
    segment(kBkFene, nfene_);
  }
  if (nonb) segment(kBkPairs14, np14_);
  if (excl && coul_) segment(kBkExcl, nx_);
  if (!W.nseg) return;
  W.first[W.nseg] = blocks;
  W.nb = nb_, W.na = na_, W.ndg = ndg_, W.nig = nig_, W.nf = nfene_, W.np14 = np14_, W.nx = nx_;
  W.bond_ij = d_bond_ij_.p, W.bond_kr = d_bond_kr_.p;
  W.angle_ijk = d_angle_ijk_.p, W.angle_kt = d_angle_kt_.p;
  W.dih_grp = d_dih_grp_.p, W.dih_ijkl = d_dih_ijkl_.p, W.dih_vd = d_dih_vd_.p, W.dih_n = d_dih_n_.p;
  W.imp_grp = d_imp_grp_.p, W.imp_ijkl = d_imp_ijkl_.p, W.imp_vd = d_imp_vd_.p, W.imp_n = d_imp_n_.p;
  W.fene_ij = d_fene_ij_.p, W.fene_p = d_fene_p_.p, W.counters = d_counters_.p, W.info = d_errinfo_.p;
  W.p14_ij = d_p14_ij_.p, W.p14_scale = p14_scaled_ ? d_p14_scale_.p : nullptr, W.lj14 = lj14_, W.type = d_type_.p, W.nt = nt_;
  W.lj14g_tab = d_lj14g_.p, W.lj14g2_tab = d_lj14g2_.p, W.lj_inner = lj_inner_, W.tables = pair_tables();
  W.lj_fsw = lj_fsw_ && !lj96_ ? 1 : 0, W.rc = rc_;
  W.lj14_tab = d_lj14_.p, W.cap14_tab = opt_.force_cap > 0 ? (const double4*)d_cap14_.p : (const double4*)nullptr, W.lj96 = lj96_ ? 1 : 0;
  W.X = ExclArgs{d_excl_ij_.p, d_excl_f_.p, d_q_.p, d_gtab_.p, ghi_, rc_, rc_ * rc_, kappa_, dsf_e0_, dsf_f0_, pme_ ? 1 : 0};
  auto run = [&](auto sink) {
    using S = decltype(sink);
    if (ener) {
      if (vir) launch_k(k_bonded<double, S, true, true>, blocks, T, 0, stream_, W, A, sink);
      else launch_k(k_bonded<double, S, true, false>, blocks, T, 0, stream_, W, A, sink);
    } else {
      if (vir) launch_k(k_bonded<double, S, false, true>, blocks, T, 0, stream_, W, A, sink);
      else launch_k(k_bonded<double, S, false, false>, blocks, T, 0, stream_, W, A, sink);
    }
  };
  if (mixed_) run(ForceSink<float>{d_F_.p, d_F_.p + n_, d_F_.p + 2 * size_t(n_), d_counters_.p + kCntErr});
  else run(ForceSink<double>{d_Fd_.p, d_Fd_.p + n_, d_Fd_.p + 2 * size_t(n_)});
}

}  // namespace capsb
