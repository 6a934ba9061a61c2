// Host side of the bonded terms, 1-4 pairs and excluded-pair corrections: one launch per term kind.
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
  auto nblk = [&](int cnt) { return std::min(blocks_for(size_t(std::max(cnt, 1)), T), dev_sms_ * 4); };
#define LAUNCH3(K, S, cnt, ...)                                                                                     \
  do {                                                                                                              \
    if (ener) { if (vir) K<double, S, true, true><<<nblk(cnt), T, 0, stream_>>>(__VA_ARGS__); else K<double, S, true, false><<<nblk(cnt), T, 0, stream_>>>(__VA_ARGS__); } \
    else { if (vir) K<double, S, false, true><<<nblk(cnt), T, 0, stream_>>>(__VA_ARGS__); else K<double, S, false, false><<<nblk(cnt), T, 0, stream_>>>(__VA_ARGS__); } \
  } while (0)
#define LAUNCHX(S, ...)                                                                                             \
  do {                                                                                                              \
    if (ener) { if (vir) k_excl_f64<S, true, true><<<nblk(nx_), T, 0, stream_>>>(__VA_ARGS__); else k_excl_f64<S, true, false><<<nblk(nx_), T, 0, stream_>>>(__VA_ARGS__); } \
    else { if (vir) k_excl_f64<S, false, true><<<nblk(nx_), T, 0, stream_>>>(__VA_ARGS__); else k_excl_f64<S, false, false><<<nblk(nx_), T, 0, stream_>>>(__VA_ARGS__); } \
  } while (0)
  auto run = [&](auto sink) {
    using S = decltype(sink);
    const S F = sink;
    if (bonded) {
      if (nb_) LAUNCH3(k_bonds, S, nb_, nb_, d_bond_ij_.p, d_bond_kr_.p, A, F);
      if (na_) LAUNCH3(k_angles, S, na_, na_, d_angle_ijk_.p, d_angle_kt_.p, A, F);
      if (ndg_) LAUNCH3(k_torsions, S, ndg_, ndg_, d_dih_grp_.p, d_dih_ijkl_.p, d_dih_vd_.p, d_dih_n_.p, A, F, int(kEDihedral));
      if (nig_) LAUNCH3(k_torsions, S, nig_, nig_, d_imp_grp_.p, d_imp_ijkl_.p, d_imp_vd_.p, d_imp_n_.p, A, F, int(kEImproper));
      if (nfene_) LAUNCH3(k_fene, S, nfene_, nfene_, d_fene_ij_.p, d_fene_p_.p, A, F, d_counters_.p);
    }
    if (nonb && np14_)
      LAUNCH3(k_pairs14, S, np14_, np14_, d_p14_ij_.p, p14_scaled_ ? d_p14_scale_.p : nullptr, lj14_, d_type_.p, nt_, d_lj14_.p,
              opt_.force_cap > 0 ? (const double4*)d_cap14_.p : (const double4*)nullptr, A, F, lj96_ ? 1 : 0);
    if (excl && coul_ && nx_) {
      ExclArgs E{d_excl_ij_.p, d_excl_f_.p, d_q_.p, d_gtab_.p, ghi_, rc_, rc_ * rc_, kappa_, dsf_e0_, dsf_f0_, pme_ ? 1 : 0};
      LAUNCHX(S, nx_, E, A, F);
    }
  };
  if (mixed_) run(ForceSink<float>{d_F_.p, d_F_.p + n_, d_F_.p + 2 * size_t(n_), d_counters_.p + kCntErr});
  else run(ForceSink<double>{d_Fd_.p, d_Fd_.p + n_, d_Fd_.p + 2 * size_t(n_)});
#undef LAUNCH3
#undef LAUNCHX
  CK(cudaGetLastError());
}

}  // namespace capsb
