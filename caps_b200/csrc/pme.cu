// Host side of PME: plans, twiddle tables and line blocking per grid, and the spread / transform / solve / gather
// launch sequence.
#include <algorithm>
#include <array>
#include <map>
#include <mutex>
#include <cmath>
#include <cstring>
#include <functional>
#include <vector>

#include "engine.h"
#include "pme.cuh"

namespace capsb {

namespace {

void factor_radices(int n, int* rad, int& nst) {
  nst = 0;
  int r = n;
  while (r % 4 == 0 && nst < kMaxRadices) rad[nst++] = 4, r /= 4;
  for (int p : {2, 3, 5, 7}) while (r % p == 0 && nst < kMaxRadices) rad[nst++] = p, r /= p;
  if (r != 1) throw ModelError(CAPS_GPU_EINVAL, "PME grid length " + std::to_string(n) + " cannot be factored for the line FFT");
}

}  // namespace

template <class R>
void Engine::pme_setup(PmePath<R>& P) {
  using T = typename Cpx<R>::T;
  const size_t half = size_t(ph1_) * pk_[1] * pk_[2];
  P.h.alloc(half);
  P.gr.alloc(size_t(pk_[0]) * pk_[1] * pk_[2]);
  P.gt.alloc(half);
  P.wt.alloc(6 * half);
  if (mixed_) d_gridq_.alloc(size_t(pk_[0]) * pk_[1] * pk_[2]);
  d_grid_.alloc(size_t(pk_[0]) * pk_[1] * pk_[2]);
  for (int d = 0; d < 3; ++d)
    for (int dir = 0; dir < 2; ++dir) {
      const int nn = pk_[d];
      const int sign = dir == 0 ? -1 : +1;   // forward e^{-i}, inverse e^{+i}: the convolution is the same either way
      std::vector<T> tw(static_cast<size_t>(nn));
      for (int k = 0; k < nn; ++k) {
        const double ang = 2 * kPi * k / nn;
        tw[size_t(k)] = T{R(std::cos(ang)), R(sign * std::sin(ang))};
      }
      P.tw[d][dir].upload(tw, stream_);
      FftPlan<R>& pl = P.plan[d][dir];
      pl.n = nn;
      factor_radices(nn, pl.rad, pl.nst);
      pl.tw = P.tw[d][dir].p;
      pl.sign = sign;
    }
  // Lines per block. x: contiguous lines, enough blocks for four per SM, two buffers within 40 KB of shared memory.
  // y, z: `la` consecutive a per block so that each row read is 128 bytes.
  const int cap = int(40 * 1024 / (2 * sizeof(T)));
  const int nlx = pk_[1] * pk_[2];
  P.lines[0] = std::max(1, std::min({cap / pk_[0], 16, (nlx + 4 * dev_sms_ - 1) / (4 * dev_sms_)}));
  const int la = int(128 / sizeof(T));
  P.lines[1] = std::max(1, std::min({la, cap / pk_[1], ph1_}));
  P.lines[2] = std::max(1, std::min({la, cap / pk_[2], ph1_}));
  if (tuning_pinned_)
    for (int d = 0; d < 3; ++d) P.lines[d] = pinned_lines_[d];
  else
    pme_tune(P);
  for (int d = 0; d < 3; ++d) P.k[d] = pk_[d];
  green_valid_ = false;
  CK(cudaStreamSynchronize(stream_));
}

void Engine::tuning(int32_t v[7]) const {
  const int* l = pme_lines();
  const int32_t t[7] = {batch_, pair_cut_, pme_cap_, bonded_cap_, l[0], l[1], l[2]};
  std::memcpy(v, t, sizeof t);
}

void Engine::pin_tuning(const int32_t v[7]) {
  if (v[0] < 1 || v[0] > kBatch || v[1] < 0 || v[2] < 0 || v[3] < 0 || v[4] < 1 || v[5] < 1 || v[6] < 1)
    throw ModelError(CAPS_GPU_EINVAL, "tuning values out of range");
  batch_ = geom_.batch = v[0];
  pair_cut_ = v[1];
  pme_cap_ = v[2];
  bonded_cap_ = v[3];
  for (int d = 0; d < 3; ++d) pinned_lines_[d] = v[4 + d];
  auto& lines = mixed_ ? pf_.lines : pd_.lines;
  for (int d = 0; d < 3; ++d) lines[d] = v[4 + d];
  tuning_pinned_ = true;
  batch_tuned_ = true;
  list_valid_ = false;
  drop_run_state();
}

// The mixed path transforms in FP32 (pf_), the FP64 path in FP64 (pd_); each path is set up for the current grid on
// first use.
void Engine::ensure_pme() {
  if (!pme_ || pk_[0] == 0) return;
  auto same = [&](const int* k) { return k[0] == pk_[0] && k[1] == pk_[1] && k[2] == pk_[2]; };
  if (mixed_) {
    if (!same(pf_.k)) pme_setup(pf_);
    d_gridq_.alloc(size_t(pk_[0]) * pk_[1] * pk_[2]);
  } else if (!same(pd_.k)) {
    pme_setup(pd_);
  }
}

// The five line-transform passes of one PME evaluation (forward x, y; z with the solve; inverse y, x).
template <class R>
void Engine::fft_passes(PmePath<R>& P, bool ener, bool vir) {
  using T = typename Cpx<R>::T;
  PmeArgs A{pk_[0], pk_[1], pk_[2], ph1_, dcell_, nullptr, d_q_.p, n_};
  // shared memory: twiddle table(s) + two line buffers
  const size_t sx = (size_t(P.lines[0]) * 2 + 1) * pk_[0] * sizeof(T), sy = (size_t(P.lines[1]) * 2 + 1) * pk_[1] * sizeof(T),
               sz = (size_t(P.lines[2]) + 1) * 2 * pk_[2] * sizeof(T);
  const int nlx = pk_[1] * pk_[2];
  // the kernels stride over their line groups: a grid cap (the tuner's pme_cap_, 0 for none) leaves SM slots to the
  // pair kernel that runs beside them
  auto capped = [&](int g) { return pme_cap_ > 0 ? std::min(g, pme_cap_) : g; };
  launch_k(k_fft_x_fwd<R>, capped(blocks_for(size_t(nlx), P.lines[0])), 128, sx, stream_, A, mixed_ ? nullptr : d_grid_.p, mixed_ ? d_gridq_.p : nullptr, P.h.p,
                                                                        P.plan[0][0], P.lines[0]);
  const int gy = capped(((ph1_ + P.lines[1] - 1) / P.lines[1]) * pk_[2]);
  launch_k(k_fft_y<R>, gy, 128, sy, stream_, A, P.h.p, P.plan[1][0], P.lines[1]);
  const int gz = capped(((ph1_ + P.lines[2] - 1) / P.lines[2]) * pk_[1]);
  EnergySink en{d_efix_.p, d_edbl_.p};
  if (ener) { if (vir) launch_k(k_fft_z_solve<R, true, true>, gz, 128, sz, stream_, A, P.h.p, P.gt.p, P.wt.p, P.plan[2][0], P.plan[2][1], P.lines[2], en, mixed_); else launch_k(k_fft_z_solve<R, true, false>, gz, 128, sz, stream_, A, P.h.p, P.gt.p, P.wt.p, P.plan[2][0], P.plan[2][1], P.lines[2], en, mixed_); }
  else { if (vir) launch_k(k_fft_z_solve<R, false, true>, gz, 128, sz, stream_, A, P.h.p, P.gt.p, P.wt.p, P.plan[2][0], P.plan[2][1], P.lines[2], en, mixed_); else launch_k(k_fft_z_solve<R, false, false>, gz, 128, sz, stream_, A, P.h.p, P.gt.p, P.wt.p, P.plan[2][0], P.plan[2][1], P.lines[2], en, mixed_); }
  launch_k(k_fft_y<R>, gy, 128, sy, stream_, A, P.h.p, P.plan[1][1], P.lines[1]);
  launch_k(k_fft_x_inv<R>, capped(blocks_for(size_t(nlx), P.lines[0])), 128, sx, stream_, A, P.h.p, P.gr.p, P.plan[0][1], P.lines[0]);
}

// Autotuner for the line transforms: every block shape that fits (x: 1-16 lines per block; y, z: 1-8 consecutive a per
// block) is timed on this grid (the transforms' time does not depend on the values), and the fastest kept. Results are
// cached per grid, precision and SM count for the process.
template <class R>
void Engine::pme_tune(PmePath<R>& P) {
  using T = typename Cpx<R>::T;
  static std::mutex mu;
  static std::map<std::array<int, 5>, std::array<int, 3>> cache;
  const std::array<int, 5> key{pk_[0], pk_[1], pk_[2], int(sizeof(R)), dev_sms_};
  {
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(key);
    if (it != cache.end()) {
      P.lines[0] = it->second[0], P.lines[1] = it->second[1], P.lines[2] = it->second[2];
      return;
    }
  }
  const size_t half = size_t(ph1_) * pk_[1] * pk_[2];
  CK(cudaMemsetAsync(P.gt.p, 0, half * sizeof(R), stream_));
  CK(cudaMemsetAsync(P.wt.p, 0, 6 * half * sizeof(R), stream_));
  CK(cudaMemsetAsync(P.h.p, 0, half * sizeof(T), stream_));
  if (mixed_) CK(cudaMemsetAsync(d_gridq_.p, 0, d_gridq_.n * sizeof(long long), stream_));
  else CK(cudaMemsetAsync(d_grid_.p, 0, d_grid_.n * sizeof(double), stream_));
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  const size_t smax = 48 * 1024;
  float best = 1e30f;
  std::array<int, 3> pick{P.lines[0], P.lines[1], P.lines[2]};
  for (int lx : {1, 2, 4, 8, 16})
    for (int la : {1, 2, 4, 8}) {
      if ((size_t(lx) * 2 + 1) * pk_[0] * sizeof(T) > smax) continue;
      const int ly = std::min(la, ph1_), lz = std::min(la, ph1_);
      if ((size_t(ly) * 2 + 1) * pk_[1] * sizeof(T) > smax || (size_t(lz) + 1) * 2 * pk_[2] * sizeof(T) > smax) continue;
      P.lines[0] = lx, P.lines[1] = ly, P.lines[2] = lz;
      fft_passes(P, false, false);   // warm
      CK(cudaEventRecord(e0, stream_));
      for (int rep = 0; rep < 3; ++rep) fft_passes(P, false, false);
      CK(cudaEventRecord(e1, stream_));
      CK(cudaEventSynchronize(e1));
      float ms = 0;
      CK(cudaEventElapsedTime(&ms, e0, e1));
      if (ms < best) best = ms, pick = {lx, ly, lz};
    }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  P.lines[0] = pick[0], P.lines[1] = pick[1], P.lines[2] = pick[2];
  std::lock_guard<std::mutex> lock(mu);
  cache[key] = pick;
}

template <class R>
void Engine::pme_run(PmePath<R>& P, const double* d_x, bool ener, bool vir) {
  using T = typename Cpx<R>::T;
  PmeArgs A{pk_[0], pk_[1], pk_[2], ph1_, dcell_, d_x, d_q_.p, n_};
  if (!green_valid_ || std::memcmp(green_cell_, cell_h_, sizeof cell_h_) != 0) {
    const size_t half = size_t(ph1_) * pk_[1] * pk_[2];
    launch_k(k_pme_green<R>, blocks_for(half, 256), 256, 0, stream_, A, d_bsp_[0].p, d_bsp_[1].p, d_bsp_[2].p, beta_, kCoulomb, P.gt.p, P.wt.p);
    std::memcpy(green_cell_, cell_h_, sizeof cell_h_);
    green_valid_ = true;
  }
  const int nb = blocks_for(size_t(n_), 128);
  if (mixed_) CK(cudaMemsetAsync(d_gridq_.p, 0, d_gridq_.n * sizeof(long long), stream_));
  else CK(cudaMemsetAsync(d_grid_.p, 0, d_grid_.n * sizeof(double), stream_));
#define SPREAD(P_)                                                                            \
  do {                                                                                        \
    if (mixed_) launch_k(k_spread<float, P_>, nb, 128, 0, stream_, A, d_grid_.p, d_gridq_.p);      \
    else launch_k(k_spread<double, P_>, nb, 128, 0, stream_, A, d_grid_.p, d_gridq_.p);            \
  } while (0)
  switch (order_) {
    case 3: SPREAD(3); break;
    case 4: SPREAD(4); break;
    case 5: SPREAD(5); break;
    case 6: SPREAD(6); break;
    case 7: SPREAD(7); break;
    default: SPREAD(8); break;
  }
#undef SPREAD
  fft_passes(P, ener, vir);
  const ForceSink<float> Ff{d_F_.p, d_F_.p + n_, d_F_.p + 2 * size_t(n_), d_counters_.p + kCntErr};
  const ForceSink<double> Fd{d_Fd_.p, d_Fd_.p + n_, d_Fd_.p + 2 * size_t(n_)};
#define GATHER(P_)                                                                            \
  do {                                                                                        \
    if (mixed_) launch_k(k_gather<float, R, P_>, nb, 128, 0, stream_, A, P.gr.p, Ff);              \
    else launch_k(k_gather<double, R, P_>, nb, 128, 0, stream_, A, P.gr.p, Fd);                     \
  } while (0)
  switch (order_) {
    case 3: GATHER(3); break;
    case 4: GATHER(4); break;
    case 5: GATHER(5); break;
    case 6: GATHER(6); break;
    case 7: GATHER(7); break;
    default: GATHER(8); break;
  }
#undef GATHER
  CK(cudaGetLastError());
}

void Engine::pme_forces(const double* d_x, bool ener, bool vir) {
  if (mixed_) pme_run(pf_, d_x, ener, vir);
  else pme_run(pd_, d_x, ener, vir);
}


template void Engine::pme_setup<double>(PmePath<double>&);
template void Engine::pme_run<double>(PmePath<double>&, const double*, bool, bool);
template void Engine::fft_passes<double>(PmePath<double>&, bool, bool);
template void Engine::pme_tune<double>(PmePath<double>&);
template void Engine::pme_setup<float>(PmePath<float>&);
template void Engine::pme_run<float>(PmePath<float>&, const double*, bool, bool);
template void Engine::fft_passes<float>(PmePath<float>&, bool, bool);
template void Engine::pme_tune<float>(PmePath<float>&);

}  // namespace capsb
