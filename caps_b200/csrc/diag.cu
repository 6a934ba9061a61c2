// Measurement entry points (include/caps_gpu_diag.h): per-step event timing of runs and the pair kernel's launch time.
#include <vector>

#include "caps_gpu_diag.h"
#include "engine.h"

namespace capsb {

void Engine::time_pair_kernel(const double* x, const double* cell, int launches, int64_t flush_bytes, double* avg_ms, double* pairs_in,
                              double* pairs_listed, double* entries) {
  caps_gpu_terms t{};
  std::vector<double> f(size_t(3) * n_);
  compute_host(x, cell, f.data(), &t);
  const double pin = mixed_ ? double(h_efix_[kEPairs]) * kInvFixE : 0.0;
  const double pl = mixed_ ? double(h_efix_[kEListed]) * kInvFixE : 0.0;
  if (pairs_in) *pairs_in = pin;
  if (pairs_listed) *pairs_listed = pl;
  if (entries) *entries = double(h_counters_[kCntEnt]);
  if (flush_bytes > 0) d_flush_.alloc(size_t(flush_bytes));
  std::vector<cudaEvent_t> ev(size_t(2 * launches));
  for (auto& e : ev) {
    if (cudaEventCreate(&e) != cudaSuccess) throw CudaError("cudaEventCreate");
  }
  // the kernel alone: its full persistent grid, whatever share of the SMs the tuner leaves it inside a step
  const int cut = pair_cut_;
  pair_cut_ = 0;
  for (int k = 0; k < launches; ++k) {
    if (flush_bytes > 0) cudaMemsetAsync(d_flush_.p, k & 255, size_t(flush_bytes), stream_);
    if (mixed_) cudaMemsetAsync(d_Fs_.p, 0, d_Fs_.n * sizeof(long long), stream_);
    else cudaMemsetAsync(d_Fsd_.p, 0, d_Fsd_.n * sizeof(double), stream_);
    cudaMemsetAsync(d_counters_.p + kCntPairNext, 0, sizeof(int), stream_);   // the pack kernel resets it in a force evaluation
    cudaEventRecord(ev[size_t(2 * k)], stream_);
    pair_forces(false, false);
    cudaEventRecord(ev[size_t(2 * k + 1)], stream_);
  }
  pair_cut_ = cut;
  if (cudaStreamSynchronize(stream_) != cudaSuccess) throw CudaError("pair timing: stream failed");
  double sum = 0;
  for (int k = 0; k < launches; ++k) {
    float ms = 0;
    cudaEventElapsedTime(&ms, ev[size_t(2 * k)], ev[size_t(2 * k + 1)]);
    sum += ms;
  }
  for (auto& e : ev) cudaEventDestroy(e);
  if (avg_ms) *avg_ms = launches > 0 ? sum / launches : 0.0;
}

// The force evaluation's branches timed one at a time, then together (force-only, as on a plain MD step; the list is
// built once first and kept): ms[0] the bonded branch (bonded terms, 1-4 pairs, excluded-pair corrections), ms[1] PME,
// ms[2] the short-range evaluation (displacement check, pack, prune check, pair kernel, and its 1-4 branch), ms[3] the
// whole evaluation. Each is the mean over `launches` repetitions, CUDA events on the engine's stream, an L2 flush of
// flush_bytes before each.
void Engine::time_phases(const double* x, const double* cell, int launches, int64_t flush_bytes, double* ms) {
  caps_gpu_terms t{};
  std::vector<double> f(size_t(3) * n_);
  compute_host(x, cell, f.data(), &t);
  if (flush_bytes > 0) d_flush_.alloc(size_t(flush_bytes));
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  for (int ph = 0; ph < 4; ++ph) {
    double sum = 0;
    for (int k = 0; k < launches; ++k) {
      if (flush_bytes > 0) CK(cudaMemsetAsync(d_flush_.p, k & 255, size_t(flush_bytes), stream_));
      CK(cudaEventRecord(e0, stream_));
      if (ph == 0) bonded_forces(d_x_.p, false, false, 7);
      else if (ph == 1) {
        if (pme_) pme_forces(d_x_.p, false, false);
      } else if (ph == 2) forces(d_x_.p, false, false, true, 2);
      else forces(d_x_.p, false, false, true);
      CK(cudaEventRecord(e1, stream_));
      CK(cudaEventSynchronize(e1));
      float m = 0;
      CK(cudaEventElapsedTime(&m, e0, e1));
      sum += m;
    }
    ms[ph] = launches > 0 ? sum / launches : 0.0;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  check_errors();
}

}  // namespace capsb

