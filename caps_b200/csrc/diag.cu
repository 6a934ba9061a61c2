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
  for (int k = 0; k < launches; ++k) {
    if (flush_bytes > 0) cudaMemsetAsync(d_flush_.p, k & 255, size_t(flush_bytes), stream_);
    if (mixed_) cudaMemsetAsync(d_Fs_.p, 0, d_Fs_.n * sizeof(long long), stream_);
    else cudaMemsetAsync(d_Fsd_.p, 0, d_Fsd_.n * sizeof(double), stream_);
    cudaMemsetAsync(d_counters_.p + kCntPairNext, 0, sizeof(int), stream_);   // the pack kernel resets it in a force evaluation
    cudaEventRecord(ev[size_t(2 * k)], stream_);
    pair_forces(false, false);
    cudaEventRecord(ev[size_t(2 * k + 1)], stream_);
  }
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

}  // namespace capsb

