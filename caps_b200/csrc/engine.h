// The device engine behind include/caps_gpu.h: owns the force field on the device, the cluster pair list, the PME
// grids and the MD state, and runs Evaluator::compute and run_dynamics for one system on one GPU.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <cstdint>
#include <functional>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "caps_gpu.h"
#include "common.cuh"
#include "list_types.cuh"
#include "pme_types.cuh"

namespace capsb {

struct PairArgs;
struct Stepper;
struct StepperDeleter {
  void operator()(Stepper* s) const;   // integrate.cu
};

inline int blocks_for(size_t n, int threads) { return int(std::max<size_t>(1, (n + size_t(threads) - 1) / size_t(threads))); }

// Bumped whenever any device buffer of the library is allocated or freed. A captured CUDA graph holds buffer addresses,
// so a run that finds this count unchanged since its step graph was captured (with everything else that shaped the
// capture) may replay that graph instead of capturing it again.
inline std::atomic<unsigned long long> g_buffer_epoch{0};

template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) {
      cudaFree(p);
      g_buffer_epoch.fetch_add(1, std::memory_order_relaxed);
    }
    p = nullptr;
    n = 0;
  }
  void alloc(size_t count);        // throws on failure; keeps the buffer when large enough
  void upload(const T* h, size_t count, cudaStream_t s);
  void upload(const std::vector<T>& h, cudaStream_t s) { upload(h.data(), h.size(), s); }
  void zero(cudaStream_t s);
};

struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

// Every CUDA runtime call of the host engine goes through CK: a failure becomes a CudaError with the call's text.
#define CK(call)                                                                                         \
  do {                                                                                                   \
    cudaError_t e_ = (call);                                                                             \
    if (e_ != cudaSuccess) throw CudaError(std::string(#call) + ": " + cudaGetErrorString(e_));          \
  } while (0)

template <class T>
void DevBuf<T>::alloc(size_t count) {
  if (count <= n && p) return;
  release();
  if (count == 0) count = 1;
  const cudaError_t e = cudaMalloc(&p, count * sizeof(T));
  if (e != cudaSuccess) {
    p = nullptr;
    throw CudaError(std::string("cudaMalloc: ") + cudaGetErrorString(e));
  }
  n = count;
  g_buffer_epoch.fetch_add(1, std::memory_order_relaxed);
}
template <class T>
void DevBuf<T>::upload(const T* h, size_t count, cudaStream_t s) {
  alloc(count);
  if (!count) return;
  const cudaError_t e = cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) throw CudaError(std::string("cudaMemcpyAsync: ") + cudaGetErrorString(e));
}
template <class T>
void DevBuf<T>::zero(cudaStream_t s) {
  if (!p) return;
  const cudaError_t e = cudaMemsetAsync(p, 0, n * sizeof(T), s);
  if (e != cudaSuccess) throw CudaError(std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
}
// Launches a kernel on a stream and turns a launch error into an exception. Arguments convert to the kernel's parameter
// types.
template <class... KP, class... A>
void launch_k(void (*kernel)(KP...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream, A&&... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  const cudaError_t e = cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...);
  if (e != cudaSuccess) throw CudaError(std::string("kernel launch: ") + cudaGetErrorString(e));
}

struct ModelError : std::runtime_error {   // the reference's FieldError and argument errors
  int code;
  ModelError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

// PME plans and buffers of one precision.
template <class R>
struct PmePath {
  using T = typename Cpx<R>::T;
  DevBuf<T> h;          // half spectrum
  DevBuf<R> gr;         // real grid after the inverse transform
  DevBuf<R> gt, wt;     // influence function, virial weights
  DevBuf<T> tw[3][2];   // twiddles per axis: forward, inverse
  FftPlan<R> plan[3][2];
  int k[3] = {0, 0, 0};      // the grid these were set up for
  int lines[3] = {1, 1, 1};  // line-transform block shapes (x lines per block; y, z consecutive a per block), tuned
};

class Engine {
 public:
  Engine(const caps_gpu_ff* ff, const caps_gpu_opts* o);
  ~Engine();
  void set_options(const caps_gpu_opts* o);
  void energies(bool on) { energies_ = on; }
  // compute on host arrays (copies in and out) or on device arrays
  void compute_host(const double* x, const double* cell, double* f, caps_gpu_terms* out);
  void compute_dev(const double* d_x, const double* cell, double* d_f, caps_gpu_terms* out);
  int list_builds();   // list builds so far (counted on the device)
  void list_counts(int64_t* v);   // v[0] list builds, v[1] dynamic prunes so far
  // Evaluator::freeze_pairs / unfreeze (field.hpp:341-347): later evaluations take exactly the pairs inside the cut-off
  // at (x, cell), on the FP64 path, and never rebuild the list
  void freeze_pairs(const double* x, const double* cell);
  void unfreeze();
  bool frozen() const { return frozen_; }
  // Evaluator::pairs() (field.hpp:348): atom pairs in the FP64 pair list (within r_c + skin at its last build)
  long long pairs();
  bool energies_on() const { return energies_; }
  int64_t timing_flush() const { return timing_flush_; }
  int sms() const { return dev_sms_; }
  void run(caps_gpu_state* st, const caps_gpu_md_opts* md, caps_gpu_progress_fn progress, caps_gpu_frame_fn frame, void* user, std::string* report);
  void validate_md(const caps_gpu_md_opts& o) const;   // the dynamics options the device path takes (throws otherwise)
  double last_steps_per_second() const { return last_sps_; }
  // measurement support (include/caps_gpu_diag.h)
  void set_timing(int64_t flush_bytes) { timing_flush_ = flush_bytes; }
  void time_pair_kernel(const double* x, const double* cell, int launches, int64_t flush_bytes, double* avg_ms, double* pairs_in,
                        double* pairs_listed, double* entries);
  void time_phases(const double* x, const double* cell, int launches, int64_t flush_bytes, double* ms);
  double last_step_ms_device() const { return last_step_ms_; }
  int graph_kernels() const { return graph_kernels_; }
  // the tuned launch shapes: j-tile depth, pair-grid cut, PME grid cap, bonded cap, PME line blocks x, y, z
  void tuning(int32_t v[7]) const;
  void pin_tuning(const int32_t v[7]);   // these shapes from now on, no tuning (profiling runs)
  long long kernels_run() const { return kernels_run_; }
  std::string err;
  // Host state that shapes a captured step graph besides the run's own options: the buffer epoch, the options, the
  // cell, the list and PME set-up and the flags forces() reads while it is captured. Two captures made with the same
  // state (and the same run options) record the same graph.
  std::string capture_state() const;
  void drop_run_state();   // the MD state kept between runs is set up again at the next run

  // --- internals used by the step kernels' launcher (integrate.cu) ---
  int n_ = 0, nt_ = 0;
  bool mixed_ = true;
  caps_gpu_opts opt_{};
  cudaStream_t stream_ = nullptr;

 private:
  friend struct Stepper;
  friend struct MdRun;
  friend void run_batch(const std::vector<Engine*>&, caps_gpu_state* const*, const caps_gpu_md_opts* const*, caps_gpu_progress_fn,
                        caps_gpu_frame_fn, void* const*);
  void setup_ff(const caps_gpu_ff* ff);
  void setup_options();
  void set_cell(const double* cell);
  void ensure_list_capacity();
  void grow_list(size_t ent, size_t mk);
  bool grow_list_for_run();
  // One force evaluation up to the AoS doubles d_out (d_f_ by default), async. parts: a mask of 1 bonded, 2 short-range
  // non-bonded, 4 long-range (PME) terms (-1: the options' parts); clear_energies = false adds this evaluation's
  // energies and virial to the previous one's.
  // reduce = false leaves the forces in the fixed-point (or FP64) sums, for a kick that reads them itself
  void forces(const double* d_x, bool ener, bool vir, bool check_rebuild, int parts = -1, double* d_out = nullptr, bool clear_energies = true,
              bool reduce = true);
  // Concurrent branches of a force evaluation: `launch` runs with stream_ pointing at side stream k, after everything
  // queued on the main stream so far; join(k) makes the main stream wait for it. Captured, these are graph branches.
  void fork(int k, const std::function<void()>& launch);
  void join(int k);
  cudaStream_t side_[2] = {nullptr, nullptr};
  int counter(int slot);   // a device counter (synchronises the stream)
  // Autotuning (timed on this system and GPU, once): the j-tile depth of the pair kernels' work items, and the PME
  // line-transform block shapes per grid.
  int batch_ = kBatch;
  int pair_cut_ = 0;   // the pair kernel's persistent grid leaves this many block slots per SM to the other branches
  int pme_cap_ = 0;    // at most this many blocks per PME line-transform launch (0: one per line group)
  int bonded_cap_ = 0; // at most this many blocks per bonded term kind (0: four per SM)
  bool tuning_pinned_ = false;
  int pinned_lines_[3] = {1, 1, 1};
  bool sums_cleared_ = false;   // the atom-order force sums were cleared by the integrator's kick (the next forces() skips it)
  bool batch_tuned_ = false;
  void tune_batch(const double* d_x);
  template <class R> void fft_passes(PmePath<R>& P, bool ener, bool vir);
  template <class R> void pme_tune(PmePath<R>& P);
  cudaEvent_t ev_fork_ = nullptr, ev_join_[2] = {nullptr, nullptr};
  void read_terms(caps_gpu_terms* out, bool ener, bool vir);
  void check_errors();
  void launch_build(const double* d_x);
  // the displacement check's arguments (SHAKE's launch: with the atoms in no constraint cluster), and whether a step may
  // fold the check into its own kernels: a non-bonded evaluation with a valid list that is not frozen
  ListCheck list_check(int nfree, const int* free_atoms) const;
  bool list_check_fusable() const;
  void pme_forces(const double* d_x, bool ener, bool vir);
  template <class R> void pme_setup(PmePath<R>& P);
  template <class R> void pme_run(PmePath<R>& P, const double* d_x, bool ener, bool vir);
  void pair_forces(bool ener, bool vir);
  PairArgs pair_args();
  void prune(const double* d_x);
  void bonded_forces(const double* d_x, bool ener, bool vir, int parts);
  void host_constants(caps_gpu_terms* t, bool ener, bool vir) const;

  // force field (device)
  DevBuf<int> d_type_;
  DevBuf<double> d_q_, d_mass_;
  std::vector<int> h_type_;
  std::vector<double> h_q_, h_mass_, h_eps_, h_sig_;   // per type pair
  std::vector<double> type_count_;
  std::vector<std::array<uint32_t, 2>> hb_;   // bonds (harmonic, then FENE) and their r0 (0: none), for constraints
  std::vector<double> hr0_;
  std::vector<std::array<uint32_t, 3>> ha_;   // angles and theta0, for rigid waters
  std::vector<double> hth0_;
  DevBuf<float4> d_tab_;
  DevBuf<float2> d_ljf_;   // per type (sqrt c6, sqrt c12), the padding type last
  bool comb_ = false;      // the pair coefficients factor per type (geometric mixing, 12-6)
  DevBuf<double4> d_tabd_, d_lj14_, d_tabcap_, d_cap14_;
  // ForceField::pair_func on the FP64 path: per type pair the form (0 LJ) and its parameters, the pair's own cut-off
  // squared; tables of (a, b, c, rc^2) beside the LJ tables (their .w holds the form)
  std::vector<int> h_form_;
  std::vector<double> h_pa_, h_pb_, h_pc_, h_prc2_;
  bool generic_ = false;
  DevBuf<double4> d_tabg_, d_lj14g_, d_tabg2_, d_lj14g2_;
  double lj_inner_ = 0;
  bool lj_fsw_ = false;   // CHARMM's force switch on every 12-6 pair (FP64 path)
  DevBuf<int> d_toff_;
  DevBuf<double> d_tr0dr_, d_te_, d_tf_;
  std::vector<int> h_toff_;   // the tabulated pairs on the host (shift and bounds)
  std::vector<double> h_tr0dr_, h_te_, h_tf_;
  PairTables pair_tables() const { return PairTables{d_toff_.p, d_tr0dr_.p, d_te_.p, d_tf_.p}; }
  DevBuf<double> d_gtab_;
  int gnodes_ = 0;
  double ghi_ = 0;
  DevBuf<uint32_t> d_bond_ij_, d_angle_ijk_, d_dih_ijkl_, d_imp_ijkl_, d_p14_ij_, d_excl_ij_, d_fene_ij_;
  DevBuf<double> d_bond_kr_, d_angle_kt_, d_dih_vd_, d_imp_vd_, d_p14_scale_, d_fene_p_;
  std::vector<double> h_fene_r0_;   // R0 of each FENE bond, for the overstretch message
  DevBuf<double> d_errinfo_;        // error details left by the kernels (ErrInfo)
  DevBuf<int> d_dih_n_, d_imp_n_, d_dih_grp_, d_imp_grp_;
  DevBuf<double> d_excl_f_;
  DevBuf<uint32_t> d_excl_off_, d_excl_list_;
  int nb_ = 0, na_ = 0, nd_ = 0, ndg_ = 0, ni_ = 0, nig_ = 0, np14_ = 0, nx_ = 0, nfene_ = 0;
  double lj14_ = 0.5;
  bool p14_scaled_ = false;
  bool lj_shift_model_ = false;
  bool lj96_ = false;   // class II 9-6 pair form (ForceField::pair_form "lj9-6")
  double model_cutoff_ = 0;

  // options derived
  double rc_ = 10, skin_ = 2, beta_ = 0, kappa_ = 0, dsf_e0_ = 0, dsf_f0_ = 0, erfc_rc_ = 0;
  bool pme_ = false, coul_ = true, tail_ = true, shifted_ = false;
  int order_ = 4;
  bool energies_ = true;

  // cell and list
  double cell_h_[12] = {0};
  bool cell_set_ = false;
  DevCell dcell_{};
  ListGeom geom_{};
  ListBufs lb_{};
  DevBuf<int> d_col_, d_ioff_, d_order_, d_iperm_, d_col_count_, d_col_fill_, d_col_start_, d_col_sc_, d_sc_col_, d_perm_, d_counters_;
  DevBuf<double> d_frac_, d_sc_z_, d_sc_org_, d_cl_box_, d_x0_, d_xp_;
  DevBuf<unsigned char> d_cl_real_;
  DevBuf<uint4> d_ent_;
  DevBuf<float4> d_ent_shift_;
  DevBuf<unsigned long long> d_masks_;
  DevBuf<int4> d_work_;
  bool list_valid_ = false;
  // a frozen pair set: per entry and i cluster, the 64 atom pairs that interact; the precision to restore at unfreeze
  bool frozen_ = false;
  int frozen_saved_precision_ = -1;
  DevBuf<unsigned long long> d_frozen_;
  long long frozen_pairs_ = 0;   // pairs() as the reference reports it on its cluster path: the list of the last freeze
  long long count_pairs();
  int nsc_cap_ = 0;

  // packed positions, forces
  DevBuf<float4> d_xq_;
  DevBuf<double4> d_xqd_;
  DevBuf<int> d_tslot_;
  DevBuf<long long> d_F_, d_Fs_;    // fixed point, SoA: atom order (3 n), slot order (3 nslots)
  DevBuf<double> d_Fd_, d_Fsd_;     // FP64 path
  DevBuf<long long> d_efix_;
  DevBuf<double> d_edbl_;
  DevBuf<double> d_x_, d_f_;        // host-call staging: positions in, forces out (3 n AoS)
  int* h_counters_ = nullptr;       // pinned
  long long* h_efix_ = nullptr;     // pinned
  double* h_edbl_ = nullptr;        // pinned

  // PME
  int pk_[3] = {0, 0, 0}, ph1_ = 0;
  DevBuf<double> d_bsp_[3];
  DevBuf<double> d_grid_;           // FP64 spread grid
  DevBuf<long long> d_gridq_;       // FP32 path: fixed-point spread grid
  PmePath<double> pd_;              // FP64 transforms: the FP64 path
  PmePath<float> pf_;               // FP32 transforms: the mixed path
  double green_cell_[12] = {0};
  bool green_valid_ = false;        // the active path's influence function matches cell_h_
  void ensure_pme();                // the active path's plans, buffers and block shapes for the current grid
  const int* pme_lines() const { return mixed_ ? pf_.lines : pd_.lines; }

  double last_sps_ = 0, last_step_ms_ = 0;
  int64_t timing_flush_ = -1;
  int graph_kernels_ = 0;
  long long kernels_run_ = 0;
  DevBuf<unsigned char> d_flush_;
  int dev_sms_ = 148;
  // The MD state kept between runs (integrate.cu): state and work buffers, pinned scalars, the constraint clusters and
  // the instantiated step graphs, so that a run on the same engine pays none of their set-up again.
  std::unique_ptr<Stepper, StepperDeleter> stepper_;
};

// Independent replicas (one engine each, on the current device) advanced in lock step; integrate.cu.
void run_batch(const std::vector<Engine*>& es, caps_gpu_state* const* states, const caps_gpu_md_opts* const* mds, caps_gpu_progress_fn progress,
               caps_gpu_frame_fn frame, void* const* users);

}  // namespace capsb
