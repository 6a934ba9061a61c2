/* caps_gpu_diag.h — measurement entry points of the B200 engine for the benchmark harness and profiling.
 * These have no counterpart in the reference (it publishes its timings from std::chrono around the step loop,
 * core/src/dynamics.cpp:776-778); they sit beside the drop-in boundary of caps_gpu.h and change no result. */
#ifndef CAPS_GPU_DIAG_H
#define CAPS_GPU_DIAG_H
#include <stdint.h>
#include "caps_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Measurement mode for caps_gpu_run: flush_bytes >= 0 brackets every MD step with a CUDA event pair on the engine's
 * stream and, when > 0, writes flush_bytes (larger than the 126 MB L2) between steps, outside the events; < 0 turns it
 * off. caps_gpu_last_steps_per_second then reports K / (sum of the per-step event times). */
int32_t caps_gpu_diag_set_timing(caps_gpu_engine* e, int64_t flush_bytes);
/* The launch shapes the engine's tuners chose (v[7]: entries per work item, pair-grid blocks per SM left free, PME
 * line-transform grid cap, bonded blocks per term kind, PME line blocks along x, y, z; a cap of 0 means none), and
 * the same shapes pinned on an engine, which then tunes nothing: a profiler, which slows the kernels it replays and
 * so misleads the tuners, can see the shapes of a plain run. */
int32_t caps_gpu_diag_get_tuning(const caps_gpu_engine* e, int32_t* v);
int32_t caps_gpu_diag_set_tuning(caps_gpu_engine* e, const int32_t* v);
/* Device milliseconds per MD step of the last run (the per-step events in measurement mode). */
double caps_gpu_diag_last_step_ms(const caps_gpu_engine* e);
/* Kernel launches in one plain MD step of the last run (the kernel nodes of its captured CUDA graph; the list-build and
 * prune kernels among them return at once on steps that do not need them). */
int32_t caps_gpu_diag_step_kernels(const caps_gpu_engine* e);
/* Kernels the last caps_gpu_run launched in its step loop: per step the kernel nodes of the step graph it replayed, plus
 * the kinetic-energy kernel of each thermo row; a barostat step (run outside a graph) counts as one thermo step. */
int64_t caps_gpu_diag_kernels_run(const caps_gpu_engine* e);
/* List builds and dynamic prunes the engine has run so far (counted on the device; v[0] builds, v[1] prunes). */
int32_t caps_gpu_diag_list_counts(caps_gpu_engine* e, int64_t* v);
/* Times the non-bonded pair kernel alone: one force evaluation at x (host, 3N) builds the list, then `launches`
 * launches of the pair kernel (forces only, its full persistent grid), each bracketed by CUDA events, an L2 flush of
 * flush_bytes before each.
 * avg_ms: mean launch time; pairs_in: atom pairs inside the cut-off per launch; pairs_listed: atom pairs the kernel
 * evaluates (list pairs, masked lanes excluded); entries: cluster-pair entries (FP32 path only; 0 on FP64). */
int32_t caps_gpu_diag_pair_timing(caps_gpu_engine* e, const double* x, const double* cell, int32_t launches, int64_t flush_bytes, double* avg_ms,
                                  double* pairs_in, double* pairs_listed, double* entries);

/* The force evaluation's concurrent branches timed one at a time and together (force-only, on the list built at x):
 * ms[0] the bonded branch (bonded terms, 1-4 pairs, excluded-pair corrections), ms[1] PME, ms[2] the short-range branch
 * (displacement check, pack, prune check, pair kernel), ms[3] the whole evaluation; means over `launches` repetitions,
 * CUDA events, an L2 flush of flush_bytes before each. */
int32_t caps_gpu_diag_phase_timing(caps_gpu_engine* e, const double* x, const double* cell, int32_t launches, int64_t flush_bytes, double* ms);

#ifdef __cplusplus
}
#endif
#endif /* CAPS_GPU_DIAG_H */
