// pct_kernels.h -- host-callable launchers of the engine's kernels.
#pragma once

#include "pct_common.cuh"
#include "pct_tables.h"

namespace pct {

// Streaming-multiprocessor count of the current device (cached after the first call).
int sm_count();

// One shared-memory carve-out for every kernel a captured DROP iteration runs concurrently (path
// kernels, DROP block kernels, image updates), set on the current device.  An SM runs CTAs of
// kernels with different carve-outs only after it has drained and been reconfigured, so the block
// chain's small kernels, interleaved with path-kernel chunks that keep 16 KB of shared memory per
// CTA, would otherwise wait for whole SMs to empty.
cudaError_t set_iteration_carveout();
cudaError_t set_image_update_carveout(int percent);

// Per-step MLP table entries 0..kmax on the device (entry 0 zero).
// The S-curve table s(k), k < kSCurveEntries, of configuration c (pct_scurve.cu).
cudaError_t launch_s_curve_table(const pct_config& c, float* out, cudaStream_t stream);
cudaError_t launch_build_step_table(const Tables& tab, unsigned sstep, unsigned pstep, int kmax, StepConst* steps,
                                    cudaStream_t stream);

// MLP + DROP scatter for histories [begin, begin+count) (exact mode).
cudaError_t launch_drop_block_exact(const Geometry& g, const Tables& tab, const StepConst* steps, int kmax,
                                    const float* x, float2* acc, const HistorySoA& h, long long begin,
                                    long long count, unsigned long long* counters, cudaStream_t stream);

// MLP voxel lists for parity checks (exact mode).
cudaError_t launch_mlp_paths_exact(const Geometry& g, const Tables& tab, const StepConst* steps, int kmax,
                                   const float* x, const HistorySoA& h, long long begin, long long count, int stride,
                                   uint32_t* counts, uint32_t* voxels, double* chord, double* a_dot_x,
                                   unsigned long long* counters, cudaStream_t stream);

// Loop trips (MLP points) of the exact walk of histories [begin, begin+count).
cudaError_t launch_mlp_steps(const Geometry& g, const Tables& tab, int kmax, const HistorySoA& h, long long begin,
                             long long count, int* steps, cudaStream_t stream);

// Two-phase DROP iteration (see pct_drop_exact.cu).
cudaError_t launch_path_bounds(const Geometry& g, const Tables& tab, const HistorySoA& h, long long n,
                               long long block_size, int histories_per_block, int* bounds, cudaStream_t stream);
// dst[p] = src[perm[p]] for the path kernel's inputs (the ten geometry fields and the first voxel),
// the path bounds and the path-storage offsets, p in [0, n).
cudaError_t launch_gather_path_inputs(const HistorySoA& src, const int* perm, const int* bounds,
                                      const long long* offsets, long long n, const HistorySoA& dst, int* bounds_sorted,
                                      long long* offsets_sorted, cudaStream_t stream);
// The path kernel over `count` histories in processing order: h, bounds and offsets hold its
// inputs in that order (from launch_gather_path_inputs, offset to the chunk), perm the history
// each position stands for (its path length and chord are written there).
cudaError_t launch_mlp_phase1_exact(const Geometry& g, const Tables& tab, const StepConst* steps, int kmax,
                                    const HistorySoA& h, const int* perm, long long count, const long long* offsets,
                                    long long offset_base, const int* bounds, uint32_t* paths, int* path_n,
                                    double* chord, unsigned long long* counters, cudaStream_t stream);
// Exact vs mixed-precision MLP points of histories [begin, begin+count): per history the largest
// deviations of t and v (cm) and the number of steps whose voxel differs, over the steps with a
// positive Sigma_2 determinant; ill_posed counts the other steps.
cudaError_t launch_mlp_precision(const Geometry& g, const Tables& tab, const StepConst* steps, int kmax,
                                 const HistorySoA& h, long long begin, long long count, double* dev_t, double* dev_v,
                                 int* mismatched, int* ill_posed, cudaStream_t stream);
cudaError_t launch_drop_phase2(const Geometry& g, const float* x, float2* acc, float* normA, const FixedAcc& fx,
                               const float* WEPL,
                               const long long* offsets, long long offset_base, const uint32_t* paths,
                               const int* path_n, const double* chord, long long begin, long long count,
                               cudaStream_t stream, bool pdl = false);

// Prefix sum of int32 values into int64 offsets (n+1 entries); tile_scratch holds
// scan_tile_scratch_elems(n) int64.
cudaError_t exclusive_scan_i32_to_i64(const int* values, long long n, long long* offsets, long long* tile_scratch,
                                      cudaStream_t stream);
long long scan_tile_scratch_elems(long long n);
// perm[0..n) = indices begin..begin+n ordered by descending key (key < max_key); hist_scratch
// holds 2*max_key unsigned.
// Counting sort of each window of `window` consecutive indices by descending key (one CTA each).
cudaError_t window_sort_by_key(const int* key, long long begin, long long n, int max_key, int window, int* perm,
                               cudaStream_t stream);
cudaError_t bucket_sort_by_key(const int* key, long long begin, long long n, int max_key, unsigned* hist_scratch,
                               int* perm, cudaStream_t stream);

// image_update_GPU (B.cu:9398): x[v] += acc[v].x / acc[v].y where acc[v].y > 0, then acc[v] = 0.
// Image update after a DROP block (normA: the ROBUSTB accumulator, else unused).
cudaError_t launch_image_update(const Geometry& g, float* x, float2* acc, float* normA, const FixedAcc& fx,
                                cudaStream_t stream, bool pdl = false);

// Read-only view of a context's device state, for entry points implemented outside
// pct_context.cu.
struct ContextView {
    Geometry geo;
    Tables tables;
    const StepConst* steps;
    int kmax;
    int device;
    cudaStream_t stream;
    unsigned long long* counters;
};
bool context_view(pct_ctx* ctx, ContextView* v);
void context_count_launches(pct_ctx* ctx, long long n);
void context_set_error(pct_ctx* ctx, const char* msg);

}  // namespace pct
