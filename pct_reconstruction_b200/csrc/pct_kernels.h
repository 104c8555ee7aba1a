// pct_kernels.h -- host-callable launchers of the engine's kernels.
#pragma once

#include "pct_common.cuh"
#include "pct_tables.h"

namespace pct {

// Streaming-multiprocessor count of the current device (cached after the first call).
int sm_count();

// Per-step MLP table entries 0..kmax on the device (entry 0 zero).
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

// image_update_GPU (B.cu:9398): x[v] += acc[v].x / acc[v].y where acc[v].y > 0, then acc[v] = 0.
cudaError_t launch_image_update(float* x, float2* acc, int num_voxels, cudaStream_t stream);

}  // namespace pct
