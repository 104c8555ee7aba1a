// pct_image.cu -- per-block image update of DROP.
//
// image_update_GPU (B.cu:9398-9419) runs one thread per voxel over a (COLUMNS, ROWS) x SLICES
// launch after every DROP block.  Here a grid-stride loop over the linear voxel index, sized to
// a multiple of the SM count, reads the interleaved accumulator {x_update, S} of two voxels as one
// 16-byte load and applies x += x_update / S with the reference's float division, then clears it.
// With IDENTIFY_X_N_AIR an updated voxel below X_N_AIR_THRESHOLD is set to 0 (B.cu:9411-9414).
// The ROBUSTB variant (DROP_update_robust2 O.cu:7570) scales the update by
// ||a||^2 / (||a||^2 + Psi), Psi = PSI_SIGN (1 - x) ETA, from the per-voxel normA accumulator.
// The deterministic variant reads the fixed-point sums and counts (x_update = sum * 2^-40).
// The compensated variant (PRECISION MIXED) applies (x_update + comp) / S, where comp holds the
// exact rounding errors of the block's float accumulation (drop_phase2_kernel), and clears both.
#include "pct_kernels.h"

namespace pct {

namespace {

__device__ __forceinline__ float air_cut(float v, double threshold) { return (double)v < threshold ? 0.0f : v; }

__global__ void __launch_bounds__(256) image_update_kernel(float* __restrict__ x, float2* __restrict__ acc, int num_voxels,
                                                           double air)
{
    allow_dependent_launch();
    grid_dependency_wait();  // the DROP block's scatter has landed
    // two voxels per thread: one 16-byte load of {x_update, S} pairs, one 8-byte load of x
    const int stride = gridDim.x * blockDim.x;
    const int pairs = num_voxels >> 1;
    float4* __restrict__ acc4 = reinterpret_cast<float4*>(acc);
    float2* __restrict__ x2 = reinterpret_cast<float2*>(x);
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < pairs; q += stride) {
        const float4 a = acc4[q];
        const bool u0 = a.y > 0.0f, u1 = a.w > 0.0f;
        if (u0 || u1) {
            float2 xv = x2[q];
            if (u0) xv.x = air_cut(xv.x + __fdiv_rn(a.x, a.y), air);
            if (u1) xv.y = air_cut(xv.y + __fdiv_rn(a.z, a.w), air);
            x2[q] = xv;
            acc4[q] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
    }
    if ((num_voxels & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
        const int v = num_voxels - 1;
        const float2 a = acc[v];
        if (a.y > 0.0f) {
            x[v] = air_cut(x[v] + __fdiv_rn(a.x, a.y), air);
            acc[v] = make_float2(0.0f, 0.0f);
        }
    }
}

// kMixed only tells the exact mode's instance from the mixed mode's: the two take the shared-memory
// carve-out of their own mode's path kernel (set_image_update_carveout).
template <bool kMixed>
__global__ void __launch_bounds__(256) image_update_fixed_kernel(float* __restrict__ x, FixedAcc fx, int num_voxels,
                                                                 double air)
{
    allow_dependent_launch();
    grid_dependency_wait();
    const int stride = gridDim.x * blockDim.x;
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < num_voxels; v += stride) {
        const unsigned c = fx.cnt[v];
        if (c > 0) {
            const float xu = (float)((double)(long long)fx.sum[v] * (1.0 / kFixedScale));
            x[v] = air_cut(x[v] + __fdiv_rn(xu, (float)c), air);
            fx.sum[v] = 0ull;
            fx.cnt[v] = 0u;
        }
    }
}

__global__ void __launch_bounds__(256) image_update_comp_kernel(float* __restrict__ x, float2* __restrict__ acc,
                                                                float* __restrict__ comp, int num_voxels, double air)
{
    allow_dependent_launch();
    grid_dependency_wait();
    const int stride = gridDim.x * blockDim.x;
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < num_voxels; v += stride) {
        const float2 a = acc[v];
        if (a.y > 0.0f) {
            x[v] = air_cut(__fadd_rn(x[v], __fdiv_rn(__fadd_rn(a.x, comp[v]), a.y)), air);
            acc[v] = make_float2(0.0f, 0.0f);
            comp[v] = 0.0f;
        }
    }
}

__global__ void __launch_bounds__(256) image_update_robustb_kernel(float* __restrict__ x, float2* __restrict__ acc,
                                                                   float* __restrict__ normA, int num_voxels,
                                                                   int psi_sign, double eta, double air)
{
    allow_dependent_launch();
    grid_dependency_wait();
    const int stride = gridDim.x * blockDim.x;
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < num_voxels; v += stride) {
        const float2 a = acc[v];
        if (a.y > 0.0f) {
            const double norm = (double)normA[v];
            const double psi = psi_sign * (1.0 - (double)x[v]) * eta;
            x[v] = air_cut((float)((double)x[v] + (norm / (norm + psi)) * (double)a.x / (double)a.y), air);
            acc[v] = make_float2(0.0f, 0.0f);
            normA[v] = 0.0f;
        }
    }
}

}  // namespace

cudaError_t set_image_update_carveout(int percent)
{
    // the exact mode's kernels; the mixed mode's path kernel keeps no shared memory, so its kernels
    // (image_update_comp_kernel, image_update_fixed_kernel<true>) keep the driver's choice
    const void* kernels[] = {(const void*)image_update_kernel, (const void*)image_update_fixed_kernel<false>,
                             (const void*)image_update_robustb_kernel};
    for (const void* k : kernels) {
        const cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, percent);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

int sm_count()
{
    static int n = 0;
    if (n == 0) {
        int dev = 0, v = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
        n = v > 0 ? v : 148;
    }
    return n;
}

cudaError_t launch_image_update(const Geometry& g, float* x, float2* acc, float* normA, const FixedAcc& fx,
                                cudaStream_t stream, bool pdl)
{
    const int num_voxels = g.num_voxels;
    if (num_voxels <= 0) return cudaSuccess;
    const int threads = 256;
    const long long cap = (long long)sm_count() * 8;  // 8 resident 256-thread CTAs per SM
    if (g.deterministic) {
        const long long want = ((long long)num_voxels + threads - 1) / threads;
        const int blocks = (int)(want < 1 ? 1 : (want < cap ? want : cap));
        return launch_kernel(pdl, g.mixed_precision ? image_update_fixed_kernel<true> : image_update_fixed_kernel<false>,
                             blocks, threads, stream, x, fx, num_voxels,
                             g.air_threshold);
    }
    if (g.projection_algorithm == PCT_ROBUSTB) {
        const long long want = ((long long)num_voxels + threads - 1) / threads;
        const int blocks = (int)(want < 1 ? 1 : (want < cap ? want : cap));
        return launch_kernel(pdl, image_update_robustb_kernel, blocks, threads, stream, x, acc, normA, num_voxels,
                             g.psi_sign, g.eta, g.air_threshold);
    }
    if (g.compensated && normA) {  // compensated FP32 accumulation: normA holds the errors
        const long long want = ((long long)num_voxels + threads - 1) / threads;
        const int blocks = (int)(want < 1 ? 1 : (want < cap ? want : cap));
        return launch_kernel(pdl, image_update_comp_kernel, blocks, threads, stream, x, acc, normA, num_voxels,
                             g.air_threshold);
    }
    const long long want = ((long long)(num_voxels >> 1) + threads - 1) / threads;
    const int blocks = (int)(want < 1 ? 1 : (want < cap ? want : cap));
    return launch_kernel(pdl, image_update_kernel, blocks, threads, stream, x, acc, num_voxels, g.air_threshold);
}

}  // namespace pct
