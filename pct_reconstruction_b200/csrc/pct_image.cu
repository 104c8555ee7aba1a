// pct_image.cu -- per-block image update of DROP.
//
// image_update_GPU (B.cu:9398-9419) runs one thread per voxel over a (COLUMNS, ROWS) x SLICES
// launch after every DROP block.  Here a grid-stride loop over the linear voxel index, sized to
// a multiple of the SM count, reads the interleaved accumulator {x_update, S} as one 8-byte load
// and applies x += x_update / S with the reference's float division, then clears the pair.
#include "pct_kernels.h"

namespace pct {

namespace {

__global__ void __launch_bounds__(256) image_update_kernel(float* __restrict__ x, float2* __restrict__ acc, int num_voxels)
{
    const int stride = gridDim.x * blockDim.x;
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < num_voxels; v += stride) {
        const float2 a = acc[v];
        if (a.y > 0.0f) {
            x[v] += __fdiv_rn(a.x, a.y);
            acc[v] = make_float2(0.0f, 0.0f);
        }
    }
}

}  // namespace

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

cudaError_t launch_image_update(float* x, float2* acc, int num_voxels, cudaStream_t stream)
{
    if (num_voxels <= 0) return cudaSuccess;
    const int threads = 256;
    long long want = ((long long)num_voxels + threads - 1) / threads;
    const long long cap = (long long)sm_count() * 8;  // 8 resident 256-thread CTAs per SM
    const int blocks = (int)(want < cap ? want : cap);
    image_update_kernel<<<blocks, threads, 0, stream>>>(x, acc, num_voxels);
    return cudaGetLastError();
}

}  // namespace pct
