// pct_image.cu -- per-block image update of DROP.
//
// image_update_GPU (B.cu:9398-9419) runs one thread per voxel over a (COLUMNS, ROWS) x SLICES
// launch after every DROP block.  Here a grid-stride loop over the linear voxel index, sized to
// a multiple of the SM count, reads the interleaved accumulator {x_update, S} of two voxels as one
// 16-byte load and applies x += x_update / S with the reference's float division, then clears it.
#include "pct_kernels.h"

namespace pct {

namespace {

__global__ void __launch_bounds__(256) image_update_kernel(float* __restrict__ x, float2* __restrict__ acc, int num_voxels)
{
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
            if (u0) xv.x += __fdiv_rn(a.x, a.y);
            if (u1) xv.y += __fdiv_rn(a.z, a.w);
            x2[q] = xv;
            acc4[q] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
    }
    if ((num_voxels & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
        const int v = num_voxels - 1;
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
    long long want = ((long long)(num_voxels >> 1) + threads - 1) / threads;
    const long long cap = (long long)sm_count() * 8;  // 8 resident 256-thread CTAs per SM
    const int blocks = (int)(want < 1 ? 1 : (want < cap ? want : cap));
    image_update_kernel<<<blocks, threads, 0, stream>>>(x, acc, num_voxels);
    return cudaGetLastError();
}

}  // namespace pct
