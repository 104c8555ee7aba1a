// pct_selftest.cu -- device self-checks of compiler/libdevice behaviour the exact mode relies on.
//
// The exact MLP mode writes the reference's powf(v, 2) (a float power of a value rounded to
// float) as a float multiply.  pct_selftest_powf_square compares CUDA's powf(f, 2.0f) with
// __fmul_rn(f, f) over n inputs spread across the float exponent range and returns the number
// of mismatches (expected 0).  Inputs are generated in-kernel from a counter-based hash.
#include "pct_common.cuh"

namespace {

__device__ __forceinline__ uint32_t mix32(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return (uint32_t)((z ^ (z >> 31)) >> 16);
}

__global__ void powf_square_kernel(long long n, unsigned long long seed, unsigned long long* mismatches)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    unsigned long long local = 0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint32_t r = mix32(seed + (uint64_t)i * 0x9e3779b97f4a7c15ull);
        // exponent in [2^-60, 2^60): squares stay finite and normal
        const uint32_t expo = 67u + (r >> 24) % 120u;
        const uint32_t bits = (expo << 23) | (r & 0x7fffffu);
        const float f = __uint_as_float(bits);
        const float a = powf(f, 2.0f);
        const float b = __fmul_rn(f, f);
        if (__float_as_uint(a) != __float_as_uint(b)) local++;
    }
    if (local) atomicAdd(mismatches, local);
}

}  // namespace

extern "C" pct_status pct_selftest_powf_square(int64_t n, uint64_t seed, int64_t* mismatches)
{
    if (n < 0 || !mismatches) return PCT_ERR_ARG;
    unsigned long long* d = nullptr;
    if (cudaMalloc(&d, sizeof(*d)) != cudaSuccess) return PCT_ERR_NOMEM;
    cudaMemset(d, 0, sizeof(*d));
    powf_square_kernel<<<148 * 4, 256>>>(n, seed, d);
    unsigned long long h = 0;
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(&h, d, sizeof(h), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return PCT_ERR_CUDA;
    *mismatches = (int64_t)h;
    return PCT_OK;
}
