// pct_selftest.cu -- device self-checks of compiler/libdevice behaviour the exact mode relies on.
//
// The reference squares values with powf(v, 2) (a float power of a value rounded to float), and
// the exact MLP mode calls CUDA's powf the same way, because powf(f, 2.0f) is not always the
// correctly rounded product.  pct_selftest_powf_square compares CUDA's powf(f, 2.0f) with
// __fmul_rn(f, f) over n inputs spread across the float exponent range and returns the number
// of mismatches (a few percent of the inputs; the CPU oracle, which squares with the correctly
// rounded product, counts its ties against that rate).  pct_selftest_powf_square_max_ulp
// compares the two on every float of magnitude in [2^-60, 2^60) and on zero and returns the
// largest distance in float ulps (1 on B200 with CUDA 12.9): the size of each such tie's cause.  Inputs are
// generated in-kernel from a counter-based hash.
//
// pct_fp64_fma_rate measures the device's FP64 issue rate: the denominator of the path kernel's
// FP64 roofline (the exact MLP is a chain of uncontracted FP64 adds, multiplies and divisions).
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

// Every float f with |f| in [2^-60, 2^60) (both signs, all mantissas), and +-0: the largest
// distance in float ulps between powf(f, 2.0f) and __fmul_rn(f, f).  Both are non-negative, so the
// distance is the difference of their bit patterns.
__global__ void powf_square_ulp_kernel(unsigned long long* max_ulp)
{
    const long long total = 2LL * 120 * (1LL << 23) + 2;
    const long long stride = (long long)gridDim.x * blockDim.x;
    unsigned long long local = 0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        uint32_t bits;
        if (i >= total - 2) {
            bits = (uint32_t)(i - (total - 2)) << 31;  // +0, -0
        } else {
            const long long j = i >> 1;
            bits = ((uint32_t)(i & 1) << 31) | ((uint32_t)(67 + (j >> 23)) << 23) | (uint32_t)(j & 0x7fffff);
        }
        const float f = __uint_as_float(bits);
        const uint32_t a = __float_as_uint(powf(f, 2.0f)), b = __float_as_uint(__fmul_rn(f, f));
        const unsigned long long d = a > b ? a - b : b - a;
        if (d > local) local = d;
    }
    if (local) atomicMax(max_ulp, local);
}

// Eight independent FMA chains per thread (x = x * a + b, |a| < 1 keeps them finite), so that the
// FP64 pipe, not the 4-cycle dependency latency, limits the issue rate.
__global__ void __launch_bounds__(256) fp64_fma_rate_kernel(int iters, double a, double b, double* sink)
{
    double x0 = threadIdx.x * 1e-3, x1 = x0 + 0.125, x2 = x0 + 0.25, x3 = x0 + 0.375, x4 = x0 + 0.5, x5 = x0 + 0.625,
           x6 = x0 + 0.75, x7 = x0 + 0.875;
#pragma unroll 4
    for (int i = 0; i < iters; i++) {
        x0 = __fma_rn(x0, a, b);
        x1 = __fma_rn(x1, a, b);
        x2 = __fma_rn(x2, a, b);
        x3 = __fma_rn(x3, a, b);
        x4 = __fma_rn(x4, a, b);
        x5 = __fma_rn(x5, a, b);
        x6 = __fma_rn(x6, a, b);
        x7 = __fma_rn(x7, a, b);
    }
    const double s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
    if (s == 1.2345e300) sink[threadIdx.x] = s;  // never taken; keeps every chain live
}

}  // namespace

extern "C" pct_status pct_fp64_fma_rate(int device, double* fma_per_second)
{
    if (!fma_per_second) return PCT_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return PCT_ERR_ARG;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || sms <= 0)
        return PCT_ERR_CUDA;
    const int threads = 256, blocks = sms * 8, iters = 16384;  // 8 CTAs x 256 threads fill an SM
    double* sink = nullptr;
    cudaStream_t s = nullptr;
    cudaEvent_t a = nullptr, b = nullptr;
    cudaError_t e = cudaMalloc(&sink, sizeof(double) * threads);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&a);
    if (e == cudaSuccess) e = cudaEventCreate(&b);
    float best = 0.0f;
    for (int rep = 0; rep < 6 && e == cudaSuccess; rep++) {  // the first launch warms up
        e = cudaEventRecord(a, s);
        fp64_fma_rate_kernel<<<blocks, threads, 0, s>>>(iters, 0.999999, 1e-7, sink);
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaEventRecord(b, s);
        if (e == cudaSuccess) e = cudaEventSynchronize(b);
        float ms = 0.0f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
        if (e == cudaSuccess && rep > 0 && (best == 0.0f || ms < best)) best = ms;
    }
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    if (s) cudaStreamDestroy(s);
    cudaFree(sink);
    if (e != cudaSuccess || best <= 0.0f) return PCT_ERR_CUDA;
    *fma_per_second = (double)blocks * threads * iters * 8.0 / (best * 1e-3);
    return PCT_OK;
}

extern "C" pct_status pct_selftest_powf_square_max_ulp(int64_t* max_ulp)
{
    if (!max_ulp) return PCT_ERR_ARG;
    unsigned long long* d = nullptr;
    if (cudaMalloc(&d, sizeof(*d)) != cudaSuccess) return PCT_ERR_NOMEM;
    cudaMemset(d, 0, sizeof(*d));
    powf_square_ulp_kernel<<<148 * 4, 256>>>(d);
    unsigned long long h = 0;
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(&h, d, sizeof(h), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return PCT_ERR_CUDA;
    *max_ulp = (int64_t)h;
    return PCT_OK;
}

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
