// pct_scan.cu -- device prefix sums and the bucket sort used to lay out MLP path storage.
//
// exclusive_scan_i32_to_i64: offsets[i] = sum(values[0..i)), total in offsets[n]; three passes
// (tile sums, one-CTA scan of the tile sums, per-tile scan plus tile prefix).
// bucket_sort_by_key: a counting sort of indices by a small integer key (the path-length bound,
// < kMaxKey), used to group histories of similar length into the same warps.
#include "pct_kernels.h"

namespace pct {

namespace {

constexpr int kScanThreads = 512;
constexpr int kScanItems = 4;  // per thread
constexpr int kTile = kScanThreads * kScanItems;

__device__ __forceinline__ long long block_exclusive_scan(long long v, long long* smem, long long* total)
{
    // warp-level inclusive scan, then scan of warp totals
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    long long x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        long long y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) smem[warp] = x;
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
        long long w = lane < nw ? smem[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            long long y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < nw) smem[lane] = w;
    }
    __syncthreads();
    const long long warp_prefix = warp > 0 ? smem[warp - 1] : 0;
    *total = smem[(blockDim.x >> 5) - 1];
    __syncthreads();
    return warp_prefix + x - v;
}

__global__ void __launch_bounds__(kScanThreads) tile_sums_kernel(const int* __restrict__ v, long long n,
                                                                 long long* __restrict__ tile_sums)
{
    __shared__ long long smem[32];
    const long long base = (long long)blockIdx.x * kTile;
    long long s = 0;
    for (int k = 0; k < kScanItems; k++) {
        const long long i = base + (long long)k * kScanThreads + threadIdx.x;
        if (i < n) s += v[i];
    }
    long long total;
    block_exclusive_scan(s, smem, &total);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanThreads) scan_tile_sums_kernel(long long* __restrict__ tile_sums, long long ntiles)
{
    __shared__ long long smem[32];
    long long carry = 0;
    for (long long base = 0; base < ntiles; base += kScanThreads) {
        const long long i = base + threadIdx.x;
        const long long v = i < ntiles ? tile_sums[i] : 0;
        long long total;
        const long long ex = block_exclusive_scan(v, smem, &total);
        if (i < ntiles) tile_sums[i] = carry + ex;
        carry += total;
    }
    if (threadIdx.x == 0) tile_sums[ntiles] = carry;
}

__global__ void __launch_bounds__(kScanThreads) tile_scan_kernel(const int* __restrict__ v, long long n,
                                                                 const long long* __restrict__ tile_prefix,
                                                                 long long* __restrict__ out)
{
    __shared__ long long smem[32];
    const long long base = (long long)blockIdx.x * kTile + (long long)threadIdx.x * kScanItems;
    long long local[kScanItems];
    long long s = 0;
    for (int k = 0; k < kScanItems; k++) {
        const long long i = base + k;
        local[k] = i < n ? v[i] : 0;
        s += local[k];
    }
    long long total;
    long long ex = block_exclusive_scan(s, smem, &total) + tile_prefix[blockIdx.x];
    for (int k = 0; k < kScanItems; k++) {
        const long long i = base + k;
        if (i < n) out[i] = ex;
        ex += local[k];
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[n] = tile_prefix[gridDim.x];
}

// Each CTA takes a contiguous range of the elements and counts its keys in shared memory, so a
// global counter sees one addition per CTA and key instead of one per element (the keys are
// path-length bounds, concentrated on a few values: per-element global atomics serialised on them).
constexpr int kSortThreads = 256;

__device__ __forceinline__ void cta_range(long long n, long long& b0, long long& b1)
{
    const long long per = (n + gridDim.x - 1) / gridDim.x;
    b0 = (long long)blockIdx.x * per;
    b1 = b0 + per < n ? b0 + per : n;
}

__device__ __forceinline__ int clamp_key(int k, int max_key) { return k < 0 ? 0 : (k >= max_key ? max_key - 1 : k); }

__global__ void __launch_bounds__(kSortThreads) key_histogram_kernel(const int* __restrict__ key, long long begin,
                                                                    long long n, int max_key,
                                                                    unsigned* __restrict__ hist)
{
    extern __shared__ unsigned cnt[];
    for (int k = threadIdx.x; k < max_key; k += blockDim.x) cnt[k] = 0;
    __syncthreads();
    long long b0, b1;
    cta_range(n, b0, b1);
    for (long long i = b0 + threadIdx.x; i < b1; i += blockDim.x) atomicAdd(&cnt[clamp_key(key[begin + i], max_key)], 1u);
    __syncthreads();
    for (int k = threadIdx.x; k < max_key; k += blockDim.x)
        if (cnt[k]) atomicAdd(hist + k, cnt[k]);
}

// descending keys: bucket 0 holds the largest key, so long paths start first.  One warp: each lane
// sums a run of keys (largest first), a warp scan gives the runs' starts.
__global__ void key_offsets_kernel(const unsigned* __restrict__ hist, int max_key, unsigned* __restrict__ cursor)
{
    const int lane = threadIdx.x;
    const int per = (max_key + 31) / 32;
    const int j0 = lane * per, j1 = j0 + per < max_key ? j0 + per : max_key;
    unsigned s = 0;
    for (int j = j0; j < j1; j++) s += hist[max_key - 1 - j];
    unsigned x = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    unsigned acc = x - s;
    for (int j = j0; j < j1; j++) {
        const int k = max_key - 1 - j;
        cursor[k] = acc;
        acc += hist[k];
    }
}

// Each CTA counts its keys again, reserves one contiguous run per key with a single global atomic,
// and places its elements inside the runs with shared-memory atomics.
__global__ void __launch_bounds__(kSortThreads) key_scatter_kernel(const int* __restrict__ key, long long begin,
                                                                  long long n, int max_key,
                                                                  unsigned* __restrict__ cursor,
                                                                  int* __restrict__ perm)
{
    extern __shared__ unsigned sh[];
    unsigned* cnt = sh;
    unsigned* base = sh + max_key;
    for (int k = threadIdx.x; k < max_key; k += blockDim.x) cnt[k] = 0;
    __syncthreads();
    long long b0, b1;
    cta_range(n, b0, b1);
    for (long long i = b0 + threadIdx.x; i < b1; i += blockDim.x) atomicAdd(&cnt[clamp_key(key[begin + i], max_key)], 1u);
    __syncthreads();
    for (int k = threadIdx.x; k < max_key; k += blockDim.x) {
        const unsigned c = cnt[k];
        base[k] = c ? atomicAdd(cursor + k, c) : 0u;
        cnt[k] = 0;
    }
    __syncthreads();
    for (long long i = b0 + threadIdx.x; i < b1; i += blockDim.x) {
        const int k = clamp_key(key[begin + i], max_key);
        perm[base[k] + atomicAdd(&cnt[k], 1u)] = (int)(begin + i);
    }
}

// Windowed variant: each CTA sorts one window of `window` consecutive indices by descending key,
// in shared memory, so the order groups similar keys within a window while every window's
// elements stay together (their data is read once, while it is in L2).
__global__ void __launch_bounds__(kSortThreads) window_sort_kernel(const int* __restrict__ key, long long begin,
                                                                  long long n, int max_key, int window,
                                                                  int* __restrict__ perm)
{
    extern __shared__ unsigned sh[];
    unsigned* cnt = sh;
    unsigned* base = sh + max_key;
    const long long w0 = (long long)blockIdx.x * window;
    const long long w1 = w0 + window < n ? w0 + window : n;
    for (int k = threadIdx.x; k < max_key; k += blockDim.x) cnt[k] = 0;
    __syncthreads();
    for (long long i = w0 + threadIdx.x; i < w1; i += blockDim.x) atomicAdd(&cnt[clamp_key(key[begin + i], max_key)], 1u);
    __syncthreads();
    if (threadIdx.x < 32) {  // descending keys: one warp scans runs of keys, largest first
        const int lane = threadIdx.x;
        const int per = (max_key + 31) / 32;
        const int j0 = lane * per, j1 = j0 + per < max_key ? j0 + per : max_key;
        unsigned sum = 0;
        for (int j = j0; j < j1; j++) sum += cnt[max_key - 1 - j];
        unsigned x = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        unsigned acc = x - sum;
        for (int j = j0; j < j1; j++) {
            const int k = max_key - 1 - j;
            base[k] = acc;
            acc += cnt[k];
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < max_key; k += blockDim.x) cnt[k] = 0;
    __syncthreads();
    for (long long i = w0 + threadIdx.x; i < w1; i += blockDim.x) {
        const int k = clamp_key(key[begin + i], max_key);
        perm[w0 + base[k] + atomicAdd(&cnt[k], 1u)] = (int)(begin + i);
    }
}

}  // namespace

cudaError_t window_sort_by_key(const int* key, long long begin, long long n, int max_key, int window, int* perm,
                               cudaStream_t stream)
{
    if (n <= 0) return cudaSuccess;
    const long long blocks = (n + window - 1) / window;
    const size_t smem = sizeof(unsigned) * 2 * (size_t)max_key;
    window_sort_kernel<<<(unsigned)blocks, kSortThreads, smem, stream>>>(key, begin, n, max_key, window, perm);
    return cudaGetLastError();
}

cudaError_t exclusive_scan_i32_to_i64(const int* values, long long n, long long* offsets, long long* tile_scratch,
                                      cudaStream_t stream)
{
    if (n <= 0) return cudaMemsetAsync(offsets, 0, sizeof(long long), stream);
    const long long ntiles = (n + kTile - 1) / kTile;
    tile_sums_kernel<<<(unsigned)ntiles, kScanThreads, 0, stream>>>(values, n, tile_scratch);
    scan_tile_sums_kernel<<<1, kScanThreads, 0, stream>>>(tile_scratch, ntiles);
    tile_scan_kernel<<<(unsigned)ntiles, kScanThreads, 0, stream>>>(values, n, tile_scratch, offsets);
    return cudaGetLastError();
}

long long scan_tile_scratch_elems(long long n) { return (n + kTile - 1) / kTile + 1; }

cudaError_t bucket_sort_by_key(const int* key, long long begin, long long n, int max_key, unsigned* hist_scratch,
                               int* perm, cudaStream_t stream)
{
    if (n <= 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(hist_scratch, 0, sizeof(unsigned) * 2 * (size_t)max_key, stream);
    if (e != cudaSuccess) return e;
    long long want = (n + 2047) / 2048;
    if (want > sm_count() * 4LL) want = sm_count() * 4LL;
    const int blocks = (int)(want < 1 ? 1 : want);
    const size_t smem = sizeof(unsigned) * (size_t)max_key;
    key_histogram_kernel<<<blocks, kSortThreads, smem, stream>>>(key, begin, n, max_key, hist_scratch);
    key_offsets_kernel<<<1, 32, 0, stream>>>(hist_scratch, max_key, hist_scratch + max_key);
    key_scatter_kernel<<<blocks, kSortThreads, 2 * smem, stream>>>(key, begin, n, max_key, hist_scratch + max_key,
                                                                    perm);
    return cudaGetLastError();
}

}  // namespace pct
