// pct_noalloc.cu -- a DROP block update that allocates no device memory.
//
// Who needs this: some callers cannot call cudaMalloc/cudaFree while they reconstruct.  A
// real-time service that streams DROP blocks cannot afford them, because allocation and release
// can synchronise the whole device and stall every other stream; a plugin host that hands this
// library a fixed device-memory budget forbids them outright; and code that keeps its CUDA work
// free of allocation calls so it can later be issued in a stream-ordered sequence cannot make
// them either.  pct_drop_block_update_noalloc serves those callers: the caller passes the block's
// histories and the image in its own device memory, and the per-voxel accumulator {x_update, S}
// that the ordinary path keeps in context-owned memory lives instead in the file-scope array
// below, which the module holds on every GPU that loads the library until the process exits.
//
// Limits and sharing:
//  * the accumulator holds kNoAllocMaxVoxels voxels (18 MiB); a configuration with more voxels is
//    rejected with PCT_ERR_ARG;
//  * every call on a device uses the same array.  Each call clears the part it uses before it
//    scatters, so a call never sees the previous call's sums, but two calls whose kernels overlap
//    on the GPU (different streams, different contexts, or different host threads) race on it;
//    serialise them;
//  * the device address of the array is looked up once per device, on that device's first call
//    (cudaGetSymbolAddress); make that first call before any stream capture begins;
//  * the image x must be 8-byte aligned (the image update moves two voxels per 8-byte access);
//    a misaligned pointer is rejected with PCT_ERR_ARG;
//  * the MLP is always the exact (FP64, reference-rounding) walk, whatever the context's
//    PRECISION setting, as in pct_calculate_x_update.
#include <stdint.h>

#include <mutex>

#include "pct_kernels.h"
#include "pct_mlp.cuh"

namespace pct {

// 2.25 Mi voxels: the reference's default 256 x 256 x 32 grid (2 Mi voxels) plus headroom.
constexpr long long kNoAllocMaxVoxels = 2359296;

// The static accumulator {x_update, S} of the no-allocation entry point.  Host code must not
// pass this name to a kernel: on the host it is only a stand-in; its device address comes from
// cudaGetSymbolAddress.
static __device__ __align__(256) float2 g_noalloc_acc[kNoAllocMaxVoxels];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
float2* g_acc_address[kMaxDevices] = {};

// Device address of g_noalloc_acc on the current device, looked up on the first call per device.
cudaError_t noalloc_accumulator(int device, float2** out)
{
    if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_acc_address[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_acc);
        if (e != cudaSuccess) return e;
        g_acc_address[device] = static_cast<float2*>(p);
    }
    *out = g_acc_address[device];
    return cudaSuccess;
}

// The fused MLP + scatter of one DROP block (the computation of drop_block_exact_kernel),
// scattering into the caller-supplied accumulator address.  Walk flags (an entry outside the
// grid, a path beyond the list cap, a depth beyond the tables) go to the context's counters,
// which the context allocated when it was created.  g.padded_voxels equals
// g.num_voxels here: the caller's image has no spare slice, so a voxel index at or beyond
// NUM_VOXELS reads as 0 and receives no update, which leaves the image identical to the padded
// ordinary path (its spare slice is zero and never applied).
__global__ void __launch_bounds__(128) noalloc_drop_block_kernel(Geometry g, Tables tab, const StepConst* __restrict__ steps,
                                                                 int kmax, const float* __restrict__ x,
                                                                 float2* __restrict__ acc, HistorySoA h, long long count,
                                                                 unsigned long long* counters)
{
    const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= count) return;
    uint32_t path[kPathCap];
    const WalkResult r = mlp_walk_exact<true>(
        g, tab, steps, kmax, x, __ldg(h.first_MLP_voxel + id), __ldg(h.x_entry + id), __ldg(h.y_entry + id),
        __ldg(h.z_entry + id), __ldg(h.x_exit + id), __ldg(h.y_exit + id), __ldg(h.z_exit + id),
        __ldg(h.xy_entry_angle + id), __ldg(h.xz_entry_angle + id), __ldg(h.xy_exit_angle + id),
        __ldg(h.xz_exit_angle + id), [&](int j, uint32_t v) { path[j] = v; });
    if (r.flags) count_flags(r.flags, counters);
    if (r.n < g.min_mlp_length) return;
    const double a_i_dot_a_i = r.aia * r.n;
    const double a_i_dot_x_k = r.axk * r.chord;
    const float upd = (float)(r.chord * (((double)__ldg(h.WEPL + id) - a_i_dot_x_k) / a_i_dot_a_i) * g.lambda);
    const float2 add = make_float2(upd, 1.0f);
    for (int j = 0; j < r.n; j++) {
        const uint32_t v = path[j];
        if (v < (uint32_t)g.num_voxels) atomicAdd(acc + v, add);
    }
}

}  // namespace

}  // namespace pct

extern "C" pct_status pct_drop_block_update_noalloc(pct_ctx* ctx, const pct_histories* h, int64_t n, float* x)
{
    pct::ContextView v;
    if (!pct::context_view(ctx, &v) || !h || !x || n < 0) return PCT_ERR_ARG;
    if (reinterpret_cast<uintptr_t>(x) & 7u) {
        pct::context_set_error(ctx, "pct_drop_block_update_noalloc: the image x must be 8-byte aligned");
        return PCT_ERR_ARG;
    }
    if ((long long)v.geo.num_voxels > pct::kNoAllocMaxVoxels) {
        pct::context_set_error(ctx, "pct_drop_block_update_noalloc: NUM_VOXELS exceeds the 2359296-voxel static "
                                    "accumulator; use pct_calculate_x_update + pct_image_update instead");
        return PCT_ERR_ARG;
    }
    if (v.geo.projection_algorithm != PCT_DROP || v.geo.deterministic || v.geo.s_curve) {
        pct::context_set_error(ctx, "pct_drop_block_update_noalloc: needs PROJECTION_ALGORITHM DROP, SCATTER_MODE ATOMIC, "
                                    "S_CURVE_ON 0");
        return PCT_ERR_ARG;
    }
    if (n > 0 && (!h->x_entry || !h->y_entry || !h->z_entry || !h->x_exit || !h->y_exit || !h->z_exit ||
                  !h->xy_entry_angle || !h->xz_entry_angle || !h->xy_exit_angle || !h->xz_exit_angle || !h->WEPL ||
                  !h->first_MLP_voxel))
        return PCT_ERR_ARG;
    cudaError_t e = cudaSetDevice(v.device);
    float2* acc = nullptr;
    if (e == cudaSuccess) e = pct::noalloc_accumulator(v.device, &acc);
    if (e != cudaSuccess) {
        pct::context_set_error(ctx, "pct_drop_block_update_noalloc: cudaGetSymbolAddress failed");
        return PCT_ERR_CUDA;
    }
    // clear the voxels this call accumulates into (the array keeps the previous call's state)
    e = cudaMemsetAsync(acc, 0, sizeof(float2) * (size_t)v.geo.num_voxels, v.stream);
    pct::Geometry g = v.geo;
    g.padded_voxels = g.num_voxels;
    // the history arrays are read-only here; HistorySoA carries non-const pointers
    pct::HistorySoA hs{const_cast<float*>(h->x_entry), const_cast<float*>(h->y_entry), const_cast<float*>(h->z_entry),
                       const_cast<float*>(h->x_exit), const_cast<float*>(h->y_exit), const_cast<float*>(h->z_exit),
                       const_cast<float*>(h->xy_entry_angle), const_cast<float*>(h->xz_entry_angle),
                       const_cast<float*>(h->xy_exit_angle), const_cast<float*>(h->xz_exit_angle),
                       const_cast<float*>(h->WEPL), const_cast<uint32_t*>(h->first_MLP_voxel)};
    if (e == cudaSuccess && n > 0) {
        const int threads = 128;
        pct::noalloc_drop_block_kernel<<<(unsigned)((n + threads - 1) / threads), threads, 0, v.stream>>>(
            g, v.tables, v.steps, v.kmax, x, acc, hs, n, v.counters);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = pct::launch_image_update(g, x, acc, nullptr, pct::FixedAcc{nullptr, nullptr}, v.stream);
        pct::context_count_launches(ctx, 2);
    }
    if (e != cudaSuccess) {
        pct::context_set_error(ctx, "pct_drop_block_update_noalloc: kernel launch failed");
        return PCT_ERR_CUDA;
    }
    return PCT_OK;
}
