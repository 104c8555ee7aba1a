// pct_unet.cu -- learned DROP initializer: a 3-D convolutional encoder-decoder in bf16 on the
// tensor cores (tcgen05, fp32 accumulation in TMEM), with its own training kernels.
//
// The reference has no learned component; this is the engine's option to replace the FBP start
// x_0 = FBP_median x hull (define_initial_iterate, B.cu:8582-8646) by a network's estimate of the
// converged DROP image.  The FBP start stays the fallback.
//
// Network (4 levels, 16 -> 128 channels, 3x3x3 kernels, padding 1, ReLU):
//   encoder  L0: 16 -> 16 -> 16   avg-pool 2  L1: 16 -> 32 -> 32   pool  L2: 32 -> 64 -> 64
//            pool  L3: 64 -> 128 -> 128
//   decoder  nearest x2 up, conv to the level's width, + the encoder output of that level, ReLU,
//            conv, ReLU: L2 128 -> 64 -> 64, L1 64 -> 32 -> 32, L0 32 -> 16 -> 16
//   output   conv 16 -> 1 (channel 0 of a 16-wide conv whose other weights stay zero);
//            image = x_0 + (hull ? output : 0), so an untrained (zero) output layer gives back x_0.
//   input    channels-last bf16, channel 0 = x_0, channel 1 = hull, channels 2..15 = 0.
// Activations are channels-last bf16 [slice][row][column][channel] in the reference voxel order.
// Grids must have COLUMNS, ROWS and SLICES divisible by 8.
//
// Kernels:
//  * conv3_fwd_kernel: implicit GEMM, one CTA per 128 output voxels (M = 128), N = output
//    channels, K = 27 taps x input channels; per tap the CTA gathers the 128 shifted input rows
//    and the tap's weights into shared memory (K-major core-matrix layout), one thread issues
//    the tcgen05.mma instructions into the TMEM accumulator, two stages overlap the gather of
//    tap t+1 with the MMAs of tap t.  The same kernel computes the data gradient with the
//    flipped, transposed weights W'[ci][26-t][co] = W[co][t][ci].  Epilogue: bias, residual,
//    ReLU, ReLU-mask (for gradients), bf16 store; or the image output.
//  * conv3_wgrad_kernel: dW[co][t][ci] = sum_v dZ[v][co] X[v + t][ci]: M = 128 (tap, channel)
//    rows, N = output channels, K = voxels (64 per stage, MN-major operands, which is how both
//    lie in memory); the voxel range is split over CTAs, partial sums are added with atomics.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "pct_api.h"
#include "pct_context.h"
#include "pct_tc.cuh"

namespace pct {
namespace unet {

using bf16 = __nv_bfloat16;
constexpr int kThreads = 128;
constexpr int kChunk = 64;          // voxels per weight-gradient stage
constexpr int kSmemPerSm = 233472;  // shared memory per SM on sm_100
constexpr int kTmemColumns = 512;   // TMEM columns per SM

// ------------------------------------------------------------------ MMA pipeline bookkeeping --

// Two shared-memory stages, each guarded by an mbarrier that the MMAs reading it commit to.
// issued/waited count commits and completed waits per stage; every thread keeps the same counts,
// only thread 0 polls the barrier, and the verdict is shared with __syncthreads_or.
struct Pipe {
    uint32_t mbar[2];
    int issued[2];
    int waited[2];
};

__device__ __forceinline__ bool stage_free(Pipe& pp, int b)
{
    int bad = 0;
    if (pp.issued[b] > pp.waited[b]) {
        if (threadIdx.x == 0) bad = !tc::mbar_wait(pp.mbar[b], pp.waited[b] & 1);
        pp.waited[b]++;
    }
    return __syncthreads_or(bad) == 0;
}

__device__ __forceinline__ bool drain(Pipe& pp)
{
    int bad = 0;
    for (int b = 0; b < 2; ++b) {
        while (pp.issued[b] > pp.waited[b]) {
            if (threadIdx.x == 0 && !bad) bad = !tc::mbar_wait(pp.mbar[b], pp.waited[b] & 1);
            pp.waited[b]++;
        }
    }
    return __syncthreads_or(bad) == 0;
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b)
{
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&h);
}

__device__ __forceinline__ void unpack8(const uint4& u, float* f)
{
    const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const float2 t = __bfloat1622float2(h[i]);
        f[2 * i] = t.x;
        f[2 * i + 1] = t.y;
    }
}

// ----------------------------------------------------------------------------- convolutions --

// Taps gathered per pipeline stage for 16-channel inputs (half as many for 32).  Measured on B200
// (200x200x32, forward 16->16 / 32->16 upsampled, ms): 1 tap 0.321 / 0.466, 2 taps 0.314 / 0.505,
// 4 taps 0.395 / 0.542 -- the deeper gather per stage costs more than the barriers it saves.
// Weight-gradient CTAs per SM: 4 -> 0.541 ms, 6 -> 0.413 ms (16->16); training step 9.06 -> 8.47 ms.
#ifndef PCT_CONV_TAPS_16
#define PCT_CONV_TAPS_16 1
#endif
#ifndef PCT_WGRAD_CTAS_PER_SM
#define PCT_WGRAD_CTAS_PER_SM 6
#endif
__host__ __device__ constexpr int taps_per_stage(int cin)
{
    return cin >= 64 ? 1 : (cin == 32 ? (PCT_CONV_TAPS_16 > 1 ? PCT_CONV_TAPS_16 / 2 : 1) : PCT_CONV_TAPS_16);
}
__host__ __device__ constexpr int conv_stage_bytes(int cin, int cout)
{
    return (taps_per_stage(cin) * (cin * tc::kTileM * 2 + cout * cin * 2) + 127) & ~127;
}

struct ConvFwdArgs {
    const bf16* in;      // [nz>>up][ny>>up][nx>>up][cin]
    int cin, up;
    const bf16* weight;  // [cout][27][cin]
    int cout;
    int nx, ny, nz;      // output grid (= the input grid after the optional x2 upsampling)
    const float* bias;   // [cout] or null
    const bf16* residual;  // [V][cout] or null: added before the ReLU
    const bf16* mask;      // [V][cout] or null: output zeroed where mask <= 0
    int relu;
    bf16* out;             // [V][cout]
    const float* base;     // image mode: image[v] = base[v] + (hull[v] ? acc0 + bias0 : 0)
    const uint8_t* hull;
    float* image;
    int* status;           // set to 1 when a bounded wait expired
};

// Epilogue of a forward / data-gradient convolution tile: this thread's TMEM lane (row) holds
// voxel v's accumulators; every thread of the CTA calls it (tcgen05.ld is warp-collective).
__device__ __forceinline__ void conv_epilogue(const ConvFwdArgs& p, uint32_t trow, long long v, bool row_ok)
{
    if (p.image) {
        float acc[16];
        tc::tmem_load16(trow, acc);
        if (row_ok) {
            const float o = acc[0] + (p.bias ? p.bias[0] : 0.f);
            p.image[v] = p.base[v] + (p.hull[v] ? o : 0.f);
        }
    } else {
        for (int c0 = 0; c0 < p.cout; c0 += 16) {
            float acc[16];
            tc::tmem_load16(trow + c0, acc);
            if (!row_ok) continue;
            const size_t o = static_cast<size_t>(v) * p.cout + c0;
            if (p.bias) {
#pragma unroll
                for (int i = 0; i < 16; ++i) acc[i] += p.bias[c0 + i];
            }
            if (p.residual) {
                float r[16];
                unpack8(__ldg(reinterpret_cast<const uint4*>(p.residual + o)), r);
                unpack8(__ldg(reinterpret_cast<const uint4*>(p.residual + o) + 1), r + 8);
#pragma unroll
                for (int i = 0; i < 16; ++i) acc[i] += r[i];
            }
            if (p.relu) {
#pragma unroll
                for (int i = 0; i < 16; ++i) acc[i] = fmaxf(acc[i], 0.f);
            }
            if (p.mask) {
                float m[16];
                unpack8(__ldg(reinterpret_cast<const uint4*>(p.mask + o)), m);
                unpack8(__ldg(reinterpret_cast<const uint4*>(p.mask + o) + 1), m + 8);
#pragma unroll
                for (int i = 0; i < 16; ++i) acc[i] = m[i] > 0.f ? acc[i] : 0.f;
            }
            uint4 w0, w1;
            w0.x = pack_bf16(acc[0], acc[1]);
            w0.y = pack_bf16(acc[2], acc[3]);
            w0.z = pack_bf16(acc[4], acc[5]);
            w0.w = pack_bf16(acc[6], acc[7]);
            w1.x = pack_bf16(acc[8], acc[9]);
            w1.y = pack_bf16(acc[10], acc[11]);
            w1.z = pack_bf16(acc[12], acc[13]);
            w1.w = pack_bf16(acc[14], acc[15]);
            reinterpret_cast<uint4*>(p.out + o)[0] = w0;
            reinterpret_cast<uint4*>(p.out + o)[1] = w1;
        }
    }
}

__global__ void __launch_bounds__(kThreads) conv3_fwd_kernel(ConvFwdArgs p)
{
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t mbar[2];
    __shared__ uint32_t tmem_slot;
    const int tid = threadIdx.x, warp = tid >> 5;
    const long long V = static_cast<long long>(p.nx) * p.ny * p.nz;
    const long long v = static_cast<long long>(blockIdx.x) * tc::kTileM + tid;
    const uint32_t ncols = tc::tmem_columns(p.cout);
    const int tps = taps_per_stage(p.cin);
    const int a_tap = p.cin * tc::kTileM * 2, b_tap = p.cout * p.cin * 2;
    const int stage_bytes = conv_stage_bytes(p.cin, p.cout);

    if (warp == 0) tc::tmem_alloc(tc::smem_addr(&tmem_slot), ncols);
    if (tid == 0) {
        tc::mbar_init(tc::smem_addr(&mbar[0]), 1);
        tc::mbar_init(tc::smem_addr(&mbar[1]), 1);
        tc::mbar_init_fence();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tmem_slot;
    Pipe pp{{tc::smem_addr(&mbar[0]), tc::smem_addr(&mbar[1])}, {0, 0}, {0, 0}};

    const bool row_ok = v < V;
    int x = 0, y = 0, z = 0;
    if (row_ok) {
        x = static_cast<int>(v % p.nx);
        const long long r = v / p.nx;
        y = static_cast<int>(r % p.ny);
        z = static_cast<int>(r / p.ny);
    }
    const int sx = p.nx >> p.up, sy = p.ny >> p.up;
    const uint32_t sbo = static_cast<uint32_t>(p.cin) * 16u;  // 8 rows x cin bf16
    const int kc = p.cin >> 3;                                // 16-byte chunks per row
    const uint32_t idesc = tc::idesc_bf16_f32(p.cout, false);
    bool ok = true;
    int it = 0;
    for (int t0 = 0; t0 < 27; t0 += tps, ++it) {
        const int b = it & 1;
        if (!stage_free(pp, b)) {
            ok = false;
            break;
        }
        uint8_t* sa = smem + b * stage_bytes;
        uint8_t* sb = sa + tps * a_tap;
        const int nt = t0 + tps <= 27 ? tps : 27 - t0;
        for (int q = 0; q < nt; ++q) {
            const int t = t0 + q;
            const int zz = z + t / 9 - 1, yy = y + (t / 3) % 3 - 1, xx = x + t % 3 - 1;
            const bool inside = row_ok && zz >= 0 && zz < p.nz && yy >= 0 && yy < p.ny && xx >= 0 && xx < p.nx;
            uint8_t* dst = sa + q * a_tap + (tid >> 3) * sbo + (tid & 7) * 16;
            if (inside) {
                const size_t src_voxel = (static_cast<size_t>(zz >> p.up) * sy + (yy >> p.up)) * sx + (xx >> p.up);
                const uint4* src = reinterpret_cast<const uint4*>(p.in + src_voxel * p.cin);
                for (int c = 0; c < kc; ++c) *reinterpret_cast<uint4*>(dst + c * 128) = __ldg(src + c);
            } else {
                for (int c = 0; c < kc; ++c) *reinterpret_cast<uint4*>(dst + c * 128) = make_uint4(0, 0, 0, 0);
            }
            uint8_t* sbq = sb + q * b_tap;
            for (int u = tid; u < p.cout * kc; u += kThreads) {
                const int n = u / kc, c = u - n * kc;
                const uint4 w = __ldg(reinterpret_cast<const uint4*>(p.weight + (static_cast<size_t>(n) * 27 + t) * p.cin) + c);
                *reinterpret_cast<uint4*>(sbq + (n >> 3) * sbo + c * 128 + (n & 7) * 16) = w;
            }
        }
        tc::fence_proxy_async();
        __syncthreads();
        if (tid == 0) {
            tc::fence_after_sync();
            for (int q = 0; q < nt; ++q) {
                const uint32_t a0 = tc::smem_addr(sa + q * a_tap), b0 = tc::smem_addr(sb + q * b_tap);
                for (int j = 0; j < (p.cin >> 4); ++j)
                    tc::mma_bf16(tmem, tc::smem_desc(a0 + j * 256, 128, sbo), tc::smem_desc(b0 + j * 256, 128, sbo),
                                 idesc, (t0 | q | j) != 0);
            }
            tc::mma_commit(pp.mbar[b]);
        }
        pp.issued[b]++;
    }
    ok = drain(pp) && ok;
    tc::fence_after_sync();
    if (ok) {
        conv_epilogue(p, tmem + (static_cast<uint32_t>(warp * 32) << 16), v, row_ok);
    } else if (tid == 0) {
        atomicExch(p.status, 1);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem, ncols);
    }
}

// ---- TMA-fed forward convolution ------------------------------------------------------------
// The same convolution with the operand tiles brought by TMA instead of thread gathers.  A CTA owns
// the 128 voxels of a 32 x 4 patch of one slice (TMEM lane = y_local * 32 + x_local).  For tap t
// the A tile is the box of the channels-last activation tensor at (x0+dx, y0+dy, z+dz) -- boxes
// that reach outside the grid are zero-filled by TMA, which is the convolution's zero padding --
// and the B tile is the tap's [cout][cin] weight slab.  Both arrive in the swizzled K-major layout
// the MMA reads (rows of 32/64/128 bytes: 16/32/64 channels per box; 128 channels take two boxes).
// One thread drives a kTmaMaxStages-deep pipeline: "full" barriers count TMA bytes, "empty"
// barriers are armed by tcgen05.commit when the MMAs of a stage are done.  Not used for an
// upsampled input (a box copy cannot duplicate voxels).
constexpr int kTmaTileX = 32, kTmaTileY = 4;
// Pipeline depth, measured on B200 (200x200x32 network, 16 -> 16 forward / training step):
// 4 stages 0.263 / 7.01 ms, 6 stages 0.286 / 7.49 ms, 8 stages 0.385 / 8.52 ms -- deeper stages
// cost CTAs per SM.
#ifndef PCT_TMA_STAGES
#define PCT_TMA_STAGES 4
#endif
constexpr int kTmaMaxStages = PCT_TMA_STAGES;
constexpr int kTmaSmemLimit = 226 * 1024;  // dynamic; the per-block maximum (227 KB) also holds the static barriers

struct TmaConvShape {
    int bc, nsub;        // channels per box (row bytes / 2), boxes per row
    int a_sub, b_sub;    // bytes of one A / B box
    int tx;              // bytes one stage receives
    int stage, stages;   // bytes per stage (1024-aligned), stages
};

__host__ __device__ inline TmaConvShape tma_conv_shape(int cin, int cout)
{
    TmaConvShape s;
    s.bc = cin < 64 ? cin : 64;
    s.nsub = cin / s.bc;
    s.a_sub = kTmaTileX * kTmaTileY * s.bc * 2;
    s.b_sub = cout * s.bc * 2;
    s.tx = s.nsub * (s.a_sub + s.b_sub);
    s.stage = (s.tx + 1023) & ~1023;
    const int fit = (kTmaSmemLimit - 2048) / s.stage;
    s.stages = fit < kTmaMaxStages ? fit : kTmaMaxStages;
    return s;
}

__global__ void __launch_bounds__(kThreads) conv3_fwd_tma_kernel(const __grid_constant__ CUtensorMap tm_in,
                                                                const __grid_constant__ CUtensorMap tm_w, ConvFwdArgs p)
{
    extern __shared__ uint8_t smem_raw[];
    __shared__ __align__(8) uint64_t full[kTmaMaxStages];
    __shared__ __align__(8) uint64_t empty[kTmaMaxStages];
    __shared__ __align__(8) uint64_t done;
    __shared__ uint32_t tmem_slot;
    __shared__ int issue_failed;
    const int tid = threadIdx.x, warp = tid >> 5;
    const TmaConvShape sh = tma_conv_shape(p.cin, p.cout);
    const uint32_t base = (tc::smem_addr(smem_raw) + 1023u) & ~1023u;
    const int tiles_x = (p.nx + kTmaTileX - 1) / kTmaTileX, tiles_y = (p.ny + kTmaTileY - 1) / kTmaTileY;
    const int tx = blockIdx.x % tiles_x, ty = (blockIdx.x / tiles_x) % tiles_y, z = blockIdx.x / (tiles_x * tiles_y);
    const int x0 = tx * kTmaTileX, y0 = ty * kTmaTileY;
    const uint32_t ncols = tc::tmem_columns(p.cout);

    if (warp == 0) tc::tmem_alloc(tc::smem_addr(&tmem_slot), ncols);
    if (tid == 0) {
        for (int i = 0; i < kTmaMaxStages; ++i) {
            tc::mbar_init(tc::smem_addr(&full[i]), 1);
            tc::mbar_init(tc::smem_addr(&empty[i]), 1);
        }
        tc::mbar_init(tc::smem_addr(&done), 1);
        tc::mbar_init_fence();
        issue_failed = 0;
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tmem_slot;

    if (tid == 0) {
        const uint32_t idesc = tc::idesc_bf16_f32(p.cout, false);
        const uint32_t row_bytes = static_cast<uint32_t>(sh.bc) * 2u;
        const int S = sh.stages;
        bool bad = false;
        for (int t = 0; t < 27 + S - 1 && !bad; ++t) {
            if (t < 27) {
                const int st = t % S, round = t / S;
                if (round > 0 && !tc::mbar_wait(tc::smem_addr(&empty[st]), (round - 1) & 1)) {
                    bad = true;
                    break;
                }
                const uint32_t sa = base + st * sh.stage, sb = sa + sh.nsub * sh.a_sub;
                const uint32_t bar = tc::smem_addr(&full[st]);
                tc::mbar_arrive_expect_tx(bar, static_cast<uint32_t>(sh.tx));
                const int dz = t / 9 - 1, dy = (t / 3) % 3 - 1, dx = t % 3 - 1;
                for (int j = 0; j < sh.nsub; ++j) {
                    tc::tma_load_4d(sa + j * sh.a_sub, &tm_in, bar, j * sh.bc, x0 + dx, y0 + dy, z + dz);
                    tc::tma_load_3d(sb + j * sh.b_sub, &tm_w, bar, j * sh.bc, t, 0);
                }
            }
            const int u = t - (S - 1);
            if (u >= 0) {
                const int su = u % S;
                if (!tc::mbar_wait(tc::smem_addr(&full[su]), (u / S) & 1)) {
                    bad = true;
                    break;
                }
                tc::fence_after_sync();
                const uint32_t sa = base + su * sh.stage, sb = sa + sh.nsub * sh.a_sub;
                for (int j = 0; j < sh.nsub; ++j)
                    for (int kk = 0; kk < sh.bc / 16; ++kk)
                        tc::mma_bf16(tmem, tc::smem_desc_swizzled(sa + j * sh.a_sub + kk * 32, row_bytes),
                                     tc::smem_desc_swizzled(sb + j * sh.b_sub + kk * 32, row_bytes), idesc,
                                     (u | j | kk) != 0);
                tc::mma_commit(tc::smem_addr(&empty[su]));
            }
        }
        tc::mma_commit(tc::smem_addr(&done));  // tracks every MMA issued above
        if (bad) issue_failed = 1;
    }
    int bad = 0;
    if (tid == 0) bad = !tc::mbar_wait(tc::smem_addr(&done), 0) || issue_failed;
    bad = __syncthreads_or(bad);
    tc::fence_after_sync();
    if (!bad) {
        const int x = x0 + (tid & (kTmaTileX - 1)), y = y0 + tid / kTmaTileX;
        const bool row_ok = x < p.nx && y < p.ny;
        const long long v = (static_cast<long long>(z) * p.ny + y) * p.nx + x;
        conv_epilogue(p, tmem + (static_cast<uint32_t>(warp * 32) << 16), v, row_ok);
    } else if (tid == 0) {
        atomicExch(p.status, 1);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem, ncols);
    }
}

struct ConvWgradArgs {
    const bf16* in;  // forward input, [nz>>up][ny>>up][nx>>up][cin]
    int cin, cin_log2, up;
    const bf16* dz;  // gradient at the conv output (before bias/ReLU), [V][cout]
    int cout;
    int nx, ny, nz;
    float* dw;       // [cout][27][cin], accumulated
    int chunks_per_cta;
    int* status;
};

__global__ void __launch_bounds__(kThreads) conv3_wgrad_kernel(ConvWgradArgs p)
{
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t mbar[2];
    __shared__ uint32_t tmem_slot;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int R = 27 * p.cin;
    const int m0 = blockIdx.x * tc::kTileM;
    const long long V = static_cast<long long>(p.nx) * p.ny * p.nz;
    const long long nchunks = (V + kChunk - 1) / kChunk;
    const long long c_begin = static_cast<long long>(blockIdx.y) * p.chunks_per_cta;
    const long long c_end = c_begin + p.chunks_per_cta < nchunks ? c_begin + p.chunks_per_cta : nchunks;
    const uint32_t ncols = tc::tmem_columns(p.cout);
    const int a_bytes = tc::kTileM * kChunk * 2;
    const int stage_bytes = a_bytes + p.cout * kChunk * 2;
    constexpr uint32_t kSbo = (kChunk / 8) * 128;  // next 8 rows along M (N): past all K groups

    if (warp == 0) tc::tmem_alloc(tc::smem_addr(&tmem_slot), ncols);
    if (tid == 0) {
        tc::mbar_init(tc::smem_addr(&mbar[0]), 1);
        tc::mbar_init(tc::smem_addr(&mbar[1]), 1);
        tc::mbar_init_fence();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tmem_slot;
    Pipe pp{{tc::smem_addr(&mbar[0]), tc::smem_addr(&mbar[1])}, {0, 0}, {0, 0}};
    const int sx = p.nx >> p.up, sy = p.ny >> p.up;
    const uint32_t idesc = tc::idesc_bf16_f32(p.cout, true);
    const int b_units = (p.cout >> 3) * kChunk;
    bool ok = true;
    int it = 0;
    for (long long ch = c_begin; ch < c_end; ++ch, ++it) {
        const int b = it & 1;
        if (!stage_free(pp, b)) {
            ok = false;
            break;
        }
        uint8_t* sa = smem + b * stage_bytes;
        uint8_t* sb = sa + a_bytes;
        const long long vb = ch * kChunk;
        // A: rows m = (tap, channel) of this tile, K = voxels; 16-byte unit = 8 channels of one voxel.
        // Thread tid always handles voxel k = tid % 64 of the stage (units j*128 + tid), so its
        // coordinates are computed once per stage; row groups g = 2j + tid / 64.
        {
            const int k = tid & (kChunk - 1);
            const long long vv = vb + k;
            const bool vok = vv < V;
            const int vi = static_cast<int>(vok ? vv : 0);
            const int x = vi % p.nx, r = vi / p.nx;
            const int y = r % p.ny, z = r / p.ny;
            uint8_t* dst = sa + (k >> 3) * 128 + (k & 7) * 16;
#pragma unroll 4
            for (int j = 0; j < (tc::kTileM / 8) * kChunk / kThreads; ++j) {
                const int g = 2 * j + (tid >> 6);
                const int m = m0 + g * 8;
                uint4 val = make_uint4(0, 0, 0, 0);
                if (vok && m < R) {
                    const int tap = m >> p.cin_log2, ci = m & (p.cin - 1);
                    const int zz = z + tap / 9 - 1, yy = y + (tap / 3) % 3 - 1, xx = x + tap % 3 - 1;
                    if (zz >= 0 && zz < p.nz && yy >= 0 && yy < p.ny && xx >= 0 && xx < p.nx) {
                        const size_t sv = (static_cast<size_t>(zz >> p.up) * sy + (yy >> p.up)) * sx + (xx >> p.up);
                        val = __ldg(reinterpret_cast<const uint4*>(p.in + sv * p.cin + ci));
                    }
                }
                *reinterpret_cast<uint4*>(dst + g * kSbo) = val;
            }
        }
        // B: N = output channels, K = voxels
        for (int u = tid; u < b_units; u += kThreads) {
            const int k = u & (kChunk - 1), g = u / kChunk;
            const long long vv = vb + k;
            const uint4 val = vv < V ? __ldg(reinterpret_cast<const uint4*>(p.dz + vv * p.cout + g * 8))
                                     : make_uint4(0, 0, 0, 0);
            *reinterpret_cast<uint4*>(sb + g * kSbo + (k >> 3) * 128 + (k & 7) * 16) = val;
        }
        tc::fence_proxy_async();
        __syncthreads();
        if (tid == 0) {
            tc::fence_after_sync();
            const uint32_t a0 = tc::smem_addr(sa), b0 = tc::smem_addr(sb);
            for (int j = 0; j < kChunk / 16; ++j)
                tc::mma_bf16(tmem, tc::smem_desc(a0 + j * 256, 128, kSbo), tc::smem_desc(b0 + j * 256, 128, kSbo),
                             idesc, (it | j) != 0);
            tc::mma_commit(pp.mbar[b]);
        }
        pp.issued[b]++;
    }
    ok = drain(pp) && ok;
    tc::fence_after_sync();
    if (ok && it > 0) {
        const uint32_t trow = tmem + (static_cast<uint32_t>(warp * 32) << 16);
        const int m = m0 + tid;
        for (int c0 = 0; c0 < p.cout; c0 += 16) {
            float acc[16];
            tc::tmem_load16(trow + c0, acc);
            if (m < R) {
#pragma unroll
                for (int i = 0; i < 16; ++i) atomicAdd(p.dw + static_cast<size_t>(c0 + i) * R + m, acc[i]);
            }
        }
    } else if (!ok && tid == 0) {
        atomicExch(p.status, 1);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem, ncols);
    }
}

// --------------------------------------------------------------------- elementwise kernels --

__global__ void pack_input_kernel(const float* __restrict__ x0, const uint8_t* __restrict__ hull, long long V,
                                  bf16* __restrict__ out)
{
    for (long long v = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; v < V;
         v += static_cast<long long>(gridDim.x) * blockDim.x) {
        uint4 a = make_uint4(pack_bf16(x0[v], hull[v] ? 1.f : 0.f), 0, 0, 0);
        reinterpret_cast<uint4*>(out + v * 16)[0] = a;
        reinterpret_cast<uint4*>(out + v * 16)[1] = make_uint4(0, 0, 0, 0);
    }
}

// 2x2x2 average; one thread per (coarse voxel, 8 channels).
__global__ void avgpool_kernel(const bf16* __restrict__ in, int nx, int ny, int nz, int c, bf16* __restrict__ out)
{
    const int cx = nx / 2, cy = ny / 2, cz = nz / 2, g = c / 8;
    const long long n = static_cast<long long>(cx) * cy * cz * g;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int cg = static_cast<int>(i % g);
        const long long cv = i / g;
        const int x = static_cast<int>(cv % cx), y = static_cast<int>((cv / cx) % cy), z = static_cast<int>(cv / (static_cast<long long>(cx) * cy));
        float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int d = 0; d < 8; ++d) {
            const long long fv = (static_cast<long long>(2 * z + (d >> 2)) * ny + 2 * y + ((d >> 1) & 1)) * nx + 2 * x + (d & 1);
            float f[8];
            unpack8(__ldg(reinterpret_cast<const uint4*>(in + fv * c) + cg), f);
#pragma unroll
            for (int k = 0; k < 8; ++k) s[k] += f[k];
        }
        uint4 o;
        o.x = pack_bf16(s[0] * 0.125f, s[1] * 0.125f);
        o.y = pack_bf16(s[2] * 0.125f, s[3] * 0.125f);
        o.z = pack_bf16(s[4] * 0.125f, s[5] * 0.125f);
        o.w = pack_bf16(s[6] * 0.125f, s[7] * 0.125f);
        reinterpret_cast<uint4*>(out + cv * c)[cg] = o;
    }
}

// Gradient through avg-pool and a skip: out = (dp[parent] / 8 + dskip) * (act > 0), fine grid.
__global__ void unpool_add_mask_kernel(const bf16* __restrict__ dp, const bf16* __restrict__ dskip,
                                       const bf16* __restrict__ act, int nx, int ny, int nz, int c,
                                       bf16* __restrict__ out)
{
    const int g = c / 8;
    const long long n = static_cast<long long>(nx) * ny * nz * g;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int cg = static_cast<int>(i % g);
        const long long v = i / g;
        const int x = static_cast<int>(v % nx), y = static_cast<int>((v / nx) % ny), z = static_cast<int>(v / (static_cast<long long>(nx) * ny));
        const long long pv = (static_cast<long long>(z / 2) * (ny / 2) + y / 2) * (nx / 2) + x / 2;
        float a[8], s[8], m[8];
        unpack8(__ldg(reinterpret_cast<const uint4*>(dp + pv * c) + cg), a);
        unpack8(__ldg(reinterpret_cast<const uint4*>(dskip + v * c) + cg), s);
        unpack8(__ldg(reinterpret_cast<const uint4*>(act + v * c) + cg), m);
        float r[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) r[k] = m[k] > 0.f ? a[k] * 0.125f + s[k] : 0.f;
        uint4 o;
        o.x = pack_bf16(r[0], r[1]);
        o.y = pack_bf16(r[2], r[3]);
        o.z = pack_bf16(r[4], r[5]);
        o.w = pack_bf16(r[6], r[7]);
        reinterpret_cast<uint4*>(out + v * c)[cg] = o;
    }
}

// Gradient through nearest x2 upsampling: out[coarse] = sum of the 8 fine children, * (act > 0).
__global__ void upsum_mask_kernel(const bf16* __restrict__ du, const bf16* __restrict__ act, int cx, int cy, int cz,
                                  int c, bf16* __restrict__ out)
{
    const int g = c / 8, nx = 2 * cx, ny = 2 * cy;
    const long long n = static_cast<long long>(cx) * cy * cz * g;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int cg = static_cast<int>(i % g);
        const long long cv = i / g;
        const int x = static_cast<int>(cv % cx), y = static_cast<int>((cv / cx) % cy), z = static_cast<int>(cv / (static_cast<long long>(cx) * cy));
        float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int d = 0; d < 8; ++d) {
            const long long fv = (static_cast<long long>(2 * z + (d >> 2)) * ny + 2 * y + ((d >> 1) & 1)) * nx + 2 * x + (d & 1);
            float f[8];
            unpack8(__ldg(reinterpret_cast<const uint4*>(du + fv * c) + cg), f);
#pragma unroll
            for (int k = 0; k < 8; ++k) s[k] += f[k];
        }
        float m[8];
        unpack8(__ldg(reinterpret_cast<const uint4*>(act + cv * c) + cg), m);
        uint4 o;
        o.x = pack_bf16(m[0] > 0.f ? s[0] : 0.f, m[1] > 0.f ? s[1] : 0.f);
        o.y = pack_bf16(m[2] > 0.f ? s[2] : 0.f, m[3] > 0.f ? s[3] : 0.f);
        o.z = pack_bf16(m[4] > 0.f ? s[4] : 0.f, m[5] > 0.f ? s[5] : 0.f);
        o.w = pack_bf16(m[6] > 0.f ? s[6] : 0.f, m[7] > 0.f ? s[7] : 0.f);
        reinterpret_cast<uint4*>(out + cv * c)[cg] = o;
    }
}

// db[c] += sum_v dz[v][c]; 256 threads, cout divides 256.
__global__ void bias_grad_kernel(const bf16* __restrict__ dz, int cout, long long V, float* __restrict__ db)
{
    __shared__ float red[256];
    const int c = threadIdx.x % cout, lanes = 256 / cout, off = threadIdx.x / cout;
    float s = 0.f;
    for (long long v = static_cast<long long>(blockIdx.x) * lanes + off; v < V; v += static_cast<long long>(gridDim.x) * lanes)
        s += __bfloat162float(dz[v * cout + c]);
    red[threadIdx.x] = s;
    __syncthreads();
    if (off == 0) {
        float t = 0.f;
        for (int l = 0; l < lanes; ++l) t += red[l * cout + c];
        atomicAdd(db + c, t);
    }
}

__global__ void count_kernel(const uint8_t* __restrict__ hull, long long V, unsigned long long* __restrict__ count)
{
    unsigned long long n = 0;
    for (long long v = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; v < V;
         v += static_cast<long long>(gridDim.x) * blockDim.x)
        n += hull[v] ? 1 : 0;
    for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(0xffffffffu, n, o);
    if ((threadIdx.x & 31) == 0 && n) atomicAdd(count, n);
}

// Masked mean-squared error over the hull voxels: loss += (y - t)^2 / count, and the gradient
// dL/dy = 2 (y - t) / count as channel 0 of a 16-channel bf16 tensor (other channels 0).
__global__ void loss_kernel(const float* __restrict__ y, const float* __restrict__ target, const uint8_t* __restrict__ hull,
                            long long V, const unsigned long long* __restrict__ count, bf16* __restrict__ dy,
                            double* __restrict__ loss)
{
    const double inv = *count ? 1.0 / static_cast<double>(*count) : 0.0;
    double acc = 0.0;
    for (long long v = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; v < V;
         v += static_cast<long long>(gridDim.x) * blockDim.x) {
        const float d = hull[v] ? y[v] - target[v] : 0.f;
        acc += static_cast<double>(d) * d;
        const float g = static_cast<float>(2.0 * d * inv);
        reinterpret_cast<uint4*>(dy + v * 16)[0] = make_uint4(pack_bf16(g, 0.f), 0, 0, 0);
        reinterpret_cast<uint4*>(dy + v * 16)[1] = make_uint4(0, 0, 0, 0);
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, acc * inv);
}

__global__ void nonfinite_kernel(const float* __restrict__ y, long long V, unsigned long long* __restrict__ count)
{
    unsigned long long n = 0;
    for (long long v = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; v < V;
         v += static_cast<long long>(gridDim.x) * blockDim.x)
        n += isfinite(y[v]) ? 0 : 1;
    for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(0xffffffffu, n, o);
    if ((threadIdx.x & 31) == 0 && n) atomicAdd(count, n);
}

__global__ void adam_kernel(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ s, long long n, float lr, float b1, float b2, float eps, float bc1,
                            float bc2)
{
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float si = b2 * s[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        s[i] = si;
        w[i] -= lr * (mi / bc1) / (sqrtf(si / bc2) + eps);
    }
}

// bf16 copies of one layer's weights: W[co][t][ci] and the data-gradient form W'[ci][26-t][co].
__global__ void emit_weights_kernel(const float* __restrict__ w, int cin, int cout, bf16* __restrict__ wb,
                                    bf16* __restrict__ wt)
{
    const int n = cout * 27 * cin;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int ci = i % cin, t = (i / cin) % 27, co = i / (27 * cin);
        const bf16 h = __float2bfloat16_rn(w[i]);
        wb[i] = h;
        wt[(static_cast<size_t>(ci) * 27 + (26 - t)) * cout + co] = h;
    }
}

// ------------------------------------------------------------------------ launch helpers --

int grid_for(long long n, int threads)
{
    long long b = (n + threads - 1) / threads;
    if (b > 148LL * 16) b = 148LL * 16;
    return static_cast<int>(b < 1 ? 1 : b);
}

// Dynamic shared memory for a conv CTA: its two stages, raised when needed so that no more CTAs
// share an SM than its TMEM columns can hold at once.
int conv_smem(int stage_bytes, int cout)
{
    const int per_sm = kTmemColumns / static_cast<int>(tc::tmem_columns(cout));
    const int floor_bytes = kSmemPerSm / (per_sm + 1) + 1;
    const int need = 2 * stage_bytes;
    return need > floor_bytes ? need : floor_bytes;
}

cudaError_t set_smem_limits()
{
    static bool done[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev >= 0 && dev < 64 && done[dev]) return cudaSuccess;
    e = cudaFuncSetAttribute(conv3_fwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(conv3_wgrad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(conv3_fwd_tma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kTmaSmemLimit);
    if (e == cudaSuccess && dev >= 0 && dev < 64) done[dev] = true;
    return e;
}

bool valid_channels(int c) { return c == 16 || c == 32 || c == 64 || c == 128; }

// Tensor maps of the TMA convolution: the activation [nz][ny][nx][c] as a 4-D tensor (c innermost)
// with a (bc, 32, 4, 1) box, and the weights [cout][27][cin] as a 3-D tensor with a (bc, 1, cout)
// box; the swizzle matches the box row (bc * 2 bytes).
// cuTensorMapEncodeTiled through the runtime's driver entry point, so the library does not link the
// driver library itself (it still loads on machines without a GPU); null if unavailable.
PFN_cuTensorMapEncodeTiled tensor_map_encoder()
{
    static PFN_cuTensorMapEncodeTiled fn = nullptr;
    static bool looked = false;
    if (!looked) {
        looked = true;
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled>(f);
        else
            cudaGetLastError();
    }
    return fn;
}

bool encode_conv_maps(const ConvFwdArgs& a, int bc, CUtensorMap* act, CUtensorMap* w)
{
    const PFN_cuTensorMapEncodeTiled cuTensorMapEncodeTiled = tensor_map_encoder();
    if (!cuTensorMapEncodeTiled) return false;
    const CUtensorMapSwizzle sw = bc == 16 ? CU_TENSOR_MAP_SWIZZLE_32B
                                : bc == 32 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_128B;
    const cuuint64_t c = a.cin;
    cuuint64_t adim[4] = {c, (cuuint64_t)a.nx, (cuuint64_t)a.ny, (cuuint64_t)a.nz};
    cuuint64_t astr[3] = {c * 2, c * 2 * a.nx, c * 2 * a.nx * a.ny};
    cuuint32_t abox[4] = {(cuuint32_t)bc, kTmaTileX, kTmaTileY, 1};
    cuuint32_t one[4] = {1, 1, 1, 1};
    if (cuTensorMapEncodeTiled(act, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<bf16*>(a.in), adim, astr, abox, one,
                               CU_TENSOR_MAP_INTERLEAVE_NONE, sw, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return false;
    cuuint64_t wdim[3] = {c, 27, (cuuint64_t)a.cout};
    cuuint64_t wstr[2] = {c * 2, c * 2 * 27};
    cuuint32_t wbox[3] = {(cuuint32_t)bc, 1, (cuuint32_t)a.cout};
    return cuTensorMapEncodeTiled(w, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<bf16*>(a.weight), wdim, wstr, wbox,
                                  one, CU_TENSOR_MAP_INTERLEAVE_NONE, sw, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

cudaError_t launch_conv_fwd(const ConvFwdArgs& a, cudaStream_t s)
{
    cudaError_t e = set_smem_limits();
    if (e != cudaSuccess) return e;
    // TMA path: inputs at full resolution whose base addresses meet TMA's 16-byte rule
    const bool aligned = (reinterpret_cast<uintptr_t>(a.in) & 15) == 0 && (reinterpret_cast<uintptr_t>(a.weight) & 15) == 0;
    if (!a.up && aligned) {
        const TmaConvShape sh = tma_conv_shape(a.cin, a.cout);
        CUtensorMap act, w;
        if (sh.stages >= 2 && encode_conv_maps(a, sh.bc, &act, &w)) {
            const int per_sm = kTmemColumns / static_cast<int>(tc::tmem_columns(a.cout));
            int smem = sh.stages * sh.stage + 1024;
            const int floor_bytes = kSmemPerSm / (per_sm + 1) + 1;
            if (smem < floor_bytes) smem = floor_bytes;
            const long long tiles = static_cast<long long>((a.nx + kTmaTileX - 1) / kTmaTileX) *
                                    ((a.ny + kTmaTileY - 1) / kTmaTileY) * a.nz;
            conv3_fwd_tma_kernel<<<static_cast<unsigned>(tiles), kThreads, smem, s>>>(act, w, a);
            return cudaGetLastError();
        }
    }
    const long long V = static_cast<long long>(a.nx) * a.ny * a.nz;
    const int blocks = static_cast<int>((V + tc::kTileM - 1) / tc::kTileM);
    conv3_fwd_kernel<<<blocks, kThreads, conv_smem(conv_stage_bytes(a.cin, a.cout), a.cout), s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_conv_wgrad(ConvWgradArgs a, cudaStream_t s)
{
    cudaError_t e = set_smem_limits();
    if (e != cudaSuccess) return e;
    a.cin_log2 = a.cin == 16 ? 4 : a.cin == 32 ? 5 : a.cin == 64 ? 6 : 7;
    const long long V = static_cast<long long>(a.nx) * a.ny * a.nz;
    const int m_tiles = (27 * a.cin + tc::kTileM - 1) / tc::kTileM;
    const long long chunks = (V + kChunk - 1) / kChunk;
    // about six resident CTAs per SM (the two 18-34 KB stages allow six to eight)
    long long splits = (148LL * PCT_WGRAD_CTAS_PER_SM + m_tiles - 1) / m_tiles;
    if (splits > chunks) splits = chunks;
    if (splits < 1) splits = 1;
    a.chunks_per_cta = static_cast<int>((chunks + splits - 1) / splits);
    splits = (chunks + a.chunks_per_cta - 1) / a.chunks_per_cta;
    const int stage = tc::kTileM * kChunk * 2 + a.cout * kChunk * 2;
    conv3_wgrad_kernel<<<dim3(m_tiles, static_cast<unsigned>(splits)), kThreads, conv_smem(stage, a.cout), s>>>(a);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------ the network --

struct LayerSpec {
    int cin, cout, level, input, up, residual;  // input/residual: activation index (-1 = network input / none)
};

// Activation k is the output of layer k; pooled tensors are separate buffers (pool[level]).
constexpr int kLayers = 15;
constexpr int kPoolInput = 100;  // input code: pool[level] of the layer's level
const LayerSpec kSpec[kLayers] = {
    {16, 16, 0, -1, 0, -1},          {16, 16, 0, 0, 0, -1},            // e1a, e1
    {16, 32, 1, kPoolInput, 0, -1},  {32, 32, 1, 2, 0, -1},            // e2a, e2
    {32, 64, 2, kPoolInput, 0, -1},  {64, 64, 2, 4, 0, -1},            // e3a, e3
    {64, 128, 3, kPoolInput, 0, -1}, {128, 128, 3, 6, 0, -1},          // e4a, e4
    {128, 64, 2, 7, 1, 5},           {64, 64, 2, 8, 0, -1},            // d3a (+e3), d3
    {64, 32, 1, 9, 1, 3},            {32, 32, 1, 10, 0, -1},           // d2a (+e2), d2
    {32, 16, 0, 11, 1, 1},           {16, 16, 0, 12, 0, -1},           // d1a (+e1), d1
    {16, 16, 0, 13, 0, -1},                                            // output (channel 0)
};

}  // namespace unet
}  // namespace pct

using namespace pct::unet;

struct pct_unet {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int nx[4], ny[4], nz[4];
    long long nv[4];
    size_t w_off[kLayers], b_off[kLayers];
    size_t n_params = 0;
    float *params = nullptr, *grads = nullptr, *adam_m = nullptr, *adam_v = nullptr;
    bf16 *wb = nullptr, *wt = nullptr;  // bf16 weights, forward and data-gradient forms
    size_t wb_off[kLayers];
    bf16* input = nullptr;
    bf16* act[kLayers] = {};
    bf16* pool[4] = {};
    bf16* dz[kLayers] = {};
    bf16* tmp = nullptr;
    float* y = nullptr;
    unsigned long long* count = nullptr;
    double* loss = nullptr;
    int* status = nullptr;
    long long step = 0;
    std::string err;
};

namespace {

pct_status fail(pct_unet* n, pct_status s, const std::string& msg)
{
    if (n) n->err = msg;
    return s;
}

pct_status cuda_fail(pct_unet* n, cudaError_t e, const char* where)
{
    return fail(n, PCT_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define UNET_CK(call, where)                              \
    do {                                                  \
        const cudaError_t e_ = (call);                    \
        if (e_ != cudaSuccess) return cuda_fail(n, e_, where); \
    } while (0)

void release(pct_unet* n)
{
    void* ptrs[] = {n->params, n->grads, n->adam_m, n->adam_v, n->wb, n->wt, n->input, n->tmp, n->y,
                    n->count, n->loss, n->status};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    for (int l = 0; l < kLayers; ++l) {
        if (n->act[l]) cudaFree(n->act[l]);
        if (n->dz[l]) cudaFree(n->dz[l]);
    }
    for (int l = 0; l < 4; ++l)
        if (n->pool[l]) cudaFree(n->pool[l]);
    if (n->own_stream && n->stream) cudaStreamDestroy(n->stream);
}

pct_status emit_weights(pct_unet* n, cudaStream_t s)
{
    for (int l = 0; l < kLayers; ++l) {
        const LayerSpec& L = kSpec[l];
        emit_weights_kernel<<<grid_for(static_cast<long long>(L.cout) * 27 * L.cin, 256), 256, 0, s>>>(
            n->params + n->w_off[l], L.cin, L.cout, n->wb + n->wb_off[l], n->wt + n->wb_off[l]);
    }
    UNET_CK(cudaGetLastError(), "emit_weights_kernel");
    return PCT_OK;
}

const bf16* layer_input(pct_unet* n, int l)
{
    const LayerSpec& L = kSpec[l];
    if (L.input == -1) return n->input;
    if (L.input == kPoolInput) return n->pool[L.level];
    return n->act[L.input];
}

pct_status check_status(pct_unet* n, cudaStream_t s)
{
    int st = 0;
    UNET_CK(cudaMemcpyAsync(&st, n->status, sizeof(int), cudaMemcpyDeviceToHost, s), "status copy");
    UNET_CK(cudaStreamSynchronize(s), "synchronize");
    if (st) return fail(n, PCT_ERR_TIMEOUT, "a tensor-core pipeline wait expired");
    return PCT_OK;
}

// Forward pass: image = x0 + hull * network(x0, hull); all on stream s.
pct_status forward(pct_unet* n, const float* x0, const uint8_t* hull, float* image, cudaStream_t s)
{
    pack_input_kernel<<<grid_for(n->nv[0], 256), 256, 0, s>>>(x0, hull, n->nv[0], n->input);
    UNET_CK(cudaGetLastError(), "pack_input_kernel");
    for (int l = 0; l < kLayers; ++l) {
        const LayerSpec& L = kSpec[l];
        if (L.input == kPoolInput) {
            const int f = L.level - 1;  // pool the previous level's last encoder output
            const int src = 2 * f + 1;
            avgpool_kernel<<<grid_for(n->nv[L.level] * (kSpec[src].cout / 8), 256), 256, 0, s>>>(
                n->act[src], n->nx[f], n->ny[f], n->nz[f], kSpec[src].cout, n->pool[L.level]);
            UNET_CK(cudaGetLastError(), "avgpool_kernel");
        }
        ConvFwdArgs a{};
        a.in = layer_input(n, l);
        a.cin = L.cin;
        a.up = L.up;
        a.weight = n->wb + n->wb_off[l];
        a.cout = L.cout;
        a.nx = n->nx[L.level];
        a.ny = n->ny[L.level];
        a.nz = n->nz[L.level];
        a.bias = n->params + n->b_off[l];
        a.residual = L.residual >= 0 ? n->act[L.residual] : nullptr;
        a.status = n->status;
        if (l == kLayers - 1) {
            a.base = x0;
            a.hull = hull;
            a.image = image;
        } else {
            a.relu = 1;
            a.out = n->act[l];
        }
        UNET_CK(launch_conv_fwd(a, s), "conv3_fwd_kernel");
    }
    return PCT_OK;
}

// Backward pass from n->dz[14] (dL/dy in channel 0): fills n->grads.
pct_status backward(pct_unet* n, cudaStream_t s)
{
    UNET_CK(cudaMemsetAsync(n->grads, 0, n->n_params * sizeof(float), s), "grad clear");
    for (int l = kLayers - 1; l >= 0; --l) {
        const LayerSpec& L = kSpec[l];
        const int nx = n->nx[L.level], ny = n->ny[L.level], nz = n->nz[L.level];
        // weights and bias
        ConvWgradArgs w{};
        w.in = layer_input(n, l);
        w.cin = L.cin;
        w.up = L.up;
        w.dz = n->dz[l];
        w.cout = L.cout;
        w.nx = nx;
        w.ny = ny;
        w.nz = nz;
        w.dw = n->grads + n->w_off[l];
        w.status = n->status;
        UNET_CK(launch_conv_wgrad(w, s), "conv3_wgrad_kernel");
        bias_grad_kernel<<<296, 256, 0, s>>>(n->dz[l], L.cout, n->nv[L.level], n->grads + n->b_off[l]);
        UNET_CK(cudaGetLastError(), "bias_grad_kernel");
        if (l == 0) break;
        // data gradient: conv of dz with the flipped, transposed weights
        ConvFwdArgs d{};
        d.cin = L.cout;
        d.cout = L.cin;
        d.in = n->dz[l];
        d.weight = n->wt + n->wb_off[l];
        d.nx = nx;
        d.ny = ny;
        d.nz = nz;
        d.status = n->status;
        const bool into_tmp = L.up || L.input == kPoolInput;
        if (into_tmp) {
            d.out = n->tmp;  // gradient wrt the upsampled / pooled tensor
        } else {
            d.out = n->dz[L.input];
            d.mask = n->act[L.input];  // ReLU of the producing layer
        }
        UNET_CK(launch_conv_fwd(d, s), "conv3_fwd_kernel (data gradient)");
        if (L.up) {
            const int src = L.input, cl = L.level + 1;
            upsum_mask_kernel<<<grid_for(n->nv[cl] * (L.cin / 8), 256), 256, 0, s>>>(
                n->tmp, n->act[src], n->nx[cl], n->ny[cl], n->nz[cl], L.cin, n->dz[src]);
            UNET_CK(cudaGetLastError(), "upsum_mask_kernel");
        } else if (L.input == kPoolInput) {
            const int f = L.level - 1, src = 2 * f + 1;
            // the decoder layer that adds act[src] as its residual
            int skip = -1;
            for (int k = 0; k < kLayers; ++k)
                if (kSpec[k].residual == src) skip = k;
            unpool_add_mask_kernel<<<grid_for(n->nv[f] * (L.cin / 8), 256), 256, 0, s>>>(
                n->tmp, n->dz[skip], n->act[src], n->nx[f], n->ny[f], n->nz[f], L.cin, n->dz[src]);
            UNET_CK(cudaGetLastError(), "unpool_add_mask_kernel");
        }
    }
    return PCT_OK;
}

pct_status loss_and_gradient(pct_unet* n, const float* x0, const uint8_t* hull, const float* target, double* loss_out,
                             cudaStream_t s)
{
    UNET_CK(cudaMemsetAsync(n->status, 0, sizeof(int), s), "status clear");
    pct_status st = forward(n, x0, hull, n->y, s);
    if (st != PCT_OK) return st;
    UNET_CK(cudaMemsetAsync(n->count, 0, sizeof(unsigned long long), s), "count clear");
    UNET_CK(cudaMemsetAsync(n->loss, 0, sizeof(double), s), "loss clear");
    count_kernel<<<grid_for(n->nv[0], 256), 256, 0, s>>>(hull, n->nv[0], n->count);
    loss_kernel<<<grid_for(n->nv[0], 256), 256, 0, s>>>(n->y, target, hull, n->nv[0], n->count, n->dz[kLayers - 1],
                                                       n->loss);
    UNET_CK(cudaGetLastError(), "loss_kernel");
    st = backward(n, s);
    if (st != PCT_OK) return st;
    if (loss_out) UNET_CK(cudaMemcpyAsync(loss_out, n->loss, sizeof(double), cudaMemcpyDeviceToHost, s), "loss copy");
    return check_status(n, s);
}

}  // namespace

extern "C" {

pct_status pct_unet_create(int columns, int rows, int slices, int64_t seed, int device, pct_unet** out)
{
    if (!out) return PCT_ERR_ARG;
    *out = nullptr;
    if (columns <= 0 || rows <= 0 || slices <= 0 || columns % 8 || rows % 8 || slices % 8) return PCT_ERR_ARG;
    pct_unet* n = new pct_unet();
    n->device = device;
    pct_status st = PCT_OK;
    auto ck = [&](cudaError_t e, const char* where) {
        if (e != cudaSuccess && st == PCT_OK) st = cuda_fail(n, e, where);
        return e == cudaSuccess;
    };
    if (ck(cudaSetDevice(device), "cudaSetDevice") && ck(cudaStreamCreateWithFlags(&n->stream, cudaStreamNonBlocking), "stream")) {
        n->own_stream = true;
        for (int l = 0; l < 4; ++l) {
            n->nx[l] = columns >> l;
            n->ny[l] = rows >> l;
            n->nz[l] = slices >> l;
            n->nv[l] = static_cast<long long>(n->nx[l]) * n->ny[l] * n->nz[l];
        }
        size_t off = 0, boff = 0;
        for (int l = 0; l < kLayers; ++l) {
            n->w_off[l] = off;
            off += static_cast<size_t>(kSpec[l].cout) * 27 * kSpec[l].cin;
            n->b_off[l] = off;
            off += kSpec[l].cout;
            n->wb_off[l] = boff;
            boff += static_cast<size_t>(kSpec[l].cout) * 27 * kSpec[l].cin;
        }
        n->n_params = off;
        // He-normal initial weights from a seeded generator; padding channels of the input layer,
        // and the whole output layer, start at zero (the untrained network returns x_0).
        std::vector<float> h(off, 0.f);
        std::mt19937_64 rng(static_cast<uint64_t>(seed));
        for (int l = 0; l < kLayers - 1; ++l) {
            const int fan_in = 27 * (l == 0 ? 2 : kSpec[l].cin);
            std::normal_distribution<float> nd(0.f, std::sqrt(2.f / fan_in));
            for (int co = 0; co < kSpec[l].cout; ++co)
                for (int t = 0; t < 27; ++t)
                    for (int ci = 0; ci < kSpec[l].cin; ++ci) {
                        const float w = nd(rng);
                        if (l != 0 || ci < 2) h[n->w_off[l] + (static_cast<size_t>(co) * 27 + t) * kSpec[l].cin + ci] = w;
                    }
        }
        const size_t pbytes = off * sizeof(float);
        ck(cudaMalloc(&n->params, pbytes), "cudaMalloc params");
        ck(cudaMalloc(&n->grads, pbytes), "cudaMalloc grads");
        ck(cudaMalloc(&n->adam_m, pbytes), "cudaMalloc adam");
        ck(cudaMalloc(&n->adam_v, pbytes), "cudaMalloc adam");
        ck(cudaMalloc(&n->wb, boff * sizeof(bf16)), "cudaMalloc weights");
        ck(cudaMalloc(&n->wt, boff * sizeof(bf16)), "cudaMalloc weights");
        ck(cudaMalloc(&n->input, n->nv[0] * 16 * sizeof(bf16)), "cudaMalloc input");
        for (int l = 0; l < kLayers; ++l) {
            const size_t bytes = n->nv[kSpec[l].level] * kSpec[l].cout * sizeof(bf16);
            ck(cudaMalloc(&n->act[l], bytes), "cudaMalloc activations");
            ck(cudaMalloc(&n->dz[l], bytes), "cudaMalloc gradients");
        }
        for (int l = 1; l < 4; ++l) ck(cudaMalloc(&n->pool[l], n->nv[l] * kSpec[2 * l].cin * sizeof(bf16)), "cudaMalloc pool");
        // largest data-gradient scratch: L0 x 32 (upsampled into d1a), L1 x 64, L2 x 128, pools
        size_t tmp = 0;
        for (int l = 0; l < kLayers; ++l)
            if (kSpec[l].up || kSpec[l].input == kPoolInput) {
                const size_t b = n->nv[kSpec[l].level] * kSpec[l].cin;
                if (b > tmp) tmp = b;
            }
        ck(cudaMalloc(&n->tmp, tmp * sizeof(bf16)), "cudaMalloc scratch");
        ck(cudaMalloc(&n->y, n->nv[0] * sizeof(float)), "cudaMalloc output");
        ck(cudaMalloc(&n->count, sizeof(unsigned long long)), "cudaMalloc");
        ck(cudaMalloc(&n->loss, sizeof(double)), "cudaMalloc");
        ck(cudaMalloc(&n->status, sizeof(int)), "cudaMalloc");
        if (st == PCT_OK) {
            ck(cudaMemcpyAsync(n->params, h.data(), pbytes, cudaMemcpyHostToDevice, n->stream), "params copy");
            ck(cudaMemsetAsync(n->adam_m, 0, pbytes, n->stream), "memset");
            ck(cudaMemsetAsync(n->adam_v, 0, pbytes, n->stream), "memset");
            ck(cudaMemsetAsync(n->status, 0, sizeof(int), n->stream), "memset");
            if (st == PCT_OK) st = emit_weights(n, n->stream);
            ck(cudaStreamSynchronize(n->stream), "synchronize");
        }
    }
    if (st != PCT_OK) {
        const cudaError_t e = cudaGetLastError();
        (void)e;
        release(n);
        delete n;
        return st;
    }
    *out = n;
    return PCT_OK;
}

pct_status pct_unet_destroy(pct_unet* n)
{
    if (!n) return PCT_OK;
    cudaSetDevice(n->device);
    if (n->stream) cudaStreamSynchronize(n->stream);
    release(n);
    delete n;
    return PCT_OK;
}

const char* pct_unet_last_error(const pct_unet* n) { return n ? n->err.c_str() : "null network"; }

pct_status pct_unet_param_count(const pct_unet* n, int64_t* count)
{
    if (!n || !count) return PCT_ERR_ARG;
    *count = static_cast<int64_t>(n->n_params);
    return PCT_OK;
}

pct_status pct_unet_get_params(pct_unet* n, float* host, int64_t count)
{
    if (!n || !host || count != static_cast<int64_t>(n->n_params)) return fail(n, PCT_ERR_ARG, "parameter count");
    UNET_CK(cudaSetDevice(n->device), "cudaSetDevice");
    UNET_CK(cudaMemcpyAsync(host, n->params, n->n_params * sizeof(float), cudaMemcpyDeviceToHost, n->stream), "copy");
    UNET_CK(cudaStreamSynchronize(n->stream), "synchronize");
    return PCT_OK;
}

pct_status pct_unet_set_params(pct_unet* n, const float* host, int64_t count)
{
    if (!n || !host || count != static_cast<int64_t>(n->n_params)) return fail(n, PCT_ERR_ARG, "parameter count");
    UNET_CK(cudaSetDevice(n->device), "cudaSetDevice");
    UNET_CK(cudaMemcpyAsync(n->params, host, n->n_params * sizeof(float), cudaMemcpyHostToDevice, n->stream), "copy");
    UNET_CK(cudaMemsetAsync(n->adam_m, 0, n->n_params * sizeof(float), n->stream), "memset");
    UNET_CK(cudaMemsetAsync(n->adam_v, 0, n->n_params * sizeof(float), n->stream), "memset");
    n->step = 0;
    const pct_status st = emit_weights(n, n->stream);
    if (st != PCT_OK) return st;
    UNET_CK(cudaStreamSynchronize(n->stream), "synchronize");
    return PCT_OK;
}

pct_status pct_unet_forward(pct_unet* n, const float* x0, const uint8_t* hull, float* image)
{
    if (!n || !x0 || !hull || !image) return fail(n, PCT_ERR_ARG, "null pointer");
    UNET_CK(cudaSetDevice(n->device), "cudaSetDevice");
    UNET_CK(cudaMemsetAsync(n->status, 0, sizeof(int), n->stream), "status clear");
    const pct_status st = forward(n, x0, hull, image, n->stream);
    if (st != PCT_OK) return st;
    return check_status(n, n->stream);
}

pct_status pct_unet_gradients(pct_unet* n, const float* x0, const uint8_t* hull, const float* target, float* grads_host,
                              double* loss)
{
    if (!n || !x0 || !hull || !target) return fail(n, PCT_ERR_ARG, "null pointer");
    UNET_CK(cudaSetDevice(n->device), "cudaSetDevice");
    const pct_status st = loss_and_gradient(n, x0, hull, target, loss, n->stream);
    if (st != PCT_OK) return st;
    if (grads_host) {
        UNET_CK(cudaMemcpyAsync(grads_host, n->grads, n->n_params * sizeof(float), cudaMemcpyDeviceToHost, n->stream),
                "gradient copy");
        UNET_CK(cudaStreamSynchronize(n->stream), "synchronize");
    }
    return PCT_OK;
}

pct_status pct_unet_train_step(pct_unet* n, const float* x0, const uint8_t* hull, const float* target, float lr,
                               double* loss)
{
    if (!n || !x0 || !hull || !target || !(lr > 0.f)) return fail(n, PCT_ERR_ARG, "invalid argument");
    UNET_CK(cudaSetDevice(n->device), "cudaSetDevice");
    pct_status st = loss_and_gradient(n, x0, hull, target, loss, n->stream);
    if (st != PCT_OK) return st;
    n->step++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float bc1 = 1.f - std::pow(b1, static_cast<float>(n->step));
    const float bc2 = 1.f - std::pow(b2, static_cast<float>(n->step));
    adam_kernel<<<grid_for(static_cast<long long>(n->n_params), 256), 256, 0, n->stream>>>(
        n->params, n->grads, n->adam_m, n->adam_v, static_cast<long long>(n->n_params), lr, b1, b2, 1e-8f, bc1, bc2);
    UNET_CK(cudaGetLastError(), "adam_kernel");
    st = emit_weights(n, n->stream);
    if (st != PCT_OK) return st;
    UNET_CK(cudaStreamSynchronize(n->stream), "synchronize");
    return PCT_OK;
}

pct_status pct_learned_initial_iterate(pct_ctx* ctx, pct_unet* n)
{
    if (!ctx || !n) return PCT_ERR_ARG;
    const pct::Geometry& g = ctx->geo;
    if (g.columns != n->nx[0] || g.rows != n->ny[0] || g.slices != n->nz[0]) {
        pct::context_set_error(ctx, "pct_learned_initial_iterate: network grid differs from the context's");
        return PCT_ERR_ARG;
    }
    const uint8_t* hull = pct::preproc_hull(ctx);
    if (!hull || !ctx->d_x) {
        pct::context_set_error(ctx, "pct_learned_initial_iterate: needs the hull and x_0 (run preprocessing first)");
        return PCT_ERR_STATE;
    }
    if (n->device != ctx->device) {
        pct::context_set_error(ctx, "pct_learned_initial_iterate: network and context on different devices");
        return PCT_ERR_ARG;
    }
    // image = x_0 + hull * network(x_0, hull) into the network's output buffer; it replaces the
    // context's image only if every voxel is finite, otherwise the FBP start x_0 is kept.
    cudaMemsetAsync(n->status, 0, sizeof(int), ctx->stream);
    pct_status st = forward(n, ctx->d_x, hull, n->y, ctx->stream);
    if (st == PCT_OK) {
        cudaMemsetAsync(n->count, 0, sizeof(unsigned long long), ctx->stream);
        nonfinite_kernel<<<grid_for(n->nv[0], 256), 256, 0, ctx->stream>>>(n->y, n->nv[0], n->count);
        unsigned long long bad = 0;
        cudaMemcpyAsync(&bad, n->count, sizeof(bad), cudaMemcpyDeviceToHost, ctx->stream);
        st = check_status(n, ctx->stream);
        if (st == PCT_OK && bad) st = fail(n, PCT_ERR_STATE, std::to_string(bad) + " non-finite voxels; the FBP start is kept");
        if (st == PCT_OK) {
            const cudaError_t e = cudaMemcpyAsync(ctx->d_x, n->y, n->nv[0] * sizeof(float), cudaMemcpyDeviceToDevice, ctx->stream);
            if (e != cudaSuccess) st = cuda_fail(n, e, "image copy");
        }
    }
    if (st != PCT_OK) pct::context_set_error(ctx, ("pct_learned_initial_iterate: " + n->err).c_str());
    return st;
}

// ---------------------------------------------------------------- single convolutions --

pct_status pct_conv3d_bf16(const uint16_t* in, int cin, int columns, int rows, int slices, int upsample,
                           const uint16_t* weight, int cout, const float* bias, const uint16_t* residual,
                           const uint16_t* mask, int relu, uint16_t* out, void* stream)
{
    if (!in || !weight || !out || !valid_channels(cin) || !valid_channels(cout) || columns <= 0 || rows <= 0 ||
        slices <= 0 || (upsample && (columns % 2 || rows % 2 || slices % 2)))
        return PCT_ERR_ARG;
    int* status = nullptr;
    if (cudaMalloc(&status, sizeof(int)) != cudaSuccess) return PCT_ERR_NOMEM;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    ConvFwdArgs a{};
    a.in = reinterpret_cast<const bf16*>(in);
    a.cin = cin;
    a.up = upsample ? 1 : 0;
    a.weight = reinterpret_cast<const bf16*>(weight);
    a.cout = cout;
    a.nx = columns;
    a.ny = rows;
    a.nz = slices;
    a.bias = bias;
    a.residual = reinterpret_cast<const bf16*>(residual);
    a.mask = reinterpret_cast<const bf16*>(mask);
    a.relu = relu;
    a.out = reinterpret_cast<bf16*>(out);
    a.status = status;
    pct_status st = PCT_OK;
    if (cudaMemsetAsync(status, 0, sizeof(int), s) != cudaSuccess || launch_conv_fwd(a, s) != cudaSuccess) st = PCT_ERR_CUDA;
    int h = 0;
    if (st == PCT_OK && (cudaMemcpyAsync(&h, status, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                         cudaStreamSynchronize(s) != cudaSuccess))
        st = PCT_ERR_CUDA;
    if (st == PCT_OK && h) st = PCT_ERR_TIMEOUT;
    cudaFree(status);
    return st;
}

pct_status pct_conv3d_bf16_wgrad(const uint16_t* in, int cin, int columns, int rows, int slices, int upsample,
                                 const uint16_t* dz, int cout, float* dweight, void* stream)
{
    if (!in || !dz || !dweight || !valid_channels(cin) || !valid_channels(cout) || columns <= 0 || rows <= 0 ||
        slices <= 0 || (upsample && (columns % 2 || rows % 2 || slices % 2)) ||
        static_cast<long long>(columns) * rows * slices > 0x7fffffffLL)
        return PCT_ERR_ARG;
    int* status = nullptr;
    if (cudaMalloc(&status, sizeof(int)) != cudaSuccess) return PCT_ERR_NOMEM;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    ConvWgradArgs a{};
    a.in = reinterpret_cast<const bf16*>(in);
    a.cin = cin;
    a.up = upsample ? 1 : 0;
    a.dz = reinterpret_cast<const bf16*>(dz);
    a.cout = cout;
    a.nx = columns;
    a.ny = rows;
    a.nz = slices;
    a.dw = dweight;
    a.status = status;
    pct_status st = PCT_OK;
    if (cudaMemsetAsync(status, 0, sizeof(int), s) != cudaSuccess || launch_conv_wgrad(a, s) != cudaSuccess) st = PCT_ERR_CUDA;
    int h = 0;
    if (st == PCT_OK && (cudaMemcpyAsync(&h, status, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                         cudaStreamSynchronize(s) != cudaSuccess))
        st = PCT_ERR_CUDA;
    if (st == PCT_OK && h) st = PCT_ERR_TIMEOUT;
    cudaFree(status);
    return st;
}

}  // extern "C"
