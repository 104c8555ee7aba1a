// pct_tvs.cu -- total variation superiorization (NTVS) of the image on the device.
//
// Restates NTVS_iteration (B.cu:10606) -> iteratively_perturb_image (B.cu:10476, the
// TVS_CONDITIONED path) / iteratively_perturb_image_unconditional (B.cu:10562), with
// generate_perturbation_array (B.cu:10246), calculate_total_variation (B.cu:10163) and the
// beta = A^L table of generate_TVS_eta_sequence (B.cu:10149).  The reference runs all of it on
// the host between DROP iterations, one sequential pass over the image per trial beta.
//
// Design: the image never leaves HBM.  One repetition is three kinds of launch:
//   gradient    G (the TV subgradient, gathered per voxel instead of scattered), ||G||^2 and
//               TV(x), reduced in fixed order by the last block to arrive (no spin waits);
//   candidates  TV(x - beta_j * G/||G||) for 16 consecutive trial exponents L0+16q .. L0+16q+15
//               in one pass over x and G; the last block picks the first trial the reference's
//               loop would accept (TV_y <= TV_x, |TV_y - TV_prev|/TV_y < TV_THRESHOLD, or
//               L > 300) and records beta and the new L.  Chunks after the accepting one exit at
//               once, so the chain of launches is fixed and graph-capturable;
//   apply       x = x - beta * G/||G|| on hull voxels.
// The L draw of NTVS (randi, B.cu:11478: uniform in [L_0 + k - 1, L]) uses a seeded
// splitmix64 hash of (seed, k) instead of the wall clock, so runs are reproducible.
//
// Arithmetic: G, ||G|| and the per-voxel TV terms are float like the reference's (the gradient
// norm through double, as std::pow(float, 2) promotes); the reference's squares of float
// differences go through glibc powf, which differs from the correctly rounded product in about
// 0.04% of inputs, so the engine uses the product.  The reference accumulates TV and ||G||^2 in
// one float in voxel order; the engine accumulates in double in a fixed tree order, which is
// deterministic and more accurate.  Past the end of the beta table the reference reads beyond
// its array (eta[L - L_0] for L > TVS_ETA_SEQUENCE_LENGTH); the engine uses beta = 0 there.
// This translation unit is compiled with -fmad=false.
#include <cmath>
#include <vector>

#include "pct_context.h"

namespace pct {

struct TvsState {
    int L;            // exponent of the next beta = A^L
    int L0;           // L at the start of the current repetition
    int done;         // the current repetition has accepted a trial
    int unused;
    float norm;       // ||G||
    float beta;       // accepted beta
    double tv_x;      // TV of the unperturbed image
    double tv_prev;   // TV of the last rejected trial (TV_y_previous)
    double tv_y;      // TV of the accepted trial
    unsigned arrive;  // blocks finished (last-block reduction)
};

struct TvsDims {
    int C, R;
    long long nv;
};

struct TvsTable {
    const float* eta;  // eta[e] = powf(A, L_0 + e), e < len
    int L_0, len;
};

struct TvsStep {
    int draw;           // draw L at the start of this repetition (NTVS)
    int k;              // DROP iteration number (1-based)
    int unconditioned;  // TVS_CONDITIONED off: beta = A^L, L++ (no TV check)
    long long seed;
};

constexpr int kTvsThreads = 256;
constexpr int kTvsWarps = kTvsThreads / 32;
constexpr int kTvsTrials = 16;

__host__ __device__ inline int tvs_randi(int lo, int hi, unsigned long long seed, int k)
{
    if (hi < lo) return lo;  // std::uniform_int_distribution needs lo <= hi
    // splitmix64 (Steele, Lea, Flood 2014) finaliser of seed + (k+1) * golden gamma
    unsigned long long z = seed + 0x9E3779B97F4A7C15ull * (unsigned long long)(k + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return lo + (int)(z % (unsigned long long)(hi - lo + 1));
}

__device__ __forceinline__ float eta_at(const TvsTable& t, int L)
{
    const int e = L - t.L_0;
    return (e >= 0 && e < t.len) ? t.eta[e] : 0.0f;
}

// Forward differences at voxel v: gx = x[v+1]-x[v], gy = x[v+C]-x[v].
__device__ __forceinline__ void forward_diff(const float* __restrict__ x, long long v, int C, float& gx, float& gy)
{
    const float x0 = x[v];
    gx = __fsub_rn(x[v + 1], x0);
    gy = __fsub_rn(x[v + C], x0);
}

// G_norm = sqrt(pow(G_x, 2) + pow(G_y, 2)) in double, stored as float (B.cu:10266).
__device__ __forceinline__ float grad_norm(float gx, float gy)
{
    const double a = (double)gx, b = (double)gy;
    return (float)__dsqrt_rn(__dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b)));
}

// One term of calculate_total_variation (B.cu:10175): sqrt(dy^2 + dx^2) in float.
__device__ __forceinline__ float tv_term(float dy, float dx)
{
    return __fsqrt_rn(__fadd_rn(__fmul_rn(dy, dy), __fmul_rn(dx, dx)));
}

// Sums N doubles over the block in a fixed order; thread 0 gets the totals.
template <int N>
__device__ void block_sum(double (&v)[N], double* smem /* [N * kTvsWarps] */)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < N; i++) {
        double a = v[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
        if (lane == 0) smem[i * kTvsWarps + warp] = a;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int i = 0; i < N; i++) {
            double a = 0.0;
            for (int w = 0; w < kTvsWarps; w++) a += smem[i * kTvsWarps + w];
            v[i] = a;
        }
    }
    __syncthreads();
}

// Writes this block's N partial sums; returns true in the last block to arrive, after which
// `totals` holds the grid totals in thread 0 (fixed order: block b's partial at [i*nblocks+b]).
template <int N>
__device__ bool grid_sum(double (&v)[N], double* __restrict__ partials, unsigned nblocks, TvsState* st, double* smem)
{
    __shared__ bool last;
    block_sum<N>(v, smem);
    if (threadIdx.x == 0) {
        for (int i = 0; i < N; i++) partials[(size_t)i * nblocks + blockIdx.x] = v[i];
        __threadfence();
        last = atomicAdd(&st->arrive, 1u) == nblocks - 1;
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
#pragma unroll
    for (int i = 0; i < N; i++) {
        double a = 0.0;
        for (unsigned b = threadIdx.x; b < nblocks; b += kTvsThreads)
            a += ((volatile double*)partials)[(size_t)i * nblocks + b];
        v[i] = a;
    }
    block_sum<N>(v, smem);
    if (threadIdx.x == 0) st->arrive = 0;
    return true;
}

// generate_perturbation_array (B.cu:10246-10324) in gather form, ||G||^2 and TV(x).
__global__ void __launch_bounds__(kTvsThreads) tvs_gradient_kernel(const float* __restrict__ x, float* __restrict__ G,
                                                                 TvsDims d, TvsTable tab, TvsStep step,
                                                                 double* __restrict__ partials, unsigned nblocks,
                                                                 TvsState* st)
{
    __shared__ double smem[2 * kTvsWarps];
    double acc[2] = {0.0, 0.0};  // TV(x), ||G||^2
    const long long stride = (long long)gridDim.x * kTvsThreads;
    for (long long v = blockIdx.x * (long long)kTvsThreads + threadIdx.x; v < d.nv; v += stride) {
        const int c = (int)(v % d.C), r = (int)((v / d.C) % d.R);
        float g = 0.0f, gx, gy, gn;
        // contributions in the reference's loop order: from v-C (row above), v-1, then v itself
        if (r > 0 && c < d.C - 1) {
            forward_diff(x, v - d.C, d.C, gx, gy);
            gn = grad_norm(gx, gy);
            if (gn > 0.0f) g = __fadd_rn(g, __fdiv_rn(gy, gn));
        }
        if (c > 0 && r < d.R - 1) {
            forward_diff(x, v - 1, d.C, gx, gy);
            gn = grad_norm(gx, gy);
            if (gn > 0.0f) g = __fadd_rn(g, __fdiv_rn(gx, gn));
        }
        if (c < d.C - 1 && r < d.R - 1) {
            forward_diff(x, v, d.C, gx, gy);
            gn = grad_norm(gx, gy);
            if (gn > 0.0f) g = __fsub_rn(g, __fdiv_rn(__fadd_rn(gx, gy), gn));
            acc[0] += (double)tv_term(gy, gx);
        }
        G[v] = g;
        acc[1] += (double)g * (double)g;
    }
    if (!grid_sum<2>(acc, partials, nblocks, st, smem)) return;
    if (threadIdx.x == 0) {
        st->tv_x = acc[0];
        st->norm = __fsqrt_rn((float)acc[1]);
        if (step.draw) st->L = tvs_randi(tab.L_0 + step.k - 1, st->L, (unsigned long long)step.seed, step.k);
        st->L0 = st->L;
        st->tv_prev = 0.0;
        st->tv_y = acc[0];
        st->done = 0;
        if (step.unconditioned) {  // for (...; n++, L++) { BETA_K_N = eta[L - L_0]; apply }
            st->beta = eta_at(tab, st->L);
            st->L += 1;
            st->done = 1;
        }
    }
}

// The perturbation direction v = G/||G|| (0 when ||G|| = 0), B.cu:10309-10316.
__device__ __forceinline__ float direction(const float* __restrict__ G, long long v, float norm)
{
    return norm != 0.0f ? __fdiv_rn(G[v], norm) : 0.0f;
}

__device__ __forceinline__ float perturbed(float x, bool in_hull, float beta, float w)
{
    return in_hull ? __fsub_rn(x, __fmul_rn(beta, w)) : x;
}

// TV of x - beta_j v for trials j = L0 + base .. L0 + base + 15 (the while loop of B.cu:10499).
__global__ void __launch_bounds__(kTvsThreads) tvs_trials_kernel(const float* __restrict__ x,
                                                               const float* __restrict__ G,
                                                               const uint8_t* __restrict__ hull, TvsDims d,
                                                               TvsTable tab, int base, double threshold,
                                                               double* __restrict__ partials, unsigned nblocks,
                                                               TvsState* st)
{
    __shared__ double smem[kTvsTrials * kTvsWarps];
    if (st->done) return;  // uniform across the grid: written by an earlier launch
    const int L0 = st->L0;
    const float norm = st->norm;
    float beta[kTvsTrials];
#pragma unroll
    for (int j = 0; j < kTvsTrials; j++) beta[j] = eta_at(tab, L0 + base + j);
    double acc[kTvsTrials];
#pragma unroll
    for (int j = 0; j < kTvsTrials; j++) acc[j] = 0.0;
    const long long stride = (long long)gridDim.x * kTvsThreads;
    for (long long v = blockIdx.x * (long long)kTvsThreads + threadIdx.x; v < d.nv; v += stride) {
        const int c = (int)(v % d.C), r = (int)((v / d.C) % d.R);
        if (c >= d.C - 1 || r >= d.R - 1) continue;
        const float x0 = x[v], x1 = x[v + 1], x2 = x[v + d.C];
        const bool h0 = hull[v] != 0, h1 = hull[v + 1] != 0, h2 = hull[v + d.C] != 0;
        const float w0 = direction(G, v, norm), w1 = direction(G, v + 1, norm), w2 = direction(G, v + d.C, norm);
#pragma unroll
        for (int j = 0; j < kTvsTrials; j++) {
            const float p0 = perturbed(x0, h0, beta[j], w0);
            const float p1 = perturbed(x1, h1, beta[j], w1);
            const float p2 = perturbed(x2, h2, beta[j], w2);
            acc[j] += (double)tv_term(__fsub_rn(p2, p0), __fsub_rn(p1, p0));
        }
    }
    if (!grid_sum<kTvsTrials>(acc, partials, nblocks, st, smem)) return;
    if (threadIdx.x == 0) {
        double prev = st->tv_prev;
        for (int j = 0; j < kTvsTrials; j++) {
            const int L_after = L0 + base + j + 1;  // L++ precedes the test
            const double tv_y = acc[j];
            const bool accept =
                (tv_y <= st->tv_x) || (fabs(tv_y - prev) / tv_y < threshold) || L_after > 300;
            if (accept) {
                st->beta = beta[j];
                st->L = L_after;
                st->tv_y = tv_y;
                st->done = 1;
                break;
            }
            prev = tv_y;
        }
        st->tv_prev = prev;
    }
}

// image = x_TVS - beta v on hull voxels (apply_TVS_perturbation B.cu:10413).
__global__ void tvs_apply_kernel(float* __restrict__ x, const float* __restrict__ G, const uint8_t* __restrict__ hull,
                                 long long nv, const TvsState* __restrict__ st, unsigned long long* counters)
{
    if (!st->done) {  // no trial accepted (cannot happen: beta = 0 is always accepted)
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&counters[kCntWaitExpired], 1ull);
        return;
    }
    const float beta = st->beta, norm = st->norm;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nv; v += stride)
        if (hull[v]) x[v] = __fsub_rn(x[v], __fmul_rn(beta, direction(G, v, norm)));
}

// calculate_total_variation alone (same term and reduction order as the gradient kernel).
__global__ void __launch_bounds__(kTvsThreads) tvs_total_variation_kernel(const float* __restrict__ x, TvsDims d,
                                                                        double* __restrict__ partials,
                                                                        unsigned nblocks, TvsState* st,
                                                                        double* __restrict__ out)
{
    __shared__ double smem[kTvsWarps];
    double acc[1] = {0.0};
    const long long stride = (long long)gridDim.x * kTvsThreads;
    for (long long v = blockIdx.x * (long long)kTvsThreads + threadIdx.x; v < d.nv; v += stride) {
        const int c = (int)(v % d.C), r = (int)((v / d.C) % d.R);
        if (c >= d.C - 1 || r >= d.R - 1) continue;
        float gx, gy;
        forward_diff(x, v, d.C, gx, gy);
        acc[0] += (double)tv_term(gy, gx);
    }
    if (grid_sum<1>(acc, partials, nblocks, st, smem) && threadIdx.x == 0) *out = acc[0];
}

__global__ void tvs_init_state_kernel(TvsState* st, int L)
{
    st->L = L;
    st->L0 = L;
    st->done = 0;
    st->unused = 0;
    st->norm = 0.0f;
    st->beta = 0.0f;
    st->tv_x = st->tv_prev = st->tv_y = 0.0;
    st->arrive = 0;
}

}  // namespace pct

// ------------------------------------------------------------------------------------------
// C ABI
// ------------------------------------------------------------------------------------------

struct pct_tvs {
    pct::TvsState* st = nullptr;
    float* G = nullptr;
    float* eta = nullptr;
    double* partials = nullptr;
    double* scalar = nullptr;
    int eta_len = 0;  // TVS_ETA_SEQUENCE_LENGTH - L_0 filled entries
    unsigned blocks = 0;
};

namespace pct {

void tvs_release(pct_tvs* t)
{
    if (!t) return;
    cudaFree(t->st);
    cudaFree(t->G);
    cudaFree(t->eta);
    cudaFree(t->partials);
    cudaFree(t->scalar);
    delete t;
}

}  // namespace pct

namespace {

pct_status tvs_fail(pct_ctx* ctx, pct_status s, const std::string& what, cudaError_t e = cudaSuccess)
{
    ctx->last_error = what;
    if (e != cudaSuccess) ctx->last_error += " -> " + pct::cuda_error_string(e);
    return s;
}

pct::TvsDims dims_of(const pct_ctx* ctx)
{
    return pct::TvsDims{ctx->cfg.COLUMNS, ctx->cfg.ROWS, (long long)ctx->cfg.NUM_VOXELS};
}

// Lazily allocates the TVS buffers and the beta table (generate_TVS_eta_sequence B.cu:10149).
pct_status ensure_tvs(pct_ctx* ctx)
{
    if (ctx->tvs) return PCT_OK;
    const pct_config& c = ctx->cfg;
    pct_tvs* t = new pct_tvs();
    // TVS_ETA_SEQUENCE_LENGTH = log(TVS_MIN_ETA)/log(A) (an int), eta[e] = powf(A, L_0 + e)
    const int seq_len = (int)(std::log(c.TVS_MIN_ETA) / std::log(c.TVS_A));
    std::vector<float> eta;
    for (int exponent = c.TVS_L_0; exponent < seq_len; exponent++)
        eta.push_back(powf((float)c.TVS_A, (float)exponent));
    t->eta_len = (int)eta.size();
    const long long nv = c.NUM_VOXELS;
    long long b = (nv + pct::kTvsThreads - 1) / pct::kTvsThreads;
    t->blocks = (unsigned)(b < 1 ? 1 : b > 148 * 4 ? 148 * 4 : b);
    cudaError_t e = cudaMalloc(&t->st, sizeof(pct::TvsState));
    if (e == cudaSuccess) e = cudaMalloc(&t->G, sizeof(float) * (size_t)nv);
    if (e == cudaSuccess) e = cudaMalloc(&t->eta, sizeof(float) * (eta.empty() ? 1 : eta.size()));
    if (e == cudaSuccess) e = cudaMalloc(&t->partials, sizeof(double) * (size_t)pct::kTvsTrials * t->blocks);
    if (e == cudaSuccess) e = cudaMalloc(&t->scalar, sizeof(double));
    if (e == cudaSuccess && !eta.empty())
        e = cudaMemcpyAsync(t->eta, eta.data(), sizeof(float) * eta.size(), cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) {
        pct::tvs_init_state_kernel<<<1, 1, 0, ctx->stream>>>(t->st, c.TVS_L_0);  // L = 0 with L_0 = 0 (B.h:438)
        e = cudaGetLastError();
        ctx->launches += 1;
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        pct::tvs_release(t);
        cudaGetLastError();
        return tvs_fail(ctx, PCT_ERR_NOMEM, "TVS buffers", e);
    }
    ctx->tvs = t;
    return PCT_OK;
}

}  // namespace

extern "C" pct_status pct_total_variation(pct_ctx* ctx, double* tv)
{
    if (!ctx || !tv) return PCT_ERR_ARG;
    cudaSetDevice(ctx->device);
    pct_status s = ensure_tvs(ctx);
    if (s != PCT_OK) return s;
    pct_tvs* t = ctx->tvs;
    pct::tvs_total_variation_kernel<<<t->blocks, pct::kTvsThreads, 0, ctx->stream>>>(ctx->d_x, dims_of(ctx),
                                                                                    t->partials, t->blocks, t->st,
                                                                                    t->scalar);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(tv, t->scalar, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return tvs_fail(ctx, PCT_ERR_CUDA, "total variation", e);
    ctx->launches += 1;
    return PCT_OK;
}

extern "C" pct_status pct_ntvs_iteration(pct_ctx* ctx, int iteration)
{
    if (!ctx || iteration < 1) return PCT_ERR_ARG;
    const uint8_t* hull = pct::preproc_hull(ctx);
    if (!hull) return tvs_fail(ctx, PCT_ERR_STATE, "TVS needs the hull: run the preprocessing or set array \"hull\"");
    cudaSetDevice(ctx->device);
    pct_status s = ensure_tvs(ctx);
    if (s != PCT_OK) return s;
    pct_tvs* t = ctx->tvs;
    const pct_config& c = ctx->cfg;
    const pct::TvsDims d = dims_of(ctx);
    const pct::TvsTable tab{t->eta, c.TVS_L_0, t->eta_len};
    const bool ntvs = !c.TVS_OLD;                            // NTVS_ON = TVS_ON && !TVS_OLD
    const int reps = c.TVS_OLD ? 1 : c.TVS_REPETITIONS;      // TVS_OLD: TVS_REPETITIONS = 1
    const bool conditioned = c.TVS_CONDITIONED != 0;
    // Trials until beta = 0 (past the table) is reached, which is always accepted.
    const int trial_chunks = (t->eta_len + 1 + pct::kTvsTrials - 1) / pct::kTvsTrials + 1;
    cudaStream_t st = ctx->stream;
    long long launches = 0;
    for (int n = 0; n < reps; n++) {
        const pct::TvsStep step{(ntvs && n == 0) ? 1 : 0, iteration, conditioned ? 0 : 1, (long long)c.TVS_SEED};
        pct::tvs_gradient_kernel<<<t->blocks, pct::kTvsThreads, 0, st>>>(ctx->d_x, t->G, d, tab, step, t->partials,
                                                                          t->blocks, t->st);
        launches++;
        if (conditioned)
            for (int q = 0; q < trial_chunks; q++) {
                pct::tvs_trials_kernel<<<t->blocks, pct::kTvsThreads, 0, st>>>(
                    ctx->d_x, t->G, hull, d, tab, q * pct::kTvsTrials, c.TV_THRESHOLD, t->partials, t->blocks, t->st);
                launches++;
            }
        pct::tvs_apply_kernel<<<t->blocks, pct::kTvsThreads, 0, st>>>(ctx->d_x, t->G, hull, d.nv, t->st,
                                                                       ctx->d_counters);
        launches++;
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return tvs_fail(ctx, PCT_ERR_CUDA, "NTVS kernels", e);
    ctx->launches += launches;
    return PCT_OK;
}

extern "C" pct_status pct_tvs_L(pct_ctx* ctx, int32_t* L_out, const int32_t* L_in)
{
    if (!ctx) return PCT_ERR_ARG;
    cudaSetDevice(ctx->device);
    pct_status s = ensure_tvs(ctx);
    if (s != PCT_OK) return s;
    cudaError_t e = cudaSuccess;
    if (L_in) {
        pct::tvs_init_state_kernel<<<1, 1, 0, ctx->stream>>>(ctx->tvs->st, *L_in);
        e = cudaGetLastError();
        ctx->launches += 1;
    }
    if (e == cudaSuccess && L_out)
        e = cudaMemcpyAsync(L_out, &ctx->tvs->st->L, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return tvs_fail(ctx, PCT_ERR_CUDA, "TVS state", e);
    return PCT_OK;
}
