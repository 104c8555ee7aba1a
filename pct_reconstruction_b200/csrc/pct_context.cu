// pct_context.cu -- the C ABI: context lifetime, data transfer and the DROP drivers.
//
// The reference keeps its state in globals and launches two kernels per DROP block from a host
// loop (DROP_full_tx_iteration, B.cu:9537-9589), synchronising once per iteration.  Here the
// context owns all device state; one DROP iteration (all blocks, both kernels per block) is
// captured once into a CUDA graph and replayed, so an iteration costs one graph launch.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <new>
#include <string>
#include <vector>

#include "pct_context.h"


namespace pct {

std::string cuda_error_string(cudaError_t e) { return std::string(cudaGetErrorName(e)) + ": " + cudaGetErrorString(e); }

// Mixed mode: distance (cm) from the entry and the exit within which Sigma_2 and M are inverted
// in FP64.  Measured on B200: 0.5, 1 and 2 cm give the same point deviations and image RMSE
// against the exact mode as inverting in FP64 everywhere (water phantom, 10M histories), and
// 0.5 cm is the fastest (head phantom, 20M histories).
#ifndef PCT_MIXED_FP64_MARGIN
#define PCT_MIXED_FP64_MARGIN 0.5
#endif
Geometry make_geometry(const pct_config& c)
{
    Geometry g{};
    g.columns = c.COLUMNS;
    g.rows = c.ROWS;
    g.slices = c.SLICES;
    g.num_voxels = c.NUM_VOXELS;
    g.padded_voxels = c.NUM_VOXELS + c.COLUMNS * c.ROWS;
    g.voxel_width = c.VOXEL_WIDTH;
    g.voxel_height = c.VOXEL_HEIGHT;
    g.voxel_thickness = c.VOXEL_THICKNESS;
    g.inv_voxel_width = 1.0 / c.VOXEL_WIDTH;
    g.inv_voxel_height = 1.0 / c.VOXEL_HEIGHT;
    g.inv_voxel_thickness = 1.0 / c.VOXEL_THICKNESS;
    g.inv_voxel_max = fmax(fmax(g.inv_voxel_width, g.inv_voxel_height), g.inv_voxel_thickness);
    g.x_zero = -c.RECON_CYL_RADIUS;      // X_ZERO_COORDINATE (B.h:918)
    g.y_zero = c.RECON_CYL_RADIUS;       // Y_ZERO_COORDINATE (B.h:919)
    g.z_zero = c.RECON_CYL_HEIGHT / 2;   // Z_ZERO_COORDINATE (B.h:920)
    g.x_zero_f = (float)g.x_zero;
    g.y_zero_f = (float)g.y_zero;
    g.z_zero_f = (float)g.z_zero;
    g.inv_voxel_width_f = (float)(1.0 / c.VOXEL_WIDTH);
    g.inv_voxel_height_f = (float)(1.0 / c.VOXEL_HEIGHT);
    g.inv_voxel_thickness_f = (float)(1.0 / c.VOXEL_THICKNESS);
    g.mlp_u_step = c.MLP_U_STEP;
    g.trig_min = trig_table_min();
    g.trig_step = trig_table_step();
    g.trig_elements = trig_table_elements();
    g.coeff_elements = coeff_table_elements();
    g.poly_elements = poly_table_elements();
    g.sigma_index_step = (unsigned)(c.MLP_U_STEP / kCoeffTableStep + 0.5);
    g.poly_index_step = (unsigned)(c.MLP_U_STEP / kPolyTableStep + 0.5);
    g.min_mlp_length = c.MIN_MLP_LENGTH;
    g.lambda = (double)c.LAMBDA;
    g.projection_algorithm = c.PROJECTION_ALGORITHM;
    g.mixed_precision = c.PRECISION != PCT_PRECISION_EXACT ? 1 : 0;
    g.compensated = c.PRECISION == PCT_PRECISION_MIXED_COMPENSATED ? 1 : 0;
    g.mixed_fp64_margin = PCT_MIXED_FP64_MARGIN;
    g.exact_fast_points = c.EXACT_FAST_POINTS;
    g.path_cta_threads = c.PATH_CTA_THREADS;
    g.deterministic = c.SCATTER_MODE == PCT_SCATTER_DETERMINISTIC ? 1 : 0;
    g.psi_sign = c.PSI_SIGN;
    g.eta = c.ETA;
    // #if IDENTIFY_X_N_AIR: if( x[voxel] < X_N_AIR_THRESHOLD ) x[voxel] = 0.0 (B.cu:9411-9414)
    g.air_threshold = c.IDENTIFY_X_N_AIR ? c.X_N_AIR_THRESHOLD : -INFINITY;
    g.s_curve = nullptr;  // set by pct_create once the table exists
    g.dual_sided_s_curve = c.DUAL_SIDED_S_CURVE;
    return g;
}

}  // namespace pct

namespace {

pct_status ctx_fail(pct_ctx* ctx, pct_status st, const char* what, cudaError_t e = cudaSuccess)
{
    if (ctx) {
        ctx->last_error = what ? what : "";
        if (e != cudaSuccess) ctx->last_error += " -> " + pct::cuda_error_string(e);
    }
    return st;
}

void release_graph(pct_ctx* ctx)
{
    if (ctx->iter_exec) cudaGraphExecDestroy(ctx->iter_exec);
    if (ctx->reuse_exec) cudaGraphExecDestroy(ctx->reuse_exec);
    if (ctx->batch_graph) cudaGraphDestroy(ctx->batch_graph);
    ctx->iter_exec = ctx->reuse_exec = nullptr;
    ctx->batch_graph = nullptr;
    ctx->graph_version++;
    ctx->iter_launches = ctx->reuse_launches = ctx->batch_launches = 0;
    ctx->paths_valid = false;
}

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// Why the calling thread's last pct_create failed: the context it was building is gone by then.
thread_local std::string g_create_error;

}  // namespace

extern "C" const char* pct_status_string(pct_status s)
{
    switch (s) {
        case PCT_OK: return "PCT_OK";
        case PCT_ERR_ARG: return "PCT_ERR_ARG";
        case PCT_ERR_CUDA: return "PCT_ERR_CUDA";
        case PCT_ERR_OOB: return "PCT_ERR_OOB";
        case PCT_ERR_TIMEOUT: return "PCT_ERR_TIMEOUT";
        case PCT_ERR_STATE: return "PCT_ERR_STATE";
        case PCT_ERR_NOMEM: return "PCT_ERR_NOMEM";
        case PCT_ERR_IO: return "PCT_ERR_IO";
    }
    return "PCT_ERR_UNKNOWN";
}

extern "C" const char* pct_last_error(const pct_ctx* ctx) { return ctx ? ctx->last_error.c_str() : g_create_error.c_str(); }

extern "C" void pct_destroy(pct_ctx* ctx)
{
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    release_graph(ctx);
    cudaFree(ctx->d_table_block);
    cudaFree(ctx->d_steps);
    if (ctx->l2_window) {
        cudaCtxResetPersistingL2Cache();
        cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, 0);
    }
    cudaFree(ctx->d_x);  // also holds d_acc
    cudaFree(ctx->d_hist_block);
    cudaFree(ctx->d_stage_block);
    if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
    if (ctx->stage_done) cudaEventDestroy(ctx->stage_done);
    if (ctx->stage_free) cudaEventDestroy(ctx->stage_free);
    if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
    cudaFree(ctx->d_counters);
    cudaFree(ctx->d_bounds);
    cudaFree(ctx->d_offsets);
    cudaFree(ctx->d_perm);
    cudaFree(ctx->d_path_n);
    cudaFree(ctx->d_chord);
    cudaFree(ctx->d_scan_tmp);
    cudaFree(ctx->d_hist_tmp);
    cudaFree(ctx->d_sorted_block);
    cudaFree(ctx->d_paths);
    cudaFree(ctx->d_normA);
    cudaFree(ctx->fixed.sum);
    cudaFree(ctx->fixed.cnt);
    pct::preproc_release(ctx->pre);
    pct::tvs_release(ctx->tvs);
    for (cudaEvent_t ev : ctx->events) cudaEventDestroy(ev);
    if (ctx->path_stream) cudaStreamDestroy(ctx->path_stream);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
}

extern "C" pct_status pct_create(const pct_config* cfg_in, int device, pct_ctx** out)
{
    g_create_error.clear();
    if (!cfg_in || !out) {
        g_create_error = "pct_create: null argument";
        return PCT_ERR_ARG;
    }
    *out = nullptr;
    pct_ctx* ctx = new (std::nothrow) pct_ctx();
    if (!ctx) {
        g_create_error = "pct_create: out of host memory";
        return PCT_ERR_NOMEM;
    }
    ctx->cfg = *cfg_in;
    if (pct_config_finalize(&ctx->cfg) != PCT_OK) {
        g_create_error = std::string("configuration: ") + pct_config_last_error();
        delete ctx;
        return PCT_ERR_ARG;
    }
    ctx->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) {
        g_create_error = "cudaSetDevice(" + std::to_string(device) + ") -> " + pct::cuda_error_string(e);
        delete ctx;
        return PCT_ERR_CUDA;
    }
    ctx->geo = pct::make_geometry(ctx->cfg);
    (void)pct::sm_count();  // cache the SM count outside any stream capture
    pct_status st = PCT_OK;
    do {
        // The DROP block chain is the critical path: it gets the highest stream priority, the
        // path kernel chunks that run ahead of it the lowest.
        int prio_low = 0, prio_high = 0;
        cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high);
        e = cudaStreamCreateWithPriority(&ctx->own_stream, cudaStreamNonBlocking, prio_high);
        if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&ctx->path_stream, cudaStreamNonBlocking, prio_low);
        if (e != cudaSuccess) { st = ctx_fail(ctx, PCT_ERR_CUDA, "cudaStreamCreate", e); break; }
        ctx->stream = ctx->own_stream;
        ctx->trace = getenv("PCT_TRACE") != nullptr;

        // MLP lookup tables (setup_MLP_lookup_tables, B.cu:8527): built on the host, uploaded.
        pct::HostTables ht;
        pct::build_host_tables(ht);
        ctx->kmax = pct::step_table_kmax(ht, ctx->cfg.MLP_U_STEP);
        if (ctx->kmax <= 0) { st = ctx_fail(ctx, PCT_ERR_ARG, "MLP_U_STEP outside the lookup tables"); break; }
        const std::vector<double>* parts[8] = {&ht.sin_table, &ht.cos_table, &ht.scattering_table, &ht.poly_1_2,
                                               &ht.poly_2_3, &ht.poly_3_4, &ht.poly_2_6, &ht.poly_3_12};
        size_t total = 0;
        for (auto* p : parts) total += align256(p->size() * sizeof(double));
        const size_t s_curve_offset = total;  // the S-curve table follows the MLP tables
        total += align256(pct::kSCurveEntries * sizeof(float));
        e = cudaMalloc(&ctx->d_table_block, total);
        if (e != cudaSuccess) { st = ctx_fail(ctx, PCT_ERR_NOMEM, "cudaMalloc(tables)", e); break; }
        const double* dptr[8];
        size_t off = 0;
        for (int i = 0; i < 8; i++) {
            double* d = reinterpret_cast<double*>(reinterpret_cast<char*>(ctx->d_table_block) + off);
            e = cudaMemcpy(d, parts[i]->data(), parts[i]->size() * sizeof(double), cudaMemcpyHostToDevice);
            if (e != cudaSuccess) break;
            dptr[i] = d;
            off += align256(parts[i]->size() * sizeof(double));
        }
        if (e != cudaSuccess) { st = ctx_fail(ctx, PCT_ERR_CUDA, "cudaMemcpy(tables)", e); break; }
        ctx->tables = pct::Tables{dptr[0], dptr[1], dptr[2], dptr[3], dptr[4], dptr[5], dptr[6], dptr[7]};
        if (ctx->cfg.S_CURVE_ON) {
            float* table = reinterpret_cast<float*>(reinterpret_cast<char*>(ctx->d_table_block) + s_curve_offset);
            e = pct::launch_s_curve_table(ctx->cfg, table, ctx->own_stream);
            if (e != cudaSuccess) { st = ctx_fail(ctx, PCT_ERR_CUDA, "S-curve table kernel", e); break; }
            ctx->launches += 1;
            ctx->geo.s_curve = table;
        }
        e = pct::set_iteration_carveout();
        if (e != cudaSuccess) { st = ctx_fail(ctx, PCT_ERR_CUDA, "shared-memory carve-out", e); break; }
        e = cudaMalloc(&ctx->d_steps, (size_t)(ctx->kmax + 1) * sizeof(pct::StepConst));
        if (e != cudaSuccess) { st = ctx_fail(ctx, PCT_ERR_NOMEM, "cudaMalloc(steps)", e); break; }
        e = pct::launch_build_step_table(ctx->tables, ctx->geo.sigma_index_step, ctx->geo.poly_index_step, ctx->kmax,
                                         ctx->d_steps, ctx->own_stream);
        if (e != cudaSuccess) { st = ctx_fail(ctx, PCT_ERR_CUDA, "step table kernel", e); break; }
        ctx->launches += 1;

        // Image and accumulator, padded by one slice (z index SLICES is reachable, B.cu:11091).
        const size_t npad = (size_t)ctx->geo.padded_voxels;
        ctx->image_block_bytes = align256(npad * sizeof(float)) + npad * sizeof(float2);
        e = cudaMalloc(&ctx->d_x, ctx->image_block_bytes);
        if (e == cudaSuccess)
            ctx->d_acc = reinterpret_cast<float2*>(reinterpret_cast<char*>(ctx->d_x) + align256(npad * sizeof(float)));
        if (e == cudaSuccess) e = cudaMalloc(&ctx->d_counters, pct::kNumCounters * sizeof(unsigned long long));
        if (e != cudaSuccess) { st = ctx_fail(ctx, PCT_ERR_NOMEM, "cudaMalloc(image)", e); break; }
        e = cudaMemset(ctx->d_x, 0, npad * sizeof(float));
        if (e == cudaSuccess) e = cudaMemset(ctx->d_acc, 0, npad * sizeof(float2));
        if (e == cudaSuccess) e = cudaMemset(ctx->d_counters, 0, pct::kNumCounters * sizeof(unsigned long long));
        if (e != cudaSuccess) { st = ctx_fail(ctx, PCT_ERR_CUDA, "cudaMemset(image)", e); break; }
        if (ctx->cfg.SCATTER_MODE == PCT_SCATTER_DETERMINISTIC) {
            e = cudaMalloc(&ctx->fixed.sum, npad * sizeof(unsigned long long));
            if (e == cudaSuccess) e = cudaMalloc(&ctx->fixed.cnt, npad * sizeof(unsigned));
            if (e == cudaSuccess) e = cudaMemset(ctx->fixed.sum, 0, npad * sizeof(unsigned long long));
            if (e == cudaSuccess) e = cudaMemset(ctx->fixed.cnt, 0, npad * sizeof(unsigned));
            if (e != cudaSuccess) { st = ctx_fail(ctx, PCT_ERR_NOMEM, "cudaMalloc(fixed-point accumulator)", e); break; }
        }
        // ROBUSTB's per-voxel ||a||^2, or in PRECISION MIXED_COMPENSATED the rounding errors of the
        // compensated float accumulation (drop_phase2_kernel)
        if (ctx->cfg.PROJECTION_ALGORITHM == PCT_ROBUSTB ||
            (ctx->cfg.PRECISION == PCT_PRECISION_MIXED_COMPENSATED && ctx->cfg.PROJECTION_ALGORITHM == PCT_DROP &&
             ctx->cfg.SCATTER_MODE == PCT_SCATTER_ATOMIC)) {
            e = cudaMalloc(&ctx->d_normA, npad * sizeof(float));
            if (e == cudaSuccess) e = cudaMemset(ctx->d_normA, 0, npad * sizeof(float));
            if (e != cudaSuccess) { st = ctx_fail(ctx, PCT_ERR_NOMEM, "cudaMalloc(normA)", e); break; }
        }
        e = cudaDeviceSynchronize();
        if (e != cudaSuccess) { st = ctx_fail(ctx, PCT_ERR_CUDA, "create sync", e); break; }
    } while (0);
    if (st != PCT_OK) {
        g_create_error = ctx->last_error;
        pct_destroy(ctx);
        return st;
    }
    *out = ctx;
    return PCT_OK;
}

extern "C" pct_status pct_set_stream(pct_ctx* ctx, void* stream)
{
    if (!ctx) return PCT_ERR_ARG;
    ctx->stream = stream ? static_cast<cudaStream_t>(stream) : ctx->own_stream;
    return PCT_OK;
}

extern "C" pct_status pct_synchronize(pct_ctx* ctx)
{
    if (!ctx) return PCT_ERR_ARG;
    cudaSetDevice(ctx->device);
    PCT_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return PCT_OK;
}

extern "C" pct_status pct_set_reconstruction_histories(pct_ctx* ctx, const pct_histories* h, int64_t n, pct_memory where)
{
    if (!ctx || !h || n < 0 || n > 0x7fffffffLL) return PCT_ERR_ARG;
    const void* src[12] = {h->x_entry, h->y_entry, h->z_entry, h->x_exit, h->y_exit, h->z_exit,
                           h->xy_entry_angle, h->xz_entry_angle, h->xy_exit_angle, h->xz_exit_angle,
                           h->WEPL, h->first_MLP_voxel};
    if (n > 0)
        for (const void* p : src)
            if (!p) return ctx_fail(ctx, PCT_ERR_ARG, "pct_set_reconstruction_histories: NULL array");
    cudaSetDevice(ctx->device);
    // The captured iteration bakes in the history count and array addresses; it stays valid
    // while both are unchanged.
    if (n != ctx->n_hist || n > ctx->cap_hist) release_graph(ctx);
    if (n > ctx->cap_hist) {
        PCT_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        cudaFree(ctx->d_hist_block);
        ctx->d_hist_block = nullptr;
        ctx->cap_hist = 0;
        const size_t per = align256((size_t)n * 4);
        cudaError_t e = cudaMalloc(&ctx->d_hist_block, per * 12);
        if (e != cudaSuccess) return ctx_fail(ctx, PCT_ERR_NOMEM, "cudaMalloc(histories)", e);
        ctx->cap_hist = n;
    }
    const size_t per = align256((size_t)(ctx->cap_hist > 0 ? ctx->cap_hist : 1) * 4);
    char* base = static_cast<char*>(ctx->d_hist_block);
    void* dst[12];
    for (int i = 0; i < 12; i++) dst[i] = base + per * i;
    pct::HistorySoA& s = ctx->hist;
    s.x_entry = (float*)dst[0];
    s.y_entry = (float*)dst[1];
    s.z_entry = (float*)dst[2];
    s.x_exit = (float*)dst[3];
    s.y_exit = (float*)dst[4];
    s.z_exit = (float*)dst[5];
    s.xy_entry_angle = (float*)dst[6];
    s.xz_entry_angle = (float*)dst[7];
    s.xy_exit_angle = (float*)dst[8];
    s.xz_exit_angle = (float*)dst[9];
    s.WEPL = (float*)dst[10];
    s.first_MLP_voxel = (uint32_t*)dst[11];
    const cudaMemcpyKind kind = where == PCT_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    for (int i = 0; i < 12 && n > 0; i++)
        PCT_CUDA_TRY(cudaMemcpyAsync(dst[i], src[i], (size_t)n * 4, kind, ctx->stream));
    ctx->n_hist = n;
    ctx->layout_ready = false;  // path bounds and order depend on the history contents
    ctx->paths_valid = false;
    return PCT_OK;
}

extern "C" int64_t pct_reconstruction_histories(const pct_ctx* ctx) { return ctx ? ctx->n_hist : -1; }

namespace {

// new[i] = old[(i * step) mod n] for the 12 history arrays (4-byte elements), step = PRIME_OFFSET
// mod n: generate_history_sequence (B.cu:8664) sets sequence[0] = 0 and
// sequence[i] = (sequence[i-1] + offset_prime) % N, i.e. sequence[i] = i * offset_prime mod N.
__global__ void history_sequence_kernel(const char* __restrict__ src, char* __restrict__ dst, size_t per,
                                        long long n, long long step)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long long r = (long long)(((unsigned long long)i * (unsigned long long)step) % (unsigned long long)n);
#pragma unroll
    for (int a = 0; a < 12; a++)
        reinterpret_cast<uint32_t*>(dst + per * a)[i] = reinterpret_cast<const uint32_t*>(src + per * a)[r];
}

long long gcd_ll(long long a, long long b)
{
    while (b) {
        const long long t = a % b;
        a = b;
        b = t;
    }
    return a;
}

}  // namespace

extern "C" pct_status pct_apply_history_sequence(pct_ctx* ctx, int64_t prime_offset)
{
    if (!ctx || prime_offset <= 0) return PCT_ERR_ARG;
    const long long n = ctx->n_hist;
    if (n <= 1) return PCT_OK;
    const long long step = prime_offset % n;
    // verify_history_sequence (B.cu:8670): the sequence is a permutation only if gcd(step, N) = 1
    if (gcd_ll(step, n) != 1)
        return ctx_fail(ctx, PCT_ERR_ARG, "PRIME_OFFSET shares a factor with the number of histories");
    cudaSetDevice(ctx->device);
    const size_t per = align256((size_t)ctx->cap_hist * 4);
    void* fresh = nullptr;
    PCT_CUDA_TRY(cudaMalloc(&fresh, per * 12));
    history_sequence_kernel<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(
        static_cast<const char*>(ctx->d_hist_block), static_cast<char*>(fresh), per, n, step);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        cudaFree(fresh);
        return ctx_fail(ctx, PCT_ERR_CUDA, "history sequence kernel", e);
    }
    ctx->launches += 1;
    release_graph(ctx);  // the captured iteration holds the old array addresses
    cudaFree(ctx->d_hist_block);
    ctx->d_hist_block = fresh;
    char* base = static_cast<char*>(fresh);
    pct::HistorySoA& hs = ctx->hist;
    float** f[11] = {&hs.x_entry, &hs.y_entry, &hs.z_entry, &hs.x_exit, &hs.y_exit, &hs.z_exit,
                     &hs.xy_entry_angle, &hs.xz_entry_angle, &hs.xy_exit_angle, &hs.xz_exit_angle, &hs.WEPL};
    for (int a = 0; a < 11; a++) *f[a] = reinterpret_cast<float*>(base + per * a);
    hs.first_MLP_voxel = reinterpret_cast<uint32_t*>(base + per * 11);
    ctx->layout_ready = false;
    ctx->paths_valid = false;
    return PCT_OK;
}

extern "C" pct_status pct_set_image(pct_ctx* ctx, const float* x, pct_memory where)
{
    if (!ctx || !x) return PCT_ERR_ARG;
    cudaSetDevice(ctx->device);
    PCT_CUDA_TRY(cudaMemcpyAsync(ctx->d_x, x, (size_t)ctx->geo.num_voxels * sizeof(float),
                                 where == PCT_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, ctx->stream));
    if (where == PCT_HOST) PCT_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return PCT_OK;
}

extern "C" pct_status pct_get_image(pct_ctx* ctx, float* x, pct_memory where)
{
    if (!ctx || !x) return PCT_ERR_ARG;
    cudaSetDevice(ctx->device);
    PCT_CUDA_TRY(cudaMemcpyAsync(x, ctx->d_x, (size_t)ctx->geo.num_voxels * sizeof(float),
                                 where == PCT_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, ctx->stream));
    if (where == PCT_HOST) PCT_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return PCT_OK;
}

namespace {

constexpr int kMaxBoundKey = PCT_MLP_PATH_CAP + 1;
// Path-kernel order (PATH_ORDER_WINDOW): 0 sorts each chunk of DROP blocks by path-length bound
// as a whole; W > 0 sorts each window of W consecutive histories on its own (the inputs a
// window's warps read stay together, so each sector is read from HBM once).

long long covered_in_block(const pct_config& c, long long n, long long start)
{
    long long hp = n - start;
    if (hp > c.DROP_BLOCK_SIZE) hp = c.DROP_BLOCK_SIZE;
    long long covered = hp;
    if (c.HISTORIES_PER_BLOCK > 0) covered = (hp / c.HISTORIES_PER_BLOCK) * c.HISTORIES_PER_BLOCK;
    return covered;
}

template <class T>
cudaError_t grow(T*& p, long long& cap_elems, long long want)
{
    if (want <= cap_elems && p) return cudaSuccess;
    cudaFree(p);
    p = nullptr;
    cap_elems = 0;
    cudaError_t e = cudaMalloc(&p, sizeof(T) * (size_t)(want > 0 ? want : 1));
    if (e == cudaSuccess) cap_elems = want;
    return e;
}

// The gathered path-kernel inputs from processing position p on.
pct::HistorySoA sorted_from(const pct_ctx* ctx, long long p)
{
    const pct::HistorySoA& s = ctx->sorted_hist;
    return pct::HistorySoA{s.x_entry + p, s.y_entry + p, s.z_entry + p, s.x_exit + p, s.y_exit + p, s.z_exit + p,
                           s.xy_entry_angle + p, s.xz_entry_angle + p, s.xy_exit_angle + p, s.xz_exit_angle + p,
                           nullptr, s.first_MLP_voxel + p};
}

// Lay out path storage for the loaded histories: per-history bounds, their prefix sum, the
// superblocks (runs of whole DROP blocks whose storage fits the budget), and per superblock a
// processing order sorted by path length so the threads of a warp walk similar distances.
pct_status prepare_layout(pct_ctx* ctx)
{
    if (ctx->layout_ready) return PCT_OK;
    ctx->paths_valid = false;
    const pct_config& c = ctx->cfg;
    const long long n = ctx->n_hist;
    cudaStream_t s = ctx->stream;
    std::vector<pct_ctx::Superblock> old = ctx->sbs;
    ctx->sbs.clear();
    ctx->two_phase = false;
    if (ctx->path_limit_bytes >= 0 && n > 0) {
        long long cap = ctx->layout_cap;
        if (n > cap) {
            long long c1 = 0, c2 = 0, c3 = 0, c4 = 0, c5 = 0, c6 = 0, c7 = 0;
            cudaError_t e = grow(ctx->d_bounds, c1, n);
            if (e == cudaSuccess) e = grow(ctx->d_offsets, c2, n + 1);
            if (e == cudaSuccess) e = grow(ctx->d_perm, c3, n);
            if (e == cudaSuccess) e = grow(ctx->d_path_n, c4, n);
            if (e == cudaSuccess) e = grow(ctx->d_chord, c5, n);
            if (e == cudaSuccess) e = grow(ctx->d_scan_tmp, c6, pct::scan_tile_scratch_elems(n));
            if (e == cudaSuccess) e = grow(ctx->d_hist_tmp, c7, 2LL * kMaxBoundKey);
            const size_t per4 = align256((size_t)n * 4), per8 = align256((size_t)n * 8);
            if (e == cudaSuccess) e = grow(ctx->d_sorted_block, ctx->sorted_cap, (long long)(12 * per4 + per8));
            if (e == cudaSuccess) {
                char* b = ctx->d_sorted_block;
                float* f[10];
                for (int i = 0; i < 10; i++) f[i] = reinterpret_cast<float*>(b + per4 * i);
                ctx->sorted_hist = pct::HistorySoA{f[0], f[1], f[2], f[3], f[4], f[5], f[6], f[7], f[8], f[9], nullptr,
                                                   reinterpret_cast<uint32_t*>(b + per4 * 10)};
                ctx->d_bounds_sorted = reinterpret_cast<int*>(b + per4 * 11);
                ctx->d_offsets_sorted = reinterpret_cast<long long*>(b + per4 * 12);
            }
            if (e != cudaSuccess) {
                cudaGetLastError();
                ctx->layout_cap = 0;
                ctx->layout_ready = true;  // fall back to the single-pass kernel
                return PCT_OK;
            }
            ctx->layout_cap = n;
        }
        cudaError_t e = pct::launch_path_bounds(ctx->geo, ctx->tables, ctx->hist, n, c.DROP_BLOCK_SIZE,
                                                c.HISTORIES_PER_BLOCK, ctx->d_bounds, s);
        if (e == cudaSuccess) e = pct::exclusive_scan_i32_to_i64(ctx->d_bounds, n, ctx->d_offsets, ctx->d_scan_tmp, s);
        if (e != cudaSuccess) return ctx_fail(ctx, PCT_ERR_CUDA, "path layout kernels", e);
        ctx->launches += 4;
        // offsets at DROP-block boundaries, and the total
        const long long B = c.DROP_BLOCK_SIZE;
        const long long nb = (n + B - 1) / B;
        std::vector<long long> boff(nb + 1);
        e = cudaMemcpy2DAsync(boff.data(), sizeof(long long), ctx->d_offsets, sizeof(long long) * B, sizeof(long long),
                              nb, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(&boff[nb], ctx->d_offsets + n, sizeof(long long), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return ctx_fail(ctx, PCT_ERR_CUDA, "path layout copy", e);
        long long limit = ctx->path_limit_bytes;
        if (limit == 0) {
            size_t free_b = 0, total_b = 0;
            cudaMemGetInfo(&free_b, &total_b);
            limit = (long long)((double)(free_b + (size_t)ctx->paths_cap * 4) * 0.75);
        }
        const long long limit_elems = limit / 4;
        long long sb_begin_blk = 0, max_elems = 0;
        bool ok = true;
        while (sb_begin_blk < nb) {
            long long end_blk = sb_begin_blk;
            while (end_blk < nb && boff[end_blk + 1] - boff[sb_begin_blk] <= limit_elems) end_blk++;
            if (end_blk == sb_begin_blk) {
                ok = false;  // one DROP block alone exceeds the budget
                break;
            }
            const long long hb = sb_begin_blk * B, he = end_blk * B < n ? end_blk * B : n;
            ctx->sbs.push_back({hb, he, boff[sb_begin_blk]});
            const long long el = boff[end_blk] - boff[sb_begin_blk];
            if (el > max_elems) max_elems = el;
            sb_begin_blk = end_blk;
        }
        if (ok) {
            e = grow(ctx->d_paths, ctx->paths_cap, max_elems);
            if (e != cudaSuccess) {
                cudaGetLastError();
                ok = false;
            }
        }
        if (ok) {
            // path kernel chunks: runs of PATH_CHUNK_BLOCKS DROP blocks inside each superblock
            // (one chunk per superblock when 0), each sorted by path-length bound
            ctx->chunks.clear();
            for (size_t i = 0; i < ctx->sbs.size(); i++) {
                const auto& sb = ctx->sbs[i];
                const long long step = c.PATH_CHUNK_BLOCKS > 0 ? (long long)c.PATH_CHUNK_BLOCKS * B : sb.h_end - sb.h_begin;
                for (long long h0 = sb.h_begin; h0 < sb.h_end; h0 += step)
                    ctx->chunks.push_back({(int)i, h0, h0 + step < sb.h_end ? h0 + step : sb.h_end});
            }
            for (const auto& ch : ctx->chunks) {
                if (c.PATH_ORDER_WINDOW > 0) {
                    e = pct::window_sort_by_key(ctx->d_bounds, ch.h_begin, ch.h_end - ch.h_begin, kMaxBoundKey,
                                                c.PATH_ORDER_WINDOW, ctx->d_perm + ch.h_begin, s);
                    ctx->launches += 1;
                } else {
                    e = pct::bucket_sort_by_key(ctx->d_bounds, ch.h_begin, ch.h_end - ch.h_begin, kMaxBoundKey,
                                                ctx->d_hist_tmp, ctx->d_perm + ch.h_begin, s);
                    ctx->launches += 3;
                }
                if (e != cudaSuccess) return ctx_fail(ctx, PCT_ERR_CUDA, "path order sort", e);
            }
            // the path kernel's inputs gathered once into its processing order, so that each of its
            // loads reads consecutive histories instead of one sector per history and field
            e = pct::launch_gather_path_inputs(ctx->hist, ctx->d_perm, ctx->d_bounds, ctx->d_offsets, n,
                                               ctx->sorted_hist, ctx->d_bounds_sorted, ctx->d_offsets_sorted, s);
            if (e != cudaSuccess) return ctx_fail(ctx, PCT_ERR_CUDA, "path input gather", e);
            ctx->launches += 1;
            ctx->two_phase = true;
        } else {
            ctx->sbs.clear();
            ctx->chunks.clear();
        }
    }
    // the captured iteration is reusable only if the launch structure is unchanged
    bool same = ctx->sbs.size() == old.size();
    for (size_t i = 0; same && i < old.size(); i++)
        same = old[i].h_begin == ctx->sbs[i].h_begin && old[i].h_end == ctx->sbs[i].h_end &&
               old[i].off_begin == ctx->sbs[i].off_begin;
    if (!same) release_graph(ctx);
    ctx->layout_ready = true;
    return PCT_OK;
}

}  // namespace

pct_status pct::layout_prepare(pct_ctx* ctx) { return prepare_layout(ctx); }

pct::HistorySoA pct::sorted_path_inputs(const pct_ctx* ctx, long long p) { return sorted_from(ctx, p); }

namespace {

#ifndef PCT_CHAIN_PDL
#define PCT_CHAIN_PDL 1
#endif
constexpr bool kChainPdl = PCT_CHAIN_PDL != 0;

// Enqueue one DROP iteration (DROP_full_tx_iteration, B.cu:9547-9582).  Two-phase: per
// superblock, the path kernel over all its covered histories, then per DROP block the
// gather/update/scatter kernel and the image update.  Single-pass fallback: per block the fused
// MLP + scatter kernel and the image update.
pct_status enqueue_iteration(pct_ctx* ctx, cudaStream_t s, long long* launches, bool with_paths, bool chain_pdl)
{
    const pct_config& c = ctx->cfg;
    const long long n = ctx->n_hist;
    long long nl = 0;
    cudaError_t e = cudaSuccess;
    // With chain_pdl, within a run of DROP blocks every kernel but the first is launched as a
    // programmatic dependent of the one before it (both wait on it in griddepcontrol.wait before
    // touching the image or the accumulator), so its launch and CTA ramp overlap the
    // predecessor's tail.  Batch graphs capture without it (their branches share the SMs).  The
    // first block kernel of a run follows a cross-stream join and keeps a full dependency.
    auto blocks = [&](const pct_ctx::Superblock& sb, long long h0, long long h1) -> pct_status {
        bool pdl = false;
        for (long long start = h0; start < h1; start += c.DROP_BLOCK_SIZE) {
            const long long covered = covered_in_block(c, n, start);
            if (covered <= 0) continue;
            e = pct::launch_drop_phase2(ctx->geo, ctx->d_x, ctx->d_acc, ctx->d_normA, ctx->fixed, ctx->hist.WEPL, ctx->d_offsets,
                                        sb.off_begin, ctx->d_paths, ctx->d_path_n, ctx->d_chord, start, covered, s,
                                        pdl && chain_pdl);
            if (e != cudaSuccess) return ctx_fail(ctx, PCT_ERR_CUDA, "DROP block kernel", e);
            e = pct::launch_image_update(ctx->geo, ctx->d_x, ctx->d_acc, ctx->d_normA, ctx->fixed, s, chain_pdl);
            if (e != cudaSuccess) return ctx_fail(ctx, PCT_ERR_CUDA, "image_update kernel", e);
            pdl = true;
            nl += 2;
        }
        return PCT_OK;
    };
    if (ctx->two_phase && !with_paths) {
        for (const auto& sb : ctx->sbs) {
            pct_status st = blocks(sb, sb.h_begin, sb.h_end);
            if (st != PCT_OK) return st;
        }
    } else if (ctx->two_phase) {
        // The path kernel of chunk k+1 runs on the low-priority path stream while the DROP blocks
        // of chunk k run on `s`; a superblock's storage is rewritten only after its last block.
        const size_t need = ctx->chunks.size() + ctx->sbs.size() + 1;
        while (ctx->events.size() < need) {
            cudaEvent_t ev = nullptr;
            e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
            if (e != cudaSuccess) return ctx_fail(ctx, PCT_ERR_CUDA, "cudaEventCreate", e);
            ctx->events.push_back(ev);
        }
        cudaStream_t p = ctx->path_stream;
        cudaEvent_t* ev_chunk = ctx->events.data();
        cudaEvent_t* ev_sb = ev_chunk + ctx->chunks.size();
        cudaEvent_t ev_fork = ev_sb[ctx->sbs.size()];
        e = cudaEventRecord(ev_fork, s);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(p, ev_fork, 0);
        if (e != cudaSuccess) return ctx_fail(ctx, PCT_ERR_CUDA, "stream fork", e);
        for (size_t k = 0; k < ctx->chunks.size(); k++) {
            const auto& ch = ctx->chunks[k];
            const auto& sb = ctx->sbs[ch.sb];
            if (ch.sb > 0 && ch.h_begin == sb.h_begin) {
                e = cudaStreamWaitEvent(p, ev_sb[ch.sb - 1], 0);
                if (e != cudaSuccess) return ctx_fail(ctx, PCT_ERR_CUDA, "stream wait", e);
            }
            e = pct::launch_mlp_phase1_exact(ctx->geo, ctx->tables, ctx->d_steps, ctx->kmax,
                                             sorted_from(ctx, ch.h_begin), ctx->d_perm + ch.h_begin,
                                             ch.h_end - ch.h_begin, ctx->d_offsets_sorted + ch.h_begin, sb.off_begin,
                                             ctx->d_bounds_sorted + ch.h_begin, ctx->d_paths, ctx->d_path_n,
                                             ctx->d_chord, ctx->d_counters, p);
            if (e != cudaSuccess) return ctx_fail(ctx, PCT_ERR_CUDA, "MLP path kernel", e);
            nl += 1;
            e = cudaEventRecord(ev_chunk[k], p);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(s, ev_chunk[k], 0);
            if (e != cudaSuccess) return ctx_fail(ctx, PCT_ERR_CUDA, "stream join", e);
            pct_status st = blocks(sb, ch.h_begin, ch.h_end);
            if (st != PCT_OK) return st;
            if (ch.h_end == sb.h_end) {
                e = cudaEventRecord(ev_sb[ch.sb], s);
                if (e != cudaSuccess) return ctx_fail(ctx, PCT_ERR_CUDA, "event record", e);
            }
        }
    } else {
        if (c.PROJECTION_ALGORITHM != PCT_DROP || c.SCATTER_MODE != PCT_SCATTER_ATOMIC)
            return ctx_fail(ctx, PCT_ERR_STATE, "robust algorithms and the deterministic scatter need path storage");
        for (long long start = 0; start < n; start += c.DROP_BLOCK_SIZE) {
            const long long covered = covered_in_block(c, n, start);
            if (covered <= 0) continue;
            e = pct::launch_drop_block_exact(ctx->geo, ctx->tables, ctx->d_steps, ctx->kmax, ctx->d_x, ctx->d_acc,
                                             ctx->hist, start, covered, ctx->d_counters, s);
            if (e != cudaSuccess) return ctx_fail(ctx, PCT_ERR_CUDA, "drop_block kernel", e);
            e = pct::launch_image_update(ctx->geo, ctx->d_x, ctx->d_acc, ctx->d_normA, ctx->fixed, s);
            if (e != cudaSuccess) return ctx_fail(ctx, PCT_ERR_CUDA, "image_update kernel", e);
            nl += 2;
        }
    }
    *launches = nl;
    return PCT_OK;
}

}  // namespace

extern "C" pct_status pct_set_path_storage_limit(pct_ctx* ctx, int64_t bytes)
{
    if (!ctx) return PCT_ERR_ARG;
    if (bytes != ctx->path_limit_bytes) {
        ctx->path_limit_bytes = bytes;
        ctx->layout_ready = false;
        release_graph(ctx);
    }
    return PCT_OK;
}

extern "C" int pct_path_storage_superblocks(pct_ctx* ctx)
{
    if (!ctx) return -1;
    if (ctx->n_hist > 0 && prepare_layout(ctx) != PCT_OK) return -1;
    return ctx->two_phase ? (int)ctx->sbs.size() : 0;
}

namespace {

// Captures one DROP iteration on the context's own stream: the full iteration or the DROP blocks
// alone (precomputed paths), instantiated for pct_drop_full_tx_iteration, or the full iteration
// kept as a graph for batches.
enum class Capture { kFull, kReuse, kBatch };

pct_status capture_iteration(pct_ctx* ctx, Capture mode)
{
    const bool reuse = mode == Capture::kReuse, batch = mode == Capture::kBatch;
    cudaGraphExec_t& exec = reuse ? ctx->reuse_exec : ctx->iter_exec;
    long long& exec_launches = batch ? ctx->batch_launches : (reuse ? ctx->reuse_launches : ctx->iter_launches);
    if (batch ? ctx->batch_graph != nullptr : exec != nullptr) return PCT_OK;
    // Capture on the context's own stream (capture is not allowed on the legacy stream).
    cudaStream_t cs = ctx->own_stream;
    if (ctx->stream != cs) PCT_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    cudaGraph_t graph = nullptr;
    PCT_CUDA_TRY(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    long long nl = 0;
    pct_status st = enqueue_iteration(ctx, cs, &nl, !reuse, kChainPdl && !batch);
    cudaError_t e = cudaStreamEndCapture(cs, &graph);
    if (st != PCT_OK) {
        if (graph) cudaGraphDestroy(graph);
        return st;
    }
    if (e != cudaSuccess) return ctx_fail(ctx, PCT_ERR_CUDA, "cudaStreamEndCapture", e);
    if (ctx->l2_window) {
        // every kernel node gets the window over the image and accumulator
        size_t count = 0;
        e = cudaGraphGetNodes(graph, nullptr, &count);
        std::vector<cudaGraphNode_t> nodes(count);
        if (e == cudaSuccess && count) e = cudaGraphGetNodes(graph, nodes.data(), &count);
        cudaKernelNodeAttrValue v{};
        v.accessPolicyWindow = ctx->l2_policy;
        for (size_t i = 0; e == cudaSuccess && i < count; ++i) {
            cudaGraphNodeType type;
            e = cudaGraphNodeGetType(nodes[i], &type);
            if (e == cudaSuccess && type == cudaGraphNodeTypeKernel)
                e = cudaGraphKernelNodeSetAttribute(nodes[i], cudaKernelNodeAttributeAccessPolicyWindow, &v);
        }
        if (e != cudaSuccess) {
            cudaGraphDestroy(graph);
            return ctx_fail(ctx, PCT_ERR_CUDA, "L2 access-policy window on the captured kernels", e);
        }
    }
    exec_launches = nl;
    if (batch) {
        ctx->batch_graph = graph;
        return PCT_OK;
    }
    // node priorities: the captured kernels keep their streams' priorities
    e = cudaGraphInstantiateWithFlags(&exec, graph, cudaGraphInstantiateFlagUseNodePriority);
    cudaGraphDestroy(graph);
    ctx->graph_captures++;
    if (e != cudaSuccess) {
        exec = nullptr;
        exec_launches = 0;
        return ctx_fail(ctx, PCT_ERR_CUDA, "cudaGraphInstantiate", e);
    }
    return PCT_OK;
}

}  // namespace

pct_status pct::iteration_graph(pct_ctx* ctx, cudaGraph_t* graph, long long* launches)
{
    if (ctx->n_hist <= 0) return ctx_fail(ctx, PCT_ERR_STATE, "no reconstruction histories loaded");
    cudaSetDevice(ctx->device);
    pct_status st = prepare_layout(ctx);
    if (st == PCT_OK) st = capture_iteration(ctx, Capture::kBatch);
    if (st != PCT_OK) return st;
    *graph = ctx->batch_graph;
    *launches = ctx->batch_launches;
    return PCT_OK;
}

void pct::iteration_ran(pct_ctx* ctx)
{
    ctx->launches += ctx->batch_launches;
    if (ctx->two_phase && ctx->sbs.size() == 1) ctx->paths_valid = true;
}

extern "C" pct_status pct_drop_full_tx_iteration(pct_ctx* ctx, int iteration)
{
    if (!ctx) return PCT_ERR_ARG;
    if (ctx->n_hist <= 0) return ctx_fail(ctx, PCT_ERR_STATE, "no reconstruction histories loaded");
    cudaSetDevice(ctx->device);
    using clock = std::chrono::steady_clock;
    const auto t0 = clock::now();
    const bool had_layout = ctx->layout_ready;
    pct_status lst = prepare_layout(ctx);
    if (lst != PCT_OK) return lst;
    const auto t1 = clock::now();
    // Precomputed-path DROP: with every path resident (one superblock) and computed by an
    // earlier iteration, the iteration is the DROP blocks alone.
    const bool resident = ctx->two_phase && ctx->sbs.size() == 1;
    const bool reuse = ctx->reuse_paths && resident && ctx->paths_valid;
    const long long captures = ctx->graph_captures;
    pct_status st = capture_iteration(ctx, reuse ? Capture::kReuse : Capture::kFull);
    if (st != PCT_OK) return st;
    const auto t2 = clock::now();
    PCT_CUDA_TRY(cudaGraphLaunch(reuse ? ctx->reuse_exec : ctx->iter_exec, ctx->stream));
    if (ctx->trace) {
        const auto ms = [](clock::time_point a, clock::time_point b) {
            return std::chrono::duration<double, std::milli>(b - a).count();
        };
        fprintf(stderr, "pct_trace: iteration %d: layout %s %.2f ms, graph %s %.2f ms, launch %.2f ms, superblocks %zu\n",
                iteration, had_layout ? "kept" : "built", ms(t0, t1),
                ctx->graph_captures != captures ? "captured" : "reused", ms(t1, t2), ms(t2, clock::now()),
                ctx->sbs.size());
    }
    ctx->launches += reuse ? ctx->reuse_launches : ctx->iter_launches;
    if (resident) ctx->paths_valid = true;
    return PCT_OK;
}

extern "C" pct_status pct_autotune_schedule(pct_ctx* ctx, int32_t chosen[3])
{
    // Times one captured DROP iteration of this context's own histories per schedule candidate and
    // keeps the fastest, one knob at a time: PATH_CHUNK_BLOCKS (how many DROP blocks one path-kernel
    // launch covers), then PATH_CTA_THREADS (histories per path-kernel CTA), then PATH_ORDER_WINDOW
    // (how far the path-length sort reaches).  These change only the schedule, never a result; the
    // image is restored afterwards.
    if (!ctx) return PCT_ERR_ARG;
    if (ctx->n_hist <= 0) return ctx_fail(ctx, PCT_ERR_STATE, "pct_autotune: no reconstruction histories loaded");
    PCT_CUDA_TRY(cudaSetDevice(ctx->device));
    const size_t bytes = (size_t)ctx->geo.padded_voxels * sizeof(float);
    float* saved = nullptr;
    cudaEvent_t a = nullptr, b = nullptr;
    cudaError_t e = cudaMalloc(&saved, bytes);
    if (e == cudaSuccess) e = cudaEventCreate(&a);
    if (e == cudaSuccess) e = cudaEventCreate(&b);
    if (e == cudaSuccess) e = cudaMemcpyAsync(saved, ctx->d_x, bytes, cudaMemcpyDeviceToDevice, ctx->stream);
    pct_status st = e == cudaSuccess ? PCT_OK : ctx_fail(ctx, PCT_ERR_CUDA, "pct_autotune setup", e);
    const bool reuse = ctx->reuse_paths;
    ctx->reuse_paths = false;
    int32_t* knobs[3] = {&ctx->cfg.PATH_CHUNK_BLOCKS, &ctx->cfg.PATH_CTA_THREADS, &ctx->cfg.PATH_ORDER_WINDOW};
    const int32_t original[3] = {*knobs[0], *knobs[1], *knobs[2]};
    static const int kChunks[] = {0, 4, 8, 16, 32, 64, 128};
    static const int kCta[] = {64, 128, 256};
    static const int kWindow[] = {0, 4096, 16384};
    const int* candidates[3] = {kChunks, kCta, kWindow};
    const int ncand[3] = {7, 3, 3};
    auto apply = [&]() {
        ctx->geo.path_cta_threads = ctx->cfg.PATH_CTA_THREADS;
        ctx->layout_ready = false;
        release_graph(ctx);
    };
    for (int knob = 0; knob < 3 && st == PCT_OK; knob++) {
        float best_ms = 0.f;
        int best = *knobs[knob];
        bool any = false;
        for (int c = 0; c < ncand[knob] && st == PCT_OK; c++) {
            cudaStreamSynchronize(ctx->stream);
            *knobs[knob] = candidates[knob][c];
            apply();
            st = pct_drop_full_tx_iteration(ctx, 1);  // layout, capture and one untimed run
            if (st != PCT_OK) break;
            e = cudaEventRecord(a, ctx->stream);
            if (e == cudaSuccess) st = pct_drop_full_tx_iteration(ctx, 1);
            if (e == cudaSuccess && st == PCT_OK) e = cudaEventRecord(b, ctx->stream);
            if (e == cudaSuccess && st == PCT_OK) e = cudaEventSynchronize(b);
            float ms = 0.f;
            if (e == cudaSuccess && st == PCT_OK) e = cudaEventElapsedTime(&ms, a, b);
            if (e != cudaSuccess && st == PCT_OK) st = ctx_fail(ctx, PCT_ERR_CUDA, "pct_autotune timing", e);
            if (st == PCT_OK && (!any || ms < best_ms)) {
                best_ms = ms;
                best = candidates[knob][c];
                any = true;
            }
        }
        *knobs[knob] = best;
    }
    cudaStreamSynchronize(ctx->stream);
    if (st != PCT_OK)
        for (int k = 0; k < 3; k++) *knobs[k] = original[k];
    apply();
    ctx->reuse_paths = reuse;
    if (saved) {
        e = cudaMemcpyAsync(ctx->d_x, saved, bytes, cudaMemcpyDeviceToDevice, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess && st == PCT_OK) st = ctx_fail(ctx, PCT_ERR_CUDA, "pct_autotune restore", e);
        cudaFree(saved);
    }
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    if (chosen)
        for (int k = 0; k < 3; k++) chosen[k] = *knobs[k];
    return st;
}

extern "C" pct_status pct_autotune(pct_ctx* ctx, int32_t* chosen_path_chunk_blocks)
{
    int32_t chosen[3] = {0, 0, 0};
    const pct_status st = pct_autotune_schedule(ctx, chosen);
    if (st == PCT_OK && chosen_path_chunk_blocks) *chosen_path_chunk_blocks = chosen[0];
    return st;
}

extern "C" pct_status pct_profile_drop_iteration(pct_ctx* ctx, double ms_out[3], int64_t launches_out[3])
{
    if (!ctx || !ms_out || !launches_out) return PCT_ERR_ARG;
    if (ctx->n_hist <= 0) return ctx_fail(ctx, PCT_ERR_STATE, "no reconstruction histories loaded");
    cudaSetDevice(ctx->device);
    pct_status lst = prepare_layout(ctx);
    if (lst != PCT_OK) return lst;
    const pct_config& c = ctx->cfg;
    const long long n = ctx->n_hist;
    cudaStream_t s = ctx->stream;
    struct Timed {
        int group;
        cudaEvent_t a, b;
    };
    std::vector<Timed> ev;
    auto begin = [&](int group) {
        Timed t{group, nullptr, nullptr};
        cudaEventCreate(&t.a);
        cudaEventCreate(&t.b);
        cudaEventRecord(t.a, s);
        ev.push_back(t);
    };
    auto end = [&]() { cudaEventRecord(ev.back().b, s); };
    cudaError_t e = cudaSuccess;
    if (ctx->two_phase) {
        for (const auto& sb : ctx->sbs) {
            begin(0);
            e = pct::launch_mlp_phase1_exact(ctx->geo, ctx->tables, ctx->d_steps, ctx->kmax,
                                             sorted_from(ctx, sb.h_begin), ctx->d_perm + sb.h_begin,
                                             sb.h_end - sb.h_begin, ctx->d_offsets_sorted + sb.h_begin, sb.off_begin,
                                             ctx->d_bounds_sorted + sb.h_begin, ctx->d_paths, ctx->d_path_n,
                                             ctx->d_chord, ctx->d_counters, s);
            end();
            for (long long st = sb.h_begin; e == cudaSuccess && st < sb.h_end; st += c.DROP_BLOCK_SIZE) {
                const long long covered = covered_in_block(c, n, st);
                if (covered <= 0) continue;
                begin(1);
                e = pct::launch_drop_phase2(ctx->geo, ctx->d_x, ctx->d_acc, ctx->d_normA, ctx->fixed, ctx->hist.WEPL, ctx->d_offsets,
                                            sb.off_begin, ctx->d_paths, ctx->d_path_n, ctx->d_chord, st, covered, s);
                end();
                begin(2);
                if (e == cudaSuccess) e = pct::launch_image_update(ctx->geo, ctx->d_x, ctx->d_acc, ctx->d_normA, ctx->fixed, s);
                end();
            }
            if (e != cudaSuccess) break;
        }
    } else {
        if (c.PROJECTION_ALGORITHM != PCT_DROP || c.SCATTER_MODE != PCT_SCATTER_ATOMIC)
            return ctx_fail(ctx, PCT_ERR_STATE, "robust algorithms and the deterministic scatter need path storage");
        for (long long st = 0; e == cudaSuccess && st < n; st += c.DROP_BLOCK_SIZE) {
            const long long covered = covered_in_block(c, n, st);
            if (covered <= 0) continue;
            begin(1);
            e = pct::launch_drop_block_exact(ctx->geo, ctx->tables, ctx->d_steps, ctx->kmax, ctx->d_x, ctx->d_acc,
                                             ctx->hist, st, covered, ctx->d_counters, s);
            end();
            begin(2);
            if (e == cudaSuccess) e = pct::launch_image_update(ctx->geo, ctx->d_x, ctx->d_acc, ctx->d_normA, ctx->fixed, s);
            end();
        }
    }
    cudaError_t se = cudaStreamSynchronize(s);
    for (int g = 0; g < 3; g++) {
        ms_out[g] = 0;
        launches_out[g] = 0;
    }
    for (auto& t : ev) {
        float ms = 0;
        if (se == cudaSuccess && e == cudaSuccess) cudaEventElapsedTime(&ms, t.a, t.b);
        ms_out[t.group] += ms;
        launches_out[t.group] += 1;
        cudaEventDestroy(t.a);
        cudaEventDestroy(t.b);
    }
    if (e != cudaSuccess) return ctx_fail(ctx, PCT_ERR_CUDA, "profiled iteration launch", e);
    if (se != cudaSuccess) return ctx_fail(ctx, PCT_ERR_CUDA, "profiled iteration sync", se);
    ctx->launches += launches_out[0] + launches_out[1] + launches_out[2];
    return PCT_OK;
}

extern "C" pct_status pct_set_path_reuse(pct_ctx* ctx, int enable)
{
    if (!ctx) return PCT_ERR_ARG;
    ctx->reuse_paths = enable != 0;
    return PCT_OK;
}

extern "C" pct_status pct_stage_reconstruction_histories(pct_ctx* ctx, const pct_histories* h, int64_t n,
                                                         pct_memory where)
{
    if (!ctx || !h || n < 0 || n > 0x7fffffffLL) return PCT_ERR_ARG;
    const void* src[12] = {h->x_entry, h->y_entry, h->z_entry, h->x_exit, h->y_exit, h->z_exit,
                           h->xy_entry_angle, h->xz_entry_angle, h->xy_exit_angle, h->xz_exit_angle,
                           h->WEPL, h->first_MLP_voxel};
    if (n > 0)
        for (const void* p : src)
            if (!p) return ctx_fail(ctx, PCT_ERR_ARG, "pct_stage_reconstruction_histories: NULL array");
    PCT_CUDA_TRY(cudaSetDevice(ctx->device));
    if (!ctx->copy_stream) {
        PCT_CUDA_TRY(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
        PCT_CUDA_TRY(cudaEventCreateWithFlags(&ctx->stage_done, cudaEventDisableTiming));
        PCT_CUDA_TRY(cudaEventCreateWithFlags(&ctx->stage_free, cudaEventDisableTiming));
        PCT_CUDA_TRY(cudaEventRecord(ctx->stage_free, ctx->stream));
    }
    if (n > ctx->stage_cap) {
        PCT_CUDA_TRY(cudaStreamSynchronize(ctx->copy_stream));
        PCT_CUDA_TRY(cudaEventSynchronize(ctx->stage_free));
        cudaFree(ctx->d_stage_block);
        ctx->d_stage_block = nullptr;
        ctx->stage_cap = 0;
        cudaError_t e = cudaMalloc(&ctx->d_stage_block, align256((size_t)n * 4) * 12);
        if (e != cudaSuccess) return ctx_fail(ctx, PCT_ERR_NOMEM, "cudaMalloc(staged histories)", e);
        ctx->stage_cap = n;
    }
    // the staging arrays are rewritten only after the last pct_use_staged_histories read them
    PCT_CUDA_TRY(cudaStreamWaitEvent(ctx->copy_stream, ctx->stage_free, 0));
    const size_t per = align256((size_t)ctx->stage_cap * 4);
    const cudaMemcpyKind kind = where == PCT_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    for (int i = 0; i < 12 && n > 0; i++)
        PCT_CUDA_TRY(cudaMemcpyAsync(static_cast<char*>(ctx->d_stage_block) + per * i, src[i], (size_t)n * 4, kind,
                                     ctx->copy_stream));
    PCT_CUDA_TRY(cudaEventRecord(ctx->stage_done, ctx->copy_stream));
    ctx->stage_n = n;
    ctx->staged = true;
    return PCT_OK;
}

extern "C" pct_status pct_use_staged_histories(pct_ctx* ctx)
{
    if (!ctx) return PCT_ERR_ARG;
    if (!ctx->staged) return ctx_fail(ctx, PCT_ERR_STATE, "pct_use_staged_histories: nothing staged");
    PCT_CUDA_TRY(cudaSetDevice(ctx->device));
    PCT_CUDA_TRY(cudaStreamWaitEvent(ctx->stream, ctx->stage_done, 0));
    const size_t per = align256((size_t)ctx->stage_cap * 4);
    char* b = static_cast<char*>(ctx->d_stage_block);
    pct_histories d{};
    d.x_entry = reinterpret_cast<const float*>(b);
    d.y_entry = reinterpret_cast<const float*>(b + per);
    d.z_entry = reinterpret_cast<const float*>(b + per * 2);
    d.x_exit = reinterpret_cast<const float*>(b + per * 3);
    d.y_exit = reinterpret_cast<const float*>(b + per * 4);
    d.z_exit = reinterpret_cast<const float*>(b + per * 5);
    d.xy_entry_angle = reinterpret_cast<const float*>(b + per * 6);
    d.xz_entry_angle = reinterpret_cast<const float*>(b + per * 7);
    d.xy_exit_angle = reinterpret_cast<const float*>(b + per * 8);
    d.xz_exit_angle = reinterpret_cast<const float*>(b + per * 9);
    d.WEPL = reinterpret_cast<const float*>(b + per * 10);
    d.first_MLP_voxel = reinterpret_cast<const uint32_t*>(b + per * 11);
    const pct_status st = pct_set_reconstruction_histories(ctx, &d, ctx->stage_n, PCT_DEVICE);
    if (st != PCT_OK) return st;
    PCT_CUDA_TRY(cudaEventRecord(ctx->stage_free, ctx->stream));
    ctx->staged = false;
    return PCT_OK;
}

extern "C" pct_status pct_set_l2_window(pct_ctx* ctx, int enable)
{
    if (!ctx || !ctx->d_x) return PCT_ERR_ARG;
    PCT_CUDA_TRY(cudaSetDevice(ctx->device));
    PCT_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    if (enable) {
        int max_persist = 0, max_window = 0;
        PCT_CUDA_TRY(cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, ctx->device));
        PCT_CUDA_TRY(cudaDeviceGetAttribute(&max_window, cudaDevAttrMaxAccessPolicyWindowSize, ctx->device));
        if (max_persist <= 0 || max_window <= 0)
            return ctx_fail(ctx, PCT_ERR_STATE, "device has no persisting L2 set-aside", cudaSuccess);
        const size_t window = std::min(ctx->image_block_bytes, static_cast<size_t>(max_window));
        const size_t aside = std::min(window, static_cast<size_t>(max_persist));
        PCT_CUDA_TRY(cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, aside));
        ctx->l2_policy.base_ptr = ctx->d_x;
        ctx->l2_policy.num_bytes = window;
        ctx->l2_policy.hitRatio = static_cast<float>(std::min(1.0, static_cast<double>(aside) / window));
        ctx->l2_policy.hitProp = cudaAccessPropertyPersisting;
        ctx->l2_policy.missProp = cudaAccessPropertyStreaming;
    } else if (ctx->l2_window) {
        PCT_CUDA_TRY(cudaCtxResetPersistingL2Cache());
        PCT_CUDA_TRY(cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, 0));
    }
    if ((enable != 0) != ctx->l2_window) {
        ctx->l2_window = enable != 0;
        release_graph(ctx);  // recaptured with (or without) the window on its kernel nodes
    }
    return PCT_OK;
}

extern "C" pct_status pct_drop_gpu(pct_ctx* ctx)
{
    // DROP_GPU (B.cu:9848) with DROP_TX_MODE = FULL_TX: TVS before (TVS_FIRST) or after each
    // iteration, on the device image.  (With TVS_FIRST off the reference perturbs only the host
    // copy it writes out, which the next iteration does not see; here the perturbation is kept.)
    if (!ctx) return PCT_ERR_ARG;
    const bool tvs = ctx->cfg.TVS_ON != 0, first = ctx->cfg.TVS_FIRST != 0;
    for (int it = 1; it <= ctx->cfg.ITERATIONS; it++) {
        pct_status st = PCT_OK;
        if (tvs && first) st = pct_ntvs_iteration(ctx, it);
        if (st == PCT_OK) st = pct_drop_full_tx_iteration(ctx, it);
        if (st == PCT_OK && tvs && !first) st = pct_ntvs_iteration(ctx, it);
        if (st != PCT_OK) return st;
    }
    return PCT_OK;
}

extern "C" pct_status pct_calculate_x_update(pct_ctx* ctx, int64_t start_position, int64_t num_histories)
{
    if (!ctx || start_position < 0 || num_histories < 0 || start_position + num_histories > ctx->n_hist)
        return PCT_ERR_ARG;
    if (ctx->cfg.PROJECTION_ALGORITHM != PCT_DROP || ctx->cfg.SCATTER_MODE != PCT_SCATTER_ATOMIC)
        return ctx_fail(ctx, PCT_ERR_STATE,
                        "calculate_x_update is the atomic DROP update; other modes run by iteration");
    cudaSetDevice(ctx->device);
    cudaError_t e = pct::launch_drop_block_exact(ctx->geo, ctx->tables, ctx->d_steps, ctx->kmax, ctx->d_x, ctx->d_acc,
                                                 ctx->hist, start_position, num_histories, ctx->d_counters, ctx->stream);
    if (e != cudaSuccess) return ctx_fail(ctx, PCT_ERR_CUDA, "drop_block kernel", e);
    if (num_histories > 0) ctx->launches += 1;
    return PCT_OK;
}

extern "C" pct_status pct_image_update(pct_ctx* ctx)
{
    if (!ctx) return PCT_ERR_ARG;
    cudaSetDevice(ctx->device);
    cudaError_t e = pct::launch_image_update(ctx->geo, ctx->d_x, ctx->d_acc, ctx->d_normA, ctx->fixed, ctx->stream);
    if (e != cudaSuccess) return ctx_fail(ctx, PCT_ERR_CUDA, "image_update kernel", e);
    ctx->launches += 1;
    return PCT_OK;
}

extern "C" pct_status pct_mlp_precision(pct_ctx* ctx, int64_t start, int64_t n, double* dev_t_cm, double* dev_v_cm,
                                        int32_t* mismatched_steps, int32_t* ill_posed_steps, pct_memory where)
{
    if (!ctx || start < 0 || n < 0 || start + n > ctx->n_hist || !dev_t_cm || !dev_v_cm || !mismatched_steps ||
        !ill_posed_steps)
        return PCT_ERR_ARG;
    if (n == 0) return PCT_OK;
    cudaSetDevice(ctx->device);
    double *dt = dev_t_cm, *dv = dev_v_cm;
    int *mm = mismatched_steps, *ip = ill_posed_steps;
    void* scratch = nullptr;
    if (where == PCT_HOST) {
        PCT_CUDA_TRY(cudaMalloc(&scratch, (size_t)n * 24));
        dt = static_cast<double*>(scratch);
        dv = dt + n;
        mm = reinterpret_cast<int*>(dv + n);
        ip = mm + n;
    }
    cudaError_t e = pct::launch_mlp_precision(ctx->geo, ctx->tables, ctx->d_steps, ctx->kmax, ctx->hist, start, n, dt,
                                              dv, mm, ip, ctx->stream);
    if (e == cudaSuccess && where == PCT_HOST) {
        e = cudaMemcpyAsync(dev_t_cm, dt, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(dev_v_cm, dv, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(mismatched_steps, mm, sizeof(int) * n, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(ill_posed_steps, ip, sizeof(int) * n, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    }
    cudaFree(scratch);
    if (e != cudaSuccess) return ctx_fail(ctx, PCT_ERR_CUDA, "MLP precision kernel", e);
    ctx->launches += 1;
    return PCT_OK;
}

extern "C" pct_status pct_mlp_paths(pct_ctx* ctx, int64_t start, int64_t n, int32_t stride, uint32_t* path_counts,
                                    uint32_t* path_voxels, double* chord_lengths, double* a_dot_x, pct_memory where)
{
    if (!ctx || start < 0 || n < 0 || start + n > ctx->n_hist || stride < 0) return PCT_ERR_ARG;
    if (path_voxels && stride == 0) return PCT_ERR_ARG;
    if (n == 0) return PCT_OK;
    cudaSetDevice(ctx->device);
    uint32_t *dc = path_counts, *dv = path_voxels;
    double *dl = chord_lengths, *da = a_dot_x;
    void* tmp = nullptr;
    if (where == PCT_HOST) {
        const size_t bc = path_counts ? align256(n * 4) : 0, bv = path_voxels ? align256((size_t)n * stride * 4) : 0;
        const size_t bl = chord_lengths ? align256(n * 8) : 0, ba = a_dot_x ? align256(n * 8) : 0;
        cudaError_t e = cudaMalloc(&tmp, bc + bv + bl + ba + 256);
        if (e != cudaSuccess) return ctx_fail(ctx, PCT_ERR_NOMEM, "cudaMalloc(mlp_paths)", e);
        char* p = static_cast<char*>(tmp);
        dc = path_counts ? (uint32_t*)p : nullptr;
        p += bc;
        dv = path_voxels ? (uint32_t*)p : nullptr;
        p += bv;
        dl = chord_lengths ? (double*)p : nullptr;
        p += bl;
        da = a_dot_x ? (double*)p : nullptr;
    }
    cudaError_t e = pct::launch_mlp_paths_exact(ctx->geo, ctx->tables, ctx->d_steps, ctx->kmax, ctx->d_x, ctx->hist,
                                                start, n, stride, dc, dv, dl, da, ctx->d_counters, ctx->stream);
    if (e != cudaSuccess) {
        cudaFree(tmp);
        return ctx_fail(ctx, PCT_ERR_CUDA, "mlp_paths kernel", e);
    }
    ctx->launches += 1;
    if (where == PCT_HOST) {
        if (path_counts) e = cudaMemcpyAsync(path_counts, dc, n * 4, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess && path_voxels)
            e = cudaMemcpyAsync(path_voxels, dv, (size_t)n * stride * 4, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess && chord_lengths) e = cudaMemcpyAsync(chord_lengths, dl, n * 8, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess && a_dot_x) e = cudaMemcpyAsync(a_dot_x, da, n * 8, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        cudaFree(tmp);
        if (e != cudaSuccess) return ctx_fail(ctx, PCT_ERR_CUDA, "mlp_paths copy-back", e);
    }
    return PCT_OK;
}

extern "C" pct_status pct_mlp_steps(pct_ctx* ctx, int64_t start, int64_t n, int32_t* steps, pct_memory where)
{
    if (!ctx || !steps || start < 0 || n < 0 || start + n > ctx->n_hist) return PCT_ERR_ARG;
    if (n == 0) return PCT_OK;
    cudaSetDevice(ctx->device);
    int* d = reinterpret_cast<int*>(steps);
    if (where == PCT_HOST) {
        cudaError_t e = cudaMalloc(&d, sizeof(int) * (size_t)n);
        if (e != cudaSuccess) return ctx_fail(ctx, PCT_ERR_NOMEM, "cudaMalloc(mlp_steps)", e);
    }
    cudaError_t e = pct::launch_mlp_steps(ctx->geo, ctx->tables, ctx->kmax, ctx->hist, start, n, d, ctx->stream);
    if (e == cudaSuccess) ctx->launches += 1;
    if (e == cudaSuccess && where == PCT_HOST) {
        e = cudaMemcpyAsync(steps, d, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    }
    if (where == PCT_HOST) cudaFree(d);
    if (e != cudaSuccess) return ctx_fail(ctx, PCT_ERR_CUDA, "mlp_steps", e);
    return PCT_OK;
}

extern "C" pct_status pct_get_counters(pct_ctx* ctx, int64_t counters[4])
{
    if (!ctx || !counters) return PCT_ERR_ARG;
    cudaSetDevice(ctx->device);
    unsigned long long h[pct::kNumCounters];
    PCT_CUDA_TRY(cudaMemcpyAsync(h, ctx->d_counters, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    PCT_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    for (int i = 0; i < 4; i++) counters[i] = (int64_t)h[i];
    return PCT_OK;
}

extern "C" pct_status pct_reset_counters(pct_ctx* ctx)
{
    if (!ctx) return PCT_ERR_ARG;
    cudaSetDevice(ctx->device);
    PCT_CUDA_TRY(cudaMemsetAsync(ctx->d_counters, 0, pct::kNumCounters * sizeof(unsigned long long), ctx->stream));
    return PCT_OK;
}

extern "C" int64_t pct_kernel_launches(const pct_ctx* ctx) { return ctx ? ctx->launches : -1; }

namespace pct {

bool context_view(pct_ctx* ctx, ContextView* v)
{
    if (!ctx || !v) return false;
    v->geo = ctx->geo;
    v->tables = ctx->tables;
    v->steps = ctx->d_steps;
    v->kmax = ctx->kmax;
    v->device = ctx->device;
    v->stream = ctx->stream;
    v->counters = ctx->d_counters;
    return true;
}

void context_count_launches(pct_ctx* ctx, long long n)
{
    if (ctx) ctx->launches += n;
}

void context_set_error(pct_ctx* ctx, const char* msg)
{
    if (ctx) ctx->last_error = msg ? msg : "";
}

}  // namespace pct
