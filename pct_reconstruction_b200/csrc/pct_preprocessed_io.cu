// pct_preprocessed_io.cu -- export and import of preprocessed data: reconstruction histories,
// WEPL, MLP voxel lists, voxels per path, chord lengths, hull and initial iterate.
//
// Follows accumulate_and_export_preprocessed_data (O.cu:6615) with export_histories (O.cu:6573),
// export_WEPL (O.cu:6562), export_voxels_per_path (O.cu:6596), export_avg_chord_lengths
// (O.cu:6605), export_hull (O.cu:6540), export_x_0 (O.cu:6551) and the matching import_*
// functions (O.cu:6660-6780).  Each file is a uint32 history count followed by the arrays, as
// there, except:
//   * histories.bin holds the engine's reconstruction histories: the ten geometry arrays
//     (x/y/z_entry, x/y/z_exit, xy/xz_entry_angle, xy/xz_exit_angle, float) and first_MLP_voxel
//     (uint32) -- the reference's voxel_x/y/z, bin and gantry-angle arrays feed nothing here;
//   * avg_chord_lengths.bin holds double chords (EffectiveChordLength_GPU B.cu:8873 is double and
//     the DROP update uses it unrounded), not the host path's float;
//   * MLP_paths.bin starts with a binary uint32 count (the reference writes it with fprintf and
//     reads it back with fread, which disagree).
// The MLP voxel lists come from the path kernel into path storage and are compacted on the device
// before the copy to the host; an import scatters them back into path storage so that
// precomputed-path DROP (pct_set_path_reuse) starts without the path kernel.
#include <algorithm>
#include <cstdio>
#include <string>
#include <vector>

#include "pct_context.h"

namespace {

// Copies each history's voxel list between path storage (at offsets[h] - base) and a packed
// array (at packed[h - h0] - packed0).  One warp per history.
template <bool kToPacked>
__global__ void move_paths_kernel(uint32_t* __restrict__ storage, const long long* __restrict__ offsets,
                                  long long base, const int* __restrict__ path_n,
                                  const long long* __restrict__ packed_off, uint32_t* __restrict__ packed,
                                  long long h0, long long count)
{
    const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= count) return;
    const long long h = h0 + w;
    const int n = path_n[h];
    uint32_t* s = storage + (offsets[h] - base);
    uint32_t* p = packed + packed_off[w];
    for (int j = lane; j < n; j += 32) {
        if (kToPacked)
            p[j] = s[j];
        else
            s[j] = p[j];
    }
}

struct File {
    FILE* f = nullptr;
    ~File()
    {
        if (f) fclose(f);
    }
};

pct_status io_fail(pct_ctx* ctx, pct_status s, const std::string& what, cudaError_t e = cudaSuccess)
{
    ctx->last_error = what;
    if (e != cudaSuccess) ctx->last_error += " -> " + pct::cuda_error_string(e);
    return s;
}

std::string join(const char* dir, const char* name) { return std::string(dir) + "/" + name; }

bool write_all(FILE* f, const void* p, size_t elem, size_t n) { return n == 0 || fwrite(p, elem, n, f) == n; }
bool read_all(FILE* f, void* p, size_t elem, size_t n) { return n == 0 || fread(p, elem, n, f) == n; }

// Writes "uint32 count, then arrays" files.
template <class T>
bool write_counted(const std::string& path, uint32_t count, const std::vector<const T*>& arrays, size_t n)
{
    File fl;
    fl.f = fopen(path.c_str(), "wb");
    if (!fl.f) return false;
    bool ok = write_all(fl.f, &count, sizeof(count), 1);
    for (const T* a : arrays) ok = ok && write_all(fl.f, a, sizeof(T), n);
    return ok && fflush(fl.f) == 0;
}

long long file_size(FILE* f)
{
    if (fseek(f, 0, SEEK_END) != 0) return -1;
    const long long sz = ftell(f);
    return fseek(f, 0, SEEK_SET) == 0 ? sz : -1;
}

}  // namespace

extern "C" pct_status pct_export_preprocessed(pct_ctx* ctx, const char* directory)
{
    if (!ctx || !directory) return PCT_ERR_ARG;
    const long long n = ctx->n_hist;
    if (n <= 0) return io_fail(ctx, PCT_ERR_STATE, "no reconstruction histories loaded");
    cudaSetDevice(ctx->device);
    pct_status st = pct::layout_prepare(ctx);
    if (st != PCT_OK) return st;
    if (!ctx->two_phase) return io_fail(ctx, PCT_ERR_STATE, "export needs path storage (pct_set_path_storage_limit >= 0)");
    cudaStream_t s = ctx->stream;
    // histories and WEPL
    const pct::HistorySoA& h = ctx->hist;
    const float* dev_geom[10] = {h.x_entry, h.y_entry, h.z_entry, h.x_exit, h.y_exit, h.z_exit,
                                 h.xy_entry_angle, h.xz_entry_angle, h.xy_exit_angle, h.xz_exit_angle};
    std::vector<float> geom((size_t)n * 10), wepl((size_t)n);
    std::vector<uint32_t> first((size_t)n);
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < 10 && e == cudaSuccess; k++)
        e = cudaMemcpyAsync(geom.data() + (size_t)k * n, dev_geom[k], sizeof(float) * n, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(wepl.data(), h.WEPL, sizeof(float) * n, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(first.data(), h.first_MLP_voxel, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, s);
    // x_0 and hull
    const long long nv = ctx->cfg.NUM_VOXELS;
    std::vector<float> x0((size_t)nv);
    if (e == cudaSuccess) e = cudaMemcpyAsync(x0.data(), ctx->d_x, sizeof(float) * nv, cudaMemcpyDeviceToHost, s);
    const uint8_t* dhull = pct::preproc_hull(ctx);
    std::vector<uint8_t> hull(dhull ? (size_t)nv : 0);
    if (e == cudaSuccess && dhull) e = cudaMemcpyAsync(hull.data(), dhull, nv, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return io_fail(ctx, PCT_ERR_CUDA, "export copies", e);
    {
        std::vector<const float*> arrays;
        for (int k = 0; k < 10; k++) arrays.push_back(geom.data() + (size_t)k * n);
        File fl;
        const std::string p = join(directory, "histories.bin");
        fl.f = fopen(p.c_str(), "wb");
        const uint32_t cnt = (uint32_t)n;
        bool ok = fl.f && write_all(fl.f, &cnt, 4, 1);
        for (const float* a : arrays) ok = ok && write_all(fl.f, a, 4, (size_t)n);
        ok = ok && write_all(fl.f, first.data(), 4, (size_t)n) && fflush(fl.f) == 0;
        if (!ok) return io_fail(ctx, PCT_ERR_IO, "cannot write " + p);
    }
    if (!write_counted<float>(join(directory, "WEPL.bin"), (uint32_t)n, {wepl.data()}, (size_t)n))
        return io_fail(ctx, PCT_ERR_IO, "cannot write WEPL.bin");
    {
        File fl;
        const std::string p = join(directory, "x_0.bin");
        fl.f = fopen(p.c_str(), "wb");
        if (!fl.f || !write_all(fl.f, x0.data(), 4, (size_t)nv) || fflush(fl.f) != 0)
            return io_fail(ctx, PCT_ERR_IO, "cannot write " + p);
    }
    if (dhull) {
        File fl;
        const std::string p = join(directory, "hull.bin");
        fl.f = fopen(p.c_str(), "wb");
        if (!fl.f || !write_all(fl.f, hull.data(), 1, (size_t)nv) || fflush(fl.f) != 0)
            return io_fail(ctx, PCT_ERR_IO, "cannot write " + p);
    }
    // MLP paths, superblock by superblock: path kernel (unless the paths are resident), packed
    // offsets by prefix sum of the path lengths, compaction, copy, append.
    File fpaths;
    const std::string ppath = join(directory, "MLP_paths.bin");
    fpaths.f = fopen(ppath.c_str(), "wb");
    const uint32_t cnt = (uint32_t)n;
    if (!fpaths.f || !write_all(fpaths.f, &cnt, 4, 1)) return io_fail(ctx, PCT_ERR_IO, "cannot write " + ppath);
    const bool resident = ctx->paths_valid && ctx->sbs.size() == 1;
    long long* d_packed_off = nullptr;
    long long* d_scan = nullptr;
    uint32_t* d_packed = nullptr;
    std::vector<uint32_t> packed;
    long long launches = 0;
    auto cleanup = [&]() {
        cudaStreamSynchronize(s);
        cudaFree(d_packed_off);
        cudaFree(d_scan);
        cudaFree(d_packed);
    };
    long long max_sb = 0;
    for (const auto& sb : ctx->sbs) max_sb = std::max(max_sb, sb.h_end - sb.h_begin);
    e = cudaMalloc(&d_packed_off, sizeof(long long) * (size_t)(max_sb + 1));
    if (e == cudaSuccess) e = cudaMalloc(&d_scan, sizeof(long long) * (size_t)pct::scan_tile_scratch_elems(max_sb));
    if (e != cudaSuccess) {
        cleanup();
        return io_fail(ctx, PCT_ERR_NOMEM, "export scratch", e);
    }
    long long d_packed_cap = 0;
    for (const auto& sb : ctx->sbs) {
        const long long m = sb.h_end - sb.h_begin;
        if (!resident) {
            // (histories outside the covered part of their DROP block get path length 0)
            e = pct::launch_mlp_phase1_exact(ctx->geo, ctx->tables, ctx->d_steps, ctx->kmax,
                                             pct::sorted_path_inputs(ctx, sb.h_begin), ctx->d_perm + sb.h_begin, m,
                                             ctx->d_offsets_sorted + sb.h_begin, sb.off_begin,
                                             ctx->d_bounds_sorted + sb.h_begin, ctx->d_paths, ctx->d_path_n,
                                             ctx->d_chord, ctx->d_counters, s);
            launches += 1;
        }
        if (e == cudaSuccess)
            e = pct::exclusive_scan_i32_to_i64(ctx->d_path_n + sb.h_begin, m, d_packed_off, d_scan, s);
        long long total = 0;
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(&total, d_packed_off + m, sizeof(long long), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e == cudaSuccess && total > d_packed_cap) {
            cudaFree(d_packed);
            d_packed = nullptr;
            e = cudaMalloc(&d_packed, sizeof(uint32_t) * (size_t)(total > 0 ? total : 1));
            d_packed_cap = e == cudaSuccess ? total : 0;
        }
        if (e == cudaSuccess && m > 0) {
            move_paths_kernel<true><<<(unsigned)((m * 32 + 255) / 256), 256, 0, s>>>(
                ctx->d_paths, ctx->d_offsets, sb.off_begin, ctx->d_path_n, d_packed_off, d_packed, sb.h_begin, m);
            e = cudaGetLastError();
            launches += 1;
        }
        packed.resize((size_t)total);
        if (e == cudaSuccess && total > 0)
            e = cudaMemcpyAsync(packed.data(), d_packed, sizeof(uint32_t) * total, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) {
            cleanup();
            return io_fail(ctx, PCT_ERR_CUDA, "export paths", e);
        }
        ctx->launches += 3;  // the scan
        if (!write_all(fpaths.f, packed.data(), 4, (size_t)total)) {
            cleanup();
            return io_fail(ctx, PCT_ERR_IO, "cannot write " + ppath);
        }
    }
    if (ctx->sbs.size() == 1) ctx->paths_valid = true;
    std::vector<int> path_n((size_t)n);
    std::vector<double> chord((size_t)n);
    e = cudaMemcpyAsync(path_n.data(), ctx->d_path_n, sizeof(int) * n, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(chord.data(), ctx->d_chord, sizeof(double) * n, cudaMemcpyDeviceToHost, s);
    cleanup();
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return io_fail(ctx, PCT_ERR_CUDA, "export path lengths", e);
    ctx->launches += launches;
    if (fflush(fpaths.f) != 0) return io_fail(ctx, PCT_ERR_IO, "cannot write " + ppath);
    std::vector<uint32_t> counts(path_n.begin(), path_n.end());
    if (!write_counted<uint32_t>(join(directory, "voxels_per_path.bin"), (uint32_t)n, {counts.data()}, (size_t)n))
        return io_fail(ctx, PCT_ERR_IO, "cannot write voxels_per_path.bin");
    if (!write_counted<double>(join(directory, "avg_chord_lengths.bin"), (uint32_t)n, {chord.data()}, (size_t)n))
        return io_fail(ctx, PCT_ERR_IO, "cannot write avg_chord_lengths.bin");
    return PCT_OK;
}

extern "C" pct_status pct_import_preprocessed(pct_ctx* ctx, const char* directory)
{
    if (!ctx || !directory) return PCT_ERR_ARG;
    cudaSetDevice(ctx->device);
    // histories + WEPL (import_histories O.cu:6694, import_WEPL O.cu:6681)
    uint32_t n32 = 0;
    std::vector<float> geom, wepl;
    std::vector<uint32_t> first;
    {
        File fl;
        const std::string p = join(directory, "histories.bin");
        fl.f = fopen(p.c_str(), "rb");
        if (!fl.f || !read_all(fl.f, &n32, 4, 1)) return io_fail(ctx, PCT_ERR_IO, "cannot read " + p);
        const long long sz = file_size(fl.f);
        if (sz != 4 + 44LL * n32) return io_fail(ctx, PCT_ERR_IO, p + ": size does not match its count");
        fseek(fl.f, 4, SEEK_SET);
        geom.resize((size_t)n32 * 10);
        first.resize(n32);
        if (!read_all(fl.f, geom.data(), 4, geom.size()) || !read_all(fl.f, first.data(), 4, first.size()))
            return io_fail(ctx, PCT_ERR_IO, "cannot read " + p);
    }
    {
        File fl;
        const std::string p = join(directory, "WEPL.bin");
        fl.f = fopen(p.c_str(), "rb");
        uint32_t c = 0;
        if (!fl.f || !read_all(fl.f, &c, 4, 1) || c != n32) return io_fail(ctx, PCT_ERR_IO, p + ": missing or count mismatch");
        wepl.resize(n32);
        if (!read_all(fl.f, wepl.data(), 4, n32)) return io_fail(ctx, PCT_ERR_IO, "cannot read " + p);
    }
    const long long n = n32;
    const float* g[10];
    for (int k = 0; k < 10; k++) g[k] = geom.data() + (size_t)k * n;
    const pct_histories hs{g[0], g[1], g[2], g[3], g[4], g[5], g[6], g[7], g[8], g[9], wepl.data(), first.data()};
    pct_status st = pct_set_reconstruction_histories(ctx, &hs, n, PCT_HOST);
    if (st != PCT_OK) return st;
    // x_0 and hull (import_x_0 O.cu:6671, import_hull O.cu:6658), when present
    const long long nv = ctx->cfg.NUM_VOXELS;
    {
        File fl;
        fl.f = fopen(join(directory, "x_0.bin").c_str(), "rb");
        if (fl.f) {
            std::vector<float> x0((size_t)nv);
            if (file_size(fl.f) != 4 * nv || !read_all(fl.f, x0.data(), 4, (size_t)nv))
                return io_fail(ctx, PCT_ERR_IO, "x_0.bin: size does not match NUM_VOXELS");
            st = pct_set_image(ctx, x0.data(), PCT_HOST);
            if (st != PCT_OK) return st;
        }
    }
    {
        File fl;
        fl.f = fopen(join(directory, "hull.bin").c_str(), "rb");
        if (fl.f) {
            std::vector<uint8_t> hull((size_t)nv);
            if (file_size(fl.f) != nv || !read_all(fl.f, hull.data(), 1, (size_t)nv))
                return io_fail(ctx, PCT_ERR_IO, "hull.bin: size does not match NUM_VOXELS");
            st = pct_set_array(ctx, "hull", hull.data(), nv, PCT_HOST);
            if (st != PCT_OK) return st;
        }
    }
    // paths, lengths, chords (import_MLP O.cu:6750, import_voxels_per_path O.cu:6726,
    // import_avg_chord_lengths O.cu:6738), when present
    File fp, fc, fa;
    fp.f = fopen(join(directory, "MLP_paths.bin").c_str(), "rb");
    fc.f = fopen(join(directory, "voxels_per_path.bin").c_str(), "rb");
    fa.f = fopen(join(directory, "avg_chord_lengths.bin").c_str(), "rb");
    if (!fp.f || !fc.f || !fa.f) return PCT_OK;  // histories only: paths are computed by the first iteration
    uint32_t c1 = 0, c2 = 0, c3 = 0;
    std::vector<uint32_t> counts(n32);
    std::vector<double> chord(n32);
    if (!read_all(fp.f, &c1, 4, 1) || !read_all(fc.f, &c2, 4, 1) || !read_all(fa.f, &c3, 4, 1) || c1 != n32 ||
        c2 != n32 || c3 != n32)
        return io_fail(ctx, PCT_ERR_IO, "path files: count mismatch with histories.bin");
    if (!read_all(fc.f, counts.data(), 4, n32) || !read_all(fa.f, chord.data(), 8, n32))
        return io_fail(ctx, PCT_ERR_IO, "path files: truncated");
    long long total = 0;
    for (uint32_t c : counts) total += c;
    if (file_size(fp.f) != 4 + 4 * total) return io_fail(ctx, PCT_ERR_IO, "MLP_paths.bin: size does not match voxels_per_path.bin");
    fseek(fp.f, 4, SEEK_SET);
    std::vector<uint32_t> packed((size_t)total);
    if (!read_all(fp.f, packed.data(), 4, (size_t)total)) return io_fail(ctx, PCT_ERR_IO, "MLP_paths.bin: truncated");
    for (uint32_t v : packed)
        if (v >= (uint32_t)ctx->geo.padded_voxels) return io_fail(ctx, PCT_ERR_IO, "MLP_paths.bin: voxel index out of range");
    st = pct::layout_prepare(ctx);
    if (st != PCT_OK) return st;
    if (!ctx->two_phase || ctx->sbs.size() != 1) return PCT_OK;  // not resident: recomputed per iteration
    cudaStream_t s = ctx->stream;
    // each imported path must fit its storage slot (the path-length bound)
    std::vector<int> bounds((size_t)n);
    cudaError_t e = cudaMemcpyAsync(bounds.data(), ctx->d_bounds, sizeof(int) * n, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return io_fail(ctx, PCT_ERR_CUDA, "import bounds", e);
    std::vector<int> path_n((size_t)n);
    std::vector<long long> packed_off((size_t)n + 1, 0);
    for (long long i = 0; i < n; i++) {
        if ((long long)counts[i] > bounds[i] && bounds[i] > 0)
            return io_fail(ctx, PCT_ERR_IO, "MLP_paths.bin: a path is longer than its MLP step bound");
        path_n[i] = bounds[i] > 0 ? (int)counts[i] : 0;
        packed_off[i + 1] = packed_off[i] + counts[i];
    }
    long long* d_off = nullptr;
    uint32_t* d_packed = nullptr;
    e = cudaMalloc(&d_off, sizeof(long long) * (size_t)(n + 1));
    if (e == cudaSuccess) e = cudaMalloc(&d_packed, sizeof(uint32_t) * (size_t)(total > 0 ? total : 1));
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_off, packed_off.data(), sizeof(long long) * (n + 1), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && total > 0)
        e = cudaMemcpyAsync(d_packed, packed.data(), sizeof(uint32_t) * total, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ctx->d_path_n, path_n.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ctx->d_chord, chord.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && n > 0) {
        move_paths_kernel<false><<<(unsigned)((n * 32 + 255) / 256), 256, 0, s>>>(
            ctx->d_paths, ctx->d_offsets, ctx->sbs[0].off_begin, ctx->d_path_n, d_off, d_packed, 0, n);
        e = cudaGetLastError();
        ctx->launches += 1;
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(d_off);
    cudaFree(d_packed);
    if (e != cudaSuccess) return io_fail(ctx, PCT_ERR_CUDA, "import paths", e);
    ctx->paths_valid = true;
    return PCT_OK;
}
