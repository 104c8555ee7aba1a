// pct_reader.cu -- projection data files (PCTD / PCTN, versions 0 and 1) to device tracker arrays.
//
// The header parse follows count_histories_v0 (B.cu:3578-3677) and the data reads follow
// read_data_chunk_v0 (B.cu:4361-4467), which is the reader the reference runs
// (DATA_FORMAT = VERSION_0, B.h:164; it reads version 0 and version 1 files alike).
//
// Design: a scan is read straight into the context's device tracker arrays.  Each file's arrays
// are read into one of two pinned staging buffers while the host-to-device copies of the other
// buffer run on the context's stream; the mm->cm conversion (convert_mm_2_cm B.cu:4070), the
// t/u/v shifts (apply_tuv_shifts B.cu:4100) and the per-history angle are applied by device
// kernels over all histories.  The conversion is the reference's `float *= double` and
// `float += double`: (float)((double)v * 0.1) and (float)((double)v + shift), both correctly
// rounded on the host and the device, so the converted arrays are bit-identical.  This
// translation unit is compiled with -fmad=false.
#include <sys/stat.h>

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "pct_context.h"

namespace {

constexpr double kMmToCm = 0.1;  // MM_TO_CM (B.h:843)
constexpr int kDataArrays = 13;  // t0..t3, v0..v3, u0..u3, WEPL

struct FileCloser {
    FILE* f = nullptr;
    ~FileCloser()
    {
        if (f) fclose(f);
    }
};

template <class T>
bool read_value(FILE* f, T* v)
{
    return fread(v, sizeof(T), 1, f) == 1;
}

// Parses the header of an open file of `file_size` bytes.  On failure *why says what was wrong.
bool parse_header(FILE* f, long long file_size, pct_projection_header* h, std::string* why)
{
    memset(h, 0, sizeof(*h));
    char magic[4];
    if (fread(magic, 1, 4, f) != 4) return *why = "file shorter than its header", false;
    if (memcmp(magic, "PCTN", 4) == 0)
        h->continuous = 1;
    else if (memcmp(magic, "PCTD", 4) != 0)
        return *why = "unknown file type (magic number is neither PCTD nor PCTN)", false;
    int32_t version = 0, n = 0, dates[2] = {0, 0};
    float angle = 0.f, energy = 0.f;
    if (!read_value(f, &version) || !read_value(f, &n) || !read_value(f, &angle) || !read_value(f, &energy) ||
        !read_value(f, &dates[0]) || !read_value(f, &dates[1]))
        return *why = "file shorter than its header", false;
    if (version != 0 && version != 1) return *why = "data format is not version 0 or 1", false;
    if (n < 0) return *why = "negative number of histories", false;
    h->version = version;
    h->num_histories = n;
    h->projection_angle = angle;
    h->beam_energy = energy;
    h->generation_date = dates[0];
    h->preprocess_date = dates[1];
    long long offset = 4 + 7 * (long long)sizeof(int32_t) + 2 * (long long)sizeof(float);  // fixed part
    char* strings[3] = {h->phantom_name, h->data_source, h->prepared_by};
    for (char* s : strings) {
        int32_t len = 0;
        if (!read_value(f, &len)) return *why = "file shorter than its header", false;
        if (len < 0 || len > file_size) return *why = "bad string length in the header", false;
        const long long keep = len < 255 ? len : 255;
        if (keep > 0 && fread(s, 1, (size_t)keep, f) != (size_t)keep)
            return *why = "file shorter than its header", false;
        s[keep] = '\0';
        if (len > keep && fseek(f, (long)(len - keep), SEEK_CUR) != 0)
            return *why = "file shorter than its header", false;
        offset += len;
    }
    h->data_offset = offset;  // SKIP_2_DATA_SIZE (B.cu:3643)
    const long long array_bytes = (long long)n * (long long)sizeof(float);
    if (file_size < offset + kDataArrays * array_bytes)
        return *why = "file shorter than its 13 data arrays (truncated)", false;
    h->has_angles = file_size >= offset + (kDataArrays + 1) * array_bytes ? 1 : 0;
    return true;
}

pct_status open_and_parse(const char* path, FileCloser* fc, pct_projection_header* h, std::string* why)
{
    if (!path || !h) return *why = "NULL argument", PCT_ERR_ARG;
    struct stat st;
    if (stat(path, &st) != 0 || !S_ISREG(st.st_mode)) return *why = std::string("cannot open ") + path, PCT_ERR_IO;
    fc->f = fopen(path, "rb");
    if (!fc->f) return *why = std::string("cannot open ") + path, PCT_ERR_IO;
    if (!parse_header(fc->f, (long long)st.st_size, h, why)) {
        *why = std::string(path) + ": " + *why;
        return PCT_ERR_IO;
    }
    return PCT_OK;
}

// Destination of file array j (t0..t3, v0..v3, u0..u3, WEPL) in the tracker-slot order
// (t_in_1..t_out_2, u_in_1..u_out_2, v_in_1..v_out_2, WEPL).
constexpr int kFileToSlot[kDataArrays] = {0, 1, 2, 3, 8, 9, 10, 11, 4, 5, 6, 7, 12};

__global__ void fill_angle_kernel(float* __restrict__ dst, long long n, float value)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] = value;
}

struct ConvertArgs {
    float* a[kDataArrays];  // tracker-slot order, WEPL last
};

// convert_mm_2_cm (B.cu:4070) then apply_tuv_shifts (B.cu:4100) over all histories.
__global__ void convert_tracker_kernel(ConvertArgs args, long long n, int to_cm, int shift, double t_shift,
                                       double u_shift, double v_shift)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
#pragma unroll
        for (int k = 0; k < kDataArrays; k++) {
            float v = args.a[k][i];
            if (to_cm) v = (float)((double)v * kMmToCm);
            if (shift && k < 12) v = (float)((double)v + (k < 4 ? t_shift : k < 8 ? u_shift : v_shift));
            args.a[k][i] = v;
        }
    }
}

unsigned grid_stride_blocks(long long n, int threads)
{
    long long b = (n + threads - 1) / threads;
    const long long cap = 148LL * 16;  // 16 resident 256-thread CTAs on each of the 148 SMs
    return (unsigned)(b < 1 ? 1 : b > cap ? cap : b);
}

pct_status fail(pct_ctx* ctx, pct_status st, const std::string& what, cudaError_t e = cudaSuccess)
{
    if (ctx) {
        ctx->last_error = what;
        if (e != cudaSuccess) ctx->last_error += " -> " + pct::cuda_error_string(e);
    }
    return st;
}

}  // namespace

extern "C" pct_status pct_read_projection_header(const char* path, pct_projection_header* header)
{
    FileCloser fc;
    std::string why;
    return open_and_parse(path, &fc, header, &why);
}

extern "C" pct_status pct_read_projection_file(const char* path, int64_t capacity, const pct_projection_arrays* out,
                                               pct_projection_header* header)
{
    if (!out || !header || capacity < 0) return PCT_ERR_ARG;
    FileCloser fc;
    std::string why;
    pct_status st = open_and_parse(path, &fc, header, &why);
    if (st != PCT_OK) return st;
    const long long n = header->num_histories;
    if (n > capacity) return PCT_ERR_ARG;
    float* dst[kDataArrays] = {out->t_in_1,  out->t_in_2,  out->t_out_1, out->t_out_2, out->v_in_1,
                               out->v_in_2,  out->v_out_1, out->v_out_2, out->u_in_1,  out->u_in_2,
                               out->u_out_1, out->u_out_2, out->WEPL};
    for (float* d : dst)
        if (!d && n > 0) return PCT_ERR_ARG;
    if (out->projection_angle && !header->has_angles) return PCT_ERR_IO;
    if (fseek(fc.f, (long)header->data_offset, SEEK_SET) != 0) return PCT_ERR_IO;
    for (float* d : dst)
        if (n > 0 && fread(d, sizeof(float), (size_t)n, fc.f) != (size_t)n) return PCT_ERR_IO;
    if (out->projection_angle && n > 0 && fread(out->projection_angle, sizeof(float), (size_t)n, fc.f) != (size_t)n)
        return PCT_ERR_IO;
    return PCT_OK;
}

extern "C" pct_status pct_write_projection_file(const char* path, const pct_projection_header* header,
                                                const pct_projection_arrays* in, int64_t n)
{
    if (!path || !header || !in || n < 0 || n > 0x7fffffffLL) return PCT_ERR_ARG;
    if (header->version != 0 && header->version != 1) return PCT_ERR_ARG;
    const float* src[kDataArrays] = {in->t_in_1,  in->t_in_2,  in->t_out_1, in->t_out_2, in->v_in_1,
                                     in->v_in_2,  in->v_out_1, in->v_out_2, in->u_in_1,  in->u_in_2,
                                     in->u_out_1, in->u_out_2, in->WEPL};
    for (const float* s : src)
        if (!s && n > 0) return PCT_ERR_ARG;
    FileCloser fc;
    fc.f = fopen(path, "wb");
    if (!fc.f) return PCT_ERR_IO;
    const int32_t fixed[3] = {header->version, (int32_t)n, 0};
    bool ok = fwrite(header->continuous ? "PCTN" : "PCTD", 1, 4, fc.f) == 4;
    ok = ok && fwrite(fixed, sizeof(int32_t), 2, fc.f) == 2;
    ok = ok && fwrite(&header->projection_angle, sizeof(float), 1, fc.f) == 1;
    ok = ok && fwrite(&header->beam_energy, sizeof(float), 1, fc.f) == 1;
    ok = ok && fwrite(&header->generation_date, sizeof(int32_t), 1, fc.f) == 1;
    ok = ok && fwrite(&header->preprocess_date, sizeof(int32_t), 1, fc.f) == 1;
    const char* strings[3] = {header->phantom_name, header->data_source, header->prepared_by};
    for (const char* s : strings) {
        const int32_t len = (int32_t)strnlen(s, 256);
        ok = ok && fwrite(&len, sizeof(int32_t), 1, fc.f) == 1;
        ok = ok && (len == 0 || fwrite(s, 1, (size_t)len, fc.f) == (size_t)len);
    }
    for (const float* s : src) ok = ok && (n == 0 || fwrite(s, sizeof(float), (size_t)n, fc.f) == (size_t)n);
    if (in->projection_angle)
        ok = ok && (n == 0 || fwrite(in->projection_angle, sizeof(float), (size_t)n, fc.f) == (size_t)n);
    ok = fflush(fc.f) == 0 && ok;
    return ok ? PCT_OK : PCT_ERR_IO;
}

extern "C" pct_status pct_load_projection_data(pct_ctx* ctx, const char* directory, int64_t* n_out)
{
    if (!ctx || !directory) return PCT_ERR_ARG;
    const pct_config& c = ctx->cfg;
    const int interval = (int)c.GANTRY_ANGLE_INTERVAL;
    if (interval <= 0) return fail(ctx, PCT_ERR_ARG, "GANTRY_ANGLE_INTERVAL below one degree");
    // count_histories_v0: headers of every file, in gantry-angle order
    struct FileInfo {
        std::string path;
        pct_projection_header h;
        long long first;
    };
    std::vector<FileInfo> files;
    long long total = 0, max_n = 0;
    bool continuous = false;
    for (int angle = 0; angle < 360; angle += interval) {
        char name[64];
        snprintf(name, sizeof(name), "/projection_%03d.bin", angle);
        FileInfo fi;
        fi.path = std::string(directory) + name;
        std::string why;
        FileCloser fc;
        pct_status st = open_and_parse(fi.path.c_str(), &fc, &fi.h, &why);
        if (st != PCT_OK) return fail(ctx, st, why);
        fi.first = total;
        total += fi.h.num_histories;
        if (fi.h.num_histories > max_n) max_n = fi.h.num_histories;
        if (fi.h.continuous) continuous = true;  // CONTINUOUS_DATA is set by any PCTN file
        files.push_back(fi);
    }
    if (total > 0x7fffffffLL) return fail(ctx, PCT_ERR_ARG, "more than 2^31-1 histories in the scan");
    const bool cont_angles = continuous && c.USE_CONT_ANGLES;
    if (cont_angles)
        for (const FileInfo& fi : files)
            if (!fi.h.has_angles) return fail(ctx, PCT_ERR_IO, fi.path + ": no per-history projection angles");

    float* dst[pct::kTrackerSlots];
    pct_status st = pct::preproc_reserve_tracker(ctx, total, dst);
    if (st != PCT_OK) return st;
    cudaStream_t s = ctx->stream;

    // read_data_chunk_v0: two pinned staging buffers, file k+1 is read while file k is copied
    const int arrays = kDataArrays + (cont_angles ? 1 : 0);
    const size_t slot_floats = (size_t)(max_n > 0 ? max_n : 1) * arrays;
    float* stage[2] = {nullptr, nullptr};
    cudaEvent_t done[2] = {nullptr, nullptr};
    bool used[2] = {false, false};
    auto cleanup = [&]() {
        cudaStreamSynchronize(s);
        for (int k = 0; k < 2; k++) {
            if (stage[k]) cudaFreeHost(stage[k]);
            if (done[k]) cudaEventDestroy(done[k]);
        }
    };
    for (int k = 0; k < 2; k++) {
        cudaError_t e = cudaHostAlloc((void**)&stage[k], slot_floats * sizeof(float), cudaHostAllocDefault);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&done[k], cudaEventDisableTiming);
        if (e != cudaSuccess) {
            cleanup();
            return fail(ctx, PCT_ERR_NOMEM, "pinned staging for projection files", e);
        }
    }
    long long launches = 0;
    for (size_t fidx = 0; fidx < files.size(); fidx++) {
        const FileInfo& fi = files[fidx];
        const long long n = fi.h.num_histories;
        if (n == 0) continue;
        const int slot = (int)(fidx & 1);
        if (used[slot]) {
            cudaError_t e = cudaEventSynchronize(done[slot]);
            if (e != cudaSuccess) {
                cleanup();
                return fail(ctx, PCT_ERR_CUDA, "staging event", e);
            }
        }
        FileCloser fc;
        fc.f = fopen(fi.path.c_str(), "rb");
        bool ok = fc.f && fseek(fc.f, (long)fi.h.data_offset, SEEK_SET) == 0;
        for (int j = 0; j < arrays && ok; j++)
            ok = fread(stage[slot] + (size_t)j * n, sizeof(float), (size_t)n, fc.f) == (size_t)n;
        if (!ok) {
            cleanup();
            return fail(ctx, PCT_ERR_IO, fi.path + ": read failed");
        }
        cudaError_t e = cudaSuccess;
        for (int j = 0; j < kDataArrays && e == cudaSuccess; j++)
            e = cudaMemcpyAsync(dst[kFileToSlot[j]] + fi.first, stage[slot] + (size_t)j * n, sizeof(float) * n,
                                cudaMemcpyHostToDevice, s);
        float* angle_dst = dst[pct::kTrackerSlots - 1] + fi.first;
        if (e == cudaSuccess && cont_angles) {
            e = cudaMemcpyAsync(angle_dst, stage[slot] + (size_t)kDataArrays * n, sizeof(float) * n,
                                cudaMemcpyHostToDevice, s);
        } else if (e == cudaSuccess) {
            // gantry_angle_h = int(projection_angles[file]) (B.cu:4429)
            fill_angle_kernel<<<grid_stride_blocks(n, 256), 256, 0, s>>>(angle_dst, n,
                                                                         (float)(int)fi.h.projection_angle);
            e = cudaGetLastError();
            launches++;
        }
        if (e == cudaSuccess) e = cudaEventRecord(done[slot], s);
        if (e != cudaSuccess) {
            cleanup();
            return fail(ctx, PCT_ERR_CUDA, "projection data copy", e);
        }
        used[slot] = true;
    }
    const bool shift = c.T_SHIFT != 0.0 || c.U_SHIFT != 0.0 || c.V_SHIFT != 0.0;
    if (total > 0 && (c.DATA_IN_MM || shift)) {
        ConvertArgs args;
        for (int k = 0; k < kDataArrays; k++) args.a[k] = dst[k];
        convert_tracker_kernel<<<grid_stride_blocks(total, 256), 256, 0, s>>>(
            args, total, c.DATA_IN_MM ? 1 : 0, shift ? 1 : 0, c.T_SHIFT, c.U_SHIFT, c.V_SHIFT);
        launches++;
    }
    cudaError_t e = cudaGetLastError();
    cleanup();
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(ctx, PCT_ERR_CUDA, "tracker conversion", e);
    ctx->launches += launches;
    pct::preproc_tracker_loaded(ctx, total, cont_angles ? 0 : 1);
    if (n_out) *n_out = total;
    return PCT_OK;
}
