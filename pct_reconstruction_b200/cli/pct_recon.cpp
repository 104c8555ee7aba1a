// pct_recon.cpp -- the reconstruction program: a C++ caller of the C ABI in include/pct_api.h.
//
// It replaces the reference's main (B.cu:369-399), which selects the GPU, runs preprocessing()
// (B.cu:7394) and image_reconstruction() (B.cu:10650) over the compile-time configuration of B.h
// and the projection files named there.  Here the configuration is a settings.cfg file read at
// run time, the data directory and the output are arguments, and every failure is a status code
// with a message (the reference printed cudaGetLastError() and carried on, or called exit(1)):
//
//   pct_recon <settings.cfg> <projection-data directory> <output image> [--device N]
//             [--iterations K] [--set KEY=VALUE ...]
//
//   1. pct_config_default + pct_config_load + pct_config_set overrides + pct_config_finalize
//      (the B.h values, then the settings file's "KEY = value" lines, as Configurations.h reads
//      settings.cfg)
//   2. pct_create on the device (the reference's cudaSetDevice loop, B.cu:373-387)
//   3. pct_preprocessing_from_files: every gantry angle's projection file, mm -> cm, the
//      intersections, binning, statistics and cuts, FBP, hulls, x_0 and the reconstruction cuts
//   4. pct_drop_gpu: ITERATIONS DROP iterations (DROP_GPU, B.cu:9848), with TVS as configured
//   5. pct_get_image, written as NUM_VOXELS little-endian float32 values (column fastest, then
//      row, then slice: the reference's voxel order)
// It prints one summary line and exits 0 on success, 1 on a usage error, 2 on a library error.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "pct_api.h"

namespace {

int usage(const char* argv0)
{
    std::fprintf(stderr,
                 "usage: %s <settings.cfg> <projection-data directory> <output image> [--device N] "
                 "[--iterations K] [--set KEY=VALUE ...]\n",
                 argv0);
    return 1;
}

int fail(const char* what, pct_status st, const pct_ctx* ctx)
{
    std::fprintf(stderr, "pct_recon: %s failed: %s%s%s\n", what, pct_status_string(st), ctx ? ": " : "",
                 ctx ? pct_last_error(ctx) : "");
    return 2;
}

// A configuration call's failure, with the library's reason.
int config_fail(const char* what, pct_status st)
{
    std::fprintf(stderr, "pct_recon: %s failed: %s: %s\n", what, pct_status_string(st), pct_config_last_error());
    return 2;
}

}  // namespace

int main(int argc, char** argv)
{
    if (argc < 4) return usage(argv[0]);
    const char* settings = argv[1];
    const char* directory = argv[2];
    const char* output = argv[3];
    int device = 0;
    std::vector<std::pair<std::string, std::string>> overrides;
    for (int i = 4; i < argc; i++) {
        if (!std::strcmp(argv[i], "--device") && i + 1 < argc) {
            device = std::atoi(argv[++i]);
        } else if (!std::strcmp(argv[i], "--iterations") && i + 1 < argc) {
            overrides.emplace_back("ITERATIONS", argv[++i]);
        } else if (!std::strcmp(argv[i], "--set") && i + 1 < argc) {
            const std::string kv = argv[++i];
            const size_t eq = kv.find('=');
            if (eq == std::string::npos || eq == 0) return usage(argv[0]);
            overrides.emplace_back(kv.substr(0, eq), kv.substr(eq + 1));
        } else {
            return usage(argv[0]);
        }
    }

    pct_config cfg;
    pct_config_default(&cfg);
    pct_status st = pct_config_load(&cfg, settings);
    if (st != PCT_OK) return config_fail("pct_config_load", st);
    for (const auto& kv : overrides) {
        st = pct_config_set(&cfg, kv.first.c_str(), kv.second.c_str());
        if (st != PCT_OK) return config_fail(("pct_config_set " + kv.first).c_str(), st);
    }
    st = pct_config_finalize(&cfg);
    if (st != PCT_OK) return config_fail("pct_config_finalize", st);

    pct_ctx* ctx = nullptr;
    st = pct_create(&cfg, device, &ctx);
    if (st != PCT_OK) {
        std::fprintf(stderr, "pct_recon: pct_create failed: %s: %s\n", pct_status_string(st), pct_last_error(nullptr));
        return 2;
    }
    const auto t0 = std::chrono::steady_clock::now();
    st = pct_preprocessing_from_files(ctx, directory);
    if (st == PCT_OK) st = pct_synchronize(ctx);
    if (st != PCT_OK) {
        const int rc = fail("pct_preprocessing_from_files", st, ctx);
        pct_destroy(ctx);
        return rc;
    }
    const auto t1 = std::chrono::steady_clock::now();
    st = pct_drop_gpu(ctx);
    if (st == PCT_OK) st = pct_synchronize(ctx);
    if (st != PCT_OK) {
        const int rc = fail("pct_drop_gpu", st, ctx);
        pct_destroy(ctx);
        return rc;
    }
    const auto t2 = std::chrono::steady_clock::now();
    std::vector<float> x((size_t)cfg.NUM_VOXELS);
    st = pct_get_image(ctx, x.data(), PCT_HOST);
    if (st != PCT_OK) {
        const int rc = fail("pct_get_image", st, ctx);
        pct_destroy(ctx);
        return rc;
    }
    const long long histories = (long long)pct_reconstruction_histories(ctx);
    int64_t counters[4] = {0, 0, 0, 0};
    pct_get_counters(ctx, counters);
    pct_destroy(ctx);

    FILE* f = std::fopen(output, "wb");
    if (!f || std::fwrite(x.data(), sizeof(float), x.size(), f) != x.size()) {
        std::fprintf(stderr, "pct_recon: cannot write %s\n", output);
        if (f) std::fclose(f);
        return 2;
    }
    std::fclose(f);
    const double pre_s = std::chrono::duration<double>(t1 - t0).count();
    const double drop_s = std::chrono::duration<double>(t2 - t1).count();
    std::printf("pct_recon: %dx%dx%d voxels, %lld reconstruction histories, preprocessing %.3f s, %d DROP "
                "iterations %.3f s, out-of-grid path entries %lld, image %s\n",
                cfg.COLUMNS, cfg.ROWS, cfg.SLICES, histories, pre_s, cfg.ITERATIONS, drop_s,
                (long long)counters[0], output);
    return 0;
}
