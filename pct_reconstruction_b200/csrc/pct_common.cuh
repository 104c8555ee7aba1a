// pct_common.cuh -- device-side parameter block, status plumbing and small helpers shared by
// the engine's translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/pct_api.h"

namespace pct {

// MLP lookup-table geometry (B.h:786-800).  The ranges and steps are fixed in the reference.
constexpr double kCoeffTableRange = 40.0;
constexpr double kCoeffTableStep = 0.00005;
constexpr double kPolyTableRange = 40.0;
constexpr double kPolyTableStep = 0.00005;

// Counter slots (pct_get_counters).
enum Counter { kCntVoxelOOB = 0, kCntPathOverflow = 1, kCntTableRange = 2, kCntWaitExpired = 3, kNumCounters = 4 };

// Everything a kernel needs from the configuration, by value (fits in kernel-parameter space).
struct Geometry {
    int columns, rows, slices;
    int num_voxels;        // COLUMNS*ROWS*SLICES
    int padded_voxels;     // num_voxels + COLUMNS*ROWS: one spare slice absorbs z = SLICES
    double voxel_width, voxel_height, voxel_thickness;
    double inv_voxel_width, inv_voxel_height, inv_voxel_thickness;  // RN(1/size)
    double inv_voxel_max;           // the largest of the three
    double x_zero, y_zero, z_zero;  // X/Y/Z_ZERO_COORDINATE (B.h:918-921)
    float x_zero_f, y_zero_f, z_zero_f;                          // float copies (mixed precision)
    float inv_voxel_width_f, inv_voxel_height_f, inv_voxel_thickness_f;
    double mlp_u_step;
    double trig_min, trig_step;     // TRIG_TABLE_MIN / TRIG_TABLE_STEP
    int trig_elements, coeff_elements, poly_elements;
    unsigned sigma_index_step;      // static_cast<unsigned>(MLP_U_STEP/COEFF_TABLE_STEP + 0.5)
    unsigned poly_index_step;       // static_cast<unsigned>(MLP_U_STEP/POLY_TABLE_STEP + 0.5)
    int min_mlp_length;
    double lambda;                  // (double)(float)LAMBDA
    int projection_algorithm;       // PCT_DROP, PCT_ROBUSTA, PCT_ROBUSTB
    int mixed_precision;            // PRECISION MIXED or MIXED_COMPENSATED (path and block kernels)
    int compensated;                // PRECISION == PCT_PRECISION_MIXED_COMPENSATED (scatter and image update)
    double mixed_fp64_margin;       // mixed mode: FP64 2x2 inversions within this distance (cm) of entry or exit
    int exact_fast_points;          // EXACT_FAST_POINTS: guarded fast MLP points in exact mode
    int path_cta_threads;           // PATH_CTA_THREADS: 64, 128 or 256
    int deterministic;              // SCATTER_MODE == PCT_SCATTER_DETERMINISTIC
    int psi_sign;                   // PSI_SIGN
    double eta;                     // ETA
    double air_threshold;           // X_N_AIR_THRESHOLD with IDENTIFY_X_N_AIR, else -infinity
    const float* s_curve;           // S_CURVE_ON: s(k) for k < kSCurveEntries (device), else nullptr
    int dual_sided_s_curve;         // DUAL_SIDED_S_CURVE
};

// Entries of the S-curve table: one per index of a path of at most PCT_MLP_PATH_CAP entries.
constexpr int kSCurveEntries = PCT_MLP_PATH_CAP;

// The S-curve index of entry j of an n-entry path (s_curve_scale_GPU, B.cu:10629-10633): the
// reference's UINT arithmetic, min(j, n-1-j) when dual-sided, else j.
__device__ __forceinline__ unsigned s_curve_index(const Geometry& g, int j, int n)
{
    const unsigned uj = (unsigned)j;
    return g.dual_sided_s_curve ? min(uj, (unsigned)n - 1u - uj) : uj;
}

// Device pointers of the MLP lookup tables (B.cu:8503-8526).
struct Tables {
    const double* sin_table;
    const double* cos_table;
    const double* scattering_table;
    const double* poly_1_2;
    const double* poly_2_3;
    const double* poly_3_4;
    const double* poly_2_6;
    const double* poly_3_12;
};

// Deterministic scatter accumulator: the updates of a DROP block as 64-bit fixed-point sums
// (scale 2^40) and their counts.  Integer addition is associative, so the sums do not depend on
// the order in which the reductions land.
struct FixedAcc {
    unsigned long long* sum;
    unsigned* cnt;
};
constexpr double kFixedScale = 1099511627776.0;  // 2^40

// Reconstruction histories in HBM, structure of arrays (B.h:1257-1271 order).
struct HistorySoA {
    float* x_entry;
    float* y_entry;
    float* z_entry;
    float* x_exit;
    float* y_exit;
    float* z_exit;
    float* xy_entry_angle;
    float* xz_entry_angle;
    float* xy_exit_angle;
    float* xz_exit_angle;
    float* WEPL;
    uint32_t* first_MLP_voxel;
};

// Programmatic dependent launch.  A kernel launched with programmatic stream serialization may
// be scheduled while the previous kernel in its stream is still finishing; it must pass
// grid_dependency_wait() (griddepcontrol.wait: returns once that kernel has completed and its
// memory is visible) before it touches anything that kernel writes.  allow_dependent_launch()
// lets the next such kernel be scheduled once every CTA of this one has issued it.  Both are
// no-ops for a kernel launched without the attribute.
__device__ __forceinline__ void grid_dependency_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void allow_dependent_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Launch `kernel`, with programmatic stream serialization when `pdl` is set.
template <typename... KArgs, typename... Args>
cudaError_t launch_kernel(bool pdl, void (*kernel)(KArgs...), unsigned grid, unsigned block, cudaStream_t stream,
                          Args... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

// Reference constants (B.h:741-754, 818).
__host__ __device__ inline double ref_pi() { return 3.141592653589793; }  // == 4*atan(1.0)

Geometry make_geometry(const pct_config& c);
std::string cuda_error_string(cudaError_t e);

}  // namespace pct

// Launch-site error check used inside the C-ABI implementation.
#define PCT_CUDA_TRY(expr)                                                      \
    do {                                                                        \
        cudaError_t _e = (expr);                                                \
        if (_e != cudaSuccess) return ctx_fail(ctx, PCT_ERR_CUDA, #expr, _e);   \
    } while (0)
