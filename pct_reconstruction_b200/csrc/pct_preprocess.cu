// pct_preprocess.cu -- the stages that turn tracker data into reconstruction histories and the
// initial image: recon-volume intersections, binning, statistical cuts, sinogram, FBP, hull
// detection, initial iterate and the hull-entry/exit (MLP endpoint) search.
//
// Each kernel restates one reference kernel (B.cu line cited at the kernel) in the same double and
// float operations -- including where the reference calls float functions on float operands
// (atan2 on float differences resolves to atan2f, abs on a float to fabsf) and where it calls
// powf on doubles -- so integer results (bins, survivors, hull voxels, first MLP voxels) come out
// identical.  This translation unit is compiled with -fmad=false.
//
// Design differences from the reference, all of which leave results unchanged:
//  * all histories are resident in HBM: no MAX_GPU_HISTORIES chunking, no host round trips;
//  * the host-side compactions (std::vector push_back loops, B.cu:5429-5450, 5892-5911,
//    8286-8294) are stable device compactions (prefix sum + scatter), so the history order -- and
//    with it the DROP block composition -- is the reference's;
//  * the filter, backprojection and median filter accumulate each output in one thread in the
//    reference's loop order, so they are deterministic (the reference's atomicAdds there each
//    touch one thread's own element);
//  * MSC edge detection runs out of place with the in-place kernel's condition (B.cu:6911-6956
//    reads neighbours that other blocks may already have overwritten; the result here is the
//    one that kernel gives when none has been);
//  * the hull voxel walks stop when an index leaves the grid on either side and after a bounded
//    number of steps: the reference's SC/MSC/SM walks (B.cu:6681-7099) only test the upper bounds
//    and would run forever (writing out of bounds) on a walk that misses its exit voxel towards
//    negative indices; such walks are counted (counter "wait_expired").
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "pct_context.h"

namespace pct {

namespace {

constexpr double kPi = 3.141592653589793;      // 4*atan(1.0)
constexpr double kPiOver4 = 0.7853981633974483;  // atan(1.0)
constexpr double kPiOver2 = 1.5707963267948966;  // 2*atan(1.0)

// Reference macro values derived from the configuration, by value for kernels.
struct PreGeom {
    int columns, rows, slices, num_voxels;
    double voxel_width, voxel_height, voxel_thickness;
    double R, H;  // RECON_CYL_RADIUS, RECON_CYL_HEIGHT
    int t_bins, v_bins, angular_bins, num_bins;
    double t_bin_size, v_bin_size, angular_bin_size;
    int sigmas_to_keep, sample_std_dev;
    int sinogram_filter;
    double source_radius, rsp_air, fbp_threshold;
    double sc_lower, sc_upper, msc_lower, msc_upper, sm_lower, sm_scale;
    int msc_diff_thresh;
};

PreGeom make_pregeom(const pct_config& c)
{
    PreGeom g{};
    g.columns = c.COLUMNS;
    g.rows = c.ROWS;
    g.slices = c.SLICES;
    g.num_voxels = c.NUM_VOXELS;
    g.voxel_width = c.VOXEL_WIDTH;
    g.voxel_height = c.VOXEL_HEIGHT;
    g.voxel_thickness = c.VOXEL_THICKNESS;
    g.R = c.RECON_CYL_RADIUS;
    g.H = c.RECON_CYL_HEIGHT;
    g.t_bins = c.T_BINS;
    g.v_bins = c.V_BINS;
    g.angular_bins = c.ANGULAR_BINS;
    g.num_bins = c.NUM_BINS;
    g.t_bin_size = c.T_BIN_SIZE;
    g.v_bin_size = c.V_BIN_SIZE;
    g.angular_bin_size = c.ANGULAR_BIN_SIZE;
    g.sigmas_to_keep = c.SIGMAS_TO_KEEP;
    g.sample_std_dev = c.SAMPLE_STD_DEV ? 1 : 0;
    g.sinogram_filter = c.SINOGRAM_FILTER;
    g.source_radius = c.SOURCE_RADIUS;
    g.rsp_air = c.RSP_AIR;
    g.fbp_threshold = c.FBP_THRESHOLD;
    g.sc_lower = c.SC_LOWER_THRESHOLD;
    g.sc_upper = c.SC_UPPER_THRESHOLD;
    g.msc_lower = c.MSC_LOWER_THRESHOLD;
    g.msc_upper = c.MSC_UPPER_THRESHOLD;
    g.sm_lower = c.SM_LOWER_THRESHOLD;
    g.sm_scale = c.SM_SCALE_THRESHOLD;
    g.msc_diff_thresh = c.MSC_DIFF_THRESH;
    return g;
}

// Per-history geometry of one history set, structure of arrays.
enum GeomArray { kXE, kYE, kZE, kXO, kYO, kZO, kXYE, kXZE, kXYO, kXZO, kNumGeom };
const char* const kGeomNames[kNumGeom] = {"x_entry", "y_entry", "z_entry", "x_exit", "y_exit", "z_exit",
                                          "xy_entry_angle", "xz_entry_angle", "xy_exit_angle", "xz_exit_angle"};
struct GeomPtrs {
    float* a[kNumGeom];
};

// Tracker inputs (B.cu:4139-4766 arrays after the mm->cm conversion).
enum TrackerArray { kTIn1, kTIn2, kTOut1, kTOut2, kUIn1, kUIn2, kUOut1, kUOut2, kVIn1, kVIn2, kVOut1, kVOut2, kNumTracker };
const char* const kTrackerNames[kNumTracker] = {"t_in_1", "t_in_2", "t_out_1", "t_out_2", "u_in_1", "u_in_2",
                                                "u_out_1", "u_out_2", "v_in_1", "v_in_2", "v_out_1", "v_out_2"};
struct TrackerPtrs {
    const float* a[kNumTracker];
};
static_assert(kTrackerSlots == kNumTracker + 2, "tracker slots: coordinates, WEPL, angle");

}  // namespace

// Device arrays of the preprocessing stages.
struct Preproc {
    long long n_raw = 0, cap_raw = 0;
    float* tracker[kNumTracker] = {};
    float* gantry_angle = nullptr;   // degrees
    int integer_angles = 0;
    float* raw_geom[kNumGeom] = {};  // intersections output
    float* raw_wepl = nullptr;
    uint8_t* missed = nullptr;
    int* raw_bin_num = nullptr;
    uint8_t* keep = nullptr;
    // current history vectors (compacted after binning, after cuts, after reconstruction cuts)
    long long n_vec = 0, cap_vec = 0;
    float* vec_geom[kNumGeom] = {};
    float* vec_wepl = nullptr;
    int* vec_bin_num = nullptr;
    uint32_t* vec_first_voxel = nullptr;
    // compaction scratch
    float* tmp_geom[kNumGeom] = {};
    float* tmp_wepl = nullptr;
    int* tmp_bin_num = nullptr;
    int* flags = nullptr;
    long long* offsets = nullptr;
    long long* scan_tmp = nullptr;
    long long cap_scratch = 0;
    // bins
    int* bin_counts = nullptr;
    float *mean_WEPL = nullptr, *mean_rel_ut_angle = nullptr, *mean_rel_uv_angle = nullptr;
    float *stddev_WEPL = nullptr, *stddev_rel_ut_angle = nullptr, *stddev_rel_uv_angle = nullptr;
    float *sinogram = nullptr, *sinogram_filtered = nullptr;
    // images
    float *FBP_image = nullptr, *FBP_median = nullptr;
    uint8_t *FBP_hull = nullptr, *SC_hull = nullptr, *hull = nullptr;
    int *MSC_counts = nullptr, *SM_counts = nullptr, *SM_differences = nullptr, *SM_thresholds = nullptr;
    int* edge_tmp = nullptr;
    unsigned* walk_hist = nullptr;  // bucket-sort scratch of the walk order
    bool hull_ready = false;
};

void preproc_release(Preproc* p)
{
    if (!p) return;
    for (int k = 0; k < kNumTracker; k++) cudaFree(p->tracker[k]);
    for (int k = 0; k < kNumGeom; k++) {
        cudaFree(p->raw_geom[k]);
        cudaFree(p->vec_geom[k]);
        cudaFree(p->tmp_geom[k]);
    }
    void* ptrs[] = {p->gantry_angle, p->raw_wepl, p->missed, p->raw_bin_num, p->keep, p->vec_wepl, p->vec_bin_num,
                    p->vec_first_voxel, p->tmp_wepl, p->tmp_bin_num, p->flags, p->offsets, p->scan_tmp,
                    p->bin_counts, p->mean_WEPL, p->mean_rel_ut_angle, p->mean_rel_uv_angle, p->stddev_WEPL,
                    p->stddev_rel_ut_angle, p->stddev_rel_uv_angle, p->sinogram, p->sinogram_filtered,
                    p->FBP_image, p->FBP_median, p->FBP_hull, p->SC_hull, p->hull, p->MSC_counts, p->SM_counts,
                    p->SM_differences, p->SM_thresholds, p->edge_tmp, p->walk_hist};
    for (void* q : ptrs) cudaFree(q);
    delete p;
}

namespace {

// ------------------------------------------------------------------------------------------
// Device helpers
// ------------------------------------------------------------------------------------------

// calculate_intercepts (B.cu:5286-5372).  The intercept stays at its initial value when the
// line misses the circle (the reference leaves it unassigned).
__device__ bool calculate_intercepts(double R, double u, double t, double ut_angle, double& u_intercept,
                                     double& t_intercept)
{
    const bool entry_in_cone = ((ut_angle > kPiOver4) && (ut_angle < 3 * kPiOver4)) ||
                               ((ut_angle > 5 * kPiOver4) && (ut_angle < 7 * kPiOver4));
    double u_temp;
    if (entry_in_cone) {
        u_temp = u;
        u = -t;
        t = u_temp;
        ut_angle += kPiOver2;
    }
    const double m = tan(ut_angle);
    const double b_in = t - m * u;
    const double a = 1 + powf((float)m, 2.0f);
    const double b = 2 * m * b_in;
    const double c = __fsub_rn(powf((float)b_in, 2.0f), powf((float)R, 2.0f));
    const double entry_discriminant = powf((float)b, 2.0f) - (4 * a * c);
    const bool intersected = (entry_discriminant > 0);
    if (intersected) {
        const double u_intercept_1 = (sqrt(entry_discriminant) - b) / (2 * a);
        const double u_intercept_2 = (sqrt(entry_discriminant) + b) / (2 * a);
        const double t_intercept_1 = m * u_intercept_1 + b_in;
        const double t_intercept_2 = m * u_intercept_2 - b_in;
        const double squared_distance_1 =
            __fadd_rn(powf((float)(u_intercept_1 - u), 2.0f), powf((float)(t_intercept_1 - t), 2.0f));
        const double squared_distance_2 =
            __fadd_rn(powf((float)(u_intercept_2 + u), 2.0f), powf((float)(t_intercept_2 + t), 2.0f));
        u_intercept = u_intercept_1 * (squared_distance_1 <= squared_distance_2) -
                      u_intercept_2 * (squared_distance_1 > squared_distance_2);
        t_intercept = t_intercept_1 * (squared_distance_1 <= squared_distance_2) -
                      t_intercept_2 * (squared_distance_1 > squared_distance_2);
    }
    if (entry_in_cone) {
        u_temp = u_intercept;
        u_intercept = t_intercept;
        t_intercept = -u_temp;
    }
    return intersected;
}

// recon_volume_intersections_GPU / _exact_angles (B.cu:4890-5153): outputs are stored as float and
// later read back as float, as the reference does.
__global__ void intersections_kernel(PreGeom g, long long n, TrackerPtrs T, const float* __restrict__ angle_deg,
                                     int integer_angles, GeomPtrs out, uint8_t* __restrict__ missed)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float t_in_1 = T.a[kTIn1][i], t_in_2 = T.a[kTIn2][i], t_out_1 = T.a[kTOut1][i], t_out_2 = T.a[kTOut2][i];
    const float u_in_1 = T.a[kUIn1][i], u_in_2 = T.a[kUIn2][i], u_out_1 = T.a[kUOut1][i], u_out_2 = T.a[kUOut2][i];
    const float v_in_1 = T.a[kVIn1][i], v_in_2 = T.a[kVIn2][i], v_out_1 = T.a[kVOut1][i], v_out_2 = T.a[kVOut2][i];
    const double ANGLE_TO_RADIANS = (kPi / 180.0);
    const double rotation_angle_radians =
        integer_angles ? (int)angle_deg[i] * ANGLE_TO_RADIANS : angle_deg[i] * ANGLE_TO_RADIANS;
    const double HALF_H = g.H * 0.5;

    const double ut_entry_angle = atan2f(__fsub_rn(t_in_2, t_in_1), __fsub_rn(u_in_2, u_in_1));
    double u_entry = 0.0, t_entry = 0.0;
    bool entered = calculate_intercepts(g.R, u_in_2, t_in_2, ut_entry_angle, u_entry, t_entry);
    const float xy_entry_angle = (float)(ut_entry_angle + rotation_angle_radians);
    float x_entry = (float)((cos(rotation_angle_radians) * u_entry) - (sin(rotation_angle_radians) * t_entry));
    float y_entry = (float)((sin(rotation_angle_radians) * u_entry) + (cos(rotation_angle_radians) * t_entry));

    const double ut_exit_angle = atan2f(__fsub_rn(t_out_2, t_out_1), __fsub_rn(u_out_2, u_out_1));
    double u_exit = 0.0, t_exit = 0.0;
    bool exited = calculate_intercepts(g.R, u_out_1, t_out_1, ut_exit_angle, u_exit, t_exit);
    const float xy_exit_angle = (float)(ut_exit_angle + rotation_angle_radians);
    float x_exit = (float)((cos(rotation_angle_radians) * u_exit) - (sin(rotation_angle_radians) * t_exit));
    float y_exit = (float)((sin(rotation_angle_radians) * u_exit) + (cos(rotation_angle_radians) * t_exit));

    const double uv_entry_slope = __fdiv_rn(__fsub_rn(v_in_2, v_in_1), __fsub_rn(u_in_2, u_in_1));
    const double uv_exit_slope = __fdiv_rn(__fsub_rn(v_out_2, v_out_1), __fsub_rn(u_out_2, u_out_1));
    const float xz_entry_angle = atan2f(__fsub_rn(v_in_2, v_in_1), __fsub_rn(u_in_2, u_in_1));
    const float xz_exit_angle = atan2f(__fsub_rn(v_out_2, v_out_1), __fsub_rn(u_out_2, u_out_1));

    u_entry = (cos(rotation_angle_radians) * x_entry) + (sin(rotation_angle_radians) * y_entry);
    u_exit = (cos(rotation_angle_radians) * x_exit) + (sin(rotation_angle_radians) * y_exit);
    float z_entry = (float)(v_in_2 + uv_entry_slope * (u_entry - u_in_2));
    float z_exit = (float)(v_out_1 - uv_exit_slope * (u_out_1 - u_exit));

    if (entered && exited) {
        if ((fabsf(z_entry) < HALF_H) && (fabsf(z_exit) > HALF_H)) {
            const double recon_cyl_fraction =
                fabs((((z_exit >= 0) - (z_exit < 0)) * g.H * 0.5 - z_entry) / (double)__fsub_rn(z_exit, z_entry));
            x_exit = (float)(x_entry + recon_cyl_fraction * __fsub_rn(x_exit, x_entry));
            y_exit = (float)(y_entry + recon_cyl_fraction * __fsub_rn(y_exit, y_entry));
            z_exit = (float)(((z_exit >= 0) - (z_exit < 0)) * g.H * 0.5);
        } else if (fabsf(z_entry) > HALF_H) {
            entered = false;
            exited = false;
        }
        if ((fabsf(z_entry) > HALF_H) && (fabsf(z_exit) < HALF_H)) {
            const double recon_cyl_fraction =
                fabs((((z_exit >= 0) - (z_exit < 0)) * g.H * 0.5 - z_exit) / (double)__fsub_rn(z_exit, z_entry));
            x_entry = (float)(x_exit + recon_cyl_fraction * __fsub_rn(x_exit, x_entry));
            y_entry = (float)(y_exit + recon_cyl_fraction * __fsub_rn(y_exit, y_entry));
            z_entry = (float)(((z_entry >= 0) - (z_entry < 0)) * g.H * 0.5);
        }
        if ((fabsf(__fsub_rn(t_out_1, t_in_2)) > 5) || (fabsf(__fsub_rn(v_out_1, v_in_2)) > 5)) {
            entered = false;
            exited = false;
        }
    }
    out.a[kXE][i] = x_entry;
    out.a[kYE][i] = y_entry;
    out.a[kZE][i] = z_entry;
    out.a[kXO][i] = x_exit;
    out.a[kYO][i] = y_exit;
    out.a[kZO][i] = z_exit;
    out.a[kXYE][i] = xy_entry_angle;
    out.a[kXZE][i] = xz_entry_angle;
    out.a[kXYO][i] = xy_exit_angle;
    out.a[kXZO][i] = xz_exit_angle;
    missed[i] = (!entered || !exited) ? 1 : 0;
}

// rel angle of a history, wrapped as B.cu:5528-5537 does
__device__ __forceinline__ double rel_angle(float exit_angle, float entry_angle)
{
    double a = __fsub_rn(exit_angle, entry_angle);
    if (a > kPi) a -= 2 * kPi;
    if (a < -kPi) a += 2 * kPi;
    return a;
}

// binning_GPU (B.cu:5482-5553); bin_num keeps its 0 default when t/v fall outside (B.cu:5380).
__global__ void binning_kernel(PreGeom g, long long n, GeomPtrs G, const float* __restrict__ WEPL,
                               const uint8_t* __restrict__ missed, int* __restrict__ bin_num, int* bin_counts,
                               float* mean_WEPL, float* mean_ut, float* mean_uv)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float xe = G.a[kXE][i], ye = G.a[kYE][i], ze = G.a[kZE][i];
    const float xo = G.a[kXO][i], yo = G.a[kYO][i], zo = G.a[kZO][i];
    const double x_midpath = __fdiv_rn(__fadd_rn(xe, xo), 2.0f);
    const double y_midpath = __fdiv_rn(__fadd_rn(ye, yo), 2.0f);
    const double z_midpath = __fdiv_rn(__fadd_rn(ze, zo), 2.0f);
    double path_angle = atan2f(__fsub_rn(yo, ye), __fsub_rn(xo, xe));
    if (path_angle < 0) path_angle += 2 * kPi;
    const double RADIANS_TO_ANGLE = (180.0 / kPi), ANGLE_TO_RADIANS = (kPi / 180.0);
    const int angle_bin = int((path_angle * RADIANS_TO_ANGLE / g.angular_bin_size) + 0.5) % g.angular_bins;
    const double angle = angle_bin * g.angular_bin_size * ANGLE_TO_RADIANS;
    const double t = y_midpath * cos(angle) - x_midpath * sin(angle);
    const int t_bin = int((t / g.t_bin_size) + g.t_bins / 2);
    const double v = z_midpath;
    const int v_bin = int((v / g.v_bin_size) + g.v_bins / 2);
    int bin = 0;
    if ((t_bin >= 0) && (v_bin >= 0) && (t_bin < g.t_bins) && (v_bin < g.v_bins)) {
        bin = t_bin + angle_bin * g.t_bins + v_bin * g.t_bins * g.angular_bins;
        if (!missed[i]) {
            const double rel_ut_angle = rel_angle(G.a[kXYO][i], G.a[kXYE][i]);
            const double rel_uv_angle = rel_angle(G.a[kXZO][i], G.a[kXZE][i]);
            atomicAdd(&bin_counts[bin], 1);
            atomicAdd(&mean_WEPL[bin], WEPL[i]);
            atomicAdd(&mean_ut[bin], (float)rel_ut_angle);
            atomicAdd(&mean_uv[bin], (float)rel_uv_angle);
        }
    }
    bin_num[i] = bin;
}

// calculate_means_GPU (B.cu:5644)
__global__ void means_kernel(int nb, const int* __restrict__ bin_counts, float* mean_WEPL, float* mean_ut, float* mean_uv)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    const int c = bin_counts[b];
    if (c > 0) {
        mean_WEPL[b] = __fdiv_rn(mean_WEPL[b], (float)c);
        mean_ut[b] = __fdiv_rn(mean_ut[b], (float)c);
        mean_uv[b] = __fdiv_rn(mean_uv[b], (float)c);
    }
}

// sum_squared_deviations_GPU (B.cu:5689)
__global__ void sum_sq_dev_kernel(long long n, const int* __restrict__ bin_num, const float* __restrict__ WEPL,
                                  GeomPtrs G, const float* __restrict__ mean_WEPL, const float* __restrict__ mean_ut,
                                  const float* __restrict__ mean_uv, float* sd_WEPL, float* sd_ut, float* sd_uv)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int b = bin_num[i];
    const double rel_ut_angle = rel_angle(G.a[kXYO][i], G.a[kXYE][i]);
    const double rel_uv_angle = rel_angle(G.a[kXZO][i], G.a[kXZE][i]);
    const double WEPL_difference = __fsub_rn(WEPL[i], mean_WEPL[b]);
    const double rel_ut_angle_difference = rel_ut_angle - mean_ut[b];
    const double rel_uv_angle_difference = rel_uv_angle - mean_uv[b];
    atomicAdd(&sd_WEPL[b], powf((float)WEPL_difference, 2.0f));
    atomicAdd(&sd_ut[b], powf((float)rel_ut_angle_difference, 2.0f));
    atomicAdd(&sd_uv[b], powf((float)rel_uv_angle_difference, 2.0f));
}

// calculate_standard_deviations_GPU (B.cu:5737); also zeroes bin_counts (B.cu:5748-5749)
__global__ void stddev_kernel(int nb, int sample, int* bin_counts, float* sd_WEPL, float* sd_ut, float* sd_uv)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    const int c = bin_counts[b];
    if (c > 1) {
        const float d = (float)(c - sample);
        sd_WEPL[b] = sqrtf(__fdiv_rn(sd_WEPL[b], d));
        sd_ut[b] = sqrtf(__fdiv_rn(sd_ut[b], d));
        sd_uv[b] = sqrtf(__fdiv_rn(sd_uv[b], d));
    }
    bin_counts[b] = 0;
}

// statistical_cuts_GPU (B.cu:5937-5971): flags survivors, accumulates counts and WEPL sums
__global__ void cuts_kernel(PreGeom g, long long n, const int* __restrict__ bin_num, const float* __restrict__ WEPL,
                            GeomPtrs G, const float* __restrict__ mean_WEPL, const float* __restrict__ mean_ut,
                            const float* __restrict__ mean_uv, const float* __restrict__ sd_WEPL,
                            const float* __restrict__ sd_ut, const float* __restrict__ sd_uv, int* bin_counts,
                            float* sinogram, int* __restrict__ keep)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int b = bin_num[i];
    const double rel_ut_angle = rel_angle(G.a[kXYO][i], G.a[kXYE][i]);
    const double rel_uv_angle = rel_angle(G.a[kXZO][i], G.a[kXZE][i]);
    const bool passed_ut_cut = (fabs(rel_ut_angle - mean_ut[b]) < (double)__fmul_rn((float)g.sigmas_to_keep, sd_ut[b]));
    const bool passed_uv_cut = (fabs(rel_uv_angle - mean_uv[b]) < (double)__fmul_rn((float)g.sigmas_to_keep, sd_uv[b]));
    const bool passed_WEPL_cut = (fabsf(__fsub_rn(mean_WEPL[b], WEPL[i])) <= __fmul_rn((float)g.sigmas_to_keep, sd_WEPL[b]));
    const bool failed = !passed_ut_cut || !passed_uv_cut || !passed_WEPL_cut;
    if (!failed) {
        atomicAdd(&bin_counts[b], 1);
        atomicAdd(&sinogram[b], WEPL[i]);
    }
    keep[i] = failed ? 0 : 1;
}

// construct_sinogram_GPU (B.cu:6073)
__global__ void sinogram_kernel(int nb, const int* __restrict__ bin_counts, float* sinogram)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    const int c = bin_counts[b];
    if (c > 0) sinogram[b] = __fdiv_rn(sinogram[b], (float)c);
}

// filter_GPU (B.cu:6206-6240): one thread per output bin, summing over the strip in the
// reference's order; each term is rounded to float as atomicAdd(float*, double) rounds it.
// The reference leaves the filter value unset for UNFILTERED; here it passes the sinogram through.
__global__ void filter_kernel(PreGeom g, const float* __restrict__ sinogram, float* __restrict__ filtered_out)
{
    const long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= g.num_bins) return;
    const int t_bin = (int)(b % g.t_bins);
    const int strip = (int)(b / g.t_bins);  // v_bin * ANGULAR_BINS + angle_bin
    const int v_bin = strip / g.angular_bins;
    const long long strip_index = (long long)strip * g.t_bins;
    if (g.sinogram_filter == PCT_UNFILTERED) {
        filtered_out[b] = sinogram[b];
        return;
    }
    const double v = (v_bin - g.v_bins / 2 + 0.5) * g.v_bin_size;
    // RAM_LAK_TAU = 2/ROOT_TWO * T_BIN_SIZE, ROOT_TWO = sqrtf(2.0): a float quotient
    const double ram_lak_tau = (double)__fdiv_rn(2.0f, sqrtf(2.0f)) * g.t_bin_size;
    float acc = 0.0f;
    for (int t_bin_ref = 0; t_bin_ref < g.t_bins; t_bin_ref++) {
        const double t = (t_bin_ref - g.t_bins / 2 + 0.5) * g.t_bin_size;
        const int t_bin_sep = t_bin - t_bin_ref;
        const double scale_factor = g.source_radius / sqrt(g.source_radius * g.source_radius + t * t + v * v);
        double filtered;
        if (g.sinogram_filter == PCT_RAM_LAK) {
            if (t_bin_sep == 0) filtered = 1.0 / (4.0 * pow(ram_lak_tau, 2.0));
            else if (t_bin_sep % 2 == 0) filtered = 0;
            else filtered = -1.0 / (pow(ram_lak_tau * kPi * t_bin_sep, 2.0));
        } else {
            filtered = 1.0 / ((g.t_bin_size * kPi * g.t_bin_size * kPi) * (1.0 - (4 * t_bin_sep * t_bin_sep)));
        }
        acc = __fadd_rn(acc, (float)(g.t_bin_size * sinogram[strip_index + t_bin_ref] * filtered * scale_factor));
    }
    filtered_out[b] = acc;
}

// voxel_2_3D_voxels_GPU (B.cu:11117-11133): the reference's loops stop at "> 0", so an index that
// is an exact multiple of COLUMNS*ROWS (or COLUMNS) is decomposed one step short; kept as is.
__device__ __forceinline__ void voxel_2_3D_voxels(const PreGeom& g, int voxel, int& vx, int& vy, int& vz)
{
    const int CR = g.columns * g.rows;
    vz = voxel > 0 ? (voxel - 1) / CR : 0;
    voxel -= vz * CR;
    vy = voxel > 0 ? (voxel - 1) / g.columns : 0;
    voxel -= vy * g.columns;
    vx = voxel;
}

__device__ __forceinline__ double voxel_2_position(int voxel_i, double size, int num_i, int progression)
{
    const double zero_voxel = (num_i - 1) / 2.0;
    return progression * (voxel_i - zero_voxel) * size;
}

// backprojection_GPU2 (B.cu:6340-6479): one thread per voxel, angles summed in order.
__global__ void backprojection_kernel(PreGeom g, const float* __restrict__ sinogram_filtered, float* __restrict__ FBP)
{
    const long long voxel = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (voxel >= g.num_voxels) return;
    const double ANGLE_TO_RADIANS = (kPi / 180.0);
    const double delta = g.angular_bin_size * ANGLE_TO_RADIANS;
    int vx, vy, vz;
    voxel_2_3D_voxels(g, (int)voxel, vx, vy, vz);
    const double x = voxel_2_position(vx, g.voxel_width, g.columns, 1);
    const double y = voxel_2_position(vy, g.voxel_height, g.rows, -1);
    const double z = voxel_2_position(vz, g.voxel_thickness, g.slices, -1);
    if ((x * x + y * y) > (g.R * g.R)) {
        FBP[voxel] = (float)g.rsp_air;
        return;
    }
    const int T = g.t_bins, V = g.v_bins, A = g.angular_bins;
    float acc = 0.0f;
    for (int angle_bin = 0; angle_bin < A; angle_bin++) {
        const double bin_angle = angle_bin * delta;
        const double u = x * cos(bin_angle) + y * sin(bin_angle);
        const double t = y * cos(bin_angle) - x * sin(bin_angle);
        const double v = z;
        const double detector_number_t = (t - u * (t / (g.source_radius + u))) / g.t_bin_size + T / 2.0;
        const int t_bin = (int)floor(detector_number_t);
        const double eta = detector_number_t - t_bin;
        const double detector_number_v = (v - u * (v / (g.source_radius + u))) / g.v_bin_size + V / 2.0;
        const int v_bin = (int)floor(detector_number_v);
        const double epsilon = detector_number_v - v_bin;
        const double scale_factor = powf((float)(g.source_radius / (g.source_radius + u)), 2.0f);
        const long long bin11 = ((long long)v_bin * A + angle_bin) * T + t_bin;
        const long long bin12 = bin11 + 1;
        const long long bin21 = bin11 + (long long)A * T;
        const long long bin22 = bin21 + 1;
        float xterm = 0.0f;
        if (t_bin > -1 && t_bin < T - 1) {
            if (v_bin > -1 && v_bin < V - 1) {
                xterm = (float)(sinogram_filtered[bin11] * (1 - eta) * (1 - epsilon) + sinogram_filtered[bin12] * eta * (1 - epsilon) +
                                sinogram_filtered[bin21] * (1 - eta) * epsilon + sinogram_filtered[bin22] * eta * epsilon);
            } else if (v_bin == -1) {
                xterm = (float)(sinogram_filtered[bin21] * (1 - eta) * epsilon + sinogram_filtered[bin22] * eta * epsilon);
            } else if (v_bin == V - 1) {
                xterm = (float)(sinogram_filtered[bin11] * (1 - eta) * (1 - epsilon) + sinogram_filtered[bin12] * eta * (1 - epsilon));
            }
        } else if (t_bin == -1) {
            if (v_bin > -1 && v_bin < V - 1) {
                xterm = (float)(sinogram_filtered[bin12] * eta * (1 - epsilon) + sinogram_filtered[bin22] * eta * epsilon);
            } else if (v_bin == -1) {
                xterm = (float)(sinogram_filtered[bin22] * eta * epsilon);
            } else if (v_bin == V - 1) {
                xterm = (float)(sinogram_filtered[bin12] * eta * (1 - epsilon));
            }
        } else if (t_bin == T - 1) {
            if (v_bin > -1 && v_bin < V - 1) {
                xterm = (float)(sinogram_filtered[bin11] * (1 - eta) * (1 - epsilon) + sinogram_filtered[bin21] * (1 - eta) * epsilon);
            } else if (v_bin == -1) {
                xterm = (float)(sinogram_filtered[bin21] * (1 - eta) * epsilon);
            } else if (v_bin == V - 1) {
                xterm = (float)(sinogram_filtered[bin11] * (1 - eta) * (1 - epsilon));
            }
        }
        acc = __fadd_rn(acc, (float)(xterm * delta * scale_factor));
    }
    FBP[voxel] = acc;
}

// median_filter_2D (B.cu:7482-7521): (2r+1)^2 neighbourhood per slice, the element at index
// n/2 of the sorted values; voxels within r of a slice edge stay 0.  Selection by counting.
__global__ void median_kernel(PreGeom g, int radius, const float* __restrict__ in, float* __restrict__ out)
{
    const long long voxel = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (voxel >= g.num_voxels) return;
    const int CR = g.columns * g.rows;
    const int slice = (int)(voxel / CR), rem = (int)(voxel % CR), row = rem / g.columns, col = rem % g.columns;
    if (col < radius || col >= g.columns - radius || row < radius || row >= g.rows - radius) {
        out[voxel] = 0.0f;
        return;
    }
    const int side = 2 * radius + 1, count = side * side, middle = count / 2;
    float vals[225];  // radius <= 7
    int k = 0;
    for (int c = col - radius; c <= col + radius; c++)
        for (int r = row - radius; r <= row + radius; r++) vals[k++] = in[c + r * g.columns + (long long)slice * CR];
    // element of rank `middle`: the value with fewer than middle+1 smaller elements and at least
    // middle+1 elements <= it
    float result = vals[0];
    for (int a = 0; a < count; a++) {
        int less = 0, less_eq = 0;
        for (int b = 0; b < count; b++) {
            less += vals[b] < vals[a];
            less_eq += vals[b] <= vals[a];
        }
        if (less <= middle && middle < less_eq) {
            result = vals[a];
            break;
        }
    }
    out[voxel] = result;
}

// FBP_image_2_hull_GPU (B.cu:6592)
__global__ void fbp_hull_kernel(PreGeom g, const float* __restrict__ FBP, uint8_t* __restrict__ hull)
{
    const long long voxel = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (voxel >= g.num_voxels) return;
    const int rem = (int)(voxel % ((long long)g.columns * g.rows)), row = rem / g.columns, column = rem % g.columns;
    const double x = -g.R + (column + 0.5) * g.voxel_width;
    const double y = g.R - (row + 0.5) * g.voxel_height;
    const double d_squared = __fadd_rn(powf((float)x, 2.0f), powf((float)y, 2.0f));
    hull[voxel] = (FBP[voxel] > g.fbp_threshold && (d_squared < powf((float)g.R, 2.0f))) ? 1 : 0;
}

// initialize_hull_GPU (B.cu:6659): 1 inside the reconstruction cylinder
template <class T>
__global__ void init_hull_kernel(PreGeom g, T* __restrict__ hull)
{
    const long long voxel = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (voxel >= g.num_voxels) return;
    const int rem = (int)(voxel % ((long long)g.columns * g.rows)), row = rem / g.columns, column = rem % g.columns;
    const double x = (column - g.columns / 2 + 0.5) * g.voxel_width;
    const double y = (g.rows / 2 - row - 0.5) * g.voxel_height;
    hull[voxel] = (__fadd_rn(powf((float)x, 2.0f), powf((float)y, 2.0f)) < powf((float)g.R, 2.0f)) ? 1 : 0;
}

// ---- straight-line voxel walks (B.cu:11313-11462) ----
__device__ __forceinline__ int calculate_voxel(double zero, double pos, double size)
{
    const double q = fabs(pos - zero) / size;
    return q < 2147483647.0 ? (int)q : 2147483647;
}
__device__ __forceinline__ double edge_coordinate(double zero, int voxel_entered, double size, int inc, int step)
{
    const int on_edge = (step == inc) ? voxel_entered : voxel_entered + 1;
    return zero + (inc * on_edge * size);
}
__device__ __forceinline__ double distance_remaining(double zero, double pos, int inc, int step, double size, int voxel)
{
    const int next_voxel = voxel + inc * step;
    return fabs(edge_coordinate(zero, next_voxel, size, inc, step) - pos);
}
__device__ __forceinline__ double corresponding_coordinate(double m, double x, double x0, double y0) { return m * (x - x0) + y0; }

struct WalkState {
    double x, y, z, x_to_go, y_to_go, z_to_go;
    int vx, vy, vz, voxel;
};

// take_3D_step_GPU (B.cu:11392-11460) with X_INCREASING_DIRECTION = RIGHT, Y/Z = DOWN
__device__ void take_3D_step(const PreGeom& g, int xd, int yd, int zd, double dy_dx, double dz_dx, double dz_dy,
                             double dx_dy, double dx_dz, double dy_dz, double x0, double y0, double z0, WalkState& w)
{
    const double X0 = -g.R, Y0 = g.R, Z0 = g.H / 2;
    const double x_extension = fabs(dz_dx) * w.x_to_go;
    const double y_extension = fabs(dz_dy) * w.y_to_go;
    if ((w.z_to_go <= x_extension) && (w.z_to_go <= y_extension)) {
        w.vz -= zd;
        w.z = edge_coordinate(Z0, w.vz, g.voxel_thickness, -1, zd);
        w.x = corresponding_coordinate(dx_dz, w.z, z0, x0);
        w.y = corresponding_coordinate(dy_dz, w.z, z0, y0);
        w.x_to_go = distance_remaining(X0, w.x, 1, xd, g.voxel_width, w.vx);
        w.y_to_go = distance_remaining(Y0, w.y, -1, yd, g.voxel_height, w.vy);
        w.z_to_go = g.voxel_thickness;
    } else if (x_extension <= y_extension) {
        w.vx += xd;
        w.x = edge_coordinate(X0, w.vx, g.voxel_width, 1, xd);
        w.y = corresponding_coordinate(dy_dx, w.x, x0, y0);
        w.z = corresponding_coordinate(dz_dx, w.x, x0, z0);
        w.x_to_go = g.voxel_width;
        w.y_to_go = distance_remaining(Y0, w.y, -1, yd, g.voxel_height, w.vy);
        w.z_to_go = distance_remaining(Z0, w.z, -1, zd, g.voxel_thickness, w.vz);
    } else {
        w.vy -= yd;
        w.y = edge_coordinate(Y0, w.vy, g.voxel_height, -1, yd);
        w.x = corresponding_coordinate(dx_dy, w.y, y0, x0);
        w.z = corresponding_coordinate(dz_dy, w.y, y0, z0);
        w.x_to_go = distance_remaining(X0, w.x, 1, xd, g.voxel_width, w.vx);
        w.y_to_go = g.voxel_height;
        w.z_to_go = distance_remaining(Z0, w.z, -1, zd, g.voxel_thickness, w.vz);
    }
    if (w.x_to_go == 0) {
        w.x_to_go = g.voxel_width;
        w.vx += xd;
    }
    if (w.y_to_go == 0) {
        w.y_to_go = g.voxel_height;
        w.vy -= yd;
    }
    if (w.z_to_go == 0) {
        w.z_to_go = g.voxel_thickness;
        w.vz -= zd;
    }
    w.vz = max(w.vz, 0);
    w.voxel = w.vx + w.vy * g.columns + w.vz * g.columns * g.rows;
}

// take_2D_step_GPU (B.cu:11346-11390)
__device__ void take_2D_step(const PreGeom& g, int xd, int yd, double dy_dx, double dx_dy, double x0, double y0, WalkState& w)
{
    const double X0 = -g.R, Y0 = g.R;
    const double y_extension = fabs(dx_dy) * w.y_to_go;
    if (w.x_to_go <= y_extension) {
        w.vx += xd;
        w.x = edge_coordinate(X0, w.vx, g.voxel_width, 1, xd);
        w.y = corresponding_coordinate(dy_dx, w.x, x0, y0);
        w.x_to_go = g.voxel_width;
        w.y_to_go = distance_remaining(Y0, w.y, -1, yd, g.voxel_height, w.vy);
    } else {
        w.vy -= yd;
        w.y = edge_coordinate(Y0, w.vy, g.voxel_height, -1, yd);
        w.x = corresponding_coordinate(dx_dy, w.y, y0, x0);
        w.x_to_go = distance_remaining(X0, w.x, 1, xd, g.voxel_width, w.vx);
        w.y_to_go = g.voxel_height;
    }
    if (w.x_to_go == 0) {
        w.x_to_go = g.voxel_width;
        w.vx += xd;
    }
    if (w.y_to_go == 0) {
        w.y_to_go = g.voxel_height;
        w.vy -= yd;
    }
    w.vz = max(w.vz, 0);
    w.voxel = w.vx + w.vy * g.columns + w.vz * g.columns * g.rows;
}

// Processing order of the voxel walks.  A history's walk lengths depend on where its line crosses
// the grid: its distance t from the z axis and its direction (the chord for the hull walk, the gap
// to the hull for the endpoint walks), and one thread walks one history, so neighbouring threads
// should have similar lines.  The key is t in kWalkT buckets of the cylinder radius, times the
// line's direction (mod pi) in dir_buckets buckets: measured on a 20M-proton head scan, direction
// buckets shorten the endpoint walks (38.2 -> 31.2 ms; t alone 33.8) but not the hull walks, which
// run entry to exit (23.0 -> 21.5 ms with t alone, 23.7 with 32 directions).  The order changes no
// result (integer counts, per-history endpoints).
constexpr int kWalkT = 32, kWalkDir = 32, kWalkKeys = kWalkT * kWalkDir;
__global__ void walk_order_key_kernel(long long n, const float* __restrict__ xe, const float* __restrict__ ye,
                                      const float* __restrict__ xo, const float* __restrict__ yo, float R,
                                      int dir_buckets, int* __restrict__ key)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float dx = xo[i] - xe[i], dy = yo[i] - ye[i];
    const float len = sqrtf(dx * dx + dy * dy);
    const float t = len > 0.f ? fabsf(xe[i] * yo[i] - xo[i] * ye[i]) / len : 0.f;
    int kt = (int)(t / R * kWalkT);
    kt = kt < 0 ? 0 : (kt >= kWalkT ? kWalkT - 1 : kt);
    float a = atan2f(dy, dx);
    if (a < 0.f) a += 3.14159265f;  // direction mod pi
    int ka = (int)(a / 3.14159265f * dir_buckets);
    ka = ka < 0 ? 0 : (ka >= dir_buckets ? dir_buckets - 1 : ka);
    key[i] = kt * dir_buckets + ka;
}

// SC_GPU / MSC_GPU / SM_GPU (B.cu:6681-7099) in one pass.  The three reference kernels walk the
// same straight line from the entry to the exit voxel and differ only in their WEPL window and in
// what they do at each voxel: SC carves (writes 0), MSC and SM count.  Here each history walks once
// and applies every hull whose window (and *_ON switch) it satisfies, so the voxel sequence each
// hull sees is the one its own kernel would walk.
__global__ void hull_walks_kernel(PreGeom g, long long n, const int* __restrict__ order, GeomPtrs G,
                                  const float* __restrict__ WEPL, const uint8_t* __restrict__ missed,
                                  uint8_t* __restrict__ sc_hull, int* __restrict__ msc_counts, int* __restrict__ sm_counts,
                                  unsigned long long* counters)
{
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const long long i = order[k];
    if (missed[i]) return;
    const float wepl = WEPL[i];
    const bool sc = sc_hull && (wepl <= g.sc_upper) && (wepl >= g.sc_lower);
    const bool msc = msc_counts && (wepl <= g.msc_upper) && (wepl >= g.msc_lower);
    const bool sm = sm_counts && (wepl >= g.sm_lower);
    if (!(sc || msc || sm)) return;
    const double X0 = -g.R, Y0 = g.R, Z0 = g.H / 2;
    const float xe = G.a[kXE][i], ye = G.a[kYE][i], ze = G.a[kZE][i], xo = G.a[kXO][i], yo = G.a[kYO][i], zo = G.a[kZO][i];
    const int xd = (xe <= xo) - (xe >= xo), yd = (ye <= yo) - (ye >= yo), zd = (ze <= zo) - (ze >= zo);
    WalkState w;
    w.x = xe;
    w.y = ye;
    w.z = ze;
    w.vx = calculate_voxel(X0, xe, g.voxel_width);
    w.vy = calculate_voxel(Y0, ye, g.voxel_height);
    w.vz = calculate_voxel(Z0, ze, g.voxel_thickness);
    w.voxel = w.vx + w.vy * g.columns + w.vz * g.columns * g.rows;
    w.x_to_go = distance_remaining(X0, w.x, 1, xd, g.voxel_width, w.vx);
    w.y_to_go = distance_remaining(Y0, w.y, -1, yd, g.voxel_height, w.vy);
    w.z_to_go = distance_remaining(Z0, w.z, -1, zd, g.voxel_thickness, w.vz);
    const double dy_dx = (double)__fdiv_rn(__fsub_rn(yo, ye), __fsub_rn(xo, xe));
    const double dz_dx = (double)__fdiv_rn(__fsub_rn(zo, ze), __fsub_rn(xo, xe));
    const double dz_dy = (double)__fdiv_rn(__fsub_rn(zo, ze), __fsub_rn(yo, ye));
    const double dx_dy = (double)__fdiv_rn(__fsub_rn(xo, xe), __fsub_rn(yo, ye));
    const double dx_dz = (double)__fdiv_rn(__fsub_rn(xo, xe), __fsub_rn(zo, ze));
    const double dy_dz = (double)__fdiv_rn(__fsub_rn(yo, ye), __fsub_rn(zo, ze));
    const int vx_out = calculate_voxel(X0, xo, g.voxel_width), vy_out = calculate_voxel(Y0, yo, g.voxel_height),
              vz_out = calculate_voxel(Z0, zo, g.voxel_thickness);
    const int voxel_out = vx_out + vy_out * g.columns + vz_out * g.columns * g.rows;
    auto outside = [&]() { return w.vx >= g.columns || w.vy >= g.rows || w.vz >= g.slices || w.vx < 0 || w.vy < 0 || w.vz < 0; };
    auto mark = [&]() {
        if (sc) sc_hull[w.voxel] = 0;
        if (msc) atomicAdd(msc_counts + w.voxel, 1);
        if (sm) atomicAdd(sm_counts + w.voxel, 1);
    };
    bool end_walk = (w.voxel == voxel_out) || outside();
    if (!end_walk) mark();
    const int max_steps = 4 * (g.columns + g.rows + g.slices) + 16;
    int steps = 0;
    while (!end_walk) {
        if (zd != 0) take_3D_step(g, xd, yd, zd, dy_dx, dz_dx, dz_dy, dx_dy, dx_dz, dy_dz, xe, ye, ze, w);
        else take_2D_step(g, xd, yd, dy_dx, dx_dy, xe, ye, w);
        end_walk = (w.voxel == voxel_out) || outside();
        if (!end_walk) mark();
        if (++steps > max_steps) {
            atomicAdd(counters + kCntWaitExpired, 1ull);
            break;
        }
    }
}

// MSC_edge_detection_GPU (B.cu:6911-6956), out of place: 3x3 maximum difference over the
// interior, threshold on the difference or the count, then the cylinder mask.
__global__ void msc_edge_kernel(PreGeom g, const int* __restrict__ counts, int* __restrict__ out)
{
    const long long voxel = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (voxel >= g.num_voxels) return;
    const long long CR = (long long)g.columns * g.rows;
    const int slice = (int)(voxel / CR), rem = (int)(voxel % CR), row = rem / g.columns, column = rem % g.columns;
    const float x = (float)((column - g.columns / 2 + 0.5) * g.voxel_width);
    const float y = (float)((g.rows / 2 - row - 0.5) * g.voxel_height);
    int max_difference = 0;
    if ((row != 0) && (row != g.rows - 1) && (column != 0) && (column != g.columns - 1)) {
        for (int r = row - 1; r <= row + 1; r++)
            for (int c = column - 1; c <= column + 1; c++) {
                const int difference = counts[voxel] - counts[c + r * g.columns + slice * CR];
                if (difference > max_difference) max_difference = difference;
            }
    }
    int result = (max_difference > g.msc_diff_thresh || counts[voxel] > g.msc_diff_thresh) ? 0 : 1;
    const double half = (g.voxel_width > g.voxel_height ? g.voxel_width : g.voxel_height) / 2;
    if (__fadd_rn(powf(x, 2.0f), powf(y, 2.0f)) >= powf((float)(g.R - half), 2.0f)) result = 0;
    out[voxel] = result;
}

// carve_differences (B.cu:6616-6634): interior 3x3 maximum difference
__global__ void carve_differences_kernel(PreGeom g, const int* __restrict__ image, int* __restrict__ diff)
{
    const long long voxel = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (voxel >= g.num_voxels) return;
    const long long CR = (long long)g.columns * g.rows;
    const int slice = (int)(voxel / CR), rem = (int)(voxel % CR), row = rem / g.columns, column = rem % g.columns;
    int max_difference = 0;
    if ((row != 0) && (row != g.rows - 1) && (column != 0) && (column != g.columns - 1)) {
        for (int r = row - 1; r <= row + 1; r++)
            for (int c = column - 1; c <= column + 1; c++) {
                const int difference = image[voxel] - image[c + r * g.columns + slice * CR];
                if (difference > max_difference) max_difference = difference;
            }
        diff[voxel] = max_difference;
    } else {
        diff[voxel] = 0;
    }
}

// SM_edge_detection's host threshold search (B.cu:7118-7133): per slice, the count at the first
// voxel (in index order) holding the slice's largest positive difference; 0 if none is positive.
// One 256-thread CTA per slice; the winner is the smallest index among maximal differences.
__global__ void sm_threshold_kernel(PreGeom g, const int* __restrict__ diff, const int* __restrict__ counts,
                                    int* __restrict__ thresholds)
{
    const int slice = blockIdx.x;
    const long long CR = (long long)g.columns * g.rows;
    const long long base = slice * CR;
    int best = 0;
    long long best_idx = -1;
    for (long long p = threadIdx.x; p < CR; p += blockDim.x) {
        const int d = diff[base + p];
        if (d > best) {  // within a thread indices increase, so the first maximum is kept
            best = d;
            best_idx = p;
        }
    }
    __shared__ int s_best[256];
    __shared__ long long s_idx[256];
    s_best[threadIdx.x] = best;
    s_idx[threadIdx.x] = best_idx;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            const int b2 = s_best[threadIdx.x + o];
            const long long i2 = s_idx[threadIdx.x + o];
            if (b2 > s_best[threadIdx.x] || (b2 == s_best[threadIdx.x] && b2 > 0 && i2 >= 0 &&
                                              (s_idx[threadIdx.x] < 0 || i2 < s_idx[threadIdx.x]))) {
                s_best[threadIdx.x] = b2;
                s_idx[threadIdx.x] = i2;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) thresholds[slice] = s_idx[0] >= 0 ? counts[base + s_idx[0]] : 0;
}

// SM_edge_detection_GPU (B.cu:7160-7175)
__global__ void sm_edge_kernel(PreGeom g, int* __restrict__ counts, const int* __restrict__ thresholds)
{
    const long long voxel = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (voxel >= g.num_voxels) return;
    const long long CR = (long long)g.columns * g.rows;
    const int slice = (int)(voxel / CR), rem = (int)(voxel % CR), row = rem / g.columns, column = rem % g.columns;
    const float x = (float)((column - g.columns / 2 + 0.5) * g.voxel_width);
    const float y = (float)((g.rows / 2 - row - 0.5) * g.voxel_height);
    int v = (counts[voxel] > g.sm_scale * thresholds[slice]) ? 1 : 0;
    const double half = (g.voxel_width > g.voxel_height ? g.voxel_width : g.voxel_height) / 2;
    if (__fadd_rn(powf(x, 2.0f), powf(y, 2.0f)) >= powf((float)(g.R - half), 2.0f)) v = 0;
    counts[voxel] = v;
}

__global__ void counts_to_hull_kernel(long long n, const int* __restrict__ counts, uint8_t* __restrict__ hull)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) hull[i] = counts[i] == 1 ? 1 : 0;
}

// initial_iterate_generate_hybrid (B.cu:8582-8591): x = FBP where the hull is set, else 0
__global__ void hybrid_kernel(long long n, const uint8_t* __restrict__ hull, const float* __restrict__ fbp, float* __restrict__ x)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] = hull[i] ? fbp[i] : 0.0f;
}

// find_MLP_endpoints_GPU (B.cu:7581-7773): walk from the cylinder point along the straight line
// (angle + PI when leaving) until the first hull voxel or the image edge.
__device__ bool find_endpoint(const PreGeom& g, const uint8_t* __restrict__ image, double x_start, double y_start,
                              double z_start, double xy_angle, double xz_angle, double& x_object, double& y_object,
                              double& z_object, int& voxel_x, int& voxel_y, int& voxel_z, bool entering)
{
    const double X0 = -g.R, Y0 = g.R, Z0 = g.H / 2;
    double x = x_start, y = y_start, z = z_start;
    bool hit_hull = false;
    if (!entering) xy_angle += kPi;
    int x_move_direction = (cos(xy_angle) >= 0) - (cos(xy_angle) <= 0);
    const int y_move_direction = (sin(xy_angle) >= 0) - (sin(xy_angle) <= 0);
    int z_move_direction = (sin(xz_angle) >= 0) - (sin(xz_angle) <= 0);
    if (x_move_direction < 0) z_move_direction *= -1;
    voxel_x = calculate_voxel(X0, x, g.voxel_width);
    voxel_y = calculate_voxel(Y0, y, g.voxel_height);
    voxel_z = calculate_voxel(Z0, z, g.voxel_thickness);
    double x_to_go = distance_remaining(X0, x, 1, x_move_direction, g.voxel_width, voxel_x);
    double y_to_go = distance_remaining(Y0, y, -1, y_move_direction, g.voxel_height, voxel_y);
    double z_to_go = distance_remaining(Z0, z, -1, z_move_direction, g.voxel_thickness, voxel_z);
    int voxel = voxel_x + (voxel_y + voxel_z * g.rows) * g.columns;
    const double delta_yx = fabs(tan(xy_angle));
    const double delta_zx = fabs(tan(xz_angle));
    const double delta_zy = fabs(tan(xz_angle) / tan(xy_angle));
    const double dy_dx = tan(xy_angle);
    const double dz_dx = tan(xz_angle);
    const double dz_dy = tan(xz_angle) / tan(xy_angle);
    const double dx_dy = powf((float)tan(xy_angle), -1.0f);
    const double dx_dz = powf((float)tan(xz_angle), -1.0f);
    const double dy_dz = tanf((float)xy_angle) / tan(xz_angle);
    auto outside = [&]() {
        return (voxel_x >= g.columns) || (voxel_y >= g.rows) || (voxel_z >= g.slices) || (voxel_x < 0) || (voxel_y < 0) || (voxel_z < 0);
    };
    bool outside_image = outside();
    if (!outside_image) hit_hull = (image[voxel] == 1);
    bool end_walk = outside_image || hit_hull;
    // every pass moves one index monotonically, so the walk leaves the grid within this bound
    const int max_steps = 2 * (g.columns + g.rows + g.slices) + 16;
    int steps = 0;
    if (z_move_direction != 0) {
        while (!end_walk && steps++ < max_steps) {
            const double x_extension = delta_zx * x_to_go;
            const double y_extension = delta_zy * y_to_go;
            if ((z_to_go <= x_extension) && (z_to_go <= y_extension)) {
                voxel_z -= z_move_direction;
                z = edge_coordinate(Z0, voxel_z, g.voxel_thickness, -1, z_move_direction);
                x = corresponding_coordinate(dx_dz, z, z_start, x_start);
                y = corresponding_coordinate(dy_dz, z, z_start, y_start);
                x_to_go = distance_remaining(X0, x, 1, x_move_direction, g.voxel_width, voxel_x);
                y_to_go = distance_remaining(Y0, y, -1, y_move_direction, g.voxel_height, voxel_y);
                z_to_go = g.voxel_thickness;
            } else if (x_extension <= y_extension) {
                voxel_x += x_move_direction;
                x = edge_coordinate(X0, voxel_x, g.voxel_width, 1, x_move_direction);
                y = corresponding_coordinate(dy_dx, x, x_start, y_start);
                z = corresponding_coordinate(dz_dx, x, x_start, z_start);
                x_to_go = g.voxel_width;
                y_to_go = distance_remaining(Y0, y, -1, y_move_direction, g.voxel_height, voxel_y);
                z_to_go = distance_remaining(Z0, z, -1, z_move_direction, g.voxel_thickness, voxel_z);
            } else {
                voxel_y -= y_move_direction;
                y = edge_coordinate(Y0, voxel_y, g.voxel_height, -1, y_move_direction);
                x = corresponding_coordinate(dx_dy, y, y_start, x_start);
                z = corresponding_coordinate(dz_dy, y, y_start, z_start);
                x_to_go = distance_remaining(X0, x, 1, x_move_direction, g.voxel_width, voxel_x);
                y_to_go = g.voxel_height;
                z_to_go = distance_remaining(Z0, z, -1, z_move_direction, g.voxel_thickness, voxel_z);
            }
            if (x_to_go == 0) {
                x_to_go = g.voxel_width;
                voxel_x += x_move_direction;
            }
            if (y_to_go == 0) {
                y_to_go = g.voxel_height;
                voxel_y -= y_move_direction;
            }
            if (z_to_go == 0) {
                z_to_go = g.voxel_thickness;
                voxel_z -= z_move_direction;
            }
            voxel_z = max(voxel_z, 0);
            voxel = voxel_x + voxel_y * g.columns + voxel_z * g.columns * g.rows;
            outside_image = outside();
            if (!outside_image) hit_hull = (image[voxel] == 1);
            end_walk = outside_image || hit_hull;
        }
    } else {
        while (!end_walk && steps++ < max_steps) {
            const double y_extension = y_to_go / delta_yx;
            if (x_to_go <= y_extension) {
                voxel_x += x_move_direction;
                x = edge_coordinate(X0, voxel_x, g.voxel_width, 1, x_move_direction);
                y = corresponding_coordinate(dy_dx, x, x_start, y_start);
                x_to_go = g.voxel_width;
                y_to_go = distance_remaining(Y0, y, -1, y_move_direction, g.voxel_height, voxel_y);
            } else {
                voxel_y -= y_move_direction;
                // the reference passes Z_INCREASING_DIRECTION here (B.cu:7736); it equals Y's
                y = edge_coordinate(Y0, voxel_y, g.voxel_height, -1, y_move_direction);
                x = corresponding_coordinate(dx_dy, y, y_start, x_start);
                x_to_go = distance_remaining(X0, x, 1, x_move_direction, g.voxel_width, voxel_x);
                y_to_go = g.voxel_height;
            }
            if (x_to_go == 0) {
                x_to_go = g.voxel_width;
                voxel_x += x_move_direction;
            }
            if (y_to_go == 0) {
                y_to_go = g.voxel_height;
                voxel_y -= y_move_direction;
            }
            voxel = voxel_x + voxel_y * g.columns + voxel_z * g.columns * g.rows;
            outside_image = outside();
            if (!outside_image) hit_hull = (image[voxel] == 1);
            end_walk = outside_image || hit_hull;
        }
    }
    if (hit_hull) {
        x_object = x;
        y_object = y;
        z_object = z;
    }
    return hit_hull;
}

// collect_MLP_endpoints_GPU_nobool (B.cu:7819-7854)
__global__ void endpoints_kernel(PreGeom g, long long n, const int* __restrict__ order, const uint8_t* __restrict__ hull,
                                 GeomPtrs G, uint32_t* __restrict__ first_voxel, int* __restrict__ keep)
{
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const long long i = order[k];
    int vx = 0, vy = 0, vz = 0, vx2 = 0, vy2 = 0, vz2 = 0;
    double xin = 0, yin = 0, zin = 0, xout = 0, yout = 0, zout = 0;
    const bool entered = find_endpoint(g, hull, G.a[kXE][i], G.a[kYE][i], G.a[kZE][i], G.a[kXYE][i], G.a[kXZE][i], xin,
                                       yin, zin, vx, vy, vz, true);
    const bool exited = find_endpoint(g, hull, G.a[kXO][i], G.a[kYO][i], G.a[kZO][i], G.a[kXYO][i], G.a[kXZO][i], xout,
                                      yout, zout, vx2, vy2, vz2, false);
    if (entered && exited) {
        first_voxel[i] = (uint32_t)(vx + g.columns * vy + g.rows * g.columns * vz);
        G.a[kXE][i] = (float)xin;
        G.a[kYE][i] = (float)yin;
        G.a[kZE][i] = (float)zin;
        G.a[kXO][i] = (float)xout;
        G.a[kYO][i] = (float)yout;
        G.a[kZO][i] = (float)zout;
        keep[i] = 1;
    } else {
        first_voxel[i] = (uint32_t)g.num_voxels;
        keep[i] = 0;
    }
}

// stable compaction of the history vectors: out[offsets[i]] = in[i] where keep[i]
struct CompactArrays {
    const float* in_f[kNumGeom + 1];
    float* out_f[kNumGeom + 1];
    const int* in_i[2];
    int* out_i[2];
    int nf, ni;
};
__global__ void compact_kernel(long long n, const int* __restrict__ keep, const long long* __restrict__ offsets, CompactArrays c)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !keep[i]) return;
    const long long o = offsets[i];
    for (int k = 0; k < c.nf; k++) c.out_f[k][o] = c.in_f[k][i];
    for (int k = 0; k < c.ni; k++) c.out_i[k][o] = c.in_i[k][i];
}

__global__ void u8_to_int_kernel(long long n, const uint8_t* __restrict__ in, int invert, int* __restrict__ out)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = invert ? !in[i] : in[i];
}

unsigned grid_for(long long n, int threads) { return (unsigned)((n + threads - 1) / threads); }

}  // namespace

}  // namespace pct

// ==========================================================================================
// C ABI
// ==========================================================================================

using pct::Preproc;

namespace {

pct_status fail(pct_ctx* ctx, pct_status st, const std::string& what, cudaError_t e = cudaSuccess)
{
    if (ctx) {
        ctx->last_error = what;
        if (e != cudaSuccess) ctx->last_error += " -> " + pct::cuda_error_string(e);
    }
    return st;
}

#define PRE_TRY(expr, what)                                             \
    do {                                                                \
        cudaError_t _e = (expr);                                        \
        if (_e != cudaSuccess) return fail(ctx, PCT_ERR_CUDA, what, _e); \
    } while (0)

template <class T>
cudaError_t alloc(T*& p, long long n)
{
    cudaFree(p);
    p = nullptr;
    return cudaMalloc(&p, sizeof(T) * (size_t)(n > 0 ? n : 1));
}

Preproc* pre_of(pct_ctx* ctx)
{
    if (!ctx->pre) ctx->pre = new Preproc();
    return ctx->pre;
}

pct::GeomPtrs geom_ptrs(float* const a[pct::kNumGeom])
{
    pct::GeomPtrs g;
    for (int k = 0; k < pct::kNumGeom; k++) g.a[k] = a[k];
    return g;
}

// bins and images, sized once per context
pct_status ensure_fixed(pct_ctx* ctx, Preproc* p)
{
    if (p->bin_counts) return PCT_OK;
    const long long nb = ctx->cfg.NUM_BINS, nv = ctx->cfg.NUM_VOXELS;
    cudaError_t e = alloc(p->bin_counts, nb);
    float** fb[] = {&p->mean_WEPL, &p->mean_rel_ut_angle, &p->mean_rel_uv_angle, &p->stddev_WEPL, &p->stddev_rel_ut_angle,
                    &p->stddev_rel_uv_angle, &p->sinogram, &p->sinogram_filtered};
    for (float** q : fb)
        if (e == cudaSuccess) e = alloc(*q, nb);
    if (e == cudaSuccess) e = alloc(p->FBP_image, nv);
    if (e == cudaSuccess) e = alloc(p->FBP_median, nv);
    if (e == cudaSuccess) e = alloc(p->FBP_hull, nv);
    if (e == cudaSuccess) e = alloc(p->SC_hull, nv);
    if (e == cudaSuccess) e = alloc(p->hull, nv);
    if (e == cudaSuccess) e = alloc(p->MSC_counts, nv);
    if (e == cudaSuccess) e = alloc(p->SM_counts, nv);
    if (e == cudaSuccess) e = alloc(p->SM_differences, nv);
    if (e == cudaSuccess) e = alloc(p->edge_tmp, nv);
    if (e == cudaSuccess) e = alloc(p->walk_hist, 2 * pct::kWalkKeys);
    if (e == cudaSuccess) e = alloc(p->SM_thresholds, ctx->cfg.SLICES);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(ctx, PCT_ERR_NOMEM, "preprocessing arrays", e);
    }
    return PCT_OK;
}

pct_status ensure_scratch(pct_ctx* ctx, Preproc* p, long long n)
{
    if (n <= p->cap_scratch) return PCT_OK;
    cudaError_t e = alloc(p->flags, n);
    if (e == cudaSuccess) e = alloc(p->offsets, n + 1);
    if (e == cudaSuccess) e = alloc(p->scan_tmp, pct::scan_tile_scratch_elems(n));
    for (int k = 0; k < pct::kNumGeom && e == cudaSuccess; k++) e = alloc(p->tmp_geom[k], n);
    if (e == cudaSuccess) e = alloc(p->tmp_wepl, n);
    if (e == cudaSuccess) e = alloc(p->tmp_bin_num, n);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(ctx, PCT_ERR_NOMEM, "compaction scratch", e);
    }
    p->cap_scratch = n;
    return PCT_OK;
}

// Walk order of n histories by the key above: keys in the compaction's int scratch, the order in
// the offsets array (both idle while the walks run).  Returns the order (device), or null if a
// launch failed.  Needs ensure_scratch(n).
int* walk_order(pct_ctx* ctx, Preproc* p, long long n, float* const geom[pct::kNumGeom], int dir_buckets)
{
    cudaStream_t s = ctx->stream;
    int* key = p->tmp_bin_num;
    int* order = reinterpret_cast<int*>(p->offsets);
    pct::walk_order_key_kernel<<<pct::grid_for(n, 256), 256, 0, s>>>(n, geom[pct::kXE], geom[pct::kYE], geom[pct::kXO],
                                                                     geom[pct::kYO], (float)ctx->cfg.RECON_CYL_RADIUS,
                                                                     dir_buckets, key);
    if (cudaGetLastError() != cudaSuccess) return nullptr;
    if (pct::bucket_sort_by_key(key, 0, n, pct::kWalkT * dir_buckets, p->walk_hist, order, s) != cudaSuccess)
        return nullptr;
    ctx->launches += 4;
    return order;
}

// Stable compaction of the current vectors by p->flags (1 = keep); returns the new length.
pct_status compact_vectors(pct_ctx* ctx, Preproc* p, long long n, long long* kept)
{
    cudaStream_t s = ctx->stream;
    PRE_TRY(pct::exclusive_scan_i32_to_i64(p->flags, n, p->offsets, p->scan_tmp, s), "compaction scan");
    long long total = 0;
    PRE_TRY(cudaMemcpyAsync(&total, p->offsets + n, sizeof(long long), cudaMemcpyDeviceToHost, s), "compaction count");
    pct::CompactArrays c{};
    int nf = 0;
    for (int k = 0; k < pct::kNumGeom; k++) {
        c.in_f[nf] = p->vec_geom[k];
        c.out_f[nf++] = p->tmp_geom[k];
    }
    c.in_f[nf] = p->vec_wepl;
    c.out_f[nf++] = p->tmp_wepl;
    c.nf = nf;
    c.in_i[0] = p->vec_bin_num;
    c.out_i[0] = p->tmp_bin_num;
    c.ni = 1;
    if (n > 0) pct::compact_kernel<<<pct::grid_for(n, 256), 256, 0, s>>>(n, p->flags, p->offsets, c);
    PRE_TRY(cudaGetLastError(), "compaction kernel");
    PRE_TRY(cudaStreamSynchronize(s), "compaction sync");
    for (int k = 0; k < pct::kNumGeom; k++) std::swap(p->vec_geom[k], p->tmp_geom[k]);
    std::swap(p->vec_wepl, p->tmp_wepl);
    std::swap(p->vec_bin_num, p->tmp_bin_num);
    p->n_vec = total;
    *kept = total;
    ctx->launches += 4;
    return PCT_OK;
}

}  // namespace

namespace pct {

// Device tracker arrays for n histories: dst[0..11] in the order of kTrackerNames, dst[12] WEPL,
// dst[13] the projection angle (degrees).  Grows the arrays when n exceeds their capacity.
pct_status preproc_reserve_tracker(pct_ctx* ctx, long long n, float* dst[kTrackerSlots])
{
    if (!ctx || n < 0 || n > 0x7fffffffLL) return PCT_ERR_ARG;
    cudaSetDevice(ctx->device);
    Preproc* p = pre_of(ctx);
    if (n > p->cap_raw) {
        cudaError_t e = cudaSuccess;
        for (int k = 0; k < kNumTracker && e == cudaSuccess; k++) e = alloc(p->tracker[k], n);
        for (int k = 0; k < kNumGeom && e == cudaSuccess; k++) e = alloc(p->raw_geom[k], n);
        if (e == cudaSuccess) e = alloc(p->gantry_angle, n);
        if (e == cudaSuccess) e = alloc(p->raw_wepl, n);
        if (e == cudaSuccess) e = alloc(p->missed, n);
        if (e == cudaSuccess) e = alloc(p->raw_bin_num, n);
        if (e != cudaSuccess) {
            cudaGetLastError();
            p->cap_raw = 0;
            return fail(ctx, PCT_ERR_NOMEM, "tracker arrays", e);
        }
        p->cap_raw = n;
    }
    for (int k = 0; k < kNumTracker; k++) dst[k] = p->tracker[k];
    dst[kNumTracker] = p->raw_wepl;
    dst[kNumTracker + 1] = p->gantry_angle;
    return PCT_OK;
}

const uint8_t* preproc_hull(pct_ctx* ctx)
{
    return (ctx && ctx->pre && ctx->pre->hull_ready) ? ctx->pre->hull : nullptr;
}

// The tracker arrays hold n histories: reset the stage state.
void preproc_tracker_loaded(pct_ctx* ctx, long long n, int integer_angles)
{
    Preproc* p = pre_of(ctx);
    p->n_raw = n;
    p->integer_angles = integer_angles ? 1 : 0;
    p->n_vec = 0;
    p->hull_ready = false;
}

}  // namespace pct

extern "C" pct_status pct_load_tracker_data(pct_ctx* ctx, const pct_tracker_data* t, int64_t n, pct_memory where,
                                            int integer_angles)
{
    if (!ctx || !t || n < 0 || n > 0x7fffffffLL) return PCT_ERR_ARG;
    const float* src[pct::kTrackerSlots] = {t->t_in_1,  t->t_in_2,  t->t_out_1, t->t_out_2, t->u_in_1,
                                            t->u_in_2,  t->u_out_1, t->u_out_2, t->v_in_1,  t->v_in_2,
                                            t->v_out_1, t->v_out_2, t->WEPL,    t->gantry_angle};
    if (n > 0)
        for (const float* q : src)
            if (!q) return fail(ctx, PCT_ERR_ARG, "pct_load_tracker_data: NULL array");
    float* dst[pct::kTrackerSlots];
    pct_status st = pct::preproc_reserve_tracker(ctx, n, dst);
    if (st != PCT_OK) return st;
    const cudaMemcpyKind kind = where == PCT_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    for (int k = 0; k < pct::kTrackerSlots && n > 0; k++)
        PRE_TRY(cudaMemcpyAsync(dst[k], src[k], sizeof(float) * n, kind, ctx->stream), "tracker copy");
    if (where == PCT_HOST) PRE_TRY(cudaStreamSynchronize(ctx->stream), "tracker sync");
    pct::preproc_tracker_loaded(ctx, n, integer_angles);
    return PCT_OK;
}

extern "C" pct_status pct_recon_volume_intersections(pct_ctx* ctx)
{
    if (!ctx || !ctx->pre) return PCT_ERR_STATE;
    Preproc* p = ctx->pre;
    cudaSetDevice(ctx->device);
    const pct::PreGeom g = pct::make_pregeom(ctx->cfg);
    pct::TrackerPtrs T;
    for (int k = 0; k < pct::kNumTracker; k++) T.a[k] = p->tracker[k];
    if (p->n_raw > 0)
        pct::intersections_kernel<<<pct::grid_for(p->n_raw, 256), 256, 0, ctx->stream>>>(
            g, p->n_raw, T, p->gantry_angle, p->integer_angles, geom_ptrs(p->raw_geom), p->missed);
    PRE_TRY(cudaGetLastError(), "intersections kernel");
    ctx->launches += 1;
    return PCT_OK;
}

extern "C" pct_status pct_binning(pct_ctx* ctx)
{
    if (!ctx || !ctx->pre) return PCT_ERR_STATE;
    Preproc* p = ctx->pre;
    cudaSetDevice(ctx->device);
    pct_status st = ensure_fixed(ctx, p);
    if (st != PCT_OK) return st;
    const long long n = p->n_raw, nb = ctx->cfg.NUM_BINS;
    cudaStream_t s = ctx->stream;
    PRE_TRY(cudaMemsetAsync(p->bin_counts, 0, sizeof(int) * nb, s), "bins clear");
    PRE_TRY(cudaMemsetAsync(p->mean_WEPL, 0, sizeof(float) * nb, s), "bins clear");
    PRE_TRY(cudaMemsetAsync(p->mean_rel_ut_angle, 0, sizeof(float) * nb, s), "bins clear");
    PRE_TRY(cudaMemsetAsync(p->mean_rel_uv_angle, 0, sizeof(float) * nb, s), "bins clear");
    PRE_TRY(cudaMemsetAsync(p->sinogram, 0, sizeof(float) * nb, s), "bins clear");
    const pct::PreGeom g = pct::make_pregeom(ctx->cfg);
    if (n > 0)
        pct::binning_kernel<<<pct::grid_for(n, 256), 256, 0, s>>>(g, n, geom_ptrs(p->raw_geom), p->raw_wepl, p->missed,
                                                                   p->raw_bin_num, p->bin_counts, p->mean_WEPL,
                                                                   p->mean_rel_ut_angle, p->mean_rel_uv_angle);
    PRE_TRY(cudaGetLastError(), "binning kernel");
    ctx->launches += 1;
    // the reference keeps histories that hit the volume with bin_num >= 0 (always, since bin_num
    // defaults to 0) in the history vectors, in order (B.cu:5429-5450)
    if (n > p->cap_vec) {
        cudaError_t e = cudaSuccess;
        for (int k = 0; k < pct::kNumGeom && e == cudaSuccess; k++) e = alloc(p->vec_geom[k], n);
        if (e == cudaSuccess) e = alloc(p->vec_wepl, n);
        if (e == cudaSuccess) e = alloc(p->vec_bin_num, n);
        if (e == cudaSuccess) e = alloc(p->vec_first_voxel, n);
        if (e != cudaSuccess) {
            cudaGetLastError();
            p->cap_vec = 0;
            return fail(ctx, PCT_ERR_NOMEM, "history vectors", e);
        }
        p->cap_vec = n;
    }
    st = ensure_scratch(ctx, p, n);
    if (st != PCT_OK) return st;
    for (int k = 0; k < pct::kNumGeom; k++)
        PRE_TRY(cudaMemcpyAsync(p->vec_geom[k], p->raw_geom[k], sizeof(float) * n, cudaMemcpyDeviceToDevice, s), "copy");
    PRE_TRY(cudaMemcpyAsync(p->vec_wepl, p->raw_wepl, sizeof(float) * n, cudaMemcpyDeviceToDevice, s), "copy");
    PRE_TRY(cudaMemcpyAsync(p->vec_bin_num, p->raw_bin_num, sizeof(int) * n, cudaMemcpyDeviceToDevice, s), "copy");
    if (n > 0) pct::u8_to_int_kernel<<<pct::grid_for(n, 256), 256, 0, s>>>(n, p->missed, 1, p->flags);
    PRE_TRY(cudaGetLastError(), "keep flags");
    long long kept = 0;
    return compact_vectors(ctx, p, n, &kept);
}

extern "C" pct_status pct_hull_detection(pct_ctx* ctx)
{
    if (!ctx || !ctx->pre) return PCT_ERR_STATE;
    Preproc* p = ctx->pre;
    cudaSetDevice(ctx->device);
    pct_status st = ensure_fixed(ctx, p);
    if (st != PCT_OK) return st;
    const pct::PreGeom g = pct::make_pregeom(ctx->cfg);
    const long long nv = ctx->cfg.NUM_VOXELS, n = p->n_raw;
    cudaStream_t s = ctx->stream;
    // hull_initializations / initialize_hull_GPU (B.cu:6636-6669)
    pct::init_hull_kernel<uint8_t><<<pct::grid_for(nv, 256), 256, 0, s>>>(g, p->SC_hull);
    pct::init_hull_kernel<int><<<pct::grid_for(nv, 256), 256, 0, s>>>(g, p->MSC_counts);
    pct::init_hull_kernel<int><<<pct::grid_for(nv, 256), 256, 0, s>>>(g, p->SM_counts);
    ctx->launches += 3;
    if (n > 0) {
        const pct::GeomPtrs G = geom_ptrs(p->raw_geom);
        if (ctx->cfg.SC_ON || ctx->cfg.MSC_ON || ctx->cfg.SM_ON) {
            st = ensure_scratch(ctx, p, n);
            if (st != PCT_OK) return st;
            int* order = walk_order(ctx, p, n, p->raw_geom, 1);
            if (!order) return fail(ctx, PCT_ERR_CUDA, "walk order", cudaGetLastError());
            pct::hull_walks_kernel<<<pct::grid_for(n, 128), 128, 0, s>>>(
                g, n, order, G, p->raw_wepl, p->missed, ctx->cfg.SC_ON ? p->SC_hull : nullptr,
                ctx->cfg.MSC_ON ? p->MSC_counts : nullptr, ctx->cfg.SM_ON ? p->SM_counts : nullptr, ctx->d_counters);
            ctx->launches += 1;
        }
    }
    PRE_TRY(cudaGetLastError(), "hull walk kernels");
    return PCT_OK;
}

extern "C" pct_status pct_calculate_means(pct_ctx* ctx)
{
    if (!ctx || !ctx->pre || !ctx->pre->bin_counts) return PCT_ERR_STATE;
    Preproc* p = ctx->pre;
    cudaSetDevice(ctx->device);
    const int nb = ctx->cfg.NUM_BINS;
    pct::means_kernel<<<pct::grid_for(nb, 256), 256, 0, ctx->stream>>>(nb, p->bin_counts, p->mean_WEPL, p->mean_rel_ut_angle,
                                                                     p->mean_rel_uv_angle);
    PRE_TRY(cudaGetLastError(), "means kernel");
    ctx->launches += 1;
    return PCT_OK;
}

extern "C" pct_status pct_sum_squared_deviations(pct_ctx* ctx)
{
    if (!ctx || !ctx->pre || !ctx->pre->bin_counts) return PCT_ERR_STATE;
    Preproc* p = ctx->pre;
    cudaSetDevice(ctx->device);
    const long long nb = ctx->cfg.NUM_BINS, n = p->n_vec;
    cudaStream_t s = ctx->stream;
    PRE_TRY(cudaMemsetAsync(p->stddev_WEPL, 0, sizeof(float) * nb, s), "clear");
    PRE_TRY(cudaMemsetAsync(p->stddev_rel_ut_angle, 0, sizeof(float) * nb, s), "clear");
    PRE_TRY(cudaMemsetAsync(p->stddev_rel_uv_angle, 0, sizeof(float) * nb, s), "clear");
    if (n > 0)
        pct::sum_sq_dev_kernel<<<pct::grid_for(n, 256), 256, 0, s>>>(n, p->vec_bin_num, p->vec_wepl, geom_ptrs(p->vec_geom),
                                                                     p->mean_WEPL, p->mean_rel_ut_angle, p->mean_rel_uv_angle,
                                                                     p->stddev_WEPL, p->stddev_rel_ut_angle, p->stddev_rel_uv_angle);
    PRE_TRY(cudaGetLastError(), "sum of squared deviations kernel");
    ctx->launches += 1;
    return PCT_OK;
}

extern "C" pct_status pct_calculate_standard_deviations(pct_ctx* ctx)
{
    if (!ctx || !ctx->pre || !ctx->pre->bin_counts) return PCT_ERR_STATE;
    Preproc* p = ctx->pre;
    cudaSetDevice(ctx->device);
    const int nb = ctx->cfg.NUM_BINS;
    pct::stddev_kernel<<<pct::grid_for(nb, 256), 256, 0, ctx->stream>>>(nb, ctx->cfg.SAMPLE_STD_DEV ? 1 : 0, p->bin_counts,
                                                                      p->stddev_WEPL, p->stddev_rel_ut_angle,
                                                                      p->stddev_rel_uv_angle);
    PRE_TRY(cudaGetLastError(), "standard deviations kernel");
    ctx->launches += 1;
    return PCT_OK;
}

extern "C" pct_status pct_statistical_cuts(pct_ctx* ctx)
{
    if (!ctx || !ctx->pre || !ctx->pre->bin_counts) return PCT_ERR_STATE;
    Preproc* p = ctx->pre;
    cudaSetDevice(ctx->device);
    const long long n = p->n_vec;
    cudaStream_t s = ctx->stream;
    PRE_TRY(cudaMemsetAsync(p->sinogram, 0, sizeof(float) * ctx->cfg.NUM_BINS, s), "sinogram clear");
    const pct::PreGeom g = pct::make_pregeom(ctx->cfg);
    if (n > 0)
        pct::cuts_kernel<<<pct::grid_for(n, 256), 256, 0, s>>>(g, n, p->vec_bin_num, p->vec_wepl, geom_ptrs(p->vec_geom),
                                                               p->mean_WEPL, p->mean_rel_ut_angle, p->mean_rel_uv_angle,
                                                               p->stddev_WEPL, p->stddev_rel_ut_angle, p->stddev_rel_uv_angle,
                                                               p->bin_counts, p->sinogram, p->flags);
    PRE_TRY(cudaGetLastError(), "cuts kernel");
    ctx->launches += 1;
    long long kept = 0;
    return compact_vectors(ctx, p, n, &kept);
}

extern "C" pct_status pct_construct_sinogram(pct_ctx* ctx)
{
    if (!ctx || !ctx->pre || !ctx->pre->bin_counts) return PCT_ERR_STATE;
    Preproc* p = ctx->pre;
    cudaSetDevice(ctx->device);
    const int nb = ctx->cfg.NUM_BINS;
    pct::sinogram_kernel<<<pct::grid_for(nb, 256), 256, 0, ctx->stream>>>(nb, p->bin_counts, p->sinogram);
    PRE_TRY(cudaGetLastError(), "sinogram kernel");
    ctx->launches += 1;
    return PCT_OK;
}

extern "C" pct_status pct_FBP(pct_ctx* ctx)
{
    if (!ctx || !ctx->pre || !ctx->pre->bin_counts) return PCT_ERR_STATE;
    Preproc* p = ctx->pre;
    cudaSetDevice(ctx->device);
    const pct::PreGeom g = pct::make_pregeom(ctx->cfg);
    const long long nb = ctx->cfg.NUM_BINS, nv = ctx->cfg.NUM_VOXELS;
    cudaStream_t s = ctx->stream;
    pct::filter_kernel<<<pct::grid_for(nb, 128), 128, 0, s>>>(g, p->sinogram, p->sinogram_filtered);
    pct::backprojection_kernel<<<pct::grid_for(nv, 128), 128, 0, s>>>(g, p->sinogram_filtered, p->FBP_image);
    ctx->launches += 2;
    const int r = ctx->cfg.FBP_MED_FILTER_RADIUS;
    if (ctx->cfg.MEDIAN_FILTER_FBP && r > 0) {
        if (r > 7) return fail(ctx, PCT_ERR_ARG, "FBP_MED_FILTER_RADIUS above 7 is not supported");
        pct::median_kernel<<<pct::grid_for(nv, 128), 128, 0, s>>>(g, r, p->FBP_image, p->FBP_median);
        ctx->launches += 1;
    } else {
        PRE_TRY(cudaMemcpyAsync(p->FBP_median, p->FBP_image, sizeof(float) * nv, cudaMemcpyDeviceToDevice, s), "copy");
    }
    // FBP_image_2_hull thresholds the unfiltered FBP image (B.cu:6163-6164, 6592)
    if (ctx->cfg.ENDPOINTS_HULL == PCT_FBP_HULL) {
        pct::fbp_hull_kernel<<<pct::grid_for(nv, 256), 256, 0, s>>>(g, p->FBP_image, p->FBP_hull);
        ctx->launches += 1;
    }
    PRE_TRY(cudaGetLastError(), "FBP kernels");
    return PCT_OK;
}

extern "C" pct_status pct_hull_detection_finish(pct_ctx* ctx)
{
    if (!ctx || !ctx->pre || !ctx->pre->bin_counts) return PCT_ERR_STATE;
    Preproc* p = ctx->pre;
    cudaSetDevice(ctx->device);
    const pct::PreGeom g = pct::make_pregeom(ctx->cfg);
    const long long nv = ctx->cfg.NUM_VOXELS;
    cudaStream_t s = ctx->stream;
    if (ctx->cfg.MSC_ON) {  // MSC_edge_detection (B.cu:6902), out of place
        pct::msc_edge_kernel<<<pct::grid_for(nv, 256), 256, 0, s>>>(g, p->MSC_counts, p->edge_tmp);
        PRE_TRY(cudaMemcpyAsync(p->MSC_counts, p->edge_tmp, sizeof(int) * nv, cudaMemcpyDeviceToDevice, s), "copy");
        ctx->launches += 1;
    }
    if (ctx->cfg.SM_ON) {  // SM_edge_detection (B.cu:7100)
        pct::carve_differences_kernel<<<pct::grid_for(nv, 256), 256, 0, s>>>(g, p->SM_counts, p->SM_differences);
        pct::sm_threshold_kernel<<<ctx->cfg.SLICES, 256, 0, s>>>(g, p->SM_differences, p->SM_counts, p->SM_thresholds);
        pct::sm_edge_kernel<<<pct::grid_for(nv, 256), 256, 0, s>>>(g, p->SM_counts, p->SM_thresholds);
        ctx->launches += 3;
    }
    PRE_TRY(cudaGetLastError(), "hull finish kernels");
    return PCT_OK;
}

extern "C" pct_status pct_hull_selection(pct_ctx* ctx)
{
    if (!ctx || !ctx->pre || !ctx->pre->bin_counts) return PCT_ERR_STATE;
    Preproc* p = ctx->pre;
    cudaSetDevice(ctx->device);
    const long long nv = ctx->cfg.NUM_VOXELS;
    cudaStream_t s = ctx->stream;
    switch (ctx->cfg.ENDPOINTS_HULL) {  // hull_selection (B.cu:7351-7393)
        case PCT_SC_HULL:
            PRE_TRY(cudaMemcpyAsync(p->hull, p->SC_hull, nv, cudaMemcpyDeviceToDevice, s), "hull copy");
            break;
        case PCT_MSC_HULL:
            pct::counts_to_hull_kernel<<<pct::grid_for(nv, 256), 256, 0, s>>>(nv, p->MSC_counts, p->hull);
            ctx->launches += 1;
            break;
        case PCT_SM_HULL:
            pct::counts_to_hull_kernel<<<pct::grid_for(nv, 256), 256, 0, s>>>(nv, p->SM_counts, p->hull);
            ctx->launches += 1;
            break;
        default:
            PRE_TRY(cudaMemcpyAsync(p->hull, p->FBP_hull, nv, cudaMemcpyDeviceToDevice, s), "hull copy");
    }
    PRE_TRY(cudaGetLastError(), "hull selection");
    p->hull_ready = true;
    return PCT_OK;
}

extern "C" pct_status pct_define_initial_iterate(pct_ctx* ctx)
{
    if (!ctx || !ctx->pre || !ctx->pre->hull_ready) return PCT_ERR_STATE;
    Preproc* p = ctx->pre;
    cudaSetDevice(ctx->device);
    const long long nv = ctx->cfg.NUM_VOXELS;
    pct::hybrid_kernel<<<pct::grid_for(nv, 256), 256, 0, ctx->stream>>>(nv, p->hull, p->FBP_median, ctx->d_x);
    PRE_TRY(cudaGetLastError(), "initial iterate");
    ctx->launches += 1;
    return PCT_OK;
}

extern "C" pct_status pct_reconstruction_cuts(pct_ctx* ctx)
{
    if (!ctx || !ctx->pre || !ctx->pre->hull_ready) return PCT_ERR_STATE;
    Preproc* p = ctx->pre;
    cudaSetDevice(ctx->device);
    const long long n = p->n_vec;
    cudaStream_t s = ctx->stream;
    const pct::PreGeom g = pct::make_pregeom(ctx->cfg);
    if (n > 0) {
        int* order = walk_order(ctx, p, n, p->vec_geom, pct::kWalkDir);
        if (!order) return fail(ctx, PCT_ERR_CUDA, "walk order", cudaGetLastError());
        pct::endpoints_kernel<<<pct::grid_for(n, 128), 128, 0, s>>>(g, n, order, p->hull, geom_ptrs(p->vec_geom),
                                                                    p->vec_first_voxel, p->flags);
    }
    PRE_TRY(cudaGetLastError(), "endpoints kernel");
    ctx->launches += 1;
    // keep histories whose entry and exit walks hit the hull, in order (B.cu:8286-8294); the first
    // MLP voxel is compacted by a second pass through the integer slot
    PRE_TRY(pct::exclusive_scan_i32_to_i64(p->flags, n, p->offsets, p->scan_tmp, s), "scan");
    long long total = 0;
    PRE_TRY(cudaMemcpyAsync(&total, p->offsets + n, sizeof(long long), cudaMemcpyDeviceToHost, s), "count");
    pct::CompactArrays c{};
    int nf = 0;
    for (int k = 0; k < pct::kNumGeom; k++) {
        c.in_f[nf] = p->vec_geom[k];
        c.out_f[nf++] = p->tmp_geom[k];
    }
    c.in_f[nf] = p->vec_wepl;
    c.out_f[nf++] = p->tmp_wepl;
    c.nf = nf;
    c.in_i[0] = reinterpret_cast<const int*>(p->vec_first_voxel);
    c.out_i[0] = p->tmp_bin_num;
    c.ni = 1;
    if (n > 0) pct::compact_kernel<<<pct::grid_for(n, 256), 256, 0, s>>>(n, p->flags, p->offsets, c);
    PRE_TRY(cudaGetLastError(), "compaction");
    PRE_TRY(cudaStreamSynchronize(s), "sync");
    ctx->launches += 4;
    for (int k = 0; k < pct::kNumGeom; k++) std::swap(p->vec_geom[k], p->tmp_geom[k]);
    std::swap(p->vec_wepl, p->tmp_wepl);
    PRE_TRY(cudaMemcpyAsync(p->vec_first_voxel, p->tmp_bin_num, sizeof(uint32_t) * total, cudaMemcpyDeviceToDevice, s), "copy");
    p->n_vec = total;
    // hand the reconstruction histories to the DROP stage (device to device)
    pct_histories h;
    h.x_entry = p->vec_geom[pct::kXE];
    h.y_entry = p->vec_geom[pct::kYE];
    h.z_entry = p->vec_geom[pct::kZE];
    h.x_exit = p->vec_geom[pct::kXO];
    h.y_exit = p->vec_geom[pct::kYO];
    h.z_exit = p->vec_geom[pct::kZO];
    h.xy_entry_angle = p->vec_geom[pct::kXYE];
    h.xz_entry_angle = p->vec_geom[pct::kXZE];
    h.xy_exit_angle = p->vec_geom[pct::kXYO];
    h.xz_exit_angle = p->vec_geom[pct::kXZO];
    h.WEPL = p->vec_wepl;
    h.first_MLP_voxel = p->vec_first_voxel;
    pct_status st = pct_set_reconstruction_histories(ctx, &h, total, PCT_DEVICE);
    // apply_history_sequence (B.cu:8691): the reconstruction order of the histories
    if (st == PCT_OK && ctx->cfg.RECON_HISTORY_ORDERING == PCT_PRIME_PERMUTATION)
        st = pct_apply_history_sequence(ctx, ctx->cfg.PRIME_OFFSET);
    return st;
}

extern "C" pct_status pct_set_history_vectors(pct_ctx* ctx, const pct_histories* h, int64_t n, pct_memory where)
{
    if (!ctx || !h || n < 0 || n > 0x7fffffffLL) return PCT_ERR_ARG;
    cudaSetDevice(ctx->device);
    Preproc* p = pre_of(ctx);
    pct_status st = ensure_fixed(ctx, p);
    if (st != PCT_OK) return st;
    if (n > p->cap_vec) {
        cudaError_t e = cudaSuccess;
        for (int k = 0; k < pct::kNumGeom && e == cudaSuccess; k++) e = alloc(p->vec_geom[k], n);
        if (e == cudaSuccess) e = alloc(p->vec_wepl, n);
        if (e == cudaSuccess) e = alloc(p->vec_bin_num, n);
        if (e == cudaSuccess) e = alloc(p->vec_first_voxel, n);
        if (e != cudaSuccess) {
            cudaGetLastError();
            p->cap_vec = 0;
            return fail(ctx, PCT_ERR_NOMEM, "history vectors", e);
        }
        p->cap_vec = n;
    }
    st = ensure_scratch(ctx, p, n);
    if (st != PCT_OK) return st;
    const float* src[pct::kNumGeom] = {h->x_entry, h->y_entry, h->z_entry, h->x_exit, h->y_exit, h->z_exit,
                                       h->xy_entry_angle, h->xz_entry_angle, h->xy_exit_angle, h->xz_exit_angle};
    const cudaMemcpyKind kind = where == PCT_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    for (int k = 0; k < pct::kNumGeom && n > 0; k++) {
        if (!src[k]) return PCT_ERR_ARG;
        PRE_TRY(cudaMemcpyAsync(p->vec_geom[k], src[k], sizeof(float) * n, kind, ctx->stream), "vector copy");
    }
    if (n > 0) {
        if (!h->WEPL) return PCT_ERR_ARG;
        PRE_TRY(cudaMemcpyAsync(p->vec_wepl, h->WEPL, sizeof(float) * n, kind, ctx->stream), "vector copy");
        PRE_TRY(cudaMemsetAsync(p->vec_bin_num, 0, sizeof(int) * n, ctx->stream), "vector clear");
    }
    PRE_TRY(cudaStreamSynchronize(ctx->stream), "vector sync");
    p->n_vec = n;
    return PCT_OK;
}

namespace {

// The stages of preprocessing() + the first half of image_reconstruction() (B.cu:7394,
// 10650-10660) after the tracker data is loaded.
pct_status preprocessing_stages(pct_ctx* ctx)
{
    pct_status st = pct_recon_volume_intersections(ctx);
    if (st == PCT_OK) st = pct_binning(ctx);
    if (st == PCT_OK) st = pct_hull_detection(ctx);
    if (st == PCT_OK) st = pct_hull_detection_finish(ctx);
    if (st == PCT_OK) st = pct_calculate_means(ctx);
    if (st == PCT_OK) st = pct_sum_squared_deviations(ctx);
    if (st == PCT_OK) st = pct_calculate_standard_deviations(ctx);
    if (st == PCT_OK) st = pct_statistical_cuts(ctx);
    if (st == PCT_OK) st = pct_construct_sinogram(ctx);
    if (st == PCT_OK) st = pct_FBP(ctx);
    if (st == PCT_OK) st = pct_hull_selection(ctx);
    if (st == PCT_OK) st = pct_define_initial_iterate(ctx);
    if (st == PCT_OK) st = pct_reconstruction_cuts(ctx);
    return st;
}

}  // namespace

extern "C" pct_status pct_preprocessing(pct_ctx* ctx, const pct_tracker_data* t, int64_t n, pct_memory where,
                                        int integer_angles)
{
    pct_status st = pct_load_tracker_data(ctx, t, n, where, integer_angles);
    return st == PCT_OK ? preprocessing_stages(ctx) : st;
}

extern "C" pct_status pct_preprocessing_from_files(pct_ctx* ctx, const char* directory)
{
    int64_t n = 0;
    pct_status st = pct_load_projection_data(ctx, directory, &n);
    return st == PCT_OK ? preprocessing_stages(ctx) : st;
}

// ---- named arrays ----
namespace {

struct NamedArray {
    void* ptr;
    size_t elem;
    long long count;
};

bool lookup(pct_ctx* ctx, const char* name, NamedArray& out)
{
    Preproc* p = ctx->pre;
    const long long nb = ctx->cfg.NUM_BINS, nv = ctx->cfg.NUM_VOXELS;
    std::string s(name);
    if (s == "x") {
        out = {ctx->d_x, 4, nv};
        return true;
    }
    // the reconstruction histories, in reconstruction order (the *_vector_reconstruction
    // vectors of apply_history_sequence, B.cu:8691)
    {
        pct::HistorySoA& h = ctx->hist;
        const struct {
            const char* n;
            void* ptr;
        } rec[] = {{"x_entry_reconstruction", h.x_entry}, {"y_entry_reconstruction", h.y_entry},
                   {"z_entry_reconstruction", h.z_entry}, {"x_exit_reconstruction", h.x_exit},
                   {"y_exit_reconstruction", h.y_exit}, {"z_exit_reconstruction", h.z_exit},
                   {"xy_entry_angle_reconstruction", h.xy_entry_angle},
                   {"xz_entry_angle_reconstruction", h.xz_entry_angle},
                   {"xy_exit_angle_reconstruction", h.xy_exit_angle},
                   {"xz_exit_angle_reconstruction", h.xz_exit_angle}, {"WEPL_reconstruction", h.WEPL},
                   {"first_MLP_voxel_reconstruction", h.first_MLP_voxel}};
        for (const auto& e : rec)
            if (s == e.n) {
                out = {e.ptr, 4, ctx->n_hist};
                return e.ptr != nullptr && ctx->n_hist > 0;
            }
    }
    if (!p) return false;
    for (int k = 0; k < pct::kNumTracker; k++)
        if (s == pct::kTrackerNames[k]) {
            out = {p->tracker[k], 4, p->n_raw};
            return true;
        }
    for (int k = 0; k < pct::kNumGeom; k++) {
        if (s == pct::kGeomNames[k]) {
            out = {p->raw_geom[k], 4, p->n_raw};
            return true;
        }
        if (s == std::string(pct::kGeomNames[k]) + "_vector") {
            out = {p->vec_geom[k], 4, p->n_vec};
            return true;
        }
    }
    const struct {
        const char* n;
        void* ptr;
        size_t elem;
        long long count;
    } table[] = {
        {"gantry_angle", p->gantry_angle, 4, p->n_raw},
        {"WEPL", p->raw_wepl, 4, p->n_raw},
        {"missed_recon_volume", p->missed, 1, p->n_raw},
        {"bin_num", p->raw_bin_num, 4, p->n_raw},
        {"WEPL_vector", p->vec_wepl, 4, p->n_vec},
        {"bin_num_vector", p->vec_bin_num, 4, p->n_vec},
        {"first_MLP_voxel_vector", p->vec_first_voxel, 4, p->n_vec},
        {"bin_counts", p->bin_counts, 4, nb},
        {"mean_WEPL", p->mean_WEPL, 4, nb},
        {"mean_rel_ut_angle", p->mean_rel_ut_angle, 4, nb},
        {"mean_rel_uv_angle", p->mean_rel_uv_angle, 4, nb},
        {"stddev_WEPL", p->stddev_WEPL, 4, nb},
        {"stddev_rel_ut_angle", p->stddev_rel_ut_angle, 4, nb},
        {"stddev_rel_uv_angle", p->stddev_rel_uv_angle, 4, nb},
        {"sinogram", p->sinogram, 4, nb},
        {"sinogram_filtered", p->sinogram_filtered, 4, nb},
        {"FBP_image", p->FBP_image, 4, nv},
        {"FBP_median_filtered", p->FBP_median, 4, nv},
        {"FBP_hull", p->FBP_hull, 1, nv},
        {"SC_hull", p->SC_hull, 1, nv},
        {"MSC_counts", p->MSC_counts, 4, nv},
        {"SM_counts", p->SM_counts, 4, nv},
        {"hull", p->hull, 1, nv},
    };
    for (const auto& e : table)
        if (s == e.n) {
            out = {e.ptr, e.elem, e.count};
            return e.ptr != nullptr;
        }
    return false;
}

}  // namespace

extern "C" int64_t pct_array_length(pct_ctx* ctx, const char* name)
{
    NamedArray a;
    if (!ctx || !name || !lookup(ctx, name, a)) return -1;
    return a.count;
}

extern "C" pct_status pct_get_array(pct_ctx* ctx, const char* name, void* dst, int64_t capacity_bytes, pct_memory where)
{
    NamedArray a;
    if (!ctx || !name || !dst) return PCT_ERR_ARG;
    if (!lookup(ctx, name, a)) return fail(ctx, PCT_ERR_ARG, std::string("unknown or unset array ") + name);
    const size_t bytes = a.elem * (size_t)a.count;
    if ((int64_t)bytes > capacity_bytes) return fail(ctx, PCT_ERR_ARG, std::string("buffer too small for ") + name);
    cudaSetDevice(ctx->device);
    if (bytes)
        PRE_TRY(cudaMemcpyAsync(dst, a.ptr, bytes, where == PCT_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice,
                                ctx->stream), "pct_get_array copy");
    PRE_TRY(cudaStreamSynchronize(ctx->stream), "pct_get_array sync");
    return PCT_OK;
}

extern "C" pct_status pct_set_array(pct_ctx* ctx, const char* name, const void* src, int64_t bytes, pct_memory where)
{
    NamedArray a;
    if (!ctx || !name || !src) return PCT_ERR_ARG;
    cudaSetDevice(ctx->device);
    if (ctx->pre) {
        pct_status st = ensure_fixed(ctx, ctx->pre);
        if (st != PCT_OK) return st;
    } else {
        pre_of(ctx);
        pct_status st = ensure_fixed(ctx, ctx->pre);
        if (st != PCT_OK) return st;
    }
    if (!lookup(ctx, name, a)) return fail(ctx, PCT_ERR_ARG, std::string("unknown or unset array ") + name);
    const std::string sn(name);
    if (sn.size() > 15 && sn.compare(sn.size() - 15, 15, "_reconstruction") == 0)
        return fail(ctx, PCT_ERR_ARG, sn + " is read-only: load histories with pct_set_reconstruction_histories");
    if ((size_t)bytes != a.elem * (size_t)a.count) return fail(ctx, PCT_ERR_ARG, std::string("size mismatch for ") + name);
    if (bytes)
        PRE_TRY(cudaMemcpyAsync(a.ptr, src, (size_t)bytes, where == PCT_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice,
                                ctx->stream), "pct_set_array copy");
    PRE_TRY(cudaStreamSynchronize(ctx->stream), "pct_set_array sync");
    if (std::string(name) == "hull") ctx->pre->hull_ready = true;
    return PCT_OK;
}
