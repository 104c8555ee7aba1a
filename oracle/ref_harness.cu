// ref_harness.cu -- runs the reference's own device code on inputs from files, to produce golden
// fixtures (TEST INFRASTRUCTURE ONLY).
//
// Linked with the reference's unmodified B.cu (src/pCT_Reconstruction_Data_Segments_Blake.cu),
// compiled for sm_100a with relocatable device code by oracle/build_reference.py.  B.cu's
// parameters are compile-time macros from B.h; each harness binary works at the configuration its
// B.cu object was compiled with: the reference's built-in one (B.h defaults: 256 x 256 x 32 voxels
// of 0.0625 x 0.0625 x 0.25 cm, RECON_CYL_RADIUS 8, MLP_U_STEP 0.03125, DROP_BLOCK_SIZE 204800,
// HISTORIES_PER_BLOCK 640, LAMBDA 1e-4, THREADS_PER_BLOCK 1024, ENDPOINTS_PER_BLOCK 320), or a
// grid set by a patched copy of B.h (the PCT_REF_* values below).
//
// Usage: ref_harness <command> <directory>
//   mlp            find_MLP_path_GPU_tabulated (B.cu:9104) per history
//   drop           one DROP iteration: per DROP block a kernel that does what
//                  calculate_x_update_GPU (B.cu:9321) does -- the reference's MLP and
//                  DROP_block_update_GPU (B.cu:9522) -- minus its device free() of a stack array,
//                  then the reference's image_update_GPU kernel (B.cu:9398)
//   time_drop      drop_params = [DROP_BLOCK_SIZE, iterations]: that many such iterations, each
//                  timed with CUDA events (out_ms.bin, float per iteration; out_x.bin the image)
//   scurve         the reference's five S-curve functions (sigmoid_GPU ... linear_over_root_GPU,
//                  B.cu:10606-10626) for k in [0, count), and s_curve_scale_GPU (B.cu:10627) on
//                  (j, n) pairs; scurve_params = [count], scurve_j / scurve_n the pairs
//   walks          the SC/MSC/SM hull walks (B.cu:6681-7099) through the reference's walk primitives
//                  (calculate_voxel_GPU, distance_remaining_GPU, take_2D/3D_step_GPU), with a step
//                  bound and a stop below index 0 that the reference's loops lack
//   tvs            calculate_total_variation and generate_perturbation_array (host code,
//                  B.cu:10163-10330) on an image
//   endpoints      the reference's collect_MLP_endpoints_GPU_nobool kernel (B.cu:7819)
//   intersections  the reference's recon_volume_intersections_GPU kernel (B.cu:4890)
//   binning        the reference's binning_GPU kernel (B.cu:5482)
//   stats_fbp      the reference's calculate_means_GPU, sum_squared_deviations_GPU,
//                  calculate_standard_deviations_GPU, statistical_cuts_GPU, construct_sinogram_GPU,
//                  filter_GPU and backprojection_GPU2 kernels in the order statistical_calculations_
//                  and_cuts / construct_sinogram / FBP launch them (B.cu:5608-6479), on binned
//                  history vectors and bin sums, then FBP()'s median_filter_2D (host, radius 3) and
//                  FBP_image_2_hull_GPU (on the unfiltered image, as FBP_image_2_hull does); every
//                  intermediate is written out
//   fbp            the same construct_sinogram ... median filter stages alone, on stored bin_counts
//                  (after the cuts) and sinogram_sums
//   edges          MSC_edge_detection_GPU (the out-of-place variant) and SM_edge_detection's
//                  carve_differences + SM_edge_detection_GPU, with the per-slice SM thresholds taken
//                  from the counts as the host loop of B.cu:7118-7133 is written, on a counts image
// Inputs are <directory>/<name>.bin raw arrays; outputs are written as <directory>/out_<name>.bin.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <string>
#include <vector>

// --- reference symbols (defined in B.cu / B.h) ---
extern double *sin_table_d, *cos_table_d, *scattering_table_d, *poly_1_2_d, *poly_2_3_d, *poly_3_4_d, *poly_2_6_d,
    *poly_3_12_d;
extern float LAMBDA;
void generate_trig_tables();
void generate_scattering_coefficient_table();
void generate_polynomial_tables();
void MLP_lookup_table_2_GPU();
__device__ void find_MLP_path_GPU_tabulated(float* x, double b_i, unsigned int first_MLP_voxel_number, double x_in_object,
                                            double y_in_object, double z_in_object, double x_out_object,
                                            double y_out_object, double z_out_object, double xy_entry_angle,
                                            double xz_entry_angle, double xy_exit_angle, double xz_exit_angle,
                                            double lambda, unsigned int* path, int& number_of_intersections,
                                            double& effective_chord_length, double& a_i_dot_x_k_partially,
                                            double& a_i_dot_a_i_partially, double* sin_table, double* cos_table,
                                            double* scattering_table, double* poly_1_2, double* poly_2_3,
                                            double* poly_3_4, double* poly_2_6, double* poly_3_12);
__device__ void DROP_block_update_GPU(int proton_id, int number_of_intersections, unsigned int* a_i, unsigned int* S,
                                      float* x_update, float* WEPL, double a_i_dot_x_k, double a_i_dot_a_i,
                                      double lambda, double effective_chord_length);
__global__ void image_update_GPU(float* x, float* x_update, unsigned int* S);
// S-curve attenuation (B.cu:10606-10649); UINT is unsigned int (B.h:82)
__device__ float sigmoid_GPU(unsigned int);
__device__ float tanh_GPU(unsigned int);
__device__ float atan_GPU(unsigned int);
__device__ float erf_GPU(unsigned int);
__device__ float linear_over_root_GPU(unsigned int);
__device__ float s_curve_scale_GPU(unsigned int, unsigned int);
__global__ void collect_MLP_endpoints_GPU_nobool(unsigned int* first_MLP_voxel, bool* hull, float* x_entry,
                                                 float* y_entry, float* z_entry, float* xy_entry_angle,
                                                 float* xz_entry_angle, float* x_exit, float* y_exit, float* z_exit,
                                                 float* xy_exit_angle, float* xz_exit_angle, int start_proton_id,
                                                 int num_histories);
__global__ void recon_volume_intersections_GPU(int num_histories, int* gantry_angle, bool* missed_recon_volume,
                                               float* t_in_1, float* t_in_2, float* t_out_1, float* t_out_2,
                                               float* u_in_1, float* u_in_2, float* u_out_1, float* u_out_2,
                                               float* v_in_1, float* v_in_2, float* v_out_1, float* v_out_2,
                                               float* x_entry, float* y_entry, float* z_entry, float* x_exit,
                                               float* y_exit, float* z_exit, float* xy_entry_angle,
                                               float* xz_entry_angle, float* xy_exit_angle, float* xz_exit_angle);
__global__ void binning_GPU(int num_histories, int* bin_counts, int* bin_num, bool* missed_recon_volume,
                            float* x_entry, float* y_entry, float* z_entry, float* x_exit, float* y_exit,
                            float* z_exit, float* mean_WEPL, float* mean_rel_ut_angle, float* mean_rel_uv_angle,
                            float* WEPL, float* xy_entry_angle, float* xz_entry_angle, float* xy_exit_angle,
                            float* xz_exit_angle);

__global__ void calculate_means_GPU(int* bin_counts, float* mean_WEPL, float* mean_rel_ut_angle, float* mean_rel_uv_angle);
__global__ void sum_squared_deviations_GPU(int num_histories, int* bin_num, float* mean_WEPL, float* mean_rel_ut_angle,
                                           float* mean_rel_uv_angle, float* WEPL, float* xy_entry_angle,
                                           float* xz_entry_angle, float* xy_exit_angle, float* xz_exit_angle,
                                           float* stddev_WEPL, float* stddev_rel_ut_angle, float* stddev_rel_uv_angle);
__global__ void calculate_standard_deviations_GPU(int* bin_counts, float* stddev_WEPL, float* stddev_rel_ut_angle,
                                                  float* stddev_rel_uv_angle);
__global__ void statistical_cuts_GPU(int num_histories, int* bin_counts, int* bin_num, float* sinogram, float* WEPL,
                                     float* xy_entry_angle, float* xz_entry_angle, float* xy_exit_angle,
                                     float* xz_exit_angle, float* mean_WEPL, float* mean_rel_ut_angle,
                                     float* mean_rel_uv_angle, float* stddev_WEPL, float* stddev_rel_ut_angle,
                                     float* stddev_rel_uv_angle, bool* failed_cuts);
__global__ void construct_sinogram_GPU(int* bin_counts, float* sinogram);
__global__ void filter_GPU(float* sinogram, float* sinogram_filtered);
__global__ void backprojection_GPU2(float* sinogram_filtered, float* FBP_image);
__global__ void FBP_image_2_hull_GPU(float* FBP_image, bool* FBP_hull);
__global__ void MSC_edge_detection_GPU(int* MSC_counts, int* MSC_counts_output);
__global__ void carve_differences(int* carve_differences, int* image);
__global__ void SM_edge_detection_GPU(int* SM_counts, int* SM_threshold);
template <typename T>
void median_filter_2D(T*& input_image, T*& median_filtered_image, unsigned int radius);
// total variation superiorization, host code (B.cu:10163-10430)
template <typename T>
float calculate_total_variation(T* image, bool print_TV);
template <typename T>
void generate_perturbation_array(T* image);
void allocate_perturbation_arrays(bool parallel);
extern float *G_x_h, *G_y_h, *G_norm_h, *G_h, *v_h, *y_h;
// straight-line voxel-walk primitives (B.cu:11091-11462)
__device__ int calculate_voxel_GPU(double zero_coordinate, double current_position, double voxel_size);
__device__ double distance_remaining_GPU(double zero_coordinate, double current_position, int increasing_direction,
                                         int step_direction, double voxel_size, int current_voxel);
__device__ void take_2D_step_GPU(const int x_move_direction, const int y_move_direction, const int z_move_direction,
                                 const double dy_dx, const double dz_dx, const double dz_dy, const double dx_dy,
                                 const double dx_dz, const double dy_dz, const double x_start, const double y_start,
                                 const double z_start, double& x, double& y, double& z, int& voxel_x, int& voxel_y,
                                 int& voxel_z, int& voxel, double& x_to_go, double& y_to_go, double& z_to_go);
__device__ void take_3D_step_GPU(const int x_move_direction, const int y_move_direction, const int z_move_direction,
                                 const double dy_dx, const double dz_dx, const double dz_dy, const double dx_dy,
                                 const double dx_dz, const double dy_dz, const double x_start, const double y_start,
                                 const double z_start, double& x, double& y, double& z, int& voxel_x, int& voxel_y,
                                 int& voxel_z, int& voxel, double& x_to_go, double& y_to_go, double& z_to_go);

// --- the configuration B.cu was compiled with (B.h:333-423) ---
// oracle/build_reference.py builds one harness per configuration: the reference's built-in B.h
// values (the defaults below), and patched copies of B.h for other grids, passing the same values
// here with -D so that the harness's arrays and launches match the macros B.cu was compiled with.
#ifndef PCT_REF_COLUMNS
#define PCT_REF_COLUMNS 256
#define PCT_REF_ROWS 256
#define PCT_REF_SLICES 32
#define PCT_REF_HISTORIES_PER_BLOCK 640
#define PCT_REF_RADIUS 8.0
#define PCT_REF_HEIGHT 8.0
#define PCT_REF_VOXEL_WIDTH 0.0625
#define PCT_REF_VOXEL_HEIGHT 0.0625
#define PCT_REF_VOXEL_THICKNESS 0.25
#endif
constexpr int kColumns = PCT_REF_COLUMNS, kRows = PCT_REF_ROWS, kSlices = PCT_REF_SLICES;
constexpr long long kVoxels = (long long)kColumns * kRows * kSlices;
constexpr long long kPadded = kVoxels + kColumns * kRows;  // spare slice: MLP z may index SLICES
constexpr int kMaxIntersections = 1280;                     // MAX_INTERSECTIONS
constexpr int kMinMlpLength = 30;                           // MIN_MLP_LENGTH
constexpr int kHistoriesPerBlock = PCT_REF_HISTORIES_PER_BLOCK;  // HISTORIES_PER_BLOCK
// X/Y/Z_ZERO_COORDINATE (-R, +R, RECON_CYL_HEIGHT/2) and X/Y/Z_INCREASING_DIRECTION (RIGHT = 1,
// DOWN = -1, DOWN), B.h:846-921
constexpr double kXZero = -PCT_REF_RADIUS, kYZero = PCT_REF_RADIUS, kZZero = PCT_REF_HEIGHT / 2;
constexpr int kXInc = 1, kYInc = -1, kZInc = -1;
constexpr double kVoxelWidth = PCT_REF_VOXEL_WIDTH, kVoxelHeight = PCT_REF_VOXEL_HEIGHT,
                 kVoxelThickness = PCT_REF_VOXEL_THICKNESS;
constexpr int kTBins = 560, kVBins = 36, kAngularBins = 120;  // T_BINS, V_BINS, ANGULAR_BINS
constexpr int kNumBins = kTBins * kVBins * kAngularBins;

#define CK(x)                                                                                  \
    do {                                                                                       \
        cudaError_t e_ = (x);                                                                  \
        if (e_ != cudaSuccess) {                                                               \
            fprintf(stderr, "%s:%d %s: %s\n", __FILE__, __LINE__, #x, cudaGetErrorString(e_)); \
            exit(2);                                                                           \
        }                                                                                      \
    } while (0)

static std::string g_dir;

template <class T>
std::vector<T> load(const char* name)
{
    std::string p = g_dir + "/" + name + ".bin";
    FILE* f = fopen(p.c_str(), "rb");
    if (!f) {
        fprintf(stderr, "missing %s\n", p.c_str());
        exit(3);
    }
    fseek(f, 0, SEEK_END);
    long b = ftell(f);
    fseek(f, 0, SEEK_SET);
    std::vector<T> v(b / sizeof(T));
    if (b && fread(v.data(), 1, b, f) != (size_t)b) exit(3);
    fclose(f);
    return v;
}

template <class T>
void save(const char* name, const T* d, size_t count)
{
    std::string p = g_dir + "/out_" + name + ".bin";
    FILE* f = fopen(p.c_str(), "wb");
    if (!f || fwrite(d, sizeof(T), count, f) != count) exit(4);
    fclose(f);
}

template <class T>
T* upload(const std::vector<T>& v, size_t pad_elems = 0)
{
    T* d = nullptr;
    CK(cudaMalloc(&d, sizeof(T) * (v.size() + pad_elems + 1)));
    CK(cudaMemset(d, 0, sizeof(T) * (v.size() + pad_elems + 1)));
    if (!v.empty()) CK(cudaMemcpy(d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
    return d;
}

template <class T>
std::vector<T> download(const T* d, size_t n)
{
    std::vector<T> v(n);
    if (n) CK(cudaMemcpy(v.data(), d, sizeof(T) * n, cudaMemcpyDeviceToHost));
    return v;
}

struct Hist {
    int n;
    float *x_entry, *y_entry, *z_entry, *x_exit, *y_exit, *z_exit, *xy_entry_angle, *xz_entry_angle, *xy_exit_angle,
        *xz_exit_angle, *WEPL;
    unsigned* first_MLP_voxel;
};

static Hist load_hist()
{
    Hist h;
    auto xe = load<float>("x_entry");
    h.n = (int)xe.size();
    h.x_entry = upload(xe);
    h.y_entry = upload(load<float>("y_entry"));
    h.z_entry = upload(load<float>("z_entry"));
    h.x_exit = upload(load<float>("x_exit"));
    h.y_exit = upload(load<float>("y_exit"));
    h.z_exit = upload(load<float>("z_exit"));
    h.xy_entry_angle = upload(load<float>("xy_entry_angle"));
    h.xz_entry_angle = upload(load<float>("xz_entry_angle"));
    h.xy_exit_angle = upload(load<float>("xy_exit_angle"));
    h.xz_exit_angle = upload(load<float>("xz_exit_angle"));
    h.WEPL = upload(load<float>("WEPL"));
    h.first_MLP_voxel = upload(load<unsigned>("first_MLP_voxel"));
    return h;
}

struct TablePtrs {
    double *sin_t, *cos_t, *scat, *p12, *p23, *p34, *p26, *p312;
};

static TablePtrs setup_tables()
{
    generate_trig_tables();
    generate_scattering_coefficient_table();
    generate_polynomial_tables();
    MLP_lookup_table_2_GPU();
    CK(cudaDeviceSynchronize());
    return {sin_table_d, cos_table_d, scattering_table_d, poly_1_2_d, poly_2_3_d, poly_3_4_d, poly_2_6_d, poly_3_12_d};
}

__global__ void harness_mlp_kernel(Hist h, float* x, double lambda, TablePtrs t, int stride, unsigned* counts,
                                   unsigned* voxels, double* chord, double* adx)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= h.n) return;
    unsigned int path[kMaxIntersections];
    int n = 0;
    double L = 0, axk = 0, aia = 0;
    find_MLP_path_GPU_tabulated(x, h.WEPL[i], h.first_MLP_voxel[i], h.x_entry[i], h.y_entry[i], h.z_entry[i],
                                h.x_exit[i], h.y_exit[i], h.z_exit[i], h.xy_entry_angle[i], h.xz_entry_angle[i],
                                h.xy_exit_angle[i], h.xz_exit_angle[i], lambda, path, n, L, axk, aia, t.sin_t, t.cos_t,
                                t.scat, t.p12, t.p23, t.p34, t.p26, t.p312);
    counts[i] = (unsigned)n;
    for (int j = 0; j < n && j < stride; j++) voxels[(long long)i * stride + j] = path[j];
    chord[i] = L;
    adx[i] = axk;
}

// The body of calculate_x_update_GPU (B.cu:9321-9380) with HISTORIES_PER_THREAD = 1, using the
// reference's own device functions, without the device free() of its stack array.
// The histories it covers are those of calculate_x_update_GPU<<<num_blocks, 640>>>: start_proton_id
// + [0, num_blocks*640), bounded by the history count; they are spread over 128-thread CTAs because
// the relocatable build of the reference's MLP function needs more registers than a 640-thread CTA
// can hold.
__global__ void harness_x_update_kernel(Hist h, float* x, float* x_update, unsigned* S, int start_proton_id,
                                        int covered, double lambda, TablePtrs t)
{
    const int k = threadIdx.x + blockIdx.x * blockDim.x;
    if (k >= covered) return;
    const int proton_id = start_proton_id + k;
    if (proton_id >= h.n) return;
    unsigned int a_i[kMaxIntersections];
    int number_of_intersections = 0;
    double a_i_dot_a_i = 0.0, a_i_dot_x_k = 0.0, effective_chord_length = 0.0;
    find_MLP_path_GPU_tabulated(x, h.WEPL[proton_id], h.first_MLP_voxel[proton_id], h.x_entry[proton_id],
                                h.y_entry[proton_id], h.z_entry[proton_id], h.x_exit[proton_id], h.y_exit[proton_id],
                                h.z_exit[proton_id], h.xy_entry_angle[proton_id], h.xz_entry_angle[proton_id],
                                h.xy_exit_angle[proton_id], h.xz_exit_angle[proton_id], lambda, a_i,
                                number_of_intersections, effective_chord_length, a_i_dot_x_k, a_i_dot_a_i, t.sin_t,
                                t.cos_t, t.scat, t.p12, t.p23, t.p34, t.p26, t.p312);
    a_i_dot_a_i *= number_of_intersections;
    a_i_dot_x_k *= effective_chord_length;
    if (number_of_intersections >= kMinMlpLength)
        DROP_block_update_GPU(proton_id, number_of_intersections, a_i, S, x_update, h.WEPL, a_i_dot_x_k, a_i_dot_a_i,
                              lambda, effective_chord_length);
}

// One thread per k: the five curves in the S_CURVES order (SIGMOID, TANH, ATAN, ERF,
// LIN_OVER_ROOT, B.h:125), then one thread per (j, n) pair for s_curve_scale_GPU.
__global__ void harness_s_curve_kernel(int count, float* curves, int pairs, const unsigned* j, const unsigned* n,
                                       float* scale)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) {
        const unsigned k = (unsigned)i;
        curves[i] = sigmoid_GPU(k);
        curves[count + i] = tanh_GPU(k);
        curves[2 * count + i] = atan_GPU(k);
        curves[3 * count + i] = erf_GPU(k);
        curves[4 * count + i] = linear_over_root_GPU(k);
    }
    if (i < pairs) scale[i] = s_curve_scale_GPU(j[i], n[i]);
}

static int cmd_scurve()
{
    const int count = load<int>("scurve_params").at(0);
    auto jv = load<unsigned>("scurve_j");
    auto nv = load<unsigned>("scurve_n");
    if (count <= 0 || jv.size() != nv.size()) {
        fprintf(stderr, "scurve: bad parameters\n");
        return 3;
    }
    const int pairs = (int)jv.size();
    float *curves, *scale;
    CK(cudaMalloc(&curves, sizeof(float) * 5 * (size_t)count));
    CK(cudaMalloc(&scale, sizeof(float) * (size_t)(pairs > 0 ? pairs : 1)));
    unsigned* dj = upload(jv);
    unsigned* dn = upload(nv);
    const int threads = 128, work = count > pairs ? count : pairs;
    harness_s_curve_kernel<<<(work + threads - 1) / threads, threads>>>(count, curves, pairs, dj, dn, scale);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    auto c = download(curves, 5 * (size_t)count);
    auto sc = download(scale, (size_t)pairs);
    save("curves", c.data(), c.size());
    save("scale", sc.data(), sc.size());
    return 0;
}

static int cmd_mlp()
{
    Hist h = load_hist();
    TablePtrs t = setup_tables();
    float* x = upload(load<float>("x"), kPadded - kVoxels);
    const int stride = kMaxIntersections;
    unsigned *counts, *voxels;
    double *chord, *adx;
    CK(cudaMalloc(&counts, sizeof(unsigned) * h.n));
    CK(cudaMalloc(&voxels, sizeof(unsigned) * (size_t)h.n * stride));
    CK(cudaMalloc(&chord, sizeof(double) * h.n));
    CK(cudaMalloc(&adx, sizeof(double) * h.n));
    harness_mlp_kernel<<<(h.n + 127) / 128, 128>>>(h, x, (double)LAMBDA, t, stride, counts, voxels, chord, adx);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    auto c = download(counts, h.n);
    auto v = download(voxels, (size_t)h.n * stride);
    std::vector<unsigned> csr;
    for (int i = 0; i < h.n; i++)
        for (unsigned j = 0; j < c[i] && j < (unsigned)stride; j++) csr.push_back(v[(size_t)i * stride + j]);
    save("counts", c.data(), c.size());
    save("voxels", csr.data(), csr.size());
    auto L = download(chord, h.n);
    auto a = download(adx, h.n);
    save("chord", L.data(), L.size());
    save("a_dot_x", a.data(), a.size());
    return 0;
}

static int cmd_drop()
{
    Hist h = load_hist();
    TablePtrs t = setup_tables();
    auto params = load<int>("drop_params");  // [DROP_BLOCK_SIZE]
    const int block_size = params.at(0);
    float* x = upload(load<float>("x"), kPadded - kVoxels);
    float* x_update;
    unsigned* S;
    CK(cudaMalloc(&x_update, sizeof(float) * kPadded));
    CK(cudaMalloc(&S, sizeof(unsigned) * kPadded));
    CK(cudaMemset(x_update, 0, sizeof(float) * kPadded));
    CK(cudaMemset(S, 0, sizeof(unsigned) * kPadded));
    // DROP_full_tx_iteration (B.cu:9537-9582)
    int remaining = h.n, start = 0;
    while (remaining > 0) {
        const int hp = remaining > block_size ? block_size : remaining;
        const int covered = (hp / kHistoriesPerBlock) * kHistoriesPerBlock;
        if (covered > 0)
            harness_x_update_kernel<<<(covered + 127) / 128, 128>>>(h, x, x_update, S, start, covered, (double)LAMBDA, t);
        CK(cudaGetLastError());
        image_update_GPU<<<dim3(kColumns, kRows), dim3(kSlices)>>>(x, x_update, S);
        CK(cudaGetLastError());
        remaining -= block_size;
        start += block_size;
    }
    CK(cudaDeviceSynchronize());
    auto out = download(x, kVoxels);
    save("x", out.data(), out.size());
    return 0;
}

// One DROP iteration of the reference's device code over all histories (DROP_full_tx_iteration
// B.cu:9537-9582 with the harness's x-update kernel).
static void drop_iteration(const Hist& h, const TablePtrs& t, float* x, float* x_update, unsigned* S, int block_size)
{
    int remaining = h.n, start = 0;
    while (remaining > 0) {
        const int hp = remaining > block_size ? block_size : remaining;
        const int covered = (hp / kHistoriesPerBlock) * kHistoriesPerBlock;
        if (covered > 0)
            harness_x_update_kernel<<<(covered + 127) / 128, 128>>>(h, x, x_update, S, start, covered, (double)LAMBDA, t);
        CK(cudaGetLastError());
        image_update_GPU<<<dim3(kColumns, kRows), dim3(kSlices)>>>(x, x_update, S);
        CK(cudaGetLastError());
        remaining -= block_size;
        start += block_size;
    }
}

static int cmd_time_drop()
{
    Hist h = load_hist();
    TablePtrs t = setup_tables();
    auto params = load<int>("drop_params");  // [DROP_BLOCK_SIZE, iterations]
    const int block_size = params.at(0), iterations = params.at(1);
    float* x = upload(load<float>("x"), kPadded - kVoxels);
    float* x_update;
    unsigned* S;
    CK(cudaMalloc(&x_update, sizeof(float) * kPadded));
    CK(cudaMalloc(&S, sizeof(unsigned) * kPadded));
    CK(cudaMemset(x_update, 0, sizeof(float) * kPadded));
    CK(cudaMemset(S, 0, sizeof(unsigned) * kPadded));
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    std::vector<float> ms;
    for (int it = 0; it < iterations; it++) {
        CK(cudaEventRecord(a));
        drop_iteration(h, t, x, x_update, S, block_size);
        CK(cudaEventRecord(b));
        CK(cudaEventSynchronize(b));
        float m = 0;
        CK(cudaEventElapsedTime(&m, a, b));
        ms.push_back(m);
    }
    save("ms", ms.data(), ms.size());
    auto out = download(x, kVoxels);
    save("x", out.data(), out.size());
    return 0;
}

// The hull walks of SC_GPU, MSC_GPU and SM_GPU (B.cu:6681-7099), driven by the reference's own
// walk primitives.  The three kernels walk the same straight line from the entry voxel to the exit
// voxel and differ only in their WEPL window and in what they do at a voxel (SC writes 0, MSC and
// SM count), so one walk per history serves all three; the loop below is their shared loop
// (B.cu:6690-6788): the same initial voxel, distances and slopes (float differences and quotient,
// as the reference's float arrays give them), the same end test, and take_3D_step_GPU or
// take_2D_step_GPU by whether z changes.  Two bounds the reference lacks make it safe to run:
//  * the walk stops before a voxel with a negative column, row or slice index.  The reference's
//    end test only checks the upper bounds, so such a walk never ends there (it keeps stepping
//    and writing wrapped or out-of-range voxels); status 1 marks these histories;
//  * at most max_steps steps (status 2), which a walk that ends in the reference never needs
//    (it crosses at most COLUMNS + ROWS + SLICES voxel faces).
// Status 0: the walk ended by the reference's own test.  Outputs: the SC carve flags (1 where an
// SC walk wrote 0), the MSC and SM counts, and per history the status and the number of steps.
struct WalkWindows {
    double sc_lower, sc_upper, msc_lower, msc_upper, sm_lower;
    int max_steps;
};

__global__ void harness_walks_kernel(int n, const float* x_entry, const float* y_entry, const float* z_entry,
                                     const float* x_exit, const float* y_exit, const float* z_exit, const float* WEPL,
                                     const uint8_t* missed, WalkWindows w, uint8_t* sc_carved, int* msc_counts,
                                     int* sm_counts, int* status_out, int* steps_out)
{
    const int i = threadIdx.x + blockIdx.x * blockDim.x;
    if (i >= n) return;
    status_out[i] = 0;
    steps_out[i] = 0;
    if (missed[i]) return;
    const bool sc = (WEPL[i] <= w.sc_upper) && (WEPL[i] >= w.sc_lower);
    const bool msc = (WEPL[i] <= w.msc_upper) && (WEPL[i] >= w.msc_lower);
    const bool sm = WEPL[i] >= w.sm_lower;
    if (!(sc || msc || sm)) return;
    int x_move_direction, y_move_direction, z_move_direction;
    double dy_dx, dz_dx, dz_dy, dx_dy, dx_dz, dy_dz;
    double x = x_entry[i], y = y_entry[i], z = z_entry[i];
    double x_to_go, y_to_go, z_to_go;
    int voxel_x, voxel_y, voxel_z, voxel;
    int voxel_x_out, voxel_y_out, voxel_z_out, voxel_out;
    x_move_direction = (x_entry[i] <= x_exit[i]) - (x_entry[i] >= x_exit[i]);
    y_move_direction = (y_entry[i] <= y_exit[i]) - (y_entry[i] >= y_exit[i]);
    z_move_direction = (z_entry[i] <= z_exit[i]) - (z_entry[i] >= z_exit[i]);
    voxel_x = calculate_voxel_GPU(kXZero, x_entry[i], kVoxelWidth);
    voxel_y = calculate_voxel_GPU(kYZero, y_entry[i], kVoxelHeight);
    voxel_z = calculate_voxel_GPU(kZZero, z_entry[i], kVoxelThickness);
    voxel = voxel_x + voxel_y * kColumns + voxel_z * kColumns * kRows;
    x_to_go = distance_remaining_GPU(kXZero, x, kXInc, x_move_direction, kVoxelWidth, voxel_x);
    y_to_go = distance_remaining_GPU(kYZero, y, kYInc, y_move_direction, kVoxelHeight, voxel_y);
    z_to_go = distance_remaining_GPU(kZZero, z, kZInc, z_move_direction, kVoxelThickness, voxel_z);
    dy_dx = (y_exit[i] - y_entry[i]) / (x_exit[i] - x_entry[i]);
    dz_dx = (z_exit[i] - z_entry[i]) / (x_exit[i] - x_entry[i]);
    dz_dy = (z_exit[i] - z_entry[i]) / (y_exit[i] - y_entry[i]);
    dx_dy = (x_exit[i] - x_entry[i]) / (y_exit[i] - y_entry[i]);
    dx_dz = (x_exit[i] - x_entry[i]) / (z_exit[i] - z_entry[i]);
    dy_dz = (y_exit[i] - y_entry[i]) / (z_exit[i] - z_entry[i]);
    voxel_x_out = calculate_voxel_GPU(kXZero, x_exit[i], kVoxelWidth);
    voxel_y_out = calculate_voxel_GPU(kYZero, y_exit[i], kVoxelHeight);
    voxel_z_out = calculate_voxel_GPU(kZZero, z_exit[i], kVoxelThickness);
    voxel_out = voxel_x_out + voxel_y_out * kColumns + voxel_z_out * kColumns * kRows;
    bool end_walk = (voxel == voxel_out) || (voxel_x >= kColumns) || (voxel_y >= kRows) || (voxel_z >= kSlices);
    bool below = (voxel_x < 0) || (voxel_y < 0) || (voxel_z < 0);
    int steps = 0;
    while (true) {
        if (end_walk || below) break;
        if (sc) sc_carved[voxel] = 1;
        if (msc) atomicAdd(msc_counts + voxel, 1);
        if (sm) atomicAdd(sm_counts + voxel, 1);
        if (steps >= w.max_steps) break;
        if (z_move_direction != 0)
            take_3D_step_GPU(x_move_direction, y_move_direction, z_move_direction, dy_dx, dz_dx, dz_dy, dx_dy, dx_dz,
                             dy_dz, x_entry[i], y_entry[i], z_entry[i], x, y, z, voxel_x, voxel_y, voxel_z, voxel,
                             x_to_go, y_to_go, z_to_go);
        else
            take_2D_step_GPU(x_move_direction, y_move_direction, z_move_direction, dy_dx, dz_dx, dz_dy, dx_dy, dx_dz,
                             dy_dz, x_entry[i], y_entry[i], z_entry[i], x, y, z, voxel_x, voxel_y, voxel_z, voxel,
                             x_to_go, y_to_go, z_to_go);
        steps++;
        end_walk = (voxel == voxel_out) || (voxel_x >= kColumns) || (voxel_y >= kRows) || (voxel_z >= kSlices);
        below = (voxel_x < 0) || (voxel_y < 0) || (voxel_z < 0);
    }
    status_out[i] = end_walk ? 0 : (below ? 1 : 2);
    steps_out[i] = steps;
}

static int cmd_walks()
{
    auto xe = load<float>("x_entry");
    const int n = (int)xe.size();
    float* in[7];
    in[0] = upload(xe);
    const char* names[6] = {"y_entry", "z_entry", "x_exit", "y_exit", "z_exit", "WEPL"};
    for (int k = 0; k < 6; k++) {
        auto v = load<float>(names[k]);
        if ((int)v.size() != n) return 5;
        in[k + 1] = upload(v);
    }
    auto missed_h = load<uint8_t>("missed_recon_volume");
    if ((int)missed_h.size() != n) return 5;
    uint8_t* missed = upload(missed_h);
    auto wp = load<double>("walk_params");  // [SC lower, SC upper, MSC lower, MSC upper, SM lower]
    if (wp.size() != 5) return 5;
    WalkWindows w{wp[0], wp[1], wp[2], wp[3], wp[4], 4 * (kColumns + kRows + kSlices) + 16};
    uint8_t* carved;
    int *msc, *sm, *status, *steps;
    CK(cudaMalloc(&carved, kVoxels));
    CK(cudaMalloc(&msc, sizeof(int) * kVoxels));
    CK(cudaMalloc(&sm, sizeof(int) * kVoxels));
    CK(cudaMalloc(&status, sizeof(int) * (n + 1)));
    CK(cudaMalloc(&steps, sizeof(int) * (n + 1)));
    CK(cudaMemset(carved, 0, kVoxels));
    CK(cudaMemset(msc, 0, sizeof(int) * kVoxels));
    CK(cudaMemset(sm, 0, sizeof(int) * kVoxels));
    if (n > 0)
        harness_walks_kernel<<<(n + 127) / 128, 128>>>(n, in[0], in[1], in[2], in[3], in[4], in[5], in[6], missed, w,
                                                       carved, msc, sm, status, steps);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    auto a = download(carved, kVoxels);
    save("SC_carved", a.data(), a.size());
    auto b = download(msc, kVoxels);
    save("MSC_counts", b.data(), b.size());
    auto c = download(sm, kVoxels);
    save("SM_counts", c.data(), c.size());
    auto d = download(status, n);
    save("status", d.data(), d.size());
    auto e = download(steps, n);
    save("steps", e.data(), e.size());
    return 0;
}

// The deterministic parts of the reference's NTVS (its draw of L is seeded from the wall clock):
// calculate_total_variation of x and generate_perturbation_array's direction v_h.
static int cmd_tvs()
{
    auto x = load<float>("x");
    if ((long long)x.size() != kVoxels) return 5;
    const float tv = calculate_total_variation(x.data(), false);
    allocate_perturbation_arrays(false);
    generate_perturbation_array(x.data());
    save("TV", &tv, 1);
    save("v", v_h, (size_t)kVoxels);
    return 0;
}

static int cmd_endpoints()
{
    Hist h = load_hist();
    auto hull = load<uint8_t>("hull");
    if ((long long)hull.size() != kVoxels) return 5;
    bool* hull_d = reinterpret_cast<bool*>(upload(hull));
    const int per_block = 320;  // ENDPOINTS_PER_BLOCK
    collect_MLP_endpoints_GPU_nobool<<<(h.n + per_block - 1) / per_block, per_block>>>(
        h.first_MLP_voxel, hull_d, h.x_entry, h.y_entry, h.z_entry, h.xy_entry_angle, h.xz_entry_angle, h.x_exit,
        h.y_exit, h.z_exit, h.xy_exit_angle, h.xz_exit_angle, 0, h.n);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    const char* names[7] = {"first_MLP_voxel", "x_entry", "y_entry", "z_entry", "x_exit", "y_exit", "z_exit"};
    auto fv = download(h.first_MLP_voxel, h.n);
    save(names[0], fv.data(), fv.size());
    float* arrs[6] = {h.x_entry, h.y_entry, h.z_entry, h.x_exit, h.y_exit, h.z_exit};
    for (int k = 0; k < 6; k++) {
        auto a = download(arrs[k], h.n);
        save(names[k + 1], a.data(), a.size());
    }
    return 0;
}

static int cmd_intersections_and_binning(bool binning)
{
    const char* in_names[12] = {"t_in_1", "t_in_2", "t_out_1", "t_out_2", "u_in_1", "u_in_2",
                                "u_out_1", "u_out_2", "v_in_1", "v_in_2", "v_out_1", "v_out_2"};
    float* in[12];
    int n = 0;
    for (int k = 0; k < 12; k++) {
        auto v = load<float>(in_names[k]);
        n = (int)v.size();
        in[k] = upload(v);
    }
    int* gantry = upload(load<int>("gantry_angle"));
    bool* missed;
    CK(cudaMalloc(&missed, n + 1));
    float* out[10];
    for (int k = 0; k < 10; k++) CK(cudaMalloc(&out[k], sizeof(float) * (n + 1)));
    recon_volume_intersections_GPU<<<n / 1024 + 1, 1024>>>(n, gantry, missed, in[0], in[1], in[2], in[3], in[4], in[5],
                                                           in[6], in[7], in[8], in[9], in[10], in[11], out[0], out[1],
                                                           out[2], out[3], out[4], out[5], out[6], out[7], out[8],
                                                           out[9]);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    const char* out_names[10] = {"x_entry", "y_entry", "z_entry", "x_exit", "y_exit",
                                 "z_exit", "xy_entry_angle", "xz_entry_angle", "xy_exit_angle", "xz_exit_angle"};
    for (int k = 0; k < 10; k++) {
        auto a = download(out[k], n);
        save(out_names[k], a.data(), a.size());
    }
    auto m = download(reinterpret_cast<uint8_t*>(missed), n);
    save("missed_recon_volume", m.data(), m.size());
    if (binning) {
        float* wepl = upload(load<float>("WEPL"));
        int *bin_counts, *bin_num;
        float *mean_wepl, *mean_ut, *mean_uv;
        CK(cudaMalloc(&bin_counts, sizeof(int) * kNumBins));
        CK(cudaMalloc(&bin_num, sizeof(int) * n));
        CK(cudaMalloc(&mean_wepl, sizeof(float) * kNumBins));
        CK(cudaMalloc(&mean_ut, sizeof(float) * kNumBins));
        CK(cudaMalloc(&mean_uv, sizeof(float) * kNumBins));
        CK(cudaMemset(bin_counts, 0, sizeof(int) * kNumBins));
        CK(cudaMemset(bin_num, 0, sizeof(int) * n));  // binning() uploads a calloc'd bin_num_h (B.cu:5380-5396)
        CK(cudaMemset(mean_wepl, 0, sizeof(float) * kNumBins));
        CK(cudaMemset(mean_ut, 0, sizeof(float) * kNumBins));
        CK(cudaMemset(mean_uv, 0, sizeof(float) * kNumBins));
        binning_GPU<<<n / 1024 + 1, 1024>>>(n, bin_counts, bin_num, missed, out[0], out[1], out[2], out[3], out[4],
                                            out[5], mean_wepl, mean_ut, mean_uv, wepl, out[6], out[7], out[8], out[9]);
        CK(cudaGetLastError());
        CK(cudaDeviceSynchronize());
        auto bn = download(bin_num, n);
        save("bin_num", bn.data(), bn.size());
        auto bc = download(bin_counts, kNumBins);
        save("bin_counts", bc.data(), bc.size());
        auto mw = download(mean_wepl, kNumBins);
        save("sum_WEPL", mw.data(), mw.size());
        auto mu = download(mean_ut, kNumBins);
        save("sum_ut", mu.data(), mu.size());
        auto mv = download(mean_uv, kNumBins);
        save("sum_uv", mv.data(), mv.size());
    }
    return 0;
}

// construct_sinogram, filter, backprojection_GPU2, FBP_image_2_hull and the host median filter on
// device bin counts and sinogram sums (the sums are overwritten by the bin means)
static int fbp_stages(int* bin_counts, float* sinogram)
{
    const dim3 bins_grid(kVBins, kAngularBins), bins_block(kTBins);
    float *filtered, *fbp;
    CK(cudaMalloc(&filtered, sizeof(float) * kNumBins));
    CK(cudaMalloc(&fbp, sizeof(float) * kVoxels));
    CK(cudaMemset(filtered, 0, sizeof(float) * kNumBins));
    CK(cudaMemset(fbp, 0, sizeof(float) * kVoxels));
    // construct_sinogram (B.cu:6039) and FBP (B.cu:6080): filter (6185) and backprojection_GPU2
    construct_sinogram_GPU<<<bins_grid, bins_block>>>(bin_counts, sinogram);
    CK(cudaGetLastError());
    filter_GPU<<<bins_grid, bins_block>>>(sinogram, filtered);
    CK(cudaGetLastError());
    backprojection_GPU2<<<dim3(kColumns, kRows), dim3(kSlices)>>>(filtered, fbp);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    auto sg = download(sinogram, kNumBins);
    save("sinogram", sg.data(), sg.size());
    auto sf = download(filtered, kNumBins);
    save("sinogram_filtered", sf.data(), sf.size());
    auto im = download(fbp, kVoxels);
    save("FBP_image", im.data(), im.size());
    // FBP_image_2_hull (B.cu:6573) thresholds the device image, which the host median filter does not touch
    bool* hull;
    CK(cudaMalloc(&hull, kVoxels));
    FBP_image_2_hull_GPU<<<dim3(kColumns, kRows), dim3(kSlices)>>>(fbp, hull);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    auto hb = download(reinterpret_cast<uint8_t*>(hull), kVoxels);
    save("FBP_hull", hb.data(), hb.size());
    // median_filter_2D( FBP_image_h, FBP_median_filtered_h, FBP_MED_FILTER_RADIUS ) (B.cu:6159): the
    // result lands in the input image and the output buffer is freed
    float* in_h = (float*)malloc(sizeof(float) * kVoxels);
    float* out_h = (float*)calloc(kVoxels, sizeof(float));
    memcpy(in_h, im.data(), sizeof(float) * kVoxels);
    median_filter_2D(in_h, out_h, 3u);
    save("FBP_median", in_h, kVoxels);
    free(in_h);
    return 0;
}

// fbp: the FBP stages alone on stored bin counts (after the cuts) and sinogram sums, so that a
// fixture of them does not depend on the float-atomic order of the cuts' sums
static int cmd_fbp()
{
    auto counts_h = load<int>("bin_counts");
    auto sums_h = load<float>("sinogram_sums");
    if ((long long)counts_h.size() != kNumBins || (long long)sums_h.size() != kNumBins) return 5;
    return fbp_stages(upload(counts_h), upload(sums_h));
}

static int cmd_stats_fbp()
{
    int* bin_num = upload(load<int>("bin_num"));
    auto wepl_h = load<float>("WEPL");
    const int n = (int)wepl_h.size();
    float* wepl = upload(wepl_h);
    float* xye = upload(load<float>("xy_entry_angle"));
    float* xze = upload(load<float>("xz_entry_angle"));
    float* xyx = upload(load<float>("xy_exit_angle"));
    float* xzx = upload(load<float>("xz_exit_angle"));
    int* bin_counts = upload(load<int>("bin_counts"));
    float* mean_wepl = upload(load<float>("sum_WEPL"));
    float* mean_ut = upload(load<float>("sum_ut"));
    float* mean_uv = upload(load<float>("sum_uv"));
    float *sd_wepl, *sd_ut, *sd_uv, *sinogram;
    bool* failed;
    CK(cudaMalloc(&sd_wepl, sizeof(float) * kNumBins));
    CK(cudaMalloc(&sd_ut, sizeof(float) * kNumBins));
    CK(cudaMalloc(&sd_uv, sizeof(float) * kNumBins));
    CK(cudaMalloc(&sinogram, sizeof(float) * kNumBins));
    CK(cudaMalloc(&failed, n + 1));
    CK(cudaMemset(sd_wepl, 0, sizeof(float) * kNumBins));
    CK(cudaMemset(sd_ut, 0, sizeof(float) * kNumBins));
    CK(cudaMemset(sd_uv, 0, sizeof(float) * kNumBins));
    CK(cudaMemset(sinogram, 0, sizeof(float) * kNumBins));
    const dim3 bins_grid(kVBins, kAngularBins), bins_block(kTBins);
    // calculate_means (B.cu:5608), sum_squared_deviations (5655), calculate_standard_deviations (5718)
    calculate_means_GPU<<<bins_grid, bins_block>>>(bin_counts, mean_wepl, mean_ut, mean_uv);
    CK(cudaGetLastError());
    sum_squared_deviations_GPU<<<n / 1024 + 1, 1024>>>(n, bin_num, mean_wepl, mean_ut, mean_uv, wepl, xye, xze, xyx,
                                                       xzx, sd_wepl, sd_ut, sd_uv);
    CK(cudaGetLastError());
    calculate_standard_deviations_GPU<<<bins_grid, bins_block>>>(bin_counts, sd_wepl, sd_ut, sd_uv);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    const char* bin_names[6] = {"mean_WEPL", "mean_rel_ut_angle", "mean_rel_uv_angle",
                                "stddev_WEPL", "stddev_rel_ut_angle", "stddev_rel_uv_angle"};
    float* bin_arrays[6] = {mean_wepl, mean_ut, mean_uv, sd_wepl, sd_ut, sd_uv};
    for (int k = 0; k < 6; k++) {
        auto a = download(bin_arrays[k], kNumBins);
        save(bin_names[k], a.data(), a.size());
    }
    // statistical_cuts (B.cu:5851) with a zeroed sinogram (initialize_sinogram B.cu:6026)
    statistical_cuts_GPU<<<n / 1024 + 1, 1024>>>(n, bin_counts, bin_num, sinogram, wepl, xye, xze, xyx, xzx, mean_wepl,
                                                 mean_ut, mean_uv, sd_wepl, sd_ut, sd_uv, failed);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    auto fc = download(reinterpret_cast<uint8_t*>(failed), n);
    save("failed_cuts", fc.data(), fc.size());
    auto bc = download(bin_counts, kNumBins);
    save("bin_counts", bc.data(), bc.size());
    auto ss = download(sinogram, kNumBins);
    save("sinogram_sums", ss.data(), ss.size());
    return fbp_stages(bin_counts, sinogram);
}

static int cmd_edges()
{
    auto counts_h = load<int>("counts");
    if ((long long)counts_h.size() != kVoxels) return 5;
    int* msc_in = upload(counts_h);
    int* msc_out;
    CK(cudaMalloc(&msc_out, sizeof(int) * kVoxels));
    MSC_edge_detection_GPU<<<dim3(kColumns, kRows), dim3(kSlices)>>>(msc_in, msc_out);
    CK(cudaGetLastError());
    // SM_edge_detection (B.cu:7100)
    int* sm = upload(counts_h);
    int* diff;
    CK(cudaMalloc(&diff, sizeof(int) * kVoxels));
    CK(cudaMemset(diff, 0, sizeof(int) * kVoxels));
    carve_differences<<<dim3(kColumns, kRows), dim3(kSlices)>>>(diff, sm);
    CK(cudaGetLastError());
    auto diff_h = download(diff, kVoxels);
    std::vector<int> thresholds(kSlices, 0);
    for (int slice = 0; slice < kSlices; slice++) {
        int max_difference = 0;
        for (int pixel = 0; pixel < kColumns * kRows; pixel++) {
            const long long voxel = pixel + (long long)slice * kColumns * kRows;
            if (diff_h[voxel] > max_difference) {
                max_difference = diff_h[voxel];
                thresholds[slice] = counts_h[voxel];
            }
        }
    }
    int* th = upload(thresholds);
    SM_edge_detection_GPU<<<dim3(kColumns, kRows), dim3(kSlices)>>>(sm, th);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    auto a = download(msc_out, kVoxels);
    save("MSC_hull", a.data(), a.size());
    auto b = download(sm, kVoxels);
    save("SM_hull", b.data(), b.size());
    save("SM_thresholds", thresholds.data(), thresholds.size());
    return 0;
}

int main(int argc, char** argv)
{
    if (argc != 3) {
        fprintf(stderr, "usage: %s mlp|drop|time_drop|walks|scurve|tvs|endpoints|intersections|binning|stats_fbp|fbp|edges <directory>\n",
                argv[0]);
        return 1;
    }
    g_dir = argv[2];
    const std::string cmd = argv[1];
    if (cmd == "mlp") return cmd_mlp();
    if (cmd == "drop") return cmd_drop();
    if (cmd == "time_drop") return cmd_time_drop();
    if (cmd == "walks") return cmd_walks();
    if (cmd == "scurve") return cmd_scurve();
    if (cmd == "tvs") return cmd_tvs();
    if (cmd == "endpoints") return cmd_endpoints();
    if (cmd == "intersections") return cmd_intersections_and_binning(false);
    if (cmd == "binning") return cmd_intersections_and_binning(true);
    if (cmd == "stats_fbp") return cmd_stats_fbp();
    if (cmd == "fbp") return cmd_fbp();
    if (cmd == "edges") return cmd_edges();
    fprintf(stderr, "unknown command %s\n", cmd.c_str());
    return 1;
}
