/*
 * pct_oracle.c -- CPU oracle for the MLP + DROP hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see pct_oracle.h).  Each function restates one reference function;
 * the citation gives the file:line it follows (B.cu = src/pCT_Reconstruction_Data_Segments_Blake.cu,
 * B.h = include/pCT_Reconstruction_Data_Segments_Blake.h, O.cu = src/pCT_Reconstruction.cu).
 *
 * Compile with -ffp-contract=off: every double/float operation is rounded on its own, in the
 * order the reference expression is written.
 */
#include "pct_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ---------------------------------------------------------------------------------------- */
/* Constants as the reference's macros evaluate them                                         */
/* ---------------------------------------------------------------------------------------- */

/* PI = 4*atan(1.0) (B.h:818); equal to M_PI in IEEE double. */
static double ref_pi(void) { return 4 * atan(1.0); }

/* TRIG_TABLE_MIN = -2*PI, TRIG_TABLE_STEP = 0.001*ANGLE_TO_RADIANS (B.h:786-789). */
double oracle_trig_table_min(void) { return -2 * ref_pi(); }
double oracle_trig_table_step(void) { return (0.001 * (ref_pi() / 180.0)); }
static int trig_table_elements(void)
{
    /* TRIG_TABLE_ELEMENTS = static_cast<int>(TRIG_TABLE_RANGE / TRIG_TABLE_STEP + 0.5),
     * TRIG_TABLE_RANGE = (4*PI - -2*PI) (B.h:787-790). */
    double range = (4 * ref_pi() - -2 * ref_pi());
    return (int)(range / oracle_trig_table_step() + 0.5);
}
#define COEFF_TABLE_RANGE 40.0  /* B.h:791 */
#define COEFF_TABLE_STEP 0.00005 /* B.h:792 */
#define POLY_TABLE_RANGE 40.0   /* B.h:795 */
#define POLY_TABLE_STEP 0.00005  /* B.h:796 */
#define E_0 13.6                 /* B.h:741 */
#define X_0 36.08                /* B.h:742 (X0) */

/* A_0..A_5 (B.h:749-754): c * pow((float)10, (float)e) -- the float overload of pow, so the
 * power of ten is rounded to float before the double multiply. */
void oracle_a_coefficients(double a[6])
{
    a[0] = 7.457 * (double)powf(10.0f, -6.0f);
    a[1] = 4.548 * (double)powf(10.0f, -7.0f);
    a[2] = -5.777 * (double)powf(10.0f, -8.0f);
    a[3] = 1.301 * (double)powf(10.0f, -8.0f);
    a[4] = -9.228 * (double)powf(10.0f, -10.0f);
    a[5] = 2.687 * (double)powf(10.0f, -11.0f);
}

/* The reference squares several double values with powf(v, 2): the value is rounded to float
 * and raised to the power 2 in float.  The oracle takes the correctly rounded float product.
 * CUDA's powf(f, 2.0f) is one float ulp away from it for a few percent of inputs (measured by
 * the engine's pct_selftest_powf_square), so GPU and oracle voxel lists may differ at boundary
 * ties; the parity tests count them. */
static double powf_sq(double v)
{
    float f = (float)v;
    return (double)(f * f);
}

/* ---------------------------------------------------------------------------------------- */
/* MLP lookup tables (B.cu:8421-8502)                                                        */
/* ---------------------------------------------------------------------------------------- */

int oracle_tables_build(const pct_config* cfg, oracle_tables* t)
{
    (void)cfg;
    memset(t, 0, sizeof(*t));
    t->trig_elements = trig_table_elements();
    t->coeff_elements = (int)(COEFF_TABLE_RANGE / COEFF_TABLE_STEP + 0.5);
    t->poly_elements = (int)(POLY_TABLE_RANGE / POLY_TABLE_STEP + 0.5);
    t->sin_table = (double*)calloc((size_t)t->trig_elements + 1, sizeof(double));
    t->cos_table = (double*)calloc((size_t)t->trig_elements + 1, sizeof(double));
    t->scattering_table = (double*)calloc((size_t)t->coeff_elements + 1, sizeof(double));
    t->poly_1_2 = (double*)calloc((size_t)t->poly_elements + 1, sizeof(double));
    t->poly_2_3 = (double*)calloc((size_t)t->poly_elements + 1, sizeof(double));
    t->poly_3_4 = (double*)calloc((size_t)t->poly_elements + 1, sizeof(double));
    t->poly_2_6 = (double*)calloc((size_t)t->poly_elements + 1, sizeof(double));
    t->poly_3_12 = (double*)calloc((size_t)t->poly_elements + 1, sizeof(double));
    if (!t->sin_table || !t->cos_table || !t->scattering_table || !t->poly_1_2 || !t->poly_2_3 ||
        !t->poly_3_4 || !t->poly_2_6 || !t->poly_3_12) {
        oracle_tables_free(t);
        return -1;
    }
    /* generate_trig_tables (B.cu:8421): argument = TRIG_TABLE_MIN + step * TRIG_TABLE_STEP */
    for (int step = 0; step <= t->trig_elements; step++) {
        double argument = -2 * ref_pi() + step * (0.001 * (ref_pi() / 180.0));
        t->sin_table[step] = sin(argument);
        t->cos_table[step] = cos(argument);
    }
    /* generate_scattering_coefficient_table (B.cu:8445) */
    for (int step_num = 0; step_num <= t->coeff_elements; step_num++) {
        double depth = step_num * COEFF_TABLE_STEP;
        t->scattering_table[step_num] = pow(E_0 * (1 + 0.038 * log(depth / X_0)), 2.0) / X_0;
    }
    /* generate_polynomial_tables (B.cu:8464): A_k_OVER_m expands to (c_k*10^e)/m */
    double A[6];
    oracle_a_coefficients(A);
    for (int step_num = 0; step_num <= t->poly_elements; step_num++) {
        double u = step_num * POLY_TABLE_STEP;
        /* The innermost "u * A_5_OVER_m" expands to "u * 2.687 * pow(10,-11)/m", evaluated
         * left to right as ((u*2.687)*p)/m -- not u*(A_5/m). */
        const double c5 = 2.687, p5 = (double)powf(10.0f, -11.0f);
        t->poly_1_2[step_num] =
            u * (A[0] + u * (A[1] / 2 + u * (A[2] / 3 + u * (A[3] / 4 + u * (A[4] / 5 + u * c5 * p5 / 6)))));
        t->poly_2_3[step_num] = pow(u, 2) * (A[0] / 2 + u * (A[1] / 3 + u * (A[2] / 4 + u * (A[3] / 5 +
                                u * (A[4] / 6 + u * c5 * p5 / 7)))));
        t->poly_3_4[step_num] = pow(u, 3) * (A[0] / 3 + u * (A[1] / 4 + u * (A[2] / 5 + u * (A[3] / 6 +
                                u * (A[4] / 7 + u * c5 * p5 / 8)))));
        t->poly_2_6[step_num] = pow(u, 2) * (A[0] / 2 + u * (A[1] / 6 + u * (A[2] / 12 + u * (A[3] / 20 +
                                u * (A[4] / 30 + u * c5 * p5 / 42)))));
        t->poly_3_12[step_num] = pow(u, 3) * (A[0] / 3 + u * (A[1] / 12 + u * (A[2] / 30 + u * (A[3] / 60 +
                                 u * (A[4] / 105 + u * c5 * p5 / 168)))));
    }
    return 0;
}

void oracle_tables_free(oracle_tables* t)
{
    free(t->sin_table);
    free(t->cos_table);
    free(t->scattering_table);
    free(t->poly_1_2);
    free(t->poly_2_3);
    free(t->poly_3_4);
    free(t->poly_2_6);
    free(t->poly_3_12);
    memset(t, 0, sizeof(*t));
}

/* ---------------------------------------------------------------------------------------- */
/* EffectiveChordLength_GPU (B.cu:8873-8894)                                                 */
/* ---------------------------------------------------------------------------------------- */

double oracle_effective_chord_length(const pct_config* cfg, double abs_angle_t, double abs_angle_v)
{
    /* The reference's compiled form: its build fuses a product into the addition that consumes it
     * (the one with fewer uses where both operands are products), so the fused multiply-adds are
     * written out; fma() rounds once, as the device's. */
    const double PI = ref_pi();
    const int quadrants = (int)(abs_angle_t / (PI / 2));
    double eff_angle_t = fma(-(double)quadrants, PI / 2, abs_angle_t);
    double eff_angle_v = fabs(abs_angle_v);
    /* sinf/cosf take float: the double arguments are rounded to float first.  A sum of two
     * float results is a float addition. */
    double step_fraction = cfg->MLP_U_STEP / cfg->VOXEL_WIDTH;
    float s2t = sinf((float)(2 * eff_angle_t));
    float ct_plus_st = cosf((float)eff_angle_t) + sinf((float)eff_angle_t);
    double sf2_s2t = (step_fraction * step_fraction) * (double)s2t;
    double chord_length_2D = (1 / 3.0) * (fma(step_fraction * step_fraction, (double)s2t, -6.0) /
                                              fma(step_fraction, (double)s2t, -(double)(2 * ct_plus_st)) +
                                          sf2_s2t / (double)(2 * ct_plus_st));
    double mean_pixel_width = cfg->VOXEL_WIDTH / ct_plus_st;
    double height_fraction = cfg->VOXEL_THICKNESS / mean_pixel_width;
    step_fraction = cfg->MLP_U_STEP / mean_pixel_width;
    float s2v = sinf((float)(2 * eff_angle_v));
    float cv = cosf((float)eff_angle_v);
    float sv = sinf((float)eff_angle_v);
    double inner2 = 2 * fma(height_fraction, (double)cv, (double)sv);
    double sf2_s2v = (step_fraction * step_fraction) * (double)s2v;
    double chord_length_3D =
        (1 / 3.0) * (fma(-6.0, height_fraction, sf2_s2v) / fma(step_fraction, (double)s2v, -inner2) + sf2_s2v / inner2);
    return cfg->VOXEL_WIDTH * chord_length_2D * chord_length_3D;
}

/* ---------------------------------------------------------------------------------------- */
/* find_MLP_path_GPU_tabulated (B.cu:9104-9262)                                              */
/* ---------------------------------------------------------------------------------------- */

static int64_t padded_voxels(const pct_config* cfg)
{
    return (int64_t)cfg->NUM_VOXELS + (int64_t)cfg->COLUMNS * cfg->ROWS;
}

/* calculate_voxel_GPU (B.cu:11091): int(|position - zero| / size); a value that does not fit
 * an int (or NaN) is reported as -1. */
static int calc_voxel(double zero_coordinate, double current_position, double voxel_size)
{
    double q = fabs(current_position - zero_coordinate) / voxel_size;
    if (!(q < 2147483647.0)) return -1;
    return (int)q;
}

int oracle_find_mlp_path_tabulated(const pct_config* cfg, const oracle_tables* tab, const float* x,
                                   uint32_t first_MLP_voxel, double x_in_object, double y_in_object,
                                   double z_in_object, double x_out_object, double y_out_object,
                                   double z_out_object, double xy_entry_angle, double xz_entry_angle,
                                   double xy_exit_angle, double xz_exit_angle, uint32_t* path,
                                   int path_cap, double* effective_chord_length,
                                   double* a_i_dot_x_k_partially, double* a_i_dot_a_i_partially,
                                   int* flags)
{
    const double PI = ref_pi();
    const double MLP_U_STEP = cfg->MLP_U_STEP;
    const double TRIG_MIN = oracle_trig_table_min();
    const double TRIG_STEP = oracle_trig_table_step();
    const double X_ZERO = -cfg->RECON_CYL_RADIUS;
    const double Y_ZERO = cfg->RECON_CYL_RADIUS;
    const double Z_ZERO = cfg->RECON_CYL_HEIGHT / 2;
    const int64_t NPAD = padded_voxels(cfg);
    *flags = 0;

    unsigned int trig_table_index = (unsigned int)((xy_entry_angle - TRIG_MIN) / TRIG_STEP + 0.5);
    double sin_term = tab->sin_table[trig_table_index];
    double cos_term = tab->cos_table[trig_table_index];
    double u_in_object = cos_term * x_in_object + sin_term * y_in_object;
    double u_out_object = cos_term * x_out_object + sin_term * y_out_object;
    if (u_in_object > u_out_object) {
        xy_entry_angle += PI;
        xy_exit_angle += PI;
        trig_table_index = (unsigned int)((xy_entry_angle - TRIG_MIN) / TRIG_STEP + 0.5);
        sin_term = tab->sin_table[trig_table_index];
        cos_term = tab->cos_table[trig_table_index];
        u_in_object = cos_term * x_in_object + sin_term * y_in_object;
        u_out_object = cos_term * x_out_object + sin_term * y_out_object;
    }
    double t_in_object = cos_term * y_in_object - sin_term * x_in_object;
    double t_out_object = cos_term * y_out_object - sin_term * x_out_object;
    double T_2_1 = xy_exit_angle - xy_entry_angle;
    double V_2_1 = xz_exit_angle - xz_entry_angle;
    double u_1 = MLP_U_STEP;
    double u_2 = fabs(u_out_object - u_in_object);
    double depth_2_go = u_2 - u_1;
    double u_shifted = u_in_object;

    unsigned int sigma_table_index_step = (unsigned int)(MLP_U_STEP / COEFF_TABLE_STEP + 0.5);
    unsigned int sigma_1_coefficient_index = sigma_table_index_step;
    unsigned int poly_table_index_step = (unsigned int)(MLP_U_STEP / POLY_TABLE_STEP + 0.5);
    unsigned int u_1_poly_index = poly_table_index_step;
    /* The reference indexes the tables without a check; u_2 beyond POLY_TABLE_RANGE (or a
     * negative depth) would read outside them.  The oracle reports it and takes no steps. */
    int tables_ok = (u_2 / POLY_TABLE_STEP + 0.5) < (double)tab->poly_elements && depth_2_go >= 0;
    unsigned int sigma_2_coefficient_index = 0, u_2_poly_index = 0;
    if (tables_ok) {
        sigma_2_coefficient_index = (unsigned int)(depth_2_go / COEFF_TABLE_STEP + 0.5);
        u_2_poly_index = (unsigned int)(u_2 / POLY_TABLE_STEP + 0.5);
    } else {
        *flags |= 4;
    }
    double u_2_poly_3_12 = tab->poly_3_12[u_2_poly_index];
    double u_2_poly_2_6 = tab->poly_2_6[u_2_poly_index];
    double u_2_poly_1_2 = tab->poly_1_2[u_2_poly_index];
    double u_2_sq = powf_sq(u_2);

    int voxel = (int)first_MLP_voxel;
    int n = 0;
    uint32_t last = first_MLP_voxel;
    if (n < path_cap) path[n] = first_MLP_voxel;
    n++;

    *effective_chord_length = oracle_effective_chord_length(
        cfg, (xy_entry_angle + xy_exit_angle) / 2.0, (xz_entry_angle + xz_exit_angle) / 2.0);
    if ((int64_t)first_MLP_voxel < NPAD) {
        *a_i_dot_x_k_partially = x[first_MLP_voxel];
    } else {
        *a_i_dot_x_k_partially = 0.0;
        *flags |= 1;
    }
    *a_i_dot_a_i_partially = powf_sq(*effective_chord_length);

    while (tables_ok && depth_2_go > MLP_U_STEP) {
        double u_1_poly_1_2 = tab->poly_1_2[u_1_poly_index];
        double u_1_poly_2_3 = tab->poly_2_3[u_1_poly_index];
        double sigma_t1 = tab->poly_3_12[u_1_poly_index];
        double sigma_t1_theta1 = tab->poly_2_6[u_1_poly_index];
        double sigma_theta1 = u_1_poly_1_2;

        double sigma_t2 = u_2_poly_3_12 - u_2_sq * u_1_poly_1_2 + 2 * u_2 * u_1_poly_2_3 -
                          tab->poly_3_4[u_1_poly_index];
        double sigma_t2_theta2 = u_2_poly_2_6 - u_2 * u_1_poly_1_2 + u_1_poly_2_3;
        double sigma_theta2 = u_2_poly_1_2 - u_1_poly_1_2;

        double determinant_Sigma_1 = tab->scattering_table[sigma_1_coefficient_index] *
                                     (sigma_t1 * sigma_theta1 - powf_sq(sigma_t1_theta1));
        double Sigma_1I_0 = sigma_theta1 / determinant_Sigma_1;
        double Sigma_1I_1 = sigma_t1_theta1 / determinant_Sigma_1;
        double Sigma_1I_2 = sigma_t1 / determinant_Sigma_1;

        double determinant_Sigma_2 = tab->scattering_table[sigma_2_coefficient_index] *
                                     (sigma_t2 * sigma_theta2 - powf_sq(sigma_t2_theta2));
        double Sigma_2I_0 = sigma_theta2 / determinant_Sigma_2;
        double Sigma_2I_1 = sigma_t2_theta2 / determinant_Sigma_2;
        double Sigma_2I_2 = sigma_t2 / determinant_Sigma_2;

        double first_term_common_24_1 = Sigma_2I_0 * depth_2_go - Sigma_2I_1;
        double first_term_0 = Sigma_1I_0 + Sigma_2I_0;
        double first_term_1 = first_term_common_24_1 - Sigma_1I_1;
        double first_term_2 = depth_2_go * Sigma_2I_0 - Sigma_1I_1 - Sigma_2I_1;
        double first_term_3 = Sigma_1I_2 + Sigma_2I_2 + depth_2_go * (first_term_common_24_1 - Sigma_2I_1);
        double determinant_first_term = first_term_0 * first_term_3 - first_term_1 * first_term_2;

        double second_term_common_3 = Sigma_2I_0 * t_out_object - Sigma_2I_1 * T_2_1;
        double second_term_0 = Sigma_1I_0 * t_in_object + second_term_common_3;
        double second_term_1 = depth_2_go * second_term_common_3 + Sigma_2I_2 * T_2_1 -
                               Sigma_2I_1 * t_out_object - Sigma_1I_1 * t_in_object;
        double t_1 = (first_term_3 * second_term_0 - first_term_1 * second_term_1) / determinant_first_term;

        second_term_common_3 = Sigma_2I_0 * z_out_object - Sigma_2I_1 * V_2_1;
        second_term_0 = Sigma_1I_0 * z_in_object + second_term_common_3;
        second_term_1 = depth_2_go * second_term_common_3 + Sigma_2I_2 * V_2_1 -
                        Sigma_2I_1 * z_out_object - Sigma_1I_1 * z_in_object;
        double v_1 = (first_term_3 * second_term_0 - first_term_1 * second_term_1) / determinant_first_term;

        u_shifted += MLP_U_STEP;
        double x_1 = cos_term * u_shifted - sin_term * t_1;
        double y_1 = sin_term * u_shifted + cos_term * t_1;
        int voxel_x = calc_voxel(X_ZERO, x_1, cfg->VOXEL_WIDTH);
        int voxel_y = calc_voxel(Y_ZERO, y_1, cfg->VOXEL_HEIGHT);
        int voxel_z = calc_voxel(Z_ZERO, v_1, cfg->VOXEL_THICKNESS);
        int64_t v64 = (int64_t)voxel_x + (int64_t)voxel_y * cfg->COLUMNS +
                      (int64_t)voxel_z * cfg->COLUMNS * cfg->ROWS;
        if (voxel_x < 0 || voxel_y < 0 || voxel_z < 0 || v64 > 0x7fffffff) v64 = 0x7fffffff;
        voxel = (int)v64;
        if ((uint32_t)voxel != last) {
            if (n < path_cap) path[n] = (uint32_t)voxel;
            else *flags |= 2;
            if (v64 < NPAD) *a_i_dot_x_k_partially += x[voxel];
            else *flags |= 1;
            last = (uint32_t)voxel;
            n++;
        }
        u_1 += MLP_U_STEP;
        depth_2_go -= MLP_U_STEP;
        sigma_1_coefficient_index += sigma_table_index_step;
        sigma_2_coefficient_index -= sigma_table_index_step;
        u_1_poly_index += poly_table_index_step;
    }
    (void)u_1;
    return n < path_cap ? n : path_cap;
}

void oracle_mlp_paths(const pct_config* cfg, const oracle_tables* tab, const float* x,
                      const pct_histories* h, int64_t start, int64_t n, int32_t stride,
                      uint32_t* counts, uint32_t* voxels, double* chord, double* a_dot_x,
                      int64_t* flag_counts)
{
    uint32_t* scratch = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(stride > 0 ? stride : 1));
    for (int64_t k = 0; k < n; k++) {
        int64_t i = start + k;
        double L, axk, aia;
        int flags;
        uint32_t* row = voxels ? voxels + k * (int64_t)stride : scratch;
        int cnt = oracle_find_mlp_path_tabulated(
            cfg, tab, x, h->first_MLP_voxel[i], h->x_entry[i], h->y_entry[i], h->z_entry[i],
            h->x_exit[i], h->y_exit[i], h->z_exit[i], h->xy_entry_angle[i], h->xz_entry_angle[i],
            h->xy_exit_angle[i], h->xz_exit_angle[i], row, stride, &L, &axk, &aia, &flags);
        if (counts) counts[k] = (uint32_t)cnt;
        if (chord) chord[k] = L;
        if (a_dot_x) a_dot_x[k] = axk;
        if (flag_counts) {
            if (flags & 1) flag_counts[0]++;
            if (flags & 2) flag_counts[1]++;
            if (flags & 4) flag_counts[2]++;
        }
    }
    free(scratch);
}

/* ---------------------------------------------------------------------------------------- */
/* S-curve attenuation of the DROP update (B.cu:10606-10649)                                 */
/* ---------------------------------------------------------------------------------------- */

/* s(k) of the configured curve: sigmoid_GPU, tanh_GPU, atan_GPU, erf_GPU, linear_over_root_GPU
 * (B.cu:10606-10626) with the reference's expressions and argument types (k an unsigned int; the
 * sigmoid's k - SIGMOID_MID_SHIFT unsigned, so k below the shift wraps and gives exactly 1).  The
 * host's libm stands in for CUDA's math functions. */
float oracle_s_curve(const pct_config* cfg, uint32_t k)
{
    const double pi = ref_pi();
    switch (cfg->S_CURVE) {
    case PCT_TANH: return tanhf((float)k);
    case PCT_ATAN: return (float)((2 / pi) * atan((pi / 2) * k));
    case PCT_ERF: return (float)erf((sqrt(pi) / 2) * k);
    case PCT_LIN_OVER_ROOT: return (float)k / sqrtf(1.0f + powf((float)k, 2.0f));
    default:
        return (float)(1 / (1 + exp(-cfg->SIGMOID_STEEPNESS * (double)(k - (uint32_t)cfg->SIGMOID_MID_SHIFT))));
    }
}

void oracle_s_curve_table(const pct_config* cfg, int32_t count, float* out)
{
    for (int32_t k = 0; k < count; k++) out[k] = oracle_s_curve(cfg, (uint32_t)k);
}

/* s_curve_scale_GPU(j, n) (B.cu:10627-10647): k = min(j, n-1-j) when DUAL_SIDED_S_CURVE, else j. */
static float s_curve_scale(const pct_config* cfg, int j, int n)
{
    const uint32_t uj = (uint32_t)j, rest = (uint32_t)n - 1u - uj;
    return oracle_s_curve(cfg, cfg->DUAL_SIDED_S_CURVE ? (uj < rest ? uj : rest) : uj);
}

/* ---------------------------------------------------------------------------------------- */
/* DROP iteration (B.cu:9537-9589, 9321-9380, 9522-9536, 9398-9419)                          */
/* ---------------------------------------------------------------------------------------- */

void oracle_drop_iteration(const pct_config* cfg, const oracle_tables* tab, const pct_histories* h,
                           int64_t num_histories, float* x, float* x_update, uint32_t* S,
                           int64_t* flag_counts)
{
    const int path_cap = PCT_MLP_PATH_CAP;
    uint32_t* a_i = (uint32_t*)malloc(sizeof(uint32_t) * path_cap);
    const double lambda = (double)cfg->LAMBDA;
    const int64_t NPAD = padded_voxels(cfg);
    float* normA = (float*)calloc((size_t)NPAD, sizeof(float)); /* ROBUSTB accumulator */
    int64_t remaining = num_histories, start_position = 0;
    while (remaining > 0) {
        int64_t histories_2_process = remaining > cfg->DROP_BLOCK_SIZE ? cfg->DROP_BLOCK_SIZE : remaining;
        /* calculate_x_update_GPU<<<floor(B/HPB), HPB>>> covers floor(B/HPB)*HPB histories,
         * each also bounded by the total history count (B.cu:9331-9334, 9557-9559). */
        int64_t covered = histories_2_process;
        if (cfg->HISTORIES_PER_BLOCK > 0)
            covered = (histories_2_process / cfg->HISTORIES_PER_BLOCK) * cfg->HISTORIES_PER_BLOCK;
        for (int64_t k = 0; k < covered; k++) {
            int64_t proton_id = start_position + k;
            if (proton_id >= num_histories) break;
            double L, axk, aia;
            int flags;
            int n = oracle_find_mlp_path_tabulated(
                cfg, tab, x, h->first_MLP_voxel[proton_id], h->x_entry[proton_id],
                h->y_entry[proton_id], h->z_entry[proton_id], h->x_exit[proton_id],
                h->y_exit[proton_id], h->z_exit[proton_id], h->xy_entry_angle[proton_id],
                h->xz_entry_angle[proton_id], h->xy_exit_angle[proton_id],
                h->xz_exit_angle[proton_id], a_i, path_cap, &L, &axk, &aia, &flags);
            if (flag_counts) {
                if (flags & 1) flag_counts[0]++;
                if (flags & 2) flag_counts[1]++;
                if (flags & 4) flag_counts[2]++;
            }
            aia *= n;
            axk *= L;
            if (n >= cfg->MIN_MLP_LENGTH && cfg->PROJECTION_ALGORITHM == PCT_DROP && cfg->S_CURVE_ON) {
                /* DROP_block_update_GPU with S_CURVE_ON (B.cu:9529-9531): entry j adds
                 * s_curve_scale_GPU(j, n) * L * ((WEPL - axk) / aia) * lambda, rounded to float. */
                const double q = ((double)h->WEPL[proton_id] - axk) / aia;
                for (int j = 0; j < n; j++) {
                    uint32_t voxel = a_i[j];
                    if ((int64_t)voxel >= NPAD) continue;
                    S[voxel] += 1;
                    x_update[voxel] += (float)((((double)s_curve_scale(cfg, j, n) * L) * q) * lambda);
                }
            } else if (n >= cfg->MIN_MLP_LENGTH && cfg->PROJECTION_ALGORITHM == PCT_DROP) {
                /* DROP_block_update_GPU (B.cu:9522): atomicAdd(float*, double) rounds the
                 * update to float; S counts every path entry. */
                float upd = (float)(L * (((double)h->WEPL[proton_id] - axk) / aia) * lambda);
                for (int j = 0; j < n; j++) {
                    uint32_t voxel = a_i[j];
                    if ((int64_t)voxel >= NPAD) continue;
                    S[voxel] += 1;
                    x_update[voxel] += upd;
                }
            } else if (n >= cfg->MIN_MLP_LENGTH && cfg->PROJECTION_ALGORITHM == PCT_ROBUSTA) {
                /* DROP_blocks_robust1 (O.cu:7537): update_j = LAMBDA * residual / (<a,a> + Psi_j),
                 * Psi_j = ((1 - x_j) * ETA) * PSI_SIGN, <a,a> = L^2 n, residual = WEPL - L sum(x). */
                const double a_dot_a = L * L * n, residual = (double)h->WEPL[proton_id] - axk;
                for (int j = 0; j < n; j++) {
                    uint32_t voxel = a_i[j];
                    if ((int64_t)voxel >= NPAD) continue;
                    const double psi = ((1.0 - (double)x[voxel]) * cfg->ETA) * cfg->PSI_SIGN;
                    S[voxel] += 1;
                    x_update[voxel] += (float)(lambda * (residual / (a_dot_a + psi)));
                }
            } else if (n >= cfg->MIN_MLP_LENGTH && cfg->PROJECTION_ALGORITHM == PCT_ROBUSTB) {
                /* DROP_blocks_robust2 (O.cu:7554): the DROP update and ||a_i||^2 = L^2 per voxel. */
                const float upd = (float)(L * lambda * (((double)h->WEPL[proton_id] - axk) / (L * L * n)));
                for (int j = 0; j < n; j++) {
                    uint32_t voxel = a_i[j];
                    if ((int64_t)voxel >= NPAD) continue;
                    S[voxel] += 1;
                    x_update[voxel] += upd;
                    normA[voxel] += (float)(L * L);
                }
            }
        }
        /* image_update_GPU (B.cu:9398) over the NUM_VOXELS image voxels, with the
         * IDENTIFY_X_N_AIR cut (B.cu:9411); DROP_update_robust2 (O.cu:7570) for ROBUSTB. */
        for (int64_t v = 0; v < cfg->NUM_VOXELS; v++) {
            if (S[v] > 0) {
                if (cfg->PROJECTION_ALGORITHM == PCT_ROBUSTB) {
                    const double norm = (double)normA[v];
                    const double psi = cfg->PSI_SIGN * (1.0 - (double)x[v]) * cfg->ETA;
                    x[v] = (float)((double)x[v] + (norm / (norm + psi)) * (double)x_update[v] / (double)(float)S[v]);
                    normA[v] = 0.0f;
                } else {
                    x[v] += x_update[v] / (float)S[v];
                }
                if (cfg->IDENTIFY_X_N_AIR && (double)x[v] < cfg->X_N_AIR_THRESHOLD) x[v] = 0.0f;
                x_update[v] = 0.0f;
                S[v] = 0;
            }
        }
        remaining -= cfg->DROP_BLOCK_SIZE;
        start_position += cfg->DROP_BLOCK_SIZE;
    }
    free(a_i);
    free(normA);
}

/* ---------------------------------------------------------------------------------------- */
/* Reference host code: calculate_MLP (O.cu:4017-4211), DROP_blocks / DROP_update            */
/* (O.cu:7680-7711), EffectiveChordLength (O.cu:3726) with the atanf chord (O.cu:6634-6636).  */
/* ---------------------------------------------------------------------------------------- */

static int host_calc_voxel(double zero_coordinate, double current_position, double voxel_size)
{
    double q = fabs(current_position - zero_coordinate) / voxel_size;
    if (!(q < 2147483647.0)) return -1;
    return (int)q;
}

static unsigned int host_calculate_MLP(const pct_config* cfg, uint32_t* path, int path_cap,
                                       uint32_t first_voxel, double x_in_object, double y_in_object,
                                       double z_in_object, double x_out_object, double y_out_object,
                                       double z_out_object, double xy_entry_angle, double xz_entry_angle,
                                       double xy_exit_angle, double xz_exit_angle)
{
    const double PI = ref_pi();
    /* Constants.h:116-121: A_i = c_i * pow(10, e) in double. */
    const double A0 = 7.457 * pow(10, -6.0), A1 = 4.548 * pow(10, -7.0), A2 = -5.777 * pow(10, -8.0);
    const double A3 = 1.301 * pow(10, -8.0), A4 = -9.228 * pow(10, -10.0);
    /* innermost "u * A_5_OVER_m" expands to ((u*2.687)*pow(10,-11))/m */
    const double P11 = pow(10, -11.0);
    const double s = cfg->MLP_U_STEP;
    int num_intersections = 0;
    path[num_intersections++] = first_voxel;

    double u_in_object = (cos(xy_entry_angle) * x_in_object) + (sin(xy_entry_angle) * y_in_object);
    double u_out_object = (cos(xy_entry_angle) * x_out_object) + (sin(xy_entry_angle) * y_out_object);
    double t_in_object = (cos(xy_entry_angle) * y_in_object) - (sin(xy_entry_angle) * x_in_object);
    double t_out_object = (cos(xy_entry_angle) * y_out_object) - (sin(xy_entry_angle) * x_out_object);
    if (u_in_object > u_out_object) {
        xy_entry_angle += PI;
        xy_exit_angle += PI;
        u_in_object = (cos(xy_entry_angle) * x_in_object) + (sin(xy_entry_angle) * y_in_object);
        u_out_object = (cos(xy_entry_angle) * x_out_object) + (sin(xy_entry_angle) * y_out_object);
        t_in_object = (cos(xy_entry_angle) * y_in_object) - (sin(xy_entry_angle) * x_in_object);
        t_out_object = (cos(xy_entry_angle) * y_out_object) - (sin(xy_entry_angle) * x_out_object);
    }
    double T0 = t_in_object, T20 = t_out_object, T21 = xy_exit_angle - xy_entry_angle;
    double V0 = z_in_object, V20 = z_out_object, V21 = xz_exit_angle - xz_entry_angle;
    double u_0 = 0.0, u_1 = s, u_2 = fabs(u_out_object - u_in_object);
    double sigma_2_pre_1 = pow(u_2, 3.0) * (A0 / 3 + u_2 * (A1 / 12 + u_2 * (A2 / 30 + u_2 * (A3 / 60 + u_2 * (A4 / 105 + u_2 * 2.687 * P11 / 168)))));
    double sigma_2_pre_2 = pow(u_2, 2.0) * (A0 / 2 + u_2 * (A1 / 6 + u_2 * (A2 / 12 + u_2 * (A3 / 20 + u_2 * (A4 / 30 + u_2 * 2.687 * P11 / 42)))));
    double sigma_2_pre_3 = u_2 * (A0 + u_2 * (A1 / 2 + u_2 * (A2 / 3 + u_2 * (A3 / 4 + u_2 * (A4 / 5 + u_2 * 2.687 * P11 / 6)))));
    const double X_ZERO = -cfg->RECON_CYL_RADIUS, Y_ZERO = cfg->RECON_CYL_RADIUS, Z_ZERO = cfg->RECON_CYL_HEIGHT / 2;
    while (u_1 < u_2 - s) {
        double R0_1 = u_1, R1_1 = u_2 - u_1;
        double c1 = pow(E_0 * (1 + 0.038 * log((u_1 - u_0) / X_0)), 2.0) / X_0;
        double st1 = c1 * (pow(u_1, 3.0) * (A0 / 3 + u_1 * (A1 / 12 + u_1 * (A2 / 30 + u_1 * (A3 / 60 + u_1 * (A4 / 105 + u_1 * 2.687 * P11 / 168))))));
        double st1th1 = c1 * (pow(u_1, 2.0) * (A0 / 2 + u_1 * (A1 / 6 + u_1 * (A2 / 12 + u_1 * (A3 / 20 + u_1 * (A4 / 30 + u_1 * 2.687 * P11 / 42))))));
        double sth1 = c1 * (u_1 * (A0 + u_1 * (A1 / 2 + u_1 * (A2 / 3 + u_1 * (A3 / 4 + u_1 * (A4 / 5 + u_1 * 2.687 * P11 / 6))))));
        double det1 = st1 * sth1 - pow(st1th1, 2);
        double S1I0 = sth1 / det1, S1I1 = -st1th1 / det1, S1I2 = -st1th1 / det1, S1I3 = st1 / det1;
        double c2 = pow(E_0 * (1 + 0.038 * log((u_2 - u_1) / X_0)), 2.0) / X_0;
        double cs1 = u_1 * (A0 + u_1 * (A1 / 2 + u_1 * (A2 / 3 + u_1 * (A3 / 4 + u_1 * (A4 / 5 + u_1 * 2.687 * P11 / 6)))));
        double cs2 = pow(u_1, 2.0) * (A0 / 2 + u_1 * (A1 / 3 + u_1 * (A2 / 4 + u_1 * (A3 / 5 + u_1 * (A4 / 6 + u_1 * 2.687 * P11 / 7)))));
        double cs3 = pow(u_1, 3.0) * (A0 / 3 + u_1 * (A1 / 4 + u_1 * (A2 / 5 + u_1 * (A3 / 6 + u_1 * (A4 / 7 + u_1 * 2.687 * P11 / 8)))));
        double st2 = c2 * (sigma_2_pre_1 - pow(u_2, 2.0) * cs1 + 2 * u_2 * cs2 - cs3);
        double st2th2 = c2 * (sigma_2_pre_2 - u_2 * cs1 + cs2);
        double sth2 = c2 * (sigma_2_pre_3 - cs1);
        double det2 = st2 * sth2 - pow(st2th2, 2);
        double S2I0 = sth2 / det2, S2I1 = -st2th2 / det2, S2I2 = -st2th2 / det2, S2I3 = st2 / det2;
        /* R_1 = [1, u_2-u_1; 0, 1], R_1T = [1, 0; u_2-u_1, 1], R_0 = [1, u_1; 0, 1] */
        double f13_1 = S2I0 * 1 + S2I1 * 0, f13_2 = S2I2 * 1 + S2I3 * 0;
        double f24_1 = S2I0 * R1_1 + S2I1 * 1, f24_2 = S2I2 * R1_1 + S2I3 * 1;
        double ft0 = S1I0 + 1 * f13_1 + 0 * f13_2;
        double ft1 = S1I1 + 1 * f24_1 + 0 * f24_2;
        double ft2 = S1I2 + R1_1 * f13_1 + 1 * f13_2;
        double ft3 = S1I3 + R1_1 * f24_1 + 1 * f24_2;
        double detft = ft0 * ft3 - ft1 * ft2;
        double tmp = ft0;
        ft0 = ft3 / detft;
        ft1 = -ft1 / detft;
        ft2 = -ft2 / detft;
        ft3 = tmp / detft;
        (void)ft2;
        (void)ft3;
        double sc1 = 1 * T0 + R0_1 * 0.0, sc2 = 0 * T0 + 1 * 0.0;
        double sc3 = S2I0 * T20 + S2I1 * T21, sc4 = S2I2 * T20 + S2I3 * T21;
        double s0 = S1I0 * sc1 + S1I1 * sc2 + 1 * sc3 + 0 * sc4;
        double s1 = S1I2 * sc1 + S1I3 * sc2 + R1_1 * sc3 + 1 * sc4;
        double t_1 = ft0 * s0 + ft1 * s1;
        sc1 = 1 * V0 + R0_1 * 0.0;
        sc2 = 0 * V0 + 1 * 0.0;
        sc3 = S2I0 * V20 + S2I1 * V21;
        sc4 = S2I2 * V20 + S2I3 * V21;
        s0 = S1I0 * sc1 + S1I1 * sc2 + 1 * sc3 + 0 * sc4;
        s1 = S1I2 * sc1 + S1I3 * sc2 + R1_1 * sc3 + 1 * sc4;
        double v_1 = ft0 * s0 + ft1 * s1;
        double x_1 = (cos(xy_entry_angle) * (u_in_object + u_1)) - (sin(xy_entry_angle) * t_1);
        double y_1 = (sin(xy_entry_angle) * (u_in_object + u_1)) + (cos(xy_entry_angle) * t_1);
        int vx = host_calc_voxel(X_ZERO, x_1, cfg->VOXEL_WIDTH);
        int vy = host_calc_voxel(Y_ZERO, y_1, cfg->VOXEL_HEIGHT);
        int vz = host_calc_voxel(Z_ZERO, v_1, cfg->VOXEL_THICKNESS);
        int voxel = (vx < 0 || vy < 0 || vz < 0) ? 0x7fffffff : vx + vy * cfg->COLUMNS + vz * cfg->COLUMNS * cfg->ROWS;
        if ((uint32_t)voxel != path[num_intersections - 1] && num_intersections < path_cap)
            path[num_intersections++] = (uint32_t)voxel;
        u_1 += s;
    }
    return (unsigned int)num_intersections;
}

/* The float overload of EffectiveChordLength (O.cu:3745-3767), which the host code calls with its
 * float avg_xy_angle / avg_xz_angle.  Each statement rounds to float where the reference stores to
 * a float variable; expressions mixing a double (PI, 1/3.0, the double parameters VOXEL_WIDTH,
 * VOXEL_THICKNESS, MLP_U_STEP) are evaluated in double first.  eff_angle_t keeps the sign of the
 * angle (no fabs), as written: atanf gives angles in (-pi/2, pi/2). */
float oracle_host_effective_chord_length(const pct_config* cfg, float abs_angle_t, float abs_angle_v)
{
    const double PI = ref_pi();
    float eff_angle_t = (float)((double)abs_angle_t - ((int)((double)abs_angle_t / (PI / 2))) * (PI / 2));
    float eff_angle_v = fabsf(abs_angle_v);
    float step_fraction = (float)(cfg->MLP_U_STEP / cfg->VOXEL_WIDTH);
    float s2t = sinf(2 * eff_angle_t), ct = cosf(eff_angle_t), st = sinf(eff_angle_t);
    float sf2 = step_fraction * step_fraction;
    float chord_length_2D = (float)((1 / 3.0) * ((sf2 * s2t - 6) / (step_fraction * s2t - 2 * (ct + st)) +
                                                 sf2 * s2t / (2 * (ct + st))));
    float mean_pixel_width = (float)(cfg->VOXEL_WIDTH / (double)(ct + st));
    float height_fraction = (float)(cfg->VOXEL_THICKNESS / (double)mean_pixel_width);
    step_fraction = (float)(cfg->MLP_U_STEP / (double)mean_pixel_width);
    sf2 = step_fraction * step_fraction;
    float s2v = sinf(2 * eff_angle_v), cv = cosf(eff_angle_v), sv = sinf(eff_angle_v);
    float chord_length_3D =
        (float)((1 / 3.0) * ((sf2 * s2v - 6 * height_fraction) / (step_fraction * s2v - 2 * (height_fraction * cv + sv)) +
                             sf2 * s2v / (2 * (height_fraction * cv + sv))));
    return (float)(cfg->VOXEL_WIDTH * (double)chord_length_2D * (double)chord_length_3D);
}

static double host_effective_chord_length(const pct_config* cfg, const pct_histories* h, int64_t i)
{
    /* O.cu:6634-6636: mean angles from atanf of the chord slopes, into the float overload */
    float avg_xy = atanf((h->y_exit[i] - h->y_entry[i]) / (h->x_exit[i] - h->x_entry[i]));
    float avg_xz = atanf((h->z_exit[i] - h->z_entry[i]) / (h->x_exit[i] - h->x_entry[i]));
    return (double)oracle_host_effective_chord_length(cfg, avg_xy, avg_xz);
}

/* The host MLP voxel lists (calculate_MLP, O.cu:4017-4211) of histories [start, start + n),
 * stride entries per history, and the atanf chord lengths. */
void oracle_host_mlp_paths(const pct_config* cfg, const pct_histories* h, int64_t start, int64_t n, int32_t stride,
                           uint32_t* counts, uint32_t* voxels, double* chord)
{
    for (int64_t k = 0; k < n; k++) {
        const int64_t i = start + k;
        counts[k] = host_calculate_MLP(cfg, voxels + k * (int64_t)stride, stride, h->first_MLP_voxel[i],
                                       h->x_entry[i], h->y_entry[i], h->z_entry[i], h->x_exit[i], h->y_exit[i],
                                       h->z_exit[i], h->xy_entry_angle[i], h->xz_entry_angle[i], h->xy_exit_angle[i],
                                       h->xz_exit_angle[i]);
        chord[k] = host_effective_chord_length(cfg, h, i);
    }
}

int64_t oracle_host_drop_iteration(const pct_config* cfg, const pct_histories* h, int64_t n,
                                   float* x, int threads)
{
    const int64_t NV = cfg->NUM_VOXELS;
    const int64_t NPAD = padded_voxels(cfg);
    const double lambda = (double)cfg->LAMBDA;
    int64_t visited = 0;
    if (threads < 1) threads = 1;
    double* x_update = (double*)calloc((size_t)NPAD, sizeof(double));
    uint32_t* counts = (uint32_t*)calloc((size_t)NPAD, sizeof(uint32_t));
    for (int64_t start = 0; start < n; start += cfg->DROP_BLOCK_SIZE) {
        int64_t end = start + cfg->DROP_BLOCK_SIZE < n ? start + cfg->DROP_BLOCK_SIZE : n;
#pragma omp parallel num_threads(threads) reduction(+ : visited)
        {
            uint32_t path[4096];
#pragma omp for schedule(dynamic, 64)
            for (int64_t i = start; i < end; i++) {
                unsigned int m = host_calculate_MLP(cfg, path, 4096, h->first_MLP_voxel[i], h->x_entry[i],
                                                    h->y_entry[i], h->z_entry[i], h->x_exit[i], h->y_exit[i],
                                                    h->z_exit[i], h->xy_entry_angle[i], h->xz_entry_angle[i],
                                                    h->xy_exit_angle[i], h->xz_exit_angle[i]);
                double L = host_effective_chord_length(cfg, h, i);
                /* DROP_blocks (O.cu:7680): scalar_dot_product2 then the scaled residual */
                double sum = 0;
                for (unsigned int j = 0; j < m; j++)
                    if ((int64_t)path[j] < NPAD) sum += x[path[j]];
                double a_i_dot_x_k = L * sum;
                double scaled_residual = ((double)h->WEPL[i] - a_i_dot_x_k) / (pow(L, 2.0) * m);
                double update_value = L * lambda * scaled_residual;
                for (unsigned int j = 0; j < m; j++) {
                    if ((int64_t)path[j] >= NPAD) continue;
#pragma omp atomic
                    x_update[path[j]] += update_value;
#pragma omp atomic
                    counts[path[j]] += 1;
                }
                visited += m;
            }
        }
        /* DROP_update (O.cu:7700) */
#pragma omp parallel for num_threads(threads) schedule(static)
        for (int64_t v = 0; v < NV; v++) {
            if (counts[v] > 0) {
                x[v] += (float)(x_update[v] / counts[v]);
                x_update[v] = 0;
                counts[v] = 0;
            }
        }
    }
    free(x_update);
    free(counts);
    return visited;
}
