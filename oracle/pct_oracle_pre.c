/*
 * pct_oracle_pre.c -- CPU oracle for the preprocessing stages (TEST INFRASTRUCTURE ONLY).
 *
 * Plain-C restatements of the reference kernels that turn tracker data into reconstruction
 * histories and the initial image (B.cu = src/pCT_Reconstruction_Data_Segments_Blake.cu).  Each
 * function cites the reference lines it follows.  Where the reference applies a float function
 * to float operands (atan2, abs, powf, sqrtf, tanf) the oracle calls the glibc float function;
 * CUDA's float functions may differ in the last bit, so integer outputs that hinge on such a
 * value can differ at boundary ties, which the tests count.  Sums the reference accumulates with
 * float atomics are accumulated here in history order.  Compiled with -ffp-contract=off.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "pct_oracle.h"

#define PI_ (4 * atan(1.0))
#define PI_OVER_4 (atan(1.0))
#define PI_OVER_2 (2 * atan(1.0))
#define ANGLE_TO_RADIANS (PI_ / 180.0)
#define RADIANS_TO_ANGLE (180.0 / PI_)

static float sqf(double v)
{
    float f = (float)v;
    return f * f;
}

/* calculate_intercepts (B.cu:5286-5372) */
static int calculate_intercepts(double R, double u, double t, double ut_angle, double* u_intercept, double* t_intercept)
{
    int entry_in_cone = ((ut_angle > PI_OVER_4) && (ut_angle < 3 * atan(1.0))) ||
                        ((ut_angle > 5 * atan(1.0)) && (ut_angle < 7 * atan(1.0)));
    double u_temp;
    if (entry_in_cone) {
        u_temp = u;
        u = -t;
        t = u_temp;
        ut_angle += PI_OVER_2;
    }
    double m = tan(ut_angle);
    double b_in = t - m * u;
    double a = 1 + (double)sqf(m);
    double b = 2 * m * b_in;
    double c = (double)(sqf(b_in) - sqf(R));
    double disc = (double)sqf(b) - (4 * a * c);
    int intersected = disc > 0;
    if (intersected) {
        double u1 = (sqrt(disc) - b) / (2 * a);
        double u2 = (sqrt(disc) + b) / (2 * a);
        double t1 = m * u1 + b_in;
        double t2 = m * u2 - b_in;
        double sd1 = (double)(sqf(u1 - u) + sqf(t1 - t));
        double sd2 = (double)(sqf(u2 + u) + sqf(t2 + t));
        *u_intercept = u1 * (sd1 <= sd2) - u2 * (sd1 > sd2);
        *t_intercept = t1 * (sd1 <= sd2) - t2 * (sd1 > sd2);
    }
    if (entry_in_cone) {
        u_temp = *u_intercept;
        *u_intercept = *t_intercept;
        *t_intercept = -u_temp;
    }
    return intersected;
}

/* recon_volume_intersections_GPU (B.cu:4890-5021) / _exact_angles (B.cu:5022) */
void oracle_recon_volume_intersections(const pct_config* cfg, int64_t n, const float* const tracker[12],
                                       const float* gantry_angle, int integer_angles, float* const out[10],
                                       uint8_t* missed)
{
    const double H = cfg->RECON_CYL_HEIGHT, R = cfg->RECON_CYL_RADIUS;
    for (int64_t i = 0; i < n; i++) {
        const float t_in_1 = tracker[0][i], t_in_2 = tracker[1][i], t_out_1 = tracker[2][i], t_out_2 = tracker[3][i];
        const float u_in_1 = tracker[4][i], u_in_2 = tracker[5][i], u_out_1 = tracker[6][i], u_out_2 = tracker[7][i];
        const float v_in_1 = tracker[8][i], v_in_2 = tracker[9][i], v_out_1 = tracker[10][i], v_out_2 = tracker[11][i];
        double rot = integer_angles ? (int)gantry_angle[i] * ANGLE_TO_RADIANS : gantry_angle[i] * ANGLE_TO_RADIANS;
        double ut_entry_angle = atan2f(t_in_2 - t_in_1, u_in_2 - u_in_1);
        double u_entry = 0, t_entry = 0;
        int entered = calculate_intercepts(R, u_in_2, t_in_2, ut_entry_angle, &u_entry, &t_entry);
        float xy_entry_angle = (float)(ut_entry_angle + rot);
        float x_entry = (float)((cos(rot) * u_entry) - (sin(rot) * t_entry));
        float y_entry = (float)((sin(rot) * u_entry) + (cos(rot) * t_entry));
        double ut_exit_angle = atan2f(t_out_2 - t_out_1, u_out_2 - u_out_1);
        double u_exit = 0, t_exit = 0;
        int exited = calculate_intercepts(R, u_out_1, t_out_1, ut_exit_angle, &u_exit, &t_exit);
        float xy_exit_angle = (float)(ut_exit_angle + rot);
        float x_exit = (float)((cos(rot) * u_exit) - (sin(rot) * t_exit));
        float y_exit = (float)((sin(rot) * u_exit) + (cos(rot) * t_exit));
        double uv_entry_slope = (v_in_2 - v_in_1) / (u_in_2 - u_in_1);
        double uv_exit_slope = (v_out_2 - v_out_1) / (u_out_2 - u_out_1);
        float xz_entry_angle = atan2f(v_in_2 - v_in_1, u_in_2 - u_in_1);
        float xz_exit_angle = atan2f(v_out_2 - v_out_1, u_out_2 - u_out_1);
        u_entry = (cos(rot) * x_entry) + (sin(rot) * y_entry);
        u_exit = (cos(rot) * x_exit) + (sin(rot) * y_exit);
        float z_entry = (float)(v_in_2 + uv_entry_slope * (u_entry - u_in_2));
        float z_exit = (float)(v_out_1 - uv_exit_slope * (u_out_1 - u_exit));
        if (entered && exited) {
            if ((fabsf(z_entry) < H * 0.5) && (fabsf(z_exit) > H * 0.5)) {
                double f = fabs((((z_exit >= 0) - (z_exit < 0)) * H * 0.5 - z_entry) / (double)(z_exit - z_entry));
                x_exit = (float)(x_entry + f * (x_exit - x_entry));
                y_exit = (float)(y_entry + f * (y_exit - y_entry));
                z_exit = (float)(((z_exit >= 0) - (z_exit < 0)) * H * 0.5);
            } else if (fabsf(z_entry) > H * 0.5) {
                entered = exited = 0;
            }
            if ((fabsf(z_entry) > H * 0.5) && (fabsf(z_exit) < H * 0.5)) {
                double f = fabs((((z_exit >= 0) - (z_exit < 0)) * H * 0.5 - z_exit) / (double)(z_exit - z_entry));
                x_entry = (float)(x_exit + f * (x_exit - x_entry));
                y_entry = (float)(y_exit + f * (y_exit - y_entry));
                z_entry = (float)(((z_entry >= 0) - (z_entry < 0)) * H * 0.5);
            }
            if ((fabsf(t_out_1 - t_in_2) > 5) || (fabsf(v_out_1 - v_in_2) > 5)) entered = exited = 0;
        }
        out[0][i] = x_entry;
        out[1][i] = y_entry;
        out[2][i] = z_entry;
        out[3][i] = x_exit;
        out[4][i] = y_exit;
        out[5][i] = z_exit;
        out[6][i] = xy_entry_angle;
        out[7][i] = xz_entry_angle;
        out[8][i] = xy_exit_angle;
        out[9][i] = xz_exit_angle;
        missed[i] = (!entered || !exited) ? 1 : 0;
    }
}

static double rel_angle(float exit_angle, float entry_angle)
{
    double a = exit_angle - entry_angle;
    if (a > PI_) a -= 2 * PI_;
    if (a < -PI_) a += 2 * PI_;
    return a;
}

/* binning_GPU (B.cu:5482-5553); sums in history order */
void oracle_binning(const pct_config* cfg, int64_t n, const float* const g[10], const float* WEPL, const uint8_t* missed,
                    int32_t* bin_num, int32_t* bin_counts, float* sum_WEPL, float* sum_ut, float* sum_uv)
{
    for (int64_t i = 0; i < n; i++) {
        double x_mid = (g[0][i] + g[3][i]) / 2, y_mid = (g[1][i] + g[4][i]) / 2, z_mid = (g[2][i] + g[5][i]) / 2;
        double path_angle = atan2f(g[4][i] - g[1][i], g[3][i] - g[0][i]);
        if (path_angle < 0) path_angle += 2 * PI_;
        int angle_bin = (int)((path_angle * RADIANS_TO_ANGLE / cfg->ANGULAR_BIN_SIZE) + 0.5) % cfg->ANGULAR_BINS;
        double angle = angle_bin * cfg->ANGULAR_BIN_SIZE * ANGLE_TO_RADIANS;
        double t = y_mid * cos(angle) - x_mid * sin(angle);
        int t_bin = (int)((t / cfg->T_BIN_SIZE) + cfg->T_BINS / 2);
        int v_bin = (int)((z_mid / cfg->V_BIN_SIZE) + cfg->V_BINS / 2);
        int bin = 0;
        if (t_bin >= 0 && v_bin >= 0 && t_bin < cfg->T_BINS && v_bin < cfg->V_BINS) {
            bin = t_bin + angle_bin * cfg->T_BINS + v_bin * cfg->T_BINS * cfg->ANGULAR_BINS;
            if (!missed[i]) {
                bin_counts[bin] += 1;
                sum_WEPL[bin] += WEPL[i];
                sum_ut[bin] += (float)rel_angle(g[8][i], g[6][i]);
                sum_uv[bin] += (float)rel_angle(g[9][i], g[7][i]);
            }
        }
        bin_num[i] = bin;
    }
}

/* calculate_means_GPU, sum_squared_deviations_GPU, calculate_standard_deviations_GPU and
 * statistical_cuts_GPU (B.cu:5644-5971) over the binned history vectors (n histories);
 * keep[i] = survivor flag, sinogram = per-bin WEPL sums of survivors, bin_counts = survivors. */
void oracle_statistics_and_cuts(const pct_config* cfg, int64_t n, const int32_t* bin_num, const float* WEPL,
                                const float* const g[10], int32_t* bin_counts, float* mean_WEPL, float* mean_ut,
                                float* mean_uv, float* sd_WEPL, float* sd_ut, float* sd_uv, float* sinogram,
                                uint8_t* keep)
{
    const int64_t nb = cfg->NUM_BINS;
    for (int64_t b = 0; b < nb; b++)
        if (bin_counts[b] > 0) {
            mean_WEPL[b] /= bin_counts[b];
            mean_ut[b] /= bin_counts[b];
            mean_uv[b] /= bin_counts[b];
        }
    memset(sd_WEPL, 0, sizeof(float) * nb);
    memset(sd_ut, 0, sizeof(float) * nb);
    memset(sd_uv, 0, sizeof(float) * nb);
    for (int64_t i = 0; i < n; i++) {
        int b = bin_num[i];
        double ru = rel_angle(g[8][i], g[6][i]), rv = rel_angle(g[9][i], g[7][i]);
        double dw = WEPL[i] - mean_WEPL[b];
        sd_WEPL[b] += sqf(dw);
        sd_ut[b] += sqf(ru - mean_ut[b]);
        sd_uv[b] += sqf(rv - mean_uv[b]);
    }
    const int sample = cfg->SAMPLE_STD_DEV ? 1 : 0;
    for (int64_t b = 0; b < nb; b++) {
        if (bin_counts[b] > 1) {
            float d = (float)(bin_counts[b] - sample);
            sd_WEPL[b] = sqrtf(sd_WEPL[b] / d);
            sd_ut[b] = sqrtf(sd_ut[b] / d);
            sd_uv[b] = sqrtf(sd_uv[b] / d);
        }
        bin_counts[b] = 0;
    }
    memset(sinogram, 0, sizeof(float) * nb);
    const float k = (float)cfg->SIGMAS_TO_KEEP;
    for (int64_t i = 0; i < n; i++) {
        int b = bin_num[i];
        double ru = rel_angle(g[8][i], g[6][i]), rv = rel_angle(g[9][i], g[7][i]);
        int pass_ut = fabs(ru - mean_ut[b]) < (double)(k * sd_ut[b]);
        int pass_uv = fabs(rv - mean_uv[b]) < (double)(k * sd_uv[b]);
        int pass_w = fabsf(mean_WEPL[b] - WEPL[i]) <= k * sd_WEPL[b];
        int failed = !pass_ut || !pass_uv || !pass_w;
        keep[i] = failed ? 0 : 1;
        if (!failed) {
            bin_counts[b] += 1;
            sinogram[b] += WEPL[i];
        }
    }
}

/* construct_sinogram_GPU (B.cu:6073) and filter_GPU (B.cu:6206-6240) */
void oracle_sinogram_filter(const pct_config* cfg, const int32_t* bin_counts, float* sinogram, float* filtered)
{
    const int T = cfg->T_BINS, V = cfg->V_BINS, A = cfg->ANGULAR_BINS;
    const int64_t nb = cfg->NUM_BINS;
    for (int64_t b = 0; b < nb; b++)
        if (bin_counts[b] > 0) sinogram[b] /= bin_counts[b];
    const double tau = (double)(2.0f / sqrtf(2.0f)) * cfg->T_BIN_SIZE;
    for (int v_bin = 0; v_bin < V; v_bin++)
        for (int angle_bin = 0; angle_bin < A; angle_bin++)
            for (int t_bin = 0; t_bin < T; t_bin++) {
                int64_t strip = ((int64_t)v_bin * A + angle_bin) * T;
                if (cfg->SINOGRAM_FILTER == PCT_UNFILTERED) {
                    filtered[strip + t_bin] = sinogram[strip + t_bin];
                    continue;
                }
                double v = (v_bin - V / 2 + 0.5) * cfg->V_BIN_SIZE;
                float acc = 0.0f;
                for (int t_ref = 0; t_ref < T; t_ref++) {
                    double t = (t_ref - T / 2 + 0.5) * cfg->T_BIN_SIZE;
                    int sep = t_bin - t_ref;
                    double scale = cfg->SOURCE_RADIUS / sqrt(cfg->SOURCE_RADIUS * cfg->SOURCE_RADIUS + t * t + v * v);
                    double f;
                    if (cfg->SINOGRAM_FILTER == PCT_RAM_LAK) {
                        if (sep == 0) f = 1.0 / (4.0 * pow(tau, 2.0));
                        else if (sep % 2 == 0) f = 0;
                        else f = -1.0 / (pow(tau * PI_ * sep, 2.0));
                    } else {
                        f = 1.0 / ((cfg->T_BIN_SIZE * PI_ * cfg->T_BIN_SIZE * PI_) * (1.0 - (4 * sep * sep)));
                    }
                    acc += (float)(cfg->T_BIN_SIZE * sinogram[strip + t_ref] * f * scale);
                }
                filtered[strip + t_bin] = acc;
            }
}

/* voxel_2_3D_voxels_GPU (B.cu:11117): loops that stop at "> 0" */
static void voxel_2_3D(const pct_config* cfg, int voxel, int* vx, int* vy, int* vz)
{
    *vx = *vy = *vz = 0;
    while (voxel - cfg->COLUMNS * cfg->ROWS > 0) {
        voxel -= cfg->COLUMNS * cfg->ROWS;
        (*vz)++;
    }
    while (voxel - cfg->COLUMNS > 0) {
        voxel -= cfg->COLUMNS;
        (*vy)++;
    }
    *vx = voxel;
}

/* backprojection_GPU2 (B.cu:6340-6479) */
void oracle_backprojection(const pct_config* cfg, const float* sf, float* FBP)
{
    const int T = cfg->T_BINS, V = cfg->V_BINS, A = cfg->ANGULAR_BINS;
    const double delta = cfg->ANGULAR_BIN_SIZE * ANGLE_TO_RADIANS, SR = cfg->SOURCE_RADIUS;
    for (int voxel = 0; voxel < cfg->NUM_VOXELS; voxel++) {
        int vx, vy, vz;
        voxel_2_3D(cfg, voxel, &vx, &vy, &vz);
        double x = 1 * (vx - (cfg->COLUMNS - 1) / 2.0) * cfg->VOXEL_WIDTH;
        double y = -1 * (vy - (cfg->ROWS - 1) / 2.0) * cfg->VOXEL_HEIGHT;
        double z = -1 * (vz - (cfg->SLICES - 1) / 2.0) * cfg->VOXEL_THICKNESS;
        if ((x * x + y * y) > (cfg->RECON_CYL_RADIUS * cfg->RECON_CYL_RADIUS)) {
            FBP[voxel] = (float)cfg->RSP_AIR;
            continue;
        }
        float acc = 0.0f;
        for (int angle_bin = 0; angle_bin < A; angle_bin++) {
            double ba = angle_bin * delta;
            double u = x * cos(ba) + y * sin(ba);
            double t = y * cos(ba) - x * sin(ba);
            double v = z;
            double dnt = (t - u * (t / (SR + u))) / cfg->T_BIN_SIZE + T / 2.0;
            int t_bin = (int)floor(dnt);
            double eta = dnt - t_bin;
            double dnv = (v - u * (v / (SR + u))) / cfg->V_BIN_SIZE + V / 2.0;
            int v_bin = (int)floor(dnv);
            double eps = dnv - v_bin;
            double scale = (double)sqf(SR / (SR + u));
            int64_t b11 = ((int64_t)v_bin * A + angle_bin) * T + t_bin, b12 = b11 + 1, b21 = b11 + (int64_t)A * T, b22 = b21 + 1;
            float xterm = 0.0f;
            if (t_bin > -1 && t_bin < T - 1) {
                if (v_bin > -1 && v_bin < V - 1)
                    xterm = (float)(sf[b11] * (1 - eta) * (1 - eps) + sf[b12] * eta * (1 - eps) + sf[b21] * (1 - eta) * eps + sf[b22] * eta * eps);
                else if (v_bin == -1)
                    xterm = (float)(sf[b21] * (1 - eta) * eps + sf[b22] * eta * eps);
                else if (v_bin == V - 1)
                    xterm = (float)(sf[b11] * (1 - eta) * (1 - eps) + sf[b12] * eta * (1 - eps));
            } else if (t_bin == -1) {
                if (v_bin > -1 && v_bin < V - 1)
                    xterm = (float)(sf[b12] * eta * (1 - eps) + sf[b22] * eta * eps);
                else if (v_bin == -1)
                    xterm = (float)(sf[b22] * eta * eps);
                else if (v_bin == V - 1)
                    xterm = (float)(sf[b12] * eta * (1 - eps));
            } else if (t_bin == T - 1) {
                if (v_bin > -1 && v_bin < V - 1)
                    xterm = (float)(sf[b11] * (1 - eta) * (1 - eps) + sf[b21] * (1 - eta) * eps);
                else if (v_bin == -1)
                    xterm = (float)(sf[b21] * (1 - eta) * eps);
                else if (v_bin == V - 1)
                    xterm = (float)(sf[b11] * (1 - eta) * (1 - eps));
            }
            acc += (float)(xterm * delta * scale);
        }
        FBP[voxel] = acc;
    }
}

static int cmp_float(const void* a, const void* b)
{
    float x = *(const float*)a, y = *(const float*)b;
    return (x > y) - (x < y);
}

/* median_filter_2D (B.cu:7482-7521) */
void oracle_median_filter(const pct_config* cfg, int radius, const float* in, float* out)
{
    const int C = cfg->COLUMNS, R = cfg->ROWS, CR = C * R;
    const int side = 2 * radius + 1, count = side * side;
    float* nb = (float*)malloc(sizeof(float) * count);
    memset(out, 0, sizeof(float) * cfg->NUM_VOXELS);
    for (int s = 0; s < cfg->SLICES; s++)
        for (int col = radius; col < C - radius; col++)
            for (int row = radius; row < R - radius; row++) {
                int k = 0;
                for (int c = col - radius; c <= col + radius; c++)
                    for (int r = row - radius; r <= row + radius; r++) nb[k++] = in[c + r * C + s * CR];
                qsort(nb, count, sizeof(float), cmp_float);
                out[col + row * C + s * CR] = nb[count / 2];
            }
    free(nb);
}

/* initialize_hull_GPU (B.cu:6659) as 0/1 ints */
void oracle_initialize_hull(const pct_config* cfg, int32_t* hull)
{
    const int C = cfg->COLUMNS, R = cfg->ROWS;
    for (int voxel = 0; voxel < cfg->NUM_VOXELS; voxel++) {
        int rem = voxel % (C * R), row = rem / C, column = rem % C;
        double x = (column - C / 2 + 0.5) * cfg->VOXEL_WIDTH;
        double y = (R / 2 - row - 0.5) * cfg->VOXEL_HEIGHT;
        hull[voxel] = (sqf(x) + sqf(y) < sqf(cfg->RECON_CYL_RADIUS)) ? 1 : 0;
    }
}

/* ---- straight-line voxel walks (B.cu:11313-11462) ---- */
static int calc_voxel(double zero, double pos, double size)
{
    double q = fabs(pos - zero) / size;
    return q < 2147483647.0 ? (int)q : 2147483647;
}
static double edge_coordinate(double zero, int voxel_entered, double size, int inc, int step)
{
    int on_edge = (step == inc) ? voxel_entered : voxel_entered + 1;
    return zero + (inc * on_edge * size);
}
static double distance_remaining(double zero, double pos, int inc, int step, double size, int voxel)
{
    return fabs(edge_coordinate(zero, voxel + inc * step, size, inc, step) - pos);
}

/* SC_GPU / MSC_GPU / SM_GPU (B.cu:6681-7099); kind 0 = SC (hull as 0/1 ints, carved),
 * 1 = MSC, 2 = SM (counts).  Walks that would leave the grid on the negative side stop there
 * (the reference does not test it).  Returns the number of walks stopped by the step bound. */
int64_t oracle_hull_walks(const pct_config* cfg, int kind, int64_t n, const float* const g[10], const float* WEPL,
                          const uint8_t* missed, int32_t* image)
{
    const double X0 = -cfg->RECON_CYL_RADIUS, Y0 = cfg->RECON_CYL_RADIUS, Z0 = cfg->RECON_CYL_HEIGHT / 2;
    const int C = cfg->COLUMNS, R = cfg->ROWS, S = cfg->SLICES;
    const double VW = cfg->VOXEL_WIDTH, VH = cfg->VOXEL_HEIGHT, VT = cfg->VOXEL_THICKNESS;
    int64_t bounded = 0;
    for (int64_t i = 0; i < n; i++) {
        if (missed[i]) continue;
        float w = WEPL[i];
        if (kind == 0 && !((w <= cfg->SC_UPPER_THRESHOLD) && (w >= cfg->SC_LOWER_THRESHOLD))) continue;
        if (kind == 1 && !((w <= cfg->MSC_UPPER_THRESHOLD) && (w >= cfg->MSC_LOWER_THRESHOLD))) continue;
        if (kind == 2 && !(w >= cfg->SM_LOWER_THRESHOLD)) continue;
        float xe = g[0][i], ye = g[1][i], ze = g[2][i], xo = g[3][i], yo = g[4][i], zo = g[5][i];
        int xd = (xe <= xo) - (xe >= xo), yd = (ye <= yo) - (ye >= yo), zd = (ze <= zo) - (ze >= zo);
        double x = xe, y = ye, z = ze;
        int vx = calc_voxel(X0, xe, VW), vy = calc_voxel(Y0, ye, VH), vz = calc_voxel(Z0, ze, VT);
        int voxel = vx + vy * C + vz * C * R;
        double xg = distance_remaining(X0, x, 1, xd, VW, vx);
        double yg = distance_remaining(Y0, y, -1, yd, VH, vy);
        double zg = distance_remaining(Z0, z, -1, zd, VT, vz);
        double dy_dx = (float)((yo - ye) / (xo - xe)), dz_dx = (float)((zo - ze) / (xo - xe));
        double dz_dy = (float)((zo - ze) / (yo - ye)), dx_dy = (float)((xo - xe) / (yo - ye));
        double dx_dz = (float)((xo - xe) / (zo - ze)), dy_dz = (float)((yo - ye) / (zo - ze));
        int voxel_out = calc_voxel(X0, xo, VW) + calc_voxel(Y0, yo, VH) * C + calc_voxel(Z0, zo, VT) * C * R;
#define OUTSIDE (vx >= C || vy >= R || vz >= S || vx < 0 || vy < 0 || vz < 0)
#define MARK                                   \
    do {                                       \
        if (kind == 0) image[voxel] = 0;       \
        else image[voxel] += 1;                \
    } while (0)
        int end_walk = (voxel == voxel_out) || OUTSIDE;
        if (!end_walk) MARK;
        int steps = 0, max_steps = 4 * (C + R + S) + 16;
        while (!end_walk) {
            if (zd != 0) { /* take_3D_step_GPU */
                double xe_ = fabs(dz_dx) * xg, ye_ = fabs(dz_dy) * yg;
                if ((zg <= xe_) && (zg <= ye_)) {
                    vz -= zd;
                    z = edge_coordinate(Z0, vz, VT, -1, zd);
                    x = dx_dz * (z - ze) + xe;
                    y = dy_dz * (z - ze) + ye;
                    xg = distance_remaining(X0, x, 1, xd, VW, vx);
                    yg = distance_remaining(Y0, y, -1, yd, VH, vy);
                    zg = VT;
                } else if (xe_ <= ye_) {
                    vx += xd;
                    x = edge_coordinate(X0, vx, VW, 1, xd);
                    y = dy_dx * (x - xe) + ye;
                    z = dz_dx * (x - xe) + ze;
                    xg = VW;
                    yg = distance_remaining(Y0, y, -1, yd, VH, vy);
                    zg = distance_remaining(Z0, z, -1, zd, VT, vz);
                } else {
                    vy -= yd;
                    y = edge_coordinate(Y0, vy, VH, -1, yd);
                    x = dx_dy * (y - ye) + xe;
                    z = dz_dy * (y - ye) + ze;
                    xg = distance_remaining(X0, x, 1, xd, VW, vx);
                    yg = VH;
                    zg = distance_remaining(Z0, z, -1, zd, VT, vz);
                }
                if (xg == 0) { xg = VW; vx += xd; }
                if (yg == 0) { yg = VH; vy -= yd; }
                if (zg == 0) { zg = VT; vz -= zd; }
            } else { /* take_2D_step_GPU */
                double ye_ = fabs(dx_dy) * yg;
                if (xg <= ye_) {
                    vx += xd;
                    x = edge_coordinate(X0, vx, VW, 1, xd);
                    y = dy_dx * (x - xe) + ye;
                    xg = VW;
                    yg = distance_remaining(Y0, y, -1, yd, VH, vy);
                } else {
                    vy -= yd;
                    y = edge_coordinate(Y0, vy, VH, -1, yd);
                    x = dx_dy * (y - ye) + xe;
                    xg = distance_remaining(X0, x, 1, xd, VW, vx);
                    yg = VH;
                }
                if (xg == 0) { xg = VW; vx += xd; }
                if (yg == 0) { yg = VH; vy -= yd; }
            }
            if (vz < 0) vz = 0;
            voxel = vx + vy * C + vz * C * R;
            end_walk = (voxel == voxel_out) || OUTSIDE;
            if (!end_walk) MARK;
            if (++steps > max_steps) {
                bounded++;
                break;
            }
        }
#undef OUTSIDE
#undef MARK
    }
    return bounded;
}

/* MSC_edge_detection_GPU (B.cu:6911-6956) out of place; SM_edge_detection (B.cu:7100-7175);
 * kind 1 = MSC, 2 = SM; counts are replaced by the 0/1 hull. */
void oracle_edge_detection(const pct_config* cfg, int kind, int32_t* counts)
{
    const int C = cfg->COLUMNS, R = cfg->ROWS, S = cfg->SLICES, CR = C * R;
    int32_t* diff = (int32_t*)calloc((size_t)cfg->NUM_VOXELS, sizeof(int32_t));
    for (int voxel = 0; voxel < cfg->NUM_VOXELS; voxel++) {
        int s = voxel / CR, rem = voxel % CR, row = rem / C, col = rem % C;
        int mx = 0;
        if (row != 0 && row != R - 1 && col != 0 && col != C - 1)
            for (int r = row - 1; r <= row + 1; r++)
                for (int c = col - 1; c <= col + 1; c++) {
                    int d = counts[voxel] - counts[c + r * C + s * CR];
                    if (d > mx) mx = d;
                }
        diff[voxel] = mx;
    }
    int32_t* thr = (int32_t*)calloc((size_t)S, sizeof(int32_t));
    if (kind == 2)
        for (int s = 0; s < S; s++) {
            int mx = 0;
            for (int p = 0; p < CR; p++)
                if (diff[p + s * CR] > mx) {
                    mx = diff[p + s * CR];
                    thr[s] = counts[p + s * CR];
                }
        }
    const double half = (cfg->VOXEL_WIDTH > cfg->VOXEL_HEIGHT ? cfg->VOXEL_WIDTH : cfg->VOXEL_HEIGHT) / 2;
    for (int voxel = 0; voxel < cfg->NUM_VOXELS; voxel++) {
        int s = voxel / CR, rem = voxel % CR, row = rem / C, col = rem % C;
        float x = (float)((col - C / 2 + 0.5) * cfg->VOXEL_WIDTH), y = (float)((R / 2 - row - 0.5) * cfg->VOXEL_HEIGHT);
        int v;
        if (kind == 1) v = (diff[voxel] > cfg->MSC_DIFF_THRESH || counts[voxel] > cfg->MSC_DIFF_THRESH) ? 0 : 1;
        else v = (counts[voxel] > cfg->SM_SCALE_THRESHOLD * thr[s]) ? 1 : 0;
        if (x * x + y * y >= sqf(cfg->RECON_CYL_RADIUS - half)) v = 0;
        diff[voxel] = v;
    }
    memcpy(counts, diff, sizeof(int32_t) * cfg->NUM_VOXELS);
    free(diff);
    free(thr);
}

/* find_MLP_endpoints_GPU (B.cu:7581-7773) */
static int find_endpoint(const pct_config* cfg, const uint8_t* image, double x_start, double y_start, double z_start,
                         double xy_angle, double xz_angle, double* xo, double* yo, double* zo, int* voxel_x,
                         int* voxel_y, int* voxel_z, int entering)
{
    const double X0 = -cfg->RECON_CYL_RADIUS, Y0 = cfg->RECON_CYL_RADIUS, Z0 = cfg->RECON_CYL_HEIGHT / 2;
    const int C = cfg->COLUMNS, R = cfg->ROWS, S = cfg->SLICES;
    const double VW = cfg->VOXEL_WIDTH, VH = cfg->VOXEL_HEIGHT, VT = cfg->VOXEL_THICKNESS;
    double x = x_start, y = y_start, z = z_start;
    int hit = 0;
    if (!entering) xy_angle += PI_;
    int xd = (cos(xy_angle) >= 0) - (cos(xy_angle) <= 0);
    int yd = (sin(xy_angle) >= 0) - (sin(xy_angle) <= 0);
    int zd = (sin(xz_angle) >= 0) - (sin(xz_angle) <= 0);
    if (xd < 0) zd *= -1;
    int vx = calc_voxel(X0, x, VW), vy = calc_voxel(Y0, y, VH), vz = calc_voxel(Z0, z, VT);
    double xg = distance_remaining(X0, x, 1, xd, VW, vx);
    double yg = distance_remaining(Y0, y, -1, yd, VH, vy);
    double zg = distance_remaining(Z0, z, -1, zd, VT, vz);
    int voxel = vx + (vy + vz * R) * C;
    double delta_yx = fabs(tan(xy_angle)), delta_zx = fabs(tan(xz_angle)), delta_zy = fabs(tan(xz_angle) / tan(xy_angle));
    double dy_dx = tan(xy_angle), dz_dx = tan(xz_angle), dz_dy = tan(xz_angle) / tan(xy_angle);
    double dx_dy = powf((float)tan(xy_angle), -1.0f), dx_dz = powf((float)tan(xz_angle), -1.0f);
    double dy_dz = tanf((float)xy_angle) / tan(xz_angle);
#define OUT (vx >= C || vy >= R || vz >= S || vx < 0 || vy < 0 || vz < 0)
    int outside = OUT;
    if (!outside) hit = image[voxel] == 1;
    int end_walk = outside || hit;
    int steps = 0, max_steps = 2 * (C + R + S) + 16;
    while (!end_walk && steps++ < max_steps) {
        if (zd != 0) {
            double xe_ = delta_zx * xg, ye_ = delta_zy * yg;
            if ((zg <= xe_) && (zg <= ye_)) {
                vz -= zd;
                z = edge_coordinate(Z0, vz, VT, -1, zd);
                x = dx_dz * (z - z_start) + x_start;
                y = dy_dz * (z - z_start) + y_start;
                xg = distance_remaining(X0, x, 1, xd, VW, vx);
                yg = distance_remaining(Y0, y, -1, yd, VH, vy);
                zg = VT;
            } else if (xe_ <= ye_) {
                vx += xd;
                x = edge_coordinate(X0, vx, VW, 1, xd);
                y = dy_dx * (x - x_start) + y_start;
                z = dz_dx * (x - x_start) + z_start;
                xg = VW;
                yg = distance_remaining(Y0, y, -1, yd, VH, vy);
                zg = distance_remaining(Z0, z, -1, zd, VT, vz);
            } else {
                vy -= yd;
                y = edge_coordinate(Y0, vy, VH, -1, yd);
                x = dx_dy * (y - y_start) + x_start;
                z = dz_dy * (y - y_start) + z_start;
                xg = distance_remaining(X0, x, 1, xd, VW, vx);
                yg = VH;
                zg = distance_remaining(Z0, z, -1, zd, VT, vz);
            }
            if (xg == 0) { xg = VW; vx += xd; }
            if (yg == 0) { yg = VH; vy -= yd; }
            if (zg == 0) { zg = VT; vz -= zd; }
            if (vz < 0) vz = 0;
        } else {
            double ye_ = yg / delta_yx;
            if (xg <= ye_) {
                vx += xd;
                x = edge_coordinate(X0, vx, VW, 1, xd);
                y = dy_dx * (x - x_start) + y_start;
                xg = VW;
                yg = distance_remaining(Y0, y, -1, yd, VH, vy);
            } else {
                vy -= yd;
                y = edge_coordinate(Y0, vy, VH, -1, yd);
                x = dx_dy * (y - y_start) + x_start;
                xg = distance_remaining(X0, x, 1, xd, VW, vx);
                yg = VH;
            }
            if (xg == 0) { xg = VW; vx += xd; }
            if (yg == 0) { yg = VH; vy -= yd; }
        }
        voxel = vx + vy * C + vz * C * R;
        outside = OUT;
        if (!outside) hit = image[voxel] == 1;
        end_walk = outside || hit;
    }
#undef OUT
    if (hit) {
        *xo = x;
        *yo = y;
        *zo = z;
    }
    *voxel_x = vx;
    *voxel_y = vy;
    *voxel_z = vz;
    return hit;
}

/* collect_MLP_endpoints_GPU_nobool (B.cu:7819-7854): g is updated in place */
void oracle_collect_mlp_endpoints(const pct_config* cfg, const uint8_t* hull, int64_t n, float* const g[10],
                                  uint32_t* first_MLP_voxel)
{
    for (int64_t i = 0; i < n; i++) {
        int vx = 0, vy = 0, vz = 0, ux = 0, uy = 0, uz = 0;
        double xin = 0, yin = 0, zin = 0, xout = 0, yout = 0, zout = 0;
        int entered = find_endpoint(cfg, hull, g[0][i], g[1][i], g[2][i], g[6][i], g[7][i], &xin, &yin, &zin, &vx, &vy, &vz, 1);
        int exited = find_endpoint(cfg, hull, g[3][i], g[4][i], g[5][i], g[8][i], g[9][i], &xout, &yout, &zout, &ux, &uy, &uz, 0);
        if (entered && exited) {
            first_MLP_voxel[i] = (uint32_t)(vx + cfg->COLUMNS * vy + cfg->ROWS * cfg->COLUMNS * vz);
            g[0][i] = (float)xin;
            g[1][i] = (float)yin;
            g[2][i] = (float)zin;
            g[3][i] = (float)xout;
            g[4][i] = (float)yout;
            g[5][i] = (float)zout;
        } else {
            first_MLP_voxel[i] = (uint32_t)cfg->NUM_VOXELS;
        }
    }
}
