// pct_mlp.cuh -- the most-likely-path (MLP) walk, exact mode.
//
// mlp_walk_exact() restates find_MLP_path_GPU_tabulated (B.cu:9104-9262) operation for
// operation in IEEE double: same table indices, same operand order, same float round trips
// (and the same CUDA powf/sinf/cosf calls) where the reference drops to float.  The translation
// unit that includes this header is compiled with -fmad=false so no multiply-add pair is fused.
// The CPU oracle squares with the correctly rounded float product instead of CUDA's powf, so the
// two voxel lists can differ where an MLP point falls within ~1e-7 cm of a voxel boundary; the
// parity tests count those ties.
//
// Two restructurings that do not change a single rounding:
//  * the Sigma_1 terms of step k depend only on k (u_1 = k*MLP_U_STEP), so they are read from a
//    per-step table built once on the device with the same expressions (build_step_table_kernel);
//  * the running depth (depth_2_go -= MLP_U_STEP) and position (u_shifted += MLP_U_STEP) are
//    carried exactly as the reference carries them.
#pragma once

#include "pct_common.cuh"
#include "pct_tables.h"

namespace pct {

// Maximum MLP voxel-list length handled per history: MLP_U_STEP >= 0.03125 cm (half of the
// reference's smallest 0.0625 cm voxel) over the 40 cm polynomial-table range gives
// <= 1281 entries (the reference's MAX_INTERSECTIONS is 1280, B.h:342).
constexpr int kPathCap = PCT_MLP_PATH_CAP;

// Flags reported per history (same bits as the oracle).
enum WalkFlag : unsigned { kFlagVoxelOOB = 1u, kFlagPathOverflow = 2u, kFlagTableRange = 4u };

struct WalkResult {
    int n;          // number_of_intersections (capped at kPathCap)
    unsigned flags;
    double chord;   // effective_chord_length
    double axk;     // a_i_dot_x_k_partially: sum of x over the path
    double aia;     // a_i_dot_a_i_partially: powf(chord, 2)
};

// powf(v, 2) on a double argument, as the reference writes it: v is rounded to float and CUDA's
// powf is called.  CUDA's powf(f, 2.0f) is not always the correctly rounded product f*f (the
// device self-test pct_selftest_powf_square counts about 6% of inputs one float ulp away), so the
// call is kept to reproduce the reference's values.
__device__ __forceinline__ double powf_square(double v)
{
    return (double)powf((float)v, 2.0f);
}

// calculate_voxel_GPU (B.cu:11091): int(|position - zero| / size); -1 when it does not fit an int.
__device__ __forceinline__ int voxel_index_1d(double zero, double pos, double size)
{
    const double q = fabs(pos - zero) / size;
    return (q < 2147483647.0) ? (int)q : -1;
}

// EffectiveChordLength_GPU (B.cu:8873-8894).  sinf/cosf receive float arguments; the sum of two
// float results is a float addition, as in the reference.
__device__ __forceinline__ double effective_chord_length(const Geometry& g, double abs_angle_t, double abs_angle_v)
{
    const double PI = ref_pi();
    const double eff_angle_t = abs_angle_t - ((int)(abs_angle_t / (PI / 2))) * (PI / 2);
    const double eff_angle_v = fabs(abs_angle_v);
    double step_fraction = g.mlp_u_step / g.voxel_width;
    const float s2t = sinf((float)(2 * eff_angle_t));
    const float ct_plus_st = __fadd_rn(cosf((float)eff_angle_t), sinf((float)eff_angle_t));
    const double chord_length_2D =
        (1 / 3.0) * ((step_fraction * step_fraction * s2t - 6) / (step_fraction * s2t - 2 * ct_plus_st) +
                     step_fraction * step_fraction * s2t / (2 * ct_plus_st));
    const double mean_pixel_width = g.voxel_width / ct_plus_st;
    const double height_fraction = g.voxel_thickness / mean_pixel_width;
    step_fraction = g.mlp_u_step / mean_pixel_width;
    const float s2v = sinf((float)(2 * eff_angle_v));
    const float cv = cosf((float)eff_angle_v);
    const float sv = sinf((float)eff_angle_v);
    const double chord_length_3D =
        (1 / 3.0) * ((step_fraction * step_fraction * s2v - 6 * height_fraction) /
                         (step_fraction * s2v - 2 * (height_fraction * cv + sv)) +
                     step_fraction * step_fraction * s2v / (2 * (height_fraction * cv + sv)));
    return g.voxel_width * chord_length_2D * chord_length_3D;
}

// u_2 = |u_out - u_in| of a history in its entry-angle frame, exactly as the walk computes it.
__device__ __forceinline__ double mlp_u_extent(const Geometry& g, const Tables& tab, double x_in, double y_in,
                                               double x_out, double y_out, double xy_entry_angle)
{
    unsigned trig_index = (unsigned)((xy_entry_angle - g.trig_min) / g.trig_step + 0.5);
    double sin_term = __ldg(tab.sin_table + trig_index);
    double cos_term = __ldg(tab.cos_table + trig_index);
    double u_in = cos_term * x_in + sin_term * y_in;
    double u_out = cos_term * x_out + sin_term * y_out;
    if (u_in > u_out) {
        trig_index = (unsigned)((xy_entry_angle + ref_pi() - g.trig_min) / g.trig_step + 0.5);
        sin_term = __ldg(tab.sin_table + trig_index);
        cos_term = __ldg(tab.cos_table + trig_index);
        u_in = cos_term * x_in + sin_term * y_in;
        u_out = cos_term * x_out + sin_term * y_out;
    }
    return fabs(u_out - u_in);
}

// One history's MLP.  emit(j, voxel) is called for every path entry j in order.  With kSumX the
// walk also sums the padded image x over the path (reads beyond it are reported and count as 0);
// without it x is not touched (the voxel list does not depend on the image).
template <bool kSumX, class Emit>
__device__ __forceinline__ WalkResult mlp_walk_exact(const Geometry& g, const Tables& tab,
                                                     const StepConst* __restrict__ steps, int kmax,
                                                     const float* __restrict__ x, uint32_t first_MLP_voxel,
                                                     double x_in_object, double y_in_object, double z_in_object,
                                                     double x_out_object, double y_out_object, double z_out_object,
                                                     double xy_entry_angle, double xz_entry_angle,
                                                     double xy_exit_angle, double xz_exit_angle, Emit emit)
{
    const double PI = ref_pi();
    const double s = g.mlp_u_step;
    WalkResult r;
    r.flags = 0;

    unsigned trig_index = (unsigned)((xy_entry_angle - g.trig_min) / g.trig_step + 0.5);
    double sin_term = __ldg(tab.sin_table + trig_index);
    double cos_term = __ldg(tab.cos_table + trig_index);
    double u_in_object = cos_term * x_in_object + sin_term * y_in_object;
    double u_out_object = cos_term * x_out_object + sin_term * y_out_object;
    if (u_in_object > u_out_object) {
        xy_entry_angle += PI;
        xy_exit_angle += PI;
        trig_index = (unsigned)((xy_entry_angle - g.trig_min) / g.trig_step + 0.5);
        sin_term = __ldg(tab.sin_table + trig_index);
        cos_term = __ldg(tab.cos_table + trig_index);
        u_in_object = cos_term * x_in_object + sin_term * y_in_object;
        u_out_object = cos_term * x_out_object + sin_term * y_out_object;
    }
    const double t_in_object = cos_term * y_in_object - sin_term * x_in_object;
    const double t_out_object = cos_term * y_out_object - sin_term * x_out_object;
    const double T_2_1 = xy_exit_angle - xy_entry_angle;
    const double V_2_1 = xz_exit_angle - xz_entry_angle;
    const double u_2 = fabs(u_out_object - u_in_object);
    double depth_2_go = u_2 - s;
    double u_shifted = u_in_object;

    const bool tables_ok = (u_2 / kPolyTableStep + 0.5) < (double)g.poly_elements && depth_2_go >= 0;
    unsigned sigma_2_index = 0, u_2_poly_index = 0;
    if (tables_ok) {
        sigma_2_index = (unsigned)(depth_2_go / kCoeffTableStep + 0.5);
        u_2_poly_index = (unsigned)(u_2 / kPolyTableStep + 0.5);
    } else {
        r.flags |= kFlagTableRange;
    }
    const double u_2_poly_3_12 = __ldg(tab.poly_3_12 + u_2_poly_index);
    const double u_2_poly_2_6 = __ldg(tab.poly_2_6 + u_2_poly_index);
    const double u_2_poly_1_2 = __ldg(tab.poly_1_2 + u_2_poly_index);
    const double u_2_sq = powf_square(u_2);
    const double two_u_2 = 2 * u_2;

    int n = 0;
    uint32_t last = first_MLP_voxel;
    emit(n, first_MLP_voxel);
    n++;
    r.chord = effective_chord_length(g, (xy_entry_angle + xy_exit_angle) / 2.0, (xz_entry_angle + xz_exit_angle) / 2.0);
    r.axk = 0.0;
    if (first_MLP_voxel < (uint32_t)g.padded_voxels) {
        if (kSumX) r.axk = (double)__ldg(x + first_MLP_voxel);
    } else {
        r.flags |= kFlagVoxelOOB;
    }
    r.aia = powf_square(r.chord);

    int k = 1;
    while (tables_ok && depth_2_go > s) {
        if (k > kmax) {  // cannot happen while the u_2 index is inside the tables
            r.flags |= kFlagTableRange;
            break;
        }
        const StepConst st = steps[k];
        const double sigma_t2 = u_2_poly_3_12 - u_2_sq * st.p12 + two_u_2 * st.p23 - st.p34;
        const double sigma_t2_theta2 = u_2_poly_2_6 - u_2 * st.p12 + st.p23;
        const double sigma_theta2 = u_2_poly_1_2 - st.p12;
        const double determinant_Sigma_2 =
            __ldg(tab.scattering_table + sigma_2_index) * (sigma_t2 * sigma_theta2 - powf_square(sigma_t2_theta2));
        const double Sigma_2I_0 = sigma_theta2 / determinant_Sigma_2;
        const double Sigma_2I_1 = sigma_t2_theta2 / determinant_Sigma_2;
        const double Sigma_2I_2 = sigma_t2 / determinant_Sigma_2;

        const double first_term_common_24_1 = Sigma_2I_0 * depth_2_go - Sigma_2I_1;
        const double first_term_0 = st.s1i0 + Sigma_2I_0;
        const double first_term_1 = first_term_common_24_1 - st.s1i1;
        const double first_term_2 = depth_2_go * Sigma_2I_0 - st.s1i1 - Sigma_2I_1;
        const double first_term_3 = st.s1i2 + Sigma_2I_2 + depth_2_go * (first_term_common_24_1 - Sigma_2I_1);
        const double determinant_first_term = first_term_0 * first_term_3 - first_term_1 * first_term_2;

        double second_term_common_3 = Sigma_2I_0 * t_out_object - Sigma_2I_1 * T_2_1;
        double second_term_0 = st.s1i0 * t_in_object + second_term_common_3;
        double second_term_1 = depth_2_go * second_term_common_3 + Sigma_2I_2 * T_2_1 -
                               Sigma_2I_1 * t_out_object - st.s1i1 * t_in_object;
        const double t_1 = (first_term_3 * second_term_0 - first_term_1 * second_term_1) / determinant_first_term;

        second_term_common_3 = Sigma_2I_0 * z_out_object - Sigma_2I_1 * V_2_1;
        second_term_0 = st.s1i0 * z_in_object + second_term_common_3;
        second_term_1 = depth_2_go * second_term_common_3 + Sigma_2I_2 * V_2_1 -
                        Sigma_2I_1 * z_out_object - st.s1i1 * z_in_object;
        const double v_1 = (first_term_3 * second_term_0 - first_term_1 * second_term_1) / determinant_first_term;

        u_shifted += s;
        const double x_1 = cos_term * u_shifted - sin_term * t_1;
        const double y_1 = sin_term * u_shifted + cos_term * t_1;
        const int vx = voxel_index_1d(g.x_zero, x_1, g.voxel_width);
        const int vy = voxel_index_1d(g.y_zero, y_1, g.voxel_height);
        const int vz = voxel_index_1d(g.z_zero, v_1, g.voxel_thickness);
        long long v64 = (long long)vx + (long long)vy * g.columns + (long long)vz * g.columns * g.rows;
        if (vx < 0 || vy < 0 || vz < 0 || v64 > 0x7fffffffLL) v64 = 0x7fffffffLL;
        const uint32_t voxel = (uint32_t)v64;
        if (voxel != last) {
            if (n < kPathCap) emit(n, voxel);
            else r.flags |= kFlagPathOverflow;
            if (voxel < (uint32_t)g.padded_voxels) {
                if (kSumX) r.axk += (double)__ldg(x + voxel);
            } else {
                r.flags |= kFlagVoxelOOB;
            }
            last = voxel;
            n++;
        }
        depth_2_go -= s;
        sigma_2_index -= g.sigma_index_step;
        k++;
    }
    r.n = n < kPathCap ? n : kPathCap;
    return r;
}

}  // namespace pct
