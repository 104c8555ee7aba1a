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
// Path storage is written in chunks of 8 entries (one 32-byte sector); kPathCap is a multiple.
constexpr int kPathChunk = 8;
static_assert(kPathCap % kPathChunk == 0, "path cap must be a multiple of the write chunk");
static_assert(kSCurveEntries >= kPathCap, "the S-curve table covers every path index");

// Flags reported per history (same bits as the oracle).
enum WalkFlag : unsigned { kFlagVoxelOOB = 1u, kFlagPathOverflow = 2u, kFlagTableRange = 4u };

// Adds one history's walk flags to the context counters read by pct_get_counters.
__device__ __forceinline__ void count_flags(unsigned flags, unsigned long long* counters)
{
    if (flags & kFlagVoxelOOB) atomicAdd(counters + kCntVoxelOOB, 1ull);
    if (flags & kFlagPathOverflow) atomicAdd(counters + kCntPathOverflow, 1ull);
    if (flags & kFlagTableRange) atomicAdd(counters + kCntTableRange, 1ull);
}

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

// The same index without the division in the common case.  p = |pos - zero| * RN(1/size) is
// within 3.4e-16 relative of the exact quotient, and the reference's RN(quotient) is within
// 1.2e-16 of it; when p is farther than 1e-14 (relative) from every integer, no integer can lie
// between p and RN(quotient), so floor(p) == (int)RN(quotient).  Otherwise (about 2e-14 of calls,
// and when p = 0) the exact division decides.
__device__ __forceinline__ int voxel_index_1d_fast(double zero, double pos, double size, double inv_size)
{
    const double a = fabs(pos - zero);
    const double p = a * inv_size;
    if (p < 2147483000.0) {
        const double f = floor(p);
        const double guard = p * 1.0e-14;
        if (p - f > guard && (f + 1.0) - p > guard) return (int)f;
    }
    return voxel_index_1d(zero, pos, size);
}

// EffectiveChordLength_GPU (B.cu:8873-8894).  sinf/cosf receive float arguments; the sum of two
// float results is a float addition, as in the reference.  The reference is compiled with
// multiply-add contraction, which fuses a product into the addition that consumes it; where both
// operands of an addition are products it fuses the one with fewer uses.  The fused forms are
// written out here (this translation unit does not contract): eff_angle_t = fma(-k, PI/2, angle),
// the numerators and denominators fma(a, b, -c), and the 3-D numerator fma(-6, h, sf^2 sin 2v),
// whose other product sf^2 sin 2v is also used by the last term.  Comparing the possible forms
// with the reference's chords on the head grid (2000 histories, tests/golden/ref_mlp_head.npz)
// singles out the 3-D numerator's; the others do not change a chord there and follow the same rule.
__device__ __forceinline__ double effective_chord_length(const Geometry& g, double abs_angle_t, double abs_angle_v)
{
    const double PI = ref_pi();
    const int quadrants = (int)(abs_angle_t / (PI / 2));
    const double eff_angle_t = __fma_rn(-(double)quadrants, PI / 2, abs_angle_t);
    const double eff_angle_v = fabs(abs_angle_v);
    double step_fraction = g.mlp_u_step / g.voxel_width;
    const float s2t = sinf((float)(2 * eff_angle_t));
    const float ct_plus_st = __fadd_rn(cosf((float)eff_angle_t), sinf((float)eff_angle_t));
    const double sf2_s2t = __dmul_rn(__dmul_rn(step_fraction, step_fraction), (double)s2t);
    const double chord_length_2D =
        (1 / 3.0) * (__fma_rn(__dmul_rn(step_fraction, step_fraction), (double)s2t, -6.0) /
                         __fma_rn(step_fraction, (double)s2t, -(double)(2 * ct_plus_st)) +
                     sf2_s2t / (double)(2 * ct_plus_st));
    const double mean_pixel_width = g.voxel_width / ct_plus_st;
    const double height_fraction = g.voxel_thickness / mean_pixel_width;
    step_fraction = g.mlp_u_step / mean_pixel_width;
    const float s2v = sinf((float)(2 * eff_angle_v));
    const float cv = cosf((float)eff_angle_v);
    const float sv = sinf((float)eff_angle_v);
    const double inner2 = 2 * __fma_rn(height_fraction, (double)cv, (double)sv);
    const double sf2_s2v = __dmul_rn(__dmul_rn(step_fraction, step_fraction), (double)s2v);
    const double chord_length_3D =
        (1 / 3.0) * (__fma_rn(-6.0, height_fraction, sf2_s2v) / __fma_rn(step_fraction, (double)s2v, -inner2) +
                     sf2_s2v / inner2);
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

// Per-history constants of the MLP loop (B.cu:9104-9158).
struct MlpHistory {
    double sin_term, cos_term;
    double t_in, t_out, z_in, z_out, T_2_1, V_2_1;
    double u_2, u_2_sq, two_u_2;
    double u_2_poly_3_12, u_2_poly_2_6, u_2_poly_1_2;
    double mag_tv;  // max(|t_in| + |t_out| + |T_2_1|, |z_in| + |z_out| + |V_2_1|): the guarded fast point's bound
};
constexpr int kHistoryFields = 15;
// 1: the walk parks its chord in the stash slot after the history's constants while it loops; 0 keeps
// it in registers.
#ifndef PCT_STASH_CHORD
#define PCT_STASH_CHORD 1
#endif
static_assert(sizeof(MlpHistory) == kHistoryFields * sizeof(double), "MlpHistory is 15 doubles");

// The constants of a history parked in shared memory: field f of this thread at byte address
// addr + f * stride.  The loads are volatile, so they stay inside the loop trip that uses them and
// the constants are not held in registers across trips.
__device__ __forceinline__ void history_stash_store(uint32_t addr, uint32_t stride, const MlpHistory& h)
{
    const double* f = reinterpret_cast<const double*>(&h);
#pragma unroll
    for (int i = 0; i < kHistoryFields; i++)
        asm volatile("st.shared.f64 [%0], %1;" ::"r"(addr + i * stride), "d"(f[i]) : "memory");
}

__device__ __forceinline__ MlpHistory history_stash_load(uint32_t addr, uint32_t stride)
{
    MlpHistory h;
    double* f = reinterpret_cast<double*>(&h);
#pragma unroll
    for (int i = 0; i < kHistoryFields; i++) asm volatile("ld.shared.f64 %0, [%1];" : "=d"(f[i]) : "r"(addr + i * stride));
    return h;
}

// Field numbers of MlpHistory (declaration order) and two ways of reading a field: from the
// struct (registers) or from the shared-memory stash, loaded where it is used.
enum HistoryField { kHSin, kHCos, kHTin, kHTout, kHZin, kHZout, kHT21, kHV21, kHU2, kHU2sq, kHTwoU2, kHP312, kHP26, kHP12, kHMag };

struct HistoryInRegisters {
    const MlpHistory& h;
    template <int F>
    __device__ __forceinline__ double get() const
    {
        static_assert(F >= 0 && F < kHistoryFields, "field");
        return reinterpret_cast<const double*>(&h)[F];
    }
};

struct HistoryInShared {
    uint32_t addr, stride;
    template <int F>
    __device__ __forceinline__ double get() const
    {
        static_assert(F >= 0 && F < kHistoryFields, "field");
        double v;
        asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(addr + F * stride));
        return v;
    }
};

// MLP point (t_1, v_1) of one loop iteration (B.cu:9180-9226): Sigma_2 from the tables, its
// inverse, the 2x2 solve for t and v.  Same operations, same order as the reference.
struct Sigma2 {
    double sigma_t2, sigma_t2_theta2, sigma_theta2, determinant;
};

// The Sigma_2 moments of one point and their determinant (B.cu:9180-9186), in the reference's
// operations and order.
template <class HA>
__device__ __forceinline__ Sigma2 sigma2_moments(const HA& h, const StepConst& st, const double* __restrict__ scattering,
                                                 unsigned sigma_2_index)
{
    Sigma2 m;
    m.sigma_t2 = h.template get<kHP312>() - h.template get<kHU2sq>() * st.p12 + h.template get<kHTwoU2>() * st.p23 - st.p34;
    m.sigma_t2_theta2 = h.template get<kHP26>() - h.template get<kHU2>() * st.p12 + st.p23;
    m.sigma_theta2 = h.template get<kHP12>() - st.p12;
    m.determinant = __ldg(scattering + sigma_2_index) * (m.sigma_t2 * m.sigma_theta2 - powf_square(m.sigma_t2_theta2));
    return m;
}

__device__ __forceinline__ Sigma2 sigma2_moments(const MlpHistory& h, const StepConst& st,
                                                 const double* __restrict__ scattering, unsigned sigma_2_index)
{
    return sigma2_moments(HistoryInRegisters{h}, st, scattering, sigma_2_index);
}

__device__ __forceinline__ void mlp_point_rest(const MlpHistory& h, const StepConst& st, const Sigma2& m,
                                               double depth_2_go, double& t_1, double& v_1)
{
    const double sigma_t2 = m.sigma_t2, sigma_t2_theta2 = m.sigma_t2_theta2, sigma_theta2 = m.sigma_theta2;
    const double determinant_Sigma_2 = m.determinant;
    const double Sigma_2I_0 = sigma_theta2 / determinant_Sigma_2;
    const double Sigma_2I_1 = sigma_t2_theta2 / determinant_Sigma_2;
    const double Sigma_2I_2 = sigma_t2 / determinant_Sigma_2;

    const double first_term_common_24_1 = Sigma_2I_0 * depth_2_go - Sigma_2I_1;
    const double first_term_0 = st.s1i0 + Sigma_2I_0;
    const double first_term_1 = first_term_common_24_1 - st.s1i1;
    const double first_term_2 = depth_2_go * Sigma_2I_0 - st.s1i1 - Sigma_2I_1;
    const double first_term_3 = st.s1i2 + Sigma_2I_2 + depth_2_go * (first_term_common_24_1 - Sigma_2I_1);
    const double determinant_first_term = first_term_0 * first_term_3 - first_term_1 * first_term_2;

    double second_term_common_3 = Sigma_2I_0 * h.t_out - Sigma_2I_1 * h.T_2_1;
    double second_term_0 = st.s1i0 * h.t_in + second_term_common_3;
    double second_term_1 =
        depth_2_go * second_term_common_3 + Sigma_2I_2 * h.T_2_1 - Sigma_2I_1 * h.t_out - st.s1i1 * h.t_in;
    t_1 = (first_term_3 * second_term_0 - first_term_1 * second_term_1) / determinant_first_term;

    second_term_common_3 = Sigma_2I_0 * h.z_out - Sigma_2I_1 * h.V_2_1;
    second_term_0 = st.s1i0 * h.z_in + second_term_common_3;
    second_term_1 =
        depth_2_go * second_term_common_3 + Sigma_2I_2 * h.V_2_1 - Sigma_2I_1 * h.z_out - st.s1i1 * h.z_in;
    v_1 = (first_term_3 * second_term_0 - first_term_1 * second_term_1) / determinant_first_term;
}

__device__ __forceinline__ void mlp_point(const MlpHistory& h, const StepConst& st, const double* __restrict__ scattering,
                                          double depth_2_go, unsigned sigma_2_index, double& t_1, double& v_1)
{
    mlp_point_rest(h, st, sigma2_moments(h, st, scattering, sigma_2_index), depth_2_go, t_1, v_1);
}

// ---- Guarded fast points (exact mode, EXACT_FAST_POINTS = 1) ----------------------------------
// Only the voxel of an MLP point enters the voxel list, so a point needs the reference's rounding
// only when it lies near a voxel face.  mlp_point_fast keeps the part of the point where the
// reference's cancellation lives -- the Sigma_2 moments and their determinant, computed by the
// caller with the reference's operations in its order -- and evaluates the rest (Sigma_2's
// inverse, M = Sigma_1^-1 + R_1^T Sigma_2^-1 R_1, its determinant, the two solves and the
// rotation) with refined reciprocals and fused multiply-adds: about half the FP64 instructions
// of five IEEE divisions and a shorter dependency chain.  Alongside it bounds the difference
// between its result and the reference's by first-order forward error analysis: every quantity q
// carries a magnitude M(q), the sum of the absolute values of the terms it is built from, and
// both evaluations' rounding errors are at most a few units in the last place times M(q); kBoundK
// (2^-40, about 8000 units) covers both with a wide margin.  For t = num / det the bound is
// K (M(num) + |t| M(det)) / |det|, valid while K M(det) is well below |det| (checked).  A point
// whose bound does not keep every coordinate clear of a voxel face, or whose M is not
// well-conditioned, returns false and is recomputed in the reference's order, so the voxel list
// is the reference's either way.
constexpr double kBoundK = 9.094947017729282e-13;  // 2^-40
#ifndef PCT_FAST_POINTS
#define PCT_FAST_POINTS 1  // 0 compiles the guarded fast points out (every point in the reference's order)
#endif

// rcp.approx.ftz.f64 (a coarse hardware reciprocal of the high word) refined by two Newton steps:
// within a few units in the last place of 1/b for the normal values it sees here.
__device__ __forceinline__ double rcp_refined(double b)
{
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(b));
    double e = __fma_rn(-b, r, 1.0);
    r = __fma_rn(r, e, r);
    e = __fma_rn(-b, r, 1.0);
    return __fma_rn(r, e, r);
}

// The three indices int(|pos - zero| / size) of (x, y, z) when every coordinate is provably more than
// err (cm) away from a voxel face, with the subtraction and scaling roundings of either evaluation
// included; false otherwise.  One tolerance serves all three axes: (K max_a + err) max(1/size) is at
// least each axis's own (K a + err) / size.  The distance to the nearest face, |p - rint(p)|, is
// exact (p and rint(p) are multiples of p's last place, and the difference is at most 1/2), and the
// index is the truncation int(p), as the reference writes it.  The conditions are combined without
// branches: every point of a warp is almost always proven.
__device__ __forceinline__ bool guarded_indices(const Geometry& g, double x, double y, double z, double err,
                                                int& vx, int& vy, int& vz)
{
    const double ax = fabs(__dsub_rn(x, g.x_zero)), ay = fabs(__dsub_rn(y, g.y_zero)), az = fabs(__dsub_rn(z, g.z_zero));
    const double amax = fmax(fmax(ax, ay), az);
    const double tol = __dmul_rn(__fma_rn(kBoundK, amax, err), g.inv_voxel_max);
    const double px = __dmul_rn(ax, g.inv_voxel_width), py = __dmul_rn(ay, g.inv_voxel_height),
                 pz = __dmul_rn(az, g.inv_voxel_thickness);
    const bool ok = (__dmul_rn(amax, g.inv_voxel_max) < 2147483000.0) & (fabs(__dsub_rn(px, rint(px))) > tol) &
                    (fabs(__dsub_rn(py, rint(py))) > tol) & (fabs(__dsub_rn(pz, rint(pz))) > tol);
    if (!ok) return false;
    vx = (int)px;
    vy = (int)py;
    vz = (int)pz;
    return true;
}

// The fast point and its voxel (see above); false when the bound cannot prove the voxel.
// h gives the history's constants (HistoryInRegisters or HistoryInShared); its mag_tv is
// |t_in| + |t_out| + |T_2_1| and the same for v, the larger of the two.
template <class HA>
__device__ __forceinline__ bool mlp_point_fast(const Geometry& g, const HA& h, const StepConst& st, double sigma_t2,
                                               double sigma_t2_theta2, double sigma_theta2, double det2, double d,
                                               double u_shifted, uint32_t& voxel)
{
    const double r2 = rcp_refined(det2);
    const double S0 = __dmul_rn(sigma_theta2, r2), S1 = __dmul_rn(sigma_t2_theta2, r2), S2 = __dmul_rn(sigma_t2, r2);
    const double c = __fma_rn(S0, d, -S1);
    const double m0 = __dadd_rn(st.s1i0, S0);
    const double m1 = __dsub_rn(c, st.s1i1);
    const double m3 = __fma_rn(d, __dsub_rn(c, S1), __dadd_rn(st.s1i2, S2));
    const double det = __fma_rn(m0, m3, -__dmul_rn(m1, m1));
    // magnitudes
    const double aS0 = fabs(S0), aS1 = fabs(S1), aS2 = fabs(S2);
    const double Mc = __fma_rn(aS0, d, aS1);
    const double Mm0 = __dadd_rn(fabs(st.s1i0), aS0);
    const double Mm1 = __dadd_rn(Mc, fabs(st.s1i1));
    const double Mm3 = __fma_rn(d, __dadd_rn(Mc, aS1), __dadd_rn(fabs(st.s1i2), aS2));
    const double Mdet = __fma_rn(Mm0, Mm3, __dmul_rn(Mm1, Mm1));
    const double adet = fabs(det);
    if (!(__dmul_rn(4.0 * kBoundK, Mdet) < adet)) return false;
    const double rdet = rcp_refined(det);
    // the right-hand sides and the solves for t and v
    double c3 = __fma_rn(S0, h.template get<kHTout>(), -__dmul_rn(S1, h.template get<kHT21>()));
    double r0 = __fma_rn(st.s1i0, h.template get<kHTin>(), c3);
    double r1 = __fma_rn(d, c3, __fma_rn(S2, h.template get<kHT21>(), -__fma_rn(S1, h.template get<kHTout>(), __dmul_rn(st.s1i1, h.template get<kHTin>()))));
    const double t_1 = __dmul_rn(__fma_rn(m3, r0, -__dmul_rn(m1, r1)), rdet);
    c3 = __fma_rn(S0, h.template get<kHZout>(), -__dmul_rn(S1, h.template get<kHV21>()));
    r0 = __fma_rn(st.s1i0, h.template get<kHZin>(), c3);
    r1 = __fma_rn(d, c3, __fma_rn(S2, h.template get<kHV21>(), -__fma_rn(S1, h.template get<kHZout>(), __dmul_rn(st.s1i1, h.template get<kHZin>()))));
    const double v_1 = __dmul_rn(__fma_rn(m3, r0, -__dmul_rn(m1, r1)), rdet);
    // one bound for both solves: each right-hand-side input is at most mag_tv in magnitude
    // M(r0) = mag (|s1i0| + |S0| + |S1|) = mag (M(m0) + |S1|) and
    // M(r1) = mag (d (|S0| + |S1|) + |S2| + |S1| + |s1i1|) = mag (M(m1) + d |S1| + |S2|), so
    // M(num) = M(m3) M(r0) + M(m1) M(r1) = mag (M(m3) (M(m0) + |S1|) + M(m1) (M(m1) + d |S1| + |S2|))
    const double mag_tv = h.template get<kHMag>();
    const double Mnum = __dmul_rn(mag_tv, __fma_rn(Mm3, __dadd_rn(Mm0, aS1), __dmul_rn(Mm1, __dadd_rn(Mm1, __fma_rn(d, aS1, aS2)))));
    const double err = __dmul_rn(kBoundK, __dmul_rn(__fma_rn(fmax(fabs(t_1), fabs(v_1)), Mdet, Mnum), fabs(rdet)));
    // rotation back to x/y (B.cu:9229-9232) and the voxel indices (calculate_voxel_GPU B.cu:11091)
    const double x_1 = __fma_rn(h.template get<kHCos>(), u_shifted, -__dmul_rn(h.template get<kHSin>(), t_1));
    const double y_1 = __fma_rn(h.template get<kHSin>(), u_shifted, __dmul_rn(h.template get<kHCos>(), t_1));
    const double Mrot = __fma_rn(fabs(h.template get<kHCos>()) + fabs(h.template get<kHSin>()), fabs(u_shifted) + fabs(t_1), 0.0);
    const double err_xy = __fma_rn(kBoundK, Mrot, err);
    int vx, vy, vz;
    if (!guarded_indices(g, x_1, y_1, v_1, err_xy, vx, vy, vz)) return false;  // err_xy >= err
    long long v64 = (long long)vx + (long long)vy * g.columns + (long long)vz * g.columns * g.rows;
    if (v64 > 0x7fffffffLL) v64 = 0x7fffffffLL;
    voxel = (uint32_t)v64;
    return true;
}

// Voxel of an MLP point after rotating back to x/y (B.cu:9229-9235); 0x7fffffff when an index
// does not fit.
__device__ __forceinline__ uint32_t mlp_voxel(const Geometry& g, const MlpHistory& h, double u_shifted, double t_1,
                                              double v_1)
{
    const double x_1 = h.cos_term * u_shifted - h.sin_term * t_1;
    const double y_1 = h.sin_term * u_shifted + h.cos_term * t_1;
    const int vx = voxel_index_1d_fast(g.x_zero, x_1, g.voxel_width, g.inv_voxel_width);
    const int vy = voxel_index_1d_fast(g.y_zero, y_1, g.voxel_height, g.inv_voxel_height);
    const int vz = voxel_index_1d_fast(g.z_zero, v_1, g.voxel_thickness, g.inv_voxel_thickness);
    long long v64 = (long long)vx + (long long)vy * g.columns + (long long)vz * g.columns * g.rows;
    if (vx < 0 || vy < 0 || vz < 0 || v64 > 0x7fffffffLL) v64 = 0x7fffffffLL;
    return (uint32_t)v64;
}

// State of one history's walk after the setup of B.cu:9104-9178: the per-history constants, the
// running depth and position, the Sigma_2 table index, and the first path entry.
struct MlpStart {
    MlpHistory h;
    double depth_2_go, u_shifted, u_in;
    unsigned sigma_2_index;
    bool tables_ok;
};

// Per-history setup of find_MLP_path_GPU_tabulated (B.cu:9104-9178), shared by both walks.
__device__ __forceinline__ MlpStart mlp_start(const Geometry& g, const Tables& tab, double x_in_object,
                                              double y_in_object, double z_in_object, double x_out_object,
                                              double y_out_object, double z_out_object, double& xy_entry_angle,
                                              double& xy_exit_angle, double xz_entry_angle, double xz_exit_angle,
                                              unsigned& flags)
{
    const double PI = ref_pi();
    const double s = g.mlp_u_step;
    MlpStart m;
    MlpHistory& h = m.h;
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
    h.sin_term = sin_term;
    h.cos_term = cos_term;
    h.t_in = cos_term * y_in_object - sin_term * x_in_object;
    h.t_out = cos_term * y_out_object - sin_term * x_out_object;
    h.z_in = z_in_object;
    h.z_out = z_out_object;
    h.T_2_1 = xy_exit_angle - xy_entry_angle;
    h.V_2_1 = xz_exit_angle - xz_entry_angle;
    h.u_2 = fabs(u_out_object - u_in_object);
    m.depth_2_go = h.u_2 - s;
    m.u_shifted = u_in_object;
    m.u_in = u_in_object;

    m.tables_ok = (h.u_2 / kPolyTableStep + 0.5) < (double)g.poly_elements && m.depth_2_go >= 0;
    unsigned u_2_poly_index = 0;
    m.sigma_2_index = 0;
    if (m.tables_ok) {
        m.sigma_2_index = (unsigned)(m.depth_2_go / kCoeffTableStep + 0.5);
        u_2_poly_index = (unsigned)(h.u_2 / kPolyTableStep + 0.5);
    } else {
        flags |= kFlagTableRange;
    }
    h.u_2_poly_3_12 = __ldg(tab.poly_3_12 + u_2_poly_index);
    h.u_2_poly_2_6 = __ldg(tab.poly_2_6 + u_2_poly_index);
    h.u_2_poly_1_2 = __ldg(tab.poly_1_2 + u_2_poly_index);
    h.u_2_sq = powf_square(h.u_2);
    h.two_u_2 = 2 * h.u_2;
    h.mag_tv = fmax(fabs(h.t_in) + fabs(h.t_out) + fabs(h.T_2_1), fabs(h.z_in) + fabs(h.z_out) + fabs(h.V_2_1));
    return m;
}

// Appends voxels to the path unless they repeat the previous entry (B.cu:9244-9251) and sums x
// over the path when kSumX.
template <bool kSumX, class Emit>
struct PathWriter {
    const Geometry& g;
    const float* __restrict__ x;
    Emit& emit;
    WalkResult& r;
    uint32_t last;
    int n;
    __device__ __forceinline__ void first(uint32_t voxel)
    {
        emit(0, voxel);
        n = 1;
        last = voxel;
        r.axk = 0.0;
        if (voxel < (uint32_t)g.padded_voxels) {
            if (kSumX) r.axk = (double)__ldg(x + voxel);
        } else {
            r.flags |= kFlagVoxelOOB;
        }
    }
    __device__ __forceinline__ void visit(uint32_t voxel)
    {
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
    }
};

// One history's MLP.  emit(j, voxel) is called for every path entry j in order.  With kSumX the
// walk also sums the padded image x over the path (reads beyond it are reported and count as 0);
// without it x is not touched (the voxel list does not depend on the image).  kUnroll = 2
// evaluates two consecutive MLP points per loop trip so their independent FP64 chains overlap;
// the depth and position recurrences are still carried one subtraction / addition at a time, so
// every value is the one the reference computes.  A non-zero stash_stride parks the per-history
// constants and the chord in shared memory at stash_addr (kHistoryFields + 1 slots, stash_stride
// bytes apart) and reads each constant where a loop trip uses it.
template <bool kSumX, int kUnroll = 1, class Emit>
__device__ __forceinline__ WalkResult mlp_walk_exact(const Geometry& g, const Tables& tab,
                                                     const StepConst* __restrict__ steps, int kmax,
                                                     const float* __restrict__ x, uint32_t first_MLP_voxel,
                                                     double x_in_object, double y_in_object, double z_in_object,
                                                     double x_out_object, double y_out_object, double z_out_object,
                                                     double xy_entry_angle, double xz_entry_angle,
                                                     double xy_exit_angle, double xz_exit_angle, Emit emit,
                                                     uint32_t stash_addr = 0, uint32_t stash_stride = 0)
{
    static_assert(kUnroll == 1 || kUnroll == 2, "unroll 1 or 2");
    const double s = g.mlp_u_step;
    WalkResult r;
    r.flags = 0;
    MlpStart m = mlp_start(g, tab, x_in_object, y_in_object, z_in_object, x_out_object, y_out_object, z_out_object,
                           xy_entry_angle, xy_exit_angle, xz_entry_angle, xz_exit_angle, r.flags);
    if (stash_stride) history_stash_store(stash_addr, stash_stride, m.h);
    double depth_2_go = m.depth_2_go, u_shifted = m.u_shifted;
    unsigned sigma_2_index = m.sigma_2_index;

    PathWriter<kSumX, Emit> w{g, x, emit, r, 0u, 0};
    w.first(first_MLP_voxel);
    r.chord = effective_chord_length(g, (xy_entry_angle + xy_exit_angle) / 2.0, (xz_entry_angle + xz_exit_angle) / 2.0);
    r.aia = powf_square(r.chord);
    if (stash_stride && PCT_STASH_CHORD)  // the chord waits in the stash slot after the history's constants
        asm volatile("st.shared.f64 [%0], %1;" ::"r"(stash_addr + kHistoryFields * stash_stride), "d"(r.chord) : "memory");

    int k = 1;
    while (m.tables_ok && depth_2_go > s) {
        if (k > kmax) {  // cannot happen while the u_2 index is inside the tables
            r.flags |= kFlagTableRange;
            break;
        }
        if (kUnroll == 1) {
            const StepConst& st = steps[k];
            const HistoryInShared hs{stash_addr, stash_stride};
            const Sigma2 m2 = stash_stride ? sigma2_moments(hs, st, tab.scattering_table, sigma_2_index)
                                           : sigma2_moments(m.h, st, tab.scattering_table, sigma_2_index);
            u_shifted += s;
            uint32_t voxel;
            bool fast = false;
            if (PCT_FAST_POINTS && g.exact_fast_points)
                fast = stash_stride ? mlp_point_fast(g, hs, st, m2.sigma_t2, m2.sigma_t2_theta2, m2.sigma_theta2,
                                                     m2.determinant, depth_2_go, u_shifted, voxel)
                                    : mlp_point_fast(g, HistoryInRegisters{m.h}, st, m2.sigma_t2, m2.sigma_t2_theta2,
                                                     m2.sigma_theta2, m2.determinant, depth_2_go, u_shifted, voxel);
            if (!fast) {
                const MlpHistory h = stash_stride ? history_stash_load(stash_addr, stash_stride) : m.h;
                double t_1, v_1;
                mlp_point_rest(h, st, m2, depth_2_go, t_1, v_1);
                voxel = mlp_voxel(g, h, u_shifted, t_1, v_1);
            }
            w.visit(voxel);
            depth_2_go -= s;
            sigma_2_index -= g.sigma_index_step;
            k++;
        } else {
            const MlpHistory& h = m.h;
            // the second point exists when the loop would run again after the first
            const double depth_b = depth_2_go - s;
            const bool have_b = depth_b > s && k + 1 <= kmax;
            const unsigned sigma_b = have_b ? sigma_2_index - g.sigma_index_step : sigma_2_index;
            double t_a, v_a, t_b, v_b;
            mlp_point(h, steps[k], tab.scattering_table, depth_2_go, sigma_2_index, t_a, v_a);
            mlp_point(h, steps[have_b ? k + 1 : k], tab.scattering_table, have_b ? depth_b : depth_2_go, sigma_b, t_b,
                      v_b);
            u_shifted += s;
            w.visit(mlp_voxel(g, h, u_shifted, t_a, v_a));
            depth_2_go = depth_b;
            sigma_2_index -= g.sigma_index_step;
            k++;
            if (have_b) {
                u_shifted += s;
                w.visit(mlp_voxel(g, h, u_shifted, t_b, v_b));
                depth_2_go -= s;
                sigma_2_index -= g.sigma_index_step;
                k++;
            }
        }
    }
    r.n = w.n < kPathCap ? w.n : kPathCap;
    if (stash_stride && PCT_STASH_CHORD)
        asm volatile("ld.shared.f64 %0, [%1];" : "=d"(r.chord) : "r"(stash_addr + kHistoryFields * stash_stride));
    return r;
}

// ------------------------------------------------------------------------------------------
// Mixed precision (PCT_PRECISION_MIXED).  FP64 is kept where cancellation needs it: the Sigma_2
// moments (differences of tabulated integrals, which cancel towards the exit) at every point, and
// within Geometry::mixed_fp64_margin of the entry or the exit also the inverse of Sigma_2, the
// matrix M = Sigma_1^-1 + R_1^T Sigma_2^-1 R_1 and its determinant (ill-conditioned there; FP32
// in between).  The right-hand sides, the solve t_1 = [M^-1]_0 . rhs, the rotation back to x/y
// and the voxel indices run in FP32.  Every operation is an explicit
// intrinsic, so the result does not depend on the translation unit's contraction flags.
// ------------------------------------------------------------------------------------------

struct MlpHistoryF {
    float sin_term, cos_term, t_in, t_out, z_in, z_out, T_2_1, V_2_1;
};

__device__ __forceinline__ MlpHistoryF mlp_history_f(const MlpHistory& h)
{
    return MlpHistoryF{(float)h.sin_term, (float)h.cos_term, (float)h.t_in, (float)h.t_out,
                       (float)h.z_in,     (float)h.z_out,    (float)h.T_2_1, (float)h.V_2_1};
}

// Whether the mixed walk inverts Sigma_2 and M in FP64 at loop trip k: within
// g.mixed_fp64_margin of the entry (u_1 = k * MLP_U_STEP, where Sigma_1 is small) or of the exit
// (depth_2_go, where Sigma_2 is small) both are ill-conditioned; in between FP32 suffices.
__device__ __forceinline__ bool mixed_fp64_inverse(const Geometry& g, int k, double depth_2_go)
{
    return depth_2_go < g.mixed_fp64_margin || (double)k * g.mlp_u_step < g.mixed_fp64_margin;
}

__device__ __forceinline__ void mlp_point_mixed(const MlpHistory& h, const MlpHistoryF& hf, const StepConst& st,
                                                const double* __restrict__ scattering, double depth_2_go,
                                                unsigned sigma_2_index, bool fp64_inverse, float& t_1, float& v_1)
{
    // FP64: the Sigma_2 moments (differences of tabulated integrals)
    const double sigma_t2 =
        __dsub_rn(__fma_rn(h.two_u_2, st.p23, __fma_rn(-h.u_2_sq, st.p12, h.u_2_poly_3_12)), st.p34);
    const double sigma_t2_theta2 = __dadd_rn(__fma_rn(-h.u_2, st.p12, h.u_2_poly_2_6), st.p23);
    const double sigma_theta2 = __dsub_rn(h.u_2_poly_1_2, st.p12);
    const double scat = __ldg(scattering + sigma_2_index);
    const float d = (float)depth_2_go;
    float i00, i01, a0, a1, a2;
    if (fp64_inverse) {
        // FP64: Sigma_2^-1, M and the first row of M^-1
        const double det2 =
            __dmul_rn(scat, __fma_rn(sigma_t2, sigma_theta2, -__dmul_rn(sigma_t2_theta2, sigma_t2_theta2)));
        const double r2 = __drcp_rn(det2);
        const double S0 = __dmul_rn(sigma_theta2, r2), S1 = __dmul_rn(sigma_t2_theta2, r2), S2 = __dmul_rn(sigma_t2, r2);
        const double c = __fma_rn(S0, depth_2_go, -S1);
        const double m0 = __dadd_rn(st.s1i0, S0);
        const double m1 = __dsub_rn(c, st.s1i1);
        const double m3 = __fma_rn(depth_2_go, __dsub_rn(c, S1), __dadd_rn(st.s1i2, S2));
        const double rM = __drcp_rn(__fma_rn(m0, m3, -__dmul_rn(m1, m1)));
        i00 = (float)__dmul_rn(m3, rM);
        i01 = (float)(-__dmul_rn(m1, rM));
        a0 = (float)S0;
        a1 = (float)S1;
        a2 = (float)S2;
    } else {
        // FP32: the same inversions away from the entry and the exit
        const float st2 = (float)sigma_t2, stt = (float)sigma_t2_theta2, sth = (float)sigma_theta2;
        const float det2 = __fmul_rn((float)scat, __fmaf_rn(st2, sth, -__fmul_rn(stt, stt)));
        const float r2 = __frcp_rn(det2);
        a0 = __fmul_rn(sth, r2);
        a1 = __fmul_rn(stt, r2);
        a2 = __fmul_rn(st2, r2);
        const float c = __fmaf_rn(a0, d, -a1);
        const float m0 = __fadd_rn(st.s1i0f, a0);
        const float m1 = __fsub_rn(c, st.s1i1f);
        const float m3 = __fmaf_rn(d, __fsub_rn(c, a1), __fadd_rn(st.s1i2f, a2));
        const float rM = __frcp_rn(__fmaf_rn(m0, m3, -__fmul_rn(m1, m1)));
        i00 = __fmul_rn(m3, rM);
        i01 = -__fmul_rn(m1, rM);
    }
    // FP32: right-hand sides and the solve
    float c3 = __fmaf_rn(a0, hf.t_out, -__fmul_rn(a1, hf.T_2_1));
    float r0 = __fmaf_rn(st.s1i0f, hf.t_in, c3);
    float r1 = __fmaf_rn(d, c3, __fmaf_rn(a2, hf.T_2_1, -__fmaf_rn(a1, hf.t_out, __fmul_rn(st.s1i1f, hf.t_in))));
    t_1 = __fmaf_rn(i00, r0, __fmul_rn(i01, r1));
    c3 = __fmaf_rn(a0, hf.z_out, -__fmul_rn(a1, hf.V_2_1));
    r0 = __fmaf_rn(st.s1i0f, hf.z_in, c3);
    r1 = __fmaf_rn(d, c3, __fmaf_rn(a2, hf.V_2_1, -__fmaf_rn(a1, hf.z_out, __fmul_rn(st.s1i1f, hf.z_in))));
    v_1 = __fmaf_rn(i00, r0, __fmul_rn(i01, r1));
}

__device__ __forceinline__ int voxel_index_1d_f(float zero, float pos, float inv_size)
{
    const float q = __fmul_rn(fabsf(__fsub_rn(pos, zero)), inv_size);
    return q < 2147483000.0f ? (int)q : -1;
}

__device__ __forceinline__ uint32_t mlp_voxel_mixed(const Geometry& g, const MlpHistoryF& hf, float u_shifted,
                                                    float t_1, float v_1)
{
    const float x_1 = __fmaf_rn(hf.cos_term, u_shifted, -__fmul_rn(hf.sin_term, t_1));
    const float y_1 = __fmaf_rn(hf.sin_term, u_shifted, __fmul_rn(hf.cos_term, t_1));
    const int vx = voxel_index_1d_f(g.x_zero_f, x_1, g.inv_voxel_width_f);
    const int vy = voxel_index_1d_f(g.y_zero_f, y_1, g.inv_voxel_height_f);
    const int vz = voxel_index_1d_f(g.z_zero_f, v_1, g.inv_voxel_thickness_f);
    long long v64 = (long long)vx + (long long)vy * g.columns + (long long)vz * g.columns * g.rows;
    if (vx < 0 || vy < 0 || vz < 0 || v64 > 0x7fffffffLL) v64 = 0x7fffffffLL;
    return (uint32_t)v64;
}

// The mixed-precision walk: same control flow, depth/position recurrences and de-duplication as
// the exact walk; the points and voxels as above.
template <bool kSumX, class Emit>
__device__ __forceinline__ WalkResult mlp_walk_mixed(const Geometry& g, const Tables& tab,
                                                     const StepConst* __restrict__ steps, int kmax,
                                                     const float* __restrict__ x, uint32_t first_MLP_voxel,
                                                     double x_in_object, double y_in_object, double z_in_object,
                                                     double x_out_object, double y_out_object, double z_out_object,
                                                     double xy_entry_angle, double xz_entry_angle,
                                                     double xy_exit_angle, double xz_exit_angle, Emit emit)
{
    const double s = g.mlp_u_step;
    WalkResult r;
    r.flags = 0;
    MlpStart m = mlp_start(g, tab, x_in_object, y_in_object, z_in_object, x_out_object, y_out_object, z_out_object,
                           xy_entry_angle, xy_exit_angle, xz_entry_angle, xz_exit_angle, r.flags);
    const MlpHistoryF hf = mlp_history_f(m.h);
    double depth_2_go = m.depth_2_go, u_shifted = m.u_shifted;
    unsigned sigma_2_index = m.sigma_2_index;
    PathWriter<kSumX, Emit> w{g, x, emit, r, 0u, 0};
    w.first(first_MLP_voxel);
    r.chord = effective_chord_length(g, (xy_entry_angle + xy_exit_angle) / 2.0, (xz_entry_angle + xz_exit_angle) / 2.0);
    r.aia = r.chord * r.chord;
    int k = 1;
    while (m.tables_ok && depth_2_go > s) {
        if (k > kmax) {
            r.flags |= kFlagTableRange;
            break;
        }
        float t_1, v_1;
        mlp_point_mixed(m.h, hf, steps[k], tab.scattering_table, depth_2_go, sigma_2_index,
                        mixed_fp64_inverse(g, k, depth_2_go), t_1, v_1);
        u_shifted = __dadd_rn(u_shifted, s);
        w.visit(mlp_voxel_mixed(g, hf, (float)u_shifted, t_1, v_1));
        depth_2_go = __dsub_rn(depth_2_go, s);
        sigma_2_index -= g.sigma_index_step;
        k++;
    }
    r.n = w.n < kPathCap ? w.n : kPathCap;
    return r;
}

}  // namespace pct
