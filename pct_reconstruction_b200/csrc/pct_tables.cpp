// pct_tables.cpp -- MLP lookup tables, built on the host.
//
// The reference builds its tables on the host with glibc double sin/cos/log/pow
// (generate_trig_tables B.cu:8421, generate_scattering_coefficient_table B.cu:8445,
// generate_polynomial_tables B.cu:8464) and uploads them (MLP_lookup_table_2_GPU B.cu:8503).
// The table values must be identical bit for bit, because the MLP voxel lists are compared
// exactly, so the expressions below keep the reference's operand order (including how the
// A_i macros expand) and this file is compiled without FMA contraction.
//
// In addition to the reference tables, build_step_table() evaluates, once per MLP step k, the
// terms of the tabulated MLP loop that depend only on u_1 = k*MLP_U_STEP (B.cu:9180-9190):
// the three u_1 polynomials and the inverse of Sigma_1.  Every history reads the same entries,
// so the loop keeps only the history-dependent Sigma_2 algebra.
#include "pct_tables.h"

#include <cmath>

namespace pct {

namespace {
constexpr double kE0 = 13.6;   // E_0 (B.h:741)
constexpr double kX0 = 36.08;  // X0  (B.h:742)
double pi() { return 4 * std::atan(1.0); }
// powf(v, 2) on a double: round to float, square in float (see powf_square in pct_mlp.cuh).
double powf_square(double v)
{
    float f = (float)v;
    return (double)(f * f);
}
}  // namespace

double trig_table_min() { return -2 * pi(); }
double trig_table_step() { return (0.001 * (pi() / 180.0)); }
int trig_table_elements() { return (int)((4 * pi() - -2 * pi()) / trig_table_step() + 0.5); }
int coeff_table_elements() { return (int)(kCoeffTableRange / kCoeffTableStep + 0.5); }
int poly_table_elements() { return (int)(kPolyTableRange / kPolyTableStep + 0.5); }

void build_host_tables(HostTables& t)
{
    const int nt = trig_table_elements(), nc = coeff_table_elements(), np = poly_table_elements();
    t.sin_table.assign(nt + 1, 0.0);
    t.cos_table.assign(nt + 1, 0.0);
    for (int s = 0; s <= nt; s++) {
        double a = -2 * pi() + s * (0.001 * (pi() / 180.0));
        t.sin_table[s] = std::sin(a);
        t.cos_table[s] = std::cos(a);
    }
    t.scattering_table.assign(nc + 1, 0.0);
    for (int s = 0; s <= nc; s++) {
        double depth = s * kCoeffTableStep;
        t.scattering_table[s] = std::pow(kE0 * (1 + 0.038 * std::log(depth / kX0)), 2.0) / kX0;
    }
    // A_i = c_i * pow((float)10, (float)e_i): the float pow overload (B.h:749-754).
    const double a0 = 7.457 * (double)powf(10.0f, -6.0f);
    const double a1 = 4.548 * (double)powf(10.0f, -7.0f);
    const double a2 = -5.777 * (double)powf(10.0f, -8.0f);
    const double a3 = 1.301 * (double)powf(10.0f, -8.0f);
    const double a4 = -9.228 * (double)powf(10.0f, -10.0f);
    const double c5 = 2.687, p5 = (double)powf(10.0f, -11.0f);  // "u * A_5_OVER_m" -> ((u*c5)*p5)/m
    t.poly_1_2.assign(np + 1, 0.0);
    t.poly_2_3.assign(np + 1, 0.0);
    t.poly_3_4.assign(np + 1, 0.0);
    t.poly_2_6.assign(np + 1, 0.0);
    t.poly_3_12.assign(np + 1, 0.0);
    for (int s = 0; s <= np; s++) {
        const double u = s * kPolyTableStep;
        const double u2 = std::pow(u, 2), u3 = std::pow(u, 3);
        t.poly_1_2[s] = u * (a0 + u * (a1 / 2 + u * (a2 / 3 + u * (a3 / 4 + u * (a4 / 5 + u * c5 * p5 / 6)))));
        t.poly_2_3[s] = u2 * (a0 / 2 + u * (a1 / 3 + u * (a2 / 4 + u * (a3 / 5 + u * (a4 / 6 + u * c5 * p5 / 7)))));
        t.poly_3_4[s] = u3 * (a0 / 3 + u * (a1 / 4 + u * (a2 / 5 + u * (a3 / 6 + u * (a4 / 7 + u * c5 * p5 / 8)))));
        t.poly_2_6[s] = u2 * (a0 / 2 + u * (a1 / 6 + u * (a2 / 12 + u * (a3 / 20 + u * (a4 / 30 + u * c5 * p5 / 42)))));
        t.poly_3_12[s] =
            u3 * (a0 / 3 + u * (a1 / 12 + u * (a2 / 30 + u * (a3 / 60 + u * (a4 / 105 + u * c5 * p5 / 168)))));
    }
}

int build_step_table(const HostTables& t, double mlp_u_step, std::vector<StepConst>& steps)
{
    const unsigned sstep = (unsigned)(mlp_u_step / kCoeffTableStep + 0.5);
    const unsigned pstep = (unsigned)(mlp_u_step / kPolyTableStep + 0.5);
    if (sstep == 0 || pstep == 0) return -1;
    const int np = (int)t.poly_1_2.size() - 1, nc = (int)t.scattering_table.size() - 1;
    // Entry k (k >= 1) is the k-th loop iteration: u_1_poly_index = k*pstep and
    // sigma_1_coefficient_index = k*sstep.  Entry 0 is unused.
    int kmax = 0;
    while ((long long)(kmax + 1) * pstep <= np && (long long)(kmax + 1) * sstep <= nc) kmax++;
    steps.assign(kmax + 1, StepConst{});
    for (int k = 1; k <= kmax; k++) {
        const unsigned pi1 = k * pstep, si1 = k * sstep;
        const double p12 = t.poly_1_2[pi1], p23 = t.poly_2_3[pi1];
        const double sigma_t1 = t.poly_3_12[pi1], sigma_t1_theta1 = t.poly_2_6[pi1], sigma_theta1 = p12;
        // determinant_Sigma_1 and Sigma_1I as at B.cu:9192-9195
        const double det1 = t.scattering_table[si1] * (sigma_t1 * sigma_theta1 - powf_square(sigma_t1_theta1));
        StepConst& e = steps[k];
        e.p12 = p12;
        e.p23 = p23;
        e.p34 = t.poly_3_4[pi1];
        e.s1i0 = sigma_theta1 / det1;
        e.s1i1 = sigma_t1_theta1 / det1;
        e.s1i2 = sigma_t1 / det1;
    }
    return kmax;
}

}  // namespace pct
