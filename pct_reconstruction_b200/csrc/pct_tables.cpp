// pct_tables.cpp -- MLP lookup tables, built on the host.
//
// The reference builds its tables on the host with glibc double sin/cos/log/pow
// (generate_trig_tables B.cu:8421, generate_scattering_coefficient_table B.cu:8445,
// generate_polynomial_tables B.cu:8464) and uploads them (MLP_lookup_table_2_GPU B.cu:8503).
// The table values must be identical bit for bit, because the MLP voxel lists are compared
// exactly, so the expressions below keep the reference's operand order (including how the
// A_i macros expand) and this file is compiled without FMA contraction.
//
// The per-step table (the terms of the MLP loop that depend only on u_1 = k*MLP_U_STEP) is
// evaluated on the device from these tables, see build_step_table_kernel.
#include "pct_tables.h"

#include <cmath>

namespace pct {

namespace {
constexpr double kE0 = 13.6;   // E_0 (B.h:741)
constexpr double kX0 = 36.08;  // X0  (B.h:742)
double pi() { return 4 * std::atan(1.0); }
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

int step_table_kmax(const HostTables& t, double mlp_u_step)
{
    const unsigned sstep = (unsigned)(mlp_u_step / kCoeffTableStep + 0.5);
    const unsigned pstep = (unsigned)(mlp_u_step / kPolyTableStep + 0.5);
    if (sstep == 0 || pstep == 0) return -1;
    const long long np = (long long)t.poly_1_2.size() - 1, nc = (long long)t.scattering_table.size() - 1;
    int kmax = 0;
    while ((long long)(kmax + 1) * pstep <= np && (long long)(kmax + 1) * sstep <= nc) kmax++;
    return kmax;
}

}  // namespace pct
