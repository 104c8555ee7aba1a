// pct_tables.h -- host construction of the MLP lookup tables and the per-step table.
#pragma once

#include <vector>

#include "pct_common.cuh"

namespace pct {

struct HostTables {
    std::vector<double> sin_table, cos_table, scattering_table;
    std::vector<double> poly_1_2, poly_2_3, poly_3_4, poly_2_6, poly_3_12;
};

// History-independent terms of MLP step k (u_1 = k*MLP_U_STEP): the u_1 polynomials used by
// Sigma_2 and the inverse of Sigma_1 (entries Sigma_1I[0..2] of B.cu:9193-9195).
struct StepConst {
    double p12, p23, p34;
    double s1i0, s1i1, s1i2;
    float s1i0f, s1i1f, s1i2f;  // float copies for the mixed-precision right-hand sides and inversions
};

double trig_table_min();
double trig_table_step();
int trig_table_elements();
int coeff_table_elements();
int poly_table_elements();

void build_host_tables(HostTables& t);
// Last MLP loop iteration k whose u_1 indices (k*pstep, k*sstep) stay inside the tables.
int step_table_kmax(const HostTables& t, double mlp_u_step);

}  // namespace pct
