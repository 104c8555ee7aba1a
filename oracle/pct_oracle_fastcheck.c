/* pct_oracle_fastcheck.c -- TEST INFRASTRUCTURE: the engine's guarded fast MLP points, checked.
 *
 * The engine's exact mode (EXACT_FAST_POINTS = 1) evaluates each MLP point by reciprocals and fused
 * multiply-adds with a forward error bound, and recomputes it in the reference's operation order
 * whenever the bound cannot prove the point's voxel (mlp_point_fast, csrc/pct_mlp.cuh).  This file
 * restates that evaluation on the CPU next to the oracle's reference-order point
 * (find_MLP_path_GPU_tabulated, B.cu:9180-9235, as oracle_find_mlp_path_tabulated computes it) and
 * counts, over every point of every history, the points the bound accepts and those accepted
 * points whose voxel differs from the reference-order voxel.  That second count must be 0.
 *
 * The hardware reciprocal rcp.approx.ftz.f64 is stood in for by the float reciprocal of the
 * mantissa (relative error below 2^-23, like the hardware's), followed by the same two Newton
 * steps; fma() is the correctly rounded fused multiply-add, as __fma_rn.  Built with
 * -ffp-contract=off.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

#include "pct_oracle.h"

static const double kBoundK = 9.094947017729282e-13; /* 2^-40, as the engine */
#define COEFF_TABLE_STEP 0.00005 /* B.h:792 */
#define POLY_TABLE_STEP 0.00005  /* B.h:796 */

static double rcp_refined(double b)
{
    int e;
    const double m = frexp(b, &e);
    double r = ldexp((double)(1.0f / (float)m), -e);
    double d = fma(-b, r, 1.0);
    r = fma(r, d, r);
    d = fma(-b, r, 1.0);
    return fma(r, d, r);
}

/* guarded_indices (pct_mlp.cuh): the three indices with one tolerance for all axes,
 * (K max_a + err) max(1/size); the exact distance |p - rint(p)| to the nearest face must exceed it,
 * and the index is the truncation int(p). */
static int guarded_indices(double x0, double y0, double z0, double inv_w, double inv_h, double inv_t, double x, double y,
                           double z, double err, int* vx, int* vy, int* vz)
{
    const double ax = fabs(x - x0), ay = fabs(y - y0), az = fabs(z - z0);
    const double amax = fmax(fmax(ax, ay), az);
    const double inv = fmax(fmax(inv_w, inv_h), inv_t);
    const double tol = fma(kBoundK, amax, err) * inv;
    const double px = ax * inv_w, py = ay * inv_h, pz = az * inv_t;
    if (!(amax * inv < 2147483000.0 && fabs(px - rint(px)) > tol && fabs(py - rint(py)) > tol &&
          fabs(pz - rint(pz)) > tol))
        return 0;
    *vx = (int)px;
    *vy = (int)py;
    *vz = (int)pz;
    return 1;
}

void oracle_guarded_indices(const pct_config* cfg, int64_t n, const double* x, const double* y, const double* z,
                            double err, int32_t* ok, int32_t* idx)
{
    const double X0 = -cfg->RECON_CYL_RADIUS, Y0 = cfg->RECON_CYL_RADIUS, Z0 = cfg->RECON_CYL_HEIGHT / 2;
    const double invW = 1.0 / cfg->VOXEL_WIDTH, invH = 1.0 / cfg->VOXEL_HEIGHT, invT = 1.0 / cfg->VOXEL_THICKNESS;
    for (int64_t i = 0; i < n; i++) {
        int vx = -1, vy = -1, vz = -1;
        ok[i] = guarded_indices(X0, Y0, Z0, invW, invH, invT, x[i], y[i], z[i], err, &vx, &vy, &vz);
        idx[3 * i] = vx;
        idx[3 * i + 1] = vy;
        idx[3 * i + 2] = vz;
    }
}

static int calc_voxel_ref(double zero, double pos, double size)
{
    double q = fabs(pos - zero) / size;
    if (!(q < 2147483647.0)) return -1;
    return (int)q;
}

static float powf_square_ref(double v)
{
    float f = (float)v;
    return f * f;
}

void oracle_fast_point_check(const pct_config* cfg, const oracle_tables* tab, const pct_histories* h, int64_t n,
                             int64_t counts[3])
{
    const double PI = 4.0 * atan(1.0);
    const double s = cfg->MLP_U_STEP;
    const double TRIG_MIN = oracle_trig_table_min(), TRIG_STEP = oracle_trig_table_step();
    const double X0 = -cfg->RECON_CYL_RADIUS, Y0 = cfg->RECON_CYL_RADIUS, Z0 = cfg->RECON_CYL_HEIGHT / 2;
    const double invW = 1.0 / cfg->VOXEL_WIDTH, invH = 1.0 / cfg->VOXEL_HEIGHT, invT = 1.0 / cfg->VOXEL_THICKNESS;
    const unsigned sstep = (unsigned)(s / COEFF_TABLE_STEP + 0.5), pstep = (unsigned)(s / POLY_TABLE_STEP + 0.5);
    int64_t points = 0, accepted = 0, mismatched = 0;
    for (int64_t i = 0; i < n; i++) {
        double xy_entry = h->xy_entry_angle[i], xy_exit = h->xy_exit_angle[i];
        const double xe = h->x_entry[i], ye = h->y_entry[i], xo = h->x_exit[i], yo = h->y_exit[i];
        unsigned ti = (unsigned)((xy_entry - TRIG_MIN) / TRIG_STEP + 0.5);
        double sn = tab->sin_table[ti], cs = tab->cos_table[ti];
        double u_in = cs * xe + sn * ye, u_out = cs * xo + sn * yo;
        if (u_in > u_out) {
            xy_entry += PI;
            xy_exit += PI;
            ti = (unsigned)((xy_entry - TRIG_MIN) / TRIG_STEP + 0.5);
            sn = tab->sin_table[ti];
            cs = tab->cos_table[ti];
            u_in = cs * xe + sn * ye;
            u_out = cs * xo + sn * yo;
        }
        const double t_in = cs * ye - sn * xe, t_out = cs * yo - sn * xo;
        const double z_in = h->z_entry[i], z_out = h->z_exit[i];
        const double T21 = xy_exit - xy_entry, V21 = (double)h->xz_exit_angle[i] - (double)h->xz_entry_angle[i];
        const double u_2 = fabs(u_out - u_in);
        double depth = u_2 - s, u_shifted = u_in;
        if (!((u_2 / POLY_TABLE_STEP + 0.5) < (double)tab->poly_elements && depth >= 0)) continue;
        unsigned s2i = (unsigned)(depth / COEFF_TABLE_STEP + 0.5), s1i = sstep, p1 = pstep;
        const unsigned p2 = (unsigned)(u_2 / POLY_TABLE_STEP + 0.5);
        const double P312 = tab->poly_3_12[p2], P26 = tab->poly_2_6[p2], P12 = tab->poly_1_2[p2];
        const double u2sq = powf_square_ref(u_2), two_u2 = 2 * u_2;
        const double mag = fmax(fabs(t_in) + fabs(t_out) + fabs(T21), fabs(z_in) + fabs(z_out) + fabs(V21));
        while (depth > s) {
            const double q12 = tab->poly_1_2[p1], q23 = tab->poly_2_3[p1], q34 = tab->poly_3_4[p1];
            const double st1 = tab->poly_3_12[p1], stt1 = tab->poly_2_6[p1], sth1 = q12;
            const double det1 = tab->scattering_table[s1i] * (st1 * sth1 - powf_square_ref(stt1));
            const double s1i0 = sth1 / det1, s1i1 = stt1 / det1, s1i2 = st1 / det1;
            /* the moments and their determinant, the reference's operations in its order */
            const double sigma_t2 = P312 - u2sq * q12 + two_u2 * q23 - q34;
            const double sigma_tt = P26 - u_2 * q12 + q23;
            const double sigma_th = P12 - q12;
            const double det2 = tab->scattering_table[s2i] * (sigma_t2 * sigma_th - powf_square_ref(sigma_tt));
            u_shifted += s;
            /* reference order */
            const double S0 = sigma_th / det2, S1 = sigma_tt / det2, S2 = sigma_t2 / det2;
            const double c24 = S0 * depth - S1;
            const double f0 = s1i0 + S0, f1 = c24 - s1i1, f2 = depth * S0 - s1i1 - S1;
            const double f3 = s1i2 + S2 + depth * (c24 - S1);
            const double fdet = f0 * f3 - f1 * f2;
            double c3 = S0 * t_out - S1 * T21, r0 = s1i0 * t_in + c3;
            double r1 = depth * c3 + S2 * T21 - S1 * t_out - s1i1 * t_in;
            const double t1 = (f3 * r0 - f1 * r1) / fdet;
            c3 = S0 * z_out - S1 * V21;
            r0 = s1i0 * z_in + c3;
            r1 = depth * c3 + S2 * V21 - S1 * z_out - s1i1 * z_in;
            const double v1 = (f3 * r0 - f1 * r1) / fdet;
            const int vx = calc_voxel_ref(X0, cs * u_shifted - sn * t1, cfg->VOXEL_WIDTH);
            const int vy = calc_voxel_ref(Y0, sn * u_shifted + cs * t1, cfg->VOXEL_HEIGHT);
            const int vz = calc_voxel_ref(Z0, v1, cfg->VOXEL_THICKNESS);
            /* the guarded fast evaluation */
            const double r2 = rcp_refined(det2);
            const double F0 = sigma_th * r2, F1 = sigma_tt * r2, F2 = sigma_t2 * r2;
            const double c = fma(F0, depth, -F1);
            const double m0 = s1i0 + F0, m1 = c - s1i1, m3 = fma(depth, c - F1, s1i2 + F2);
            const double det = fma(m0, m3, -(m1 * m1));
            const double aS0 = fabs(F0), aS1 = fabs(F1), aS2 = fabs(F2);
            const double Mc = fma(aS0, depth, aS1);
            const double Mm0 = fabs(s1i0) + aS0, Mm1 = Mc + fabs(s1i1);
            const double Mm3 = fma(depth, Mc + aS1, fabs(s1i2) + aS2);
            const double Mdet = fma(Mm0, Mm3, Mm1 * Mm1);
            int ok = (4.0 * kBoundK) * Mdet < fabs(det);
            int fx = 0, fy = 0, fz = 0;
            if (ok) {
                const double rdet = rcp_refined(det);
                double e3 = fma(F0, t_out, -(F1 * T21)), e0 = fma(s1i0, t_in, e3);
                double e1 = fma(depth, e3, fma(F2, T21, -fma(F1, t_out, s1i1 * t_in)));
                const double ft = fma(m3, e0, -(m1 * e1)) * rdet;
                e3 = fma(F0, z_out, -(F1 * V21));
                e0 = fma(s1i0, z_in, e3);
                e1 = fma(depth, e3, fma(F2, V21, -fma(F1, z_out, s1i1 * z_in)));
                const double fv = fma(m3, e0, -(m1 * e1)) * rdet;
                const double Mnum = mag * fma(Mm3, Mm0 + aS1, Mm1 * (Mm1 + fma(depth, aS1, aS2)));
                const double err = kBoundK * (fma(fmax(fabs(ft), fabs(fv)), Mdet, Mnum) * fabs(rdet));
                const double x1 = fma(cs, u_shifted, -(sn * ft)), y1 = fma(sn, u_shifted, cs * ft);
                const double Mrot = fma(fabs(cs) + fabs(sn), fabs(u_shifted) + fabs(ft), 0.0);
                const double exy = fma(kBoundK, Mrot, err);
                ok = guarded_indices(X0, Y0, Z0, invW, invH, invT, x1, y1, fv, exy, &fx, &fy, &fz);
            }
            points++;
            if (ok) {
                accepted++;
                if (fx != vx || fy != vy || fz != vz) mismatched++;
            }
            depth -= s;
            s1i += sstep;
            s2i -= sstep;
            p1 += pstep;
        }
    }
    counts[0] = points;
    counts[1] = accepted;
    counts[2] = mismatched;
}
