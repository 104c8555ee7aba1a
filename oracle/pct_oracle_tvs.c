/*
 * pct_oracle_tvs.c -- CPU oracle for total variation superiorization.  TEST INFRASTRUCTURE ONLY.
 *
 * Restates calculate_total_variation (B.cu:10163), generate_perturbation_array (B.cu:10246),
 * iteratively_perturb_image (B.cu:10476), iteratively_perturb_image_unconditional (B.cu:10562),
 * NTVS_iteration (B.cu:10606) and generate_TVS_eta_sequence (B.cu:10149) in the reference's
 * sequential loop order.
 *
 * Two accumulation modes:
 *   ORACLE_TVS_REFERENCE  the reference literally: TV terms with powf(d, 2), TV and ||G||^2
 *                         accumulated in one float in voxel order;
 *   ORACLE_TVS_ENGINE     the engine's stated arithmetic: TV terms with d*d, TV and ||G||^2
 *                         accumulated in double (voxel order here, a fixed tree on the device,
 *                         so sums may differ in the last double bits).
 * Everything else (G, the gradient norms, the directions, the perturbation) is the same float
 * arithmetic in both modes.  The L draw is the engine's seeded hash (the reference draws from a
 * wall-clock-seeded std::default_random_engine, which nothing can reproduce).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "pct_oracle.h"

int oracle_tvs_randi(int lo, int hi, uint64_t seed, int k)
{
    if (hi < lo) return lo;
    uint64_t z = seed + 0x9E3779B97F4A7C15ull * (uint64_t)(k + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return lo + (int)(z % (uint64_t)(hi - lo + 1));
}

/* TVS_ETA_SEQUENCE_LENGTH = log(TVS_MIN_ETA)/log(A) (int); eta[e] = powf(A, L_0 + e). */
int oracle_tvs_eta(const pct_config* cfg, float* eta, int capacity)
{
    const int len = (int)(log(cfg->TVS_MIN_ETA) / log(cfg->TVS_A));
    int n = 0;
    for (int exponent = cfg->TVS_L_0; exponent < len; exponent++, n++)
        if (eta && n < capacity) eta[n] = powf((float)cfg->TVS_A, (float)exponent);
    return n;
}

static float eta_at(const pct_config* cfg, const float* eta, int n, int L)
{
    const int e = L - cfg->TVS_L_0;
    return (e >= 0 && e < n) ? eta[e] : 0.0f; /* the reference reads past its table here */
}

double oracle_total_variation(const pct_config* cfg, const float* x, int mode)
{
    const int C = cfg->COLUMNS, R = cfg->ROWS, S = cfg->SLICES;
    float tv_f = 0.0f;
    double tv_d = 0.0;
    for (int s = 0; s < S; s++)
        for (int r = 0; r < R - 1; r++)
            for (int c = 0; c < C - 1; c++) {
                const long v = c + (long)r * C + (long)s * R * C;
                const float dy = x[v + C] - x[v], dx = x[v + 1] - x[v];
                if (mode == ORACLE_TVS_REFERENCE)
                    tv_f += sqrtf(powf(dy, 2.0f) + powf(dx, 2.0f));
                else
                    tv_d += (double)sqrtf(dy * dy + dx * dx);
            }
    return mode == ORACLE_TVS_REFERENCE ? (double)tv_f : tv_d;
}

/* generate_perturbation_array: G (scatter form, reference loop order) and v = G/||G||. */
void oracle_tvs_direction(const pct_config* cfg, const float* x, float* G, float* v, float* norm_out, int mode)
{
    const int C = cfg->COLUMNS, R = cfg->ROWS, S = cfg->SLICES;
    const long nv = (long)C * R * S;
    float* gx = calloc((size_t)nv, sizeof(float));
    float* gy = calloc((size_t)nv, sizeof(float));
    float* gn = calloc((size_t)nv, sizeof(float));
    memset(G, 0, sizeof(float) * (size_t)nv);
    for (int s = 0; s < S; s++)
        for (int r = 0; r < R - 1; r++)
            for (int c = 0; c < C - 1; c++) {
                const long p = c + (long)r * C + (long)s * R * C;
                gx[p] = x[p + 1] - x[p];
                gy[p] = x[p + C] - x[p];
                gn[p] = (float)sqrt((double)gx[p] * gx[p] + (double)gy[p] * gy[p]);
            }
    for (int s = 0; s < S; s++)
        for (int r = 0; r < R - 1; r++)
            for (int c = 0; c < C - 1; c++) {
                const long p = c + (long)r * C + (long)s * R * C;
                if (gn[p] > 0.0f) {
                    G[p] -= (gx[p] + gy[p]) / gn[p];
                    G[p + C] += gy[p] / gn[p];
                    G[p + 1] += gx[p] / gn[p];
                }
            }
    float norm_f = 0.0f;
    double norm_d = 0.0;
    for (long p = 0; p < nv; p++) {
        if (mode == ORACLE_TVS_REFERENCE)
            norm_f = (float)((double)norm_f + pow((double)G[p], 2));
        else
            norm_d += (double)G[p] * (double)G[p];
    }
    const float norm = mode == ORACLE_TVS_REFERENCE ? sqrtf(norm_f) : sqrtf((float)norm_d);
    for (long p = 0; p < nv; p++) v[p] = norm != 0.0f ? G[p] / norm : 0.0f;
    if (norm_out) *norm_out = norm;
    free(gx);
    free(gy);
    free(gn);
}

static void apply(long nv, const float* in, float* out, const float* v, float beta, const uint8_t* hull)
{
    for (long p = 0; p < nv; p++)
        if (hull[p]) out[p] = in[p] - beta * v[p];
}

int oracle_ntvs_iteration(const pct_config* cfg, float* x, const uint8_t* hull, int k, int* L, int mode,
                          int* accepted_L, int capacity)
{
    const long nv = (long)cfg->COLUMNS * cfg->ROWS * cfg->SLICES;
    float* G = malloc(sizeof(float) * (size_t)nv);
    float* v = malloc(sizeof(float) * (size_t)nv);
    float* x_tvs = malloc(sizeof(float) * (size_t)nv);
    const int n_eta = oracle_tvs_eta(cfg, NULL, 0);
    float* eta = malloc(sizeof(float) * (size_t)(n_eta + 1));
    oracle_tvs_eta(cfg, eta, n_eta);
    const int reps = cfg->TVS_OLD ? 1 : cfg->TVS_REPETITIONS;
    int written = 0;
    if (!cfg->TVS_OLD) *L = oracle_tvs_randi(cfg->TVS_L_0 + k - 1, *L, (uint64_t)cfg->TVS_SEED, k);
    for (int n = 0; n < reps; n++) {
        if (!cfg->TVS_CONDITIONED) { /* iteratively_perturb_image_unconditional */
            oracle_tvs_direction(cfg, x, G, v, NULL, mode);
            apply(nv, x, x, v, eta_at(cfg, eta, n_eta, *L), hull);
            *L += 1;
        } else { /* iteratively_perturb_image */
            oracle_tvs_direction(cfg, x, G, v, NULL, mode);
            float beta = eta_at(cfg, eta, n_eta, *L);
            const double tv_x = oracle_total_variation(cfg, x, mode);
            double tv_prev = 0.0;
            memcpy(x_tvs, x, sizeof(float) * (size_t)nv);
            apply(nv, x_tvs, x, v, beta, hull);
            for (;;) {
                *L += 1;
                const double tv_y = oracle_total_variation(cfg, x, mode);
                if (tv_y <= tv_x || fabs(tv_y - tv_prev) / tv_y < cfg->TV_THRESHOLD || *L > 300) break;
                beta = eta_at(cfg, eta, n_eta, *L);
                tv_prev = tv_y;
                apply(nv, x_tvs, x, v, beta, hull);
            }
        }
        if (accepted_L && written < capacity) accepted_L[written++] = *L;
    }
    free(G);
    free(v);
    free(x_tvs);
    free(eta);
    return written;
}
