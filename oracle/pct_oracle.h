/*
 * pct_oracle.h -- CPU oracle for the proton-CT hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference algorithm
 * (BlakeSchultze/pCT_Reconstruction, src/pCT_Reconstruction_Data_Segments_Blake.cu = "B.cu",
 * src/pCT_Reconstruction.cu = "O.cu") that tests/, the smoke check and bench.py's CPU-baseline
 * leg compare against.  The engine (libpct_b200.so) never links, loads or calls it.
 *
 * Parity pinning: the reference ships no golden vectors or tests.  The oracle is pinned by
 * (a) known-answer cases derived by hand (tests/test_oracle_known_answers.py) and (b) fixtures
 * produced by the reference's own device functions compiled for sm_100a and run on a B200
 * (oracle/ref_harness.cu, fixtures under tests/golden/).
 *
 * Arithmetic: IEEE double / float exactly as the reference expressions are written, left to
 * right, with no FMA contraction (built with -ffp-contract=off).  Where the reference calls a
 * float function on double data (powf, sinf, cosf) the oracle does the same conversion.
 */
#ifndef PCT_ORACLE_H
#define PCT_ORACLE_H

#include <stdint.h>
#include "../include/pct_api.h"

#ifdef __cplusplus
extern "C" {
#endif

/* MLP lookup tables (B.cu:8421-8502). */
typedef struct oracle_tables {
    int trig_elements, coeff_elements, poly_elements;
    double* sin_table;
    double* cos_table;
    double* scattering_table;
    double* poly_1_2;
    double* poly_2_3;
    double* poly_3_4;
    double* poly_2_6;
    double* poly_3_12;
} oracle_tables;

int oracle_tables_build(const pct_config* cfg, oracle_tables* t);
void oracle_tables_free(oracle_tables* t);
/* The A_i fit coefficients of 1/(beta^2 p^2) at 200 MeV as the reference evaluates them
 * (B.h:749-754): A_i = c_i * (double)powf(10, e_i). */
void oracle_a_coefficients(double a[6]);
/* Table geometry constants (B.h:786-800). */
double oracle_trig_table_min(void);
double oracle_trig_table_step(void);

/* EffectiveChordLength_GPU (B.cu:8873-8894). */
double oracle_effective_chord_length(const pct_config* cfg, double abs_angle_t, double abs_angle_v);

/* find_MLP_path_GPU_tabulated (B.cu:9104-9262).  x is the padded image
 * (NUM_VOXELS + COLUMNS*ROWS floats).  Returns number_of_intersections (path entries written,
 * capped at path_cap); *flags gets bit0 = voxel beyond the padded image (read as 0),
 * bit1 = path longer than path_cap, bit2 = u-extent outside the polynomial tables (no steps). */
int oracle_find_mlp_path_tabulated(const pct_config* cfg, const oracle_tables* tab, const float* x,
                                   uint32_t first_MLP_voxel, double x_in, double y_in, double z_in,
                                   double x_out, double y_out, double z_out, double xy_entry_angle,
                                   double xz_entry_angle, double xy_exit_angle, double xz_exit_angle,
                                   uint32_t* path, int path_cap, double* effective_chord_length,
                                   double* a_i_dot_x_k_partially, double* a_i_dot_a_i_partially,
                                   int* flags);

/* Batch form for tests: histories [start, start+n) of the SoA h (n_total entries). */
void oracle_mlp_paths(const pct_config* cfg, const oracle_tables* tab, const float* x,
                      const pct_histories* h, int64_t start, int64_t n, int32_t stride,
                      uint32_t* counts, uint32_t* voxels, double* chord, double* a_dot_x,
                      int64_t* flag_counts /* [3] */);

/* One DROP iteration (DROP_full_tx_iteration B.cu:9537 -> calculate_x_update_GPU B.cu:9321 ->
 * DROP_block_update_GPU B.cu:9522 -> image_update_GPU B.cu:9398), histories processed in input
 * order, float accumulation in history order.  x, x_update, S are padded images. */
/* S-curve attenuation (B.cu:10606-10649): s(k) of cfg's curve, and the table of k < count. */
float oracle_s_curve(const pct_config* cfg, uint32_t k);
void oracle_s_curve_table(const pct_config* cfg, int32_t count, float* out);

void oracle_drop_iteration(const pct_config* cfg, const oracle_tables* tab, const pct_histories* h,
                           int64_t n, float* x, float* x_update, uint32_t* S,
                           int64_t* flag_counts /* [3] */);

/* The reference's host MLP + DROP (O.cu:4017 calculate_MLP, O.cu:7680 DROP_blocks,
 * O.cu:7700 DROP_update): explicit FP64 MLP with pow/log per step, double x_update.  This is
 * the reference's own CPU implementation of the path, used as the timed CPU baseline.
 * Histories [0, n) are processed in DROP blocks; within a block `threads` OpenMP threads
 * split the histories and add into the shared double accumulators atomically.  Returns the
 * number of path voxels visited (sum of path lengths). */
int64_t oracle_host_drop_iteration(const pct_config* cfg, const pct_histories* h, int64_t n,
                                   float* x, int threads);

/* The host code's chord length: the float overload of EffectiveChordLength (O.cu:3745-3767). */
float oracle_host_effective_chord_length(const pct_config* cfg, float abs_angle_t, float abs_angle_v);

/* The host MLP voxel lists (calculate_MLP, O.cu:4017-4211) and atanf chord lengths
 * (O.cu:6634-6636) of histories [start, start + n), stride entries per history. */
void oracle_host_mlp_paths(const pct_config* cfg, const pct_histories* h, int64_t start, int64_t n, int32_t stride,
                           uint32_t* counts, uint32_t* voxels, double* chord);

/* The engine's guarded fast MLP points checked against the reference-order points
 * (pct_oracle_fastcheck.c): counts[0] MLP points of histories [0, n), counts[1] points whose
 * voxel the fast evaluation's error bound proves, counts[2] of those whose voxel differs from the
 * reference-order voxel (must be 0). */
void oracle_fast_point_check(const pct_config* cfg, const oracle_tables* tab, const pct_histories* h, int64_t n,
                             int64_t counts[3]);
/* The fast point's voxel guard (guarded_indices, the engine's pct_mlp.cuh) on n positions at cfg's
 * grid with error bound err (cm): ok[i] 1 when it proves the voxel, idx[3i..3i+2] the indices. */
void oracle_guarded_indices(const pct_config* cfg, int64_t n, const double* x, const double* y, const double* z,
                            double err, int32_t* ok, int32_t* idx);

/* ---- preprocessing stages (pct_oracle_pre.c) ---- */
/* geometry arrays g[10]: x/y/z_entry, x/y/z_exit, xy/xz_entry_angle, xy/xz_exit_angle;
 * tracker arrays [12]: t/u/v in_1, in_2, out_1, out_2 in the order t_in_1, t_in_2, t_out_1,
 * t_out_2, u_in_1, ..., v_out_2 */
void oracle_recon_volume_intersections(const pct_config* cfg, int64_t n, const float* const tracker[12],
                                       const float* gantry_angle, int integer_angles, float* const out[10],
                                       uint8_t* missed);
void oracle_binning(const pct_config* cfg, int64_t n, const float* const g[10], const float* WEPL, const uint8_t* missed,
                    int32_t* bin_num, int32_t* bin_counts, float* sum_WEPL, float* sum_ut, float* sum_uv);
void oracle_statistics_and_cuts(const pct_config* cfg, int64_t n, const int32_t* bin_num, const float* WEPL,
                                const float* const g[10], int32_t* bin_counts, float* mean_WEPL, float* mean_ut,
                                float* mean_uv, float* sd_WEPL, float* sd_ut, float* sd_uv, float* sinogram,
                                uint8_t* keep);
void oracle_sinogram_filter(const pct_config* cfg, const int32_t* bin_counts, float* sinogram, float* filtered);
void oracle_backprojection(const pct_config* cfg, const float* sinogram_filtered, float* FBP);
void oracle_median_filter(const pct_config* cfg, int radius, const float* in, float* out);
void oracle_initialize_hull(const pct_config* cfg, int32_t* hull);
int64_t oracle_hull_walks(const pct_config* cfg, int kind, int64_t n, const float* const g[10], const float* WEPL,
                          const uint8_t* missed, int32_t* image);
void oracle_edge_detection(const pct_config* cfg, int kind, int32_t* counts);
void oracle_collect_mlp_endpoints(const pct_config* cfg, const uint8_t* hull, int64_t n, float* const g[10],
                                  uint32_t* first_MLP_voxel);

/* ---- total variation superiorization (pct_oracle_tvs.c) ---- */
enum { ORACLE_TVS_REFERENCE = 0, ORACLE_TVS_ENGINE = 1 };
int oracle_tvs_randi(int lo, int hi, uint64_t seed, int k);
int oracle_tvs_eta(const pct_config* cfg, float* eta, int capacity);
double oracle_total_variation(const pct_config* cfg, const float* x, int mode);
void oracle_tvs_direction(const pct_config* cfg, const float* x, float* G, float* v, float* norm_out, int mode);
/* NTVS_iteration for DROP iteration k on x (NUM_VOXELS floats); *L is the exponent state;
 * accepted_L receives L after each repetition.  Returns the number of repetitions. */
int oracle_ntvs_iteration(const pct_config* cfg, float* x, const uint8_t* hull, int k, int* L, int mode,
                          int* accepted_L, int capacity);

#ifdef __cplusplus
}
#endif
#endif
