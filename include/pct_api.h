/*
 * pct_api.h -- C ABI of the B200 proton-CT reconstruction engine (libpct_b200.so).
 *
 * Every entry point is extern "C", takes plain pointers and sizes, never lets a C++
 * exception cross the boundary, and returns a pct_status.  A context (pct_ctx) owns all
 * device memory, the CUDA stream, the MLP lookup tables and the per-scan arrays; it is not
 * thread-safe, separate contexts on separate streams are.
 *
 * The reference (BlakeSchultze/pCT_Reconstruction) has no plugin layer: its stages are free
 * functions over global std::vectors and device pointers, configured by compile-time
 * macros.  Each entry point below names the reference function it replaces
 * (src/pCT_Reconstruction_Data_Segments_Blake.cu, "B.cu" below; include/
 * pCT_Reconstruction_Data_Segments_Blake.h, "B.h" below).
 *
 * Layout contract (identical to the reference):
 *   voxel = column + row*COLUMNS + slice*COLUMNS*ROWS   row 0 at +y, slice 0 at +z
 *   bin   = t_bin + angle_bin*T_BINS + v_bin*T_BINS*ANGULAR_BINS
 *   units: cm and radians inside the engine (tracker files are mm, converted on read).
 */
#ifndef PCT_API_H
#define PCT_API_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PCT_API_VERSION 1

/* Longest MLP voxel list handled per history (MLP_U_STEP >= 0.03125 cm over the 40 cm
 * polynomial-table range; the reference's MAX_INTERSECTIONS is 1280, B.h:342). */
#define PCT_MLP_PATH_CAP 1312

typedef enum pct_status {
    PCT_OK = 0,
    PCT_ERR_ARG = 1,      /* invalid argument or configuration                          */
    PCT_ERR_CUDA = 2,     /* a CUDA runtime call failed (message in pct_last_error)     */
    PCT_ERR_OOB = 3,      /* a device bounds counter tripped (index outside its array)  */
    PCT_ERR_TIMEOUT = 4,  /* a bounded device wait or host watchdog expired             */
    PCT_ERR_STATE = 5,    /* call out of order (e.g. DROP before histories are loaded)  */
    PCT_ERR_NOMEM = 6,    /* device allocation failed                                   */
    PCT_ERR_IO = 7        /* file missing, truncated or malformed                       */
} pct_status;

typedef enum pct_memory { PCT_HOST = 0, PCT_DEVICE = 1 } pct_memory;

/* Enumerations with the reference's names and values (B.h:115-124). */
enum { PCT_RAM_LAK = 0, PCT_SHEPP_LOGAN = 1, PCT_UNFILTERED = 2 };              /* FBP_FILTER_TYPES */
enum { PCT_SC_HULL = 0, PCT_MSC_HULL = 1, PCT_SM_HULL = 2, PCT_FBP_HULL = 3 };  /* HULL_TYPES       */
enum { PCT_DROP = 2, PCT_ROBUSTA = 5, PCT_ROBUSTB = 6 };  /* PROJECTION_ALGORITHMS (B.h:124) built here */
enum { PCT_SEQUENTIAL = 0, PCT_PRIME_PERMUTATION = 1 };   /* HISTORY_ORDERING (B.h:134)             */
enum { PCT_SIGMOID = 0, PCT_TANH = 1, PCT_ATAN = 2, PCT_ERF = 3, PCT_LIN_OVER_ROOT = 4 }; /* S_CURVES (B.h:125) */
/* Engine options (no reference counterpart). */
enum { PCT_PRECISION_EXACT = 0, PCT_PRECISION_MIXED = 1, PCT_PRECISION_MIXED_COMPENSATED = 2 };
enum { PCT_SCATTER_ATOMIC = 0, PCT_SCATTER_DETERMINISTIC = 1 };

/*
 * Runtime configuration.  Field names are the reference's macro / settings.cfg key names
 * (B.h:333-480, settings.cfg:21-164); values are runtime instead of compile-time.
 * Fields marked "derived" are filled by pct_config_finalize exactly as B.h derives them.
 */
typedef struct pct_config {
    /* reconstruction grid (B.h:382-393) */
    int32_t COLUMNS, ROWS, SLICES, NUM_VOXELS;             /* NUM_VOXELS derived           */
    double VOXEL_WIDTH, VOXEL_HEIGHT, VOXEL_THICKNESS;      /* cm                           */
    double RECON_CYL_RADIUS, RECON_CYL_HEIGHT;              /* cm                           */
    /* tracker planes and binning (B.h:347-367) */
    double GANTRY_ANGLE_INTERVAL;                           /* degrees                      */
    double SSD_T_SIZE, SSD_V_SIZE;                          /* cm                           */
    double T_BIN_SIZE, V_BIN_SIZE, ANGULAR_BIN_SIZE;        /* cm, cm, degrees              */
    int32_t T_BINS, V_BINS, ANGULAR_BINS, NUM_BINS;         /* derived                      */
    int32_t SIGMAS_TO_KEEP, SAMPLE_STD_DEV;
    /* FBP (B.h:368-371, 474-480, 745) */
    int32_t SINOGRAM_FILTER, MEDIAN_FILTER_FBP;
    int32_t FBP_MED_FILTER_RADIUS;
    int32_t PATH_CTA_THREADS;      /* histories per CTA of the MLP path kernel: 64, 128 (default)
                                      or 256; chosen by pct_autotune                           */
    double SOURCE_RADIUS, FBP_THRESHOLD, RSP_AIR;
    /* hull detection (B.h:395-405) */
    double SC_LOWER_THRESHOLD, SC_UPPER_THRESHOLD;
    double MSC_LOWER_THRESHOLD, MSC_UPPER_THRESHOLD;
    double SM_LOWER_THRESHOLD, SM_UPPER_THRESHOLD, SM_SCALE_THRESHOLD;
    int32_t MSC_DIFF_THRESH, ENDPOINTS_HULL;
    int32_t SC_ON, MSC_ON, SM_ON;
    int32_t PATH_ORDER_WINDOW;     /* order of the MLP path kernel's histories: 0 (default) sorts
                                      each chunk of DROP blocks by path length; W > 0 sorts each
                                      window of W consecutive histories on its own; chosen by
                                      pct_autotune                                             */
    /* MLP (B.h:407-412) */
    double MLP_U_STEP;                                      /* cm (reference: VOXEL_WIDTH/2) */
    int32_t MIN_MLP_LENGTH;
    /* DROP (B.h:335, 419-423) */
    float LAMBDA;                                           /* float, as the reference global */
    int32_t DROP_BLOCK_SIZE, ITERATIONS;
    int32_t HISTORIES_PER_BLOCK;   /* >0: process floor(B/HPB)*HPB histories per DROP block
                                      (the reference launch arithmetic, B.cu:9558); 0: all   */
    /* engine options */
    int32_t PRECISION;             /* PCT_PRECISION_EXACT: the reference's arithmetic (voxel
                                      lists bit-identical); PCT_PRECISION_MIXED: FP64 Sigma
                                      algebra, FP32 solve and voxel indices in the path kernel
                                      (path storage and pct_mlp_paths; the single-pass kernel
                                      stays exact), and the DROP update in FP32 with a
                                      compensated sum of x; PCT_PRECISION_MIXED_COMPENSATED:
                                      MIXED plus a compensated per-voxel accumulation of the
                                      updates (a second float array of rounding errors)        */
    int32_t SCATTER_MODE;          /* PCT_SCATTER_*                                            */
    int32_t THREADS_PER_HISTORY;   /* lanes per history in the DROP-block kernel: 0 or 32 (one warp) */
    int32_t PATH_CHUNK_BLOCKS;     /* path kernel launched per run of this many DROP blocks on a
                                      second stream, overlapping the DROP blocks of the previous
                                      run; 0: one launch per path-storage superblock, before
                                      its DROP blocks                                          */
    int32_t EXACT_FAST_POINTS;     /* exact mode: 1 (default) computes each MLP point with
                                      reciprocals and fused multiply-adds plus a forward error
                                      bound, and recomputes the point in the reference's
                                      operation order whenever the bound cannot prove its voxel
                                      (the voxel lists are the reference's either way); 0: every
                                      point in the reference's operation order               */
    /* projection data reader (B.h:291, 302, 355-357) */
    int32_t DATA_IN_MM;            /* tracker files hold mm: multiply by MM_TO_CM on read      */
    int32_t USE_CONT_ANGLES;       /* PCTN files: use the per-history projection angles        */
    double T_SHIFT, U_SHIFT, V_SHIFT;                       /* cm, added after the conversion */
    /* total variation superiorization (B.h:427-443) */
    int32_t TVS_ON, TVS_OLD;       /* NTVS_ON = TVS_ON && !TVS_OLD                             */
    int32_t TVS_FIRST;             /* perturb before (1) or after (0) each DROP iteration       */
    int32_t TVS_CONDITIONED;       /* accept a perturbation only if it does not raise the TV    */
    int32_t TVS_REPETITIONS;       /* perturbations per DROP iteration (TVS_OLD: 1)             */
    int32_t TVS_L_0;               /* L_0: first exponent of the beta = A^L sequence            */
    double TVS_A;                  /* A                                                        */
    double TVS_MIN_ETA;            /* smallest tabulated beta                                   */
    double TV_THRESHOLD;           /* B.h defines (1/1000), an integer division: 0             */
    int64_t TVS_SEED;              /* seed of the NTVS draw of L (the reference seeds it from
                                      the wall clock)                                          */
    /* projection algorithm and history ordering (B.h:175, 181, 416-419, 464-465) */
    int32_t PROJECTION_ALGORITHM;  /* PCT_DROP; PCT_ROBUSTA / PCT_ROBUSTB: the robust updates
                                      DROP_blocks_robust1 / _robust2 (O.cu:7537, 7554)          */
    int32_t PSI_SIGN;              /* +1 / -1: sign of the robust perturbation Psi              */
    double ETA;                    /* robust perturbation coefficient                           */
    int32_t RECON_HISTORY_ORDERING;/* PCT_SEQUENTIAL or PCT_PRIME_PERMUTATION                   */
    int32_t IDENTIFY_X_N_AIR;      /* image update: voxels below X_N_AIR_THRESHOLD become 0     */
    int64_t PRIME_OFFSET;          /* step of the prime-permutation history order               */
    double X_N_AIR_THRESHOLD;
    /* S-curve attenuation of the DROP update along each path (B.h:178, 467-470; B.cu:9529-9534,
       10606-10649): entry j of an n-entry path adds s(k) * L * residual / <a,a> * LAMBDA, with
       k = min(j, n-1-j) (DUAL_SIDED_S_CURVE) or k = j, and s the curve S_CURVE.  The reference's
       kernel selects the curve with `#if (S_CURVE == SIGMOID)`, where both names are enum
       constants and so evaluate to 0 in the preprocessor: its build always uses SIGMOID.        */
    int32_t S_CURVE_ON;            /* 0 (default, the reference's OFF) or 1; needs PRECISION EXACT
                                      and PROJECTION_ALGORITHM DROP                              */
    int32_t S_CURVE;               /* PCT_SIGMOID (default) ... PCT_LIN_OVER_ROOT               */
    int32_t DUAL_SIDED_S_CURVE;    /* 1 (default): attenuate both ends of the path; 0: the start */
    int32_t SIGMOID_MID_SHIFT;     /* 10: the sigmoid's midpoint k0.  The reference subtracts it
                                      from the unsigned index in unsigned arithmetic, so indices
                                      below it wrap to about 4.3e9 and scale by exactly 1        */
    double SIGMOID_STEEPNESS;      /* 1.25: s(k) = 1 / (1 + exp(-STEEPNESS * (k - MID_SHIFT)))  */
} pct_config;

/* Size of pct_config as compiled into the library (bindings check their mirror against it). */
size_t pct_config_size(void);
/* Fill cfg with the reference's built-in defaults (B.h values). */
void pct_config_default(pct_config* cfg);
/* Set one parameter by its reference / settings.cfg key name ("LAMBDA", "COLUMNS", ...). */
pct_status pct_config_set(pct_config* cfg, const char* key, const char* value);
/* Parse a settings.cfg file ("KEY = value // comment" lines; replaces Configurations.h:838-987). */
pct_status pct_config_load(pct_config* cfg, const char* path);
/* Compute derived fields (NUM_VOXELS, T_BINS, ...) as B.h:356-393 does and validate. */
pct_status pct_config_finalize(pct_config* cfg);
/* Why the calling thread's last failed pct_config_set, pct_config_load or pct_config_finalize
 * failed ("" after a success of pct_config_load or pct_config_finalize); valid until the thread's
 * next call of one of them. */
const char* pct_config_last_error(void);

typedef struct pct_ctx pct_ctx;

/* Create a context on CUDA device `device` (the reference's cudaSetDevice loop, B.cu:373-387,
 * becomes an explicit argument).  Builds the MLP lookup tables (B.cu:8527) on the host and
 * uploads them. */
pct_status pct_create(const pct_config* cfg, int device, pct_ctx** out);
void pct_destroy(pct_ctx* ctx);
const char* pct_status_string(pct_status s);
/* Last error message of this context ("" if none).  With ctx NULL: why the calling thread's last
 * pct_create failed ("" after a success). */
const char* pct_last_error(const pct_ctx* ctx);
/* Use an external cudaStream_t (passed as void*); NULL restores the context's own stream. */
pct_status pct_set_stream(pct_ctx* ctx, void* stream);
pct_status pct_synchronize(pct_ctx* ctx);

/*
 * Histories entering reconstruction: the reference's global vectors after
 * reconstruction_cuts (B.h:1257-1271; filled at B.cu:8286-8294), structure-of-arrays.
 */
typedef struct pct_histories {
    const float* x_entry;
    const float* y_entry;
    const float* z_entry;
    const float* x_exit;
    const float* y_exit;
    const float* z_exit;
    const float* xy_entry_angle;
    const float* xz_entry_angle;
    const float* xy_exit_angle;
    const float* xz_exit_angle;
    const float* WEPL;
    const uint32_t* first_MLP_voxel;
} pct_histories;

/* Copy n histories into the context (replaces DROP_allocations + DROP_host_2_device,
 * B.cu:9459-9500).  `where` says whether the pointers are host or device memory. */
pct_status pct_set_reconstruction_histories(pct_ctx* ctx, const pct_histories* h, int64_t n,
                                            pct_memory where);

/* Double-buffered history upload (no reference counterpart; the reference copies the histories
 * once before DROP_GPU, B.cu:9481).  pct_stage_reconstruction_histories starts copying n histories
 * into a staging area on a separate copy stream and returns at once: the current histories and
 * any DROP work in flight are untouched, so the upload overlaps the running iteration.  The
 * arrays must stay valid until the copy has run (pinned host memory for an asynchronous copy).
 * pct_use_staged_histories then makes them the reconstruction histories, ordered after the
 * upload on the context's stream (a device-side copy), exactly as pct_set_reconstruction_histories
 * would.  A second stage call waits on the device until the previous staged set has been used. */
pct_status pct_stage_reconstruction_histories(pct_ctx* ctx, const pct_histories* h, int64_t n, pct_memory where);
pct_status pct_use_staged_histories(pct_ctx* ctx);
int64_t pct_reconstruction_histories(const pct_ctx* ctx);

/* Reorder the loaded histories by the prime permutation of apply_history_sequence (B.cu:8691,
 * generate_history_sequence B.cu:8664): history i of the new order is old history
 * (i * prime_offset) mod n.  PCT_ERR_ARG when prime_offset and n share a factor (the sequence
 * would repeat).  pct_reconstruction_cuts applies it with PRIME_OFFSET when
 * RECON_HISTORY_ORDERING is PCT_PRIME_PERMUTATION. */
pct_status pct_apply_history_sequence(pct_ctx* ctx, int64_t prime_offset);

/* Image transfers: x_host_2_GPU / x_GPU_2_host (B.cu:9420-9427).  NUM_VOXELS floats. */
pct_status pct_set_image(pct_ctx* ctx, const float* x, pct_memory where);
pct_status pct_get_image(pct_ctx* ctx, float* x, pct_memory where);

/* One DROP iteration over all loaded histories: sequential blocks of DROP_BLOCK_SIZE, each an
 * MLP + scatter kernel followed by the image update (DROP_full_tx_iteration, B.cu:9537). */
pct_status pct_drop_full_tx_iteration(pct_ctx* ctx, int iteration);
/* ITERATIONS DROP iterations (DROP_GPU, B.cu:9848), each preceded (TVS_FIRST) or followed by
 * pct_ntvs_iteration when TVS_ON; the reference's text and image dumps are left out. */
pct_status pct_drop_gpu(pct_ctx* ctx);

/* Total variation superiorization on the device image (NTVS_iteration B.cu:10606 ->
 * iteratively_perturb_image B.cu:10476, or iteratively_perturb_image_unconditional B.cu:10562
 * when TVS_CONDITIONED is off).  `iteration` is the DROP iteration k (>= 1) of the L draw
 * L = randi(L_0 + k - 1, L); the draw is a seeded hash of (TVS_SEED, k).  Needs the hull
 * (preprocessing, or pct_set_array "hull").  Kernels only, no host synchronisation. */
pct_status pct_ntvs_iteration(pct_ctx* ctx, int iteration);
/* calculate_total_variation (B.cu:10163) of the current image, accumulated in double. */
pct_status pct_total_variation(pct_ctx* ctx, double* tv);
/* Read (*L_out) and/or set (*L_in) the TVS exponent L (the reference's global L, B.h:438). */
pct_status pct_tvs_L(pct_ctx* ctx, int32_t* L_out, const int32_t* L_in);

/* Path storage (no reference counterpart).  An iteration first writes every history's MLP voxel
 * list to device memory (one launch over many DROP blocks), then runs the DROP blocks over the
 * stored lists.  `bytes` caps that storage: 0 = 75% of free device memory, > 0 = that many bytes
 * (the histories are then processed in runs of whole DROP blocks that fit), < 0 = no storage
 * (each block recomputes its paths in a single fused kernel).  Results are the same either way. */
pct_status pct_set_path_storage_limit(pct_ctx* ctx, int64_t bytes);
/* Number of path-storage runs the loaded histories need (0 = single-pass kernel, -1 = error). */
int pct_path_storage_superblocks(pct_ctx* ctx);
/* Precomputed-path DROP (no reference API; the reference's precalculated-MLP mode is
 * DROP_calculate_update_GPU_blocks O.cu:7145 over paths written by
 * accumulate_and_export_preprocessed_data O.cu:6615).  With enable != 0 and every history's path
 * resident (pct_path_storage_superblocks == 1), the first iteration computes and keeps the MLP
 * paths and later iterations run the DROP blocks alone; the paths do not depend on the image, so
 * the result is that of recomputing them.  Loading new histories drops the kept paths. */
pct_status pct_set_path_reuse(pct_ctx* ctx, int enable);

/* L2 persistence for the image and the {x_update, S} accumulator (no reference counterpart).
 * enable != 0 sets aside persisting L2 (up to the device's maximum, for this context's lifetime)
 * and gives every kernel of the captured DROP iteration an access-policy window over the image
 * and accumulator (one allocation), so the streamed history and path data cannot evict them;
 * 0 releases it.  The captured iteration is rebuilt on the next call.  Off by default. */
pct_status pct_set_l2_window(pct_ctx* ctx, int enable);

/* Schedule autotuner (no reference counterpart): times one DROP iteration of this context's
 * histories per candidate and keeps the fastest, one knob at a time: PATH_CHUNK_BLOCKS in
 * {0, 4, 8, 16, 32, 64, 128}, then PATH_CTA_THREADS (histories per path-kernel CTA) in
 * {64, 128, 256}, then PATH_ORDER_WINDOW in {0, 4096, 16384}; chosen[] receives the three.  The
 * knobs only change the schedule, so results do not change; the image is restored.  Call after
 * loading the histories (and before pct_batch_create).  pct_autotune runs the same search and
 * reports the chunking. */
pct_status pct_autotune_schedule(pct_ctx* ctx, int32_t chosen[3]);
pct_status pct_autotune(pct_ctx* ctx, int32_t* chosen_path_chunk_blocks);

/* One DROP iteration launched kernel by kernel (not from the captured graph) with CUDA events
 * around every launch on the context's stream; synchronises.  ms_out / launches_out receive, per
 * launch group, the summed kernel time and the launch count: [0] MLP path kernel (two-phase
 * only), [1] DROP block kernel (gather/update/scatter, or the fused MLP+scatter kernel),
 * [2] image update.  The image advances by one iteration, as with pct_drop_full_tx_iteration. */
pct_status pct_profile_drop_iteration(pct_ctx* ctx, double ms_out[3], int64_t launches_out[3]);

/* The two per-block launches of a DROP iteration, for callers that drive blocks themselves:
 * MLP + scatter for histories [start_position, start_position + num_histories)
 * (calculate_x_update_GPU launch, B.cu:9558-9564), and the image update that applies and clears
 * the accumulated block (image_update_GPU, B.cu:9576).  Both are enqueued on the context's
 * stream and return without synchronising. */
pct_status pct_calculate_x_update(pct_ctx* ctx, int64_t start_position, int64_t num_histories);
pct_status pct_image_update(pct_ctx* ctx);

/*
 * MLP voxel lists for histories [start, start+n) of the loaded set, for parity checks
 * (find_MLP_path_GPU_tabulated, B.cu:9104, as called from calculate_x_update_GPU, B.cu:9321).
 * Outputs (all `where` memory): path_counts[n]; path_voxels[n*stride] (row h holds
 * path_counts[h] voxels, truncated at stride, overflow reported as PCT_ERR_OOB);
 * chord_lengths[n] (effective chord length, cm); a_dot_x[n] (sum of x over the path,
 * before the chord-length factor).  Any output pointer may be NULL.
 */
pct_status pct_mlp_paths(pct_ctx* ctx, int64_t start, int64_t n, int32_t stride,
                         uint32_t* path_counts, uint32_t* path_voxels, double* chord_lengths,
                         double* a_dot_x, pct_memory where);

/* Precision report of the mixed-precision MLP (no reference counterpart): for histories
 * [start, start+n) the exact (reference) and mixed-precision MLP points of every step are
 * computed side by side; per history the largest |t_mixed - t_exact| and |v_mixed - v_exact|
 * (cm) and the number of steps whose voxel differs, over the steps where the reference's Sigma_2
 * is well conditioned (1 - rho^2 > 1e-3; the scattering model gives about 1/4); ill_posed_steps
 * counts the others (near the exit the tabulated moments cancel to noise and the reference's
 * point there is arbitrary in any precision). */
pct_status pct_mlp_precision(pct_ctx* ctx, int64_t start, int64_t n, double* dev_t_cm, double* dev_v_cm,
                             int32_t* mismatched_steps, int32_t* ill_posed_steps, pct_memory where);

/* One DROP block without allocating device memory (no counterpart in the reference).  For
 * callers that cannot call cudaMalloc/cudaFree while they reconstruct -- a real-time service
 * whose allocations would synchronise the device and stall other streams, or a host that gives
 * the library a fixed device-memory budget.  h (n histories) and x (NUM_VOXELS floats, updated in
 * place) are the caller's device memory; the block's MLP + scatter and the image update run on
 * the context's stream.  The {x_update, S} accumulator is a static 2359296-voxel array in the
 * library (18 MiB held on every GPU that loads it); configurations with more voxels get
 * PCT_ERR_ARG.  All calls on a device share that array: calls that overlap on the GPU race and
 * must be serialised.  The first call on a device looks up the array's address; make it before
 * any stream capture begins.  The context's own image and histories are not touched.
 * x must be 8-byte aligned (PCT_ERR_ARG otherwise).  A path entry at or beyond NUM_VOXELS reads
 * x as 0 and receives no update, and is counted in pct_get_counters like any out-of-grid entry.
 * The MLP is always the exact (FP64) walk, whatever the context's PRECISION setting, as in
 * pct_calculate_x_update; PROJECTION_ALGORITHM must be DROP, SCATTER_MODE ATOMIC and S_CURVE_ON 0. */
pct_status pct_drop_block_update_noalloc(pct_ctx* ctx, const pct_histories* h, int64_t n, float* x);

/* ---------------------------------------------------------------------------------------
 * Preprocessing: tracker data -> reconstruction histories and the initial image
 * (preprocessing() B.cu:7394 and the start of image_reconstruction() B.cu:10650).
 * Stage calls run on the context's stream in the reference's order; each names the
 * reference function it replaces.  Intermediate arrays are readable by their reference
 * names through pct_get_array.
 * --------------------------------------------------------------------------------------- */

/* Tracker hits per history after the reader's mm->cm conversion (read_data_chunk, B.cu:4361):
 * t/u/v on the two entry and two exit planes, WEPL, and the projection angle in degrees. */
typedef struct pct_tracker_data {
    const float *t_in_1, *t_in_2, *t_out_1, *t_out_2;
    const float *u_in_1, *u_in_2, *u_out_1, *u_out_2;
    const float *v_in_1, *v_in_2, *v_out_1, *v_out_2;
    const float* WEPL;
    const float* gantry_angle; /* degrees */
} pct_tracker_data;

/* Load n histories of tracker data.  integer_angles != 0 truncates the angle to whole degrees,
 * as the discrete-angle reader does (gantry_angle is an int there); 0 keeps the continuous
 * angle (the USE_CONT_ANGLES path, recon_volume_intersections_GPU_exact_angles B.cu:5022). */
pct_status pct_load_tracker_data(pct_ctx* ctx, const pct_tracker_data* t, int64_t n, pct_memory where,
                                 int integer_angles);
/* recon_volume_intersections (B.cu:4767): entry/exit points and angles, missed_recon_volume. */
pct_status pct_recon_volume_intersections(pct_ctx* ctx);
/* binning (B.cu:5373): bin numbers, per-bin counts and sums, then the history vectors keep the
 * histories that hit the volume, in order. */
pct_status pct_binning(pct_ctx* ctx);
/* hull_detection (B.cu:6607): SC carving / MSC and SM counts over the histories of the last
 * pct_binning call, for the hulls switched on by SC_ON / MSC_ON / SM_ON. */
pct_status pct_hull_detection(pct_ctx* ctx);
/* calculate_means / sum_squared_deviations / calculate_standard_deviations / statistical_cuts
 * (B.cu:5608-5971); statistical_cuts keeps the surviving histories, in order, and builds the
 * sinogram sums. */
pct_status pct_calculate_means(pct_ctx* ctx);
pct_status pct_sum_squared_deviations(pct_ctx* ctx);
pct_status pct_calculate_standard_deviations(pct_ctx* ctx);
pct_status pct_statistical_cuts(pct_ctx* ctx);
/* construct_sinogram (B.cu:6039) and FBP (B.cu:6080): filter, backprojection, median filter,
 * and the FBP hull when ENDPOINTS_HULL is FBP_HULL. */
pct_status pct_construct_sinogram(pct_ctx* ctx);
pct_status pct_FBP(pct_ctx* ctx);
/* hull_detection_finish (B.cu:7276: MSC / SM edge detection) and hull_selection (B.cu:7351). */
pct_status pct_hull_detection_finish(pct_ctx* ctx);
pct_status pct_hull_selection(pct_ctx* ctx);
/* define_initial_iterate with X_0 = HYBRID (B.cu:8612): x = median-filtered FBP inside the hull. */
pct_status pct_define_initial_iterate(pct_ctx* ctx);
/* reconstruction_cuts (B.cu:8296): hull entry/exit search for each history vector entry; the
 * histories that hit the hull on both sides become the reconstruction histories of the DROP
 * stage (as pct_set_reconstruction_histories). */
pct_status pct_reconstruction_cuts(pct_ctx* ctx);
/* All of the above in the reference's order. */
pct_status pct_preprocessing(pct_ctx* ctx, const pct_tracker_data* t, int64_t n, pct_memory where,
                             int integer_angles);
/* Replace the history vectors (geometry and WEPL of h; bin numbers cleared), e.g. to run
 * pct_reconstruction_cuts on histories prepared elsewhere. */
pct_status pct_set_history_vectors(pct_ctx* ctx, const pct_histories* h, int64_t n, pct_memory where);

/* Named arrays, by the reference's variable names: tracker inputs ("t_in_1", ...), per-history
 * stage outputs ("x_entry", ..., "missed_recon_volume" uint8, "bin_num" int32), the current
 * history vectors ("x_entry_vector", ..., "WEPL_vector", "bin_num_vector",
 * "first_MLP_voxel_vector"), bins ("bin_counts" int32, "mean_WEPL", "stddev_WEPL",
 * "sinogram", "sinogram_filtered", ...), images ("FBP_image", "FBP_median_filtered",
 * "SC_hull"/"FBP_hull"/"hull" uint8, "MSC_counts"/"SM_counts" int32, "x"), and the loaded
 * reconstruction histories in reconstruction order ("x_entry_reconstruction", ...,
 * "WEPL_reconstruction", "first_MLP_voxel_reconstruction" uint32).
 * pct_array_length gives the element count (-1 if unknown or not yet produced). */
int64_t pct_array_length(pct_ctx* ctx, const char* name);
pct_status pct_get_array(pct_ctx* ctx, const char* name, void* dst, int64_t capacity_bytes, pct_memory where);
pct_status pct_set_array(pct_ctx* ctx, const char* name, const void* src, int64_t bytes, pct_memory where);

/* ---------------------------------------------------------------------------------------
 * Projection data files (count_histories_v0 B.cu:3578, read_data_chunk_v0 B.cu:4361).
 * One file per gantry angle, named "<directory>/projection_<angle %03d>.bin" (B.h:596-597).
 * Layout (little endian): magic "PCTD" (or "PCTN": continuous-angle data), int32 version
 * (0 or 1), int32 number of histories N, float projection angle (degrees), float beam energy
 * (MeV), int32 generation date, int32 preprocess date, three strings each preceded by its
 * int32 length (phantom name, data source, prepared by), then 13 float arrays of N values in
 * the order t0..t3, v0..v3, u0..u3, WEPL (mm), optionally followed by N per-history projection
 * angles (degrees; PCTN files and version 1).
 * --------------------------------------------------------------------------------------- */
typedef struct pct_projection_header {
    int32_t continuous;        /* 1 for magic "PCTN" (CONTINUOUS_DATA), 0 for "PCTD"        */
    int32_t version;           /* VERSION_ID: 0 or 1                                         */
    int32_t num_histories;
    float projection_angle;    /* degrees                                                    */
    float beam_energy;         /* MeV                                                        */
    int32_t generation_date, preprocess_date;     /* Unix time                               */
    int32_t has_angles;        /* the file holds the per-history angle array                 */
    int64_t data_offset;       /* bytes before the first t0 value (SKIP_2_DATA_SIZE)         */
    char phantom_name[256], data_source[256], prepared_by[256];  /* NUL-terminated, cut    */
} pct_projection_header;

/* Host arrays of one file's data in file units (mm); angles may be NULL. */
typedef struct pct_projection_arrays {
    float *t_in_1, *t_in_2, *t_out_1, *t_out_2;   /* t0..t3 */
    float *v_in_1, *v_in_2, *v_out_1, *v_out_2;   /* v0..v3 */
    float *u_in_1, *u_in_2, *u_out_1, *u_out_2;   /* u0..u3 */
    float* WEPL;
    float* projection_angle;                      /* per-history angles (degrees) */
} pct_projection_arrays;

/* Parse the header of one file (count_histories_v0 B.cu:3578).  PCT_ERR_IO for a missing file,
 * an unknown magic number or version, or a file shorter than its 13 data arrays. */
pct_status pct_read_projection_header(const char* path, pct_projection_header* header);
/* Read one file's data arrays as stored (the fread sequence of read_data_chunk_v0 B.cu:4401-4422),
 * at most `capacity` histories per array; a non-NULL out->projection_angle needs has_angles. */
pct_status pct_read_projection_file(const char* path, int64_t capacity, const pct_projection_arrays* out,
                                    pct_projection_header* header);
/* Write one file in the format above (the writer of combine_data_sets B.cu:3822, no reference
 * API); header->continuous / version / projection_angle / beam_energy / dates / strings are
 * written, num_histories and data_offset are set from n.  in->projection_angle may be NULL
 * (then no angle array is written). */
pct_status pct_write_projection_file(const char* path, const pct_projection_header* header,
                                     const pct_projection_arrays* in, int64_t n);
/* count_histories + read_data_chunk for a whole scan (B.cu:3504, 4139): read every gantry
 * angle's file (0 <= angle < 360 in steps of int(GANTRY_ANGLE_INTERVAL)) into the context's
 * tracker arrays, convert mm to cm (DATA_IN_MM, convert_mm_2_cm B.cu:4070) and add the
 * T/U/V shifts (apply_tuv_shifts B.cu:4100) on the device, and set the angle of each history:
 * int(file projection angle), or the per-history angle when a file is PCTN and
 * USE_CONT_ANGLES is set.  Equivalent to pct_load_tracker_data with the converted arrays;
 * *n_out receives the number of histories.  File reads overlap the host-to-device copies. */
pct_status pct_load_projection_data(pct_ctx* ctx, const char* directory, int64_t* n_out);
/* preprocessing() as the reference runs it (B.cu:7394): pct_load_projection_data, then the
 * stages of pct_preprocessing. */
pct_status pct_preprocessing_from_files(pct_ctx* ctx, const char* directory);

/* ---------------------------------------------------------------------------------------
 * Batches (no reference counterpart: the reference reconstructs one compile-time grid per run).
 * A batch runs one DROP iteration of several scans' contexts -- each with its own grid, histories
 * and image, all on one device -- as a single graph launch; each context's captured iteration is
 * a child graph on its own branch, so the scans run concurrently.  Every scan's result is the one
 * its own pct_drop_full_tx_iteration gives (bit for bit with SCATTER_MODE DETERMINISTIC).  The
 * batch runs on its own stream: call pct_batch_synchronize before touching a context again.
 * --------------------------------------------------------------------------------------- */
typedef struct pct_batch pct_batch;
pct_status pct_batch_create(pct_ctx* const* ctxs, int n, pct_batch** out);
void pct_batch_destroy(pct_batch* batch);
pct_status pct_batch_drop_iteration(pct_batch* batch, int iteration);
pct_status pct_batch_synchronize(pct_batch* batch);
const char* pct_batch_last_error(const pct_batch* batch);
/* The batch's cudaStream_t (as void*), e.g. to time a batch iteration with events. */
void* pct_batch_stream(pct_batch* batch);

/* ---------------------------------------------------------------------------------------
 * Preprocessed data (accumulate_and_export_preprocessed_data O.cu:6615 and the export_* /
 * import_* functions O.cu:6540-6780).  Files in `directory`, each a uint32 history count then
 * the arrays: histories.bin (x/y/z_entry, x/y/z_exit, xy/xz_entry_angle, xy/xz_exit_angle as
 * float[n] each, first_MLP_voxel uint32[n]), WEPL.bin (float[n]), voxels_per_path.bin
 * (uint32[n]), avg_chord_lengths.bin (double[n]), MLP_paths.bin (the concatenated voxel lists,
 * uint32); and without a count x_0.bin (the current image, float[NUM_VOXELS]) and hull.bin
 * (uint8[NUM_VOXELS], when a hull exists).
 * --------------------------------------------------------------------------------------- */
/* Write the loaded reconstruction histories, their MLP paths, the image and the hull. */
pct_status pct_export_preprocessed(pct_ctx* ctx, const char* directory);
/* Load histories (and image, hull when present); when the path files are present and every path
 * is resident, the paths go straight into path storage for precomputed-path DROP. */
pct_status pct_import_preprocessed(pct_ctx* ctx, const char* directory);

/* The context's S-curve scale table: scales[k] = s(k) for k in [0, count), count at most
 * PCT_MLP_PATH_CAP, computed on the device with the reference's expressions and CUDA's math
 * functions (sigmoid_GPU ... linear_over_root_GPU, B.cu:10606-10626).  PCT_ERR_STATE when the
 * configuration has S_CURVE_ON 0. */
pct_status pct_get_s_curve(pct_ctx* ctx, float* scales, int32_t count);

/* Device counters accumulated since the last reset: [0] MLP voxel indices outside the padded
 * image, [1] MLP paths longer than the path buffer, [2] histories whose u-extent exceeds the
 * MLP polynomial tables, [3] bounded loops that hit their bound (hull walks that would not
 * terminate in the reference). */
pct_status pct_get_counters(pct_ctx* ctx, int64_t counters[4]);
pct_status pct_reset_counters(pct_ctx* ctx);

/* Kernel launches issued by this context since creation (for launch accounting). */
int64_t pct_kernel_launches(const pct_ctx* ctx);

/* Device self-check (no reference counterpart): compares CUDA powf(f, 2.0f) with the correctly
 * rounded float product f*f over n inputs spread across the float range on the current device;
 * *mismatches receives the count (the exact MLP mode relies on it being 0). */
pct_status pct_selftest_powf_square(int64_t n, uint64_t seed, int64_t* mismatches);
/* The largest distance, in float ulps, between powf(f, 2.0f) and the correctly rounded f*f over
 * every float f of magnitude in [2^-60, 2^60) and zero (the CPU oracle squares with f*f, so this
 * bounds each square behind an engine-vs-oracle tie). */
pct_status pct_selftest_powf_square_max_ulp(int64_t* max_ulp);

/* Measurement support (no reference counterpart).  pct_fp64_fma_rate: the FP64 fused-multiply-add
 * issue rate of `device` (FMA instructions per second, all SMs, timed with CUDA events), the peak
 * against which the exact MLP's FP64 work is reported.  pct_mlp_steps: per history of
 * [start, start+n) the number of MLP points the walk computes (the loop trips of
 * find_MLP_path_GPU_tabulated, B.cu:9159-9255). */
pct_status pct_fp64_fma_rate(int device, double* fma_per_second);
pct_status pct_mlp_steps(pct_ctx* ctx, int64_t start, int64_t n, int32_t* steps, pct_memory where);

/* ---------------------------------------------------------------------------------------
 * Learned DROP initializer (no reference counterpart).  The reference starts DROP from
 * x_0 = FBP_median x hull (define_initial_iterate, B.cu:8582-8646); these calls let a 3-D
 * convolutional encoder-decoder (4 levels, 16 -> 128 channels, 3x3x3 kernels, bf16 weights and
 * activations, fp32 accumulation on the tensor cores) replace x_0 by an estimate of the
 * converged DROP image: image = x_0 + hull * network(x_0, hull).  The network is trained on the
 * device by its own forward and backward kernels (masked mean-squared error over the hull,
 * Adam).  A network is made for one grid (COLUMNS, ROWS, SLICES, each divisible by 8); its
 * parameters (a flat fp32 vector: per layer W[cout][27][cin] then bias[cout]) do not depend on
 * the grid.  Device pointers throughout; calls return when their work is done.
 * --------------------------------------------------------------------------------------- */
typedef struct pct_unet pct_unet;
pct_status pct_unet_create(int columns, int rows, int slices, int64_t seed, int device, pct_unet** out);
pct_status pct_unet_destroy(pct_unet* net);
const char* pct_unet_last_error(const pct_unet* net);
pct_status pct_unet_param_count(const pct_unet* net, int64_t* count);
pct_status pct_unet_get_params(pct_unet* net, float* host_params, int64_t count);
/* Sets the parameters and restarts the optimizer state. */
pct_status pct_unet_set_params(pct_unet* net, const float* host_params, int64_t count);
/* image[V] = x0 + hull * network(x0, hull); x0, hull (uint8 0/1) and image are NUM_VOXELS long. */
pct_status pct_unet_forward(pct_unet* net, const float* x0, const uint8_t* hull, float* image);
/* Loss (mean squared error over hull voxels against target) and its gradient with respect to
 * every parameter (host array of pct_unet_param_count floats, or NULL); no update. */
pct_status pct_unet_gradients(pct_unet* net, const float* x0, const uint8_t* hull, const float* target,
                              float* host_grads, double* loss);
/* One Adam step (beta 0.9 / 0.999) on one volume; *loss receives the loss before the step. */
pct_status pct_unet_train_step(pct_unet* net, const float* x0, const uint8_t* hull, const float* target,
                               float learning_rate, double* loss);
/* Replaces the context's image (x_0 after preprocessing) by the network's estimate, on the
 * context's stream; the hull of the preprocessing stages is the network's second input.  If any
 * voxel of the estimate is not finite the image is left at x_0 (the FBP start) and
 * PCT_ERR_STATE is returned. */
pct_status pct_learned_initial_iterate(pct_ctx* ctx, pct_unet* net);
/* One 3x3x3 convolution (padding 1) on channels-last bf16 tensors, as the network runs it:
 * out[v][co] = ReLU?( sum_{t,ci} weight[co][t][ci] in[v+t][ci] + bias[co] + residual[v][co] ),
 * then zeroed where mask[v][co] <= 0; upsample != 0 reads in at half resolution (nearest).
 * cin, cout in {16, 32, 64, 128}; bias, residual and mask may be NULL.  stream: cudaStream_t. */
pct_status pct_conv3d_bf16(const uint16_t* in, int cin, int columns, int rows, int slices, int upsample,
                           const uint16_t* weight, int cout, const float* bias, const uint16_t* residual,
                           const uint16_t* mask, int relu, uint16_t* out, void* stream);
/* Weight gradient of that convolution: dweight[co][t][ci] += sum_v dz[v][co] in[v+t][ci]. */
pct_status pct_conv3d_bf16_wgrad(const uint16_t* in, int cin, int columns, int rows, int slices, int upsample,
                                 const uint16_t* dz, int cout, float* dweight, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* PCT_API_H */
