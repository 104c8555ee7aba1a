// pct_context.h -- the context behind the opaque pct_ctx handle (internal to the engine).
#pragma once

#include <string>
#include <vector>

#include "pct_common.cuh"
#include "pct_kernels.h"
#include "pct_tables.h"

namespace pct {
struct Preproc;  // preprocessing-stage arrays (pct_preprocess.cu)
void preproc_release(Preproc* p);
// Device tracker arrays: 12 tracker coordinates (t_in_1, t_in_2, t_out_1, t_out_2, u_in_1, ...,
// v_out_2), WEPL, projection angle in degrees.
constexpr int kTrackerSlots = 14;
}  // namespace pct
struct pct_ctx;
struct pct_tvs;  // total variation superiorization buffers (pct_tvs.cu)
namespace pct {
void tvs_release(pct_tvs* t);
// The hull of the preprocessing stages (or set through pct_set_array), NULL if none.
const uint8_t* preproc_hull(pct_ctx* ctx);
// Reserve device tracker arrays for n histories and return them (pct_preprocess.cu).
pct_status preproc_reserve_tracker(pct_ctx* ctx, long long n, float* dst[kTrackerSlots]);
// Lay out path storage for the loaded histories (pct_context.cu); no-op when up to date.
pct_status layout_prepare(pct_ctx* ctx);
// The path kernel's gathered inputs (processing order) from position p on.
HistorySoA sorted_path_inputs(const pct_ctx* ctx, long long p);
// The captured full DROP iteration of the context (built on first use); *launches its kernels.
pct_status iteration_graph(pct_ctx* ctx, cudaGraph_t* graph, long long* launches);
// After a batch ran the context's iteration: account launches and path residency.
void iteration_ran(pct_ctx* ctx);
// Mark the tracker arrays as holding n histories (resets the later stages).
void preproc_tracker_loaded(pct_ctx* ctx, long long n, int integer_angles);
}  // namespace pct

struct pct_ctx {
    pct_config cfg;
    pct::Geometry geo;
    int device = 0;
    cudaStream_t own_stream = nullptr;   // highest priority: the DROP block chain
    cudaStream_t path_stream = nullptr;  // lowest priority: path kernel chunks running ahead
    cudaStream_t stream = nullptr;
    std::vector<cudaEvent_t> events;     // fork/join events of the captured iteration
    // MLP tables (one allocation) and per-step table
    double* d_table_block = nullptr;
    pct::Tables tables{};
    pct::StepConst* d_steps = nullptr;
    int kmax = 0;
    // image and accumulator, padded by one slice; one allocation (d_acc follows d_x) so that a
    // single L2 access-policy window can cover both
    float* d_x = nullptr;
    float2* d_acc = nullptr;
    size_t image_block_bytes = 0;
    bool l2_window = false;           // pct_set_l2_window: captured kernels carry the window
    bool trace = false;               // PCT_TRACE set in the environment at pct_create: one stderr line per iteration
    long long graph_captures = 0;     // iteration graphs captured and instantiated
    cudaAccessPolicyWindow l2_policy{};
    float* d_normA = nullptr;  // ROBUSTB: sum of ||a||^2 per voxel over the block
    pct::FixedAcc fixed{nullptr, nullptr};  // SCATTER_MODE DETERMINISTIC accumulator
    // reconstruction histories
    void* d_hist_block = nullptr;
    pct::HistorySoA hist{};
    long long n_hist = 0, cap_hist = 0;
    unsigned long long* d_counters = nullptr;
    // staged histories (pct_stage_reconstruction_histories): uploaded on copy_stream while the
    // current histories are in use, made current by pct_use_staged_histories
    void* d_stage_block = nullptr;
    long long stage_cap = 0, stage_n = 0;
    bool staged = false;
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t stage_done = nullptr, stage_free = nullptr;
    // two-phase layout: per-history path-length bound, offsets into path storage, processing
    // order, voxel-list length and chord; path storage for one superblock of DROP blocks
    struct Superblock {
        long long h_begin, h_end;  // history range (whole DROP blocks)
        long long off_begin;       // offsets[h_begin]
    };
    struct Chunk {
        int sb;                    // superblock index
        long long h_begin, h_end;  // history range (PATH_CHUNK_BLOCKS whole DROP blocks)
    };
    std::vector<Chunk> chunks;
    bool layout_ready = false;
    bool two_phase = false;
    long long path_limit_bytes = 0;  // 0: automatic, < 0: path storage disabled
    long long layout_cap = 0;        // histories the layout arrays hold
    int* d_bounds = nullptr;
    long long* d_offsets = nullptr;
    int* d_perm = nullptr;
    int* d_path_n = nullptr;
    double* d_chord = nullptr;
    long long* d_scan_tmp = nullptr;
    unsigned* d_hist_tmp = nullptr;
    // the path kernel's inputs in its processing order (perm): the ten geometry fields and the
    // first voxel of each history, its path bound and its path-storage offset
    char* d_sorted_block = nullptr;
    long long sorted_cap = 0;  // bytes
    pct::HistorySoA sorted_hist{};
    int* d_bounds_sorted = nullptr;
    long long* d_offsets_sorted = nullptr;
    uint32_t* d_paths = nullptr;
    long long paths_cap = 0;  // elements
    std::vector<Superblock> sbs;
    // captured DROP iteration; with path reuse, a second graph without the path kernel
    cudaGraphExec_t iter_exec = nullptr;
    long long iter_launches = 0;
    // the full iteration for batches (a child graph), captured without programmatic dependent
    // launch: its waiting CTAs would hold SM slots that the other scans' branches can use
    cudaGraph_t batch_graph = nullptr;
    long long batch_launches = 0;
    long long graph_version = 0;       // bumped whenever the captured iterations are released
    bool reuse_paths = false;   // precomputed-path DROP: compute the MLP paths once, reuse them
    bool paths_valid = false;   // d_paths holds every history's path (one superblock)
    cudaGraphExec_t reuse_exec = nullptr;
    long long reuse_launches = 0;
    long long launches = 0;
    std::string last_error;
    // preprocessing stages (tracker data -> reconstruction histories), allocated on first use
    pct::Preproc* pre = nullptr;
    // total variation superiorization, allocated on first use
    pct_tvs* tvs = nullptr;
};
