// pct_drop_exact.cu -- DROP block kernel and MLP-path kernel, exact (FP64, reference-rounding)
// mode.  Compiled with -fmad=false (see pct_mlp.cuh).
//
// drop_block_exact_kernel fuses the reference's calculate_x_update_GPU (B.cu:9321-9380) and
// DROP_block_update_GPU (B.cu:9522-9536): one thread per history computes the MLP voxel list,
// the sum of x over it, the DROP update value
//     upd = L * ((WEPL - L*sum_x) / (powf(L,2)*n)) * lambda        (rounded to float)
// and, when n >= MIN_MLP_LENGTH, scatters (upd, 1) into the interleaved accumulator
// acc[v] = {x_update[v], S[v]} with one 8-byte vector reduction per path entry
// (red.global.add.v2.f32) instead of the reference's two scalar atomics.
#include "pct_kernels.h"
#include "pct_mlp.cuh"

namespace pct {

namespace {

__global__ void __launch_bounds__(128) drop_block_exact_kernel(Geometry g, Tables tab, const StepConst* __restrict__ steps,
                                                               int kmax, const float* __restrict__ x, float2* __restrict__ acc,
                                                               HistorySoA h, long long begin, long long count,
                                                               unsigned long long* counters)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const long long id = begin + i;
    uint32_t path[kPathCap];
    const WalkResult r = mlp_walk_exact<true>(
        g, tab, steps, kmax, x, __ldg(h.first_MLP_voxel + id), __ldg(h.x_entry + id), __ldg(h.y_entry + id),
        __ldg(h.z_entry + id), __ldg(h.x_exit + id), __ldg(h.y_exit + id), __ldg(h.z_exit + id),
        __ldg(h.xy_entry_angle + id), __ldg(h.xz_entry_angle + id), __ldg(h.xy_exit_angle + id),
        __ldg(h.xz_exit_angle + id), [&](int j, uint32_t v) { path[j] = v; });
    if (r.flags) count_flags(r.flags, counters);
    if (r.n < g.min_mlp_length) return;
    const double a_i_dot_a_i = r.aia * r.n;
    const double a_i_dot_x_k = r.axk * r.chord;
    if (g.s_curve) {
        // S_CURVE_ON (B.cu:9530-9531): s(k) * L * ((WEPL - a_i_dot_x_k) / a_i_dot_a_i) * lambda per entry
        const double q = ((double)__ldg(h.WEPL + id) - a_i_dot_x_k) / a_i_dot_a_i;
        for (int j = 0; j < r.n; j++) {
            const uint32_t v = path[j];
            const float s = __ldg(g.s_curve + s_curve_index(g, j, r.n));
            if (v < (uint32_t)g.padded_voxels)
                atomicAdd(acc + v, make_float2((float)((((double)s * r.chord) * q) * g.lambda), 1.0f));
        }
        return;
    }
    const float upd = (float)(r.chord * (((double)__ldg(h.WEPL + id) - a_i_dot_x_k) / a_i_dot_a_i) * g.lambda);
    const float2 add = make_float2(upd, 1.0f);
    for (int j = 0; j < r.n; j++) {
        const uint32_t v = path[j];
        if (v < (uint32_t)g.padded_voxels) atomicAdd(acc + v, add);
    }
}

template <bool kMixed>
__global__ void __launch_bounds__(128) mlp_paths_kernel(Geometry g, Tables tab, const StepConst* __restrict__ steps,
                                                        int kmax, const float* __restrict__ x, HistorySoA h,
                                                        long long begin, long long count, int stride,
                                                        uint32_t* __restrict__ counts, uint32_t* __restrict__ voxels,
                                                        double* __restrict__ chord, double* __restrict__ a_dot_x,
                                                        unsigned long long* counters)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const long long id = begin + i;
    uint32_t* row = voxels ? voxels + i * (long long)stride : nullptr;
    auto emit = [&](int j, uint32_t v) {
        if (row && j < stride) row[j] = v;
    };
    WalkResult r;
    if constexpr (kMixed)
        r = mlp_walk_mixed<true>(g, tab, steps, kmax, x, h.first_MLP_voxel[id], h.x_entry[id], h.y_entry[id],
                                 h.z_entry[id], h.x_exit[id], h.y_exit[id], h.z_exit[id], h.xy_entry_angle[id],
                                 h.xz_entry_angle[id], h.xy_exit_angle[id], h.xz_exit_angle[id], emit);
    else
        r = mlp_walk_exact<true>(g, tab, steps, kmax, x, h.first_MLP_voxel[id], h.x_entry[id], h.y_entry[id],
                                 h.z_entry[id], h.x_exit[id], h.y_exit[id], h.z_exit[id], h.xy_entry_angle[id],
                                 h.xz_entry_angle[id], h.xy_exit_angle[id], h.xz_exit_angle[id], emit);
    if (r.flags) count_flags(r.flags, counters);
    if (r.n > stride && voxels) atomicAdd(counters + kCntPathOverflow, 1ull);
    if (counts) counts[i] = (uint32_t)r.n;
    if (chord) chord[i] = r.chord;
    if (a_dot_x) a_dot_x[i] = r.axk;
}

// Loop trips of the MLP walk per history (the number of MLP points find_MLP_path_GPU_tabulated
// computes, B.cu:9159-9255): the walk's own setup and loop condition (depth_2_go > MLP_U_STEP,
// carried by repeated subtraction), without the point algebra.  The measurement of the path
// kernel's FP64 work multiplies these by the operations of one point.
__global__ void __launch_bounds__(128) mlp_steps_kernel(Geometry g, Tables tab, int kmax, HistorySoA h, long long begin,
                                                        long long count, int* __restrict__ steps)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const long long id = begin + i;
    double xy_entry = h.xy_entry_angle[id], xy_exit = h.xy_exit_angle[id];
    unsigned flags = 0;
    const MlpStart m = mlp_start(g, tab, h.x_entry[id], h.y_entry[id], h.z_entry[id], h.x_exit[id], h.y_exit[id],
                                 h.z_exit[id], xy_entry, xy_exit, h.xz_entry_angle[id], h.xz_exit_angle[id], flags);
    double depth_2_go = m.depth_2_go;
    int k = 1;
    while (m.tables_ok && depth_2_go > g.mlp_u_step && k <= kmax) {
        depth_2_go -= g.mlp_u_step;
        k++;
    }
    steps[i] = k - 1;
}

// Exact and mixed-precision MLP points of the same steps side by side (the precision report):
// per history the largest |t_mixed - t_exact| and |v_mixed - v_exact| (cm) and the number of steps
// whose voxel differs, over the steps where the reference's Sigma_2 is well conditioned
// (1 - rho^2 > 1e-3); the other steps are counted in ill_posed.  Near the exit the tabulated Sigma_2 moments cancel to
// noise (u_2 enters the polynomials at its table grid point but the u_2 factors exactly), the
// determinant goes non-positive and the reference's point there is arbitrary in any precision.
__global__ void __launch_bounds__(128) mlp_precision_kernel(Geometry g, Tables tab, const StepConst* __restrict__ steps,
                                                            int kmax, HistorySoA h, long long begin, long long count,
                                                            double* __restrict__ dev_t, double* __restrict__ dev_v,
                                                            int* __restrict__ mismatched, int* __restrict__ ill_posed)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const long long id = begin + i;
    unsigned flags = 0;
    double xy_entry = h.xy_entry_angle[id], xy_exit = h.xy_exit_angle[id];
    MlpStart m = mlp_start(g, tab, h.x_entry[id], h.y_entry[id], h.z_entry[id], h.x_exit[id], h.y_exit[id],
                           h.z_exit[id], xy_entry, xy_exit, h.xz_entry_angle[id], h.xz_exit_angle[id], flags);
    const MlpHistoryF hf = mlp_history_f(m.h);
    const double s = g.mlp_u_step;
    double depth_2_go = m.depth_2_go, u_shifted = m.u_shifted, dt = 0.0, dv = 0.0;
    unsigned sigma_2_index = m.sigma_2_index;
    int bad = 0, ill = 0;
    for (int k = 1; m.tables_ok && depth_2_go > s && k <= kmax; k++) {
        double te, ve;
        float tm, vm;
        const StepConst& st = steps[k];
        mlp_point(m.h, st, tab.scattering_table, depth_2_go, sigma_2_index, te, ve);
        mlp_point_mixed(m.h, hf, st, tab.scattering_table, depth_2_go, sigma_2_index,
                        mixed_fp64_inverse(g, k, depth_2_go), tm, vm);
        u_shifted += s;
        // the reference's Sigma_2 determinant at this step (B.cu:9197)
        const MlpHistory& q = m.h;
        const double sigma_t2 = q.u_2_poly_3_12 - q.u_2_sq * st.p12 + q.two_u_2 * st.p23 - st.p34;
        const double sigma_t2_theta2 = q.u_2_poly_2_6 - q.u_2 * st.p12 + st.p23;
        const double sigma_theta2 = q.u_2_poly_1_2 - st.p12;
        // well posed: 1 - rho^2 of Sigma_2 above 1e-3 (its value for the scattering model is about 1/4)
        const double prod = sigma_t2 * sigma_theta2;
        if (sigma_theta2 > 0.0 && prod > 0.0 && prod - powf_square(sigma_t2_theta2) > 1e-3 * prod) {
            dt = fmax(dt, fabs((double)tm - te));
            dv = fmax(dv, fabs((double)vm - ve));
            if (mlp_voxel(g, m.h, u_shifted, te, ve) != mlp_voxel_mixed(g, hf, (float)u_shifted, tm, vm)) bad++;
        } else {
            ill++;
        }
        depth_2_go -= s;
        sigma_2_index -= g.sigma_index_step;
    }
    dev_t[i] = dt;
    dev_v[i] = dv;
    mismatched[i] = bad;
    ill_posed[i] = ill;
}

// ---- two-phase DROP iteration -------------------------------------------------------------
// Phase 1 (x-independent): every covered history's MLP voxel list is written to path storage.
// Phase 2 (per DROP block): gather x over the stored list, the DROP update, and the scatter.

// The path kernel's inputs in its processing order: dst[p] = src[perm[p]] (the ten geometry fields
// and the first voxel), with the path bound and the path-storage offset of the same history.
__global__ void gather_path_inputs_kernel(HistorySoA src, const int* __restrict__ perm, const int* __restrict__ bounds,
                                          const long long* __restrict__ offsets, long long n, HistorySoA dst,
                                          int* __restrict__ bounds_sorted, long long* __restrict__ offsets_sorted)
{
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const long long id = perm[p];
    dst.x_entry[p] = src.x_entry[id];
    dst.y_entry[p] = src.y_entry[id];
    dst.z_entry[p] = src.z_entry[id];
    dst.x_exit[p] = src.x_exit[id];
    dst.y_exit[p] = src.y_exit[id];
    dst.z_exit[p] = src.z_exit[id];
    dst.xy_entry_angle[p] = src.xy_entry_angle[id];
    dst.xz_entry_angle[p] = src.xz_entry_angle[id];
    dst.xy_exit_angle[p] = src.xy_exit_angle[id];
    dst.xz_exit_angle[p] = src.xz_exit_angle[id];
    dst.first_MLP_voxel[p] = src.first_MLP_voxel[id];
    bounds_sorted[p] = bounds[id];
    offsets_sorted[p] = offsets[id];
}

// Upper bound on the voxel-list length of each history (0 for histories the block launch does
// not cover): the loop runs at most u_2/MLP_U_STEP + 1 times and adds at most one entry per run.
// Rounded up to a multiple of kPathChunk entries so every history's slot starts on a 32-byte
// boundary and the path kernel writes whole sectors.
__global__ void path_bounds_kernel(Geometry g, Tables tab, HistorySoA h, long long n, long long block_size,
                                   int histories_per_block, int* __restrict__ bounds)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long long blk = i / block_size, pos = i - blk * block_size;
    long long hp = n - blk * block_size;
    if (hp > block_size) hp = block_size;
    const long long covered = histories_per_block > 0 ? (hp / histories_per_block) * histories_per_block : hp;
    int bound = 0;
    if (pos < covered) {
        const double u_2 = mlp_u_extent(g, tab, h.x_entry[i], h.y_entry[i], h.x_exit[i], h.y_exit[i], h.xy_entry_angle[i]);
        const double q = u_2 / g.mlp_u_step;
        bound = (q >= 0 && q < (double)(kPathCap - 3)) ? (int)q + 3 : kPathCap;
        bound = (bound + kPathChunk - 1) / kPathChunk * kPathChunk;
    }
    bounds[i] = bound;
}

// Launch shape of the path kernel, chosen by measurement on B200: one MLP point per loop trip
// (two points per trip need 108 registers and ran 21.7 vs 16.4 ms at 5M head histories), and the
// register budget of 7 resident 128-thread CTAs per SM (72 registers).  With the guarded fast
// points the kernel needs more live values than the reference-order points did: at 8 CTAs (64
// registers) it spilled 140 bytes and the 20M head iteration took 87.4 ms, at 7 CTAs it spills 68
// and takes 77.5 ms, against 80.4 ms for reference-order points at 8 CTAs.  With the per-history
// constants in shared memory (PCT_PHASE1_STASH, below) nothing spills at 7 CTAs and the iteration
// takes 74.1 ms (78.2 without; 74.8 at 8 CTAs, 20 bytes spilled).
#ifndef PCT_PHASE1_UNROLL
#define PCT_PHASE1_UNROLL 1
#endif
#ifndef PCT_PHASE1_MIN_BLOCKS
#define PCT_PHASE1_MIN_BLOCKS 7
#endif
// The mixed-precision path kernel keeps 8 CTAs (64 registers), as measured when it was tuned.
#ifndef PCT_PHASE1_MIXED_MIN_BLOCKS
#define PCT_PHASE1_MIXED_MIN_BLOCKS 8
#endif
// 0: each voxel-list entry is stored as it is found; 1: entries are staged in shared memory and
// written a 32-byte sector at a time.  Measured on B200 (10M head histories): staging cuts the
// kernel's DRAM traffic from ~1.9 KB to ~1.3 KB per history but costs 4% in time (34.3 vs
// 32.9 ms) -- the kernel is FP64-issue bound, not memory bound -- so 0 is the default.  (An L2
// evict-last policy on the direct stores was slower still, 34.4 ms.)  With the stash below and one
// shared-memory carve-out for the iteration's kernels (PCT_ITERATION_CARVEOUT), staging costs
// nothing: 74.0 vs 73.8 ms per 20M-history head iteration, 30.6 vs 31.5 ms per 10M-history
// small-block iteration, and the path kernel's DRAM writes fall to the lists' own bytes.  1 is the
// default.
#ifndef PCT_PHASE1_STAGE
#define PCT_PHASE1_STAGE 1
#endif
// 1: the per-history constants of the exact walk and its chord live in shared memory (16 doubles
// per thread, 16 KB per 128-thread CTA) and each is read where a loop trip uses it, instead of
// being held in registers across trips.
#ifndef PCT_PHASE1_STASH
#define PCT_PHASE1_STASH 1
#endif
// Entries per staged list write: 8 (one 32-byte sector) or 4 (16 bytes, a smaller staging buffer).
#ifndef PCT_STAGE_ENTRIES
#define PCT_STAGE_ENTRIES 8
#endif
// Staging applies to the exact mode's kernel only: the mixed-precision kernel keeps no shared memory,
// so that it and its block chain share the driver's carve-out.
// The voxel list goes to the history's slot in path storage (PCT_PHASE1_STAGE selects direct
// stores or shared-memory staging of whole 32-byte sectors, see above).
template <bool kMixed, int kThreads>
__device__ __forceinline__ void mlp_phase1_body(const Geometry& g, const Tables& tab, const StepConst* __restrict__ steps,
                                                int kmax, const HistorySoA& h, const int* __restrict__ perm,
                                                long long count, const long long* __restrict__ offsets,
                                                long long offset_base, const int* __restrict__ bounds,
                                                uint32_t* __restrict__ paths, int* __restrict__ path_n,
                                                double* __restrict__ chord, unsigned long long* counters)
{
    constexpr bool kStage = PCT_PHASE1_STAGE == 1 && !kMixed;
    // position i of the processing order: its inputs at i (gathered into this order), its
    // history id for the outputs
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const long long id = perm[i];
    const int cap = bounds[i];
    if (cap <= 0) {  // not covered by its DROP block: no path
        path_n[id] = 0;
        chord[id] = 0.0;
        return;
    }
    uint32_t* out = paths + (offsets[i] - offset_base);  // 32-byte aligned, cap a multiple of 8
    constexpr int kN = PCT_STAGE_ENTRIES;  // entries per flush: 8 (a 32-byte sector) or 4 (16 bytes)
    static_assert(kN == 4 || kN == 8, "staging flushes 4 or 8 entries");
    __shared__ uint32_t stage[kThreads * (kN + 1)];
    uint32_t* mine = stage + threadIdx.x * (kN + 1);  // odd stride in words: no bank conflicts
    auto flush = [&](int j0) {
        uint4* dst = reinterpret_cast<uint4*>(out + j0);
        dst[0] = make_uint4(mine[0], mine[1], mine[2], mine[3]);
        if (kN == 8) dst[1] = make_uint4(mine[4], mine[5], mine[6], mine[7]);
    };
    auto emit = [&](int j, uint32_t v) {
        if (j >= cap) return;
        if (!kStage) {
            out[j] = v;
            return;
        }
        mine[j & (kN - 1)] = v;
        if ((j & (kN - 1)) == kN - 1) flush(j - (kN - 1));
    };
    WalkResult r;
    if constexpr (kMixed)
        r = mlp_walk_mixed<false>(g, tab, steps, kmax, nullptr, __ldg(h.first_MLP_voxel + i), __ldg(h.x_entry + i),
                                  __ldg(h.y_entry + i), __ldg(h.z_entry + i), __ldg(h.x_exit + i),
                                  __ldg(h.y_exit + i), __ldg(h.z_exit + i), __ldg(h.xy_entry_angle + i),
                                  __ldg(h.xz_entry_angle + i), __ldg(h.xy_exit_angle + i),
                                  __ldg(h.xz_exit_angle + i), emit);
    else {
        __shared__ double stash[PCT_PHASE1_STASH ? (kHistoryFields + PCT_STASH_CHORD) * kThreads : 1];
        r = mlp_walk_exact<false, PCT_PHASE1_UNROLL>(
            g, tab, steps, kmax, nullptr, __ldg(h.first_MLP_voxel + i), __ldg(h.x_entry + i), __ldg(h.y_entry + i),
            __ldg(h.z_entry + i), __ldg(h.x_exit + i), __ldg(h.y_exit + i), __ldg(h.z_exit + i),
            __ldg(h.xy_entry_angle + i), __ldg(h.xz_entry_angle + i), __ldg(h.xy_exit_angle + i),
            __ldg(h.xz_exit_angle + i), emit, (uint32_t)__cvta_generic_to_shared(stash + threadIdx.x),
            PCT_PHASE1_STASH ? kThreads * (uint32_t)sizeof(double) : 0u);
    }
    unsigned flags = r.flags;
    int n = r.n;
    if (n > cap) {  // cannot happen: cap bounds the loop count
        flags |= kFlagPathOverflow;
        n = cap;
    }
    if (kStage && (n & (kN - 1))) flush(n & ~(kN - 1));  // the last partial flush, padded (cap is a multiple of 8)
    if (flags) count_flags(flags, counters);
    path_n[id] = n;
    chord[id] = r.chord;
}

// kThreads histories per CTA (PATH_CTA_THREADS), with the same resident threads per SM, hence the
// same register budget (72 for the exact kernel, 64 for the mixed one), at every size.
template <int kThreads>
__global__ void __launch_bounds__(kThreads, PCT_PHASE1_MIN_BLOCKS * 128 / kThreads) mlp_phase1_exact_kernel(
    Geometry g, Tables tab, const StepConst* __restrict__ steps, int kmax, HistorySoA h, const int* __restrict__ perm,
    long long count, const long long* __restrict__ offsets, long long offset_base, const int* __restrict__ bounds,
    uint32_t* __restrict__ paths, int* __restrict__ path_n, double* __restrict__ chord, unsigned long long* counters)
{
    mlp_phase1_body<false, kThreads>(g, tab, steps, kmax, h, perm, count, offsets, offset_base, bounds, paths, path_n,
                                     chord, counters);
}

template <int kThreads>
__global__ void __launch_bounds__(kThreads, PCT_PHASE1_MIXED_MIN_BLOCKS * 128 / kThreads) mlp_phase1_mixed_kernel(
    Geometry g, Tables tab, const StepConst* __restrict__ steps, int kmax, HistorySoA h, const int* __restrict__ perm,
    long long count, const long long* __restrict__ offsets, long long offset_base, const int* __restrict__ bounds,
    uint32_t* __restrict__ paths, int* __restrict__ path_n, double* __restrict__ chord, unsigned long long* counters)
{
    mlp_phase1_body<true, kThreads>(g, tab, steps, kmax, h, perm, count, offsets, offset_base, bounds, paths, path_n,
                                    chord, counters);
}

// One warp per history.  Lane l holds entries l, l+32, ..., l+224 of the stored voxel list in
// registers: they are loaded once (eight independent loads in flight per lane), gathered for
// the sum of x, and reused for the scatter; longer lists stream their tail from memory twice.
//
// kAlgo selects the update: PCT_DROP (DROP_block_update_GPU B.cu:9522), PCT_ROBUSTA (a per-voxel
// perturbation Psi_j = (1 - x_j) ETA PSI_SIGN of the denominator, DROP_blocks_robust1 O.cu:7537)
// or PCT_ROBUSTB (the DROP update plus ||a||^2 per voxel into normA, DROP_blocks_robust2
// O.cu:7554).
//
// kMixed (PRECISION MIXED = 1 or MIXED_COMPENSATED = 2, PCT_DROP) runs the DROP arithmetic in FP32
// with compensation: each lane sums its entries of x with TwoSum (a float sum and its exact
// rounding error), the warp reduces the (sum, error) pairs with TwoSum, the residual WEPL - L*sum
// is formed from the exact product error (an FMA), and the update is a float expression of the
// float chord.  The scatter then adds (update, 1) to the float accumulator as the exact mode does.
// With 2 it instead returns each accumulator's old value, recomputes the float addition locally
// and adds its exact rounding error into a second per-voxel float array (comp), so a block's
// per-voxel partial sum is held as hi + lo and the image update applies (hi + lo) / S; that costs
// a returning atomic and a second reduction per entry.
//
// kSCurve (S_CURVE_ON, exact PCT_DROP only) scales the update of entry j by the S-curve table's
// s(k), k = s_curve_index(j, n), in the reference's order s * L * q * lambda (B.cu:9530-9531).
// Its launch bound asks for 6 CTAs per SM, which holds it to 40 registers without spills (48
// unbounded): the kernel is bound by the latency of its L2 reductions, so it keeps the warps per
// SM of the plain instantiations (39 registers, 6 CTAs).  A minimum of 0 leaves the others as
// they are (a minimum of 1 moves them to 48 registers).
constexpr int kRegEntries = 8;

// TwoSum (Knuth): s = RN(a + b) and the exact error e with a + b = s + e, six float operations.
__device__ __forceinline__ float two_sum(float a, float b, float& e)
{
    const float s = __fadd_rn(a, b);
    const float bp = __fsub_rn(s, a);
    e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bp)), __fsub_rn(b, bp));
    return s;
}

template <int kAlgo, bool kDet, int kMixed, bool kSCurve = false>
__global__ void __launch_bounds__(256, kSCurve ? 6 : 0) drop_phase2_kernel(Geometry g, const float* __restrict__ x, float2* __restrict__ acc,
                                                          float* __restrict__ normA, FixedAcc fx,
                                                          const float* __restrict__ WEPL,
                                                          const long long* __restrict__ offsets, long long offset_base,
                                                          const uint32_t* __restrict__ paths, const int* __restrict__ path_n,
                                                          const double* __restrict__ chord, long long begin, long long count)
{
    allow_dependent_launch();
    const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= count) return;
    // The voxel lists were written by the path kernel, which completed before the first block
    // kernel of this run started (a full dependency), so they are read before the wait.
    const long long id = begin + w;
    const int n = path_n[id];
    const uint32_t* p = paths + (offsets[id] - offset_base);
    const uint32_t npad = (uint32_t)g.padded_voxels;
    uint32_t v[kRegEntries];
#pragma unroll
    for (int m = 0; m < kRegEntries; m++) {
        const int j = lane + 32 * m;
        v[m] = j < n ? __ldg(p + j) : 0xffffffffu;
    }
    grid_dependency_wait();  // the previous block's image update has landed
    if constexpr (kMixed != 0 && kAlgo == PCT_DROP) {
        float hi = 0.0f, lo = 0.0f, e;
#pragma unroll
        for (int m = 0; m < kRegEntries; m++)
            if (v[m] < npad) {
                hi = two_sum(hi, __ldg(x + v[m]), e);
                lo = __fadd_rn(lo, e);
            }
        for (int j = lane + 32 * kRegEntries; j < n; j += 32) {
            const uint32_t u = __ldg(p + j);
            if (u < npad) {
                hi = two_sum(hi, __ldg(x + u), e);
                lo = __fadd_rn(lo, e);
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const float h2 = __shfl_xor_sync(0xffffffffu, hi, o), l2 = __shfl_xor_sync(0xffffffffu, lo, o);
            hi = two_sum(hi, h2, e);
            lo = __fadd_rn(__fadd_rn(lo, l2), e);
        }
        if (n < g.min_mlp_length) return;
        // residual = WEPL - L * (hi + lo) with the product's rounding error recovered by an FMA
        const float L = (float)chord[id];
        const float prod = __fmul_rn(L, hi);
        const float prod_err = __fmaf_rn(L, hi, -prod);
        const float residual =
            __fsub_rn(__fsub_rn(__fsub_rn(__ldg(WEPL + id), prod), prod_err), __fmul_rn(L, lo));
        const float a_i_dot_a_i = __fmul_rn(__fmul_rn(L, L), (float)n);
        const float upd = __fmul_rn(__fmul_rn(L, __fdiv_rn(residual, a_i_dot_a_i)), (float)g.lambda);
        auto put = [&](uint32_t u) {
            if (kDet) {
                atomicAdd(fx.sum + u, (unsigned long long)__double2ll_rn((double)upd * kFixedScale));
                atomicAdd(fx.cnt + u, 1u);
            } else if (kMixed == 2) {
                const float2 old = atomicAdd(acc + u, make_float2(upd, 1.0f));
                float err;
                two_sum(old.x, upd, err);
                if (err != 0.0f) atomicAdd(normA + u, err);
            } else {
                atomicAdd(acc + u, make_float2(upd, 1.0f));
            }
        };
#pragma unroll
        for (int m = 0; m < kRegEntries; m++)
            if (v[m] < npad) put(v[m]);
        for (int j = lane + 32 * kRegEntries; j < n; j += 32) {
            const uint32_t u = __ldg(p + j);
            if (u < npad) put(u);
        }
        return;
    }
    double sum = 0.0;
#pragma unroll
    for (int m = 0; m < kRegEntries; m++)
        if (v[m] < npad) sum += (double)__ldg(x + v[m]);
    for (int j = lane + 32 * kRegEntries; j < n; j += 32) {
        const uint32_t u = __ldg(p + j);
        if (u < npad) sum += (double)__ldg(x + u);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if (n < g.min_mlp_length) return;
    const double L = chord[id];
    // one path entry's contribution: a float update and a count
    auto put = [&](uint32_t u, float upd) {
        if (kDet) {
            atomicAdd(fx.sum + u, (unsigned long long)__double2ll_rn((double)upd * kFixedScale));
            atomicAdd(fx.cnt + u, 1u);
        } else {
            atomicAdd(acc + u, make_float2(upd, 1.0f));
        }
    };
    if (kAlgo == PCT_DROP && kSCurve) {
        const double a_i_dot_a_i = powf_square(L) * n;
        const double a_i_dot_x_k = sum * L;
        const double q = ((double)__ldg(WEPL + id) - a_i_dot_x_k) / a_i_dot_a_i;
        auto scaled = [&](int j) {
            const double s = (double)__ldg(g.s_curve + s_curve_index(g, j, n));
            return (float)(((s * L) * q) * g.lambda);
        };
#pragma unroll
        for (int m = 0; m < kRegEntries; m++)
            if (v[m] < npad) put(v[m], scaled(lane + 32 * m));
        for (int j = lane + 32 * kRegEntries; j < n; j += 32) {
            const uint32_t u = __ldg(p + j);
            if (u < npad) put(u, scaled(j));
        }
    } else if (kAlgo == PCT_DROP) {
        const double a_i_dot_a_i = powf_square(L) * n;
        const double a_i_dot_x_k = sum * L;
        const float upd = (float)(L * (((double)__ldg(WEPL + id) - a_i_dot_x_k) / a_i_dot_a_i) * g.lambda);
#pragma unroll
        for (int m = 0; m < kRegEntries; m++)
            if (v[m] < npad) put(v[m], upd);
        for (int j = lane + 32 * kRegEntries; j < n; j += 32) {
            const uint32_t u = __ldg(p + j);
            if (u < npad) put(u, upd);
        }
    } else if (kAlgo == PCT_ROBUSTA) {
        // update_j = LAMBDA * residual / (<a,a> + Psi_j), Psi_j = ((1 - x_j) * ETA) * PSI_SIGN
        const double a_i_dot_a_i = L * L * n;
        const double residual = (double)__ldg(WEPL + id) - sum * L;
        auto add = [&](uint32_t u) {
            const double psi = ((1.0 - (double)__ldg(x + u)) * g.eta) * g.psi_sign;
            put(u, (float)(g.lambda * (residual / (a_i_dot_a_i + psi))));
        };
#pragma unroll
        for (int m = 0; m < kRegEntries; m++)
            if (v[m] < npad) add(v[m]);
        for (int j = lane + 32 * kRegEntries; j < n; j += 32) {
            const uint32_t u = __ldg(p + j);
            if (u < npad) add(u);
        }
    } else {  // PCT_ROBUSTB: update = L * LAMBDA * residual / <a,a>; normA_j += L^2 (float atomics)
        const double a_i_dot_a_i = L * L * n;
        const float upd = (float)(L * g.lambda * (((double)__ldg(WEPL + id) - sum * L) / a_i_dot_a_i));
        const float2 add = make_float2(upd, 1.0f);
        const float l2 = (float)(L * L);
#pragma unroll
        for (int m = 0; m < kRegEntries; m++)
            if (v[m] < npad) {
                atomicAdd(acc + v[m], add);
                atomicAdd(normA + v[m], l2);
            }
        for (int j = lane + 32 * kRegEntries; j < n; j += 32) {
            const uint32_t u = __ldg(p + j);
            if (u < npad) {
                atomicAdd(acc + u, add);
                atomicAdd(normA + u, l2);
            }
        }
    }
}

// Per-step table (see pct_tables.h): the u_1 polynomials and Sigma_1I of loop iteration k,
// evaluated on the device like the reference's loop does (B.cu:9180-9195, powf on the device).
__global__ void build_step_table_kernel(Tables tab, unsigned sstep, unsigned pstep, int kmax, StepConst* steps)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k > kmax) return;
    StepConst e{};
    if (k >= 1) {
        const unsigned pi1 = (unsigned)k * pstep, si1 = (unsigned)k * sstep;
        const double p12 = tab.poly_1_2[pi1];
        const double sigma_t1 = tab.poly_3_12[pi1], sigma_t1_theta1 = tab.poly_2_6[pi1], sigma_theta1 = p12;
        const double det1 = tab.scattering_table[si1] * (sigma_t1 * sigma_theta1 - powf_square(sigma_t1_theta1));
        e.p12 = p12;
        e.p23 = tab.poly_2_3[pi1];
        e.p34 = tab.poly_3_4[pi1];
        e.s1i0 = sigma_theta1 / det1;
        e.s1i1 = sigma_t1_theta1 / det1;
        e.s1i2 = sigma_t1 / det1;
        e.s1i0f = (float)e.s1i0;
        e.s1i1f = (float)e.s1i1;
        e.s1i2f = (float)e.s1i2;
    }
    steps[k] = e;
}

}  // namespace

cudaError_t launch_build_step_table(const Tables& tab, unsigned sstep, unsigned pstep, int kmax, StepConst* steps,
                                    cudaStream_t stream)
{
    const int threads = 128;
    build_step_table_kernel<<<(kmax + threads) / threads, threads, 0, stream>>>(tab, sstep, pstep, kmax, steps);
    return cudaGetLastError();
}

cudaError_t launch_path_bounds(const Geometry& g, const Tables& tab, const HistorySoA& h, long long n,
                               long long block_size, int histories_per_block, int* bounds, cudaStream_t stream)
{
    if (n <= 0) return cudaSuccess;
    const int threads = 256;
    path_bounds_kernel<<<(unsigned)((n + threads - 1) / threads), threads, 0, stream>>>(g, tab, h, n, block_size,
                                                                                        histories_per_block, bounds);
    return cudaGetLastError();
}

cudaError_t launch_gather_path_inputs(const HistorySoA& src, const int* perm, const int* bounds,
                                      const long long* offsets, long long n, const HistorySoA& dst, int* bounds_sorted,
                                      long long* offsets_sorted, cudaStream_t stream)
{
    if (n <= 0) return cudaSuccess;
    const int threads = 256;
    gather_path_inputs_kernel<<<(unsigned)((n + threads - 1) / threads), threads, 0, stream>>>(
        src, perm, bounds, offsets, n, dst, bounds_sorted, offsets_sorted);
    return cudaGetLastError();
}

cudaError_t launch_mlp_phase1_exact(const Geometry& g, const Tables& tab, const StepConst* steps, int kmax,
                                    const HistorySoA& h, const int* perm, long long count, const long long* offsets,
                                    long long offset_base, const int* bounds, uint32_t* paths, int* path_n,
                                    double* chord, unsigned long long* counters, cudaStream_t stream)
{
    if (count <= 0) return cudaSuccess;
#define PCT_PHASE1(T)                                                                                             \
    do {                                                                                                          \
        const unsigned blocks = (unsigned)((count + (T) - 1) / (T));                                              \
        if (g.mixed_precision)                                                                                    \
            mlp_phase1_mixed_kernel<T><<<blocks, T, 0, stream>>>(g, tab, steps, kmax, h, perm, count, offsets,    \
                                                                 offset_base, bounds, paths, path_n, chord, counters); \
        else                                                                                                      \
            mlp_phase1_exact_kernel<T><<<blocks, T, 0, stream>>>(g, tab, steps, kmax, h, perm, count, offsets,    \
                                                                 offset_base, bounds, paths, path_n, chord, counters); \
    } while (0)
    if (g.path_cta_threads == 64) PCT_PHASE1(64);
    else if (g.path_cta_threads == 256) PCT_PHASE1(256);
    else PCT_PHASE1(128);
#undef PCT_PHASE1
    return cudaGetLastError();
}

cudaError_t launch_drop_phase2(const Geometry& g, const float* x, float2* acc, float* normA, const FixedAcc& fx,
                               const float* WEPL, const long long* offsets, long long offset_base,
                               const uint32_t* paths, const int* path_n, const double* chord, long long begin,
                               long long count, cudaStream_t stream, bool pdl)
{
    if (count <= 0) return cudaSuccess;
    const int threads = 256;
    const unsigned blocks = (unsigned)((count * 32 + threads - 1) / threads);
    cudaError_t e = cudaSuccess;
#define PCT_PHASE2(ALGO, DET, MIXED, SC)                                                                    \
    e = launch_kernel(pdl, drop_phase2_kernel<ALGO, DET, MIXED, SC>, blocks, threads, stream, g, x, acc, normA, \
                      fx, WEPL, offsets, offset_base, paths, path_n, chord, begin, count)
    if (g.projection_algorithm == PCT_ROBUSTA) {
        if (g.deterministic) PCT_PHASE2(PCT_ROBUSTA, true, 0, false);
        else PCT_PHASE2(PCT_ROBUSTA, false, 0, false);
    } else if (g.projection_algorithm == PCT_ROBUSTB) {
        PCT_PHASE2(PCT_ROBUSTB, false, 0, false);
    } else if (g.mixed_precision) {
        if (g.deterministic) PCT_PHASE2(PCT_DROP, true, 1, false);  // fixed-point sums need no compensation
        else if (g.compensated) PCT_PHASE2(PCT_DROP, false, 2, false);
        else PCT_PHASE2(PCT_DROP, false, 1, false);
    } else if (g.s_curve) {
        if (g.deterministic) PCT_PHASE2(PCT_DROP, true, 0, true);
        else PCT_PHASE2(PCT_DROP, false, 0, true);
    } else {
        if (g.deterministic) PCT_PHASE2(PCT_DROP, true, 0, false);
        else PCT_PHASE2(PCT_DROP, false, 0, false);
    }
#undef PCT_PHASE2
    return e;
}

// The carve-out, in percent of the largest shared memory an SM offers (228 KB on B200).  58% asks for
// a little over 132 KB, so the driver takes the 164 KB configuration: 7 path-kernel CTAs of 20.5 KB
// (stash and list staging) plus the per-CTA reserve fit, and registers, not shared memory, limit them.
// 57% gives the 132 KB configuration, 6 path CTAs and room in the register file for one DROP-block
// CTA beside them; measured 74.7 vs 72.9 ms per 20M-history head iteration, so 58% stays.  A
// negative value leaves each kernel to the driver's choice.  Measured on B200 (exact
// mode, ms per iteration): small configuration at 10M histories (blocks of 3200, 196 path chunks)
// 31.5 with it, 66.0 without; 2M histories 6.33 vs 13.25; head 20M 73.6 vs 73.9.
#ifndef PCT_ITERATION_CARVEOUT
#define PCT_ITERATION_CARVEOUT 58
#endif

cudaError_t set_iteration_carveout()
{
    const int percent = PCT_ITERATION_CARVEOUT;
    if (percent < 0) return cudaSuccess;
    // the exact mode's kernels only: the mixed-precision path kernel keeps no shared memory, and it
    // and its block kernels run best with the driver's choice (its L1 holds the table gathers)
    const void* kernels[] = {
        (const void*)mlp_phase1_exact_kernel<64>, (const void*)mlp_phase1_exact_kernel<128>,
        (const void*)mlp_phase1_exact_kernel<256>,
        (const void*)drop_phase2_kernel<PCT_DROP, false, 0>, (const void*)drop_phase2_kernel<PCT_DROP, true, 0>,
        (const void*)drop_phase2_kernel<PCT_ROBUSTA, false, 0>, (const void*)drop_phase2_kernel<PCT_ROBUSTA, true, 0>,
        (const void*)drop_phase2_kernel<PCT_ROBUSTB, false, 0>,
        (const void*)drop_phase2_kernel<PCT_DROP, false, 0, true>, (const void*)drop_phase2_kernel<PCT_DROP, true, 0, true>};
    for (const void* k : kernels) {
        const cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, percent);
        if (e != cudaSuccess) return e;
    }
    return set_image_update_carveout(percent);
}

cudaError_t launch_drop_block_exact(const Geometry& g, const Tables& tab, const StepConst* steps, int kmax,
                                    const float* x, float2* acc, const HistorySoA& h, long long begin,
                                    long long count, unsigned long long* counters, cudaStream_t stream)
{
    if (count <= 0) return cudaSuccess;
    const int threads = 128;
    const long long blocks = (count + threads - 1) / threads;
    drop_block_exact_kernel<<<(unsigned)blocks, threads, 0, stream>>>(g, tab, steps, kmax, x, acc, h, begin, count,
                                                                      counters);
    return cudaGetLastError();
}

cudaError_t launch_mlp_paths_exact(const Geometry& g, const Tables& tab, const StepConst* steps, int kmax,
                                   const float* x, const HistorySoA& h, long long begin, long long count, int stride,
                                   uint32_t* counts, uint32_t* voxels, double* chord, double* a_dot_x,
                                   unsigned long long* counters, cudaStream_t stream)
{
    if (count <= 0) return cudaSuccess;
    const int threads = 128;
    const long long blocks = (count + threads - 1) / threads;
    if (g.mixed_precision)
        mlp_paths_kernel<true><<<(unsigned)blocks, threads, 0, stream>>>(g, tab, steps, kmax, x, h, begin, count,
                                                                         stride, counts, voxels, chord, a_dot_x,
                                                                         counters);
    else
        mlp_paths_kernel<false><<<(unsigned)blocks, threads, 0, stream>>>(g, tab, steps, kmax, x, h, begin, count,
                                                                          stride, counts, voxels, chord, a_dot_x,
                                                                          counters);
    return cudaGetLastError();
}

cudaError_t launch_mlp_steps(const Geometry& g, const Tables& tab, int kmax, const HistorySoA& h, long long begin,
                             long long count, int* steps, cudaStream_t stream)
{
    if (count <= 0) return cudaSuccess;
    const int threads = 128;
    const long long blocks = (count + threads - 1) / threads;
    mlp_steps_kernel<<<(unsigned)blocks, threads, 0, stream>>>(g, tab, kmax, h, begin, count, steps);
    return cudaGetLastError();
}

cudaError_t launch_mlp_precision(const Geometry& g, const Tables& tab, const StepConst* steps, int kmax,
                                 const HistorySoA& h, long long begin, long long count, double* dev_t, double* dev_v,
                                 int* mismatched, int* ill_posed, cudaStream_t stream)
{
    if (count <= 0) return cudaSuccess;
    const int threads = 128;
    mlp_precision_kernel<<<(unsigned)((count + threads - 1) / threads), threads, 0, stream>>>(
        g, tab, steps, kmax, h, begin, count, dev_t, dev_v, mismatched, ill_posed);
    return cudaGetLastError();
}

}  // namespace pct
