// pct_batch.cu -- many scans' DROP iterations as one graph launch.
//
// The reference reconstructs one scan per program run (its grid is compile-time).  A batch holds
// the contexts of several scans -- each with its own grid, histories, image and path storage on the
// same device -- and runs one DROP iteration of all of them as a single CUDA graph: every context's
// captured iteration becomes a child graph on its own branch, so the scans' path kernels and DROP
// block chains run concurrently and small scans fill the GPU together.  Each scan's result is what
// its own pct_drop_full_tx_iteration would give (bit for bit with SCATTER_MODE DETERMINISTIC; up to
// the float-atomic order otherwise).  The batch graph is rebuilt when a context's captured
// iteration changes (new histories, a new path-storage layout).
#include <vector>

#include "pct_context.h"

struct pct_batch {
    int device = 0;
    std::vector<pct_ctx*> ctxs;
    std::vector<long long> versions;  // graph_version of each context when the batch graph was built
    cudaStream_t stream = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::string last_error;
};

namespace {

pct_status batch_fail(pct_batch* b, pct_status s, const std::string& what, cudaError_t e = cudaSuccess)
{
    b->last_error = what;
    if (e != cudaSuccess) b->last_error += " -> " + pct::cuda_error_string(e);
    return s;
}

pct_status build(pct_batch* b)
{
    bool fresh = b->exec != nullptr;
    for (size_t i = 0; fresh && i < b->ctxs.size(); i++) fresh = b->versions[i] == b->ctxs[i]->graph_version;
    if (fresh) return PCT_OK;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
    cudaGraph_t parent = nullptr;
    cudaError_t e = cudaGraphCreate(&parent, 0);
    if (e != cudaSuccess) return batch_fail(b, PCT_ERR_CUDA, "cudaGraphCreate", e);
    for (size_t i = 0; i < b->ctxs.size(); i++) {
        cudaGraph_t child = nullptr;
        long long launches = 0;
        pct_status st = pct::iteration_graph(b->ctxs[i], &child, &launches);
        if (st != PCT_OK) {
            cudaGraphDestroy(parent);
            return batch_fail(b, st, "scan " + std::to_string(i) + ": " + b->ctxs[i]->last_error);
        }
        cudaGraphNode_t node;
        e = cudaGraphAddChildGraphNode(&node, parent, nullptr, 0, child);  // no dependencies: parallel
        if (e != cudaSuccess) {
            cudaGraphDestroy(parent);
            return batch_fail(b, PCT_ERR_CUDA, "cudaGraphAddChildGraphNode", e);
        }
        b->versions[i] = b->ctxs[i]->graph_version;
    }
    e = cudaGraphInstantiateWithFlags(&b->exec, parent, cudaGraphInstantiateFlagUseNodePriority);
    cudaGraphDestroy(parent);
    if (e != cudaSuccess) {
        b->exec = nullptr;
        return batch_fail(b, PCT_ERR_CUDA, "cudaGraphInstantiate(batch)", e);
    }
    return PCT_OK;
}

}  // namespace

extern "C" pct_status pct_batch_create(pct_ctx* const* ctxs, int n, pct_batch** out)
{
    if (!ctxs || n <= 0 || !out) return PCT_ERR_ARG;
    *out = nullptr;
    for (int i = 0; i < n; i++) {
        if (!ctxs[i] || ctxs[i]->device != ctxs[0]->device) return PCT_ERR_ARG;
        for (int j = 0; j < i; j++)
            if (ctxs[j] == ctxs[i]) return PCT_ERR_ARG;  // a context appears once
    }
    pct_batch* b = new pct_batch();
    b->device = ctxs[0]->device;
    b->ctxs.assign(ctxs, ctxs + n);
    b->versions.assign(n, -1);
    cudaSetDevice(b->device);
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete b;
        return PCT_ERR_CUDA;
    }
    *out = b;
    return PCT_OK;
}

extern "C" void pct_batch_destroy(pct_batch* b)
{
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

extern "C" pct_status pct_batch_drop_iteration(pct_batch* b, int iteration)
{
    (void)iteration;
    if (!b) return PCT_ERR_ARG;
    cudaSetDevice(b->device);
    // work a context queued on its own stream (images, histories) comes first
    for (pct_ctx* c : b->ctxs) {
        cudaError_t e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) return batch_fail(b, PCT_ERR_CUDA, "context stream", e);
    }
    pct_status st = build(b);
    if (st != PCT_OK) return st;
    cudaError_t e = cudaGraphLaunch(b->exec, b->stream);
    if (e != cudaSuccess) return batch_fail(b, PCT_ERR_CUDA, "cudaGraphLaunch(batch)", e);
    for (pct_ctx* c : b->ctxs) pct::iteration_ran(c);
    return PCT_OK;
}

extern "C" pct_status pct_batch_synchronize(pct_batch* b)
{
    if (!b) return PCT_ERR_ARG;
    cudaSetDevice(b->device);
    cudaError_t e = cudaStreamSynchronize(b->stream);
    return e == cudaSuccess ? PCT_OK : batch_fail(b, PCT_ERR_CUDA, "batch stream", e);
}

extern "C" const char* pct_batch_last_error(const pct_batch* b) { return b ? b->last_error.c_str() : ""; }

extern "C" void* pct_batch_stream(pct_batch* b) { return b ? static_cast<void*>(b->stream) : nullptr; }
