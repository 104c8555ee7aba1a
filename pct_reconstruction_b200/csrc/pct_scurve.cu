// pct_scurve.cu -- S-curve attenuation table of the DROP update (B.cu:10606-10649).
//
// With S_CURVE_ON the reference scales the update that entry j of an n-entry MLP path adds by
// s_curve_scale_GPU(j, n) (DROP_block_update_GPU, B.cu:9529-9534): the index is k = min(j, n-1-j)
// with DUAL_SIDED_S_CURVE, else k = j, and s(k) is one of five curves of the unsigned k.  s depends
// on k alone and k < PCT_MLP_PATH_CAP, so the context evaluates it once per k into a float table
// that the DROP kernels read per entry.  Each curve below is the reference's expression with the
// same CUDA math function and the same argument types; this file is compiled with nvcc's default
// contraction setting, as the reference is, so the table holds the values the reference computes
// inline.
#include "pct_context.h"
#include "pct_kernels.h"

namespace pct {

namespace {

__global__ void s_curve_table_kernel(int curve, double steepness, int mid_shift, int count, float* out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const unsigned k = (unsigned)i;      // the reference's UINT index
    const double pi = 4 * atan(1.0);     // PI (B.h:833)
    float s;
    switch (curve) {
    case PCT_TANH:  // tanh_GPU (B.cu:10618): the float overload of tanh
        s = tanhf((float)k);
        break;
    case PCT_ATAN:  // atan_GPU (B.cu:10614): TWO_OVER_PI * atan(PI_OVER_TWO * k)
        s = (float)((2 / pi) * atan((pi / 2) * k));
        break;
    case PCT_ERF:  // erf_GPU (B.cu:10610): erf(ROOT_PI_OVER_TWO * k)
        s = (float)erf((sqrt(pi) / 2) * k);
        break;
    case PCT_LIN_OVER_ROOT:  // linear_over_root_GPU (B.cu:10622): k / sqrt(1 + powf(k, 2.0)), all float
        s = (float)k / sqrtf(1.0f + powf((float)k, 2.0f));
        break;
    default:  // sigmoid_GPU (B.cu:10606): 1 / (1 + exp(-STEEPNESS * (k - MID_SHIFT))), k - MID_SHIFT unsigned
        s = (float)(1 / (1 + exp(-steepness * (double)(k - (unsigned)mid_shift))));
        break;
    }
    out[i] = s;
}

}  // namespace

cudaError_t launch_s_curve_table(const pct_config& c, float* out, cudaStream_t stream)
{
    const int count = kSCurveEntries;
    s_curve_table_kernel<<<(count + 127) / 128, 128, 0, stream>>>(c.S_CURVE, c.SIGMOID_STEEPNESS, c.SIGMOID_MID_SHIFT,
                                                                  count, out);
    return cudaGetLastError();
}

}  // namespace pct

extern "C" pct_status pct_get_s_curve(pct_ctx* ctx, float* scales, int32_t count)
{
    if (!ctx || !scales || count < 0 || count > pct::kSCurveEntries) return PCT_ERR_ARG;
    if (!ctx->geo.s_curve) {
        ctx->last_error = "pct_get_s_curve: the configuration has S_CURVE_ON 0";
        return PCT_ERR_STATE;
    }
    if (count == 0) return PCT_OK;
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(scales, ctx->geo.s_curve, sizeof(float) * (size_t)count, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        ctx->last_error = "pct_get_s_curve: " + pct::cuda_error_string(e);
        return PCT_ERR_CUDA;
    }
    return PCT_OK;
}
