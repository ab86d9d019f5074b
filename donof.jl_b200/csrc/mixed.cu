// Mixed-precision form of the RI hot path (tensor-core TF32x3 contractions
// with FP32 accumulation).  FP32 copy of b kept next to the FP64 one.
#include "kernels.cuh"

namespace donof {

namespace {

__global__ void to_f32_kernel(const double* __restrict__ in, long long count, float* __restrict__ out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = (float)in[i];
}

}  // namespace

int convert_b_f32(donof_job* job) {
    donof_ctx* ctx = job->ctx;
    const long long count = (long long)job->nbf * job->nbf * job->naux;
    void* d = nullptr;
    DONOF_CUDA(ctx, cudaMalloc(&d, sizeof(float) * (size_t)count));
    to_f32_kernel<<<8 * ctx->sm_count, 256, 0, ctx->stream>>>(job->b, count, static_cast<float*>(d)); count_launch();
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        cudaFree(d);
        set_error(ctx, "FP32 conversion of b: %s", cudaGetErrorString(e));
        return DONOF_ERR_CUDA;
    }
    job->b32 = static_cast<const float*>(d);
    job->own_b32 = true;
    return DONOF_OK;
}

int transforms_mixed(donof_job* job, cudaStream_t, const double*, int) {
    set_error(job->ctx, "mixed-precision transform not available in this build");
    return DONOF_ERR_STATE;
}

int lagrange2_mixed(donof_job* job, cudaStream_t, const double*, const double*, const double*,
                    const double*, const double*, int, int, int, double*, double*, double*) {
    set_error(job->ctx, "mixed-precision Lagrangian not available in this build");
    return DONOF_ERR_STATE;
}

int jkh_mo_mixed(donof_job* job, cudaStream_t, const double*, const double*, int, double*, double*,
                 double*) {
    set_error(job->ctx, "mixed-precision JKH_MO not available in this build");
    return DONOF_ERR_STATE;
}

}  // namespace donof
