// The RI tensor on the device from the two- and three-centre integrals:
//   b[m, n, l] = sum_k I[m, n, k] G^{-1/2}[k, l]
// (Iaux, src/integrals.jl:68-91; GPU form Iaux_gpu, ext/DoNOFGPUExt.jl:9-33):
// eigen-decomposition of Symmetric(G) (upper triangle), inverse square roots of
// the eigenvalues with negative ones set to zero, G^{-1/2} = V diag(s) V^T, and
// the contraction as one GEMM of I seen as an (nbf^2 x naux) column-major
// matrix, whose product is b in the layout of the rest of the library.
//
// The symmetric eigensolver is the library's own parallel Jacobi kernel
// (eigh.cu); the two products run on the library's FP64 tensor-core GEMM.
#include <math.h>

#include "kernels.cuh"

namespace donof {

namespace {

// Vs[i + n j] = V[i + n j] s_j,  VT[j + n i] = V[i + n j];  s_j = 1/sqrt(w_j), 0 for w_j < 0
__global__ void gmsqrt_factors_kernel(const double* __restrict__ V, const double* __restrict__ w, int n,
                                      double* __restrict__ Vs, double* __restrict__ VT) {
    const long long total = (long long)n * n;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(idx % n), j = (int)(idx / n);
        const double s = (w[j] < 0.0) ? 0.0 : 1.0 / sqrt(w[j]);
        const double v = V[idx];
        Vs[idx] = v * s;
        VT[j + (long long)n * i] = v;
    }
}

struct DeviceScratch {
    void* p[16] = {};
    int n = 0;
    donof_ctx* ctx;
    explicit DeviceScratch(donof_ctx* c) : ctx(c) {}
    template <class T>
    int alloc(T** out, size_t count) {
        if (n >= 16) {
            set_error(ctx, "Iaux scratch: too many buffers");
            return DONOF_ERR_STATE;
        }
        void* d = nullptr;
        DONOF_CHECK(dev_alloc(ctx, &d, sizeof(T) * count));
        p[n++] = d;
        *out = static_cast<T*>(d);
        return DONOF_OK;
    }
    ~DeviceScratch() {  // stream-ordered after the work that used the scratch
        for (int i = 0; i < n; ++i) dev_free(ctx, p[i]);
    }
};

}  // namespace

int iaux_f64(donof_ctx* ctx, cudaStream_t st, const double* G_host, const double* I_host, int nbf, int naux,
             double* b, DevBuf* part) {
    const size_t nn = (size_t)nbf * nbf, na2 = (size_t)naux * naux;
    DeviceScratch s(ctx);
    double *dI = nullptr, *dG = nullptr, *dw = nullptr, *dVs = nullptr, *dVT = nullptr, *dGm = nullptr,
           *dA = nullptr, *dV = nullptr;
    unsigned char* escr = nullptr;
    DONOF_CHECK(s.alloc(&dI, nn * naux));
    DONOF_CHECK(s.alloc(&dG, na2));
    DONOF_CHECK(s.alloc(&dw, (size_t)naux));
    DONOF_CHECK(s.alloc(&dVs, na2));
    DONOF_CHECK(s.alloc(&dVT, na2));
    DONOF_CHECK(s.alloc(&dGm, na2));
    DONOF_CHECK(s.alloc(&dA, na2));
    DONOF_CHECK(s.alloc(&dV, na2));
    DONOF_CHECK(s.alloc(&escr, eigh_scratch_bytes(naux)));
    DONOF_CUDA(ctx, cudaMemcpyAsync(dI, I_host, sizeof(double) * nn * naux, cudaMemcpyHostToDevice, st));
    DONOF_CUDA(ctx, cudaMemcpyAsync(dG, G_host, sizeof(double) * na2, cudaMemcpyHostToDevice, st));
    // eigen-decomposition of Symmetric(G) (its upper triangle)
    DONOF_CHECK(eigh_jacobi(ctx, st, dG, naux, dA, dV, dw, escr));
    {
        long long blocks = ((long long)na2 + 255) / 256;
        if (blocks > 8LL * ctx->sm_count) blocks = 8LL * ctx->sm_count;
        gmsqrt_factors_kernel<<<(int)blocks, 256, 0, st>>>(dV, dw, naux, dVs, dVT); count_launch();
        DONOF_CUDA(ctx, cudaGetLastError());
    }
    // G^{-1/2} = Vs V^T (A: Vs, M-contiguous; B: V^T stored K-contiguous)
    DONOF_CHECK(gemm_f64_auto(ctx, st, false, true, naux, naux, naux, dVs, naux, dVT, naux, dGm, naux, 1.0, 0.0,
                              part));
    // b = I G^{-1/2}: I as an (nbf^2 x naux) column-major matrix
    DONOF_CHECK(gemm_f64_auto(ctx, st, false, true, (int)nn, naux, naux, dI, (long long)nn, dGm, naux, b,
                              (long long)nn, 1.0, 0.0, part));
    DONOF_CUDA(ctx, cudaStreamSynchronize(st));  // the scratch is freed on return
    return DONOF_OK;
}

}  // namespace donof
