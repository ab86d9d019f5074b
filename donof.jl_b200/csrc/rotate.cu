// rotate_orbital in FP64 on the device (src/utils.jl:499-521):
//   Y = unpack(y) (antisymmetric, nonzero rows/cols only in the first nbf5),
//   C_new = C exp(Y).
//
// exp(Y) by scaling and squaring with a degree-12 Taylor polynomial evaluated
// Paterson-Stockmeyer style in X^4 (3 + 2 GEMMs):
//   X = Y / 2^s  with s = max(0, ceil(log2(||Y||_1 / 0.25))), so ||X||_1 <= 1/4
//   and the truncation error is below 0.25^13/13! ~ 2.4e-18;
//   E = sum_{k<=12} X^k / k!,   exp(Y) = E^(2^s).
// s is chosen on the device; the SMAX squaring launches are gated by it
// (a launch with k >= s returns at once), and the final C E^(2^s) GEMM reads
// the matching buffer through a device-side pointer, so the whole sequence
// has no host round trip and can be captured in a graph.  Norms beyond
// 0.25 * 2^SMAX are flagged in the status word (accuracy would degrade).
#include <math.h>

#include "kernels.cuh"

namespace donof {

namespace {

constexpr int SMAX = 10;

struct RotState {
    unsigned long long norm_bits;  // ||Y||_1 as the bit pattern of a non-negative double
    int s;
    int overflow;
    double scale;
    const double* U;  // E^(2^s)
};

__device__ __forceinline__ long long packed_index(int i, int j, int nbf) {
    // row-wise packing over i < nbf5, j > i (src/utils.jl:503-510)
    return (long long)i * (nbf - 1) - (long long)i * (i - 1) / 2 + (j - i - 1);
}

__global__ void unpack_kernel(const double* __restrict__ y, int nbf, int nbf5,
                              double* __restrict__ Y, const int* done) {
    if (done != nullptr && *done) return;
    const long long total = (long long)nbf * nbf;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(idx % nbf), j = (int)(idx / nbf);
        double v = 0.0;
        if (i < j && i < nbf5) v = y[packed_index(i, j, nbf)];
        else if (j < i && j < nbf5) v = -y[packed_index(j, i, nbf)];
        Y[idx] = v;
    }
}

// one CTA per column: ||Y||_1 = max_j sum_i |Y_ij|
__global__ void colnorm_kernel(const double* __restrict__ Y, int nbf, RotState* st, const int* done) {
    if (done != nullptr && *done) return;
    __shared__ double red[32];
    const int j = blockIdx.x;
    double s = 0.0;
    for (int i = threadIdx.x; i < nbf; i += blockDim.x) s += fabs(Y[i + (long long)nbf * j]);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        atomicMax(&st->norm_bits, (unsigned long long)__double_as_longlong(t));
    }
}

__global__ void select_kernel(RotState* st, const double* bufs, long long nn, const int* done) {
    if (done != nullptr && *done) return;
    const double norm = __longlong_as_double((long long)st->norm_bits);
    int s = 0;
    if (norm > 0.25) s = (int)ceil(log2(norm / 0.25));
    st->overflow = (s > SMAX) ? 1 : 0;
    if (s > SMAX) s = SMAX;
    if (s < 0) s = 0;
    st->s = s;
    st->scale = ldexp(1.0, -s);
    st->U = bufs + (long long)s * nn;
}

// out = a4 X4 + a3 X3 + a2 X2 + a1 X + a0 I (null inputs have zero weight);
// with scale_from != nullptr, X is replaced by (*scale_from) * X.
__global__ void lincomb_kernel(int nbf, double a0, double a1, const double* __restrict__ X,
                               double a2, const double* __restrict__ X2, double a3,
                               const double* __restrict__ X3, double a4,
                               const double* __restrict__ X4, const RotState* scale_from,
                               double* __restrict__ out, const int* done) {
    if (done != nullptr && *done) return;
    const double sc = scale_from ? scale_from->scale : 1.0;
    const long long total = (long long)nbf * nbf;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        double v = ((idx % nbf) == (idx / nbf)) ? a0 : 0.0;
        if (X) v += a1 * sc * X[idx];
        if (X2) v += a2 * X2[idx];
        if (X3) v += a3 * X3[idx];
        if (X4) v += a4 * X4[idx];
        out[idx] = v;
    }
}

int blocks_for(long long total, int sm) {
    long long b = (total + 255) / 256;
    if (b > 4LL * sm) b = 4LL * sm;
    return (int)(b < 1 ? 1 : b);
}

}  // namespace

size_t rotate_scratch_bytes(int nbf) {
    const size_t nn = (size_t)nbf * nbf;
    return sizeof(double) * nn * (5 + SMAX + 1) + 256;
}

int rotate_f64_gated(donof_ctx* ctx, cudaStream_t st, const double* y, int nbf, int nbf5,
                     const double* C, double* Cnew, const int* done, DevBuf* part) {
    const long long nn = (long long)nbf * nbf;
    DONOF_CHECK(ctx->rot.ensure(ctx, rotate_scratch_bytes(nbf)));
    char* base = ctx->rot.as<char>();
    RotState* rs = reinterpret_cast<RotState*>(base);
    double* Y = reinterpret_cast<double*>(base + 256);
    double* X = Y;  // scaled in place by the first lincomb
    double* X2 = Y + nn;
    double* X3 = Y + 2 * nn;
    double* X4 = Y + 3 * nn;
    double* P = Y + 4 * nn;
    double* bufs = Y + 5 * nn;  // E^(2^k), k = 0..SMAX
    const int nb = blocks_for(nn, ctx->sm_count);
    const double c[13] = {1.0,
                          1.0,
                          1.0 / 2,
                          1.0 / 6,
                          1.0 / 24,
                          1.0 / 120,
                          1.0 / 720,
                          1.0 / 5040,
                          1.0 / 40320,
                          1.0 / 362880,
                          1.0 / 3628800,
                          1.0 / 39916800,
                          1.0 / 479001600};

    DONOF_CUDA(ctx, cudaMemsetAsync(rs, 0, sizeof(RotState), st));
    unpack_kernel<<<nb, 256, 0, st>>>(y, nbf, nbf5, Y, done); count_launch();
    colnorm_kernel<<<nbf, 128, 0, st>>>(Y, nbf, rs, done); count_launch();
    select_kernel<<<1, 1, 0, st>>>(rs, bufs, nn, done); count_launch();
    // X = Y * 2^-s (in place)
    lincomb_kernel<<<nb, 256, 0, st>>>(nbf, 0.0, 1.0, Y, 0.0, nullptr, 0.0, nullptr, 0.0, nullptr, rs,
                                       X, done); count_launch();
    DONOF_CUDA(ctx, cudaGetLastError());

    auto mm = [&](const double* A, const double* B, double* Cm, double beta, const int* skip_le,
                  int level, const double* const* bptr) -> int {
        int splits = 1;
        const GemmTile tile = pick_tile(ctx, nbf, nbf, nbf, false, &splits);
        GemmF64Args p{};
        p.M = nbf; p.N = nbf; p.K = nbf;
        p.A = A; p.lda = nbf; p.B = B; p.ldb = nbf; p.C = Cm; p.ldc = nbf;
        p.alpha = 1.0; p.beta = beta; p.batch = 1; p.splits = 1; p.kchunk = nbf;
        p.skip_le = skip_le; p.skip_level = level; p.skip_nz = done; p.B_ptr = bptr;
        return gemm_f64(ctx, st, false, true, p, tile);
    };
    (void)part;
    DONOF_CHECK(mm(X, X, X2, 0.0, nullptr, 0, nullptr));
    DONOF_CHECK(mm(X2, X, X3, 0.0, nullptr, 0, nullptr));
    DONOF_CHECK(mm(X2, X2, X4, 0.0, nullptr, 0, nullptr));
    // P = c12 X4 + c11 X3 + c10 X2 + c9 X + c8 I
    lincomb_kernel<<<nb, 256, 0, st>>>(nbf, c[8], c[9], X, c[10], X2, c[11], X3, c[12], X4, nullptr, P,
                                       done); count_launch();
    // E1 = P X4 + (c7 X3 + c6 X2 + c5 X + c4 I)
    double* E1 = bufs;  // reuse bufs[0] as a temporary, overwritten below
    lincomb_kernel<<<nb, 256, 0, st>>>(nbf, c[4], c[5], X, c[6], X2, c[7], X3, 0.0, nullptr, nullptr,
                                       E1, done); count_launch();
    DONOF_CUDA(ctx, cudaGetLastError());
    DONOF_CHECK(mm(P, X4, E1, 1.0, nullptr, 0, nullptr));
    // E0 = E1 X4 + (c3 X3 + c2 X2 + c1 X + c0 I)   -> bufs[0] via P as staging
    lincomb_kernel<<<nb, 256, 0, st>>>(nbf, c[0], c[1], X, c[2], X2, c[3], X3, 0.0, nullptr, nullptr, P,
                                       done); count_launch();
    DONOF_CUDA(ctx, cudaGetLastError());
    DONOF_CHECK(mm(E1, X4, P, 1.0, nullptr, 0, nullptr));
    DONOF_CUDA(ctx, cudaMemcpyAsync(bufs, P, sizeof(double) * nn, cudaMemcpyDeviceToDevice, st));
    // repeated squaring, gated by s
    for (int k = 0; k < SMAX; ++k)
        DONOF_CHECK(mm(bufs + k * nn, bufs + k * nn, bufs + (k + 1) * nn, 0.0, &rs->s, k, nullptr));
    // C_new = C * E^(2^s)
    DONOF_CHECK(mm(C, nullptr, Cnew, 0.0, nullptr, 0, &rs->U));
    return DONOF_OK;
}

int rotate_f64(donof_ctx* ctx, cudaStream_t st, const double* y, int nbf, int nbf5,
               const double* C, double* Cnew) {
    return rotate_f64_gated(ctx, st, y, nbf, nbf5, C, Cnew, nullptr, nullptr);
}

}  // namespace donof
