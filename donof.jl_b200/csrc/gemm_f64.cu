// Host-side dispatch of the FP64 DMMA GEMM (tile shape, operand layout,
// 16-byte vs 8-byte staging) and the split-K reduction.
#include <atomic>
#include "gemm_f64.cuh"
#include "kernels.cuh"

namespace donof {

namespace {

template <int BM, int BN, int WM, int WN, bool AK, bool BKM, bool VEC>
cudaError_t launch_cfg(const GemmF64Args& p, cudaStream_t st) {
    constexpr int BK = 16, STAGES = 3;
    using Cfg = GemmF64Cfg<BM, BN, BK, WM, WN, STAGES, AK, BKM, VEC>;
    auto kern = gemm_f64_kernel<BM, BN, BK, WM, WN, STAGES, AK, BKM, VEC>;
    // the shared-memory opt-in is per function and device; remember it per device
    static std::atomic<unsigned long long> attr_mask{0};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const unsigned long long bit = 1ull << (dev & 63);
    if (!(attr_mask.load(std::memory_order_acquire) & bit)) {
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)Cfg::SMEM_BYTES);
        if (e != cudaSuccess) return e;
        attr_mask.fetch_or(bit, std::memory_order_acq_rel);
    }
    dim3 grid((p.M + BM - 1) / BM, (p.N + BN - 1) / BN, p.batch * p.splits);
    kern<<<grid, Cfg::THREADS, Cfg::SMEM_BYTES, st>>>(p); count_launch();
    return cudaGetLastError();
}

template <int BM, int BN, int WM, int WN, bool AK, bool BKM>
cudaError_t launch_vec(const GemmF64Args& p, bool vec, cudaStream_t st) {
    return vec ? launch_cfg<BM, BN, WM, WN, AK, BKM, true>(p, st)
               : launch_cfg<BM, BN, WM, WN, AK, BKM, false>(p, st);
}

template <int BM, int BN, int WM, int WN>
cudaError_t launch_layout(const GemmF64Args& p, bool ak, bool bk, bool vec, cudaStream_t st) {
    if (ak && bk) return launch_vec<BM, BN, WM, WN, true, true>(p, vec, st);
    if (ak && !bk) return launch_vec<BM, BN, WM, WN, true, false>(p, vec, st);
    if (!ak && bk) return launch_vec<BM, BN, WM, WN, false, true>(p, vec, st);
    return launch_vec<BM, BN, WM, WN, false, false>(p, vec, st);
}

bool aligned16(const void* ptr) { return (reinterpret_cast<uintptr_t>(ptr) & 15u) == 0; }

}  // namespace

int gemm_f64(donof_ctx* ctx, cudaStream_t st, bool a_kmajor, bool b_kmajor, GemmF64Args p,
             GemmTile tile) {
    if (p.M <= 0 || p.N <= 0 || p.batch <= 0) return DONOF_OK;
    if (p.splits < 1) p.splits = 1;
    if (p.splits == 1 || p.kchunk <= 0) p.kchunk = p.K;
    // 16-byte staging needs 16-byte aligned bases and even strides along and
    // across the copied direction, and an even extent along it.
    const bool va = aligned16(p.A) && (p.lda % 2 == 0) && (p.strideA % 2 == 0) &&
                    (a_kmajor ? (p.K % 2 == 0 && p.kchunk % 2 == 0) : (p.M % 2 == 0));
    const bool vb = aligned16(p.B) && (p.ldb % 2 == 0) && (p.strideB % 2 == 0) &&
                    (b_kmajor ? (p.K % 2 == 0 && p.kchunk % 2 == 0) : (p.N % 2 == 0));
    const bool vec = va && vb;
    cudaError_t e;
    if (tile == GemmTile::Large)
        e = launch_layout<128, 64, 4, 2>(p, a_kmajor, b_kmajor, vec, st);
    else if (tile == GemmTile::Small)
        e = launch_layout<64, 64, 2, 2>(p, a_kmajor, b_kmajor, vec, st);
    else
        e = launch_layout<32, 32, 2, 2>(p, a_kmajor, b_kmajor, vec, st);
    if (e != cudaSuccess) {
        set_error(ctx, "gemm_f64 launch (M=%d N=%d K=%d batch=%d splits=%d): %s", p.M, p.N, p.K,
                  p.batch, p.splits, cudaGetErrorString(e));
        return DONOF_ERR_CUDA;
    }
    return DONOF_OK;
}

GemmTile pick_tile(donof_ctx* ctx, int M, int N, int K, bool can_split, int* splits_out) {
    struct Cand { GemmTile t; int bm, bn; };
    const Cand cands[3] = {{GemmTile::Large, 128, 64}, {GemmTile::Small, 64, 64}, {GemmTile::Tiny, 32, 32}};
    const int want = 2 * ctx->sm_count;
    for (int c = 0; c < 3; ++c) {
        const long long tiles = (long long)((M + cands[c].bm - 1) / cands[c].bm) * ((N + cands[c].bn - 1) / cands[c].bn);
        int splits = 1;
        if (can_split && tiles < want) {
            const int max_splits = K / 64 > 1 ? K / 64 : 1;  // keep every split >= 64 deep
            long long s = (want + tiles - 1) / tiles;
            splits = (int)(s < max_splits ? s : max_splits);
        }
        if (tiles * splits >= ctx->sm_count || c == 2) {
            *splits_out = splits;
            return cands[c].t;
        }
    }
    *splits_out = 1;
    return GemmTile::Tiny;
}

int gemm_f64_auto(donof_ctx* ctx, cudaStream_t st, bool a_kmajor, bool b_kmajor, int M, int N,
                  int K, const double* A, long long lda, const double* B, long long ldb,
                  double* C, long long ldc, double alpha, double beta, DevBuf* part) {
    GemmF64Args p{};
    p.M = M; p.N = N; p.K = K;
    p.A = A; p.lda = lda; p.B = B; p.ldb = ldb; p.C = C; p.ldc = ldc;
    p.alpha = alpha; p.beta = beta; p.batch = 1; p.splits = 1; p.kchunk = K;
    int splits = 1, kchunk = K;
    const GemmTile tile = pick_tile(ctx, M, N, K, part != nullptr, &splits);
    if (splits > 1) {
        kchunk = ((K + splits - 1) / splits + 15) / 16 * 16;
        splits = (K + kchunk - 1) / kchunk;
    }
    if (splits > 1) {
        const long long per = (long long)M * N;
        DONOF_CHECK(part->ensure(ctx, sizeof(double) * per * splits));
        GemmF64Args q = p;
        q.C = part->as<double>(); q.ldc = M; q.splits = splits;
        q.kchunk = kchunk;
        q.strideSplit = per; q.beta = 0.0;
        DONOF_CHECK(gemm_f64(ctx, st, a_kmajor, b_kmajor, q, tile));
        if (ldc == M) return splitk_reduce(ctx, st, q.C, per, splits, per, C, beta);
        // strided destination: reduce column by column
        for (int j = 0; j < N; ++j)
            DONOF_CHECK(splitk_reduce(ctx, st, q.C + (long long)j * M, per, splits, M,
                                      C + (long long)j * ldc, beta));
        return DONOF_OK;
    }
    return gemm_f64(ctx, st, a_kmajor, b_kmajor, p, tile);
}

int gemm_f64_partials(donof_ctx* ctx, cudaStream_t st, bool a_kmajor, bool b_kmajor, int M, int N, int K,
                      const double* A, long long lda, const double* B, long long ldb, DevBuf* part,
                      const double** out, int* nparts) {
    GemmF64Args p{};
    p.M = M; p.N = N; p.K = K;
    p.A = A; p.lda = lda; p.B = B; p.ldb = ldb;
    p.alpha = 1.0; p.beta = 0.0; p.batch = 1; p.splits = 1; p.kchunk = K;
    int splits = 1, kchunk = K;
    const GemmTile tile = pick_tile(ctx, M, N, K, true, &splits);
    if (splits > 1) {
        kchunk = ((K + splits - 1) / splits + 15) / 16 * 16;
        splits = (K + kchunk - 1) / kchunk;
    }
    const long long per = (long long)M * N;
    DONOF_CHECK(part->ensure(ctx, sizeof(double) * per * splits));
    p.C = part->as<double>(); p.ldc = M;
    if (splits > 1) {
        p.splits = splits;
        p.kchunk = kchunk;
        p.strideSplit = per;
    }
    DONOF_CHECK(gemm_f64(ctx, st, a_kmajor, b_kmajor, p, tile));
    *out = part->as<double>();
    *nparts = splits;
    return DONOF_OK;
}

__global__ void splitk_reduce_kernel(const double* __restrict__ part, long long stride, int splits,
                                     long long count, double* __restrict__ out, double beta) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int k = 0; k < splits; ++k) s += part[i + k * stride];
        out[i] = (beta != 0.0) ? s + beta * out[i] : s;
    }
}

int splitk_reduce(donof_ctx* ctx, cudaStream_t st, const double* part, long long stride,
                  int splits, long long count, double* out, double beta) {
    const int threads = 256;
    long long blocks = (count + threads - 1) / threads;
    if (blocks > 4 * (long long)ctx->sm_count) blocks = 4 * (long long)ctx->sm_count;
    if (blocks < 1) blocks = 1;
    splitk_reduce_kernel<<<(unsigned)blocks, threads, 0, st>>>(part, stride, splits, count, out, beta); count_launch();
    DONOF_CUDA(ctx, cudaGetLastError());
    return DONOF_OK;
}

}  // namespace donof
