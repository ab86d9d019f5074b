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
#include <atomic>
#include <math.h>
#include <stdlib.h>

#include "dtile.cuh"
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
    return sizeof(double) * nn * (5 + SMAX + 2) + 256;  // + one slot for the single-launch form
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

// ---------------------------------------------------------------------------
// Single-launch form: one cooperative kernel runs every stage of the same
// algorithm (unpack + norm, X^2, X^3 and X^4, the Paterson-Stockmeyer
// combinations, the two Horner products, the s squarings and C E^(2^s)) with
// a bounded grid barrier between stages, instead of ~25 separate launches.
// The products are split into 32 x 16 tiles (dtile.cuh) spread over the SMs.
// On a barrier timeout the kernel records the error and returns (its output
// is then not valid).
// ---------------------------------------------------------------------------
namespace {

constexpr int RT_TN = 16;  // tile width of the rotation products

struct CoopState {
    unsigned long long norm_bits;
    dtile::GridSync gs;
};

struct CoopArgs {
    const double* y;
    int nbf, nbf5;
    const double* C;
    double* Cnew;
    double *Y, *X2, *X3, *X4, *P, *E1, *bufs;
    CoopState* cs;
    dtile::WaitCtl wc;
};

__device__ __forceinline__ dtile::Gemm sq_gemm(int n, const double* A, const double* B, double* C, double alpha,
                                               bool accumulate) {
    dtile::Gemm g;
    g.A = A; g.lda = n; g.ta = false;
    g.B = B; g.ldb = n; g.tb = false;
    g.C = C; g.ldc = n;
    g.M = n; g.N = n; g.K = n;
    g.alpha = alpha; g.accumulate = accumulate;
    return g;
}

__device__ __forceinline__ void run_tiles(const dtile::Gemm& g, double* sm, int cta, int G) {
    const int nt = dtile::tiles<RT_TN>(g);
    for (int w = cta; w < nt; w += G) dtile::tile<RT_TN>(g, w, sm);
}

// The whole rotation of one job on CTAs cta = 0..G-1 (of a cooperative launch).
__device__ __forceinline__ void rotate_body(const CoopArgs& a, int cta, int G, double* sm) {
    __shared__ double red[dtile::WARPS];
    const int n = a.nbf, tid = threadIdx.x;
    const long long nn = (long long)n * n;
    CoopState* cs = a.cs;
    dtile::GridSync* gs = &cs->gs;
    unsigned epoch = 0;
    // S0: unpack y into Y, column sums of |Y| -> ||Y||_1
    for (int j = cta; j < n; j += G) {
        double s = 0.0;
        for (int i = tid; i < n; i += dtile::THREADS) {
            double v = 0.0;
            if (i < j && i < a.nbf5) v = a.y[packed_index(i, j, n)];
            else if (j < i && j < a.nbf5) v = -a.y[packed_index(j, i, n)];
            a.Y[i + (long long)n * j] = v;
            s += fabs(v);
        }
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if ((tid & 31) == 0) red[tid >> 5] = s;
        __syncthreads();
        if (tid == 0) {
            double t = 0.0;
            for (int w = 0; w < dtile::WARPS; ++w) t += red[w];
            atomicMax(&cs->norm_bits, (unsigned long long)__double_as_longlong(t));
        }
        __syncthreads();
    }
    if (!dtile::grid_barrier(gs, epoch, G, a.wc)) return;
    const double norm = __longlong_as_double((long long)cs->norm_bits);
    int s = 0;
    if (norm > 0.25) s = (int)ceil(log2(norm / 0.25));
    if (s > SMAX) s = SMAX;
    const double sc = ldexp(1.0, -s);  // X = sc * Y (a power of two: exact)
    // S1: X2 = X X
    run_tiles(sq_gemm(n, a.Y, a.Y, a.X2, sc * sc, false), sm, cta, G);
    if (!dtile::grid_barrier(gs, epoch, G, a.wc)) return;
    // S2: X3 = X2 X, X4 = X2 X2
    {
        const dtile::Gemm g3 = sq_gemm(n, a.X2, a.Y, a.X3, sc, false);
        const dtile::Gemm g4 = sq_gemm(n, a.X2, a.X2, a.X4, 1.0, false);
        const int nt = dtile::tiles<RT_TN>(g3);
        for (int w = cta; w < 2 * nt; w += G) {
            if (w < nt) dtile::tile<RT_TN>(g3, w, sm);
            else dtile::tile<RT_TN>(g4, w - nt, sm);
        }
    }
    if (!dtile::grid_barrier(gs, epoch, G, a.wc)) return;
    // S3: the three polynomial blocks of the degree-12 Taylor sum (1/k! coefficients)
    {
        double c[13];
        c[0] = 1.0;
        for (int k = 1; k <= 12; ++k) c[k] = c[k - 1] / k;
        // four elements per thread and pass: every load is issued before the stores
        constexpr int U = 4;
        const long long stride = (long long)G * dtile::THREADS;
        for (long long base = cta * (long long)dtile::THREADS + tid; base < nn; base += U * stride) {
            double x[U], x2[U], x3[U], x4[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const long long idx = base + u * stride;
                const bool in = idx < nn;
                x[u] = in ? sc * a.Y[idx] : 0.0;
                x2[u] = in ? a.X2[idx] : 0.0;
                x3[u] = in ? a.X3[idx] : 0.0;
                x4[u] = in ? a.X4[idx] : 0.0;
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const long long idx = base + u * stride;
                if (idx >= nn) break;
                const double dg = ((idx % n) == (idx / n)) ? 1.0 : 0.0;
                a.P[idx] = c[12] * x4[u] + c[11] * x3[u] + c[10] * x2[u] + c[9] * x[u] + c[8] * dg;
                a.E1[idx] = c[7] * x3[u] + c[6] * x2[u] + c[5] * x[u] + c[4] * dg;
                a.bufs[idx] = c[3] * x3[u] + c[2] * x2[u] + c[1] * x[u] + c[0] * dg;
            }
        }
    }
    if (!dtile::grid_barrier(gs, epoch, G, a.wc)) return;
    // S4: E1 += P X4;  S5: E0 = bufs[0] += E1 X4
    run_tiles(sq_gemm(n, a.P, a.X4, a.E1, 1.0, true), sm, cta, G);
    if (!dtile::grid_barrier(gs, epoch, G, a.wc)) return;
    run_tiles(sq_gemm(n, a.E1, a.X4, a.bufs, 1.0, true), sm, cta, G);
    if (!dtile::grid_barrier(gs, epoch, G, a.wc)) return;
    // squarings: bufs[k+1] = bufs[k]^2
    for (int k = 0; k < s; ++k) {
        run_tiles(sq_gemm(n, a.bufs + k * nn, a.bufs + k * nn, a.bufs + (k + 1) * nn, 1.0, false), sm, cta, G);
        if (!dtile::grid_barrier(gs, epoch, G, a.wc)) return;
    }
    // C_new = C E^(2^s)
    run_tiles(sq_gemm(n, a.C, a.bufs + s * nn, a.Cnew, 1.0, false), sm, cta, G);
}

__global__ void __launch_bounds__(dtile::THREADS) rotate_coop_kernel(const CoopArgs a) {
    extern __shared__ __align__(16) double sm[];
    rotate_body(a, blockIdx.x, gridDim.x, sm);
}

static_assert(sizeof(CoopState) <= GROUP_STATE_BYTES, "rotation state slot too small");

// Grouped form: the rotations of several jobs in one cooperative launch, job j
// on CTAs [cta0, cta0 + ctas) with its own barrier state.  A CTA that lies in
// several jobs' ranges (only jobs with ctas == 1 share CTAs) runs them in order.
__global__ void __launch_bounds__(dtile::THREADS) rotate_grouped_kernel(const RotJob* __restrict__ jobs, int njobs,
                                                                        const dtile::WaitCtl wc) {
    extern __shared__ __align__(16) double sm[];
    const int cta = blockIdx.x;
    for (int j = 0; j < njobs; ++j) {
        const int c0 = jobs[j].cta0, cn = jobs[j].ctas;
        if (cta < c0 || cta >= c0 + cn) continue;
        const RotJob r = jobs[j];
        if (r.skip != nullptr && *r.skip != 0) continue;
        const long long nn = (long long)r.nbf * r.nbf;
        CoopArgs a{};
        a.y = r.y; a.nbf = r.nbf; a.nbf5 = r.nbf5; a.C = r.C; a.Cnew = r.Cnew;
        a.cs = static_cast<CoopState*>(r.state);
        a.Y = r.work;
        a.X2 = a.Y + nn; a.X3 = a.Y + 2 * nn; a.X4 = a.Y + 3 * nn; a.P = a.Y + 4 * nn;
        a.bufs = a.Y + 5 * nn;
        a.E1 = a.bufs + (SMAX + 1) * nn;
        a.wc = wc;
        rotate_body(a, cta - c0, cn, sm);
        __syncthreads();
    }
}

}  // namespace

size_t rotate_work_doubles(int nbf) { return (size_t)nbf * nbf * (5 + SMAX + 2); }

int rotate_grouped(donof_ctx* ctx, cudaStream_t st, const RotJob* jobs, int njobs, void* states, int grid) {
    const int smem = (int)sizeof(double) * dtile::smem_doubles<RT_TN>();
    static std::atomic<unsigned long long> attr_mask{0};
    const unsigned long long bit = 1ull << (ctx->device & 63);
    if (!(attr_mask.load(std::memory_order_acquire) & bit)) {
        DONOF_CUDA(ctx, cudaFuncSetAttribute(rotate_grouped_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        attr_mask.fetch_or(bit, std::memory_order_acq_rel);
    }
    if (grid < 1 || grid > ctx->sm_count) {
        set_error(ctx, "rotate_grouped: %d CTAs (1..%d allowed)", grid, ctx->sm_count);
        return DONOF_ERR_ARG;
    }
    DONOF_CUDA(ctx, cudaMemsetAsync(states, 0, (size_t)GROUP_STATE_BYTES * njobs, st));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(dtile::THREADS);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    DONOF_CUDA(ctx, cudaLaunchKernelEx(&cfg, rotate_grouped_kernel, jobs, njobs, dtile::wait_ctl(ctx)));
    count_launch();
    return DONOF_OK;
}

int rotate_f64(donof_ctx* ctx, cudaStream_t st, const double* y, int nbf, int nbf5,
               const double* C, double* Cnew) {
    // DONOF_ROTATE_MULTI=1 selects the multi-launch form (same arithmetic)
    static const bool multi = [] {
        const char* e = getenv("DONOF_ROTATE_MULTI");
        return e != nullptr && e[0] == '1';
    }();
    if (multi) return rotate_f64_gated(ctx, st, y, nbf, nbf5, C, Cnew, nullptr, nullptr);
    const long long nn = (long long)nbf * nbf;
    DONOF_CHECK(ctx->rot.ensure(ctx, rotate_scratch_bytes(nbf)));
    char* base = ctx->rot.as<char>();
    CoopArgs a{};
    a.y = y; a.nbf = nbf; a.nbf5 = nbf5; a.C = C; a.Cnew = Cnew;
    a.cs = reinterpret_cast<CoopState*>(base);
    a.Y = reinterpret_cast<double*>(base + 256);
    a.X2 = a.Y + nn; a.X3 = a.Y + 2 * nn; a.X4 = a.Y + 3 * nn; a.P = a.Y + 4 * nn;
    a.bufs = a.Y + 5 * nn;           // E^(2^k), k = 0..SMAX
    a.E1 = a.bufs + (SMAX + 1) * nn;  // extra slot
    a.wc = dtile::wait_ctl(ctx);
    const int smem = (int)sizeof(double) * dtile::smem_doubles<RT_TN>();
    static std::atomic<unsigned long long> attr_mask{0};
    const unsigned long long bit = 1ull << (ctx->device & 63);
    if (!(attr_mask.load(std::memory_order_acquire) & bit)) {
        DONOF_CUDA(ctx, cudaFuncSetAttribute(rotate_coop_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        attr_mask.fetch_or(bit, std::memory_order_acq_rel);
    }
    int per_sm = 0;
    DONOF_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, rotate_coop_kernel, dtile::THREADS, smem));
    if (per_sm < 1) {
        set_error(ctx, "rotate_coop_kernel does not fit on an SM");
        return DONOF_ERR_CUDA;
    }
    const int mt = (nbf + dtile::TM - 1) / dtile::TM, ntile = mt * ((nbf + RT_TN - 1) / RT_TN);
    int grid = ctx_ctas(ctx);                  // at most one CTA per SM (co-resident: the kernel has grid barriers)
    if (grid > 2 * ntile) grid = 2 * ntile;    // stage S2 has 2 * ntile tiles
    if (grid < 1) grid = 1;
    DONOF_CUDA(ctx, cudaMemsetAsync(a.cs, 0, sizeof(CoopState), st));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(dtile::THREADS);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    DONOF_CUDA(ctx, cudaLaunchKernelEx(&cfg, rotate_coop_kernel, a));
    count_launch();
    return DONOF_OK;
}

}  // namespace donof
