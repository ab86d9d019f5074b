// The FP64 tail of the orbital-gradient Lagrangian, in one cooperative launch
// (src/utils.jl:17-18 and :39 for H_mat and elag, :216-227 for the energy):
//
//   Y      = sum_g part_g            partial sums of Y = sum_l tmp_l W_l (FP32 per-CTA
//                                    partials of the mixed kernel, or FP64 split-K partials)
//   HC     = H C5                    (nbf x nbf5)
//   Bp     = HC diag(n) + Y
//   H_mat  = C^T HC                  (nbf x nbf5)
//   elag   = [C^T Bp | 0]            = n o H_mat + C^T Y on the first nbf5 columns
//   E_elec = sum_{i < nbf5} elag[i, i] + n_i H_mat[i, i]
//
// Stage 1 runs the HC tiles and the reduction of the Y partials side by side,
// stage 2 forms Bp, stage 3 the H_mat and elag tiles; the last CTA to finish
// stage 3 sums the energy in a fixed order.  Bounded grid barriers separate
// the stages.
#include <atomic>
#include "dtile.cuh"
#include "kernels.cuh"

namespace donof {

namespace {

constexpr int TL_TN = 16;

struct TailState {
    dtile::GridSync gs;
    unsigned done;
    unsigned pad[3];
};

struct TailArgs {
    const double* C;
    const double* H;
    const double* n;
    int nbf, nbf5;
    const void* part;  // part[g * pstride + m + nbf * b]
    int part_f32;
    int nparts;
    long long pstride;
    double *Y, *HC, *Bp;  // scratch, nbf x nbf5 each
    double *Hmat, *elag, *E;
    TailState* ts;
    dtile::WaitCtl wc;
};

// The whole tail of one job on CTAs cta = 0..G-1 (of a cooperative launch).
__device__ __forceinline__ void tail_body(const TailArgs& a, int cta, int G, double* sm) {
    const int nbf = a.nbf, nbf5 = a.nbf5, tid = threadIdx.x;
    const long long ny = (long long)nbf * nbf5;
    dtile::GridSync* gs = &a.ts->gs;
    unsigned epoch = 0;

    // ---- stage 1: HC = H C5 (tiles on the first CTAs), Y = sum of partials (the rest)
    dtile::Gemm ghc;
    ghc.A = a.H; ghc.lda = nbf; ghc.ta = false;
    ghc.B = a.C; ghc.ldb = nbf; ghc.tb = false;
    ghc.C = a.HC; ghc.ldc = nbf;
    ghc.M = nbf; ghc.N = nbf5; ghc.K = nbf;
    ghc.alpha = 1.0; ghc.accumulate = false;
    const int nt_hc = dtile::tiles<TL_TN>(ghc);
    const int red_ctas = G > nt_hc ? G - nt_hc : G;  // CTAs that reduce Y
    const int red_first = G > nt_hc ? nt_hc : 0;
    for (int w = cta; w < nt_hc; w += G) dtile::tile<TL_TN>(ghc, w, sm);
    if (cta >= red_first) {
        // Warp w sums the partials g = w (mod WARPS) of a block of elements, then the
        // warps' sums are added in a fixed order (the result does not depend on timing).
        __shared__ double wsum[dtile::WARPS][128];
        const int lane = tid & 31, warp = tid >> 5;
        const bool vec = a.part_f32 && (a.pstride & 3) == 0 && (ny & 3) == 0 &&
                         (reinterpret_cast<uintptr_t>(a.part) & 15) == 0;
        if (vec) {
            // FP32 partials, blocks of 128 elements: four consecutive elements per lane
            const long long nblk = (ny + 127) / 128;
            const float* p = static_cast<const float*>(a.part);
            for (long long blk = cta - red_first; blk < nblk; blk += red_ctas) {
                const long long e = blk * 128 + 4 * lane;
                double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
                if (e < ny) {
                    // up to PF partials per warp in flight at once
                    constexpr int PF = 20;
                    for (int g0 = warp; g0 < a.nparts; g0 += PF * dtile::WARPS) {
                        float4 v[PF];
#pragma unroll
                        for (int i = 0; i < PF; ++i) {
                            const int g = g0 + i * dtile::WARPS;
                            v[i] = (g < a.nparts) ? __ldg(reinterpret_cast<const float4*>(p + g * a.pstride + e))
                                                  : make_float4(0.f, 0.f, 0.f, 0.f);
                        }
#pragma unroll
                        for (int i = 0; i < PF; ++i) {
                            s0 += (double)v[i].x; s1 += (double)v[i].y; s2 += (double)v[i].z; s3 += (double)v[i].w;
                        }
                    }
                }
                wsum[warp][4 * lane] = s0;
                wsum[warp][4 * lane + 1] = s1;
                wsum[warp][4 * lane + 2] = s2;
                wsum[warp][4 * lane + 3] = s3;
                __syncthreads();
                if (tid < 128 && blk * 128 + tid < ny) {
                    double t = 0.0;
#pragma unroll
                    for (int w = 0; w < dtile::WARPS; ++w) t += wsum[w][tid];
                    a.Y[blk * 128 + tid] = t;
                }
                __syncthreads();
            }
        } else {
            // blocks of 64 elements, two per lane
            const long long nblk = (ny + 63) / 64;
            for (long long blk = cta - red_first; blk < nblk; blk += red_ctas) {
                const long long e0 = blk * 64 + lane, e1 = e0 + 32;
                double s0 = 0.0, s1 = 0.0;
                if (a.part_f32) {
                    const float* p = static_cast<const float*>(a.part);
#pragma unroll 4
                    for (int g = warp; g < a.nparts; g += dtile::WARPS) {
                        const float* q = p + g * a.pstride;
                        if (e0 < ny) s0 += (double)__ldg(q + e0);
                        if (e1 < ny) s1 += (double)__ldg(q + e1);
                    }
                } else {
                    const double* p = static_cast<const double*>(a.part);
#pragma unroll 4
                    for (int g = warp; g < a.nparts; g += dtile::WARPS) {
                        const double* q = p + g * a.pstride;
                        if (e0 < ny) s0 += __ldg(q + e0);
                        if (e1 < ny) s1 += __ldg(q + e1);
                    }
                }
                wsum[warp][lane] = s0;
                wsum[warp][32 + lane] = s1;
                __syncthreads();
                if (tid < 64 && blk * 64 + tid < ny) {
                    double t = 0.0;
#pragma unroll
                    for (int w = 0; w < dtile::WARPS; ++w) t += wsum[w][tid];
                    a.Y[blk * 64 + tid] = t;
                }
                __syncthreads();
            }
        }
    }
    // columns nbf5.. of elag are zero
    {
        const long long z0 = (long long)nbf * nbf5, zn = (long long)nbf * nbf;
        for (long long i = z0 + (long long)cta * dtile::THREADS + tid; i < zn; i += (long long)G * dtile::THREADS)
            a.elag[i] = 0.0;
    }
    if (!dtile::grid_barrier(gs, epoch, G, a.wc)) return;

    // ---- stage 2: Bp = HC diag(n) + Y
    for (long long i = (long long)cta * dtile::THREADS + tid; i < ny; i += (long long)G * dtile::THREADS)
        a.Bp[i] = a.HC[i] * a.n[i / nbf] + a.Y[i];
    if (!dtile::grid_barrier(gs, epoch, G, a.wc)) return;

    // ---- stage 3: H_mat = C^T HC, elag[:, :nbf5] = C^T Bp
    dtile::Gemm gh;
    gh.A = a.C; gh.lda = nbf; gh.ta = true;
    gh.B = a.HC; gh.ldb = nbf; gh.tb = false;
    gh.C = a.Hmat; gh.ldc = nbf;
    gh.M = nbf; gh.N = nbf5; gh.K = nbf;
    gh.alpha = 1.0; gh.accumulate = false;
    dtile::Gemm ge = gh;
    ge.B = a.Bp;
    ge.C = a.elag;
    const int nt = dtile::tiles<TL_TN>(gh);
    for (int w = cta; w < 2 * nt; w += G) {
        if (w < nt) dtile::tile<TL_TN>(gh, w, sm);
        else dtile::tile<TL_TN>(ge, w - nt, sm);
    }
    if (a.E == nullptr) return;
    // ---- energy: the last CTA to finish sums the diagonals in a fixed order
    __shared__ unsigned last;
    __shared__ double red[dtile::WARPS];
    __syncthreads();
    if (tid == 0) {
        __threadfence();
        last = (atomicAdd(&a.ts->done, 1u) == (unsigned)G - 1) ? 1u : 0u;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double s = 0.0;
    for (int i = tid; i < nbf5; i += dtile::THREADS) {
        const volatile double* el = a.elag;
        const volatile double* hm = a.Hmat;
        s += el[i + (long long)nbf * i] + a.n[i] * hm[i + (long long)nbf * i];
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((tid & 31) == 0) red[tid >> 5] = s;
    __syncthreads();
    if (tid == 0) {
        double t = 0.0;
        for (int w = 0; w < dtile::WARPS; ++w) t += red[w];
        *a.E = t;
    }
}

__global__ void __launch_bounds__(dtile::THREADS) elag_tail_kernel(const TailArgs a) {
    extern __shared__ __align__(16) double sm[];
    tail_body(a, blockIdx.x, gridDim.x, sm);
}

static_assert(sizeof(TailState) <= GROUP_STATE_BYTES, "tail state slot too small");

// Grouped form: the tails of several jobs in one cooperative launch, job j on
// CTAs [cta0, cta0 + ctas) with its own barrier state (as rotate_grouped_kernel).
__global__ void __launch_bounds__(dtile::THREADS) tail_grouped_kernel(const TailJob* __restrict__ jobs, int njobs,
                                                                      const dtile::WaitCtl wc) {
    extern __shared__ __align__(16) double sm[];
    const int cta = blockIdx.x;
    for (int j = 0; j < njobs; ++j) {
        const int c0 = jobs[j].cta0, cn = jobs[j].ctas;
        if (cta < c0 || cta >= c0 + cn) continue;
        const TailJob t = jobs[j];
        if (t.skip != nullptr && *t.skip != 0) continue;
        const long long ny = (long long)t.nbf * t.nbf5;
        TailArgs a{};
        a.C = t.C; a.H = t.H; a.n = t.n;
        a.nbf = t.nbf; a.nbf5 = t.nbf5;
        a.part = t.part; a.part_f32 = t.part_f32; a.nparts = t.nparts; a.pstride = t.pstride;
        a.ts = static_cast<TailState*>(t.state);
        a.Y = t.work; a.HC = a.Y + ny; a.Bp = a.HC + ny;
        a.Hmat = t.Hmat; a.elag = t.elag; a.E = t.E;
        a.wc = wc;
        tail_body(a, cta - c0, cn, sm);
        __syncthreads();
    }
}

}  // namespace

int tail_grouped(donof_ctx* ctx, cudaStream_t st, const TailJob* jobs, int njobs, void* states, int grid) {
    const int smem = (int)sizeof(double) * dtile::smem_doubles<TL_TN>();
    static std::atomic<unsigned long long> attr_mask{0};
    const unsigned long long bit = 1ull << (ctx->device & 63);
    if (!(attr_mask.load(std::memory_order_acquire) & bit)) {
        DONOF_CUDA(ctx, cudaFuncSetAttribute(tail_grouped_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        attr_mask.fetch_or(bit, std::memory_order_acq_rel);
    }
    if (grid < 1 || grid > ctx->sm_count) {
        set_error(ctx, "tail_grouped: %d CTAs (1..%d allowed)", grid, ctx->sm_count);
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
    DONOF_CUDA(ctx, cudaLaunchKernelEx(&cfg, tail_grouped_kernel, jobs, njobs, dtile::wait_ctl(ctx)));
    count_launch();
    return DONOF_OK;
}

int elag_tail_f64(donof_job* job, cudaStream_t st, const double* C, const double* H, const double* n, int nbf5,
                  const void* part, bool part_f32, int nparts, long long pstride, double* Hmat, double* elag,
                  double* E) {
    donof_ctx* ctx = job->ctx;
    const int nbf = job->nbf;
    const size_t ny = (size_t)nbf * nbf5;
    DONOF_CHECK(job->small.ensure(ctx, 256 + sizeof(double) * 3 * ny));
    char* base = job->small.as<char>();
    TailArgs a{};
    a.C = C; a.H = H; a.n = n;
    a.nbf = nbf; a.nbf5 = nbf5;
    a.part = part; a.part_f32 = part_f32 ? 1 : 0; a.nparts = nparts; a.pstride = pstride;
    a.ts = reinterpret_cast<TailState*>(base);
    a.Y = reinterpret_cast<double*>(base + 256);
    a.HC = a.Y + ny;
    a.Bp = a.HC + ny;
    a.Hmat = Hmat; a.elag = elag; a.E = E;
    a.wc = dtile::wait_ctl(ctx);
    const int smem = (int)sizeof(double) * dtile::smem_doubles<TL_TN>();
    static std::atomic<unsigned long long> attr_mask{0};
    const unsigned long long bit = 1ull << (ctx->device & 63);
    if (!(attr_mask.load(std::memory_order_acquire) & bit)) {
        DONOF_CUDA(ctx, cudaFuncSetAttribute(elag_tail_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        attr_mask.fetch_or(bit, std::memory_order_acq_rel);
    }
    int per_sm = 0;
    DONOF_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, elag_tail_kernel, dtile::THREADS, smem));
    if (per_sm < 1) {
        set_error(ctx, "elag_tail_kernel does not fit on an SM");
        return DONOF_ERR_CUDA;
    }
    const int grid = ctx_ctas(ctx);  // at most one CTA per SM (co-resident: the kernel has grid barriers)
    DONOF_CUDA(ctx, cudaMemsetAsync(a.ts, 0, sizeof(TailState), st));
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
    DONOF_CUDA(ctx, cudaLaunchKernelEx(&cfg, elag_tail_kernel, a));
    count_launch();
    return DONOF_OK;
}

}  // namespace donof
