// Grouped orbital optimiser: a batch of jobs (molecules of different sizes,
// each with its own RI tensor b) runs the orbital loop of DoNOF.jl
// (orbopt_adam / _adabelief / _yogi / _demon, src/minimization.jl:242-630,
// iteration body :387-422) side by side, and every stage of a gradient step is
// ONE launch over all jobs of the batch:
//
//   update      grouped elementwise kernel (each job's own AMSGrad state)
//   rotation    grouped cooperative kernel (rotate.cu): job j on its own CTA range
//   T1, T2, Y   grouped persistent FP64 tensor-core GEMMs (gemm_f64.cuh) over a
//               work list that spans every job; one launch per tile shape in use,
//               the shapes picked per job by the batch's autotuner
//   W           grouped elementwise kernels (wbuild.cuh)
//   tail        grouped cooperative kernel (tail.cu): H_mat, elag, E_elec
//   gradient    grouped packing of 4(elag - elag^T) with max|g| per job
//   end, copy, commit   the reference's stopping rule and best-C bookkeeping
//
// The loop is one captured CUDA graph whose conditional WHILE node repeats the
// step until every job has stopped.  A job that has stopped is skipped by every
// launch (device-side gates), so each job takes exactly the iterations it
// takes alone.  Every product sums in the same order as the single-job FP64
// path: the same tile routine (the tile shape does not change the summation
// order), and for the Lagrangian GEMM the same split of its K range (the
// autotuner's entry for the job's shape).  A job's result is bit-for-bit what
// the single-job path gives it, whatever else the batch holds.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "kernels.cuh"
#include "orbupd.cuh"
#include "wbuild.cuh"

namespace donof {
namespace {

constexpr int CH = 1024;  // elements per work unit of the chunked elementwise kernels

struct BOrbState {
    double E, bestE, alpha, thresh;
    unsigned long long gmax_bits;  // max|g| of the latest gradient, as the bits of a non-negative double
    int it, maxloop, improved, improved_now, success, nit, stopped, stop_pending;
};

// Per-job view for the elementwise kernels.
struct BJob {
    int nbf, naux, nbf5, nalpha, nbeta, pad;
    long long nvar, nn;
    const double *n, *cj12, *ck12, *Cin;
    const double* bpq;
    double *W, *tv;
    double *m, *v, *vm, *y, *g;
    double *Ccur, *Cnew, *Cbest, *elag;
    BOrbState* S;
};

// job owning work unit u: the largest j with pre[j] <= u (pre[njobs] = total)
__device__ __forceinline__ int job_of(const int* __restrict__ pre, int njobs, int u) {
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (pre[mid] <= u) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ long long packed_row_start(int i, int nbf) {
    return (long long)i * (nbf - 1) - (long long)i * (i - 1) / 2;
}

__global__ void __launch_bounds__(256) b_update_kernel(const BJob* __restrict__ jobs, const int* __restrict__ pre,
                                                       int njobs, int method) {
    const int total = pre[njobs];
    for (int u = blockIdx.x; u < total; u += gridDim.x) {
        const int j = job_of(pre, njobs, u);
        const BJob& J = jobs[j];
        const BOrbState* s = J.S;
        if (s->stopped) continue;
        const orbupd::Coef c = orbupd::coef(method, s->it + 1, s->maxloop, s->alpha);
        const long long k0 = (long long)(u - pre[j]) * CH, k1 = min(J.nvar, k0 + CH);
        for (long long k = k0 + threadIdx.x; k < k1; k += blockDim.x) orbupd::step(c, k, J.g, J.m, J.v, J.vm, J.y);
        if (u == pre[j] && threadIdx.x == 0) J.S->gmax_bits = 0ull;  // the gradient of this step re-reduces it
    }
}

// g = 4 elag[i, j] - 4 elag[j, i] packed row-wise over i < nbf5, j > i
// (src/pnof.jl:1395-1403), max|g| per job.
__global__ void __launch_bounds__(256) b_pack_kernel(const BJob* __restrict__ jobs, const int* __restrict__ pre,
                                                     int njobs) {
    __shared__ double red[8];
    const int total = pre[njobs];
    for (int u = blockIdx.x; u < total; u += gridDim.x) {
        const int j = job_of(pre, njobs, u);
        const BJob& J = jobs[j];
        if (J.S->stopped) continue;
        const int nbf = J.nbf, nbf5 = J.nbf5;
        const long long k0 = (long long)(u - pre[j]) * CH, k1 = min(J.nvar, k0 + CH);
        double local = 0.0;
        for (long long k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
            int lo = 0, hi = nbf5 - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (packed_row_start(mid, nbf) <= k) lo = mid; else hi = mid - 1;
            }
            const int i = lo;
            const int c = (int)(k - packed_row_start(i, nbf)) + i + 1;
            const double v = 4.0 * J.elag[i + (long long)nbf * c] - 4.0 * J.elag[c + (long long)nbf * i];
            J.g[k] = v;
            local = fmax(local, fabs(v));
        }
        for (int o = 16; o > 0; o >>= 1) local = fmax(local, __shfl_xor_sync(0xffffffffu, local, o));
        __syncthreads();  // red of the previous unit is consumed
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = local;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t = fmax(t, red[w]);
            atomicMax(&J.S->gmax_bits, (unsigned long long)__double_as_longlong(t));
        }
    }
}

enum CopyMode { COPY_IN_TO_NEW = 0, COPY_NEW_TO_CUR_BEST = 1, COPY_LOOP_END = 2 };

// Orbital-matrix copies of every job (nbf x nbf each):
//   COPY_IN_TO_NEW        C_new <- C_in          (start of a call)
//   COPY_NEW_TO_CUR_BEST  C_cur, C_best <- C_new (after the first evaluation)
//   COPY_LOOP_END         C_best <- C_new if the energy improved; C_cur <- C_new
//                         (end of an iteration, for jobs still running)
__global__ void __launch_bounds__(256) b_copy_kernel(const BJob* __restrict__ jobs, const int* __restrict__ pre,
                                                     int njobs, int mode) {
    const int total = pre[njobs];
    for (int u = blockIdx.x; u < total; u += gridDim.x) {
        const int j = job_of(pre, njobs, u);
        const BJob& J = jobs[j];
        const long long k0 = (long long)(u - pre[j]) * CH, k1 = min(J.nn, k0 + CH);
        if (J.S->stopped) continue;  // jobs left out of the call, and jobs that have stopped
        if (mode == COPY_IN_TO_NEW) {
            for (long long k = k0 + threadIdx.x; k < k1; k += blockDim.x) J.Cnew[k] = J.Cin[k];
        } else if (mode == COPY_NEW_TO_CUR_BEST) {
            for (long long k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
                const double c = J.Cnew[k];
                J.Ccur[k] = c;
                J.Cbest[k] = c;
            }
        } else {
            const bool best = J.S->improved_now != 0;
            for (long long k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
                const double c = J.Cnew[k];
                if (best) J.Cbest[k] = c;
                J.Ccur[k] = c;
            }
        }
    }
}

__global__ void __launch_bounds__(256) b_wdiag_kernel(const BJob* __restrict__ jobs, const int* __restrict__ pre,
                                                      int njobs) {
    __shared__ double sd[wbuild::DIAG_SM];
    const int total = pre[njobs];
    for (int u = blockIdx.x; u < total; u += gridDim.x) {
        const int j = job_of(pre, njobs, u);
        const BJob& J = jobs[j];
        if (J.S->stopped) continue;
        wbuild::diag_unit(J.bpq, J.n, J.cj12, J.nbf5, J.naux, J.nalpha, J.nbeta, J.tv, u - pre[j], sd);
    }
}

__global__ void __launch_bounds__(256, 4) b_buildw_kernel(const BJob* __restrict__ jobs, const int* __restrict__ pre,
                                                       int njobs) {
    __shared__ double tb[wbuild::LT][32][33];
    const int total = pre[njobs];
    for (int u = blockIdx.x; u < total; u += gridDim.x) {
        const int j = job_of(pre, njobs, u);
        const BJob& J = jobs[j];
        if (J.S->stopped) continue;
        wbuild::tile(J.bpq, J.ck12, J.tv, J.nbf5, J.naux, J.W, u - pre[j], tb);
    }
}

// bestE = E of the first evaluation
__global__ void b_start_kernel(const BJob* __restrict__ jobs, int njobs) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < njobs; j += gridDim.x * blockDim.x) {
        BOrbState* s = jobs[j].S;
        s->bestE = s->E;
    }
}

// End of iteration it+1 of every running job: best-E tracking and the stopping
// rule the reference evaluates at the start of the next iteration
// (src/minimization.jl:387-422), as orb_end_kernel of the single-job loop.
__global__ void b_end_kernel(const BJob* __restrict__ jobs, int njobs) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < njobs; j += gridDim.x * blockDim.x) {
        BOrbState* s = jobs[j].S;
        if (s->stopped) continue;
        s->it += 1;
        const int i = s->it;
        const double E = s->E;
        int now = 0;
        if (E < s->bestE) {
            s->bestE = E;
            s->improved = 1;
            now = 1;
        }
        s->improved_now = now;
        const double gmax = __longlong_as_double((long long)s->gmax_bits);
        int stop = 0;
        if (i >= s->maxloop) {
            stop = 1;
            s->nit = i;
        } else if (2.0 * gmax < s->thresh && s->improved) {
            stop = 1;
            s->success = 1;
            s->nit = i + 1;
        }
        s->stop_pending = stop;
    }
}

// Jobs that met their stopping rule leave the loop; the WHILE condition stays
// set while any job is running.  One block.
__global__ void b_commit_kernel(const BJob* __restrict__ jobs, int njobs, cudaGraphConditionalHandle h) {
    int running = 0;
    for (int j = threadIdx.x; j < njobs; j += blockDim.x) {
        BOrbState* s = jobs[j].S;
        if (s->stop_pending) s->stopped = 1;
        running |= (s->stopped == 0);
    }
    running = __syncthreads_or(running);
    if (threadIdx.x == 0) cudaGraphSetConditional(h, running ? 1u : 0u);
}

size_t al32(size_t doubles) { return (doubles + 31) / 32 * 32; }  // 256-byte segments

// Heuristic tile shape of an M x N output: the largest tile that the output fills.
GemmTile heuristic_tile(int M, int N) {
    if (M >= 128 && N >= 48) return GemmTile::Large;
    if (M >= 48 && N >= 48) return GemmTile::Small;
    return GemmTile::Tiny;
}

enum Stage { ST_T1 = 0, ST_T2 = 1, ST_Y = 2, NSTAGE = 3 };
constexpr int NTILE = 4;  // tile shapes a stage's launch list can hold (GemmTile values)

}  // namespace
}  // namespace donof

using namespace donof;

struct donof_batch {
    donof_ctx* ctx = nullptr;
    int nj = 0;
    struct Shape {
        donof_job* job;       // the job bound to the slot (not dereferenced once bound: it may be freed)
        const double* b;      // its RI tensor, read by T1 while the slot runs
        int nbf, naux, nbf5, nalpha, nbeta;
        long long nvar, nn;
        int splits, kchunk;
    };
    std::vector<Shape> sh;
    // per-job arena pointers (device)
    struct Ptrs {
        double *tmp, *bpq, *W, *tv, *ypart, *twork, *rwork;
        double *m, *v, *vm, *y, *g, *Ccur, *Cnew, *Cbest, *elag, *Hmat;
    };
    std::vector<Ptrs> pt;
    DevBuf arena, tab, ypbuf;  // ypbuf: the split-K partials of the Lagrangian GEMM
    double* mvv = nullptr;  // m, v, vmax of every job (one contiguous span)
    size_t mvv_doubles = 0;
    // device table addresses
    BJob* d_jobs = nullptr;
    RotJob* d_rot = nullptr;
    TailJob* d_tail = nullptr;
    GemmF64Args* d_gemm[NSTAGE] = {};
    int* d_start[NSTAGE] = {};
    int* d_pre[4] = {};  // units of: nvar chunks, nn chunks, W diagonal groups, build_w tiles
    void* d_rstate = nullptr;
    void* d_tstate = nullptr;
    BOrbState* d_state = nullptr;
    int pre_total[4] = {};
    int rot_grid = 1, tail_grid = 1;
    // tile shape per stage and job, and the launch list it gives
    std::vector<GemmTile> tile[NSTAGE];
    struct Launch {
        GemmTile tile;
        bool ak, bk, vec;
        int args_off, start_off, ngroups, total;
    };
    std::vector<Launch> launches[NSTAGE];
    bool tuned = false;
    // mixed form (donof_batch_set_precision): the fused tcgen05 kernel over every job
    int precision = DONOF_PREC_FP64;
    DevBuf mix;                          // per job: Cs, n32, cj32, ck32, Y partials; the split table
    std::vector<MixedGroupJob> mjobs;
    MixedSplitJob* d_split = nullptr;
    int max_ldk = 0;
    // captured loop
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int graph_method = -1, graph_ctas = -1;
    int per_iter = 0;
};

namespace {

void stage_layout(int s, bool* ak, bool* bk) {
    // T1: A = b (M-contiguous), B = C K-major; T2: A = C^T (K-major), B = tmp K-major;
    // Y: A = tmp (M-contiguous), B = W K-major.
    *ak = (s == ST_T2);
    *bk = true;
}

GemmF64Args stage_args(const donof_batch* B, int s, int j) {
    const donof_batch::Shape& h = B->sh[j];
    const donof_batch::Ptrs& p = B->pt[j];
    GemmF64Args a{};
    if (s == ST_T1) {  // tmp_l(m, q) = sum_n b[m, n, l] C[n, q]
        a.M = h.nbf; a.N = h.nbf5; a.K = h.nbf;
        a.A = h.b; a.lda = h.nbf; a.strideA = (long long)h.nbf * h.nbf;
        a.B = p.Cnew; a.ldb = h.nbf; a.strideB = 0;
        a.C = p.tmp; a.ldc = h.nbf; a.strideC = (long long)h.nbf * h.nbf5;
        a.batch = h.naux; a.splits = 1; a.kchunk = h.nbf;
    } else if (s == ST_T2) {  // bpq_l(p, q) = sum_m C[m, p] tmp_l[m, q]
        a.M = h.nbf5; a.N = h.nbf5; a.K = h.nbf;
        a.A = p.Cnew; a.lda = h.nbf; a.strideA = 0;
        a.B = p.tmp; a.ldb = h.nbf; a.strideB = (long long)h.nbf * h.nbf5;
        a.C = p.bpq; a.ldc = h.nbf5; a.strideC = (long long)h.nbf5 * h.nbf5;
        a.batch = h.naux; a.splits = 1; a.kchunk = h.nbf;
    } else {  // Y = sum_{q,l} tmp[m, q + nbf5 l] W[q + nbf5 l, b], split-K partials
        const long long Kt = (long long)h.nbf5 * h.naux;
        a.M = h.nbf; a.N = h.nbf5; a.K = (int)Kt;
        a.A = p.tmp; a.lda = h.nbf; a.strideA = 0;
        a.B = p.W; a.ldb = Kt; a.strideB = 0;
        a.C = p.ypart; a.ldc = h.nbf; a.strideC = 0;
        a.batch = 1; a.splits = h.splits; a.kchunk = h.kchunk;
        a.strideSplit = (long long)h.nbf * h.nbf5;
    }
    a.alpha = 1.0;
    a.beta = 0.0;
    a.skip_nz = &B->d_state[j].stopped;
    return a;
}

// Host images of the GEMM tables for the current tile choice: per stage the
// args grouped by tile shape (largest K first within a shape) and each shape's
// start array; uploaded to the device tables.
int upload_gemm_tables(donof_batch* B, cudaStream_t st) {
    donof_ctx* ctx = B->ctx;
    for (int s = 0; s < NSTAGE; ++s) {
        bool ak, bk;
        stage_layout(s, &ak, &bk);
        std::vector<GemmF64Args> args;
        std::vector<int> starts;
        B->launches[s].clear();
        const GemmTile order[NTILE] = {GemmTile::Large, GemmTile::SmallW8, GemmTile::Small, GemmTile::Tiny};
        for (GemmTile t : order) {
            std::vector<int> js;
            for (int j = 0; j < B->nj; ++j)
                if (B->tile[s][j] == t) js.push_back(j);
            if (js.empty()) continue;
            std::vector<GemmF64Args> ga;
            for (int j : js) ga.push_back(stage_args(B, s, j));
            std::stable_sort(ga.begin(), ga.end(), [](const GemmF64Args& x, const GemmF64Args& y) {
                const int kx = x.splits > 1 ? x.kchunk : x.K, ky = y.splits > 1 ? y.kchunk : y.K;
                return kx > ky;
            });
            donof_batch::Launch L{};
            L.tile = t; L.ak = ak; L.bk = bk; L.vec = true;
            L.args_off = (int)args.size();
            L.start_off = (int)starts.size();
            L.ngroups = (int)ga.size();
            int acc = 0;
            for (const GemmF64Args& a : ga) {
                starts.push_back(acc);
                acc += gemm_f64_tiles(a, t);
                L.vec = L.vec && gemm_f64_vec_ok(ak, bk, a);
                args.push_back(a);
            }
            starts.push_back(acc);
            L.total = acc;
            B->launches[s].push_back(L);
        }
        DONOF_CUDA(ctx, cudaMemcpyAsync(B->d_gemm[s], args.data(), sizeof(GemmF64Args) * args.size(),
                                        cudaMemcpyHostToDevice, st));
        DONOF_CUDA(ctx, cudaMemcpyAsync(B->d_start[s], starts.data(), sizeof(int) * starts.size(),
                                        cudaMemcpyHostToDevice, st));
    }
    return DONOF_OK;
}

int run_stage(donof_batch* B, cudaStream_t st, int s) {
    donof_ctx* ctx = B->ctx;
    const int max_ctas = ctx->cta_limit > 0 ? ctx->cta_limit : 0;
    for (const donof_batch::Launch& L : B->launches[s])
        DONOF_CHECK(gemm_f64_grouped(ctx, st, L.ak, L.bk, L.vec, L.tile, B->d_gemm[s] + L.args_off,
                                     B->d_start[s] + L.start_off, L.ngroups, L.total, max_ctas));
    return DONOF_OK;
}

int grid_units(int total, int per_sm, int sm) {
    long long g = total;
    if (g > (long long)per_sm * sm) g = (long long)per_sm * sm;
    return (int)(g < 1 ? 1 : g);
}

// The Lagrangian of every running job at C_new: T1, T2, W, Y, tail (energy into the job state).
int lagrangian(donof_batch* B, cudaStream_t st) {
    donof_ctx* ctx = B->ctx;
    if (B->precision == DONOF_PREC_MIXED) {
        // every job's fused T1, T2, W, Y on its CTA range (bf16 split products, FP32 Y
        // partials), then the grouped FP64 tail on those partials
        DONOF_CHECK(split_c_grouped(ctx, st, B->d_split, B->nj, B->max_ldk));
        DONOF_CHECK(launch_mixed_grouped(ctx, st, B->mjobs.data(), B->nj));
        return tail_grouped(ctx, st, B->d_tail, B->nj, B->d_tstate, B->tail_grid);
    }
    DONOF_CHECK(run_stage(B, st, ST_T1));
    DONOF_CHECK(run_stage(B, st, ST_T2));
    b_wdiag_kernel<<<grid_units(B->pre_total[2], 4, ctx->sm_count), 256, 0, st>>>(B->d_jobs, B->d_pre[2], B->nj);
    count_launch();
    b_buildw_kernel<<<grid_units(B->pre_total[3], 16, ctx->sm_count), 256, 0, st>>>(B->d_jobs, B->d_pre[3], B->nj);
    count_launch();
    DONOF_CUDA(ctx, cudaGetLastError());
    DONOF_CHECK(run_stage(B, st, ST_Y));
    return tail_grouped(ctx, st, B->d_tail, B->nj, B->d_tstate, B->tail_grid);
}

int gradient(donof_batch* B, cudaStream_t st) {
    b_pack_kernel<<<grid_units(B->pre_total[0], 4, B->ctx->sm_count), 256, 0, st>>>(B->d_jobs, B->d_pre[0], B->nj);
    count_launch();
    DONOF_CUDA(B->ctx, cudaGetLastError());
    return DONOF_OK;
}

// CTA ranges of the grouped cooperative kernels: one CTA per job, the rest of
// the grid in proportion to the job's work (at most cap_j each).  More jobs
// than CTAs: one CTA each, job j on CTA j mod grid.
int assign_ctas(const std::vector<double>& w, const std::vector<int>& cap, int G, std::vector<int>* c0,
                std::vector<int>* cn) {
    const int nj = (int)w.size();
    c0->assign(nj, 0);
    cn->assign(nj, 1);
    if (nj > G) {
        for (int j = 0; j < nj; ++j) (*c0)[j] = j % G;
        return G;
    }
    double tw = 0.0;
    for (double x : w) tw += x;
    const int rem = G - nj;
    for (int j = 0; j < nj && tw > 0.0; ++j) {
        int extra = (int)floor(rem * w[j] / tw);
        if (extra > cap[j] - 1) extra = cap[j] - 1;
        if (extra < 0) extra = 0;
        (*cn)[j] += extra;
    }
    int acc = 0;
    for (int j = 0; j < nj; ++j) {
        (*c0)[j] = acc;
        acc += (*cn)[j];
    }
    return acc;
}

int upload_call_tables(donof_batch* B, cudaStream_t st, const donof_batch_item* items,
                       const std::vector<BOrbState>& states, bool with_states) {
    donof_ctx* ctx = B->ctx;
    const int nj = B->nj;
    std::vector<BJob> bj(nj);
    std::vector<TailJob> tj(nj);
    std::vector<RotJob> rj(nj);
    std::vector<double> wr(nj), wt(nj);
    std::vector<int> capr(nj), capt(nj);
    for (int j = 0; j < nj; ++j) {
        const donof_batch::Shape& h = B->sh[j];
        wr[j] = (double)h.nbf * h.nbf * h.nbf;
        wt[j] = (double)h.nbf * h.nbf * h.nbf5 + (double)h.splits * h.nbf * h.nbf5;
        capr[j] = 2 * ((h.nbf + 31) / 32) * ((h.nbf + 15) / 16);
        capt[j] = 2 * ((h.nbf + 31) / 32) * ((h.nbf5 + 15) / 16);
    }
    const int G = ctx_ctas(ctx);
    std::vector<int> r0, rn, t0, tn;
    B->rot_grid = assign_ctas(wr, capr, G, &r0, &rn);
    B->tail_grid = assign_ctas(wt, capt, G, &t0, &tn);
    for (int j = 0; j < nj; ++j) {
        const donof_batch::Shape& h = B->sh[j];
        const donof_batch::Ptrs& p = B->pt[j];
        const donof_batch_item& it = items[j];
        BJob& J = bj[j];
        J.nbf = h.nbf; J.naux = h.naux; J.nbf5 = h.nbf5; J.nalpha = h.nalpha; J.nbeta = h.nbeta;
        J.nvar = h.nvar; J.nn = h.nn;
        J.n = it.n; J.cj12 = it.cj12; J.ck12 = it.ck12; J.Cin = it.C;
        J.bpq = p.bpq; J.W = p.W; J.tv = p.tv;
        J.m = p.m; J.v = p.v; J.vm = p.vm; J.y = p.y; J.g = p.g;
        J.Ccur = p.Ccur; J.Cnew = p.Cnew; J.Cbest = p.Cbest; J.elag = p.elag;
        J.S = B->d_state + j;
        RotJob& R = rj[j];
        R.y = p.y; R.C = p.Ccur; R.Cnew = p.Cnew; R.work = p.rwork;
        R.state = static_cast<char*>(B->d_rstate) + (size_t)GROUP_STATE_BYTES * j;
        R.skip = &B->d_state[j].stopped;
        R.nbf = h.nbf; R.nbf5 = h.nbf5; R.cta0 = r0[j]; R.ctas = rn[j];
        TailJob& T = tj[j];
        T.C = p.Cnew; T.H = it.H; T.n = it.n;
        T.part = p.ypart; T.pstride = (long long)h.nbf * h.nbf5;
        T.Hmat = p.Hmat; T.elag = p.elag; T.E = &B->d_state[j].E;
        T.work = p.twork;
        T.state = static_cast<char*>(B->d_tstate) + (size_t)GROUP_STATE_BYTES * j;
        T.skip = &B->d_state[j].stopped;
        T.nbf = h.nbf; T.nbf5 = h.nbf5; T.part_f32 = 0; T.nparts = h.splits; T.cta0 = t0[j]; T.ctas = tn[j];
        if (B->precision == DONOF_PREC_MIXED) {
            T.part = B->mjobs[j].ypart;
            T.part_f32 = 1;
            T.nparts = B->mjobs[j].ctas;
        }
    }
    DONOF_CUDA(ctx, cudaMemcpyAsync(B->d_jobs, bj.data(), sizeof(BJob) * nj, cudaMemcpyHostToDevice, st));
    DONOF_CUDA(ctx, cudaMemcpyAsync(B->d_rot, rj.data(), sizeof(RotJob) * nj, cudaMemcpyHostToDevice, st));
    DONOF_CUDA(ctx, cudaMemcpyAsync(B->d_tail, tj.data(), sizeof(TailJob) * nj, cudaMemcpyHostToDevice, st));
    if (with_states)
        DONOF_CUDA(ctx, cudaMemcpyAsync(B->d_state, states.data(), sizeof(BOrbState) * nj, cudaMemcpyHostToDevice,
                                        st));
    return DONOF_OK;
}

// The batch's own tile autotuner: for each grouped GEMM stage, times the launch
// list of five candidate assignments (the per-job heuristic, all 128 x 64, all
// 64 x 64, all 32 x 32, all 64 x 64 over 8 warps) on the batch's operands with
// CUDA events (one warm-up and two timed runs each) and keeps the fastest.  Every candidate
// writes the same result (the tile shape does not change any summation order).
int autotune(donof_batch* B, cudaStream_t st) {
    donof_ctx* ctx = B->ctx;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    DONOF_CUDA(ctx, cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        set_error(ctx, "batch autotune: cudaEventCreate failed");
        return DONOF_ERR_CUDA;
    }
    int rc = DONOF_OK;
    std::vector<GemmTile> best[NSTAGE];
    for (int s = 0; s < NSTAGE && rc == DONOF_OK; ++s) {
        float best_ms = -1.f;
        for (int c = 0; c < 5 && rc == DONOF_OK; ++c) {
            for (int j = 0; j < B->nj; ++j) {
                const donof_batch::Shape& h = B->sh[j];
                const int M = (s == ST_T2) ? h.nbf5 : h.nbf;
                const GemmTile cand[5] = {heuristic_tile(M, h.nbf5), GemmTile::Large, GemmTile::Small, GemmTile::Tiny,
                                          GemmTile::SmallW8};
                B->tile[s][j] = cand[c];
            }
            if ((rc = upload_gemm_tables(B, st)) != DONOF_OK) break;
            if ((rc = run_stage(B, st, s)) != DONOF_OK) break;
            cudaEventRecord(e0, st);
            if ((rc = run_stage(B, st, s)) != DONOF_OK) break;
            if ((rc = run_stage(B, st, s)) != DONOF_OK) break;
            cudaEventRecord(e1, st);
            if (cudaEventSynchronize(e1) != cudaSuccess) {
                set_error(ctx, "batch autotune: %s", cudaGetErrorString(cudaGetLastError()));
                rc = DONOF_ERR_CUDA;
                break;
            }
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (best_ms < 0.f || ms < best_ms) {
                best_ms = ms;
                best[s] = B->tile[s];
            }
        }
        // later stages are timed with this stage at its heuristic choice
        for (int j = 0; j < B->nj && rc == DONOF_OK; ++j) {
            const donof_batch::Shape& h = B->sh[j];
            B->tile[s][j] = heuristic_tile((s == ST_T2) ? h.nbf5 : h.nbf, h.nbf5);
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc != DONOF_OK) return rc;
    for (int s = 0; s < NSTAGE; ++s) B->tile[s] = best[s];
    DONOF_CHECK(upload_gemm_tables(B, st));
    B->tuned = true;
    return DONOF_OK;
}

int check_items(donof_batch* B, const donof_batch_item* items, bool orbopt) {
    donof_ctx* ctx = B->ctx;
    for (int j = 0; j < B->nj; ++j) {
        const donof_batch_item& it = items[j];
        if (!it.n || !it.cj12 || !it.ck12 || !it.H || !it.C) {
            set_error(ctx, "batch item %d: null device pointer", j);
            return DONOF_ERR_ARG;
        }
        if (orbopt && it.maxloop < 0) {
            set_error(ctx, "batch item %d: maxloop must be >= 0", j);
            return DONOF_ERR_ARG;
        }
    }
    return DONOF_OK;
}

cudaStream_t batch_stream(donof_batch* B) {
    donof_ctx* ctx = B->ctx;
    cudaStream_t st = ctx->stream;
    if (st == nullptr || st == cudaStreamLegacy) {
        // the legacy default stream cannot be captured: run on a private stream,
        // ordered after the work already queued
        if (!ctx->aux_stream && cudaStreamCreateWithFlags(&ctx->aux_stream, cudaStreamNonBlocking) != cudaSuccess)
            return nullptr;
        if (cudaStreamSynchronize(st) != cudaSuccess) return nullptr;
        st = ctx->aux_stream;
    }
    return st;
}

// Start of a call: inputs, optimiser state, first evaluation at C_in.
int start_call(donof_batch* B, cudaStream_t st, const donof_batch_item* items, const std::vector<BOrbState>& hs) {
    donof_ctx* ctx = B->ctx;
    DONOF_CHECK(upload_call_tables(B, st, items, hs, true));
    if (!B->tuned) DONOF_CHECK(autotune(B, st));
    if (B->precision == DONOF_PREC_MIXED)
        for (int j = 0; j < B->nj; ++j) {
            MixedGroupJob& g = B->mjobs[j];
            DONOF_CHECK(prep_coef(B->ctx, st, items[j].n, items[j].cj12, items[j].ck12, g.nbf5,
                                  const_cast<float*>(g.n32), const_cast<float*>(g.cj32), const_cast<float*>(g.ck32)));
        }
    DONOF_CUDA(ctx, cudaMemsetAsync(B->mvv, 0, sizeof(double) * B->mvv_doubles, st));
    b_copy_kernel<<<grid_units(B->pre_total[1], 4, ctx->sm_count), 256, 0, st>>>(B->d_jobs, B->d_pre[1], B->nj,
                                                                               COPY_IN_TO_NEW);
    count_launch();
    DONOF_CUDA(ctx, cudaGetLastError());
    DONOF_CHECK(lagrangian(B, st));
    return DONOF_OK;
}

}  // namespace

extern "C" {

int donof_batch_create(donof_ctx* ctx, int count, const donof_batch_shape* shapes, donof_batch** out) {
    if (!ctx || !out) return DONOF_ERR_ARG;
    *out = nullptr;
    if (count <= 0 || !shapes) {
        set_error(ctx, "donof_batch_create: count must be > 0 and shapes non-null");
        return DONOF_ERR_ARG;
    }
    for (int j = 0; j < count; ++j) {
        const donof_batch_shape& s = shapes[j];
        if (!s.job || s.job->ctx == nullptr || s.job->ctx->device != ctx->device) {
            set_error(ctx, "donof_batch_create: shape %d has no job on this context's device", j);
            return DONOF_ERR_ARG;
        }
        if (s.job->b == nullptr) {
            set_error(ctx, "donof_batch_create: shape %d: the job holds no FP64 RI tensor", j);
            return DONOF_ERR_ARG;
        }
        const int nbf = s.job->nbf;
        if (s.nbf5 <= 0 || s.nbf5 > nbf || s.nbeta < 0 || s.nalpha < s.nbeta || s.nalpha > s.nbf5) {
            set_error(ctx, "donof_batch_create: shape %d has invalid sizes nbf=%d nbf5=%d nalpha=%d nbeta=%d", j, nbf,
                      s.nbf5, s.nalpha, s.nbeta);
            return DONOF_ERR_ARG;
        }
        if ((long long)s.nbf5 * s.job->naux > 0x7fffffffLL) {
            set_error(ctx, "donof_batch_create: shape %d: nbf5 * naux exceeds the 32-bit GEMM extent", j);
            return DONOF_ERR_ARG;
        }
    }
    if (cudaSetDevice(ctx->device) != cudaSuccess) {
        set_error(ctx, "donof_batch_create: cudaSetDevice(%d) failed", ctx->device);
        return DONOF_ERR_CUDA;
    }
    donof_batch* B = new (std::nothrow) donof_batch();
    if (!B) return DONOF_ERR_OOM;
    B->ctx = ctx;
    B->nj = count;
    B->sh.resize(count);
    B->pt.resize(count);
    for (int j = 0; j < count; ++j) {
        donof_batch::Shape& h = B->sh[j];
        h.job = shapes[j].job;
        h.b = h.job->b;
        h.nbf = h.job->nbf; h.naux = h.job->naux; h.nbf5 = shapes[j].nbf5;
        h.nalpha = shapes[j].nalpha; h.nbeta = shapes[j].nbeta;
        h.nvar = nvar_of(h.nbf, h.nbf5);
        h.nn = (long long)h.nbf * h.nbf;
        h.splits = 1;  // set below, once the operands exist
        h.kchunk = h.nbf5 * h.naux;
    }
    // arena: per-field spans, so that m, v and vmax of every job form one block
    std::vector<size_t> off_tmp(count), off_bpq(count), off_W(count), off_tv(count), off_yp(count), off_tw(count),
        off_rw(count), off_m(count), off_v(count), off_vm(count), off_y(count), off_g(count), off_Cc(count),
        off_Cn(count), off_Cb(count), off_el(count), off_Hm(count);
    size_t acc = 0;
    auto field = [&](std::vector<size_t>& off, auto size_of) {
        for (int j = 0; j < count; ++j) {
            off[j] = acc;
            acc += al32(size_of(B->sh[j]));
        }
    };
    using S = donof_batch::Shape;
    field(off_m, [](const S& h) { return (size_t)h.nvar; });
    field(off_v, [](const S& h) { return (size_t)h.nvar; });
    field(off_vm, [](const S& h) { return (size_t)h.nvar; });
    const size_t mvv_end = acc;
    field(off_y, [](const S& h) { return (size_t)h.nvar; });
    field(off_g, [](const S& h) { return (size_t)h.nvar; });
    field(off_Cc, [](const S& h) { return (size_t)h.nn; });
    field(off_Cn, [](const S& h) { return (size_t)h.nn; });
    field(off_Cb, [](const S& h) { return (size_t)h.nn; });
    field(off_el, [](const S& h) { return (size_t)h.nn; });
    field(off_Hm, [](const S& h) { return (size_t)h.nbf * h.nbf5; });
    field(off_tmp, [](const S& h) { return (size_t)h.nbf * h.nbf5 * h.naux; });
    field(off_bpq, [](const S& h) { return (size_t)h.nbf5 * h.nbf5 * h.naux; });
    field(off_W, [](const S& h) { return (size_t)h.nbf5 * h.nbf5 * h.naux; });
    field(off_tv, [](const S& h) { return (size_t)h.nbf5 * h.naux; });
    field(off_tw, [](const S& h) { return (size_t)3 * h.nbf * h.nbf5; });
    field(off_rw, [](const S& h) { return rotate_work_doubles(h.nbf); });
    int rc = B->arena.ensure(ctx, sizeof(double) * acc);
    if (rc != DONOF_OK) {
        delete B;
        return rc;
    }
    double* base = B->arena.as<double>();
    B->mvv = base;
    B->mvv_doubles = mvv_end;
    for (int j = 0; j < count; ++j) {
        donof_batch::Ptrs& p = B->pt[j];
        p.m = base + off_m[j]; p.v = base + off_v[j]; p.vm = base + off_vm[j];
        p.y = base + off_y[j]; p.g = base + off_g[j];
        p.Ccur = base + off_Cc[j]; p.Cnew = base + off_Cn[j]; p.Cbest = base + off_Cb[j]; p.elag = base + off_el[j];
        p.Hmat = base + off_Hm[j];
        p.tmp = base + off_tmp[j]; p.bpq = base + off_bpq[j]; p.W = base + off_W[j]; p.tv = base + off_tv[j];
        p.twork = base + off_tw[j]; p.rwork = base + off_rw[j];
    }
    // Split of each job's Lagrangian GEMM (K = nbf5 naux): the one the single-job
    // FP64 path uses for that shape (the process's autotuner entry, timed now on
    // the batch's operands if there is none yet), so that a job sums in the same
    // order in a batch and alone.  Then the partials' storage.
    {
        DevBuf scratch;
        size_t yp = 0;
        std::vector<size_t> off_yp(count);
        for (int j = 0; j < count && rc == DONOF_OK; ++j) {
            S& h = B->sh[j];
            const long long Kt = (long long)h.nbf5 * h.naux;
            rc = gemm_f64_partials_splits(ctx, ctx->stream, false, true, h.nbf, h.nbf5, (int)Kt, B->pt[j].tmp, h.nbf,
                                          B->pt[j].W, Kt, &scratch, &h.splits, &h.kchunk);
            off_yp[j] = yp;
            yp += al32((size_t)h.splits * h.nbf * h.nbf5);
        }
        scratch.release(ctx);
        if (rc == DONOF_OK) rc = B->ypbuf.ensure(ctx, sizeof(double) * yp);
        if (rc != DONOF_OK) {
            B->ypbuf.release(ctx);
            B->arena.release(ctx);
            delete B;
            return rc;
        }
        for (int j = 0; j < count; ++j) B->pt[j].ypart = B->ypbuf.as<double>() + off_yp[j];
    }
    // device tables
    size_t tb = 0;
    auto take = [&](size_t bytes) { size_t o = tb; tb += (bytes + 255) / 256 * 256; return o; };
    const size_t o_jobs = take(sizeof(BJob) * count), o_rot = take(sizeof(RotJob) * count),
                 o_tail = take(sizeof(TailJob) * count), o_state = take(sizeof(BOrbState) * count),
                 o_rs = take((size_t)GROUP_STATE_BYTES * count), o_ts = take((size_t)GROUP_STATE_BYTES * count);
    size_t o_gemm[NSTAGE], o_start[NSTAGE], o_pre[4];
    for (int s = 0; s < NSTAGE; ++s) {
        o_gemm[s] = take(sizeof(GemmF64Args) * count);
        o_start[s] = take(sizeof(int) * (count + NTILE));  // one start array of n_k + 1 entries per tile shape
    }
    for (int k = 0; k < 4; ++k) o_pre[k] = take(sizeof(int) * (count + 1));
    rc = B->tab.ensure(ctx, tb);
    if (rc != DONOF_OK) {
        B->ypbuf.release(ctx);
        B->arena.release(ctx);
        delete B;
        return rc;
    }
    char* t = B->tab.as<char>();
    B->d_jobs = reinterpret_cast<BJob*>(t + o_jobs);
    B->d_rot = reinterpret_cast<RotJob*>(t + o_rot);
    B->d_tail = reinterpret_cast<TailJob*>(t + o_tail);
    B->d_state = reinterpret_cast<BOrbState*>(t + o_state);
    B->d_rstate = t + o_rs;
    B->d_tstate = t + o_ts;
    for (int s = 0; s < NSTAGE; ++s) {
        B->d_gemm[s] = reinterpret_cast<GemmF64Args*>(t + o_gemm[s]);
        B->d_start[s] = reinterpret_cast<int*>(t + o_start[s]);
    }
    for (int k = 0; k < 4; ++k) B->d_pre[k] = reinterpret_cast<int*>(t + o_pre[k]);
    // work-unit prefixes of the elementwise kernels
    std::vector<int> pre[4];
    for (int k = 0; k < 4; ++k) pre[k].assign(count + 1, 0);
    for (int j = 0; j < count; ++j) {
        const S& h = B->sh[j];
        const long long u[4] = {(h.nvar + CH - 1) / CH, (h.nn + CH - 1) / CH,
                                wbuild::diag_units(h.nbf5, h.naux), wbuild::tiles(h.nbf5, h.naux)};
        for (int k = 0; k < 4; ++k) {
            const long long v = pre[k][j] + u[k];
            if (v > 0x7fffffffLL) {
                set_error(ctx, "donof_batch_create: too much work for one batch");
                B->tab.release(ctx);
                B->ypbuf.release(ctx);
                B->arena.release(ctx);
                delete B;
                return DONOF_ERR_ARG;
            }
            pre[k][j + 1] = (int)v;
        }
    }
    for (int k = 0; k < 4; ++k) {
        B->pre_total[k] = pre[k][count];
        if (cudaMemcpyAsync(B->d_pre[k], pre[k].data(), sizeof(int) * (count + 1), cudaMemcpyHostToDevice,
                            ctx->stream) != cudaSuccess) {
            set_error(ctx, "donof_batch_create: upload of the work tables failed");
            B->tab.release(ctx);
            B->ypbuf.release(ctx);
            B->arena.release(ctx);
            delete B;
            return DONOF_ERR_CUDA;
        }
    }
    for (int s = 0; s < NSTAGE; ++s) {
        B->tile[s].resize(count);
        for (int j = 0; j < count; ++j) {
            const S& h = B->sh[j];
            B->tile[s][j] = heuristic_tile((s == ST_T2) ? h.nbf5 : h.nbf, h.nbf5);
        }
    }
    rc = upload_gemm_tables(B, ctx->stream);
    if (rc == DONOF_OK && cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
        set_error(ctx, "donof_batch_create: %s", cudaGetErrorString(cudaGetLastError()));
        rc = DONOF_ERR_CUDA;
    }
    if (rc != DONOF_OK) {
        B->tab.release(ctx);
        B->ypbuf.release(ctx);
        B->arena.release(ctx);
        delete B;
        return rc;
    }
    *out = B;
    return DONOF_OK;
}

int donof_batch_set_precision(donof_batch* B, int precision) {
    if (!B) return DONOF_ERR_ARG;
    donof_ctx* ctx = B->ctx;
    if (precision == DONOF_PREC_FP64) {
        B->precision = precision;
        B->graph_method = -1;  // the captured loop is taken again
        return DONOF_OK;
    }
    if (precision != DONOF_PREC_MIXED) {
        set_error(ctx, "donof_batch_set_precision: unknown precision %d", precision);
        return DONOF_ERR_ARG;
    }
    const int nj = B->nj;
    for (int j = 0; j < nj; ++j) {
        const donof_batch::Shape& h = B->sh[j];
        if (h.job->b16hi == nullptr) {
            set_error(ctx, "donof_batch_set_precision: job %d holds no bf16 split of b (upload it as mixed)", j);
            return DONOF_ERR_ARG;
        }
        if (!mixed_fused_fits(h.nbf, h.nbf5)) {
            set_error(ctx, "donof_batch_set_precision: job %d (nbf %d, nbf5 %d) exceeds the fused mixed kernel "
                           "(nbf <= 256, nbf5 <= 64)", j, h.nbf, h.nbf5);
            return DONOF_ERR_ARG;
        }
    }
    DONOF_CUDA(ctx, cudaSetDevice(ctx->device));
    // CTAs per job in proportion to its b (nbf^2 naux), at least one, about one wave in all
    std::vector<double> w(nj);
    double wsum = 0.0;
    for (int j = 0; j < nj; ++j) wsum += (w[j] = (double)B->sh[j].nbf * B->sh[j].nbf * B->sh[j].naux);
    const int G = ctx_ctas(ctx) > nj ? ctx_ctas(ctx) : nj;
    std::vector<int> ctas(nj);
    for (int j = 0; j < nj; ++j) {
        int c = (int)(w[j] / wsum * (G - nj)) + 1;
        if (c > B->sh[j].naux) c = B->sh[j].naux;
        ctas[j] = c;
    }
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o = off; off += (bytes + 255) / 256 * 256; return o; };
    std::vector<size_t> o_cs(nj), o_n(nj), o_cj(nj), o_ck(nj), o_y(nj);
    int max_ldk = 0;
    for (int j = 0; j < nj; ++j) {
        const donof_batch::Shape& h = B->sh[j];
        const int ldk = mixed_ldk(h.nbf);
        if (ldk > max_ldk) max_ldk = ldk;
        o_cs[j] = take(2 * (size_t)ldk * 128);
        o_n[j] = take(sizeof(float) * 64);
        o_cj[j] = take(sizeof(float) * 64 * 64);
        o_ck[j] = take(sizeof(float) * 64 * 64);
        o_y[j] = take(sizeof(float) * (size_t)ctas[j] * h.nbf * h.nbf5);
    }
    const size_t o_split = take(sizeof(MixedSplitJob) * nj);
    DONOF_CHECK(B->mix.ensure(ctx, off));
    char* base = B->mix.as<char>();
    B->mjobs.resize(nj);
    std::vector<MixedSplitJob> sj(nj);
    for (int j = 0; j < nj; ++j) {
        const donof_batch::Shape& h = B->sh[j];
        MixedGroupJob& g = B->mjobs[j];
        g.job = h.job;
        g.nbf5 = h.nbf5; g.nalpha = h.nalpha; g.nbeta = h.nbeta; g.ctas = ctas[j];
        g.cs = base + o_cs[j];
        g.n32 = reinterpret_cast<float*>(base + o_n[j]);
        g.cj32 = reinterpret_cast<float*>(base + o_cj[j]);
        g.ck32 = reinterpret_cast<float*>(base + o_ck[j]);
        g.ypart = reinterpret_cast<float*>(base + o_y[j]);
        sj[j] = MixedSplitJob{B->pt[j].Cnew, g.cs, h.nbf, h.nbf5, mixed_ldk(h.nbf), 0};
    }
    B->d_split = reinterpret_cast<MixedSplitJob*>(base + o_split);
    B->max_ldk = max_ldk;
    DONOF_CUDA(ctx, cudaMemcpyAsync(B->d_split, sj.data(), sizeof(MixedSplitJob) * nj, cudaMemcpyHostToDevice,
                                    ctx->stream));
    DONOF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    B->precision = precision;
    B->graph_method = -1;  // the captured loop is taken again
    return DONOF_OK;
}

int donof_batch_destroy(donof_batch* B) {
    if (!B) return DONOF_OK;
    donof_ctx* ctx = B->ctx;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    if (ctx->aux_stream) cudaStreamSynchronize(ctx->aux_stream);
    if (B->exec) cudaGraphExecDestroy(B->exec);
    if (B->graph) cudaGraphDestroy(B->graph);
    B->tab.release(ctx);
    B->ypbuf.release(ctx);
    B->arena.release(ctx);
    B->mix.release(ctx);
    cudaStreamSynchronize(ctx->stream);
    delete B;
    return DONOF_OK;
}

size_t donof_batch_device_bytes(const donof_batch* B) {
    return B ? B->arena.bytes + B->tab.bytes + B->ypbuf.bytes + B->mix.bytes : 0;
}

int donof_batch_lagrange2(donof_batch* B, const donof_batch_item* items, double* const* elag, double* const* H_mat,
                          double* E) {
    if (!B) return DONOF_ERR_ARG;
    donof_ctx* ctx = B->ctx;
    if (!items) {
        set_error(ctx, "donof_batch_lagrange2: null items");
        return DONOF_ERR_ARG;
    }
    DONOF_CHECK(check_items(B, items, false));
    DONOF_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = batch_stream(B);
    if (!st) {
        set_error(ctx, "donof_batch_lagrange2: no stream");
        return DONOF_ERR_CUDA;
    }
    std::vector<BOrbState> hs(B->nj);
    memset(hs.data(), 0, sizeof(BOrbState) * hs.size());
    DONOF_CHECK(start_call(B, st, items, hs));
    for (int j = 0; j < B->nj; ++j) {
        const donof_batch::Shape& h = B->sh[j];
        if (elag && elag[j])
            DONOF_CUDA(ctx, cudaMemcpyAsync(elag[j], B->pt[j].elag, sizeof(double) * h.nn, cudaMemcpyDeviceToDevice, st));
        if (H_mat && H_mat[j])
            DONOF_CUDA(ctx, cudaMemcpyAsync(H_mat[j], B->pt[j].Hmat, sizeof(double) * h.nbf * h.nbf5,
                                            cudaMemcpyDeviceToDevice, st));
    }
    DONOF_CUDA(ctx, cudaMemcpyAsync(hs.data(), B->d_state, sizeof(BOrbState) * B->nj, cudaMemcpyDeviceToHost, st));
    DONOF_CUDA(ctx, cudaStreamSynchronize(st));
    DONOF_CHECK(failure_status(ctx));
    if (E)
        for (int j = 0; j < B->nj; ++j) E[j] = hs[j].E;
    return DONOF_OK;
}

int donof_batch_orbopt(donof_batch* B, int method, donof_batch_item* items) {
    if (!B) return DONOF_ERR_ARG;
    donof_ctx* ctx = B->ctx;
    if (!items) {
        set_error(ctx, "donof_batch_orbopt: null items");
        return DONOF_ERR_ARG;
    }
    if (method < DONOF_ORB_ADAM || method > DONOF_ORB_DEMON) {
        set_error(ctx, "donof_batch_orbopt: unknown optimiser %d", method);
        return DONOF_ERR_ARG;
    }
    DONOF_CHECK(check_items(B, items, true));
    DONOF_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = batch_stream(B);
    if (!st) {
        set_error(ctx, "donof_batch_orbopt: no stream");
        return DONOF_ERR_CUDA;
    }
    const bool prof = ctx->profile;
    ctx->profile = false;  // event records are not allowed in a conditional body
    struct Restore {
        donof_ctx* c;
        bool p;
        ~Restore() { c->profile = p; }
    } restore{ctx, prof};
    const int nj = B->nj;
    std::vector<BOrbState> hs(nj);
    memset(hs.data(), 0, sizeof(BOrbState) * nj);
    for (int j = 0; j < nj; ++j) {
        hs[j].alpha = items[j].alpha;
        hs[j].thresh = items[j].threshgorb;
        hs[j].maxloop = items[j].maxloop;
        hs[j].stopped = (items[j].maxloop == 0) ? 1 : 0;  // left out of this call
    }
    DONOF_CHECK(start_call(B, st, items, hs));
    DONOF_CHECK(gradient(B, st));
    b_copy_kernel<<<grid_units(B->pre_total[1], 4, ctx->sm_count), 256, 0, st>>>(B->d_jobs, B->d_pre[1], nj,
                                                                               COPY_NEW_TO_CUR_BEST);
    count_launch();
    b_start_kernel<<<1, 256, 0, st>>>(B->d_jobs, nj);
    count_launch();
    DONOF_CUDA(ctx, cudaGetLastError());

    // (re)build the loop graph when the optimiser or the CTA budget changed
    if (!B->exec || B->graph_method != method || B->graph_ctas != ctx_ctas(ctx)) {
        if (B->exec) cudaGraphExecDestroy(B->exec);
        if (B->graph) cudaGraphDestroy(B->graph);
        B->exec = nullptr;
        B->graph = nullptr;
        cudaGraph_t graph = nullptr;
        DONOF_CUDA(ctx, cudaGraphCreate(&graph, 0));
        B->graph = graph;
        cudaGraphConditionalHandle handle;
        DONOF_CUDA(ctx, cudaGraphConditionalHandleCreate(&handle, graph, 1, cudaGraphCondAssignDefault));
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = handle;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        DONOF_CUDA(ctx, cudaGraphAddNode(&node, graph, nullptr, 0, &cp));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        const unsigned long long l0 = donof_launch_count();
        DONOF_CUDA(ctx, cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        int rc = DONOF_OK;
        do {
            b_update_kernel<<<grid_units(B->pre_total[0], 4, ctx->sm_count), 256, 0, st>>>(B->d_jobs, B->d_pre[0],
                                                                                         nj, method);
            count_launch();
            if ((rc = rotate_grouped(ctx, st, B->d_rot, nj, B->d_rstate, B->rot_grid)) != DONOF_OK) break;
            if ((rc = lagrangian(B, st)) != DONOF_OK) break;
            if ((rc = gradient(B, st)) != DONOF_OK) break;
            b_end_kernel<<<(nj + 127) / 128, 128, 0, st>>>(B->d_jobs, nj);
            count_launch();
            b_copy_kernel<<<grid_units(B->pre_total[1], 4, ctx->sm_count), 256, 0, st>>>(B->d_jobs, B->d_pre[1], nj,
                                                                                       COPY_LOOP_END);
            count_launch();
            b_commit_kernel<<<1, 256, 0, st>>>(B->d_jobs, nj, handle);
            count_launch();
        } while (false);
        cudaGraph_t captured = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(st, &captured);
        if (rc != DONOF_OK) return rc;
        if (ce != cudaSuccess) {
            set_error(ctx, "capture of the grouped optimiser body: %s", cudaGetErrorString(ce));
            return DONOF_ERR_CUDA;
        }
        B->per_iter = (int)(donof_launch_count() - l0);
        g_launch_adjust(-(long long)B->per_iter);
        cudaGraphExec_t exec = nullptr;
        DONOF_CUDA(ctx, cudaGraphInstantiate(&exec, graph, 0));
        B->exec = exec;
        B->graph_method = method;
        B->graph_ctas = ctx_ctas(ctx);
    }
    DONOF_CUDA(ctx, cudaGraphLaunch(B->exec, st));
    DONOF_CUDA(ctx, cudaMemcpyAsync(hs.data(), B->d_state, sizeof(BOrbState) * nj, cudaMemcpyDeviceToHost, st));
    DONOF_CUDA(ctx, cudaStreamSynchronize(st));
    DONOF_CHECK(failure_status(ctx));
    int iters = 0;
    for (int j = 0; j < nj; ++j) iters = std::max(iters, hs[j].it);
    g_launch_adjust((long long)B->per_iter * iters);
    // back-off and result of each job, as the single-job loop (src/minimization.jl:425-437)
    for (int j = 0; j < nj; ++j) {
        donof_batch_item& it = items[j];
        if (it.maxloop == 0) continue;
        if (!hs[j].improved) {
            it.alpha = 0.3 * it.alpha;
            it.maxloop = it.maxloop + 10;
        }
        const bool return_best = (it.maxloop < 100);
        DONOF_CUDA(ctx, cudaMemcpyAsync(it.C, return_best ? B->pt[j].Cbest : B->pt[j].Ccur,
                                        sizeof(double) * B->sh[j].nn, cudaMemcpyDeviceToDevice, st));
        it.E = return_best ? hs[j].bestE : hs[j].E;
        it.nit = hs[j].nit;
        it.success = hs[j].success;
    }
    DONOF_CUDA(ctx, cudaStreamSynchronize(st));
    return DONOF_OK;
}

struct donof_batch_queue {
    struct Req {
        donof_batch_request r;
        unsigned long long ticket;
        bool taken = false, done = false;
        int status = DONOF_OK;
        donof_energy_result res{};
    };
    std::mutex mu;
    std::condition_variable cv;       // serve loop: new request or close
    std::condition_variable cv_done;  // pollers: a request finished
    std::deque<std::shared_ptr<Req>> all;
    unsigned long long next = 1;
    bool closed = false;
    int method = -1;
    std::shared_ptr<Req> find(unsigned long long t) {
        for (auto& q : all)
            if (q->ticket == t) return q;
        return nullptr;
    }
};

int donof_batch_queue_create(donof_batch_queue** q) {
    if (!q) return DONOF_ERR_ARG;
    *q = new (std::nothrow) donof_batch_queue();
    return *q ? DONOF_OK : DONOF_ERR_OOM;
}

int donof_batch_queue_push(donof_batch_queue* q, const donof_batch_request* r, unsigned long long* ticket) {
    if (!q || !r || !ticket || !r->job || !r->H || !r->C_inout || !r->gamma_inout) return DONOF_ERR_ARG;
    std::lock_guard<std::mutex> lk(q->mu);
    if (q->closed) return DONOF_ERR_STATE;
    if (q->method < 0) q->method = r->params.orb_method;
    if (r->params.orb_method != q->method) return DONOF_ERR_ARG;  // one optimiser per queue
    auto req = std::make_shared<donof_batch_queue::Req>();
    req->r = *r;
    req->ticket = q->next++;
    q->all.push_back(req);
    *ticket = req->ticket;
    q->cv.notify_all();
    return DONOF_OK;
}

int donof_batch_queue_close(donof_batch_queue* q) {
    if (!q) return DONOF_ERR_ARG;
    std::lock_guard<std::mutex> lk(q->mu);
    q->closed = true;
    q->cv.notify_all();
    return DONOF_OK;
}

int donof_batch_queue_poll(donof_batch_queue* q, unsigned long long ticket, int wait, int* done, int* status,
                           donof_energy_result* res) {
    if (!q || !done) return DONOF_ERR_ARG;
    std::unique_lock<std::mutex> lk(q->mu);
    auto req = q->find(ticket);
    if (!req) return DONOF_ERR_ARG;
    if (wait) q->cv_done.wait(lk, [&] { return req->done; });
    *done = req->done ? 1 : 0;
    if (req->done) {
        if (status) *status = req->status;
        if (res) *res = req->res;
    }
    return DONOF_OK;
}

int donof_batch_queue_destroy(donof_batch_queue* q) {
    delete q;
    return DONOF_OK;
}

int donof_batch_energy(donof_batch* B, donof_energy_params* params, const double* const* H, double* const* C_inout,
                       double* const* gamma_inout, double* const* n_out, donof_energy_result* results) {
    if (!B) return DONOF_ERR_ARG;
    donof_ctx* ctx = B->ctx;
    if (!params || !H || !C_inout || !gamma_inout || !results) {
        set_error(ctx, "donof_batch_energy: null argument");
        return DONOF_ERR_ARG;
    }
    const int nj = B->nj;
    const int method = params[0].orb_method;
    for (int j = 0; j < nj; ++j) {
        const donof_batch::Shape& h = B->sh[j];
        const donof_energy_params& q = params[j];
        if (!H[j] || !C_inout[j] || !gamma_inout[j]) {
            set_error(ctx, "donof_batch_energy: job %d: null array", j);
            return DONOF_ERR_ARG;
        }
        if (q.occ.nbf5 != h.nbf5 || q.occ.nalpha != h.nalpha || q.occ.nbeta != h.nbeta) {
            set_error(ctx, "donof_batch_energy: job %d: nbf5/nalpha/nbeta differ from the batch's shape", j);
            return DONOF_ERR_ARG;
        }
        if (q.orb_method != method) {
            set_error(ctx, "donof_batch_energy: every job of a call uses the same orbital optimiser");
            return DONOF_ERR_ARG;
        }
        if (h.job->precision != DONOF_PREC_FP64) {
            set_error(ctx, "donof_batch_energy: job %d is not in the FP64 form", j);
            return DONOF_ERR_ARG;
        }
    }
    std::vector<EnergyJob> E(nj);
    for (int j = 0; j < nj; ++j)
        DONOF_CHECK(E[j].setup(B->sh[j].job, &params[j], H[j], C_inout[j], gamma_inout[j], nullptr));
    std::vector<donof_batch_item> items(nj);
    for (;;) {
        bool any = false;
        for (int j = 0; j < nj; ++j) {
            donof_batch_item& it = items[j];
            it.n = E[j].dev_n(); it.cj12 = E[j].dev_cj(); it.ck12 = E[j].dev_ck(); it.H = E[j].dev_H();
            it.C = E[j].dev_C();
            it.alpha = params[j].alpha;
            it.threshgorb = params[j].threshgorb;
            it.maxloop = 0;  // left out unless running
            if (E[j].done()) continue;
            DONOF_CHECK(E[j].begin());
            // the job's coefficient upload is on its own context's stream
            DONOF_CUDA(ctx, cudaStreamSynchronize(B->sh[j].job->ctx->stream));
            it.maxloop = params[j].maxloop;
            any = true;
        }
        if (!any) break;
        DONOF_CHECK(donof_batch_orbopt(B, method, items.data()));
        std::vector<int> run;
        for (int j = 0; j < nj; ++j) {
            if (items[j].maxloop == 0) continue;
            params[j].alpha = items[j].alpha;
            params[j].maxloop = items[j].maxloop;
            DONOF_CHECK(E[j].occ_fetch());
            run.push_back(j);
        }
        // the occupation optimisations of the running jobs, on host threads
        std::vector<int> st(run.size(), DONOF_OK);
        {
            std::atomic<size_t> next{0};
            auto work = [&]() {
                for (size_t i = next.fetch_add(1); i < run.size(); i = next.fetch_add(1)) st[i] = E[run[i]].occ_solve();
            };
            const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
            const size_t nt = std::min<size_t>(run.size(), hw);
            std::vector<std::thread> pool;
            for (size_t t = 1; t < nt; ++t) pool.emplace_back(work);
            work();
            for (std::thread& t : pool) t.join();
        }
        for (size_t i = 0; i < run.size(); ++i) {
            DONOF_CHECK(st[i]);
            DONOF_CHECK(E[run[i]].end_iteration(items[run[i]].E, items[run[i]].nit));
        }
    }
    for (int j = 0; j < nj; ++j)
        DONOF_CHECK(E[j].finish(C_inout[j], gamma_inout[j], n_out ? n_out[j] : nullptr, nullptr, &results[j]));
    return DONOF_OK;
}

int donof_batch_serve(donof_batch* B, donof_batch_queue* q) {
    if (!B || !q) return DONOF_ERR_ARG;
    donof_ctx* ctx = B->ctx;
    if (B->precision != DONOF_PREC_FP64) {
        set_error(ctx, "donof_batch_serve: continuous batching runs the FP64 form");
        return DONOF_ERR_STATE;
    }
    DONOF_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t bst = batch_stream(B);
    if (!bst) {
        set_error(ctx, "donof_batch_serve: no stream");
        return DONOF_ERR_CUDA;
    }
    using Req = donof_batch_queue::Req;
    const int nj = B->nj;
    std::vector<std::shared_ptr<Req>> slot(nj);
    std::vector<std::unique_ptr<EnergyJob>> E(nj);
    std::vector<donof_energy_params> prm(nj);
    std::vector<donof_batch_item> items(nj);
    // zero device arrays standing in for an idle slot's inputs (the grouped step skips the slot)
    DevBuf idle;
    std::vector<size_t> ioff(nj);
    size_t per = 0;
    for (int j = 0; j < nj; ++j) {
        const donof_batch::Shape& h = B->sh[j];
        ioff[j] = per;
        per += al32((size_t)h.nbf5 + 2 * (size_t)h.nbf5 * h.nbf5 + 2 * (size_t)h.nn);
    }
    DONOF_CHECK(idle.ensure(ctx, sizeof(double) * per));
    DONOF_CUDA(ctx, cudaMemsetAsync(idle.ptr, 0, sizeof(double) * per, bst));
    struct Release {
        donof_ctx* c;
        DevBuf* b;
        cudaStream_t s;
        ~Release() {
            cudaStreamSynchronize(s);
            b->release(c);
        }
    } release{ctx, &idle, bst};
    auto fits = [&](const Req& r, int j) {
        const donof_batch::Shape& h = B->sh[j];
        const donof_job* jb = r.r.job;
        return jb->ctx != nullptr && jb->ctx->device == ctx->device && jb->b != nullptr &&
               jb->precision == DONOF_PREC_FP64 && jb->nbf == h.nbf && jb->naux == h.naux &&
               r.r.params.occ.nbf5 == h.nbf5 && r.r.params.occ.nalpha == h.nalpha && r.r.params.occ.nbeta == h.nbeta;
    };
    auto complete = [&](const std::shared_ptr<Req>& r, int status, const donof_energy_result* res) {
        std::lock_guard<std::mutex> lk(q->mu);
        r->status = status;
        if (res) r->res = *res;
        r->done = true;
        q->cv_done.notify_all();
    };
    auto retire = [&](int j, int status) {
        donof_energy_result res{};
        int s = status;
        if (s == DONOF_OK)
            s = E[j]->finish(slot[j]->r.C_inout, slot[j]->r.gamma_inout, slot[j]->r.n_out, nullptr, &res);
        complete(slot[j], s, s == DONOF_OK ? &res : nullptr);
        slot[j].reset();
        E[j].reset();
    };
    auto fail_all = [&](int status) {
        for (int j = 0; j < nj; ++j)
            if (slot[j]) {
                complete(slot[j], status, nullptr);
                slot[j].reset();
                E[j].reset();
            }
        return status;
    };
    int method = -1;
    for (;;) {
        // ---- free slots take the oldest waiting request of their shape
        std::vector<int> fresh;
        {
            std::unique_lock<std::mutex> lk(q->mu);
            for (;;) {
                method = q->method;
                for (auto& r : q->all) {
                    if (r->taken) continue;
                    bool some = false;
                    for (int j = 0; j < nj && !some; ++j) some = fits(*r, j);
                    if (!some) {  // no slot of the batch has this request's shape
                        r->taken = r->done = true;
                        r->status = DONOF_ERR_ARG;
                        q->cv_done.notify_all();
                    }
                }
                for (int j = 0; j < nj; ++j) {
                    if (slot[j]) continue;
                    for (auto& r : q->all)
                        if (!r->taken && fits(*r, j)) {
                            r->taken = true;
                            slot[j] = r;
                            fresh.push_back(j);
                            break;
                        }
                }
                bool active = false, pending = false;
                for (int j = 0; j < nj; ++j) active = active || (bool)slot[j];
                for (auto& r : q->all) pending = pending || !r->taken;
                if (active) break;
                if (q->closed && !pending) return DONOF_OK;
                q->cv.wait_for(lk, std::chrono::milliseconds(20));
            }
        }
        // ---- bind the new requests' RI tensors and start their energy loops
        bool rebound = false;
        for (int j : fresh) {
            // always rebind: a freed job's address may have been reused by this one
            B->sh[j].job = slot[j]->r.job;
            B->sh[j].b = slot[j]->r.job->b;
            rebound = true;
            prm[j] = slot[j]->r.params;
            E[j].reset(new (std::nothrow) EnergyJob());
            const int s = E[j] ? E[j]->setup(slot[j]->r.job, &prm[j], slot[j]->r.H, slot[j]->r.C_inout,
                                             slot[j]->r.gamma_inout, nullptr)
                               : DONOF_ERR_OOM;
            if (s != DONOF_OK) retire(j, s);
        }
        if (rebound) {
            const int s = upload_gemm_tables(B, bst);
            if (s != DONOF_OK) return fail_all(s);
        }
        // ---- one outer iteration of every running request, the orbital steps grouped
        bool any = false;
        for (int j = 0; j < nj; ++j) {
            donof_batch_item& it = items[j];
            it.maxloop = 0;  // left out unless running
            if (E[j] && !E[j]->done()) {
                int s = E[j]->begin();
                if (s == DONOF_OK && cudaStreamSynchronize(slot[j]->r.job->ctx->stream) != cudaSuccess) s = DONOF_ERR_CUDA;
                if (s != DONOF_OK) {
                    retire(j, s);
                } else {
                    it.n = E[j]->dev_n(); it.cj12 = E[j]->dev_cj(); it.ck12 = E[j]->dev_ck(); it.H = E[j]->dev_H();
                    it.C = E[j]->dev_C();
                    it.alpha = prm[j].alpha;
                    it.threshgorb = prm[j].threshgorb;
                    it.maxloop = prm[j].maxloop;
                    any = true;
                    continue;
                }
            }
            const donof_batch::Shape& h = B->sh[j];
            double* z = idle.as<double>() + ioff[j];
            it.n = z; it.cj12 = z + h.nbf5; it.ck12 = z + h.nbf5 + (size_t)h.nbf5 * h.nbf5;
            it.H = z + h.nbf5 + 2 * (size_t)h.nbf5 * h.nbf5;
            it.C = const_cast<double*>(it.H) + h.nn;
            it.alpha = 0.01;
            it.threshgorb = 1.0;
        }
        if (any) {
            int s = donof_batch_orbopt(B, method, items.data());
            if (s != DONOF_OK) return fail_all(s);
            std::vector<int> run;
            for (int j = 0; j < nj; ++j) {
                if (items[j].maxloop == 0 || !E[j]) continue;
                prm[j].alpha = items[j].alpha;
                prm[j].maxloop = items[j].maxloop;
                s = E[j]->occ_fetch();
                if (s != DONOF_OK) retire(j, s);
                else run.push_back(j);
            }
            std::vector<int> st(run.size(), DONOF_OK);
            {
                std::atomic<size_t> next{0};
                auto work = [&]() {
                    for (size_t i = next.fetch_add(1); i < run.size(); i = next.fetch_add(1))
                        st[i] = E[run[i]]->occ_solve();
                };
                const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
                const size_t nt = std::min<size_t>(run.size(), hw);
                std::vector<std::thread> pool;
                for (size_t k = 1; k < nt; ++k) pool.emplace_back(work);
                work();
                for (std::thread& th : pool) th.join();
            }
            for (size_t i = 0; i < run.size(); ++i) {
                const int j = run[i];
                s = st[i];
                if (s == DONOF_OK) s = E[j]->end_iteration(items[j].E, items[j].nit);
                if (s != DONOF_OK) retire(j, s);
            }
        }
        // ---- converged (or out of iterations) requests return now; their slots free up
        for (int j = 0; j < nj; ++j)
            if (E[j] && E[j]->done()) retire(j, DONOF_OK);
    }
}

}  // extern "C"
