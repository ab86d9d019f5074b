// Plain FP64 form of the RI hot path: compute_Lagrange2 and JKH_MO.
//
// Restructured contraction (exact in exact arithmetic):
//   T1   tmp_l  = B_l C5                  (per aux index l; nbf x nbf5)
//   T2   b_pq^l = C5^T tmp_l              (nbf5 x nbf5)
//   W[q,l,b]    = delta_qb (n'_b d_b^l + sum_q' cj12[b,q'] d_q'^l) - ck12[b,q] b_bq^l
//                 with d_q^l = b_qq^l and n'_b = n_b on the beta/alpha-virtual
//                 blocks (src/utils.jl:42-47), 0 elsewhere
//   Y[m,b]      = sum_{q,l} tmp_l[m,q] W[q,l,b]          (one GEMM, K = nbf5*naux)
//   elag[:, :nbf5] = C^T Y + n_b H_mat[:, b]
// which equals src/utils.jl:17-55 term by term: every elag term there is
// sum_k b_MO[a,.,k] X[.,k,b] with b_MO = C^T tmp, so C^T factors out and the
// full nbf x nbf second transform of the reference is never formed.
// JKH_MO (src/integrals.jl:144-172) reuses T1/T2: J = D D^T with D[p,l] = d_p^l
// and K = sum_l (b_pq^l)^2.
#include <math.h>

#include <mutex>

#include "kernels.cuh"
#include "wbuild.cuh"

namespace donof {

namespace {

// W of every aux index (wbuild.cuh) in two fully parallel passes: w_diag_kernel
// forms n'_b d_b^l + t_b^l (one thread per (b, l), cj12 read along b, the
// diagonals d^l staged in shared memory per group of aux indices);
// build_w_kernel the elementwise part over tiles of 32 x 32 (b, q) and
// wbuild::LT aux indices, one tile per CTA step (b need not be symmetric).
__global__ void __launch_bounds__(256) w_diag_kernel(const double* __restrict__ bpq, const double* __restrict__ n,
                                                     const double* __restrict__ cj12, int nbf5, int naux, int nalpha,
                                                     int nbeta, double* __restrict__ tv) {
    __shared__ double sd[wbuild::DIAG_SM];
    const long long units = wbuild::diag_units(nbf5, naux);
    for (long long u = blockIdx.x; u < units; u += gridDim.x)
        wbuild::diag_unit(bpq, n, cj12, nbf5, naux, nalpha, nbeta, tv, u, sd);
}

__global__ void __launch_bounds__(256, 4) build_w_kernel(const double* __restrict__ bpq, const double* __restrict__ ck12,
                                                      const double* __restrict__ tv, int nbf5, int naux,
                                                      double* __restrict__ W) {
    __shared__ double tb[wbuild::LT][32][33];
    const long long tiles = wbuild::tiles(nbf5, naux);
    for (long long t = blockIdx.x; t < tiles; t += gridDim.x) wbuild::tile(bpq, ck12, tv, nbf5, naux, W, t, tb);
}

// W in one pass for nbf5 <= FUSED_W_MAX: the tiles of build_w_kernel, where a
// diagonal tile (b0 == q0) first computes its own n'_b d_b^l + t_b^l for its 32
// b and LT aux indices -- one thread per (b, l), summing over q in the order of
// wbuild::diag_unit, so W is bit-for-bit the two-kernel W (the grouped path of
// batch.cu still builds it in two passes and must agree with this one).
constexpr int FUSED_W_MAX = 256;

__global__ void __launch_bounds__(256, 4) build_w_fused_kernel(const double* __restrict__ bpq,
                                                            const double* __restrict__ n,
                                                            const double* __restrict__ cj12,
                                                            const double* __restrict__ ck12, int nbf5, int naux,
                                                            int nalpha, int nbeta, double* __restrict__ W) {
    __shared__ double tb[wbuild::LT][32][33];
    __shared__ double sd[wbuild::LT * FUSED_W_MAX];
    __shared__ double stv[wbuild::LT][32];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const long long n55 = (long long)nbf5 * nbf5, Kt = (long long)nbf5 * naux;
    const int nt = (nbf5 + 31) / 32;
    const long long tiles = wbuild::tiles(nbf5, naux);
    for (long long t = blockIdx.x; t < tiles; t += gridDim.x) {
        const int b0 = (int)(t % nt) * 32, q0 = (int)((t / nt) % nt) * 32;
        const long long l0 = (t / ((long long)nt * nt)) * wbuild::LT;
        const int b = b0 + tx;
        const bool diag = (b0 == q0);
        if (diag) {
            __syncthreads();  // the previous tile's reads of sd are done
            for (int i = threadIdx.x; i < wbuild::LT * nbf5; i += blockDim.x) {
                const int k = i / nbf5, q = i - k * nbf5;
                const long long l = l0 + k;
                sd[i] = (l < naux) ? bpq[n55 * l + (long long)q * (nbf5 + 1)] : 0.0;
            }
            __syncthreads();
            if (threadIdx.x < 32 * wbuild::LT) {
                const int k = threadIdx.x >> 5, bb = b0 + tx;
                const long long l = l0 + k;
                if (l < naux && bb < nbf5) {
                    const double* d = sd + k * nbf5;
                    double s = 0.0;
                    for (int q = 0; q < nbf5; ++q) s = wbuild::tv_step(s, cj12[bb + (long long)nbf5 * q], d[q]);
                    const bool dj = (nbeta > 0) && (bb < nbeta || bb >= nalpha);
                    stv[k][tx] = wbuild::tv_value(dj, n[bb], d[bb], s);
                }
            }
        }
        double ck[4], v[wbuild::LT][4];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int q = q0 + ty + 8 * r;
            ck[r] = (b < nbf5 && q < nbf5) ? ck12[b + (long long)nbf5 * q] : 0.0;
        }
#pragma unroll
        for (int k = 0; k < wbuild::LT; ++k) {
            const long long l = l0 + k;
            const double* B = bpq + n55 * l;
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const int q = q0 + ty + 8 * r;
                v[k][r] = (l < naux && b < nbf5 && q < nbf5) ? B[b + (long long)nbf5 * q] : 0.0;
            }
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < wbuild::LT; ++k) {
            const long long l = l0 + k;
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const int q = q0 + ty + 8 * r;
                double w = wbuild::w_value(ck[r], v[k][r]);
                if (diag && q == b && l < naux && b < nbf5) w = wbuild::w_diag(w, stv[k][tx]);
                tb[k][ty + 8 * r][tx] = w;  // [l - l0][q - q0][b - b0]
            }
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < wbuild::LT; ++k) {
            const long long l = l0 + k;
            if (l >= naux) break;
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const int q = q0 + tx, bb = b0 + ty + 8 * r;
                if (bb < nbf5 && q < nbf5) W[q + (long long)nbf5 * l + Kt * bb] = tb[k][tx][ty + 8 * r];
            }
        }
    }
}

// elag[a, b] = n_b H_mat[a, b] for b < nbf5 (the 2ndH/dy_ab term,
// src/utils.jl:39), columns >= nbf5 set to zero.
__global__ void elag_init_kernel(const double* __restrict__ Hmat, const double* __restrict__ n,
                                 int nbf, int nbf5, double* __restrict__ elag) {
    const long long total = (long long)nbf * nbf;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(i / nbf);
        elag[i] = (b < nbf5) ? n[b] * Hmat[i] : 0.0;
    }
}

// E_elec = sum_{i<nbf5} elag[i,i] + sum_i n_i H_mat[i,i]   (src/utils.jl:216-227)
__global__ void e_elec_kernel(const double* __restrict__ elag, const double* __restrict__ Hmat,
                              const double* __restrict__ n, int nbf, int nbf5, double* E) {
    __shared__ double red[32];
    double s = 0.0;
    for (int i = threadIdx.x; i < nbf5; i += blockDim.x)
        s += elag[i + (long long)nbf * i] + n[i] * Hmat[i + (long long)nbf * i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0) *E = s;
    }
}

// J/K partial sums over a chunk of aux indices; thread per (p, q).
__global__ void jk_partial_kernel(const double* __restrict__ bpq, int nbf5, int naux, int lchunk,
                                  double* __restrict__ part) {
    const long long n55 = (long long)nbf5 * nbf5;
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const int c = blockIdx.y;
    if (idx >= n55) return;
    const int p = (int)(idx % nbf5), q = (int)(idx / nbf5);
    const int l0 = c * lchunk, l1 = min(naux, l0 + lchunk);
    double sj = 0.0, sk = 0.0;
    for (int l = l0; l < l1; ++l) {
        const double* B = bpq + n55 * l;
        const double v = B[idx];
        sj += B[(long long)p * (nbf5 + 1)] * B[(long long)q * (nbf5 + 1)];
        sk += v * v;
    }
    part[(long long)c * 2 * n55 + idx] = sj;
    part[(long long)c * 2 * n55 + n55 + idx] = sk;
}

// H_core[i] = sum_m C[m,i] (H C5)[m,i]; one warp per i.
__global__ void hcore_kernel(const double* __restrict__ C, const double* __restrict__ HC, int nbf,
                             int nbf5, double* __restrict__ Hcore) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= nbf5) return;
    double s = 0.0;
    for (int m = lane; m < nbf; m += 32) s += C[m + (long long)nbf * warp] * HC[m + (long long)nbf * warp];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) Hcore[warp] = s;
}

// W of every aux index into W (Kt * nbf5 values; W + Kt * nbf5 holds the Kt
// diagonal terms when they are built in a pass of their own).
int build_w(donof_ctx* ctx, cudaStream_t st, const double* bpq, const double* n, const double* cj12,
            const double* ck12, int nbf5, int naux, int nalpha, int nbeta, double* W) {
    long long blocks = wbuild::tiles(nbf5, naux);
    if (blocks > 16LL * ctx->sm_count) blocks = 16LL * ctx->sm_count;
    if (nbf5 <= FUSED_W_MAX) {
        build_w_fused_kernel<<<(int)blocks, 256, 0, st>>>(bpq, n, cj12, ck12, nbf5, naux, nalpha, nbeta, W);
        count_launch();
    } else {
        double* tv = W + (size_t)nbf5 * naux * nbf5;  // n'_b d_b^l + t_b^l (Kt values)
        long long dblocks = wbuild::diag_units(nbf5, naux);
        if (dblocks > 8LL * ctx->sm_count) dblocks = 8LL * ctx->sm_count;
        w_diag_kernel<<<(int)dblocks, 256, 0, st>>>(bpq, n, cj12, nbf5, naux, nalpha, nbeta, tv); count_launch();
        build_w_kernel<<<(int)blocks, 256, 0, st>>>(bpq, ck12, tv, nbf5, naux, W); count_launch();
    }
    DONOF_CUDA(ctx, cudaGetLastError());
    return DONOF_OK;
}

int grid_for(long long total, int threads, int sm) {
    long long b = (total + threads - 1) / threads;
    if (b > 8LL * sm) b = 8LL * sm;
    return (int)(b < 1 ? 1 : b);
}

}  // namespace

// T1 + T2 into the job scratch: tmp (nbf x nbf5 x naux) and bpq (nbf5^2 x naux).
int transforms_f64(donof_job* job, cudaStream_t st, const double* C, int nbf5) {
    donof_ctx* ctx = job->ctx;
    const int nbf = job->nbf, naux = job->naux;
    DONOF_CHECK(job->tmp.ensure(ctx, sizeof(double) * (size_t)nbf * nbf5 * naux));
    DONOF_CHECK(job->bpq.ensure(ctx, sizeof(double) * (size_t)nbf5 * nbf5 * naux));
    double* tmp = job->tmp.as<double>();
    double* bpq = job->bpq.as<double>();
    // T1: tmp_l(m,q) = sum_n b[m,n,l] C[n,q]; A(i=m,k=n) = b[m + nbf*n] (M-contiguous).
    // With b's digit slices on the device it runs on the tensor cores (ozaki.cu).
    if (job->oz_b) {
        DONOF_CHECK(t1_ozaki(job, st, C, nbf5, tmp));
    } else {
        GemmF64Args p{};
        p.M = nbf; p.N = nbf5; p.K = nbf;
        p.A = job->b; p.lda = nbf; p.strideA = (long long)nbf * nbf;
        p.B = C; p.ldb = nbf; p.strideB = 0;
        p.C = tmp; p.ldc = nbf; p.strideC = (long long)nbf * nbf5;
        p.alpha = 1.0; p.beta = 0.0; p.batch = naux; p.splits = 1;
        prof_begin(ctx, st);
        DONOF_CHECK(gemm_f64_tuned(ctx, st, false, true, p, nbf >= 128 ? GemmTile::Large : GemmTile::Small));
        prof_end(ctx, st);
    }
    // T2: bpq_l(p,q) = sum_m C[m,p] tmp_l[m,q]
    {
        GemmF64Args p{};
        p.M = nbf5; p.N = nbf5; p.K = nbf;
        p.A = C; p.lda = nbf; p.strideA = 0;
        p.B = tmp; p.ldb = nbf; p.strideB = (long long)nbf * nbf5;
        p.C = bpq; p.ldc = nbf5; p.strideC = (long long)nbf5 * nbf5;
        p.alpha = 1.0; p.beta = 0.0; p.batch = naux; p.splits = 1;
        DONOF_CHECK(gemm_f64_tuned(ctx, st, true, true, p, nbf5 > 64 ? GemmTile::Large : GemmTile::Small));
    }
    return DONOF_OK;
}

int lagrange2_f64(donof_job* job, cudaStream_t st, const double* C, const double* n,
                  const double* H, const double* cj12, const double* ck12, int nbf5, int nalpha,
                  int nbeta, double* elag, double* Hmat, double* E) {
    donof_ctx* ctx = job->ctx;
    const int nbf = job->nbf, naux = job->naux;
    const long long Kt = (long long)nbf5 * naux;

    DONOF_CHECK(transforms_f64(job, st, C, nbf5));

    DONOF_CHECK(job->W.ensure(ctx, sizeof(double) * (size_t)Kt * (nbf5 + 1)));
    double* W = job->W.as<double>();
    DONOF_CHECK(build_w(ctx, st, job->bpq.as<double>(), n, cj12, ck12, nbf5, naux, nalpha, nbeta, W));

    // Y = sum_{q,l} tmp[m, q + nbf5*l] W[q + nbf5*l, b], left as split-K partials
    const double* ypart = nullptr;
    int nparts = 1;
    DONOF_CHECK(gemm_f64_partials(ctx, st, false, true, nbf, nbf5, (int)Kt, job->tmp.as<double>(), nbf, W, Kt,
                                  &job->part, &ypart, &nparts));
    // H_mat = C^T (H C5) (src/utils.jl:17-18), elag = [n o H_mat + C^T Y | 0], E_elec
    return elag_tail_f64(job, st, C, H, n, nbf5, ypart, false, nparts, (long long)nbf * nbf5, Hmat, elag, E);
}

// The Lagrangian of a slice of the aux index (the job's b holds naux_r aux
// indices of a larger tensor): Y_r = sum_{q, l in slice} tmp_l[m, q] W[q, l, b],
// reduced to one nbf x nbf5 FP64 matrix.  Every term of Y is a sum over l, so the
// Y of the whole tensor is the sum of the slices' Y (an all-reduce across the
// ranks that hold the slices); lagrange2_finish_f64 then gives elag, H_mat, E.
int lagrange2_partial_f64(donof_job* job, cudaStream_t st, const double* C, const double* n, const double* cj12,
                          const double* ck12, int nbf5, int nalpha, int nbeta, double* Y) {
    donof_ctx* ctx = job->ctx;
    const int nbf = job->nbf, naux = job->naux;
    const long long Kt = (long long)nbf5 * naux;
    DONOF_CHECK(transforms_f64(job, st, C, nbf5));
    DONOF_CHECK(job->W.ensure(ctx, sizeof(double) * (size_t)Kt * (nbf5 + 1)));
    double* W = job->W.as<double>();
    DONOF_CHECK(build_w(ctx, st, job->bpq.as<double>(), n, cj12, ck12, nbf5, naux, nalpha, nbeta, W));
    const double* ypart = nullptr;
    int nparts = 1;
    DONOF_CHECK(gemm_f64_partials(ctx, st, false, true, nbf, nbf5, (int)Kt, job->tmp.as<double>(), nbf, W, Kt,
                                  &job->part, &ypart, &nparts));
    const long long ny = (long long)nbf * nbf5;
    return splitk_reduce(ctx, st, ypart, ny, nparts, ny, Y, 0.0);
}

// elag, H_mat and E_elec from the Y of the whole aux range (the fused tail).
int lagrange2_finish_f64(donof_job* job, cudaStream_t st, const double* C, const double* n, const double* H,
                         int nbf5, const double* Y, double* elag, double* Hmat, double* E) {
    return elag_tail_f64(job, st, C, H, n, nbf5, Y, false, 1, (long long)job->nbf * nbf5, Hmat, elag, E);
}

int hcore_f64(donof_job* job, cudaStream_t st, const double* C, const double* HC, int nbf5, double* Hcore) {
    hcore_kernel<<<(nbf5 * 32 + 255) / 256, 256, 0, st>>>(C, HC, job->nbf, nbf5, Hcore); count_launch();
    DONOF_CUDA(job->ctx, cudaGetLastError());
    return DONOF_OK;
}

int jkh_mo_f64(donof_job* job, cudaStream_t st, const double* C, const double* H, int nbf5,
               double* J, double* K, double* Hcore) {
    donof_ctx* ctx = job->ctx;
    const int nbf = job->nbf, naux = job->naux;
    DONOF_CHECK(transforms_f64(job, st, C, nbf5));
    const long long n55 = (long long)nbf5 * nbf5;
    // chunk the aux index so that about 2 CTAs per SM are busy
    const int xblocks = (int)((n55 + 255) / 256);
    int chunks = (2 * ctx->sm_count + xblocks - 1) / xblocks;
    if (chunks > naux) chunks = naux;
    if (chunks < 1) chunks = 1;
    const int lchunk = (naux + chunks - 1) / chunks;
    chunks = (naux + lchunk - 1) / lchunk;
    DONOF_CHECK(job->part.ensure(ctx, sizeof(double) * (size_t)chunks * 2 * n55));
    double* part = job->part.as<double>();
    jk_partial_kernel<<<dim3(xblocks, chunks), 256, 0, st>>>(job->bpq.as<double>(), nbf5, naux, lchunk,
                                                             part); count_launch();
    DONOF_CUDA(ctx, cudaGetLastError());
    DONOF_CHECK(splitk_reduce(ctx, st, part, 2 * n55, chunks, n55, J, 0.0));
    DONOF_CHECK(splitk_reduce(ctx, st, part + n55, 2 * n55, chunks, n55, K, 0.0));
    // H_core
    DONOF_CHECK(job->small.ensure(ctx, sizeof(double) * (size_t)nbf * nbf5 * 2));
    double* HC = job->small.as<double>();
    DONOF_CHECK(gemm_f64_auto(ctx, st, false, true, nbf, nbf5, nbf, H, nbf, C, nbf, HC, nbf, 1.0,
                              0.0, nullptr));
    hcore_kernel<<<(nbf5 * 32 + 255) / 256, 256, 0, st>>>(C, HC, nbf, nbf5, Hcore); count_launch();
    DONOF_CUDA(ctx, cudaGetLastError());
    return DONOF_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free compute_Lagrange2 (donof_lagrange2_noalloc_dev).
//
// Some callers cannot call cudaMalloc at all: a host whose device memory is
// owned by another runtime's pool (a Julia or PyTorch process that hands this
// library only the arrays it already holds), code that must not add to a fixed
// device-memory budget while it serves, or a caller that may not block on the
// synchronising allocator in the middle of its own stream work.  This variant
// runs the same FP64 pipeline as lagrange2_f64 but takes every intermediate
// from one file-scope device array of NOALLOC_SCRATCH_BYTES, which every GPU
// that loads the library holds until the process exits.  It never calls
// cudaMalloc, cudaFree or an allocating library routine.
//
// The first call on a device looks the array up with cudaGetSymbolAddress
// (with that device current) and caches the address; make that first call
// before any stream capture.  Every call shares the one array, so calls that
// overlap on the GPU (other streams, other host threads) race on it; each
// call writes every scratch element it later reads, so nothing has to start
// at zero and the contents left by the previous call are never used.
// ---------------------------------------------------------------------------
constexpr size_t NOALLOC_SCRATCH_BYTES = size_t(32) << 20;  // 32 MiB
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

namespace {

std::mutex g_noalloc_mutex;
void* g_noalloc_addr[64] = {};

// Device address of g_noalloc_scratch on the current device (set-up once per device).
int noalloc_scratch(donof_ctx* ctx, double** out) {
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (ctx->device < 0 || ctx->device >= 64) {
        set_error(ctx, "device index %d out of range for the scratch table", ctx->device);
        return DONOF_ERR_ARG;
    }
    if (g_noalloc_addr[ctx->device] == nullptr) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr) {
            set_error(ctx, "cudaGetSymbolAddress(scratch) on device %d: %s", ctx->device,
                      cudaGetErrorString(e));
            return DONOF_ERR_CUDA;
        }
        g_noalloc_addr[ctx->device] = p;
    }
    *out = static_cast<double*>(g_noalloc_addr[ctx->device]);
    return DONOF_OK;
}

size_t round256(size_t doubles) { return (doubles * sizeof(double) + 255) / 256 * 256 / sizeof(double); }

}  // namespace

int lagrange2_f64_noalloc(donof_job* job, cudaStream_t st, const double* C, const double* n,
                          const double* H, const double* cj12, const double* ck12, int nbf5,
                          int nalpha, int nbeta, double* elag, double* Hmat, double* E) {
    donof_ctx* ctx = job->ctx;
    const int nbf = job->nbf, naux = job->naux;
    const long long Kt = (long long)nbf5 * naux;
    // split count of the Lagrangian GEMM (K = nbf5 * naux), as in gemm_f64_auto
    int splits = 1;
    const GemmTile ytile = pick_tile(ctx, nbf, nbf5, (int)Kt, true, &splits);
    int kchunk = (int)Kt;
    if (splits > 1) {
        kchunk = (int)(((Kt + splits - 1) / splits + 15) / 16 * 16);
        splits = (int)((Kt + kchunk - 1) / kchunk);
    }
    const size_t s_tmp = round256((size_t)nbf * nbf5 * naux);
    const size_t s_bpq = round256((size_t)nbf5 * nbf5 * naux);
    const size_t s_w = round256((size_t)Kt * (nbf5 + 1));  // W and the diagonal terms
    const size_t s_small = round256((size_t)nbf * nbf5);
    const size_t s_part = round256((size_t)splits * nbf * nbf5);
    const size_t need = (s_tmp + s_bpq + s_w + 2 * s_small + s_part) * sizeof(double);
    if (need > NOALLOC_SCRATCH_BYTES) {
        set_error(ctx,
                  "donof_lagrange2_noalloc_dev: nbf=%d nbf5=%d naux=%d needs %zu bytes of scratch, "
                  "more than the fixed %zu bytes; use donof_lagrange2_dev",
                  nbf, nbf5, naux, need, NOALLOC_SCRATCH_BYTES);
        return DONOF_ERR_ARG;
    }
    double* base = nullptr;
    DONOF_CHECK(noalloc_scratch(ctx, &base));
    double* tmp = base;
    double* bpq = tmp + s_tmp;
    double* W = bpq + s_bpq;
    double* HC = W + s_w;
    double* Y = HC + s_small;
    double* part = Y + s_small;

    auto plain = [&](bool ak, const double* A, const double* B, double* Cm, double beta) -> int {
        int sp = 1;
        const GemmTile t = pick_tile(ctx, nbf, nbf5, nbf, false, &sp);
        GemmF64Args p{};
        p.M = nbf; p.N = nbf5; p.K = nbf;
        p.A = A; p.lda = nbf; p.B = B; p.ldb = nbf; p.C = Cm; p.ldc = nbf;
        p.alpha = 1.0; p.beta = beta; p.batch = 1; p.splits = 1; p.kchunk = nbf;
        return gemm_f64(ctx, st, ak, true, p, t);
    };
    // H_mat = C^T (H C5)
    DONOF_CHECK(plain(false, H, C, HC, 0.0));
    DONOF_CHECK(plain(true, C, HC, Hmat, 0.0));
    // T1 / T2
    {
        GemmF64Args p{};
        p.M = nbf; p.N = nbf5; p.K = nbf;
        p.A = job->b; p.lda = nbf; p.strideA = (long long)nbf * nbf;
        p.B = C; p.ldb = nbf; p.strideB = 0;
        p.C = tmp; p.ldc = nbf; p.strideC = (long long)nbf * nbf5;
        p.alpha = 1.0; p.beta = 0.0; p.batch = naux; p.splits = 1;
        DONOF_CHECK(gemm_f64(ctx, st, false, true, p, nbf >= 128 ? GemmTile::Large : GemmTile::Small));
    }
    {
        GemmF64Args p{};
        p.M = nbf5; p.N = nbf5; p.K = nbf;
        p.A = C; p.lda = nbf; p.strideA = 0;
        p.B = tmp; p.ldb = nbf; p.strideB = (long long)nbf * nbf5;
        p.C = bpq; p.ldc = nbf5; p.strideC = (long long)nbf5 * nbf5;
        p.alpha = 1.0; p.beta = 0.0; p.batch = naux; p.splits = 1;
        DONOF_CHECK(gemm_f64(ctx, st, true, true, p, nbf5 > 64 ? GemmTile::Large : GemmTile::Small));
    }
    {
        double* tv = W + (size_t)Kt * nbf5;
        w_diag_kernel<<<grid_for(wbuild::diag_units(nbf5, naux) * 256, 256, ctx->sm_count), 256, 0, st>>>(
            bpq, n, cj12, nbf5, naux, nalpha, nbeta, tv); count_launch();
        build_w_kernel<<<grid_for(wbuild::tiles(nbf5, naux) * 256, 256, ctx->sm_count), 256, 0, st>>>(
            bpq, ck12, tv, nbf5, naux, W); count_launch();
        DONOF_CUDA(ctx, cudaGetLastError());
    }
    // Y = tmp W (split-K partials in the scratch, then reduced)
    {
        GemmF64Args p{};
        p.M = nbf; p.N = nbf5; p.K = (int)Kt;
        p.A = tmp; p.lda = nbf; p.B = W; p.ldb = Kt;
        p.alpha = 1.0; p.beta = 0.0; p.batch = 1;
        if (splits > 1) {
            p.C = part; p.ldc = nbf; p.splits = splits; p.kchunk = kchunk;
            p.strideSplit = (long long)nbf * nbf5;
            DONOF_CHECK(gemm_f64(ctx, st, false, true, p, ytile));
            DONOF_CHECK(splitk_reduce(ctx, st, part, (long long)nbf * nbf5, splits, (long long)nbf * nbf5, Y, 0.0));
        } else {
            p.C = Y; p.ldc = nbf; p.splits = 1; p.kchunk = (int)Kt;
            DONOF_CHECK(gemm_f64(ctx, st, false, true, p, ytile));
        }
    }
    elag_init_kernel<<<grid_for((long long)nbf * nbf, 256, ctx->sm_count), 256, 0, st>>>(Hmat, n, nbf, nbf5,
                                                                                      elag); count_launch();
    DONOF_CUDA(ctx, cudaGetLastError());
    DONOF_CHECK(plain(true, C, Y, elag, 1.0));
    if (E != nullptr) {
        e_elec_kernel<<<1, 256, 0, st>>>(elag, Hmat, n, nbf, nbf5, E); count_launch();
        DONOF_CUDA(ctx, cudaGetLastError());
    }
    return DONOF_OK;
}

}  // namespace donof

extern "C" int donof_lagrange2_noalloc_dev(donof_job* job, const double* C, const double* n, const double* H,
                                           const double* cj12, const double* ck12, int nbf5, int nalpha,
                                           int nbeta, double* elag, double* H_mat, double* E_elec) {
    using namespace donof;
    if (!job) return DONOF_ERR_ARG;
    donof_ctx* ctx = job->ctx;
    if (nbf5 <= 0 || nbf5 > job->nbf || nbeta < 0 || nalpha < nbeta || nalpha > nbf5) {
        set_error(ctx, "donof_lagrange2_noalloc_dev: invalid sizes nbf=%d nbf5=%d nalpha=%d nbeta=%d", job->nbf,
                  nbf5, nalpha, nbeta);
        return DONOF_ERR_ARG;
    }
    if (!C || !n || !H || !cj12 || !ck12 || !elag || !H_mat) {
        set_error(ctx, "donof_lagrange2_noalloc_dev: null array argument");
        return DONOF_ERR_ARG;
    }
    DONOF_CUDA(ctx, cudaSetDevice(ctx->device));
    return lagrange2_f64_noalloc(job, ctx->stream, C, n, H, cj12, ck12, nbf5, nalpha, nbeta, elag, H_mat,
                                 E_elec);
}
