// Symmetric eigen-decomposition on the device for Iaux (src/integrals.jl:68-91,
// ext/DoNOFGPUExt.jl:9-33: eigen(Symmetric(G))) by the parallel cyclic
// Jacobi method: two-sided plane rotations on disjoint index pairs, the pairs
// of a round chosen by the round-robin (circle) ordering of Brent and Luk
// (J. Sci. Stat. Comput. 6, 1985), the rotation angle by Rutishauser's formulas
// (t = sign(theta) / (|theta| + sqrt(1 + theta^2)), theta = (a_qq - a_pp) / (2 a_pq)),
// and a pair skipped when |a_pq| <= eps sqrt(|a_pp a_qq|) (the relative test of
// Demmel and Veselic).  A sweep is npad - 1 rounds (npad = n rounded up to
// even; with n odd, index n is a dummy whose pair is skipped); the iteration
// stops after the first sweep that rotates no pair.
//
// One cooperative kernel runs every sweep.  Per round: phase A computes the
// rotation of each pair (one thread per pair) and counts the rotations of the
// sweep; after a grid barrier, phase B updates A two-sided block by block --
// the 2 x 2 block of rows {p1, q1} and columns {p2, q2} becomes
// R1^T A_blk R2, the diagonal blocks by the closed form a_pp - t a_pq,
// a_qq + t a_pq, 0 -- and the column pairs of V (V <- V J); a second grid
// barrier ends the round.  Every barrier is bounded (dtile.cuh); a sweep
// count above the limit is reported as non-convergence.
#include <math.h>

#include "dtile.cuh"
#include "kernels.cuh"

namespace donof {

namespace {

constexpr int EIG_THREADS = 256;
constexpr int EIG_MAX_SWEEPS = 40;
constexpr double EIG_EPS = 2.220446049250313e-16;

struct Rot {
    int p, q;       // q >= n: no rotation (dummy index)
    int active;     // rotated in this round
    int pad;
    double c, s, t;
};

struct EigState {
    dtile::GridSync gs;
    int rotations[EIG_MAX_SWEEPS];  // per sweep, zeroed before the launch
    int sweeps;                     // sweeps run, the last one without a rotation
    int converged;
};

struct EigArgs {
    double* A;      // n x n, symmetric (both triangles), overwritten: diagonal = eigenvalues
    double* V;      // n x n eigenvectors (columns), starts as the identity
    Rot* rot;       // npad / 2
    EigState* st;
    int n, npad;
    dtile::WaitCtl wc;
};

// Index at position pos of round r of the circle ordering (position 0 fixed).
__device__ __forceinline__ int circle(int pos, int r, int npad) {
    return pos == 0 ? 0 : 1 + (pos - 1 + r) % (npad - 1);
}

__global__ void __launch_bounds__(EIG_THREADS) jacobi_kernel(const EigArgs a) {
    const int n = a.n, npad = a.npad, P = npad / 2;
    const long long ln = n;
    double* A = a.A;
    double* V = a.V;
    unsigned epoch = 0;
    const unsigned members = gridDim.x;
    const long long gtid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long gstride = (long long)gridDim.x * blockDim.x;
    __shared__ int block_rot;
    int sweep = 0;
    bool ok = true, done = false;
    for (; sweep < EIG_MAX_SWEEPS && ok && !done; ++sweep) {
        for (int r = 0; r < npad - 1 && ok; ++r) {
            // ---- phase A: the rotation of every pair of this round
            if (threadIdx.x == 0) block_rot = 0;
            __syncthreads();
            for (long long k = gtid; k < P; k += gstride) {
                const int i0 = circle((int)k, r, npad), i1 = circle(npad - 1 - (int)k, r, npad);
                Rot R;
                R.p = i0 < i1 ? i0 : i1;
                R.q = i0 < i1 ? i1 : i0;
                R.active = 0;
                R.c = 1.0;
                R.s = 0.0;
                R.t = 0.0;
                if (R.q < n) {
                    const double app = A[R.p + ln * R.p], aqq = A[R.q + ln * R.q], apq = A[R.p + ln * R.q];
                    if (apq != 0.0 && fabs(apq) > EIG_EPS * sqrt(fabs(app * aqq))) {
                        const double th = (aqq - app) / (2.0 * apq);
                        const double t = (th >= 0.0 ? 1.0 : -1.0) / (fabs(th) + sqrt(1.0 + th * th));
                        R.c = 1.0 / sqrt(1.0 + t * t);
                        R.s = t * R.c;
                        R.t = t;
                        R.active = 1;
                        atomicAdd(&block_rot, 1);
                    }
                }
                a.rot[k] = R;
            }
            __syncthreads();
            if (threadIdx.x == 0 && block_rot) atomicAdd(&a.st->rotations[sweep], block_rot);
            if (!dtile::grid_barrier(&a.st->gs, epoch, members, a.wc)) { ok = false; break; }
            // ---- phase B: A <- J^T A J by 2 x 2 blocks (pairs k2 <= k1), V <- V J
            const long long nblk = (long long)P * (P + 1) / 2;
            for (long long idx = gtid; idx < nblk; idx += gstride) {
                // idx -> (k1, k2) with k2 <= k1, row by row over the lower triangle of pairs
                int k1 = (int)((sqrtf(8.0f * (float)idx + 1.0f) - 1.0f) * 0.5f);  // then corrected exactly
                while ((long long)(k1 + 1) * (k1 + 2) / 2 <= idx) ++k1;
                while ((long long)k1 * (k1 + 1) / 2 > idx) --k1;
                const int k2 = (int)(idx - (long long)k1 * (k1 + 1) / 2);  // k2 <= k1
                const Rot R1 = a.rot[k2], R2 = a.rot[k1];                   // R1: rows, R2: columns
                if (!R1.active && !R2.active) continue;
                if (k1 == k2) {
                    // diagonal block: closed form
                    const long long pp = R1.p + ln * R1.p, qq = R1.q + ln * R1.q, pq = R1.p + ln * R1.q,
                                    qp = R1.q + ln * R1.p;
                    const double apq = A[pq];
                    A[pp] -= R1.t * apq;
                    A[qq] += R1.t * apq;
                    A[pq] = 0.0;
                    A[qp] = 0.0;
                    continue;
                }
                const bool q1ok = R1.q < n, q2ok = R2.q < n;
                const double x00 = A[R1.p + ln * R2.p];
                const double x01 = q2ok ? A[R1.p + ln * R2.q] : 0.0;
                const double x10 = q1ok ? A[R1.q + ln * R2.p] : 0.0;
                const double x11 = (q1ok && q2ok) ? A[R1.q + ln * R2.q] : 0.0;
                // M = X J2, then Y = J1^T M  (J = [[c, s], [-s, c]] on {p, q})
                const double m00 = x00 * R2.c - x01 * R2.s, m01 = x00 * R2.s + x01 * R2.c;
                const double m10 = x10 * R2.c - x11 * R2.s, m11 = x10 * R2.s + x11 * R2.c;
                const double y00 = R1.c * m00 - R1.s * m10, y01 = R1.c * m01 - R1.s * m11;
                const double y10 = R1.s * m00 + R1.c * m10, y11 = R1.s * m01 + R1.c * m11;
                A[R1.p + ln * R2.p] = y00;
                A[R2.p + ln * R1.p] = y00;
                if (q2ok) {
                    A[R1.p + ln * R2.q] = y01;
                    A[R2.q + ln * R1.p] = y01;
                }
                if (q1ok) {
                    A[R1.q + ln * R2.p] = y10;
                    A[R2.p + ln * R1.q] = y10;
                }
                if (q1ok && q2ok) {
                    A[R1.q + ln * R2.q] = y11;
                    A[R2.q + ln * R1.q] = y11;
                }
            }
            const long long nv = ln * P;
            for (long long idx = gtid; idx < nv; idx += gstride) {
                const int i = (int)(idx % ln), k = (int)(idx / ln);
                const Rot R = a.rot[k];
                if (!R.active) continue;
                double* vp = V + ln * R.p + i;
                double* vq = V + ln * R.q + i;
                const double x = *vp, y = *vq;
                *vp = R.c * x - R.s * y;
                *vq = R.s * x + R.c * y;
            }
            if (!dtile::grid_barrier(&a.st->gs, epoch, members, a.wc)) { ok = false; break; }
        }
        if (ok) done = *(volatile int*)&a.st->rotations[sweep] == 0;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.st->sweeps = sweep;
        a.st->converged = (ok && done) ? 1 : 0;
    }
}

// A = Symmetric(G) (upper triangle of the column-major G), V = identity.
__global__ void eig_init_kernel(const double* __restrict__ G, int n, double* __restrict__ A, double* __restrict__ V) {
    const long long total = (long long)n * n;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(idx % n), j = (int)(idx / n);
        A[idx] = (i <= j) ? G[idx] : G[j + (long long)n * i];
        V[idx] = (i == j) ? 1.0 : 0.0;
    }
}

__global__ void eig_diag_kernel(const double* __restrict__ A, int n, double* __restrict__ w) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        w[i] = A[i + (long long)n * i];
}

}  // namespace

size_t eigh_scratch_bytes(int n) {
    const int npad = n + (n & 1);
    return ((sizeof(EigState) + 255) / 256 + (sizeof(Rot) * (size_t)(npad / 2) + 255) / 256) * 256;
}

// Eigenvalues w (unsorted) and eigenvectors V (columns, n x n) of Symmetric(G)
// (the upper triangle of the column-major n x n device matrix G); A is n x n
// scratch, `scratch` eigh_scratch_bytes(n) of device memory.  Synchronises the
// stream; DONOF_ERR_STATE if the sweeps do not converge, DONOF_ERR_TIMEOUT if a
// grid barrier ran out.
int eigh_jacobi(donof_ctx* ctx, cudaStream_t st, const double* G, int n, double* A, double* V, double* w,
                void* scratch) {
    const int npad = n + (n & 1);
    EigState* es = static_cast<EigState*>(scratch);
    Rot* rot = reinterpret_cast<Rot*>(static_cast<char*>(scratch) + (sizeof(EigState) + 255) / 256 * 256);
    long long blocks = ((long long)n * n + 255) / 256;
    if (blocks > 8LL * ctx->sm_count) blocks = 8LL * ctx->sm_count;
    eig_init_kernel<<<(int)blocks, 256, 0, st>>>(G, n, A, V); count_launch();
    DONOF_CUDA(ctx, cudaGetLastError());
    DONOF_CUDA(ctx, cudaMemsetAsync(es, 0, sizeof(EigState), st));
    int per_sm = 0;
    DONOF_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, jacobi_kernel, EIG_THREADS, 0));
    if (per_sm < 1) {
        set_error(ctx, "jacobi_kernel does not fit on an SM");
        return DONOF_ERR_CUDA;
    }
    int grid = ctx_ctas(ctx);  // at most one CTA per SM: co-resident (the kernel has grid barriers)
    const long long work = (long long)(npad / 2) * (npad / 2 + 1) / 2;
    if (grid > (work + EIG_THREADS - 1) / EIG_THREADS) grid = (int)((work + EIG_THREADS - 1) / EIG_THREADS);
    if (grid < 1) grid = 1;
    EigArgs a{A, V, rot, es, n, npad, dtile::wait_ctl(ctx)};
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(EIG_THREADS);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    DONOF_CUDA(ctx, cudaLaunchKernelEx(&cfg, jacobi_kernel, a));
    count_launch();
    eig_diag_kernel<<<(n + 255) / 256, 256, 0, st>>>(A, n, w); count_launch();
    DONOF_CUDA(ctx, cudaGetLastError());
    int hs[2] = {0, 0};
    DONOF_CUDA(ctx, cudaMemcpyAsync(hs, &es->sweeps, sizeof(hs), cudaMemcpyDeviceToHost, st));
    DONOF_CHECK(sync_and_check(ctx));
    if (!hs[1]) {
        set_error(ctx, "Jacobi eigen-decomposition of G did not converge in %d sweeps", hs[0]);
        return DONOF_ERR_STATE;
    }
    return DONOF_OK;
}

}  // namespace donof
