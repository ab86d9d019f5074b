// Orbital optimisers on the device: gradient packing and the AMSGrad-style
// updates of orbopt_adam / orbopt_adabelief / orbopt_yogi / orbopt_demon
// (src/minimization.jl:242-630), plus the optimiser loop itself.
#include <math.h>
#include <string.h>

#include <vector>

#include "kernels.cuh"
#include <type_traits>

#include "orbupd.cuh"

namespace donof {

namespace {

__device__ __forceinline__ long long packed_row_start(int i, int nbf) {
    return (long long)i * (nbf - 1) - (long long)i * (i - 1) / 2;
}

// g[k] = 4 elag[i,j] - 4 elag[j,i] for the k-th pair (i < nbf5, j > i),
// row-wise (src/pnof.jl:1395-1403).  One thread per packed entry; the pair
// is recovered from k by walking rows (nbf5 <= a few hundred).
__global__ void pack_grad_kernel(const double* __restrict__ elag, int nbf, int nbf5,
                                 double* __restrict__ g, unsigned long long* maxabs,
                                 const int* done) {
    if (done != nullptr && *done) return;
    const long long nvar = (long long)nbf5 * nbf - (long long)nbf5 * (nbf5 + 1) / 2;
    double local = 0.0;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nvar;
         k += (long long)gridDim.x * blockDim.x) {
        // row i: largest i with packed_row_start(i) <= k
        int lo = 0, hi = nbf5 - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (packed_row_start(mid, nbf) <= k) lo = mid; else hi = mid - 1;
        }
        const int i = lo;
        const int j = (int)(k - packed_row_start(i, nbf)) + i + 1;
        const double v = 4.0 * elag[i + (long long)nbf * j] - 4.0 * elag[j + (long long)nbf * i];
        g[k] = v;
        local = fmax(local, fabs(v));
    }
    if (maxabs != nullptr) {
        for (int o = 16; o > 0; o >>= 1) local = fmax(local, __shfl_xor_sync(0xffffffffu, local, o));
        if ((threadIdx.x & 31) == 0) atomicMax(maxabs, (unsigned long long)__double_as_longlong(local));
    }
}

struct UpdCoef {
    double beta1, beta2, bc1, bc2, alpha;  // bc = 1 - beta^i
};

// AMSGrad-style update shared by the four methods; `method` picks the second
// moment rule (src/minimization.jl:310-316, 406-411, 503-508, 598-603).
__global__ void update_kernel(int method, long long nvar, const double* __restrict__ g,
                              double* __restrict__ m, double* __restrict__ v,
                              double* __restrict__ vmax, double* __restrict__ y, UpdCoef c,
                              const int* done) {
    if (done != nullptr && *done) return;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nvar;
         k += (long long)gridDim.x * blockDim.x) {
        const double gk = g[k];
        const double mk = c.beta1 * m[k] + (1.0 - c.beta1) * gk;
        double vk;
        if (method == DONOF_ORB_ADABELIEF) {
            const double d = gk - mk;
            vk = c.beta2 * v[k] + (1.0 - c.beta2) * (d * d);
        } else if (method == DONOF_ORB_YOGI) {
            const double g2 = gk * gk;
            const double dv = v[k] - g2;
            const double sg = (dv > 0.0) ? 1.0 : ((dv < 0.0) ? -1.0 : 0.0);
            vk = v[k] - (1.0 - c.beta2) * sg * g2;
        } else {
            vk = c.beta2 * v[k] + (1.0 - c.beta2) * (gk * gk);
        }
        const double mhat = mk / c.bc1;
        const double vhat = vk / c.bc2;
        const double vm = fmax(vmax[k], vhat);
        m[k] = mk;
        v[k] = vk;
        vmax[k] = vm;
        y[k] = -c.alpha * mhat / sqrt(vm + 1e-16);
    }
}

int nblocks(long long total, int sm) {
    long long b = (total + 255) / 256;
    if (b > 4LL * sm) b = 4LL * sm;
    return (int)(b < 1 ? 1 : b);
}

}  // namespace

int pack_grad(donof_ctx* ctx, cudaStream_t st, const double* elag, int nbf, int nbf5, double* g,
              unsigned long long* maxabs_bits) {
    const long long nvar = nvar_of(nbf, nbf5);
    pack_grad_kernel<<<nblocks(nvar, ctx->sm_count), 256, 0, st>>>(elag, nbf, nbf5, g, maxabs_bits,
                                                                   nullptr); count_launch();
    DONOF_CUDA(ctx, cudaGetLastError());
    return DONOF_OK;
}

// ---------------------------------------------------------------------------
// Graph form of the optimiser loop: one CUDA graph whose conditional WHILE
// node repeats the iteration body (update, rotation, Lagrangian, gradient,
// best-E bookkeeping) on the device; the body's last kernel evaluates the
// reference's stopping rule and clears the loop condition.  The host launches
// the graph once per orbopt call and reads the final state once.
// ---------------------------------------------------------------------------
namespace {

struct OrbState {
    double E, bestE, alpha, thresh;
    unsigned long long gmax_bits;  // max|g| of the latest gradient, as the bits of a non-negative double
    int it, maxloop, method, improved, improved_now, success, nit, pad;
};

// update of the AMSGrad family with the iteration count and step size read
// from the device state (src/minimization.jl:307-316, 406-411, 503-508, 598-603);
// it also clears max|g| for the gradient this iteration reduces (the first
// node of the iteration, so no memset node is needed)
__global__ void orb_update_kernel(OrbState* __restrict__ s, long long nvar, const double* __restrict__ g,
                                  double* __restrict__ m, double* __restrict__ v, double* __restrict__ vmax,
                                  double* __restrict__ y) {
    const orbupd::Coef c = orbupd::coef(s->method, s->it + 1, s->maxloop, s->alpha);
    if (blockIdx.x == 0 && threadIdx.x == 0) s->gmax_bits = 0ull;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nvar;
         k += (long long)gridDim.x * blockDim.x)
        orbupd::step(c, k, g, m, v, vmax, y);
}

// End of iteration it+1: best-E tracking and the stopping rule evaluated at the
// start of the next iteration in the reference (src/minimization.jl:387-422).
__global__ void orb_end_kernel(OrbState* s, cudaGraphConditionalHandle h) {
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
    cudaGraphSetConditional(h, stop ? 0u : 1u);
}

// The rotated orbitals become the current ones, and the best ones when this
// iteration improved E (one pass over C_new for both copies).
__global__ void copy_step_kernel(const double* __restrict__ src, double* __restrict__ cur, double* __restrict__ best,
                                 long long count, const int* flag) {
    const bool improved = *flag != 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x) {
        const double v = src[i];
        cur[i] = v;
        if (improved) best[i] = v;
    }
}

}  // namespace

int orbopt_run_host(donof_job* job, int method, const double* n, const double* cj12, const double* ck12,
                    const double* H, int nbf5, int nalpha, int nbeta, double* alpha, int* maxloop,
                    double threshgorb, double* C, double* E_out, int* nit_out, int* success_out, int precision);

int orbopt_run(donof_job* job, int method, const double* n, const double* cj12, const double* ck12,
               const double* H, int nbf5, int nalpha, int nbeta, double* alpha, int* maxloop,
               double threshgorb, double* C, double* E_out, int* nit_out, int* success_out,
               int precision) {
    const char* env = getenv("DONOF_ORBOPT_HOST_LOOP");
    if (env && env[0] == '1')
        return orbopt_run_host(job, method, n, cj12, ck12, H, nbf5, nalpha, nbeta, alpha, maxloop, threshgorb, C,
                               E_out, nit_out, success_out, precision);
    donof_ctx* ctx = job->ctx;
    cudaStream_t st = ctx->stream;
    if (st == nullptr || st == cudaStreamLegacy) {
        // the legacy default stream cannot be captured: run this synchronous
        // call on a private stream, ordered after the work already queued
        if (!ctx->aux_stream) DONOF_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->aux_stream, cudaStreamNonBlocking));
        DONOF_CUDA(ctx, cudaStreamSynchronize(st));
        st = ctx->aux_stream;
    }
    struct ProfileOff {  // event records are not allowed in a conditional body
        donof_ctx* c;
        bool was;
        ~ProfileOff() { c->profile = was; }
    } profile_off{ctx, ctx->profile};
    ctx->profile = false;
    const int nbf = job->nbf;
    const long long nvar = nvar_of(nbf, nbf5);
    const long long nn = (long long)nbf * nbf;
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o = off; off += (bytes + 255) / 256 * 256; return o; };
    const size_t o_m = take(8 * nvar), o_v = take(8 * nvar), o_vm = take(8 * nvar), o_y = take(8 * nvar),
                 o_g = take(8 * nvar);
    const size_t o_C = take(8 * nn), o_Cn = take(8 * nn), o_best = take(8 * nn), o_elag = take(8 * nn);
    const size_t o_H = take(8 * (size_t)nbf * nbf5), o_st = take(sizeof(OrbState));
    DONOF_CHECK(job->orb.ensure(ctx, off));
    DONOF_CHECK(ctx->rot.ensure(ctx, rotate_scratch_bytes(nbf)));
    char* base = job->orb.as<char>();
    double* m = (double*)(base + o_m);
    double* v = (double*)(base + o_v);
    double* vm = (double*)(base + o_vm);
    double* y = (double*)(base + o_y);
    double* g = (double*)(base + o_g);
    double* Ccur = (double*)(base + o_C);
    double* Cnew = (double*)(base + o_Cn);
    double* Cbest = (double*)(base + o_best);
    double* elag = (double*)(base + o_elag);
    double* Hmat = (double*)(base + o_H);
    OrbState* S = (OrbState*)(base + o_st);

    auto lagr = [&](const double* Cin) -> int {
        if (precision == DONOF_PREC_MIXED)
            return lagrange2_mixed(job, st, Cin, n, H, cj12, ck12, nbf5, nalpha, nbeta, elag, Hmat, &S->E);
        return lagrange2_f64(job, st, Cin, n, H, cj12, ck12, nbf5, nalpha, nbeta, elag, Hmat, &S->E);
    };
    auto grad = [&]() -> int {
        DONOF_CUDA(ctx, cudaMemsetAsync(&S->gmax_bits, 0, sizeof(unsigned long long), st));
        return pack_grad(ctx, st, elag, nbf, nbf5, g, &S->gmax_bits);
    };

    // initial evaluation (also sizes every scratch buffer the graph will use)
    DONOF_CUDA(ctx, cudaMemsetAsync(base + o_m, 0, o_y - o_m, st));  // m, v, vmax = 0
    DONOF_CUDA(ctx, cudaMemcpyAsync(Ccur, C, sizeof(double) * nn, cudaMemcpyDeviceToDevice, st));
    DONOF_CHECK(lagr(Ccur));
    DONOF_CHECK(grad());
    DONOF_CUDA(ctx, cudaMemcpyAsync(Cbest, Ccur, sizeof(double) * nn, cudaMemcpyDeviceToDevice, st));
    OrbState hs{};
    DONOF_CUDA(ctx, cudaMemcpyAsync(&hs, S, sizeof(OrbState), cudaMemcpyDeviceToHost, st));
    DONOF_CUDA(ctx, cudaStreamSynchronize(st));
    DONOF_CHECK(failure_status(ctx));
    const double E0 = hs.E;
    hs.bestE = E0;
    hs.alpha = *alpha;
    hs.thresh = threshgorb;
    hs.it = 0;
    hs.maxloop = *maxloop;
    hs.method = method;
    hs.improved = hs.improved_now = hs.success = hs.nit = 0;
    DONOF_CUDA(ctx, cudaMemcpyAsync(S, &hs, sizeof(OrbState), cudaMemcpyHostToDevice, st));

    if (*maxloop >= 1) {
        // (re)build the graph when its inputs or any buffer it references changed
        const unsigned long long gens = (unsigned long long)job->tmp.gen + job->bpq.gen + job->W.gen + job->part.gen +
                                        job->small.gen + job->orb.gen + ctx->rot.gen + job->oz_c.gen +
                                        ((unsigned long long)job->oz_gen << 32);
        const unsigned long long key[10] = {(unsigned long long)(uintptr_t)n, (unsigned long long)(uintptr_t)cj12,
                                            (unsigned long long)(uintptr_t)ck12, (unsigned long long)(uintptr_t)H,
                                            (unsigned long long)nbf5 | ((unsigned long long)nalpha << 20) |
                                                ((unsigned long long)nbeta << 40),
                                            (unsigned long long)method | ((unsigned long long)ctx_ctas(ctx) << 8),
                                            (unsigned long long)precision, gens,
                                            (unsigned long long)(uintptr_t)base, (unsigned long long)(uintptr_t)st};
        bool valid = job->orb_exec != nullptr;
        for (int k = 0; k < 10 && valid; ++k) valid = (job->orb_key[k] == key[k]);
        if (!valid) {
            if (job->orb_exec) cudaGraphExecDestroy(job->orb_exec);
            if (job->orb_graph) cudaGraphDestroy(job->orb_graph);
            job->orb_exec = nullptr;
            job->orb_graph = nullptr;
            cudaGraph_t graph = nullptr;
            DONOF_CUDA(ctx, cudaGraphCreate(&graph, 0));
            job->orb_graph = graph;
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
            DONOF_CUDA(ctx, cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0,
                                                          cudaStreamCaptureModeThreadLocal));
            int rc = DONOF_OK;
            do {
                orb_update_kernel<<<nblocks(nvar, ctx->sm_count), 256, 0, st>>>(S, nvar, g, m, v, vm, y); count_launch();
                if ((rc = rotate_f64(ctx, st, y, nbf, nbf5, Ccur, Cnew)) != DONOF_OK) break;
                if ((rc = lagr(Cnew)) != DONOF_OK) break;
                // max|g| was cleared by orb_update_kernel
                if ((rc = pack_grad(ctx, st, elag, nbf, nbf5, g, &S->gmax_bits)) != DONOF_OK) break;
                orb_end_kernel<<<1, 1, 0, st>>>(S, handle); count_launch();
                copy_step_kernel<<<nblocks(nn, ctx->sm_count), 256, 0, st>>>(Cnew, Ccur, Cbest, nn, &S->improved_now);
                count_launch();
            } while (false);
            cudaGraph_t captured = nullptr;
            const cudaError_t ce = cudaStreamEndCapture(st, &captured);
            if (rc != DONOF_OK) return rc;
            if (ce != cudaSuccess) {
                set_error(ctx, "capture of the optimiser body: %s", cudaGetErrorString(ce));
                return DONOF_ERR_CUDA;
            }
            job->orb_per_iter = (int)(donof_launch_count() - l0);
            // the capture counted the body's launches once; replays are counted below
            g_launch_adjust(-(long long)job->orb_per_iter);
            cudaGraphExec_t exec = nullptr;
            DONOF_CUDA(ctx, cudaGraphInstantiate(&exec, graph, 0));
            job->orb_exec = exec;
            for (int k = 0; k < 10; ++k) job->orb_key[k] = key[k];
        }
        DONOF_CUDA(ctx, cudaGraphLaunch(job->orb_exec, st));
        DONOF_CUDA(ctx, cudaMemcpyAsync(&hs, S, sizeof(OrbState), cudaMemcpyDeviceToHost, st));
        DONOF_CUDA(ctx, cudaStreamSynchronize(st));
        DONOF_CHECK(failure_status(ctx));
        g_launch_adjust((long long)job->orb_per_iter * hs.it);
    }
    if (!hs.improved) {
        *alpha = 0.3 * (*alpha);
        *maxloop = *maxloop + 10;
    }
    const bool return_best = (*maxloop < 100);
    DONOF_CUDA(ctx, cudaMemcpyAsync(C, return_best ? Cbest : Ccur, sizeof(double) * nn, cudaMemcpyDeviceToDevice, st));
    *E_out = return_best ? hs.bestE : hs.E;
    *nit_out = hs.nit;
    *success_out = hs.success;
    return DONOF_OK;
}

// Host-driven form of the same loop (one 16-byte read per iteration); kept as
// a reference execution mode, selected with DONOF_ORBOPT_HOST_LOOP=1.
int orbopt_run_host(donof_job* job, int method, const double* n, const double* cj12, const double* ck12,
                    const double* H, int nbf5, int nalpha, int nbeta, double* alpha, int* maxloop,
                    double threshgorb, double* C, double* E_out, int* nit_out, int* success_out,
                    int precision) {
    donof_ctx* ctx = job->ctx;
    cudaStream_t st = ctx->stream;
    const int nbf = job->nbf;
    const long long nvar = nvar_of(nbf, nbf5);
    const long long nn = (long long)nbf * nbf;
    // layout of the optimiser state
    size_t off = 0;
    auto take = [&](size_t count) { size_t o = off; off += ((count * sizeof(double) + 255) / 256) * 256; return o; };
    const size_t o_m = take(nvar), o_v = take(nvar), o_vm = take(nvar), o_y = take(nvar), o_g = take(nvar);
    const size_t o_C = take(nn), o_Cn = take(nn), o_best = take(nn), o_elag = take(nn);
    const size_t o_H = take((size_t)nbf * nbf5), o_stat = take(4);
    DONOF_CHECK(job->orb.ensure(ctx, off));
    char* base = job->orb.as<char>();
    double* m = (double*)(base + o_m);
    double* v = (double*)(base + o_v);
    double* vm = (double*)(base + o_vm);
    double* y = (double*)(base + o_y);
    double* g = (double*)(base + o_g);
    double* Ccur = (double*)(base + o_C);
    double* Cnew = (double*)(base + o_Cn);
    double* Cbest = (double*)(base + o_best);
    double* elag = (double*)(base + o_elag);
    double* Hmat = (double*)(base + o_H);
    double* stat = (double*)(base + o_stat);  // [0] = E, [1] = max|g| bits
    DONOF_CUDA(ctx, cudaMemsetAsync(base + o_m, 0, o_y - o_m, st));  // m, v, vmax = 0

    auto lagr = [&](const double* Cin) -> int {
        if (precision == DONOF_PREC_MIXED)
            return lagrange2_mixed(job, st, Cin, n, H, cj12, ck12, nbf5, nalpha, nbeta, elag, Hmat, stat);
        return lagrange2_f64(job, st, Cin, n, H, cj12, ck12, nbf5, nalpha, nbeta, elag, Hmat, stat);
    };
    auto eval = [&](const double* Cin, double* E, double* gmax) -> int {
        DONOF_CHECK(lagr(Cin));
        DONOF_CUDA(ctx, cudaMemsetAsync(stat + 1, 0, sizeof(double), st));
        DONOF_CHECK(pack_grad(ctx, st, elag, nbf, nbf5, g, (unsigned long long*)(stat + 1)));
        double h[2];
        DONOF_CUDA(ctx, cudaMemcpyAsync(h, stat, sizeof(h), cudaMemcpyDeviceToHost, st));
        DONOF_CUDA(ctx, cudaStreamSynchronize(st));
        DONOF_CHECK(failure_status(ctx));
        *E = h[0];
        *gmax = h[1];
        return DONOF_OK;
    };

    DONOF_CUDA(ctx, cudaMemcpyAsync(Ccur, C, sizeof(double) * nn, cudaMemcpyDeviceToDevice, st));
    double E = 0.0, gmax = 0.0;
    DONOF_CHECK(eval(Ccur, &E, &gmax));
    double bestE = E;
    DONOF_CUDA(ctx, cudaMemcpyAsync(Cbest, Ccur, sizeof(double) * nn, cudaMemcpyDeviceToDevice, st));

    const double a = *alpha;
    double beta1 = (method == DONOF_ORB_DEMON) ? 0.6 : 0.5;
    const double beta2 = (method == DONOF_ORB_DEMON) ? 0.999 : 0.9;
    const double binit = beta1;
    const int loops = *maxloop;
    bool improved = false, success = false;
    int nit = 0;
    for (int i = 1; i <= loops; ++i) {
        ++nit;
        if (2.0 * gmax < threshgorb && improved) {
            success = true;
            break;
        }
        if (method == DONOF_ORB_DEMON) {
            const double rate = (i - 1.0) / (loops - 1.0);
            beta1 = binit * (1.0 - rate) / ((1.0 - binit) + binit * (1.0 - rate));
        }
        UpdCoef c{beta1, beta2, 1.0 - pow(beta1, i), 1.0 - pow(beta2, i), a};
        update_kernel<<<nblocks(nvar, ctx->sm_count), 256, 0, st>>>(method, nvar, g, m, v, vm, y, c, nullptr); count_launch();
        DONOF_CUDA(ctx, cudaGetLastError());
        DONOF_CHECK(rotate_f64(ctx, st, y, nbf, nbf5, Ccur, Cnew));
        double* t = Ccur; Ccur = Cnew; Cnew = t;
        DONOF_CHECK(eval(Ccur, &E, &gmax));
        if (E < bestE) {
            bestE = E;
            DONOF_CUDA(ctx, cudaMemcpyAsync(Cbest, Ccur, sizeof(double) * nn, cudaMemcpyDeviceToDevice, st));
            improved = true;
        }
    }
    if (!improved) {
        *alpha = 0.3 * (*alpha);
        *maxloop = *maxloop + 10;
    }
    const bool return_best = (*maxloop < 100);
    DONOF_CUDA(ctx, cudaMemcpyAsync(C, return_best ? Cbest : Ccur, sizeof(double) * nn,
                                    cudaMemcpyDeviceToDevice, st));
    *E_out = return_best ? bestE : E;
    *nit_out = nit;
    *success_out = success ? 1 : 0;
    return DONOF_OK;
}

}  // namespace donof

// The host side of one optimiser iteration (src/minimization.jl:390-412, which
// the reference runs on the host between its GPU calls): calcorbg's packing of
// 4 (elag - elag^T) and the update of the AMSGrad family, with the same
// per-element arithmetic as the device loop (orbupd.cuh).
extern "C" int donof_orb_step_host(int method, int it, int maxloop, double alpha, const double* elag, int nbf,
                                   int nbf5, double* g, double* m, double* v, double* vmax, double* y,
                                   double* gmax) {
    if (!elag || !g || !m || !v || !vmax || !y || nbf < 1 || nbf5 < 1 || nbf5 > nbf || it < 1 ||
        method < DONOF_ORB_ADAM || method > DONOF_ORB_DEMON || (method == DONOF_ORB_DEMON && maxloop < 2)) {
        donof::set_error(nullptr, "donof_orb_step_host: invalid arguments");
        return DONOF_ERR_ARG;
    }
    // rows i of the packing in groups of 8: for each column j the group's
    // elag[i + nbf j] share a cache line and elag[j + nbf i], g run along j
    double mx = 0.0;
    auto start = [nbf](long long i) { return i * (nbf - 1) - i * (i - 1) / 2; };  // first k of row i
    for (int i0 = 0; i0 < nbf5; i0 += 8) {
        const int i1 = i0 + 8 < nbf5 ? i0 + 8 : nbf5;
        for (int j = i0 + 1; j < nbf; ++j) {
            const double* col = elag + (long long)nbf * j;
            for (int i = i0; i < i1 && i < j; ++i) {
                const double val = 4.0 * col[i] - 4.0 * elag[j + (long long)nbf * i];
                g[start(i) + (j - i - 1)] = val;
                mx = fmax(mx, fabs(val));
            }
        }
    }
    const long long nvar = start(nbf5);
    const donof::orbupd::Coef c = donof::orbupd::coef(method, it, maxloop, alpha);
    // one loop per method, so that the per-element branch on it folds away; the
    // bias corrections as reciprocals (one division and one square root per
    // element; within an ulp of orbupd::step)
    auto run = [&](auto tag) {
        constexpr int M = decltype(tag)::value;
        const double b1 = c.beta1, b2 = c.beta2, ib1 = 1.0 / c.bc1, ib2 = 1.0 / c.bc2, a = c.alpha;
        double* __restrict__ mm = m;
        double* __restrict__ vv = v;
        double* __restrict__ vx = vmax;
        double* __restrict__ yy = y;
        const double* __restrict__ gg = g;
        for (long long q = 0; q < nvar; ++q) {
            const double gk = gg[q];
            const double mk = b1 * mm[q] + (1.0 - b1) * gk;
            double vk;
            if (M == DONOF_ORB_ADABELIEF) {
                const double dd = gk - mk;
                vk = b2 * vv[q] + (1.0 - b2) * (dd * dd);
            } else if (M == DONOF_ORB_YOGI) {
                const double g2 = gk * gk, dv = vv[q] - g2;
                vk = vv[q] - (1.0 - b2) * ((dv > 0.0) ? g2 : ((dv < 0.0) ? -g2 : 0.0));
            } else {
                vk = b2 * vv[q] + (1.0 - b2) * (gk * gk);
            }
            const double vh = vk * ib2, vo = vx[q];
            const double vm = (vo > vh) ? vo : vh;
            mm[q] = mk;
            vv[q] = vk;
            vx[q] = vm;
            yy[q] = -a * (mk * ib1) / sqrt(vm + 1e-16);
        }
    };
    switch (method) {
        case DONOF_ORB_ADABELIEF: run(std::integral_constant<int, DONOF_ORB_ADABELIEF>{}); break;
        case DONOF_ORB_YOGI: run(std::integral_constant<int, DONOF_ORB_YOGI>{}); break;
        case DONOF_ORB_DEMON: run(std::integral_constant<int, DONOF_ORB_DEMON>{}); break;
        default: run(std::integral_constant<int, DONOF_ORB_ADAM>{}); break;
    }
    if (gmax) *gmax = mx;
    return DONOF_OK;
}
