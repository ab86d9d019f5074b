// occoptr's minimisation over gamma on the GPU (donof_occ_cg_dev).
//
// The same Hager-Zhang conjugate gradient with a strong-Wolfe line search and
// the approximate-Wolfe acceptance as the host solver (occupation.cu), run by
// one CTA (a line search that finds no step along a conjugate direction is
// retried once from steepest descent before the solver stops): every evaluation of the occupation energy and gradient (calce /
// calcoccg, src/pnof.jl:1273-1377) is a few CTA-wide passes over the shared
// per-orbital formulas (occ_math.cuh) -- the occupations and dn blocks of the
// pairs, n_d and phi(n), the class-range row sums of J_MO / K_MO (one warp per
// orbital), the row energy terms and the pairs' gradient entries -- and the
// scalar control flow of the line search runs identically in every thread on
// values broadcast through shared memory.  Sums are reduced in a fixed order,
// so a call gives the same result every time; they are not summed in the host
// solver's order, so the two agree to rounding.
//
// Every loop is bounded (max_iter iterations, 30 line-search and 30 zoom
// steps); there is no wait on another CTA.  J_MO, K_MO, H_core, gamma and the
// result live in device memory; the index tables travel in the kernel
// argument, so the call allocates nothing.
#include <math.h>

#include <atomic>

#include "kernels.cuh"
#include "occ.cuh"
#include "occ_math.cuh"

namespace donof {
namespace occ {
namespace {

constexpr int NT = 256;               // threads of the solver's CTA
constexpr int NW = NT / 32;
constexpr int MAX_N = 1024;           // nbf5
constexpr int MAX_PAIR = 512;         // ndoc
constexpr int MAX_PV = 2048;          // ndoc * ncwo
constexpr int CACHE = 64;             // line-search points kept (a, f, da)
constexpr size_t OCC_SMEM_MAX = 220 * 1024;  // dynamic shared memory of the largest solver launch

struct Tables {
    int S[MAX_PAIR];
    int P[MAX_PV], G[MAX_PV], KG[MAX_PV];
    int grp[MAX_N];
};

struct CgArgs {
    int N, no1, ndoc, nsoc, nbeta, nalpha, ncwo, nv, ista, high_spin, method;
    double h_cut;
    const double *J, *K, *Hc;
    double* gamma;      // in/out
    double* result;     // [0] E, [1] iterations, [2] converged, [3, 3 + nv) the gradient
    double g_abstol;
    int max_iter;
};

struct Smem {
    OccView o;
    double *n, *fi, *nd12, *nd, *w, *F, *coc, *blk, *x, *d, *gx, *gt, *xa;
    RowSums* rs;
    double* red;    // 2 x NW x 3 per-warp partials (two buffers, used in turn)
    double *ca, *cf, *cd;  // line-search cache
    int* ncache;
    int rbuf;       // the red buffer of the next reduction (the same in every thread)
};

// Butterfly sum over a warp: every lane ends with the same value (each step
// adds two values that are each other's mirror, and a + b == b + a).
__device__ __forceinline__ double warp_allsum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_allmax(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Sums (or maxima) of up to three values over the CTA with one barrier: each
// warp's partials go to the current buffer, and every thread adds the warps'
// partials in the same order, so every thread gets the same result.  The two
// buffers alternate, so a buffer is written again only after the barrier of
// the next reduction, by which time every thread has read it.
template <int NVAL, bool MAX>
__device__ __forceinline__ void block_reduce(Smem& m, double (&v)[NVAL]) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double* buf = m.red + m.rbuf * (NW * 3);
#pragma unroll
    for (int k = 0; k < NVAL; ++k) v[k] = MAX ? warp_allmax(v[k]) : warp_allsum(v[k]);
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NVAL; ++k) buf[warp * 3 + k] = v[k];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NVAL; ++k) {
        double t = MAX ? buf[k] : 0.0;
        for (int i = MAX ? 1 : 0; i < NW; ++i) t = MAX ? fmax(t, buf[i * 3 + k]) : t + buf[i * 3 + k];
        v[k] = t;
    }
    m.rbuf ^= 1;
}

__device__ __forceinline__ double block_sum(Smem& m, double v) {
    double a[1] = {v};
    block_reduce<1, false>(m, a);
    return a[0];
}

__device__ __forceinline__ double block_max(Smem& m, double v) {
    double a[1] = {v};
    block_reduce<1, true>(m, a);
    return a[0];
}

__device__ double dot(Smem& m, const double* a, const double* b, int nv) {
    double s = 0.0;
    for (int k = threadIdx.x; k < nv; k += NT) s += a[k] * b[k];
    return block_sum(m, s);
}

__device__ double maxabs(Smem& m, const double* a, int nv) {
    double s = 0.0;
    for (int k = threadIdx.x; k < nv; k += NT) s = fmax(s, fabs(a[k]));
    return block_max(m, s);
}

// Occupation energy at gamma = xa and, with g != nullptr, its gradient (every thread gets E).
__device__ double eval(const CgArgs& A, Smem& m, const double* xa, double* g) {
    const OccView& o = m.o;
    const int N = o.N, nc = o.ncwo, nd = o.ndoc, tid = threadIdx.x;
    const double *J = A.J, *K = A.K;
    // occupations: orbitals outside the pairs, then each pair (pass 1); the dn
    // blocks and n_d (pass 2, which reads n of every pair)
    for (int i = tid; i < N; i += NT) {
        if (o.grp[i] < 0) {
            double v = 0.0;
            if (i < o.no1) v = 1.0;
            else if (i >= o.no1 + nd && i < o.no1 + nd + o.nsoc) v = o.high_spin ? 1.0 : 0.5;
            m.n[i] = v;
            m.nd[i] = 0.0;
        }
    }
    for (int gi = tid; gi < nd; gi += NT) pair_n(o, xa, gi, m.n);
    __syncthreads();
    for (int gi = tid; gi < nd; gi += NT) {
        pair_dn(o, xa, gi, m.n, m.blk + (size_t)gi * (nc + 1) * nc);
        pair_dynamic(o, m.n, gi, m.nd, m.F, m.coc);
    }
    __syncthreads();
    double part[3] = {0.0, 0.0, 0.0};  // linear terms, sum of the J rows, sum of the K rows
    for (int i = tid; i < N; i += NT) {
        m.fi[i] = phi_fn(m.n[i], o.ista);
        m.nd12[i] = sqrt(m.nd[i]);
        const double wi = 2.0 * A.Hc[i] + J[i + (size_t)N * i];
        m.w[i] = wi;
        if (i < o.nbeta || i >= o.nalpha) part[0] += m.n[i] * wi;
        else part[0] += 2.0 * m.n[i] * A.Hc[i];
    }
    __syncthreads();
    // class-range row sums and the row's energy terms, one thread per orbital
    const VecView vv{m.n, m.fi, m.nd12, m.nd, m.F, m.coc};
    {
        const int bnd[5] = {0, o.no1, o.nbeta, o.nalpha, N};
        for (int i = tid; i < N; i += NT) {
            const double* Kc = K + (size_t)N * i;
            const double* Jc = J + (size_t)N * i;
            RowSums& r = m.rs[i];
            for (int R = 0; R < 4; ++R) {
                double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0, a4 = 0.0;
                for (int j = bnd[R]; j < bnd[R + 1]; ++j) {
                    const double kj = Kc[j];
                    a0 += m.n[j] * kj;
                    a1 += m.fi[j] * kj;
                    a2 += m.nd12[j] * kj;
                    a3 += m.nd[j] * kj;
                    a4 += kj;
                }
                r.S[R][V_N] = a0; r.S[R][V_FI] = a1; r.S[R][V_ND12] = a2; r.S[R][V_ND] = a3; r.S[R][V_ONE] = a4;
            }
            double jn = 0.0;
            for (int j = 0; j < N; ++j) jn += m.n[j] * Jc[j];
            r.jn = jn;
            double rj, rk;
            row_energy(o, vv, i, r, J, K, &rj, &rk);
            part[1] += rj;
            part[2] += rk;
        }
    }
    block_reduce<3, false>(m, part);  // its barrier also publishes every row's sums
    const double E = part[0] + (part[1] - part[2]);
    if (g != nullptr) {
        // each gamma entry belongs to exactly one pair: the pair's thread sets it
        for (int gi = tid; gi < nd; gi += NT) {
            for (int c = 0; c < nc; ++c) g[o.KG[gi * nc + c]] = 0.0;
            pair_grad(o, vv, m.rs, J, K, m.w, m.blk + (size_t)gi * (nc + 1) * nc, gi, g);
        }
        __syncthreads();
    }
    return E;
}

struct Pt {
    double a, f, da;
};

// phi(a) = E(x + a d) with its gradient in m.gt (every call evaluates, so the
// point returned by the line search is always the last one evaluated and m.gt
// holds its gradient); the scalars are also kept for phi_f.
__device__ Pt phi(const CgArgs& A, Smem& m, double a) {
    const int nv = m.o.nv;
    for (int k = threadIdx.x; k < nv; k += NT) m.xa[k] = m.x[k] + a * m.d[k];
    __syncthreads();
    Pt p;
    p.a = a;
    p.f = eval(A, m, m.xa, m.gt);
    p.da = dot(m, m.gt, m.d, nv);
    if (threadIdx.x == 0 && *m.ncache < CACHE) {
        m.ca[*m.ncache] = a;
        m.cf[*m.ncache] = p.f;
        m.cd[*m.ncache] = p.da;
        *m.ncache += 1;
    }
    __syncthreads();
    return p;
}

// E(x + a d) only: from the points of this line search when a was evaluated
__device__ double phi_f(const CgArgs& A, Smem& m, double a) {
    const int nc = *m.ncache;
    for (int i = 0; i < nc; ++i)
        if (m.ca[i] == a) return m.cf[i];
    return phi(A, m, a).f;
}

__device__ bool decrease_ok(double fa, double da, double a, double f0, double d0, double c1) {
    if (fa <= f0 + c1 * a * d0) return true;
    return fa <= f0 + 1e-6 * fabs(f0) && da <= (2 * 0.1 - 1.0) * d0;
}

__device__ Pt zoom(const CgArgs& A, Smem& m, double a_lo, double a_hi, double f_lo, double d_lo, double f0,
                   double d0, double c1, double c2) {
    double f_hi = phi_f(A, m, a_hi);
    for (int it = 0; it < 30; ++it) {
        const double denom = 2.0 * (f_hi - f_lo - d_lo * (a_hi - a_lo));
        double a = denom > 0 ? a_lo - d_lo * (a_hi - a_lo) * (a_hi - a_lo) / denom : 0.5 * (a_lo + a_hi);
        const double lo = fmin(a_lo, a_hi), hi = fmax(a_lo, a_hi);
        if (!(lo + 0.1 * (hi - lo) <= a && a <= hi - 0.1 * (hi - lo))) a = 0.5 * (a_lo + a_hi);
        const Pt pa = phi(A, m, a);
        if (!decrease_ok(pa.f, pa.da, a, f0, d0, c1) || pa.f > f_lo + 1e-6 * fabs(f0)) {
            a_hi = a;
            f_hi = pa.f;
        } else {
            if (fabs(pa.da) <= -c2 * d0) return pa;
            if (pa.da * (a_hi - a_lo) >= 0) {
                a_hi = a_lo;
                f_hi = f_lo;
            }
            a_lo = a;
            f_lo = pa.f;
            d_lo = pa.da;
        }
    }
    return phi(A, m, a_lo);
}

__device__ Pt wolfe(const CgArgs& A, Smem& m, double fx, double d0, double a1) {
    const double c1 = 1e-4, c2 = 0.1, a_max = 1e6;
    if (threadIdx.x == 0) *m.ncache = 0;
    __syncthreads();
    double a_prev = 0.0, f_prev = fx, dp_prev = d0, a = a1;
    Pt pa{0.0, fx, d0};
    for (int i = 0; i < 30; ++i) {
        pa = phi(A, m, a);
        if (!decrease_ok(pa.f, pa.da, a, fx, d0, c1) || (i > 0 && pa.f > f_prev + 1e-6 * fabs(fx)))
            return zoom(A, m, a_prev, a, f_prev, dp_prev, fx, d0, c1, c2);
        if (fabs(pa.da) <= -c2 * d0) return pa;
        if (pa.da >= 0) return zoom(A, m, a, a_prev, pa.f, pa.da, fx, d0, c1, c2);
        a_prev = a;
        f_prev = pa.f;
        dp_prev = pa.da;
        a = fmin(2.0 * a, a_max);
    }
    return pa;
}

__global__ void __launch_bounds__(NT, 1) occ_cg_kernel(const __grid_constant__ Tables T, const CgArgs A) {
    extern __shared__ __align__(16) double sm[];
    const int tid = threadIdx.x;
    const int N = A.N, nv = A.nv, nd = A.ndoc, nc = A.ncwo;
    // shared-memory map (sizes checked on the host, occ_cg_smem_bytes)
    Smem m;
    double* p = sm;
    auto take = [&](size_t count) { double* q = p; p += (count + 1) & ~size_t(1); return q; };
    m.n = take(N); m.fi = take(N); m.nd12 = take(N); m.nd = take(N); m.w = take(N);
    m.F = take(nd); m.coc = take(nd);
    m.blk = take((size_t)nd * (nc + 1) * nc);
    m.x = take(nv); m.d = take(nv); m.gx = take(nv); m.gt = take(nv); m.xa = take(nv);
    m.rs = reinterpret_cast<RowSums*>(take((size_t)N * sizeof(RowSums) / sizeof(double)));
    m.red = take(2 * NW * 3);
    m.rbuf = 0;
    m.ca = take(CACHE); m.cf = take(CACHE); m.cd = take(CACHE);
    m.ncache = reinterpret_cast<int*>(take(2));
    int* tab = reinterpret_cast<int*>(p);
    int* S = tab;
    int* P = S + nd;
    int* G = P + nd * nc;
    int* KG = G + nd * nc;
    int* grp = KG + nd * nc;
    for (int i = tid; i < nd; i += NT) S[i] = T.S[i];
    for (int i = tid; i < nd * nc; i += NT) {
        P[i] = T.P[i];
        G[i] = T.G[i];
        KG[i] = T.KG[i];
    }
    for (int i = tid; i < N; i += NT) grp[i] = T.grp[i];
    m.o = OccView{N, A.no1, nd, A.nsoc, A.nbeta, A.nalpha, nc, nv, A.ista, A.high_spin, A.method, A.h_cut,
                  S, P, G, KG, grp};
    for (int k = tid; k < nv; k += NT) m.x[k] = A.gamma[k];
    __syncthreads();

    const double eta = 0.4;
    double fx = eval(A, m, m.x, m.gx);
    int nit = 0, conv = 0;
    if (maxabs(m, m.gx, nv) <= A.g_abstol) {
        conv = 1;
    } else {
        for (int k = tid; k < nv; k += NT) m.d[k] = -m.gx[k];
        __syncthreads();
        double a = 1.0 / fmax(maxabs(m, m.gx, nv), 1e-12);
        bool have_prev = false, steepest = true;
        double gd_prev = 0.0;
        nit = A.max_iter;
        for (int it = 1; it <= A.max_iter; ++it) {
            double gd = dot(m, m.gx, m.d, nv);
            if (gd >= 0) {  // not a descent direction: restart
                for (int k = tid; k < nv; k += NT) m.d[k] = -m.gx[k];
                __syncthreads();
                gd = dot(m, m.gx, m.d, nv);
                steepest = true;
            }
            if (have_prev) a = fmin(fmax(a * gd_prev / gd, 1e-10), 1e6);
            const Pt pt = wolfe(A, m, fx, gd, a);
            a = pt.a;
            // x += a d, y = g_new - g_old (y kept in xa), |a d|_max
            double smax = 0.0;
            for (int k = tid; k < nv; k += NT) {
                const double s = a * m.d[k];
                smax = fmax(smax, fabs(s));
                m.x[k] += s;
                m.xa[k] = m.gt[k] - m.gx[k];
            }
            smax = block_max(m, smax);
            if (maxabs(m, m.gt, nv) <= A.g_abstol) {
                fx = pt.f;
                nit = it;
                conv = 1;
                break;
            }
            if (fabs(pt.f - fx) <= 0.0 && smax == 0.0) {
                // the line search found no step: once along a conjugate direction, restart
                // from steepest descent; along steepest descent, stop
                if (!steepest) {
                    for (int k = tid; k < nv; k += NT) m.d[k] = -m.gx[k];
                    __syncthreads();
                    steepest = true;
                    have_prev = false;
                    a = 1.0 / fmax(maxabs(m, m.gx, nv), 1e-12);
                    continue;
                }
                fx = pt.f;
                nit = it;
                break;
            }
            const double dy = dot(m, m.d, m.xa, nv);
            double beta = 0.0;
            if (dy != 0.0) {
                const double yy = dot(m, m.xa, m.xa, nv);
                double t = 0.0;
                for (int k = tid; k < nv; k += NT) t += (m.xa[k] - 2.0 * m.d[k] * yy / dy) * m.gt[k];
                t = block_sum(m, t);
                beta = t / dy;
                const double eta_k = -1.0 / (sqrt(dot(m, m.d, m.d, nv)) * fmin(eta, sqrt(dot(m, m.gx, m.gx, nv))));
                beta = fmax(beta, eta_k);
            }
            gd_prev = gd;
            have_prev = true;
            steepest = false;
            for (int k = tid; k < nv; k += NT) {
                m.d[k] = -m.gt[k] + beta * m.d[k];
                m.gx[k] = m.gt[k];
            }
            __syncthreads();
            fx = pt.f;
        }
    }
    // the gradient at the returned gamma: gx unless the loop stopped on a new point
    const double* gfin = (nit > 0) ? m.gt : m.gx;
    for (int k = tid; k < nv; k += NT) {
        A.gamma[k] = m.x[k];
        A.result[3 + k] = gfin[k];
    }
    if (tid == 0) {
        A.result[0] = fx;
        A.result[1] = (double)nit;
        A.result[2] = (double)conv;
    }
}

}  // namespace

size_t occ_cg_smem_bytes(int N, int ndoc, int ncwo, int nv) {
    auto r2 = [](size_t c) { return (c + 1) & ~size_t(1); };
    size_t d = 5 * r2(N) + 2 * r2(ndoc) + r2((size_t)ndoc * (ncwo + 1) * ncwo) + 5 * r2(nv) +
               r2((size_t)N * sizeof(RowSums) / sizeof(double)) + r2(2 * NW * 3) + 3 * r2(CACHE) + r2(2);
    const size_t ints = (size_t)ndoc + 3 * (size_t)ndoc * ncwo + N;
    return d * sizeof(double) + ints * sizeof(int);
}

bool occ_cg_fits(const Occ& o) {
    return o.N <= MAX_N && o.ndoc <= MAX_PAIR && o.ndoc * o.ncwo <= MAX_PV &&
           occ_cg_smem_bytes(o.N, o.ndoc, o.ncwo, o.nv) <= OCC_SMEM_MAX;
}

int occ_cg_launch(donof_ctx* ctx, cudaStream_t st, const Occ& o, const double* J, const double* K, const double* Hc,
                  double* gamma, double g_abstol, int max_iter, double* result) {
    if (!occ_cg_fits(o)) {
        set_error(ctx, "occupation solver on the device: nbf5=%d ndoc=%d ncwo=%d exceed its shared-memory tables",
                  o.N, o.ndoc, o.ncwo);
        return DONOF_ERR_ARG;
    }
    Tables T;
    for (int g = 0; g < o.ndoc; ++g) T.S[g] = o.S[g];
    for (int i = 0; i < o.ndoc * o.ncwo; ++i) {
        T.P[i] = o.P[i];
        T.G[i] = o.G[i];
        T.KG[i] = o.KG[i];
    }
    for (int i = 0; i < o.N; ++i) T.grp[i] = o.grp[i];
    CgArgs A{};
    A.N = o.N; A.no1 = o.no1; A.ndoc = o.ndoc; A.nsoc = o.nsoc; A.nbeta = o.nbeta; A.nalpha = o.nalpha;
    A.ncwo = o.ncwo; A.nv = o.nv; A.ista = o.ista; A.high_spin = o.high_spin; A.method = o.method; A.h_cut = o.h_cut;
    A.J = J; A.K = K; A.Hc = Hc; A.gamma = gamma; A.result = result; A.g_abstol = g_abstol;
    A.max_iter = max_iter;
    const size_t smem = occ_cg_smem_bytes(o.N, o.ndoc, o.ncwo, o.nv);
    // the attribute is set once per device to the largest size a launch may ask
    // for (setting it per launch would race with launches from other host threads)
    static std::atomic<unsigned long long> attr_mask{0};
    const unsigned long long bit = 1ull << (ctx->device & 63);
    if (!(attr_mask.load(std::memory_order_acquire) & bit)) {
        DONOF_CUDA(ctx, cudaFuncSetAttribute(occ_cg_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)OCC_SMEM_MAX));
        attr_mask.fetch_or(bit, std::memory_order_acq_rel);
    }
    occ_cg_kernel<<<1, NT, smem, st>>>(T, A); count_launch();
    DONOF_CUDA(ctx, cudaGetLastError());
    return DONOF_OK;
}

}  // namespace occ
}  // namespace donof

extern "C" int donof_occ_cg_dev(donof_ctx* ctx, const donof_occ_params* prm, const double* J_MO, const double* K_MO,
                                const double* H_core, double* gamma, double g_abstol, int max_iter, double* result) {
    using namespace donof;
    if (!ctx) return DONOF_ERR_ARG;
    occ::Occ o;
    if (!occ::setup(prm, o) || !J_MO || !K_MO || !H_core || !gamma || !result || max_iter < 0) {
        set_error(ctx, "donof_occ_cg_dev: invalid sizes, null pointer or max_iter < 0");
        return DONOF_ERR_ARG;
    }
    DONOF_CUDA(ctx, cudaSetDevice(ctx->device));
    return occ::occ_cg_launch(ctx, ctx->stream, o, J_MO, K_MO, H_core, gamma, g_abstol, max_iter, result);
}
