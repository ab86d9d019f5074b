// The orbital / occupation alternation of DoNOF.energy (src/energy.jl:140-224)
// as one native call, donof_energy.
//
// Per outer iteration, like the reference:
//   orbopt           the device-resident orbital optimiser (optim.cu) at the
//                    occupations of the current gamma
//   occoptr          J_MO, K_MO, H_core on the device, then the conjugate
//                    gradient over gamma on the host (src/minimization.jl:100-139;
//                    maxloop + 10 when it takes no iteration)
//   ordering         order_occupations_softmax (src/utils.jl:586-616): each
//                    pair's orbitals sorted by gamma, descending (Softmax only)
//   convergence      max|g_orb| from the Lagrangian at the new occupations
//                    (calcorbg, src/pnof.jl:1389-1407) and |g_occ| from calcoccg
//                    at fresh J_MO, K_MO, H_core; stop when both are below
//                    threshgorb and threshgocc.
// ENERGY1r's Lagrangian (src/utils.jl:117-136), which the loop only prints, is
// evaluated once, for the last iteration, to give elag and the final
// order_subspaces (src/guess.jl:58-106, ipnof > 4).
//
// C, H and the functional's coefficients stay on the device; only gamma's
// couplings (nbf5^2), J_MO, K_MO, H_core and a few scalars cross PCIe per
// iteration.  The whole loop runs without the caller's interpreter, so that
// jobs served from several host threads advance in parallel.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <numeric>
#include <vector>

#include "kernels.cuh"
#include "occ.cuh"

namespace donof {

int orbopt_run(donof_job* job, int method, const double* n, const double* cj12, const double* ck12,
               const double* H, int nbf5, int nalpha, int nbeta, double* alpha, int* maxloop,
               double threshgorb, double* C, double* E_out, int* nit_out, int* success_out,
               int precision);

namespace {

// Cout[:, j] = Cin[:, perm[j]]
__global__ void permute_cols_kernel(const double* __restrict__ Cin, const int* __restrict__ perm, int nbf,
                                    double* __restrict__ Cout) {
    const long long nn = (long long)nbf * nbf;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nn;
         i += (long long)gridDim.x * blockDim.x) {
        const int m = (int)(i % nbf), j = (int)(i / nbf);
        Cout[i] = Cin[m + (long long)nbf * perm[j]];
    }
}

struct Dev {
    double *H, *C, *C2, *n, *cj, *ck, *elag, *Hmat, *E, *J, *K, *Hc, *g;
    unsigned long long* gmax;
    int* perm;
};

struct Loop {
    donof_job* job;
    donof_ctx* ctx;
    cudaStream_t st;
    const donof::occ::Occ& o;
    int nbf, N, nalpha, nbeta, prec;
    Dev D;

    int put(double* d, const std::vector<double>& h) {
        DONOF_CUDA(ctx, cudaMemcpyAsync(d, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice, st));
        return DONOF_OK;
    }
    int put_coef(const std::vector<double>& n, const std::vector<double>& cj, const std::vector<double>& ck) {
        DONOF_CHECK(put(D.n, n));
        DONOF_CHECK(put(D.cj, cj));
        return put(D.ck, ck);
    }
    int lagrangian() {
        if (prec == DONOF_PREC_MIXED)
            return lagrange2_mixed(job, st, D.C, D.n, D.H, D.cj, D.ck, N, nalpha, nbeta, D.elag, D.Hmat, D.E);
        return lagrange2_f64(job, st, D.C, D.n, D.H, D.cj, D.ck, N, nalpha, nbeta, D.elag, D.Hmat, D.E);
    }
    // J_MO, K_MO, H_core at the current C, brought to the host
    int jkh(std::vector<double>& J, std::vector<double>& K, std::vector<double>& Hc) {
        if (prec == DONOF_PREC_MIXED) DONOF_CHECK(jkh_mo_mixed(job, st, D.C, D.H, N, D.J, D.K, D.Hc));
        else DONOF_CHECK(jkh_mo_f64(job, st, D.C, D.H, N, D.J, D.K, D.Hc));
        DONOF_CUDA(ctx, cudaMemcpyAsync(J.data(), D.J, sizeof(double) * J.size(), cudaMemcpyDeviceToHost, st));
        DONOF_CUDA(ctx, cudaMemcpyAsync(K.data(), D.K, sizeof(double) * K.size(), cudaMemcpyDeviceToHost, st));
        DONOF_CUDA(ctx, cudaMemcpyAsync(Hc.data(), D.Hc, sizeof(double) * Hc.size(), cudaMemcpyDeviceToHost, st));
        DONOF_CUDA(ctx, cudaStreamSynchronize(st));
        return DONOF_OK;
    }
    // C <- C[:, perm]
    int permute(const std::vector<int>& perm) {
        DONOF_CUDA(ctx, cudaMemcpyAsync(D.perm, perm.data(), sizeof(int) * nbf, cudaMemcpyHostToDevice, st));
        const long long nn = (long long)nbf * nbf;
        long long blocks = (nn + 255) / 256;
        if (blocks > 4LL * ctx->sm_count) blocks = 4LL * ctx->sm_count;
        permute_cols_kernel<<<(int)blocks, 256, 0, st>>>(D.C, D.perm, nbf, D.C2); count_launch();
        DONOF_CUDA(ctx, cudaGetLastError());
        DONOF_CUDA(ctx, cudaMemcpyAsync(D.C, D.C2, sizeof(double) * nn, cudaMemcpyDeviceToDevice, st));
        return DONOF_OK;
    }
};

// order_occupations_softmax: per pair, the strong orbital and its weak ones
// sorted by (0, gamma) descending (a stable ascending sort, reversed), gamma
// shifted so that the largest is 0.  Fills perm (identity elsewhere); returns
// whether any column moved.
bool order_softmax(const donof::occ::Occ& o, std::vector<double>& gamma, std::vector<int>& perm) {
    std::iota(perm.begin(), perm.end(), 0);
    bool any_pos = false;
    for (double g : gamma) any_pos = any_pos || (g > 0.0);
    if (!any_pos) return false;
    bool moved = false;
    const int nc = o.ncwo;
    std::vector<int> cols(nc + 1), idx(nc + 1);
    std::vector<double> vals(nc + 1);
    for (int g = 0; g < o.ndoc; ++g) {
        cols[0] = o.no1 + g;
        vals[0] = 0.0;
        for (int w = 0; w < nc; ++w) {
            cols[w + 1] = o.P[g * nc + w];
            vals[w + 1] = gamma[o.G[g * nc + w]];
        }
        std::iota(idx.begin(), idx.end(), 0);
        std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return vals[a] < vals[b]; });
        std::reverse(idx.begin(), idx.end());
        const double vmax = *std::max_element(vals.begin(), vals.end());
        for (int w = 0; w < nc; ++w) gamma[o.G[g * nc + w]] = vals[idx[w + 1]] - vmax;
        for (int k = 0; k <= nc; ++k) {
            perm[cols[k]] = cols[idx[k]];
            moved = moved || (idx[k] != k);
        }
    }
    return moved;
}

// order_subspaces: strong orbitals (with their weak partners) and singly
// occupied ones sorted by the Lagrangian diagonal (stable, ascending).  The
// reference sorts the first no1 columns and then overwrites them with the
// originals; the result is the identity on those columns, kept here.
void order_subspaces(const donof::occ::Occ& o, const std::vector<double>& ed, std::vector<double>& n,
                     std::vector<int>& perm) {
    std::iota(perm.begin(), perm.end(), 0);
    const std::vector<double> n0 = n;
    auto sorted = [&](int lo, int cnt) {
        std::vector<int> s(cnt);
        std::iota(s.begin(), s.end(), 0);
        std::stable_sort(s.begin(), s.end(), [&](int a, int b) { return ed[lo + a] < ed[lo + b]; });
        return s;
    };
    const std::vector<int> srt = sorted(o.no1, o.ndoc);
    for (int i = 0; i < o.ndoc; ++i) {
        const int io = srt[i];
        perm[o.no1 + i] = o.no1 + io;
        n[o.no1 + i] = n0[o.no1 + io];
        for (int w = 0; w < o.ncwo; ++w) {
            perm[o.P[i * o.ncwo + w]] = o.P[io * o.ncwo + w];
            n[o.P[i * o.ncwo + w]] = n0[o.P[io * o.ncwo + w]];
        }
    }
    const std::vector<int> srs = sorted(o.no1 + o.ndoc, o.nsoc);
    for (int i = 0; i < o.nsoc; ++i) {
        perm[o.no1 + o.ndoc + i] = o.no1 + o.ndoc + srs[i];
        n[o.no1 + o.ndoc + i] = n0[o.no1 + o.ndoc + srs[i]];
    }
}

}  // namespace

}  // namespace donof

using namespace donof;

extern "C" int donof_energy(donof_job* job, donof_energy_params* prm, const double* H, double* C_inout,
                            double* gamma_inout, double* n_out, double* elag_out, double* history,
                            donof_energy_result* res) {
    if (!job || !prm || !H || !C_inout || !gamma_inout || !res) return DONOF_ERR_ARG;
    donof_ctx* ctx = job->ctx;
    donof::occ::Occ o;
    if (!donof::occ::setup(&prm->occ, o) || prm->occ.nbf5 > job->nbf || prm->maxit < 1 || prm->maxloop < 1 ||
        prm->orb_method < DONOF_ORB_ADAM || prm->orb_method > DONOF_ORB_DEMON) {
        set_error(ctx, "donof_energy: invalid sizes, switches, maxit or maxloop");
        return DONOF_ERR_ARG;
    }
    DONOF_CUDA(ctx, cudaSetDevice(ctx->device));
    const int nbf = job->nbf, N = o.N, nv = o.nv;
    const size_t nn = (size_t)nbf * nbf, n55 = (size_t)N * N;
    const long long nvar = nvar_of(nbf, N);
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t q = off; off += (bytes + 255) / 256 * 256; return q; };
    const size_t oH = take(8 * nn), oC = take(8 * nn), oC2 = take(8 * nn), on = take(8 * (size_t)N),
                 ocj = take(8 * n55), ock = take(8 * n55), oel = take(8 * nn), oHm = take(8 * (size_t)nbf * N),
                 oE = take(8), oJ = take(8 * n55), oK = take(8 * n55), oHc = take(8 * (size_t)N),
                 og = take(8 * (size_t)nvar), ogm = take(8), op = take(sizeof(int) * (size_t)nbf);
    DONOF_CHECK(job->drv.ensure(ctx, off));
    char* base = job->drv.as<char>();
    Loop L{job, ctx, ctx->stream, o, nbf, N, prm->occ.nalpha, prm->occ.nbeta, job->precision, {}};
    L.D.H = (double*)(base + oH);
    L.D.C = (double*)(base + oC);
    L.D.C2 = (double*)(base + oC2);
    L.D.n = (double*)(base + on);
    L.D.cj = (double*)(base + ocj);
    L.D.ck = (double*)(base + ock);
    L.D.elag = (double*)(base + oel);
    L.D.Hmat = (double*)(base + oHm);
    L.D.E = (double*)(base + oE);
    L.D.J = (double*)(base + oJ);
    L.D.K = (double*)(base + oK);
    L.D.Hc = (double*)(base + oHc);
    L.D.g = (double*)(base + og);
    L.D.gmax = (unsigned long long*)(base + ogm);
    L.D.perm = (int*)(base + op);
    cudaStream_t st = L.st;
    DONOF_CUDA(ctx, cudaMemcpyAsync(L.D.H, H, 8 * nn, cudaMemcpyHostToDevice, st));
    DONOF_CUDA(ctx, cudaMemcpyAsync(L.D.C, C_inout, 8 * nn, cudaMemcpyHostToDevice, st));

    std::vector<double> gamma(gamma_inout, gamma_inout + nv), dn((size_t)N * (nv > 0 ? nv : 1));
    std::vector<double> n(N), cj(n55), ck(n55), n_occ(N), cj_occ(n55), ck_occ(n55);
    std::vector<double> J(n55), K(n55), Hc(N), gocc(nv > 0 ? nv : 1);
    std::vector<int> perm(nbf);
    donof::occ::occupations(o, gamma.data(), n.data(), dn.data());
    donof::occ::coupling(o, n.data(), cj.data(), ck.data());

    double E = 9999.0, E_old = 9999.0, gorb = 0.0, gocc_norm = 0.0;
    int it = 0, tot_orb = 0, tot_occ = 0, converged = 0;
    for (it = 1; it <= prm->maxit; ++it) {
        // ---- orbopt at the occupations of gamma
        DONOF_CHECK(L.put_coef(n, cj, ck));
        double E_orb = 0.0;
        int nit_orb = 0, ok_orb = 0;
        DONOF_CHECK(orbopt_run(job, prm->orb_method, L.D.n, L.D.cj, L.D.ck, L.D.H, N, L.nalpha, L.nbeta,
                               &prm->alpha, &prm->maxloop, prm->threshgorb, L.D.C, &E_orb, &nit_orb, &ok_orb,
                               L.prec));
        // ---- occoptr
        int nit_occ = 0;
        if (o.ndoc > 0 && !prm->freeze_occ) {
            DONOF_CHECK(L.jkh(J, K, Hc));
            double E_occ = 0.0;
            int conv = 0;
            DONOF_CHECK(donof::occ::cg(o, J.data(), K.data(), Hc.data(), gamma.data(), prm->threshen, 1000, &E_occ,
                                       &nit_occ, &conv));
            if (nit_occ < 1) prm->maxloop += 10;
        }
        donof::occ::occupations(o, gamma.data(), n_occ.data(), dn.data());
        donof::occ::coupling(o, n_occ.data(), cj_occ.data(), ck_occ.data());
        // ---- order_occupations_softmax
        if (o.method == 0 && order_softmax(o, gamma, perm)) DONOF_CHECK(L.permute(perm));
        tot_orb += nit_orb;
        tot_occ += nit_occ;
        E = E_orb;
        const double E_diff = E - E_old;
        E_old = E;
        // ---- convergence: orbital gradient at the new occupations, occupation gradient
        donof::occ::occupations(o, gamma.data(), n.data(), dn.data());
        donof::occ::coupling(o, n.data(), cj.data(), ck.data());
        DONOF_CHECK(L.put_coef(n, cj, ck));
        DONOF_CHECK(L.lagrangian());
        DONOF_CUDA(ctx, cudaMemsetAsync(L.D.gmax, 0, sizeof(unsigned long long), st));
        DONOF_CHECK(pack_grad(ctx, st, L.D.elag, nbf, N, L.D.g, L.D.gmax));
        unsigned long long gbits = 0;
        DONOF_CUDA(ctx, cudaMemcpyAsync(&gbits, L.D.gmax, sizeof(gbits), cudaMemcpyDeviceToHost, st));
        DONOF_CHECK(L.jkh(J, K, Hc));  // synchronises the stream
        memcpy(&gorb, &gbits, sizeof(double));
        donof::occ::energy_grad(o, gamma.data(), J.data(), K.data(), Hc.data(), gocc.data());
        double s2 = 0.0;
        for (int k = 0; k < nv; ++k) s2 += gocc[k] * gocc[k];
        gocc_norm = sqrt(s2);
        if (history) {
            double* h = history + 6 * (size_t)(it - 1);
            h[0] = E; h[1] = E_diff; h[2] = gorb; h[3] = gocc_norm; h[4] = nit_orb; h[5] = nit_occ;
        }
        if (gorb < prm->threshgorb && gocc_norm < prm->threshgocc) {
            converged = 1;
            break;
        }
        if (prm->stop_rel_de > 0.0 && it > 1 && fabs(E_diff) <= prm->stop_rel_de * fabs(E)) break;
    }
    if (it > prm->maxit) it = prm->maxit;
    // ---- ENERGY1r of the last iteration: elag at (C, occupations before the ordering)
    DONOF_CHECK(L.put_coef(n_occ, cj_occ, ck_occ));
    DONOF_CHECK(L.lagrangian());
    if (prm->order_subspaces) {
        std::vector<double> el(nn), ed(N);
        DONOF_CUDA(ctx, cudaMemcpyAsync(el.data(), L.D.elag, 8 * nn, cudaMemcpyDeviceToHost, st));
        DONOF_CUDA(ctx, cudaStreamSynchronize(st));
        for (int i = 0; i < N; ++i) ed[i] = el[i + (size_t)nbf * i];
        order_subspaces(o, ed, n, perm);
        DONOF_CHECK(L.permute(perm));
        donof::occ::coupling(o, n.data(), cj.data(), ck.data());
        DONOF_CHECK(L.put_coef(n, cj, ck));
        DONOF_CHECK(L.lagrangian());
    }
    DONOF_CUDA(ctx, cudaMemcpyAsync(C_inout, L.D.C, 8 * nn, cudaMemcpyDeviceToHost, st));
    if (elag_out) DONOF_CUDA(ctx, cudaMemcpyAsync(elag_out, L.D.elag, 8 * nn, cudaMemcpyDeviceToHost, st));
    DONOF_CUDA(ctx, cudaStreamSynchronize(st));
    std::copy(gamma.begin(), gamma.end(), gamma_inout);
    if (n_out) std::copy(n.begin(), n.end(), n_out);
    res->E_elec = E;
    res->iterations = it;
    res->converged = converged;
    res->tot_it_orb = tot_orb;
    res->tot_it_occ = tot_occ;
    res->max_grad_orb = gorb;
    res->norm_grad_occ = gocc_norm;
    return DONOF_OK;
}
