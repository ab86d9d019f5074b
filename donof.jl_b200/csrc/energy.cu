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
#include <atomic>
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
    double *gam, *occres;  // gamma and the result of the device occupation solver
    unsigned long long* gmax;
    int* perm;
};

struct Loop {
    donof_job* job;
    donof_ctx* ctx;
    cudaStream_t st;
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
    // J_MO, K_MO, H_core at the current C, left on the device
    int jkh_dev() {
        if (prec == DONOF_PREC_MIXED) return jkh_mo_mixed(job, st, D.C, D.H, N, D.J, D.K, D.Hc);
        return jkh_mo_f64(job, st, D.C, D.H, N, D.J, D.K, D.Hc);
    }
    // J_MO, K_MO, H_core at the current C, brought to the host
    int jkh(std::vector<double>& J, std::vector<double>& K, std::vector<double>& Hc) {
        if (prec == DONOF_PREC_MIXED) DONOF_CHECK(jkh_mo_mixed(job, st, D.C, D.H, N, D.J, D.K, D.Hc));
        else DONOF_CHECK(jkh_mo_f64(job, st, D.C, D.H, N, D.J, D.K, D.Hc));
        DONOF_CUDA(ctx, cudaMemcpyAsync(J.data(), D.J, sizeof(double) * J.size(), cudaMemcpyDeviceToHost, st));
        DONOF_CUDA(ctx, cudaMemcpyAsync(K.data(), D.K, sizeof(double) * K.size(), cudaMemcpyDeviceToHost, st));
        DONOF_CUDA(ctx, cudaMemcpyAsync(Hc.data(), D.Hc, sizeof(double) * Hc.size(), cudaMemcpyDeviceToHost, st));
        DONOF_CUDA(ctx, cudaStreamSynchronize(st));
        return failure_status(ctx);
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

// One job's pass through DoNOF.energy's alternation (see the file header):
// setup, then per outer iteration begin() (the occupations of gamma on the
// device), the orbital optimisation of D.C at them, after_orbopt() (occoptr,
// ordering, convergence; sets done), and finish() once done.  donof_energy
// drives one with the single-job optimiser; donof_batch_energy (batch.cu)
// drives several, with the orbital optimisation of all of them as one grouped
// call.
struct EnergyJob::Impl {
    donof_job* job = nullptr;
    donof_energy_params* prm = nullptr;
    donof::occ::Occ o;
    Loop L{};
    double* history = nullptr;
    std::vector<double> gamma, dn, n, cj, ck, n_occ, cj_occ, ck_occ, J, K, Hc, gocc;
    std::vector<int> perm;
    double E = 9999.0, E_old = 9999.0, gorb = 0.0, gocc_norm = 0.0;
    int it = 1, tot_orb = 0, tot_occ = 0, converged = 0, nit_occ = 0;
    bool done = false, moved = false;
    bool occ_dev = false;      // occoptr's CG runs on the device (occ_device and the sizes fit)
    bool occ_dev_done = false;  // this iteration's device CG has run (occ_fetch)
};

EnergyJob::EnergyJob() : p(new Impl) {}
EnergyJob::~EnergyJob() { delete p; }
bool EnergyJob::done() const { return p->done; }
const double* EnergyJob::dev_n() const { return p->L.D.n; }
const double* EnergyJob::dev_cj() const { return p->L.D.cj; }
const double* EnergyJob::dev_ck() const { return p->L.D.ck; }
const double* EnergyJob::dev_H() const { return p->L.D.H; }
double* EnergyJob::dev_C() const { return p->L.D.C; }

int EnergyJob::setup(donof_job* job, donof_energy_params* prm, const double* H, const double* C,
                     const double* gamma_in, double* history) {
    Impl& S = *p;
    donof_ctx* ctx = job->ctx;
    if (!donof::occ::setup(&prm->occ, S.o) || prm->occ.nbf5 > job->nbf || prm->maxit < 1 || prm->maxloop < 1 ||
        prm->orb_method < DONOF_ORB_ADAM || prm->orb_method > DONOF_ORB_DEMON) {
        set_error(ctx, "donof_energy: invalid sizes, switches, maxit or maxloop");
        return DONOF_ERR_ARG;
    }
    DONOF_CUDA(ctx, cudaSetDevice(ctx->device));
    S.job = job;
    S.prm = prm;
    S.history = history;
    const donof::occ::Occ& o = S.o;
    const int nbf = job->nbf, N = o.N, nv = o.nv;
    const size_t nn = (size_t)nbf * nbf, n55 = (size_t)N * N;
    const long long nvar = nvar_of(nbf, N);
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t q = off; off += (bytes + 255) / 256 * 256; return q; };
    const size_t oH = take(8 * nn), oC = take(8 * nn), oC2 = take(8 * nn), on = take(8 * (size_t)N),
                 ocj = take(8 * n55), ock = take(8 * n55), oel = take(8 * nn), oHm = take(8 * (size_t)nbf * N),
                 oE = take(8), oJ = take(8 * n55), oK = take(8 * n55), oHc = take(8 * (size_t)N),
                 og = take(8 * (size_t)nvar), ogm = take(8), op = take(sizeof(int) * (size_t)nbf),
                 ogam = take(8 * (size_t)(nv > 0 ? nv : 1)), ores = take(8 * (size_t)(3 + nv));
    DONOF_CHECK(job->drv.ensure(ctx, off));
    char* base = job->drv.as<char>();
    S.L = Loop{job, ctx, ctx->stream, nbf, N, prm->occ.nalpha, prm->occ.nbeta, job->precision, {}};
    Dev& D = S.L.D;
    D.H = (double*)(base + oH);
    D.C = (double*)(base + oC);
    D.C2 = (double*)(base + oC2);
    D.n = (double*)(base + on);
    D.cj = (double*)(base + ocj);
    D.ck = (double*)(base + ock);
    D.elag = (double*)(base + oel);
    D.Hmat = (double*)(base + oHm);
    D.E = (double*)(base + oE);
    D.J = (double*)(base + oJ);
    D.K = (double*)(base + oK);
    D.Hc = (double*)(base + oHc);
    D.g = (double*)(base + og);
    D.gmax = (unsigned long long*)(base + ogm);
    D.perm = (int*)(base + op);
    D.gam = (double*)(base + ogam);
    D.occres = (double*)(base + ores);
    DONOF_CUDA(ctx, cudaMemcpyAsync(D.H, H, 8 * nn, cudaMemcpyHostToDevice, S.L.st));
    DONOF_CUDA(ctx, cudaMemcpyAsync(D.C, C, 8 * nn, cudaMemcpyHostToDevice, S.L.st));
    S.gamma.assign(gamma_in, gamma_in + nv);
    S.dn.assign((size_t)N * (nv > 0 ? nv : 1), 0.0);
    S.n.assign(N, 0.0); S.n_occ.assign(N, 0.0);
    S.cj.assign(n55, 0.0); S.ck.assign(n55, 0.0); S.cj_occ.assign(n55, 0.0); S.ck_occ.assign(n55, 0.0);
    S.J.assign(n55, 0.0); S.K.assign(n55, 0.0); S.Hc.assign(N, 0.0);
    S.gocc.assign(nv > 0 ? nv : 1, 0.0);
    S.perm.assign(nbf, 0);
    donof::occ::occupations(o, S.gamma.data(), S.n.data(), S.dn.data());
    donof::occ::coupling(o, S.n.data(), S.cj.data(), S.ck.data());
    S.occ_dev = prm->occ_device != 0 && donof::occ::occ_cg_fits(o);
    return DONOF_OK;
}

int EnergyJob::begin() { return p->L.put_coef(p->n, p->cj, p->ck); }

int EnergyJob::after_orbopt(double E_orb, int nit_orb) {
    DONOF_CHECK(occ_fetch());
    DONOF_CHECK(occ_solve());
    return end_iteration(E_orb, nit_orb);
}

// occoptr, device part: J_MO, K_MO, H_core at the optimised orbitals, to the host
// for the host solver; with the device solver, they stay on the device and the
// conjugate gradient runs there too (one CTA), only gamma and its result come back.
int EnergyJob::occ_fetch() {
    Impl& S = *p;
    S.occ_dev_done = false;
    if (S.o.ndoc <= 0 || S.prm->freeze_occ) return DONOF_OK;
    if (!S.occ_dev) return S.L.jkh(S.J, S.K, S.Hc);
    Loop& L = S.L;
    const int nv = S.o.nv;
    DONOF_CHECK(L.jkh_dev());
    DONOF_CUDA(L.ctx, cudaMemcpyAsync(L.D.gam, S.gamma.data(), 8 * (size_t)nv, cudaMemcpyHostToDevice, L.st));
    DONOF_CHECK(donof::occ::occ_cg_launch(L.ctx, L.st, S.o, L.D.J, L.D.K, L.D.Hc, L.D.gam, S.prm->threshen, 1000,
                                          L.D.occres));
    double res[3];
    DONOF_CUDA(L.ctx, cudaMemcpyAsync(S.gamma.data(), L.D.gam, 8 * (size_t)nv, cudaMemcpyDeviceToHost, L.st));
    DONOF_CUDA(L.ctx, cudaMemcpyAsync(res, L.D.occres, sizeof(res), cudaMemcpyDeviceToHost, L.st));
    DONOF_CUDA(L.ctx, cudaStreamSynchronize(L.st));
    DONOF_CHECK(failure_status(L.ctx));
    S.nit_occ = (int)res[1];
    S.occ_dev_done = true;
    return DONOF_OK;
}

// occoptr, host part (no CUDA call: jobs may run it on several threads at once):
// the conjugate gradient over gamma, the occupations and couplings it gives, and
// the column order of order_occupations_softmax.
int EnergyJob::occ_solve() {
    Impl& S = *p;
    const donof::occ::Occ& o = S.o;
    donof_energy_params* prm = S.prm;
    if (o.ndoc > 0 && !prm->freeze_occ) {
        if (!S.occ_dev_done) {
            S.nit_occ = 0;
            double E_occ = 0.0;
            int conv = 0;
            const int rc = donof::occ::cg(o, S.J.data(), S.K.data(), S.Hc.data(), S.gamma.data(), prm->threshen,
                                          1000, &E_occ, &S.nit_occ, &conv);
            if (rc != DONOF_OK) return rc;
        }
        if (S.nit_occ < 1) prm->maxloop += 10;
    } else {
        S.nit_occ = 0;
    }
    donof::occ::occupations(o, S.gamma.data(), S.n_occ.data(), S.dn.data());
    donof::occ::coupling(o, S.n_occ.data(), S.cj_occ.data(), S.ck_occ.data());
    S.moved = (o.method == 0) && order_softmax(o, S.gamma, S.perm);
    return DONOF_OK;
}

int EnergyJob::end_iteration(double E_orb, int nit_orb) {
    Impl& S = *p;
    Loop& L = S.L;
    const donof::occ::Occ& o = S.o;
    donof_energy_params* prm = S.prm;
    donof_ctx* ctx = L.ctx;
    cudaStream_t st = L.st;
    const int nv = o.nv;
    const int nit_occ = S.nit_occ;
    // ---- order_occupations_softmax on the device
    if (S.moved) DONOF_CHECK(L.permute(S.perm));
    S.tot_orb += nit_orb;
    S.tot_occ += nit_occ;
    S.E = E_orb;
    const double E_diff = S.E - S.E_old;
    S.E_old = S.E;
    // ---- convergence: orbital gradient at the new occupations, occupation gradient
    donof::occ::occupations(o, S.gamma.data(), S.n.data(), S.dn.data());
    donof::occ::coupling(o, S.n.data(), S.cj.data(), S.ck.data());
    DONOF_CHECK(L.put_coef(S.n, S.cj, S.ck));
    DONOF_CHECK(L.lagrangian());
    DONOF_CUDA(ctx, cudaMemsetAsync(L.D.gmax, 0, sizeof(unsigned long long), st));
    DONOF_CHECK(pack_grad(ctx, st, L.D.elag, L.nbf, L.N, L.D.g, L.D.gmax));
    unsigned long long gbits = 0;
    DONOF_CUDA(ctx, cudaMemcpyAsync(&gbits, L.D.gmax, sizeof(gbits), cudaMemcpyDeviceToHost, st));
    DONOF_CHECK(L.jkh(S.J, S.K, S.Hc));  // synchronises the stream
    memcpy(&S.gorb, &gbits, sizeof(double));
    donof::occ::energy_grad(o, S.gamma.data(), S.J.data(), S.K.data(), S.Hc.data(), S.gocc.data());
    double s2 = 0.0;
    for (int k = 0; k < nv; ++k) s2 += S.gocc[k] * S.gocc[k];
    S.gocc_norm = sqrt(s2);
    if (S.history) {
        double* h = S.history + 6 * (size_t)(S.it - 1);
        h[0] = S.E; h[1] = E_diff; h[2] = S.gorb; h[3] = S.gocc_norm; h[4] = nit_orb; h[5] = nit_occ;
    }
    if (S.gorb < prm->threshgorb && S.gocc_norm < prm->threshgocc) {
        S.converged = 1;
        S.done = true;
    } else if (prm->stop_rel_de > 0.0 && S.it > 1 && fabs(E_diff) <= prm->stop_rel_de * fabs(S.E)) {
        S.done = true;
    } else if (S.it >= prm->maxit) {
        S.done = true;
    } else {
        ++S.it;
    }
    return DONOF_OK;
}

int EnergyJob::finish(double* C_out, double* gamma_out, double* n_out, double* elag_out, donof_energy_result* res) {
    Impl& S = *p;
    Loop& L = S.L;
    donof_ctx* ctx = L.ctx;
    cudaStream_t st = L.st;
    const int nbf = L.nbf, N = L.N;
    const size_t nn = (size_t)nbf * nbf;
    // ---- ENERGY1r of the last iteration: elag at (C, occupations before the ordering)
    DONOF_CHECK(L.put_coef(S.n_occ, S.cj_occ, S.ck_occ));
    DONOF_CHECK(L.lagrangian());
    if (S.prm->order_subspaces) {
        std::vector<double> el(nn), ed(N);
        DONOF_CUDA(ctx, cudaMemcpyAsync(el.data(), L.D.elag, 8 * nn, cudaMemcpyDeviceToHost, st));
        DONOF_CUDA(ctx, cudaStreamSynchronize(st));
        for (int i = 0; i < N; ++i) ed[i] = el[i + (size_t)nbf * i];
        order_subspaces(S.o, ed, S.n, S.perm);
        DONOF_CHECK(L.permute(S.perm));
        donof::occ::coupling(S.o, S.n.data(), S.cj.data(), S.ck.data());
        DONOF_CHECK(L.put_coef(S.n, S.cj, S.ck));
        DONOF_CHECK(L.lagrangian());
    }
    DONOF_CUDA(ctx, cudaMemcpyAsync(C_out, L.D.C, 8 * nn, cudaMemcpyDeviceToHost, st));
    if (elag_out) DONOF_CUDA(ctx, cudaMemcpyAsync(elag_out, L.D.elag, 8 * nn, cudaMemcpyDeviceToHost, st));
    DONOF_CUDA(ctx, cudaStreamSynchronize(st));
    DONOF_CHECK(failure_status(ctx));
    std::copy(S.gamma.begin(), S.gamma.end(), gamma_out);
    if (n_out) std::copy(S.n.begin(), S.n.end(), n_out);
    res->E_elec = S.E;
    res->iterations = S.it;
    res->converged = S.converged;
    res->tot_it_orb = S.tot_orb;
    res->tot_it_occ = S.tot_occ;
    res->max_grad_orb = S.gorb;
    res->norm_grad_occ = S.gocc_norm;
    return DONOF_OK;
}

}  // namespace donof

using namespace donof;

namespace donof {

int energy_run(donof_job* job, donof_energy_params* prm, const double* H, double* C_inout, double* gamma_inout,
               double* n_out, double* elag_out, double* history, donof_energy_result* res,
               const std::atomic<int>* cancel) {
    EnergyJob E;
    DONOF_CHECK(E.setup(job, prm, H, C_inout, gamma_inout, history));
    while (!E.done()) {
        if (cancel && cancel->load(std::memory_order_relaxed)) {
            set_error(job->ctx, "cancelled");
            return DONOF_ERR_STATE;
        }
        DONOF_CHECK(E.begin());
        double E_orb = 0.0;
        int nit_orb = 0, ok_orb = 0;
        DONOF_CHECK(orbopt_run(job, prm->orb_method, E.dev_n(), E.dev_cj(), E.dev_ck(), E.dev_H(), prm->occ.nbf5,
                               prm->occ.nalpha, prm->occ.nbeta, &prm->alpha, &prm->maxloop, prm->threshgorb,
                               E.dev_C(), &E_orb, &nit_orb, &ok_orb, job->precision));
        DONOF_CHECK(E.after_orbopt(E_orb, nit_orb));
    }
    return E.finish(C_inout, gamma_inout, n_out, elag_out, res);
}

}  // namespace donof

extern "C" int donof_energy(donof_job* job, donof_energy_params* prm, const double* H, double* C_inout,
                            double* gamma_inout, double* n_out, double* elag_out, double* history,
                            donof_energy_result* res) {
    if (!job || !prm || !H || !C_inout || !gamma_inout || !res) return DONOF_ERR_ARG;
    return energy_run(job, prm, H, C_inout, gamma_inout, n_out, elag_out, history, res, nullptr);
}
