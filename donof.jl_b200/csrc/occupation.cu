// Occupation layer and occupation optimiser of GNOF in native host code (FP64).
//
// DoNOF.jl runs this part on the host, even with its GPU extension loaded: the
// occupation energy and gradient from cached J_MO, K_MO, H_core (src/pnof.jl:
// 1273-1377), the occupation parametrisations (softmax src/pnof.jl:1122-1163,
// trigonometric :1047-1120), the GNOF couplings cj12/ck12 and their
// derivatives (CJCKD8 / der_CJCKD8, :488-793) and the conjugate-gradient
// minimisation over gamma of occoptr (src/minimization.jl:100-139, Optim.jl
// ConjugateGradient with g_abstol = threshen).
//
// The gradient contracts the derivative tensors of der_CJCKD8 through their
// separable terms (every term is a per-row derivative a_t[i, k] times a
// matrix M_t[i, j]), O(nbf5^2 + nbf5 nv) per evaluation instead of
// O(nbf5^2 nv).  The minimiser is a Hager-Zhang conjugate gradient (Hager &
// Zhang, SIAM J. Optim. 16 (2005) 170-192, eta = 0.4) with a strong-Wolfe line
// search (Nocedal & Wright, Alg. 3.5/3.6) and Hager-Zhang's approximate-Wolfe
// acceptance, stopped on max|grad| <= g_abstol.
//
// Matrices (J_MO, K_MO) are column-major, X(i, j) = X[i + nbf5 j], like the rest
// of the C ABI.  Nothing here touches the GPU.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "occ.cuh"
#include "occ_math.cuh"

namespace donof {
namespace occ {

bool setup(const donof_occ_params* q, Occ& o) {
    if (!q) return false;
    o.N = q->nbf5;
    o.no1 = q->no1;
    o.nbeta = q->nbeta;
    o.nalpha = q->nalpha;
    o.ndoc = q->nbeta - q->no1;
    o.nsoc = q->nalpha - q->nbeta;
    o.ncwo = q->ncwo;
    o.nv = o.ncwo * o.ndoc;
    o.ista = q->ista;
    o.high_spin = q->high_spin;
    o.method = q->occ_method;
    o.h_cut = q->h_cut;
    if (o.N <= 0 || o.ndoc < 0 || o.nsoc < 0 || o.ncwo < 0 || o.ncwo > 64 || o.no1 < 0 || o.ista < 0 || o.ista > 5 ||
        (o.method != 0 && o.method != 1) || o.h_cut <= 0.0)
        return false;
    const int ndns = o.ndoc + o.nsoc;
    if (o.no1 + ndns + o.ndoc * o.ncwo > o.N) return false;
    o.S.resize(o.ndoc);
    o.P.resize((size_t)o.ndoc * o.ncwo);
    o.G.resize((size_t)o.ndoc * o.ncwo);
    o.KG.resize((size_t)o.ndoc * o.ncwo);
    o.grp.assign(o.N, -1);
    for (int g = 0; g < o.ndoc; ++g) {
        o.S[g] = o.no1 + g;
        o.grp[o.S[g]] = g;
        for (int w = 0; w < o.ncwo; ++w) {
            // Julia's ll:ndoc:ul for strong orbital g+1 (src/param.jl, pnof.jl)
            o.P[g * o.ncwo + w] = o.no1 + ndns + (o.ndoc - (g + 1)) + o.ndoc * w;
            o.G[g * o.ncwo + w] = (o.ndoc - (g + 1)) + o.ndoc * w;
            o.grp[o.P[g * o.ncwo + w]] = g;
            // columns of dn in the pair's rows: softmax, its gamma entries; trigonometric,
            // the strong angle g and the ncwo - 1 weak angles of the pair
            o.KG[g * o.ncwo + w] = (o.method == 0) ? o.G[g * o.ncwo + w]
                                   : (w == 0 ? g : o.ndoc + (o.ndoc - (g + 1)) + o.ndoc * (w - 1));
        }
    }
    return true;
}

namespace {

// n and dn; with full, every entry of dn is written, else only the pair blocks
// (the rows of a pair's members at the pair's gamma columns, KG), the only
// entries energy_grad reads.
void occupations_impl(const Occ& o, const double* gamma, double* n, double* dn, bool full) {
    const int N = o.N, nv = o.nv, nd = o.ndoc, nc = o.ncwo;
    const OccView ov = view(o);
    for (int i = 0; i < N; ++i) n[i] = 0.0;
    for (int i = 0; i < o.no1; ++i) n[i] = 1.0;
    for (int i = o.no1 + nd; i < o.no1 + nd + o.nsoc; ++i) n[i] = o.high_spin ? 1.0 : 0.5;
    if (full) std::fill(dn, dn + (size_t)N * nv, 0.0);
    for (int g = 0; g < nd; ++g) pair_n(ov, gamma, g, n);
    std::vector<double> blk((size_t)(nc + 1) * (nc > 0 ? nc : 1));
    for (int g = 0; g < nd; ++g) {
        pair_dn(ov, gamma, g, n, blk.data());
        for (int m = 0; m <= nc; ++m)
            for (int c = 0; c < nc; ++c) dn[(size_t)member(ov, g, m) * nv + o.KG[g * nc + c]] = blk[m * nc + c];
    }
}

}  // namespace

OccView view(const Occ& o) {
    return OccView{o.N, o.no1, o.ndoc, o.nsoc, o.nbeta, o.nalpha, o.ncwo, o.nv, o.ista, o.high_spin, o.method,
                   o.h_cut, o.S.data(), o.P.data(), o.G.data(), o.KG.data(), o.grp.data()};
}

// n (N) and dn (N x nv, dn[i * nv + k]) for the configured occupation map
void occupations(const Occ& o, const double* gamma, double* n, double* dn) {
    occupations_impl(o, gamma, n, dn, true);
}

// n_d, F and coc of the dynamic part (src/pnof.jl:488-601)
void dynamic(const Occ& o, const double* n, std::vector<double>& nd, std::vector<double>& F,
             std::vector<double>& coc) {
    const OccView ov = view(o);
    nd.assign(o.N, 0.0);
    F.assign(o.ndoc, 0.0);
    coc.assign(o.ndoc, 0.0);
    for (int g = 0; g < o.ndoc; ++g) pair_dynamic(ov, n, g, nd.data(), F.data(), coc.data());
}

bool in(int i, int a, int b) { return i >= a && i < b; }

// cj12, ck12 (row-major C[i * N + j]) with zeroed diagonals (PNOFi_selector, CJCKD8)
void coupling(const Occ& o, const double* n, double* cj, double* ck) {
    const int N = o.N;
    std::vector<double> nd, F, coc;
    dynamic(o, n, nd, F, coc);
    std::vector<double> nd12(N), fi(N);
    for (int i = 0; i < N; ++i) {
        nd12[i] = sqrt(nd[i]);
        fi[i] = phi_fn(n[i], o.ista);
    }
    const int b0 = o.no1, b1 = o.nbeta, a1 = o.nalpha, c1 = N;  // be [b0,b1), al [b1,a1), cw [a1,c1)
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) {
            cj[i * N + j] = 2.0 * n[i] * n[j];
            double k = n[i] * n[j];
            const bool ibe = in(i, b0, b1), ial = in(i, b1, a1), icw = in(i, a1, c1);
            const bool jbe = in(j, b0, b1), jal = in(j, b1, a1), jcw = in(j, a1, c1);
            if (o.ista == 0) {
                if ((ibe && jcw) || (icw && jbe) || (icw && jcw)) k += fi[i] * fi[j];
                if (o.nsoc > 0) {
                    if (ibe && jal) k += 0.25 * fi[i];
                    if (ial && jbe) k += 0.25 * fi[j];
                    if (ial && jcw) k += 0.5 * fi[j];
                    if (icw && jal) k += 0.5 * fi[i];
                }
                if (o.nsoc > 1 && ial && jal) k = 0.5;
            } else {
                k += fi[i] * fi[j];
            }
            if ((ibe && jcw) || (icw && jbe)) k += nd12[i] * nd12[j] - nd[i] * nd[j];
            if (icw && jcw) k -= nd12[i] * nd12[j] + nd[i] * nd[j];
            ck[i * N + j] = k;
        }
    for (int g = 0; g < o.ndoc; ++g) {
        const int s = o.S[g];
        for (int a = 0; a < o.ncwo; ++a) {
            const int w = o.P[g * o.ncwo + a];
            cj[s * N + w] = cj[w * N + s] = 0.0;
            const double r = sqrt(n[s] * n[w]);
            ck[s * N + w] = ck[w * N + s] = r;
            for (int b = 0; b < o.ncwo; ++b) {
                const int v = o.P[g * o.ncwo + b];
                cj[w * N + v] = 0.0;
                ck[w * N + v] = -(sqrt(n[w]) * sqrt(n[v]));
            }
        }
    }
    for (int i = 0; i < N; ++i) cj[i * N + i] = ck[i * N + i] = 0.0;
}

// ---------------------------------------------------------------- energy, gradient
// The couplings of CJCKD8 (coupling() above) and the factors of their
// derivatives (der_CJCKD8, src/pnof.jl:603-793) are, away from the pairs, a
// function of the index classes of the two orbitals -- [0, no1), beta-occupied
// [no1, nbeta), alpha-only [nbeta, nalpha), weak [nalpha, nbf5) -- and of four
// per-orbital vectors (n, phi(n), n_d^{1/2}, n_d); inside a pair (a strong
// orbital and its weak partners) they take special values.  Every double sum
// over (i, j) therefore reduces to, per orbital i, a few dot products of
// column i of J_MO / K_MO with those vectors over the class ranges (RowSums),
// plus corrections for the 1 + ncwo members of its pair (occ_math.cuh).  The
// gradient contracts the separable terms
//   Dcj[i,j,:] = Mcj[i,j] dn[i,:],   Dck[i,j,:] = sum_t M_t[i,j] A_t[i,:],
//   A = (dn, dphi, dn_d^{1/2}, dn_d),
// whose rows A_t[i,:] are nonzero only on the ncwo gamma entries of i's pair.

struct OrbVecs {
    std::vector<double> n, fi, nd12, nd, F, coc;  // per orbital; F, coc per pair (dynamic())
    VecView view() const { return VecView{n.data(), fi.data(), nd12.data(), nd.data(), F.data(), coc.data()}; }
};

// Rows are taken four at a time (the last ones one at a time): every row keeps
// its own accumulators summed in order of j, so the result is the same as row by
// row, with four independent chains per sum in flight instead of one.
void row_sums(const Occ& o, const OrbVecs& v, const double* J, const double* K, std::vector<RowSums>& rs) {
    const int N = o.N;
    const int bnd[5] = {0, o.no1, o.nbeta, o.nalpha, N};
    const double *vn = v.n.data(), *vf = v.fi.data(), *v12 = v.nd12.data(), *vd = v.nd.data();
    rs.resize(N);
    constexpr int RB = 4;
    int i0 = 0;
    for (; i0 + RB <= N; i0 += RB) {
        const double* Kc[RB];
        const double* Jc[RB];
        for (int u = 0; u < RB; ++u) {
            Kc[u] = K + (size_t)N * (i0 + u);
            Jc[u] = J + (size_t)N * (i0 + u);
        }
        for (int R = 0; R < 4; ++R) {
            double a0[RB] = {}, a1[RB] = {}, a2[RB] = {}, a3[RB] = {}, a4[RB] = {};
            for (int j = bnd[R]; j < bnd[R + 1]; ++j) {
                const double n_ = vn[j], f_ = vf[j], h_ = v12[j], d_ = vd[j];
                for (int u = 0; u < RB; ++u) {
                    const double kj = Kc[u][j];
                    a0[u] += n_ * kj;
                    a1[u] += f_ * kj;
                    a2[u] += h_ * kj;
                    a3[u] += d_ * kj;
                    a4[u] += kj;
                }
            }
            for (int u = 0; u < RB; ++u) {
                RowSums& r = rs[i0 + u];
                r.S[R][V_N] = a0[u]; r.S[R][V_FI] = a1[u]; r.S[R][V_ND12] = a2[u]; r.S[R][V_ND] = a3[u];
                r.S[R][V_ONE] = a4[u];
            }
        }
        double jn[RB] = {};
        for (int j = 0; j < N; ++j) {
            const double n_ = vn[j];
            for (int u = 0; u < RB; ++u) jn[u] += n_ * Jc[u][j];
        }
        for (int u = 0; u < RB; ++u) rs[i0 + u].jn = jn[u];
    }
    for (int i = i0; i < N; ++i) {
        const double* Kc = K + (size_t)N * i;
        const double* Jc = J + (size_t)N * i;
        RowSums& r = rs[i];
        for (int R = 0; R < 4; ++R) {
            double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0, a4 = 0.0;
            for (int j = bnd[R]; j < bnd[R + 1]; ++j) {
                const double kj = Kc[j];
                a0 += vn[j] * kj;
                a1 += vf[j] * kj;
                a2 += v12[j] * kj;
                a3 += vd[j] * kj;
                a4 += kj;
            }
            r.S[R][V_N] = a0; r.S[R][V_FI] = a1; r.S[R][V_ND12] = a2; r.S[R][V_ND] = a3; r.S[R][V_ONE] = a4;
        }
        double jn = 0.0;
        for (int j = 0; j < N; ++j) jn += vn[j] * Jc[j];
        r.jn = jn;
    }
}

// Occupation energy (calce, src/pnof.jl:1273-1300) and, when grad != nullptr,
// its gamma-gradient (calcoccg, :1324-1377).
double energy_grad(const Occ& o, const double* gamma, const double* J, const double* K, const double* Hc,
                   double* grad) {
    const int N = o.N, nv = o.nv, nc = o.ncwo;
    const OccView ov = view(o);
    thread_local OrbVecs v;
    thread_local std::vector<double> dn, w, blk;
    thread_local std::vector<RowSums> rs;
    v.n.resize(N);
    dn.resize((size_t)N * (nv > 0 ? nv : 1));
    occupations_impl(o, gamma, v.n.data(), dn.data(), false);  // only the pair blocks are read below
    dynamic(o, v.n.data(), v.nd, v.F, v.coc);
    v.fi.resize(N);
    v.nd12.resize(N);
    for (int i = 0; i < N; ++i) {
        v.fi[i] = phi_fn(v.n[i], o.ista);
        v.nd12[i] = sqrt(v.nd[i]);
    }
    const VecView vv = v.view();
    w.resize(N);
    for (int i = 0; i < N; ++i) w[i] = 2.0 * Hc[i] + J[i + (size_t)N * i];
    double E = 0.0;
    for (int i = 0; i < o.nbeta; ++i) E += v.n[i] * w[i];
    if (o.nsoc > 0)
        for (int i = o.nbeta; i < o.nalpha; ++i) E += 2.0 * v.n[i] * Hc[i];
    for (int i = o.nalpha; i < N; ++i) E += v.n[i] * w[i];
    row_sums(o, v, J, K, rs);
    // sum_ij cj12[i,j] J(j,i) - ck12[i,j] K(j,i)
    double sj = 0.0, sk = 0.0;
    for (int i = 0; i < N; ++i) {
        double rj, rk;
        row_energy(ov, vv, i, rs[i], J, K, &rj, &rk);
        sj += rj;
        sk += rk;
    }
    E += sj - sk;
    if (grad) {
        for (int k = 0; k < nv; ++k) grad[k] = 0.0;
        blk.resize((size_t)(nc + 1) * (nc > 0 ? nc : 1));
        for (int g = 0; g < o.ndoc; ++g) {
            for (int m = 0; m <= nc; ++m)
                for (int c = 0; c < nc; ++c) blk[m * nc + c] = dn[(size_t)member(ov, g, m) * nv + o.KG[g * nc + c]];
            pair_grad(ov, vv, rs.data(), J, K, w.data(), blk.data(), g, grad);
        }
    }
    return E;
}

// ------------------------------------------------------------------ CG minimiser
struct Point {
    double a, f, da;
    std::vector<double> g;
};

struct LineFn {
    const Occ& o;
    const double *J, *K, *Hc;
    const std::vector<double>& x;
    const std::vector<double>& d;
    std::vector<Point> cache;
    std::vector<double> xa;

    const Point& operator()(double a) {
        for (const Point& p : cache)
            if (p.a == a) return p;
        const int nv = o.nv;
        xa.resize(nv);
        for (int k = 0; k < nv; ++k) xa[k] = x[k] + a * d[k];
        Point p;
        p.a = a;
        p.g.resize(nv);
        p.f = energy_grad(o, xa.data(), J, K, Hc, p.g.data());
        p.da = 0.0;
        for (int k = 0; k < nv; ++k) p.da += p.g[k] * d[k];
        cache.push_back(std::move(p));
        return cache.back();
    }
};

// Armijo sufficient decrease, or Hager-Zhang's approximate Wolfe test.
bool decrease_ok(double fa, double da, double a, double f0, double d0, double c1) {
    if (fa <= f0 + c1 * a * d0) return true;
    return fa <= f0 + 1e-6 * fabs(f0) && da <= (2 * 0.1 - 1.0) * d0;
}

Point zoom(LineFn& phi, double a_lo, double a_hi, double f_lo, double d_lo, double f0, double d0, double c1,
           double c2, int max_it = 30) {
    double f_hi = phi(a_hi).f;
    for (int it = 0; it < max_it; ++it) {
        const double denom = 2.0 * (f_hi - f_lo - d_lo * (a_hi - a_lo));
        double a = denom > 0 ? a_lo - d_lo * (a_hi - a_lo) * (a_hi - a_lo) / denom : 0.5 * (a_lo + a_hi);
        const double lo = std::min(a_lo, a_hi), hi = std::max(a_lo, a_hi);
        if (!(lo + 0.1 * (hi - lo) <= a && a <= hi - 0.1 * (hi - lo))) a = 0.5 * (a_lo + a_hi);
        const Point pa = phi(a);
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
    return phi(a_lo);
}

Point wolfe(LineFn& phi, double fx, double d0, double a1, double c1 = 1e-4, double c2 = 0.1, double a_max = 1e6,
            int max_it = 30) {
    double a_prev = 0.0, f_prev = fx, dp_prev = d0, a = a1;
    Point pa;
    for (int i = 0; i < max_it; ++i) {
        pa = phi(a);
        if (!decrease_ok(pa.f, pa.da, a, fx, d0, c1) || (i > 0 && pa.f > f_prev + 1e-6 * fabs(fx)))
            return zoom(phi, a_prev, a, f_prev, dp_prev, fx, d0, c1, c2);
        if (fabs(pa.da) <= -c2 * d0) return pa;
        if (pa.da >= 0) return zoom(phi, a, a_prev, pa.f, pa.da, fx, d0, c1, c2);
        a_prev = a;
        f_prev = pa.f;
        dp_prev = pa.da;
        a = std::min(2.0 * a, a_max);
    }
    return pa;
}

double maxabs(const std::vector<double>& v) {
    double m = 0.0;
    for (double x : v) m = std::max(m, fabs(x));
    return m;
}
double dot(const std::vector<double>& a, const std::vector<double>& b) {
    double s = 0.0;
    for (size_t i = 0; i < a.size(); ++i) s += a[i] * b[i];
    return s;
}

int cg(const Occ& o, const double* J_MO, const double* K_MO, const double* H_core, double* gamma,
       double g_abstol, int max_iter, double* E, int* nit, int* converged) {
    const int nv = o.nv;
    const double eta = 0.4;
    std::vector<double> x(gamma, gamma + nv), gx(nv), d(nv), gn(nv), y(nv);
    double fx = energy_grad(o, x.data(), J_MO, K_MO, H_core, gx.data());
    *nit = 0;
    *converged = 0;
    if (maxabs(gx) <= g_abstol) {
        *E = fx;
        *converged = 1;
        return DONOF_OK;
    }
    for (int k = 0; k < nv; ++k) d[k] = -gx[k];
    double a = 1.0 / std::max(maxabs(gx), 1e-12);
    bool have_prev = false;
    double gd_prev = 0.0;
    for (int it = 1; it <= max_iter; ++it) {
        double gd = dot(gx, d);
        if (gd >= 0) {  // not a descent direction: restart
            for (int k = 0; k < nv; ++k) d[k] = -gx[k];
            gd = dot(gx, d);
        }
        if (have_prev) a = std::min(std::max(a * gd_prev / gd, 1e-10), 1e6);
        LineFn phi{o, J_MO, K_MO, H_core, x, d, {}, {}};
        const Point pt = wolfe(phi, fx, gd, a);
        a = pt.a;
        double smax = 0.0;
        for (int k = 0; k < nv; ++k) {
            const double s = a * d[k];
            smax = std::max(smax, fabs(s));
            x[k] += s;
            gn[k] = pt.g[k];
            y[k] = gn[k] - gx[k];
        }
        if (maxabs(gn) <= g_abstol) {
            std::copy(x.begin(), x.end(), gamma);
            *E = pt.f;
            *nit = it;
            *converged = 1;
            return DONOF_OK;
        }
        if (fabs(pt.f - fx) <= 0.0 && smax == 0.0) {
            std::copy(x.begin(), x.end(), gamma);
            *E = pt.f;
            *nit = it;
            return DONOF_OK;
        }
        const double dy = dot(d, y);
        double beta = 0.0;
        if (dy != 0.0) {
            const double yy = dot(y, y);
            double t = 0.0;
            for (int k = 0; k < nv; ++k) t += (y[k] - 2.0 * d[k] * yy / dy) * gn[k];
            beta = t / dy;
            const double eta_k = -1.0 / (sqrt(dot(d, d)) * std::min(eta, sqrt(dot(gx, gx))));
            beta = std::max(beta, eta_k);
        }
        gd_prev = gd;
        have_prev = true;
        for (int k = 0; k < nv; ++k) d[k] = -gn[k] + beta * d[k];
        fx = pt.f;
        gx = gn;
    }
    std::copy(x.begin(), x.end(), gamma);
    *E = fx;
    *nit = max_iter;
    return DONOF_OK;
}

}  // namespace occ
}  // namespace donof

extern "C" {

using donof::occ::Occ;
using donof::occ::setup;
using donof::occ::energy_grad;

int donof_occ_energy(const donof_occ_params* prm, const double* gamma, const double* J_MO, const double* K_MO,
                     const double* H_core, double* E, double* grad) {
    Occ o;
    if (!setup(prm, o) || !gamma || !J_MO || !K_MO || !H_core || !E) {
        donof::set_error(nullptr, "donof_occ_energy: invalid sizes or null pointer");
        return DONOF_ERR_ARG;
    }
    *E = energy_grad(o, gamma, J_MO, K_MO, H_core, grad);
    return DONOF_OK;
}

int donof_occupations(const donof_occ_params* prm, const double* gamma, double* n, double* dn_dgamma) {
    Occ o;
    if (!setup(prm, o) || !gamma || !n) {
        donof::set_error(nullptr, "donof_occupations: invalid sizes or null pointer");
        return DONOF_ERR_ARG;
    }
    std::vector<double> dn((size_t)o.N * (o.nv > 0 ? o.nv : 1), 0.0);  // dn[i * nv + k]
    donof::occ::occupations(o, gamma, n, dn.data());
    if (dn_dgamma)  // column-major N x nv (Julia's layout)
        for (int i = 0; i < o.N; ++i)
            for (int k = 0; k < o.nv; ++k) dn_dgamma[i + (size_t)o.N * k] = dn[(size_t)i * o.nv + k];
    return DONOF_OK;
}

int donof_coupling(const donof_occ_params* prm, const double* n, double* cj12, double* ck12) {
    Occ o;
    if (!setup(prm, o) || !n || !cj12 || !ck12) {
        donof::set_error(nullptr, "donof_coupling: invalid sizes or null pointer");
        return DONOF_ERR_ARG;
    }
    donof::occ::coupling(o, n, cj12, ck12);
    return DONOF_OK;
}

int donof_occ_cg(const donof_occ_params* prm, const double* J_MO, const double* K_MO, const double* H_core,
                 double* gamma, double g_abstol, int max_iter, double* E, int* nit, int* converged) {
    Occ o;
    if (!setup(prm, o) || !gamma || !J_MO || !K_MO || !H_core || !E || !nit || !converged || max_iter < 0) {
        donof::set_error(nullptr, "donof_occ_cg: invalid sizes, null pointer or max_iter < 0");
        return DONOF_ERR_ARG;
    }
    return donof::occ::cg(o, J_MO, K_MO, H_core, gamma, g_abstol, max_iter, E, nit, converged);
}

}  // extern "C"
