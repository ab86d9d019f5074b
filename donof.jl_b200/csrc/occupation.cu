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
    if (o.N <= 0 || o.ndoc < 0 || o.nsoc < 0 || o.ncwo < 0 || o.no1 < 0 || o.ista < 0 || o.ista > 5 ||
        (o.method != 0 && o.method != 1) || o.h_cut <= 0.0)
        return false;
    const int ndns = o.ndoc + o.nsoc;
    if (o.no1 + ndns + o.ndoc * o.ncwo > o.N) return false;
    o.S.resize(o.ndoc);
    o.P.resize((size_t)o.ndoc * o.ncwo);
    o.G.resize((size_t)o.ndoc * o.ncwo);
    for (int g = 0; g < o.ndoc; ++g) {
        o.S[g] = o.no1 + g;
        for (int w = 0; w < o.ncwo; ++w) {
            // Julia's ll:ndoc:ul for strong orbital g+1 (src/param.jl, pnof.jl)
            o.P[g * o.ncwo + w] = o.no1 + ndns + (o.ndoc - (g + 1)) + o.ndoc * w;
            o.G[g * o.ncwo + w] = (o.ndoc - (g + 1)) + o.ndoc * w;
        }
    }
    return true;
}

// n (N) and dn (N x nv, dn[i * nv + k]) for the configured occupation map
void occupations(const Occ& o, const double* gamma, double* n, double* dn) {
    const int N = o.N, nv = o.nv, nd = o.ndoc, nc = o.ncwo;
    for (int i = 0; i < N; ++i) n[i] = 0.0;
    for (int i = 0; i < o.no1; ++i) n[i] = 1.0;
    for (int i = o.no1 + nd; i < o.no1 + nd + o.nsoc; ++i) n[i] = o.high_spin ? 1.0 : 0.5;
    std::fill(dn, dn + (size_t)N * nv, 0.0);
    if (o.method == 0) {  // softmax (src/pnof.jl:1122-1163)
        std::vector<double> w((size_t)nd * nc);
        for (int g = 0; g < nd; ++g) {
            double s = 1.0;
            for (int c = 0; c < nc; ++c) {
                w[g * nc + c] = exp(gamma[o.G[g * nc + c]]);
                s += w[g * nc + c];
            }
            const double inv = 1.0 / s;
            n[o.S[g]] = inv;
            for (int c = 0; c < nc; ++c) {
                w[g * nc + c] *= inv;
                n[o.P[g * nc + c]] = w[g * nc + c];
            }
        }
        for (int g = 0; g < nd; ++g) {
            // src/pnof.jl:1152 multiplies by n[i] with i the pair index (kept as is)
            for (int c = 0; c < nc; ++c) dn[(size_t)o.S[g] * nv + o.G[g * nc + c]] = -n[g] * w[g * nc + c];
            for (int a = 0; a < nc; ++a)
                for (int b = 0; b < nc; ++b)
                    dn[(size_t)o.P[g * nc + a] * nv + o.G[g * nc + b]] =
                        (a == b ? w[g * nc + a] : 0.0) - w[g * nc + a] * w[g * nc + b];
        }
        return;
    }
    // trigonometric (src/pnof.jl:1047-1120)
    std::vector<double> dstrong(nd);
    for (int g = 0; g < nd; ++g) {
        const double c = cos(gamma[g]);
        n[o.S[g]] = 0.5 * (1.0 + c * c);
        dstrong[g] = -0.5 * sin(2.0 * gamma[g]);
    }
    std::vector<int> cols(std::max(nc - 1, 0));
    std::vector<double> th(std::max(nc - 1, 0)), s2(std::max(nc - 1, 0)), c2(std::max(nc - 1, 0)), fac(nc),
        blk((size_t)nc * std::max(nc - 1, 1)), col(nc);
    for (int g = 0; g < nd; ++g) {
        for (int j = 0; j < nc - 1; ++j) {
            cols[j] = nd + (nd - (g + 1)) + nd * j;
            th[j] = gamma[cols[j]];
            const double sn = sin(th[j]), cs = cos(th[j]);
            s2[j] = sn * sn;
            c2[j] = cs * cs;
        }
        const double h = 1.0 - n[o.S[g]];
        std::fill(fac.begin(), fac.end(), 1.0);
        for (int k = 0; k < nc - 1; ++k) {
            fac[k] *= s2[k];
            for (int m = k + 1; m < nc; ++m) fac[m] *= c2[k];
        }
        for (int w = 0; w < nc; ++w) n[o.P[g * nc + w]] = h * fac[w];
        dn[(size_t)o.S[g] * nv + g] = dstrong[g];
        for (int w = 0; w < nc; ++w) dn[(size_t)o.P[g * nc + w] * nv + g] = -dstrong[g] * fac[w];
        const int nb = nc - 1;
        auto B = [&](int r, int c) -> double& { return blk[(size_t)r * nb + c]; };
        for (int j = 0; j < nb; ++j) {
            for (int r = 0; r < nc; ++r) col[r] = n[o.S[g]] - 1.0;
            for (int r = 0; r <= j; ++r) col[r] = 0.0;
            for (int k = 0; k < j; ++k)
                for (int r = j + 1; r < nc; ++r) col[r] *= c2[k];
            for (int r = j + 1; r < nc; ++r) col[r] *= sin(2.0 * th[j]);
            for (int k = j + 1; k < nb; ++k) {
                col[k] *= s2[k];
                for (int r = k + 1; r < nc; ++r) col[r] *= c2[k];
            }
            for (int r = 0; r < nc; ++r) B(r, j) = col[r];
        }
        for (int j = 0; j < nb; ++j) B(j, j) = 1.0 - n[o.S[g]];
        for (int k = 0; k < nb; ++k) {
            B(k, k) *= sin(2.0 * th[k]);
            for (int l = k + 1; l < nb; ++l) B(l, l) *= c2[k];
        }
        for (int r = 0; r < nc; ++r)
            for (int j = 0; j < nb; ++j) dn[(size_t)o.P[g * nc + r] * nv + cols[j]] = B(r, j);
    }
}

double phi_fn(double ni, int ista) {
    double f = ni * (1.0 - ni);
    if (f < 0.0) f = 0.0;
    switch (ista) {
        case 0: case 1: case 5: return sqrt(f);
        case 2: return 0.9 * sqrt(f);
        case 3: {
            const double a = 0.55, aa = pow(pow(2.0, 2.0 * a - 1.0), 1.0 / a);
            return pow(aa * f, a);
        }
        default: return sqrt(f) * exp(-(ni - 0.5) * (ni - 0.5));  // ista 4
    }
}

// n_d, F and coc of the dynamic part (src/pnof.jl:488-601)
void dynamic(const Occ& o, const double* n, std::vector<double>& nd, std::vector<double>& F,
             std::vector<double>& coc) {
    const double c = (o.ista == 5) ? 0.8 : 1.0;
    nd.assign(o.N, 0.0);
    F.assign(o.ndoc, 0.0);
    coc.assign(o.ndoc, 0.0);
    for (int g = 0; g < o.ndoc; ++g) {
        coc[g] = (1.0 - n[o.S[g]]) / o.h_cut;
        F[g] = c * exp(-coc[g] * coc[g]);
        nd[o.S[g]] = n[o.S[g]] * F[g];
        for (int w = 0; w < o.ncwo; ++w) nd[o.P[g * o.ncwo + w]] = n[o.P[g * o.ncwo + w]] * F[g];
    }
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

// Separable terms of der_CJCKD8: Dcj[i,j,:] = Mcj[i,j] dn[i,:],
// Dck[i,j,:] = sum_t M[t][i,j] A[t][i,:], A = (dn, dfi, dnd12, dnd).
void derivative_factors(const Occ& o, const double* n, const double* dn, std::vector<double>& dfi,
                        std::vector<double>& dnd12, std::vector<double>& dnd, std::vector<double>& Mcj,
                        std::vector<double> (&M)[4]) {
    const int N = o.N, nv = o.nv;
    std::vector<double> nd, F, coc;
    dynamic(o, n, nd, F, coc);
    dnd.assign((size_t)N * nv, 0.0);
    for (int g = 0; g < o.ndoc; ++g) {
        const int s = o.S[g];
        const double k = 2.0 * coc[g] / o.h_cut;
        for (int c = 0; c < nv; ++c) dnd[(size_t)s * nv + c] = F[g] * dn[(size_t)s * nv + c] * (1.0 + n[s] * k);
        for (int a = 0; a < o.ncwo; ++a) {
            const int w = o.P[g * o.ncwo + a];
            for (int c = 0; c < nv; ++c)
                dnd[(size_t)w * nv + c] = F[g] * dn[(size_t)w * nv + c] + F[g] * k * n[w] * dn[(size_t)s * nv + c];
        }
    }
    std::vector<double> nd12(N), fi(N);
    dnd12.assign((size_t)N * nv, 0.0);
    for (int i = 0; i < N; ++i) {
        nd12[i] = sqrt(nd[i]);
        const double den = std::max(nd12[i], 1e-15);
        for (int c = 0; c < nv; ++c) dnd12[(size_t)i * nv + c] = 0.5 * dnd[(size_t)i * nv + c] / den;
    }
    dfi.assign((size_t)N * nv, 0.0);
    for (int i = 0; i < N; ++i) {
        double f = n[i] * (1.0 - n[i]);
        if (f < 0.0) f = 0.0;
        fi[i] = phi_fn(n[i], o.ista);
        if (i < o.no1) continue;
        double fac;
        if (o.ista == 3) {
            const double al = 0.55, aa = pow(pow(2.0, 2.0 * al - 1.0), 1.0 / al);
            const double a = std::max(aa * n[i] * (1.0 - n[i]), 1e-15);
            fac = al * pow(a, al - 1.0) * aa * (1.0 - 2.0 * n[i]);
        } else {
            const double fi0 = sqrt(f) * (o.ista == 2 ? 0.9 : 1.0);
            const double a = std::max(fi0, 1e-15);
            const double scale = (o.ista == 2) ? 0.81 : 1.0;
            fac = scale / (2.0 * a) * (1.0 - 2.0 * n[i]);
            if (o.ista == 4) {
                const double e = exp(-(n[i] - 0.5) * (n[i] - 0.5));
                fac = fac * e - fi0 * 2.0 * (n[i] - 0.5) * e;
            }
        }
        for (int c = 0; c < nv; ++c) dfi[(size_t)i * nv + c] = fac * dn[(size_t)i * nv + c];
    }
    const int b0 = o.no1, b1 = o.nbeta, a1 = o.nalpha, c1 = N;
    Mcj.assign((size_t)N * N, 0.0);
    for (auto& m : M) m.assign((size_t)N * N, 0.0);
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) {
            const bool ibe = in(i, b0, b1), ial = in(i, b1, a1), icw = in(i, a1, c1);
            const bool jbe = in(j, b0, b1), jal = in(j, b1, a1), jcw = in(j, a1, c1);
            const size_t ij = (size_t)i * N + j;
            Mcj[ij] = 2.0 * n[j];
            M[0][ij] = n[j];
            if (o.ista == 0) {
                if ((ibe && jcw) || (icw && jbe) || (icw && jcw)) M[1][ij] += fi[j];
                if (o.nsoc > 0) {
                    if (ibe && jal) M[1][ij] += 0.25;
                    if (icw && jal) M[1][ij] += 0.5;
                }
            } else {
                M[1][ij] += fi[j];
            }
            if (o.nsoc > 1 && ial && jal)
                for (auto& m : M) m[ij] = 0.0;
            if ((ibe && jcw) || (icw && jbe)) {
                M[2][ij] += nd12[j];
                M[3][ij] -= nd[j];
            }
            if (icw && jcw) {
                M[2][ij] -= nd12[j];
                M[3][ij] -= nd[j];
            }
        }
    for (int g = 0; g < o.ndoc; ++g) {
        const int s = o.S[g];
        const double sa = sqrt(std::max(n[s], 1e-15));
        for (int a = 0; a < o.ncwo; ++a) {
            const int w = o.P[g * o.ncwo + a];
            const double sb = sqrt(std::max(n[w], 1e-15));
            Mcj[(size_t)s * N + w] = Mcj[(size_t)w * N + s] = 0.0;
            for (auto& m : M) m[(size_t)s * N + w] = m[(size_t)w * N + s] = 0.0;
            M[0][(size_t)s * N + w] = 0.5 / sa * sqrt(n[w]);
            M[0][(size_t)w * N + s] = 0.5 / sb * sqrt(n[s]);
            for (int b = 0; b < o.ncwo; ++b) {
                const int v = o.P[g * o.ncwo + b];
                Mcj[(size_t)w * N + v] = 0.0;
                for (auto& m : M) m[(size_t)w * N + v] = 0.0;
                M[0][(size_t)w * N + v] = -0.5 * (1.0 / sb) * sqrt(n[v]);
            }
        }
    }
    for (int i = 0; i < N; ++i) {
        Mcj[(size_t)i * N + i] = 0.0;
        for (auto& m : M) m[(size_t)i * N + i] = 0.0;
    }
}

// Occupation energy (calce, src/pnof.jl:1273-1300) and, when grad != nullptr,
// its gamma-gradient (calcoccg, :1324-1377).
double energy_grad(const Occ& o, const double* gamma, const double* J, const double* K, const double* Hc,
                   double* grad) {
    const int N = o.N, nv = o.nv;
    std::vector<double> n(N), dn((size_t)N * nv), cj((size_t)N * N), ck((size_t)N * N);
    occupations(o, gamma, n.data(), dn.data());
    coupling(o, n.data(), cj.data(), ck.data());
    auto Jm = [&](int i, int j) { return J[i + (size_t)N * j]; };
    auto Km = [&](int i, int j) { return K[i + (size_t)N * j]; };
    std::vector<double> w(N);
    for (int i = 0; i < N; ++i) w[i] = 2.0 * Hc[i] + Jm(i, i);
    double E = 0.0;
    for (int i = 0; i < o.nbeta; ++i) E += n[i] * w[i];
    if (o.nsoc > 0)
        for (int i = o.nbeta; i < o.nalpha; ++i) E += 2.0 * n[i] * Hc[i];
    for (int i = o.nalpha; i < N; ++i) E += n[i] * w[i];
    double sj = 0.0, sk = 0.0;
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) {
            sj += cj[(size_t)i * N + j] * Jm(j, i);
            sk += ck[(size_t)i * N + j] * Km(j, i);
        }
    E += sj - sk;
    if (grad) {
        std::vector<double> dfi, dnd12, dnd, Mcj;
        std::vector<double> M[4];
        derivative_factors(o, n.data(), dn.data(), dfi, dnd12, dnd, Mcj, M);
        const double* A[4] = {dn.data(), dfi.data(), dnd12.data(), dnd.data()};
        for (int k = 0; k < nv; ++k) grad[k] = 0.0;
        auto row = [&](int r) { return (r >= o.no1 && r < o.nbeta) || (r >= o.nalpha && r < N); };
        for (int r = 0; r < N; ++r) {
            if (!row(r)) continue;
            double vj = 0.0, vk[4] = {0.0, 0.0, 0.0, 0.0};
            for (int j = 0; j < N; ++j) {
                vj += Mcj[(size_t)r * N + j] * Jm(j, r);
                for (int t = 0; t < 4; ++t) vk[t] += M[t][(size_t)r * N + j] * Km(j, r);
            }
            for (int k = 0; k < nv; ++k) {
                double g = dn[(size_t)r * nv + k] * w[r] + 2.0 * dn[(size_t)r * nv + k] * vj;
                for (int t = 0; t < 4; ++t) g -= 2.0 * A[t][(size_t)r * nv + k] * vk[t];
                grad[k] += g;
            }
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
