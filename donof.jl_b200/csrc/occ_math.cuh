// Per-orbital and per-pair formulas of the GNOF occupation layer, shared by
// the host code (occupation.cu) and the device occupation solver
// (occ_device.cu), so that both evaluate the same expressions:
//   occupations of a pair       ocupacion_softmax / _trigonometric (src/pnof.jl:1047-1163)
//   n_d, F, coc of a pair       the dynamic part of CJCKD8 (src/pnof.jl:488-601)
//   phi(n), d phi / d n         CJCKD8 / der_CJCKD8 per ista (src/pnof.jl:488-793)
//   generic / special ck12, derivative factors, their row sums
//   the energy terms of one row and the gradient of one pair (calce /
//   calcoccg through the separable terms of der_CJCKD8, src/pnof.jl:1273-1377)
// Matrices J, K are column-major, X(i, j) = X[i + N j].
#pragma once

#include <math.h>

namespace donof {
namespace occ {

#define OCC_HD __host__ __device__ __forceinline__

// Sizes and index tables (names of src/param.jl): strong orbital S[g] of pair
// g, its weak partners P[g*ncwo + w] and their gamma entries G[g*ncwo + w], the
// ncwo gamma entries of the pair's dn block KG[g*ncwo + c], and the pair of each
// orbital grp[i] (-1 outside the pairs).
struct OccView {
    int N, no1, ndoc, nsoc, nbeta, nalpha, ncwo, nv, ista, high_spin, method;
    double h_cut;
    const int *S, *P, *G, *KG, *grp;
};

// Per-orbital vectors n, phi(n), n_d^{1/2}, n_d and per-pair F, coc.
struct VecView {
    const double *n, *fi, *nd12, *nd, *F, *coc;
};

enum : int { V_N = 0, V_FI, V_ND12, V_ND, V_ONE, NVEC };

// S[R][k] = sum over j in class range R of vec_k[j] K(j, i); jn = sum_j n_j J(j, i)
struct RowSums {
    double S[4][NVEC];
    double jn;
};

OCC_HD int cls(const OccView& o, int i) { return i < o.no1 ? 0 : (i < o.nbeta ? 1 : (i < o.nalpha ? 2 : 3)); }

// member m of pair g: 0 the strong orbital, 1..ncwo the weak ones
OCC_HD int member(const OccView& o, int g, int m) { return m == 0 ? o.S[g] : o.P[g * o.ncwo + m - 1]; }

OCC_HD double phi_fn(double ni, int ista) {
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

// d phi / d n_i (the factor of dfi = dphi * dn, der_CJCKD8)
OCC_HD double dphi_factor(int ista, double ni) {
    double f = ni * (1.0 - ni);
    if (f < 0.0) f = 0.0;
    if (ista == 3) {
        const double al = 0.55, aa = pow(pow(2.0, 2.0 * al - 1.0), 1.0 / al);
        const double t = aa * ni * (1.0 - ni);
        const double a = t > 1e-15 ? t : 1e-15;
        return al * pow(a, al - 1.0) * aa * (1.0 - 2.0 * ni);
    }
    const double fi0 = sqrt(f) * (ista == 2 ? 0.9 : 1.0);
    const double a = fi0 > 1e-15 ? fi0 : 1e-15;
    const double scale = (ista == 2) ? 0.81 : 1.0;
    double fac = scale / (2.0 * a) * (1.0 - 2.0 * ni);
    if (ista == 4) {
        const double e = exp(-(ni - 0.5) * (ni - 0.5));
        fac = fac * e - fi0 * 2.0 * (ni - 0.5) * e;
    }
    return fac;
}

// ---- occupations of one pair ---------------------------------------------------
// Pass 1 (every pair before pass 2): n of the pair's members.
OCC_HD void pair_n(const OccView& o, const double* gamma, int g, double* n) {
    const int nc = o.ncwo, nd = o.ndoc;
    if (o.method == 0) {  // softmax (src/pnof.jl:1122-1163)
        double s = 1.0;
        for (int c = 0; c < nc; ++c) s += exp(gamma[o.G[g * nc + c]]);
        const double inv = 1.0 / s;
        n[o.S[g]] = inv;
        for (int c = 0; c < nc; ++c) n[o.P[g * nc + c]] = exp(gamma[o.G[g * nc + c]]) * inv;
        return;
    }
    // trigonometric (src/pnof.jl:1047-1120)
    const double cs = cos(gamma[g]);
    const double ns = 0.5 * (1.0 + cs * cs);
    n[o.S[g]] = ns;
    const double h = 1.0 - ns;
    for (int w = 0; w < nc; ++w) {
        double fac = 1.0;
        for (int k = 0; k < nc - 1; ++k) {
            const double th = gamma[nd + (nd - (g + 1)) + nd * k];
            const double sn = sin(th), c = cos(th);
            if (k == w) fac *= sn * sn;
            else if (k < w) fac *= c * c;
        }
        n[o.P[g * nc + w]] = h * fac;
    }
}

// Pass 2: the pair's dn block, blk[m * ncwo + c] = dn[member m, KG[g*ncwo + c]]
// (the only nonzero entries of the pair's rows).  Softmax reads n[g], the
// pair index (the reference's src/pnof.jl:1152, kept as is), so every pair's n
// must be set first.
OCC_HD void pair_dn(const OccView& o, const double* gamma, int g, const double* n, double* blk) {
    const int nc = o.ncwo, nd = o.ndoc;
    if (o.method == 0) {
        for (int c = 0; c < nc; ++c) {
            const double wc = n[o.P[g * nc + c]];
            blk[c] = -n[g] * wc;
        }
        for (int a = 0; a < nc; ++a)
            for (int b = 0; b < nc; ++b) {
                const double wa = n[o.P[g * nc + a]], wb = n[o.P[g * nc + b]];
                blk[(a + 1) * nc + b] = (a == b ? wa : 0.0) - wa * wb;
            }
        return;
    }
    // trigonometric: column 0 is the strong angle g, columns 1.. the weak angles
    // (the strong orbital's row is zero there)
    for (int c = 1; c < nc; ++c) blk[c] = 0.0;
    const double nsg = n[o.S[g]];
    const double dstrong = -0.5 * sin(2.0 * gamma[g]);
    const int nb = nc - 1;
    double s2[64], c2[64], th[64];  // ncwo <= 65 (checked by setup)
    for (int j = 0; j < nb; ++j) {
        th[j] = gamma[nd + (nd - (g + 1)) + nd * j];
        const double sn = sin(th[j]), cs = cos(th[j]);
        s2[j] = sn * sn;
        c2[j] = cs * cs;
    }
    blk[0] = dstrong;
    for (int w = 0; w < nc; ++w) {
        double fac = 1.0;
        for (int k = 0; k < nb; ++k) {
            if (k == w) fac *= s2[k];
            else if (k < w) fac *= c2[k];
        }
        blk[(w + 1) * nc + 0] = -dstrong * fac;
    }
    // weak-angle columns: B(r, j) of the host formulation, r over the weak members
    for (int j = 0; j < nb; ++j) {
        for (int r = 0; r < nc; ++r) {
            double v;
            if (r < j) {
                v = 0.0;
            } else if (r == j) {
                v = 1.0 - nsg;
                for (int k = 0; k <= j; ++k) v *= (k == j) ? sin(2.0 * th[k]) : c2[k];
            } else {
                v = nsg - 1.0;
                for (int k = 0; k < j; ++k) v *= c2[k];
                v *= sin(2.0 * th[j]);
                for (int k = j + 1; k < nb; ++k) {
                    if (k == r) v *= s2[k];
                    else if (k < r) v *= c2[k];
                }
            }
            blk[(r + 1) * nc + 1 + j] = v;
        }
    }
}

// n_d, F and coc of pair g (src/pnof.jl:488-601); nd is zero outside the pairs
OCC_HD void pair_dynamic(const OccView& o, const double* n, int g, double* nd, double* F, double* coc) {
    const double c = (o.ista == 5) ? 0.8 : 1.0;
    coc[g] = (1.0 - n[o.S[g]]) / o.h_cut;
    F[g] = c * exp(-coc[g] * coc[g]);
    nd[o.S[g]] = n[o.S[g]] * F[g];
    for (int w = 0; w < o.ncwo; ++w) nd[o.P[g * o.ncwo + w]] = n[o.P[g * o.ncwo + w]] * F[g];
}

// ---- couplings ---------------------------------------------------------------------
// generic ck(i, j) of CJCKD8, before the pair overrides
OCC_HD double gen_ck(const OccView& o, const VecView& v, int i, int j) {
    const int ci = cls(o, i), cj = cls(o, j);
    const bool ibe = ci == 1, ial = ci == 2, icw = ci == 3, jbe = cj == 1, jal = cj == 2, jcw = cj == 3;
    double k = v.n[i] * v.n[j];
    if (o.ista == 0) {
        if ((ibe && jcw) || (icw && jbe) || (icw && jcw)) k += v.fi[i] * v.fi[j];
        if (o.nsoc > 0) {
            if (ibe && jal) k += 0.25 * v.fi[i];
            if (ial && jbe) k += 0.25 * v.fi[j];
            if (ial && jcw) k += 0.5 * v.fi[j];
            if (icw && jal) k += 0.5 * v.fi[i];
        }
        if (o.nsoc > 1 && ial && jal) k = 0.5;
    } else {
        k += v.fi[i] * v.fi[j];
    }
    if ((ibe && jcw) || (icw && jbe)) k += v.nd12[i] * v.nd12[j] - v.nd[i] * v.nd[j];
    if (icw && jcw) k -= v.nd12[i] * v.nd12[j] + v.nd[i] * v.nd[j];
    return k;
}

// sum_j gen_ck(i, j) K(j, i) from the row sums
OCC_HD double row_ck(const OccView& o, const VecView& v, int i, const RowSums& r) {
    const int ci = cls(o, i);
    const double ni = v.n[i], fi = v.fi[i];
    double s = ni * (r.S[0][V_N] + r.S[1][V_N] + r.S[2][V_N] + r.S[3][V_N]);
    if (o.ista == 0) {
        if (ci == 1) s += fi * r.S[3][V_FI];
        if (ci == 3) s += fi * (r.S[1][V_FI] + r.S[3][V_FI]);
        if (o.nsoc > 0) {
            if (ci == 1) s += 0.25 * fi * r.S[2][V_ONE];
            if (ci == 2) s += 0.25 * r.S[1][V_FI] + 0.5 * r.S[3][V_FI];
            if (ci == 3) s += 0.5 * fi * r.S[2][V_ONE];
        }
        if (o.nsoc > 1 && ci == 2) s += 0.5 * r.S[2][V_ONE] - ni * r.S[2][V_N];
    } else {
        s += fi * (r.S[0][V_FI] + r.S[1][V_FI] + r.S[2][V_FI] + r.S[3][V_FI]);
    }
    if (ci == 1) s += v.nd12[i] * r.S[3][V_ND12] - v.nd[i] * r.S[3][V_ND];
    if (ci == 3)
        s += v.nd12[i] * (r.S[1][V_ND12] - r.S[3][V_ND12]) - v.nd[i] * (r.S[1][V_ND] + r.S[3][V_ND]);
    return s;
}

// ck(i, j) inside a pair, i != j: strong-weak sqrt(n_s n_w), weak-weak -sqrt(n_w) sqrt(n_v)
OCC_HD double spec_ck(const OccView& o, const VecView& v, int i, int j) {
    const int g = o.grp[i];
    if (i == o.S[g]) return sqrt(v.n[i] * v.n[j]);
    if (j == o.S[g]) return sqrt(v.n[j] * v.n[i]);
    return -(sqrt(v.n[i]) * sqrt(v.n[j]));
}

// generic derivative factors M_t(r, j) (t = 0..3) and Mcj(r, j) for a row r in a pair
OCC_HD void gen_m(const OccView& o, const VecView& v, int r, int j, double (&m)[4], double& mcj) {
    const int cr = cls(o, r), cj = cls(o, j);
    const bool rbe = cr == 1, rcw = cr == 3, jbe = cj == 1, jal = cj == 2, jcw = cj == 3;
    mcj = 2.0 * v.n[j];
    m[0] = v.n[j];
    m[1] = m[2] = m[3] = 0.0;
    if (o.ista == 0) {
        if ((rbe && jcw) || (rcw && jbe) || (rcw && jcw)) m[1] += v.fi[j];
        if (o.nsoc > 0) {
            if (rbe && jal) m[1] += 0.25;
            if (rcw && jal) m[1] += 0.5;
        }
    } else {
        m[1] += v.fi[j];
    }
    if ((rbe && jcw) || (rcw && jbe)) {
        m[2] += v.nd12[j];
        m[3] -= v.nd[j];
    }
    if (rcw && jcw) {
        m[2] -= v.nd12[j];
        m[3] -= v.nd[j];
    }
}

// sum_j M_t(r, j) K(j, r) for the generic factors of a row r in a pair
OCC_HD void row_m(const OccView& o, int r, const RowSums& s, double (&vk)[4]) {
    const int cr = cls(o, r);
    vk[0] = s.S[0][V_N] + s.S[1][V_N] + s.S[2][V_N] + s.S[3][V_N];
    if (o.ista == 0) {
        vk[1] = (cr == 1) ? s.S[3][V_FI] : s.S[1][V_FI] + s.S[3][V_FI];
        if (o.nsoc > 0) vk[1] += (cr == 1 ? 0.25 : 0.5) * s.S[2][V_ONE];
    } else {
        vk[1] = s.S[0][V_FI] + s.S[1][V_FI] + s.S[2][V_FI] + s.S[3][V_FI];
    }
    if (cr == 1) {
        vk[2] = s.S[3][V_ND12];
        vk[3] = -s.S[3][V_ND];
    } else {
        vk[2] = s.S[1][V_ND12] - s.S[3][V_ND12];
        vk[3] = -s.S[1][V_ND] - s.S[3][V_ND];
    }
}

// ---- energy and gradient ---------------------------------------------------------
// Row i of sum_ij cj12[i,j] J(j,i) and of sum_ij ck12[i,j] K(j,i): the generic
// row from the row sums, minus the generic values on i's pair (or on the
// diagonal), plus the pair's special values.
OCC_HD void row_energy(const OccView& o, const VecView& v, int i, const RowSums& r, const double* J, const double* K,
                       double* rj_out, double* rk_out) {
    const int N = o.N, nc = o.ncwo;
    double rj = 2.0 * v.n[i] * r.jn, rk = row_ck(o, v, i, r);
    const int g = o.grp[i];
    const int cnt = (g < 0) ? 1 : nc + 1;
    for (int m = 0; m < cnt; ++m) {
        const int j = (g < 0) ? i : member(o, g, m);
        const double Jji = J[j + (size_t)N * i], Kji = K[j + (size_t)N * i];
        rj -= 2.0 * v.n[i] * v.n[j] * Jji;
        rk -= gen_ck(o, v, i, j) * Kji;
        if (j != i) rk += spec_ck(o, v, i, j) * Kji;
    }
    *rj_out = rj;
    *rk_out = rk;
}

// The gradient entries of pair g: grad[KG[g*ncwo + c]] += its members'
// contributions (calcoccg through the separable terms of der_CJCKD8).  rs[r]
// holds the row sums of orbital r, blk the pair's dn block (pair_dn), w[r] =
// 2 H_core[r] + J(r, r).
OCC_HD void pair_grad(const OccView& o, const VecView& v, const RowSums* rs, const double* J, const double* K,
                      const double* w, const double* blk, int g, double* grad) {
    const int N = o.N, nc = o.ncwo;
    const int s = o.S[g];
    const double kk = 2.0 * v.coc[g] / o.h_cut;
    const double sa = sqrt(v.n[s] > 1e-15 ? v.n[s] : 1e-15);
    for (int m = 0; m <= nc; ++m) {
        const int r = member(o, g, m);
        const RowSums& rr = rs[r];
        // vj = sum_j Mcj(r,j) J(j,r), vk_t = sum_j M_t(r,j) K(j,r)
        double vj = 2.0 * rr.jn, vk[4];
        row_m(o, r, rr, vk);
        const double sb = sqrt(v.n[r] > 1e-15 ? v.n[r] : 1e-15);
        for (int q = 0; q <= nc; ++q) {  // the pair's members: generic values out, special in
            const int j = member(o, g, q);
            double mg[4], mcj;
            gen_m(o, v, r, j, mg, mcj);
            const double Jjr = J[j + (size_t)N * r], Kjr = K[j + (size_t)N * r];
            vj -= mcj * Jjr;
            for (int t = 0; t < 4; ++t) vk[t] -= mg[t] * Kjr;
            if (j == r) continue;
            double m0;
            if (r == s) m0 = 0.5 / sa * sqrt(v.n[j]);
            else if (j == s) m0 = 0.5 / sb * sqrt(v.n[s]);
            else m0 = -0.5 * (1.0 / sb) * sqrt(v.n[j]);
            vk[0] += m0 * Kjr;
        }
        const double cdn = w[r] + 2.0 * vj;
        const double fac = dphi_factor(o.ista, v.n[r]);
        const double den = v.nd12[r] > 1e-15 ? v.nd12[r] : 1e-15;
        for (int c = 0; c < nc; ++c) {
            const int k = o.KG[g * nc + c];
            const double a0 = blk[m * nc + c];
            const double a3 = (r == s) ? v.F[g] * a0 * (1.0 + v.n[s] * kk)
                                       : v.F[g] * a0 + v.F[g] * kk * v.n[r] * blk[c];
            const double a1 = fac * a0, a2 = 0.5 * a3 / den;
            grad[k] += a0 * cdn - 2.0 * (a0 * vk[0] + a1 * vk[1] + a2 * vk[2] + a3 * vk[3]);
        }
    }
}

}  // namespace occ
}  // namespace donof
