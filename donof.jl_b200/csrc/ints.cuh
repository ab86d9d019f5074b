// Gaussian integrals by the McMurchie-Davidson scheme (McMurchie and Davidson,
// J. Comput. Phys. 26, 218 (1978); as set out in Helgaker, Jorgensen and
// Olsen, "Molecular Electronic-Structure Theory", ch. 9): products of
// Cartesian Gaussians expanded in Hermite Gaussians (coefficients E^{ij}_t by
// the two-term recursion), Coulomb-type integrals from the Hermite integrals
// R^n_{tuv} (recursion from the Boys function).  The same __host__ __device__
// code computes the integrals on the host (tests, one-electron matrices) and
// in the B200 kernel of the three-centre integrals (ints.cu).
//
// Replaces the integral engine the reference calls through GaussianBasis.jl
// (src/integrals.jl:1-49: overlap, kinetic, nuclear, ERI_2e2c, ERI_2e3c,
// ERI_2e4c).
#pragma once

#include <math.h>

namespace donof {
namespace ints {

constexpr int LMAX = 5;                 // highest angular momentum of a shell (h)
constexpr int NBOYS = 4 * LMAX + 1;     // Boys orders for a four-centre integral

__host__ __device__ constexpr int ncart(int l) { return (l + 1) * (l + 2) / 2; }

// Cartesian exponents of component c of shell l, in the order
// xx..x, xx..y, ..., zz..z (x power descending, then y power descending).
__host__ __device__ inline void cart_xyz(int l, int c, int* lx, int* ly, int* lz) {
    int k = 0;
    for (int a = l; a >= 0; --a)
        for (int b = l - a; b >= 0; --b) {
            if (k == c) {
                *lx = a;
                *ly = b;
                *lz = l - a - b;
                return;
            }
            ++k;
        }
    *lx = *ly = *lz = 0;
}

// Boys function F_n(T) for n = 0..nmax (nmax < NBOYS + 1).  For T <= 35 the
// highest order comes from the series F_m(T) = e^-T sum_k (2T)^k /
// ((2m+1)(2m+3)...(2m+2k+1)) (all terms positive) and the others by the
// downward recursion F_{m-1} = (2T F_m + e^-T) / (2m - 1); above 35, F_0 =
// sqrt(pi/T)/2 (erf(sqrt T) is 1 to double precision there) and the upward
// recursion F_{m+1} = ((2m+1) F_m - e^-T) / (2T), stable for large T.
__host__ __device__ inline void boys(int nmax, double T, double* F) {
    if (T < 1e-14) {
        for (int n = 0; n <= nmax; ++n) F[n] = 1.0 / (2 * n + 1) - T / (2 * n + 3);
        return;
    }
    const double et = exp(-T);
    if (T <= 35.0) {
        double term = 1.0 / (2 * nmax + 1), sum = term;
        for (int k = 1; k < 200; ++k) {
            term *= 2.0 * T / (2 * nmax + 2 * k + 1);
            sum += term;
            if (term < 1e-17 * sum) break;
        }
        F[nmax] = et * sum;
        for (int m = nmax; m > 0; --m) F[m - 1] = (2.0 * T * F[m] + et) / (2 * m - 1);
    } else {
        F[0] = 0.5 * sqrt(3.14159265358979323846 / T);
        for (int m = 0; m < nmax; ++m) F[m + 1] = ((2 * m + 1) * F[m] - et) / (2.0 * T);
    }
}

// 1-D Hermite expansion coefficients E^{ij}_t (i <= la, j <= lb, t <= i + j)
// of the product of x^i e^{-a x_A^2} and x^j e^{-b x_B^2}, with XAB = A - B:
//   E^{00}_0 = exp(-ab/(a+b) XAB^2),
//   E^{i+1,j}_t = E^{ij}_{t-1} / (2p) + X_PA E^{ij}_t + (t+1) E^{ij}_{t+1}  (and j alike),
// stored E[e_index(la, lb, i, j, t)] ((la+1)(lb+1)(la+lb+1) doubles); b = 0 with
// XAB = 0 gives the expansion of a single Gaussian (an auxiliary function).
__host__ __device__ constexpr int e_size(int la, int lb) { return (la + 1) * (lb + 1) * (la + lb + 1); }
__host__ __device__ inline int e_index(int la, int lb, int i, int j, int t) {
    return (i * (lb + 1) + j) * (la + lb + 1) + t;
}
__host__ __device__ inline void hermite_e(int la, int lb, double a, double b, double XAB, double* E) {
    const double p = a + b, mu = a * b / p;
    const double XPA = -b / p * XAB, XPB = a / p * XAB, h = 0.5 / p;
    const int T = la + lb + 1;
    for (int k = 0; k < e_size(la, lb); ++k) E[k] = 0.0;
    E[0] = exp(-mu * XAB * XAB);
    for (int i = 0; i <= la; ++i) {
        for (int j = 0; j <= lb; ++j) {
            if (i == 0 && j == 0) continue;
            double* out = E + (i * (lb + 1) + j) * T;
            const double* src = (i > 0) ? E + ((i - 1) * (lb + 1) + j) * T : E + (j - 1) * T;
            const double X = (i > 0) ? XPA : XPB;
            const int top = i + j - 1;  // highest t of the source
            for (int t = 0; t <= i + j; ++t) {
                double v = (t <= top) ? X * src[t] : 0.0;
                if (t > 0) v += h * src[t - 1];
                if (t + 1 <= top) v += (t + 1) * src[t + 1];
                out[t] = v;
            }
        }
    }
}

// Packed index of (t, u, v) among all t + u + v <= L (shells of s = t + u + v).
__host__ __device__ constexpr int tri_size(int L) { return (L + 1) * (L + 2) * (L + 3) / 6; }
__host__ __device__ inline int tri(int t, int u, int v) {
    const int s = t + u + v, r = s - t;
    return s * (s + 1) * (s + 2) / 6 + r * (r + 1) / 2 + v;
}

// Hermite Coulomb integrals R_{tuv} = R^0_{tuv}(alpha, PC) for t + u + v <= L,
// stored R[tri(t, u, v)]; scratch holds 2 * tri_size(L) doubles (two levels n
// of the recursion R^n_{t+1,u,v} = t R^{n+1}_{t-1,u,v} + X_PC R^{n+1}_{t,u,v}).
__host__ __device__ inline void hermite_r(int L, double alpha, double X, double Y, double Z, double* R,
                                          double* scratch) {
    double F[NBOYS + 2];
    boys(L, alpha * (X * X + Y * Y + Z * Z), F);
    double* lv[2] = {scratch, scratch + tri_size(L)};
    // level n holds R^n_{tuv} for t + u + v <= L - n
    double fpow[NBOYS + 2];
    fpow[0] = 1.0;
    for (int n = 1; n <= L; ++n) fpow[n] = fpow[n - 1] * (-2.0 * alpha);
    double* up = lv[L & 1];
    up[0] = fpow[L] * F[L];
    for (int n = L - 1; n >= 0; --n) {
        double* cur = (n == 0) ? R : lv[n & 1];
        const int m = L - n;
        cur[0] = fpow[n] * F[n];
        for (int t = 0; t <= m; ++t)
            for (int u = 0; u + t <= m; ++u)
                for (int v = 0; v + u + t <= m; ++v) {
                    if (t + u + v == 0) continue;
                    double r;
                    if (t > 0) {
                        r = X * up[tri(t - 1, u, v)];
                        if (t > 1) r += (t - 1) * up[tri(t - 2, u, v)];
                    } else if (u > 0) {
                        r = Y * up[tri(t, u - 1, v)];
                        if (u > 1) r += (u - 1) * up[tri(t, u - 2, v)];
                    } else {
                        r = Z * up[tri(t, u, v - 1)];
                        if (v > 1) r += (v - 1) * up[tri(t, u, v - 2)];
                    }
                    cur[tri(t, u, v)] = r;
                }
        up = cur;
    }
    if (L == 0) R[0] = F[0];
}

// Scratch doubles coulomb_prim needs for angular momenta la, lb, lc, ld.
__host__ __device__ constexpr int coulomb_scratch(int la, int lb, int lc, int ld) {
    return 3 * e_size(la, lb) + 3 * e_size(lc, ld) + 3 * tri_size(la + lb + lc + ld) + tri_size(la + lb);
}

// w (ab|cd) over one primitive of each of a, b, c, d (exponents a..d, centres
// A..D, Cartesian components of the shells' angular momenta), added into
// out[((ia * nb + ib) * nc + ic) * nd + id]:
//   (ab|cd) = 2 pi^{5/2} / (p q sqrt(p + q)) sum_{tuv} E^{ab}_{tuv}
//             sum_{t'u'v'} (-1)^{t'+u'+v'} E^{cd}_{t'u'v'} R_{t+t',u+u',v+v'}(pq/(p+q), P - Q).
// A single (auxiliary) Gaussian is a pair with the second exponent 0 and l 0.
__host__ __device__ inline void coulomb_prim(int la, int lb, double a, double b, const double* A, const double* B,
                                             int lc, int ld, double c, double d, const double* C, const double* D,
                                             double w, double* out, double* scr) {
    const double p = a + b, q = c + d, alpha = p * q / (p + q);
    double P[3], Q[3];
    for (int k = 0; k < 3; ++k) {
        P[k] = (a * A[k] + b * B[k]) / p;
        Q[k] = (c * C[k] + d * D[k]) / q;
    }
    const int e1 = e_size(la, lb), e2 = e_size(lc, ld), L = la + lb + lc + ld, lab = la + lb;
    double* E1 = scr;
    double* E2 = E1 + 3 * e1;
    double* R = E2 + 3 * e2;
    double* rs = R + tri_size(L);
    double* G = rs + 2 * tri_size(L);
    for (int k = 0; k < 3; ++k) {
        hermite_e(la, lb, a, b, A[k] - B[k], E1 + k * e1);
        hermite_e(lc, ld, c, d, C[k] - D[k], E2 + k * e2);
    }
    hermite_r(L, alpha, P[0] - Q[0], P[1] - Q[1], P[2] - Q[2], R, rs);
    const double pref = w * 34.986836655249725 / (p * q * sqrt(p + q));  // 2 pi^{5/2}
    const int na = ncart(la), nb = ncart(lb), nc = ncart(lc), nd = ncart(ld);
    for (int ic = 0; ic < nc; ++ic) {
        int cx, cy, cz;
        cart_xyz(lc, ic, &cx, &cy, &cz);
        for (int id = 0; id < nd; ++id) {
            int dx, dy, dz;
            cart_xyz(ld, id, &dx, &dy, &dz);
            const double* ex = E2 + 0 * e2;
            const double* ey = E2 + 1 * e2;
            const double* ez = E2 + 2 * e2;
            for (int t = 0; t <= lab; ++t)
                for (int u = 0; u + t <= lab; ++u)
                    for (int v = 0; v + u + t <= lab; ++v) {
                        double g = 0.0;
                        for (int t2 = 0; t2 <= cx + dx; ++t2) {
                            const double fx = ex[e_index(lc, ld, cx, dx, t2)];
                            if (fx == 0.0) continue;
                            for (int u2 = 0; u2 <= cy + dy; ++u2) {
                                const double fxy = fx * ey[e_index(lc, ld, cy, dy, u2)];
                                if (fxy == 0.0) continue;
                                for (int v2 = 0; v2 <= cz + dz; ++v2) {
                                    const double f = fxy * ez[e_index(lc, ld, cz, dz, v2)];
                                    const double r = R[tri(t + t2, u + u2, v + v2)];
                                    g += ((t2 + u2 + v2) & 1) ? -f * r : f * r;
                                }
                            }
                        }
                        G[tri(t, u, v)] = g;
                    }
            for (int ia = 0; ia < na; ++ia) {
                int ax, ay, az;
                cart_xyz(la, ia, &ax, &ay, &az);
                for (int ib = 0; ib < nb; ++ib) {
                    int bx, by, bz;
                    cart_xyz(lb, ib, &bx, &by, &bz);
                    double val = 0.0;
                    for (int t = 0; t <= ax + bx; ++t) {
                        const double fx = E1[e_index(la, lb, ax, bx, t)];
                        for (int u = 0; u <= ay + by; ++u) {
                            const double fxy = fx * E1[e1 + e_index(la, lb, ay, by, u)];
                            for (int v = 0; v <= az + bz; ++v)
                                val += fxy * E1[2 * e1 + e_index(la, lb, az, bz, v)] * G[tri(t, u, v)];
                        }
                    }
                    out[((ia * nb + ib) * nc + ic) * nd + id] += pref * val;
                }
            }
        }
    }
}

// Scratch doubles one_e_prim needs.
__host__ __device__ inline int one_e_scratch(int la, int lb) {
    return 3 * e_size(la, lb + 2) + 3 * tri_size(la + lb);
}

// w times the overlap, kinetic energy and nuclear attraction (sum over the
// natom nuclei of charge Z[k] at xyz[3k..3k+2]) between one primitive of a
// and one of b, for every pair of Cartesian components, added into
// S/T/V[ia * nb + ib] (T or V may be null):
//   S = E^x_0 E^y_0 E^z_0 (pi/p)^{3/2};
//   T from the 1-D kinetic integrals -2b^2 S_{i,j+2} + b(2j+1) S_{ij} - j(j-1)/2 S_{i,j-2};
//   V = -sum_C Z_C (2 pi / p) sum_{tuv} E^x_t E^y_u E^z_v R_{tuv}(p, P - C).
__host__ __device__ inline void one_e_prim(int la, int lb, double a, double b, const double* A, const double* B,
                                           int natom, const double* Z, const double* xyz, double w, double* S,
                                           double* T, double* V, double* scr) {
    const double p = a + b;
    const int es = e_size(la, lb + 2), lab = la + lb;
    double* E = scr;
    double* R = E + 3 * es;
    double* rs = R + tri_size(lab);
    double P[3];
    for (int k = 0; k < 3; ++k) {
        P[k] = (a * A[k] + b * B[k]) / p;
        hermite_e(la, lb + 2, a, b, A[k] - B[k], E + k * es);
    }
    const double s1 = sqrt(3.14159265358979323846 / p);
    const int na = ncart(la), nb = ncart(lb);
    auto s1d = [&](int k, int i, int j) -> double {
        return (j < 0) ? 0.0 : E[k * es + e_index(la, lb + 2, i, j, 0)] * s1;
    };
    auto t1d = [&](int k, int i, int j) -> double {
        return -2.0 * b * b * s1d(k, i, j + 2) + b * (2 * j + 1) * s1d(k, i, j) - 0.5 * j * (j - 1) * s1d(k, i, j - 2);
    };
    for (int ia = 0; ia < na; ++ia) {
        int ax[3];
        cart_xyz(la, ia, &ax[0], &ax[1], &ax[2]);
        for (int ib = 0; ib < nb; ++ib) {
            int bx[3];
            cart_xyz(lb, ib, &bx[0], &bx[1], &bx[2]);
            const double sx = s1d(0, ax[0], bx[0]), sy = s1d(1, ax[1], bx[1]), sz = s1d(2, ax[2], bx[2]);
            S[ia * nb + ib] += w * sx * sy * sz;
            if (T)
                T[ia * nb + ib] += w * (t1d(0, ax[0], bx[0]) * sy * sz + sx * t1d(1, ax[1], bx[1]) * sz +
                                        sx * sy * t1d(2, ax[2], bx[2]));
        }
    }
    if (!V) return;
    for (int c = 0; c < natom; ++c) {
        hermite_r(lab, p, P[0] - xyz[3 * c], P[1] - xyz[3 * c + 1], P[2] - xyz[3 * c + 2], R, rs);
        const double f = -w * Z[c] * 2.0 * 3.14159265358979323846 / p;
        for (int ia = 0; ia < na; ++ia) {
            int ax[3];
            cart_xyz(la, ia, &ax[0], &ax[1], &ax[2]);
            for (int ib = 0; ib < nb; ++ib) {
                int bx[3];
                cart_xyz(lb, ib, &bx[0], &bx[1], &bx[2]);
                double val = 0.0;
                for (int t = 0; t <= ax[0] + bx[0]; ++t)
                    for (int u = 0; u <= ax[1] + bx[1]; ++u)
                        for (int v = 0; v <= ax[2] + bx[2]; ++v)
                            val += E[e_index(la, lb + 2, ax[0], bx[0], t)] *
                                   E[es + e_index(la, lb + 2, ax[1], bx[1], u)] *
                                   E[2 * es + e_index(la, lb + 2, ax[2], bx[2], v)] * R[tri(t, u, v)];
                V[ia * nb + ib] += f * val;
            }
        }
    }
}

}  // namespace ints
}  // namespace donof
