/*
 * CPU oracle for the DoNOF.jl RI hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * This file restates, in plain C with OpenMP, the reference's FP64 CPU
 * algorithm for the three contractions on the per-iteration path:
 *
 *   oracle_jkh_mo      src/integrals.jl:144-172  (JKH_MO, RI method)
 *   oracle_lagrange2   src/utils.jl:1-59         (compute_Lagrange2, RI method)
 *   oracle_expm        src/utils.jl:515          (LinearAlgebra.exp of the
 *                                                 antisymmetric rotation generator)
 *   oracle_rotate      src/utils.jl:499-521      (rotate_orbital)
 *
 * Contraction order follows the reference (full b_MO = C^T (b x_2 C5) for the
 * Lagrangian, b_pnl then b_pql for J/K).  Only the test suite, the smoke check
 * and the CPU-baseline leg of the benchmark load this library; the product
 * path never calls it.
 *
 * Parity status: the reference is Julia (Tullio/LoopVectorization) and ships
 * no tests, fixtures or golden vectors; Julia is not installed here, so these
 * restatements are pinned by the identities the reference code implies
 * (calce == computeE_elec, finite-difference gradients, orthonormality) and by
 * an independent numpy restatement, not by outputs of the reference itself:
 * parity against reference-run outputs is unpinned.
 *
 * Layout: every array is column-major with 0-based indices, exactly as Julia
 * stores it:  C[m + nbf*p], b[m + nbf*n + nbf*nbf*l], H[m + nbf*n],
 * cj12[p + nbf5*q], elag[a + nbf*b], Hmat[i + nbf*j] (nbf x nbf5),
 * J_MO[p + nbf5*q].
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static int max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

static int thread_id(void) {
#ifdef _OPENMP
    return omp_get_thread_num();
#else
    return 0;
#endif
}

int oracle_num_threads(void) { return max_threads(); }

void oracle_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* tmp[m + nbf*q] = sum_n B[m + nbf*n] * C[n + nbf*q]  for q < ncol.
 * (utils.jl:19, integrals.jl:159 with the m<->n roles as written there) */
static void mat_BC(int nbf, int ncol, const double *B, const double *C, double *tmp) {
    memset(tmp, 0, sizeof(double) * (size_t)nbf * ncol);
    for (int q = 0; q < ncol; ++q) {
        double *t = tmp + (size_t)nbf * q;
        for (int n = 0; n < nbf; ++n) {
            const double c = C[n + (size_t)nbf * q];
            const double *Bn = B + (size_t)nbf * n;
            for (int m = 0; m < nbf; ++m) t[m] += Bn[m] * c;
        }
    }
}

/* out[p + ldo*q] = sum_m A[m + nbf*p] * X[m + nbf*q]  (A^T X), p < np, q < nq */
static void mat_AtX(int nbf, int np, int nq, const double *A, const double *X,
                    double *out, int ldo) {
    for (int q = 0; q < nq; ++q) {
        const double *x = X + (size_t)nbf * q;
        for (int p = 0; p < np; ++p) {
            const double *a = A + (size_t)nbf * p;
            double s = 0.0;
            for (int m = 0; m < nbf; ++m) s += a[m] * x[m];
            out[p + (size_t)ldo * q] = s;
        }
    }
}

/*
 * compute_Lagrange2, RI method (src/utils.jl:1-59).
 *   H_mat[i,j]  = sum_mn C[m,i] H[m,n] C[n,j]                 j < nbf5   (:17-18)
 *   tmp[m,q,l]  = sum_n C5[n,q] b[m,n,l]                                 (:19)
 *   b_MO[p,q,l] = sum_m C[m,p] tmp[m,q,l]                                (:20)
 *   elag[a,b]  += n[b] H_mat[a,b]                                        (:39)
 *   elag[a,b]  += n[b] sum_k b_MO[a,b,k] b_MO[b,b,k]   b<nbeta | b>=nalpha (:42-47)
 *   elag[a,b]  += sum_k b_MO[a,b,k] sum_q cj12[b,q] b_MO[q,q,k]          (:50-51)
 *   elag[a,b]  -= sum_qk ck12[b,q] b_MO[a,q,k] b_MO[b,q,k]               (:54-55)
 * elag is nbf x nbf (columns >= nbf5 stay zero); H_mat is nbf x nbf5.
 * The per-k work is independent, so k is distributed over threads with
 * per-thread partial sums reduced in thread order.
 */
void oracle_lagrange2(int nbf, int nbf5, int naux, int nalpha, int nbeta,
                      const double *C, const double *n, const double *H,
                      const double *b, const double *cj12, const double *ck12,
                      double *elag, double *Hmat) {
    const size_t nn = (size_t)nbf * nbf;
    /* H_mat = C^T (H C5) */
    double *HC = (double *)malloc(sizeof(double) * nbf * nbf5);
    mat_BC(nbf, nbf5, H, C, HC);
    mat_AtX(nbf, nbf, nbf5, C, HC, Hmat, nbf);
    free(HC);

    const int nt = max_threads();
    double *part = (double *)calloc((size_t)nt * nbf * nbf5, sizeof(double));
    memset(elag, 0, sizeof(double) * nn);

#pragma omp parallel
    {
        double *acc = part + (size_t)thread_id() * nbf * nbf5;
        double *tmp = (double *)malloc(sizeof(double) * nbf * nbf5);
        double *bmo = (double *)malloc(sizeof(double) * nbf * nbf5);
        double *dg = (double *)malloc(sizeof(double) * nbf5);
        double *t = (double *)malloc(sizeof(double) * nbf5);
#pragma omp for schedule(static)
        for (int l = 0; l < naux; ++l) {
            const double *Bl = b + nn * l;
            mat_BC(nbf, nbf5, Bl, C, tmp);
            mat_AtX(nbf, nbf, nbf5, C, tmp, bmo, nbf); /* b_MO[:, :, l], nbf x nbf5 */
            for (int q = 0; q < nbf5; ++q) dg[q] = bmo[q + (size_t)nbf * q];
            /* dJ_pp/dy_ab */
            if (nbeta > 0) {
                for (int bb = 0; bb < nbf5; ++bb) {
                    if (!(bb < nbeta || bb >= nalpha)) continue;
                    const double f = n[bb] * dg[bb];
                    for (int a = 0; a < nbf; ++a) acc[a + (size_t)nbf * bb] += f * bmo[a + (size_t)nbf * bb];
                }
            }
            /* C^J_pq dJ_pq/dy_ab */
            for (int bb = 0; bb < nbf5; ++bb) {
                double s = 0.0;
                for (int q = 0; q < nbf5; ++q) s += cj12[bb + (size_t)nbf5 * q] * dg[q];
                t[bb] = s;
            }
            for (int bb = 0; bb < nbf5; ++bb)
                for (int a = 0; a < nbf; ++a) acc[a + (size_t)nbf * bb] += bmo[a + (size_t)nbf * bb] * t[bb];
            /* -C^K_pq dK_pq/dy_ab */
            for (int bb = 0; bb < nbf5; ++bb) {
                double *ac = acc + (size_t)nbf * bb;
                for (int q = 0; q < nbf5; ++q) {
                    const double f = ck12[bb + (size_t)nbf5 * q] * bmo[bb + (size_t)nbf * q];
                    if (f == 0.0) continue;
                    const double *bq = bmo + (size_t)nbf * q;
                    for (int a = 0; a < nbf; ++a) ac[a] -= f * bq[a];
                }
            }
        }
        free(tmp); free(bmo); free(dg); free(t);
    }
    for (int th = 0; th < nt; ++th) {
        const double *p = part + (size_t)th * nbf * nbf5;
        for (size_t i = 0; i < (size_t)nbf * nbf5; ++i) elag[i] += p[i];
    }
    free(part);
    /* 2ndH/dy_ab (added last; addition order differs from :39 only by rounding) */
    for (int bb = 0; bb < nbf5; ++bb)
        for (int a = 0; a < nbf; ++a) elag[a + (size_t)nbf * bb] += n[bb] * Hmat[a + (size_t)nbf * bb];
}

/*
 * JKH_MO, RI method (src/integrals.jl:144-172).
 *   b_pnl[p,n,l] = sum_m C5[m,p] b[m,n,l];  b_pql[p,q,l] = sum_n C5[n,q] b_pnl[p,n,l]
 *   J_MO[p,q] = sum_l b_pql[p,p,l] b_pql[q,q,l];  K_MO[p,q] = sum_l b_pql[p,q,l]^2
 *   H_core[i] = sum_mn C[m,i] C[n,i] H[m,n]
 */
void oracle_jkh_mo(int nbf, int nbf5, int naux, const double *C, const double *H,
                   const double *b, double *J, double *K, double *Hcore) {
    const size_t nn = (size_t)nbf * nbf;
    const size_t n55 = (size_t)nbf5 * nbf5;
    const int nt = max_threads();
    double *part = (double *)calloc((size_t)nt * 2 * n55, sizeof(double));
#pragma omp parallel
    {
        double *pJ = part + (size_t)thread_id() * 2 * n55;
        double *pK = pJ + n55;
        double *bpn = (double *)malloc(sizeof(double) * nbf5 * nbf); /* [p + nbf5*n] */
        double *bpq = (double *)malloc(sizeof(double) * n55);
#pragma omp for schedule(static)
        for (int l = 0; l < naux; ++l) {
            const double *Bl = b + nn * l;
            /* b_pn[p,n] = sum_m C[m,p] B[m,n] */
            for (int nq = 0; nq < nbf; ++nq) {
                const double *Bn = Bl + (size_t)nbf * nq;
                for (int p = 0; p < nbf5; ++p) {
                    const double *cp = C + (size_t)nbf * p;
                    double s = 0.0;
                    for (int m = 0; m < nbf; ++m) s += cp[m] * Bn[m];
                    bpn[p + (size_t)nbf5 * nq] = s;
                }
            }
            /* b_pq[p,q] = sum_n C[n,q] b_pn[p,n] */
            memset(bpq, 0, sizeof(double) * n55);
            for (int q = 0; q < nbf5; ++q)
                for (int nq = 0; nq < nbf; ++nq) {
                    const double c = C[nq + (size_t)nbf * q];
                    const double *src = bpn + (size_t)nbf5 * nq;
                    double *dst = bpq + (size_t)nbf5 * q;
                    for (int p = 0; p < nbf5; ++p) dst[p] += c * src[p];
                }
            for (int q = 0; q < nbf5; ++q) {
                const double dq = bpq[q + (size_t)nbf5 * q];
                for (int p = 0; p < nbf5; ++p) {
                    const double v = bpq[p + (size_t)nbf5 * q];
                    pJ[p + (size_t)nbf5 * q] += bpq[p + (size_t)nbf5 * p] * dq;
                    pK[p + (size_t)nbf5 * q] += v * v;
                }
            }
        }
        free(bpn); free(bpq);
    }
    memset(J, 0, sizeof(double) * n55);
    memset(K, 0, sizeof(double) * n55);
    for (int th = 0; th < nt; ++th) {
        const double *pJ = part + (size_t)th * 2 * n55;
        for (size_t i = 0; i < n55; ++i) { J[i] += pJ[i]; K[i] += pJ[n55 + i]; }
    }
    free(part);
    for (int i = 0; i < nbf5; ++i) {
        const double *ci = C + (size_t)nbf * i;
        double s = 0.0;
        for (int nq = 0; nq < nbf; ++nq) {
            double hs = 0.0;
            for (int m = 0; m < nbf; ++m) hs += ci[m] * H[m + (size_t)nbf * nq];
            s += hs * ci[nq];
        }
        Hcore[i] = s;
    }
}

/* ---------------------------------------------------------------------------
 * Matrix exponential: scaling and squaring with the [13/13] Pade approximant
 * (N. J. Higham, "The scaling and squaring method for the matrix exponential
 * revisited", SIAM J. Matrix Anal. Appl. 26 (2005) 1179-1193), the method
 * behind Julia's LinearAlgebra.exp used at src/utils.jl:515.  Pade
 * coefficients are generated from their closed form
 *   c_j = (2m-j)! m! / ((2m)! j! (m-j)!),  m = 13.
 * ------------------------------------------------------------------------- */
static void gemm_nn(int n, const double *A, const double *B, double *Cm) {
#pragma omp parallel for schedule(static)
    for (int j = 0; j < n; ++j) {
        double *c = Cm + (size_t)n * j;
        for (int i = 0; i < n; ++i) c[i] = 0.0;
        for (int k = 0; k < n; ++k) {
            const double bk = B[k + (size_t)n * j];
            const double *a = A + (size_t)n * k;
            for (int i = 0; i < n; ++i) c[i] += a[i] * bk;
        }
    }
}

/* Solve A X = B in place (B overwritten by X), LU with partial pivoting. */
static int lu_solve(int n, double *A, double *B, int nrhs) {
    int *piv = (int *)malloc(sizeof(int) * n);
    for (int k = 0; k < n; ++k) {
        int p = k;
        double amax = fabs(A[k + (size_t)n * k]);
        for (int i = k + 1; i < n; ++i) {
            double v = fabs(A[i + (size_t)n * k]);
            if (v > amax) { amax = v; p = i; }
        }
        piv[k] = p;
        if (amax == 0.0) { free(piv); return -1; }
        if (p != k)
            for (int j = 0; j < n; ++j) {
                double t = A[k + (size_t)n * j];
                A[k + (size_t)n * j] = A[p + (size_t)n * j];
                A[p + (size_t)n * j] = t;
            }
        const double inv = 1.0 / A[k + (size_t)n * k];
        for (int i = k + 1; i < n; ++i) A[i + (size_t)n * k] *= inv;
        for (int j = k + 1; j < n; ++j) {
            const double akj = A[k + (size_t)n * j];
            if (akj == 0.0) continue;
            for (int i = k + 1; i < n; ++i) A[i + (size_t)n * j] -= A[i + (size_t)n * k] * akj;
        }
    }
    for (int r = 0; r < nrhs; ++r) {
        double *x = B + (size_t)n * r;
        for (int k = 0; k < n; ++k)
            if (piv[k] != k) { double t = x[k]; x[k] = x[piv[k]]; x[piv[k]] = t; }
        for (int k = 0; k < n; ++k) {
            const double xk = x[k];
            for (int i = k + 1; i < n; ++i) x[i] -= A[i + (size_t)n * k] * xk;
        }
        for (int k = n - 1; k >= 0; --k) {
            x[k] /= A[k + (size_t)n * k];
            const double xk = x[k];
            for (int i = 0; i < k; ++i) x[i] -= A[i + (size_t)n * k] * xk;
        }
    }
    free(piv);
    return 0;
}

int oracle_expm(int n, const double *A, double *E) {
    const size_t nn = (size_t)n * n;
    const int m = 13;
    const double theta13 = 5.371920351148152; /* Higham 2005, Table 2.3 */
    double c[14];
    /* c_j = (2m-j)! m! / ((2m)! j! (m-j)!) built as a running product */
    c[0] = 1.0;
    for (int j = 1; j <= m; ++j) c[j] = c[j - 1] * (double)(m - j + 1) / ((double)j * (double)(2 * m - j + 1));
    double norm1 = 0.0;
    for (int j = 0; j < n; ++j) {
        double s = 0.0;
        for (int i = 0; i < n; ++i) s += fabs(A[i + (size_t)n * j]);
        if (s > norm1) norm1 = s;
    }
    int s = 0;
    if (norm1 > theta13) s = (int)ceil(log2(norm1 / theta13));
    const double scale = ldexp(1.0, -s);
    double *As = (double *)malloc(sizeof(double) * nn);
    double *A2 = (double *)malloc(sizeof(double) * nn);
    double *A4 = (double *)malloc(sizeof(double) * nn);
    double *A6 = (double *)malloc(sizeof(double) * nn);
    double *W = (double *)malloc(sizeof(double) * nn);
    double *T = (double *)malloc(sizeof(double) * nn);
    double *U = (double *)malloc(sizeof(double) * nn);
    double *V = (double *)malloc(sizeof(double) * nn);
    for (size_t i = 0; i < nn; ++i) As[i] = A[i] * scale;
    gemm_nn(n, As, As, A2);
    gemm_nn(n, A2, A2, A4);
    gemm_nn(n, A4, A2, A6);
    /* U = A [A6 (c13 A6 + c11 A4 + c9 A2) + c7 A6 + c5 A4 + c3 A2 + c1 I] */
    for (size_t i = 0; i < nn; ++i) W[i] = c[13] * A6[i] + c[11] * A4[i] + c[9] * A2[i];
    gemm_nn(n, A6, W, T);
    for (size_t i = 0; i < nn; ++i) T[i] += c[7] * A6[i] + c[5] * A4[i] + c[3] * A2[i];
    for (int i = 0; i < n; ++i) T[i + (size_t)n * i] += c[1];
    gemm_nn(n, As, T, U);
    /* V = A6 (c12 A6 + c10 A4 + c8 A2) + c6 A6 + c4 A4 + c2 A2 + c0 I */
    for (size_t i = 0; i < nn; ++i) W[i] = c[12] * A6[i] + c[10] * A4[i] + c[8] * A2[i];
    gemm_nn(n, A6, W, V);
    for (size_t i = 0; i < nn; ++i) V[i] += c[6] * A6[i] + c[4] * A4[i] + c[2] * A2[i];
    for (int i = 0; i < n; ++i) V[i + (size_t)n * i] += c[0];
    /* (V - U) X = (V + U) */
    for (size_t i = 0; i < nn; ++i) { T[i] = V[i] - U[i]; E[i] = V[i] + U[i]; }
    int rc = lu_solve(n, T, E, n);
    for (int k = 0; k < s; ++k) {
        gemm_nn(n, E, E, T);
        memcpy(E, T, sizeof(double) * nn);
    }
    free(As); free(A2); free(A4); free(A6); free(W); free(T); free(U); free(V);
    return rc;
}

/*
 * rotate_orbital (src/utils.jl:499-521): unpack y row-wise over i < nbf5,
 * j > i into the antisymmetric Y (Y[i,j] = y, Y[j,i] = -y), U = exp(Y),
 * Cnew = C U.
 */
int oracle_rotate(int nbf, int nbf5, const double *y, const double *C, double *Cnew) {
    const size_t nn = (size_t)nbf * nbf;
    double *Y = (double *)calloc(nn, sizeof(double));
    double *U = (double *)malloc(sizeof(double) * nn);
    size_t k = 0;
    for (int i = 0; i < nbf5; ++i)
        for (int j = i + 1; j < nbf; ++j) {
            Y[i + (size_t)nbf * j] = y[k];
            Y[j + (size_t)nbf * i] = -y[k];
            ++k;
        }
    int rc = oracle_expm(nbf, Y, U);
    gemm_nn(nbf, C, U, Cnew);
    free(Y); free(U);
    return rc;
}
