"""Oracle (test infrastructure only): restatement of Iaux (src/integrals.jl:68-91).

    G = Symmetric(G)                        (the upper triangle)
    evals, evecs = eigen(G)
    sqrtinv_i = 0 if evals_i < 0 else 1 / sqrt(evals_i)
    Gmsqrt = evecs * Diagonal(sqrtinv) * evecs'
    I[m, :, :] = I[m, :, :] * Gmsqrt        for every m

Used only by tests to check the library's donof_iaux.
"""
import numpy as np


def iaux(G, I):
    """b[m, n, l] = sum_k I[m, n, k] Gmsqrt[k, l] (FP64, numpy)."""
    G = np.asarray(G, dtype=np.float64)
    Gs = np.triu(G) + np.triu(G, 1).T          # Symmetric(G, :U)
    w, V = np.linalg.eigh(Gs)
    s = np.where(w < 0.0, 0.0, 1.0 / np.sqrt(np.where(w < 0.0, 1.0, w)))
    Gm = (V * s) @ V.T
    nbf, _, naux = I.shape
    return np.tensordot(np.asarray(I, dtype=np.float64), Gm, axes=([2], [0]))
