"""BLAS mirror of the reference's threaded CPU path -- test infrastructure
and CPU baseline only, never the product.

The reference evaluates compute_Lagrange2 (src/utils.jl:1-59) and JKH_MO
(src/integrals.jl:144-172) with threaded Tullio/LoopVectorization loop nests.
This module states the same contractions, in the same order, as FP64 BLAS
GEMMs on the host CPU (torch's CPU matmul: MKL/OpenBLAS over all host
threads), so that the CPU baseline is a tuned CPU code and not the scalar
loops of donof_oracle.c:

  tmp    = H C5,                 H_mat = C^T tmp                  (utils.jl:17-18)
  tmp_l  = b_l C5,               b_MO_l = C^T tmp_l  for every l   (utils.jl:19-20)
  elag[:, b] = n_b H_mat[:, b]
             + [b < nbeta or b >= nalpha] n_b sum_k b_MO[:, b, k] b_MO[b, b, k]
             + sum_k b_MO[:, b, k] (cj12 D)[b, k]
             - sum_{q,k} b_MO[:, q, k] ck12[b, q] b_MO[b, q, k]      (utils.jl:39-55)

with D[q, k] = b_MO[q, q, k]; the last three terms are one GEMM over (q, k)
(the first two sit on its diagonal q = b).  rotate_orbital (src/utils.jl:
499-521) uses scipy's expm (Pade scaling and squaring, like Julia's exp).
Results agree with the C oracle to rounding (tests/test_oracle.py).
"""
from __future__ import annotations

import numpy as np
import scipy.linalg
import torch


def threads() -> int:
    """Host threads the CPU GEMMs use."""
    return int(torch.get_num_threads())


def _t(a):
    return torch.from_numpy(np.asarray(a, dtype=np.float64))


def _bl(b):
    """b[m, n, l] (Julia layout) as a stack over l of nbf x nbf matrices [m, n]."""
    return _t(b).permute(2, 0, 1)


def transform(C, b, nbf5):
    """tmp[l] = b_l C5 and b_MO[l] = C^T tmp[l]: tensors (naux, nbf, nbf5)."""
    tC = _t(C)
    tmp = torch.matmul(_bl(b), tC[:, :nbf5].contiguous())
    b_MO = torch.matmul(tC.T, tmp)
    return tmp, b_MO


def lagrange2(C, n, H, b, cj12, ck12, nalpha, nbeta):
    """compute_Lagrange2, RI method (src/utils.jl:1-59) -> elag, H_mat."""
    tC, tn = _t(C), _t(n)
    nbf, nbf5 = tC.shape[0], tn.shape[0]
    H_mat = tC.T @ (_t(H) @ tC[:, :nbf5])
    _, bm = transform(C, b, nbf5)                       # bm[k, a, b] = b_MO[a, b, k]
    naux = bm.shape[0]
    D = torch.diagonal(bm[:, :nbf5, :nbf5], dim1=1, dim2=2).T.contiguous()   # D[q, k]
    # dJ_pp/dy_ab and the C^J term are sum_k b_MO[a, b, k] w[b, k]
    w = _t(cj12) @ D
    if nbeta > 0:
        sel = torch.zeros(nbf5, dtype=torch.bool)
        sel[:nbeta] = True
        sel[nalpha:] = True
        w[sel] += tn[sel, None] * D[sel]
    # -C^K_pq dK_pq/dy_ab is -sum_{q,k} b_MO[a, q, k] ck12[b, q] b_MO[b, q, k]; with the
    # w terms on the diagonal q = b, all three are one GEMM over (q, k)
    Wk = _t(ck12)[:, :, None] * bm[:, :nbf5, :].permute(1, 2, 0)            # Wk[b, q, k]
    idx = torch.arange(nbf5)
    Wk[idx, idx, :] -= w
    A = bm.permute(1, 2, 0).reshape(nbf, nbf5 * naux)                      # A[a, (q, k)]
    g = H_mat * tn[None, :] - A @ Wk.reshape(nbf5, nbf5 * naux).T
    elag = np.zeros((nbf, nbf), order="F")
    elag[:, :nbf5] = g.numpy()
    return elag, np.asfortranarray(H_mat.numpy())


def jkh_mo(C, H, b, nbf5):
    """JKH_MO, RI method (src/integrals.jl:144-172) -> J_MO, K_MO, H_core."""
    tC = _t(C)
    C5 = tC[:, :nbf5].contiguous()
    t = torch.matmul(C5.T, _bl(b))                       # b_pnl[l] = C5^T b_l      (p x n)
    bpq = torch.matmul(t, C5)                            # b_pql[l] = b_pnl[l] C5   (p x q)
    d = torch.diagonal(bpq, dim1=1, dim2=2)              # d[l, p] = b_pp^l
    J = d.T @ d
    K = torch.square(bpq).sum(dim=0)
    Hc = (C5 * (_t(H) @ C5)).sum(dim=0)
    return np.asfortranarray(J.numpy()), np.asfortranarray(K.numpy()), Hc.numpy()


def rotate(y, C, nbf5):
    """rotate_orbital (src/utils.jl:499-521): C exp(Y), Y antisymmetric from y."""
    C = np.asarray(C, dtype=np.float64)
    nbf = C.shape[0]
    Y = np.zeros((nbf, nbf))
    iu = np.triu_indices(nbf, 1)
    sel = iu[0] < nbf5
    Y[iu[0][sel], iu[1][sel]] = y
    Y -= Y.T
    return np.asfortranarray(C @ scipy.linalg.expm(Y))
