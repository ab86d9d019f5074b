"""Host-side GNOF functional layer (FP64): occupation parametrisations, the
coupling coefficients cj12/ck12, and the occupation energy / gradient from
cached J_MO, K_MO, H_core.

In DoNOF.jl these functions run on the host even with the GPU extension
loaded.  Here they are the library's native host code (occupation.cu, the one
implementation the energy loop uses as well), reached through the C ABI;
the numpy restatement of the reference lives in the oracle only.  Reference
definitions:
  ocupacion / _softmax / _trigonometric   src/pnof.jl:1024-1163
  PNOFi_selector + CJCKD8                 src/pnof.jl:1-53, 488-601
  der_PNOFi_selector + der_CJCKD8         src/pnof.jl:55-117, 603-793 (inside calcoccg)
  calce / calcocce / calcoccg             src/pnof.jl:1273-1377
  guess_gamma_softmax / _trigonometric    src/guess.jl:184-213
  order_occupations_softmax               src/utils.jl:586-616
"""
from __future__ import annotations

import ctypes as ct
import math

import numpy as np

from . import _lib
from .param import Param


def _prm(p: Param):
    from .api import _occ_params
    if p.ipnof != 8:
        raise ValueError("only GNOF (ipnof = 8) is on this path")
    return _occ_params(p)


def occupations(gamma, p: Param):
    """n (nbf5) and dn/dgamma (nbf5 x nv) for p.occ_method (donof_occupations)."""
    prm = _prm(p)
    g = np.ascontiguousarray(gamma, dtype=np.float64)
    if g.shape != (p.nv,):
        raise ValueError(f"gamma has shape {g.shape}, nv = {p.nv}")
    n = np.zeros(p.nbf5)
    dn = np.zeros((p.nbf5, p.nv), order="F")
    _lib.check(_lib.load().donof_occupations(ct.byref(prm), g.ctypes.data, n.ctypes.data, dn.ctypes.data))
    return n, dn


ocupacion = occupations


def coupling(n, p: Param):
    """cj12, ck12 of GNOF (ipnof = 8) with zeroed diagonals (donof_coupling)."""
    prm = _prm(p)
    n = np.ascontiguousarray(n, dtype=np.float64)
    cj = np.zeros((p.nbf5, p.nbf5), order="F")
    ck = np.zeros((p.nbf5, p.nbf5), order="F")
    _lib.check(_lib.load().donof_coupling(ct.byref(prm), n.ctypes.data, cj.ctypes.data, ck.ctypes.data))
    return cj, ck


PNOFi_selector = coupling


def calce(n, cj12, ck12, J_MO, K_MO, H_core, p: Param) -> float:
    """Occupation-space energy (src/pnof.jl:1273-1300)."""
    dJ = np.diag(J_MO)
    w = 2.0 * H_core + dJ
    E = float(n[: p.nbeta] @ w[: p.nbeta])
    if p.nsoc > 0:
        E += float(2.0 * n[p.nbeta: p.nalpha] @ H_core[p.nbeta: p.nalpha])
    E += float(n[p.nalpha: p.nbf5] @ w[p.nalpha: p.nbf5])
    E += float(np.sum(cj12 * J_MO.T) - np.sum(ck12 * K_MO.T))
    return E


def calcocce(gamma, J_MO, K_MO, H_core, p: Param) -> float:
    """Occupation energy at gamma (src/pnof.jl:1302-1322), native."""
    from .api import occ_energy
    return occ_energy(gamma, J_MO, K_MO, H_core, p, grad=False)[0]


def calcoccg(gamma, J_MO, K_MO, H_core, p: Param) -> np.ndarray:
    """Occupation gradient (src/pnof.jl:1324-1377), native: the nbf5 x nbf5 x nv
    derivative tensors of der_CJCKD8 are contracted with J_MO, K_MO through
    their separable terms, O(nbf5^2 + nbf5 nv) instead of O(nbf5^2 nv)."""
    from .api import occ_energy
    return occ_energy(gamma, J_MO, K_MO, H_core, p, grad=True)[1]


def guess_gamma(p: Param) -> np.ndarray:
    """Initial gamma (src/guess.jl:184-213)."""
    g = np.zeros(p.nv)
    if p.occ_method == "Softmax":
        g[p.gamma_table()] = math.log(max(0.001 / p.ncwo, 1e-16)) - math.log(0.999)
    elif p.occ_method == "Trigonometric":
        g[: p.ndoc] = math.acos(math.sqrt(2.0 * 0.999 - 1.0))
        for i in range(1, p.ndoc + 1):
            for j in range(1, p.ncwo):
                g[p.ndoc + (p.ndoc - i) + p.ndoc * (j - 1)] = math.asin(math.sqrt(1.0 / (p.ncwo - j + 1)))
    else:
        raise ValueError(p.occ_method)
    return g


def n_to_gammas(n, p: Param) -> np.ndarray:
    """gamma whose occupations are n: the restart path of DoNOF.energy
    (src/energy.jl:95-99), n_to_gammas_softmax (src/utils.jl:539-561) and
    n_to_gammas_trigonometric (src/utils.jl:563-584)."""
    n = np.asarray(n, dtype=np.float64)
    g = np.zeros(p.nv)
    nd, nc = p.ndoc, p.ncwo
    P = p.pair_table()
    if p.occ_method == "Softmax":
        # the reference divides by n[i] with i the pair index (1-based), kept as is
        g[p.gamma_table()] = np.log(np.maximum(n[P], 1e-16)) - np.log(n[:nd])[:, None]
    elif p.occ_method == "Trigonometric":
        strong = p.no1 + np.arange(nd)
        g[:nd] = np.arccos(np.sqrt(2.0 * n[strong] - 1.0))
        for i in range(nd):
            pref = max(1.0 - n[strong[i]], 1e-14)
            cols = nd + (nd - (i + 1)) + nd * np.arange(nc - 1)
            for j in range(nc - 1):
                g[cols[j]] = math.asin(math.sqrt(n[P[i, j]] / pref))
                pref *= math.cos(g[cols[j]]) ** 2
    else:
        raise ValueError(f"occupation method {p.occ_method!r} is not supported")
    return g


def order_occupations_softmax(C, gamma, p: Param):
    """Sort each pair's orbitals by gamma, descending (src/utils.jl:586-616)."""
    C = np.array(C, copy=True, order="F")
    gamma = np.array(gamma, copy=True)
    if not np.any(gamma > 0):
        return C, gamma
    C0 = C.copy()
    for g, (ws, gi) in enumerate(zip(p.pair_table(), p.gamma_table())):
        cols = np.r_[p.no1 + g, ws]
        vals = np.r_[0.0, gamma[gi]]
        order = np.argsort(vals, kind="stable")[::-1]
        vals = vals[order] - vals.max()
        gamma[gi] = vals[1:]
        C[:, cols] = C0[:, cols[order]]
    return C, gamma
