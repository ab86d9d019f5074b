"""ctypes wrapper of liboracle.so (the C/OpenMP oracle) -- test infrastructure only."""
from __future__ import annotations

import ctypes as ct
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def lib() -> ct.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = ct.CDLL(str(LIB))
        vp, i = ct.c_void_p, ct.c_int
        L.oracle_lagrange2.argtypes = [i, i, i, i, i] + [vp] * 8
        L.oracle_lagrange2.restype = None
        L.oracle_jkh_mo.argtypes = [i, i, i] + [vp] * 6
        L.oracle_jkh_mo.restype = None
        L.oracle_expm.argtypes = [i, vp, vp]
        L.oracle_expm.restype = i
        L.oracle_rotate.argtypes = [i, i, vp, vp, vp]
        L.oracle_rotate.restype = i
        L.oracle_num_threads.restype = i
        L.oracle_set_threads.argtypes = [i]
        _lib = L
    return _lib


def _f(a):
    return np.asfortranarray(np.asarray(a, dtype=np.float64))


def _p(a):
    return a.ctypes.data


def set_threads(n: int) -> None:
    lib().oracle_set_threads(int(n))


def num_threads() -> int:
    return int(lib().oracle_num_threads())


def lagrange2(C, n, H, b, cj12, ck12, nalpha, nbeta):
    """compute_Lagrange2, RI (src/utils.jl:1-59) -> elag, H_mat."""
    C, n, H, b, cj12, ck12 = map(_f, (C, n, H, b, cj12, ck12))
    nbf, naux, nbf5 = C.shape[0], b.shape[2], n.shape[0]
    elag = np.zeros((nbf, nbf), order="F")
    Hmat = np.zeros((nbf, nbf5), order="F")
    lib().oracle_lagrange2(nbf, nbf5, naux, int(nalpha), int(nbeta), _p(C), _p(n), _p(H), _p(b), _p(cj12),
                           _p(ck12), _p(elag), _p(Hmat))
    return elag, Hmat


def jkh_mo(C, H, b, nbf5):
    """JKH_MO, RI (src/integrals.jl:144-172) -> J_MO, K_MO, H_core."""
    C, H, b = map(_f, (C, H, b))
    nbf, naux = C.shape[0], b.shape[2]
    J = np.zeros((nbf5, nbf5), order="F")
    K = np.zeros((nbf5, nbf5), order="F")
    Hc = np.zeros(nbf5)
    lib().oracle_jkh_mo(nbf, nbf5, naux, _p(C), _p(H), _p(b), _p(J), _p(K), _p(Hc))
    return J, K, Hc


def expm(A):
    A = _f(A)
    E = np.zeros_like(A, order="F")
    rc = lib().oracle_expm(A.shape[0], _p(A), _p(E))
    if rc != 0:
        raise np.linalg.LinAlgError("singular Pade denominator")
    return E


def rotate(y, C, nbf5):
    """rotate_orbital (src/utils.jl:499-521)."""
    y, C = _f(y), _f(C)
    Cn = np.zeros_like(C, order="F")
    rc = lib().oracle_rotate(C.shape[0], int(nbf5), _p(y), _p(C), _p(Cn))
    if rc != 0:
        raise np.linalg.LinAlgError("singular Pade denominator")
    return Cn
