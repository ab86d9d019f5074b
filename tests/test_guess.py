"""Starting orbitals (eigen(H, S) + check_ortho, src/energy.jl:67-80,
src/utils.jl:431-496) against an independent restatement: Cholesky reduction
of the generalized problem, the same sign convention."""
import numpy as np

from donof_b200 import gnof
from donof_b200.guess import check_ortho, guess, guess_C
from donof_b200.param import Param


def _hs(n, seed):
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((n, n))
    H = 0.5 * (A + A.T) + np.diag(np.linspace(-3.0, 3.0, n))
    B = rng.standard_normal((n, n)) * 0.1
    S = np.eye(n) + 0.5 * (B + B.T)
    S = S @ S.T / n + np.eye(n)          # symmetric positive definite
    return H, S


def _reference_guess(H, S):
    L = np.linalg.cholesky(S)
    Li = np.linalg.inv(L)
    e, V = np.linalg.eigh(Li @ H @ Li.T)
    C = Li.T @ V
    idx = np.argmax(np.abs(C), axis=0)
    return e, C * np.sign(C[idx, np.arange(C.shape[1])])[None, :]


def test_guess_c_matches_cholesky_reduction():
    for n, seed in ((13, 1), (40, 2)):
        H, S = _hs(n, seed)
        e, C = guess_C(H, S)
        e0, C0 = _reference_guess(H, S)
        assert np.max(np.abs(e - e0)) <= 1e-10 * np.max(np.abs(e0))
        assert np.max(np.abs(C - C0)) <= 1e-8
        assert np.max(np.abs(C.T @ S @ C - np.eye(n))) <= 1e-10
        assert np.max(np.abs(H @ C - S @ C * e[None, :])) <= 1e-9
        idx = np.argmax(np.abs(C), axis=0)
        assert np.all(C[idx, np.arange(n)] > 0)


def test_check_ortho_repairs_a_perturbed_set():
    H, S = _hs(24, 3)
    _, C = guess_C(H, S)
    rng = np.random.default_rng(4)
    Cp = C + 1e-3 * rng.standard_normal(C.shape)
    C2 = check_ortho(Cp, S)
    assert np.max(np.abs(C2.T @ S @ C2 - np.eye(24))) <= 1e-10
    assert np.max(np.abs(C2 - C)) <= 1e-2               # close to the orbitals it repaired
    idx = np.argmax(np.abs(C2), axis=0)
    assert np.all(C2[idx, np.arange(24)] > 0)
    # an orthonormal set only has its signs adjusted
    C3 = check_ortho(-C, S)
    assert np.max(np.abs(C3 - C)) == 0.0


def test_guess_returns_reference_gamma():
    p = Param(nbf=24, nbfaux=10, nbeta=5, nalpha=5)
    H, S = _hs(24, 5)
    C, g = guess(H, p, S)
    assert np.array_equal(g, gnof.guess_gamma(p))
    assert np.max(np.abs(C.T @ S @ C - np.eye(24))) <= 1e-10
