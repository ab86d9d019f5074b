"""Starting orbitals and occupations of an energy job (host, FP64, one-time
set-up; DoNOF.jl does this on the host too).

  guess_C        src/energy.jl:67-71, 80:  Ei, Cguess = eigen(H, S); check_ortho
  check_ortho    src/utils.jl:431-466: orthonormality test (1e-6), orthonormalize
                 on violation, then each orbital's sign set so that its largest
                 coefficient (the first one among equals) is positive
  orthonormalize src/utils.jl:468-496: Loewdin-type S^{-1/2} frame (negative
                 eigenvalues of S dropped), Gram-Schmidt, back-transform
  guess_gamma    src/guess.jl:184-213 (gnof.guess_gamma)

The generalized eigenvectors come from SciPy's symmetric-definite solver
(S-orthonormal, ascending eigenvalues), so check_ortho only applies the sign
convention; for non-degenerate spectra this is the orbital set the reference's
eigen + check_ortho produce.
"""
from __future__ import annotations

from typing import Optional, Tuple

import numpy as np
import scipy.linalg

from . import gnof
from .param import Param


def orthonormalize(C, S):
    """src/utils.jl:468-496."""
    C = np.array(C, dtype=np.float64)
    S = np.asarray(S, dtype=np.float64)
    evals, evecs = np.linalg.eigh(S)
    inv = np.where(evals < 0.0, 0.0, 1.0 / np.sqrt(np.where(evals < 0.0, 1.0, evals)))
    S12 = evecs * inv[None, :]
    C2 = S12.T @ (S @ C)
    nbf = C.shape[0]
    ncol = min(C2.shape)  # the reference's inner bound is the row count; C is square there
    for i in range(C2.shape[1]):
        C2[:nbf, i] = C2[:nbf, i] / np.linalg.norm(C2[:nbf, i])
        for j in range(i + 1, ncol):
            val = -np.sum(C2[:nbf, i] * C2[:nbf, j])
            C2[:nbf, j] = C2[:nbf, j] + val * C2[:nbf, i]
    return S12 @ C2


def check_ortho(C, S, max_rounds: int = 10):
    """src/utils.jl:431-466 (returns a new array)."""
    C = np.array(C, dtype=np.float64, order="F")
    S = np.asarray(S, dtype=np.float64)
    for _ in range(max_rounds):
        dev = np.abs(C.T @ S @ C - np.eye(C.shape[1]))
        if np.max(dev) <= 1e-6:
            break
        C = np.asfortranarray(orthonormalize(C, S))
    idx = np.argmax(np.abs(C), axis=0)  # first maximum, like the reference's strict '>' scan
    signs = np.sign(C[idx, np.arange(C.shape[1])])
    signs[signs == 0] = 1.0
    return np.asfortranarray(C * signs[None, :])


def guess_C(H, S=None):
    """Orbitals of the core Hamiltonian: the generalized eigenvectors of (H, S)
    in ascending order of eigenvalue, S-orthonormal, sign convention of
    check_ortho.  Returns (eigenvalues, C)."""
    H = np.asarray(H, dtype=np.float64)
    S = np.eye(H.shape[0]) if S is None else np.asarray(S, dtype=np.float64)
    e, C = scipy.linalg.eigh(H, S)
    return e, check_ortho(C, S)


def guess(H, p: Param, S=None, C: Optional[np.ndarray] = None) -> Tuple[np.ndarray, np.ndarray]:
    """(C, gamma) to start DoNOF.energy from: the given C (orthonormalised) or
    the core-Hamiltonian guess, and the reference's initial gamma."""
    S = np.eye(np.asarray(H).shape[0]) if S is None else S
    if C is None:
        _, C = guess_C(H, S)
    C = check_ortho(C, S)
    return C, gnof.guess_gamma(p)
