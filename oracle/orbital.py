"""numpy restatement of the orbital-optimiser loops -- TEST INFRASTRUCTURE ONLY.

  orbopt (ADAM / ADABelief / YOGI / Demon)   src/minimization.jl:242-630
  calcorbg                                    src/pnof.jl:1389-1407
  computeE_elec(Hmat, n, elag)                src/utils.jl:216-227

The heavy contractions come from the C oracle (``native``).  Trajectory parity
with the Julia reference is unpinned (no Julia here); these loops pin the
device optimiser to the reference's update rules step by step.
"""
from __future__ import annotations

import numpy as np

from . import gnof, native


def e_elec(Hmat, n, elag, nbf5):
    return float(np.trace(elag[:nbf5, :nbf5]) + np.sum(n[:nbf5] * np.diag(Hmat[:nbf5, :nbf5])))


def calcorbg(y, n, cj12, ck12, C, H, b, p: gnof.Sizes):
    Cn = C if y is None else native.rotate(y, C, p.nbf5)
    elag, _ = native.lagrange2(Cn, n, H, b, cj12, ck12, p.nalpha, p.nbeta)
    return gnof.pack_orbital_gradient(elag, p.nbf5)


def orbopt(method, n, cj12, ck12, C, H, b, p: gnof.Sizes, alpha: float, maxloop: int, threshgorb: float):
    """One call of orbopt_<method>; returns (E, C, nit, success, alpha, maxloop)."""
    elag, Hmat = native.lagrange2(C, n, H, b, cj12, ck12, p.nalpha, p.nbeta)
    E = e_elec(Hmat, n, elag, p.nbf5)
    nvar = p.nvar
    beta1, beta2 = (0.6, 0.999) if method == "Demon" else (0.5, 0.9)
    binit = beta1
    m = np.zeros(nvar)
    v = np.zeros(nvar)
    vmax = np.zeros(nvar)
    improved = False
    success = False
    best_E, best_C = E, C
    nit = 0
    for i in range(1, maxloop + 1):
        nit += 1
        g = gnof.pack_orbital_gradient(elag, p.nbf5)
        if 2.0 * np.max(np.abs(g)) < threshgorb and improved:
            success = True
            break
        if method == "Demon":
            rate = (i - 1.0) / (maxloop - 1.0)
            beta1 = binit * (1.0 - rate) / ((1.0 - binit) + binit * (1.0 - rate))
        m = beta1 * m + (1.0 - beta1) * g
        if method == "ADABelief":
            v = beta2 * v + (1.0 - beta2) * (g - m) ** 2
        elif method == "YOGI":
            v = v - (1.0 - beta2) * np.sign(v - g ** 2) * g ** 2
        else:
            v = beta2 * v + (1.0 - beta2) * g ** 2
        mhat = m / (1.0 - beta1 ** i)
        vhat = v / (1.0 - beta2 ** i)
        vmax = np.maximum(vmax, vhat)
        y = -alpha * mhat / np.sqrt(vmax + 1e-16)
        C = native.rotate(y, C, p.nbf5)
        elag, Hmat = native.lagrange2(C, n, H, b, cj12, ck12, p.nalpha, p.nbeta)
        E = e_elec(Hmat, n, elag, p.nbf5)
        if E < best_E:
            best_C, best_E = C, E
            improved = True
    if not improved:
        alpha = 0.3 * alpha
        maxloop = maxloop + 10
    if maxloop < 100:
        return best_E, best_C, nit, success, alpha, maxloop
    return E, C, nit, success, alpha, maxloop
