"""numpy/C restatement of the occupation optimiser and the energy outer loop --
TEST INFRASTRUCTURE ONLY.

  occoptr   src/minimization.jl:100-139, with SciPy's CG standing in for
            Optim.jl 1.13.2 ConjugateGradient (not vendored; same stopping
            rule: max|grad| <= g_abstol = threshen)
  energy    src/energy.jl:140-220
  ENERGY1r  src/utils.jl:117-136

Trajectories differ from Optim.jl's line search; converged energies are what
the tests compare.
"""
from __future__ import annotations

import numpy as np
import scipy.optimize

from . import gnof, native, orbital


def occoptr(gamma, C, H, b, s: gnof.Sizes, threshen: float, maxloop: int):
    J, K, Hc = native.jkh_mo(C, H, b, s.nbf5)
    res = scipy.optimize.minimize(lambda x: gnof.calcocce(x, J, K, Hc, s), gamma,
                                  jac=lambda x: gnof.calcoccg(x, J, K, Hc, s), method="CG",
                                  options={"gtol": threshen, "norm": np.inf, "maxiter": 1000})
    gamma = res.x
    if res.nit < 1:
        maxloop += 10
    n, _ = gnof.ocupacion(gamma, s)
    cj12, ck12 = gnof.PNOFi_selector(n, s)
    return float(res.fun), gamma, n, cj12, ck12, maxloop


def energy1r(C, n, H, b, cj12, ck12, s: gnof.Sizes):
    elag, _ = native.lagrange2(C, n, H, b, cj12, ck12, s.nalpha, s.nbeta)
    E = gnof.computeE_elec_HC(H, C, n, elag, s)
    return E, elag


def energy(H, b, s: gnof.Sizes, C, gamma, method="ADAM", alpha=0.01, maxloop=10, threshgorb=4e-3,
           threshgocc=1e-3, threshen=1e-4, maxit=200):
    n, _ = gnof.ocupacion(gamma, s)
    cj12, ck12 = gnof.PNOFi_selector(n, s)
    E = 9999.0
    for it in range(1, maxit + 1):
        E, C, nit, ok, alpha, maxloop = orbital.orbopt(method, n, cj12, ck12, C, H, b, s, alpha, maxloop,
                                                       threshgorb)
        _, gamma, n, cj12, ck12, maxloop = occoptr(gamma, C, H, b, s, threshen, maxloop)
        if s.occ_method == "Softmax":
            C, gamma = gnof.order_occupations_softmax(C, gamma, s)
        n, _ = gnof.ocupacion(gamma, s)
        cj12, ck12 = gnof.PNOFi_selector(n, s)
        g_orb = orbital.calcorbg(None, n, cj12, ck12, C, H, b, s)
        J, K, Hc = native.jkh_mo(C, H, b, s.nbf5)
        g_occ = gnof.calcoccg(gamma, J, K, Hc, s)
        if np.max(np.abs(g_orb)) < threshgorb and np.linalg.norm(g_occ) < threshgocc:
            return E, C, gamma, it, True
    return E, C, gamma, maxit, False
