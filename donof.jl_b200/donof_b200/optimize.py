"""Occupation optimiser and the GNOF energy outer loop, driving the device
hot path.

  occoptr            src/minimization.jl:100-139  (Optim.jl ConjugateGradient on gamma)
  ENERGY1r           src/utils.jl:117-136
  order_subspaces    src/guess.jl:58-106
  energy             src/energy.jl:140-231 (the iteration part of DoNOF.energy)

Optim.jl is not available here, so the conjugate-gradient minimiser is our own:
Hager-Zhang directions (Hager & Zhang, SIAM J. Optim. 16 (2005) 170-192,
eta = 0.4 as in Optim.jl's default) with a strong-Wolfe line search
(Nocedal & Wright, Numerical Optimization, Alg. 3.5/3.6), stopped on
max|grad| <= g_abstol like Optim.Options(g_abstol = p.threshen).  Its
trajectory therefore differs from Optim.jl's; converged results agree.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Callable, Optional

import numpy as np

from . import api, gnof
from .param import Param


# ---------------------------------------------------------------- CG minimiser
def _decrease_ok(fa, da, a, f0, d0, c1):
    """Armijo sufficient decrease, or Hager-Zhang's approximate Wolfe test
    (phi(a) <= phi(0) + eps |phi(0)| and phi'(a) <= (2 delta - 1) phi'(0)),
    which stays decidable when the decrease is below the rounding of f."""
    if fa <= f0 + c1 * a * d0:
        return True
    return fa <= f0 + 1e-6 * abs(f0) and da <= (2 * 0.1 - 1.0) * d0


def _zoom(phi, dphi, a_lo, a_hi, f_lo, d_lo, f0, d0, c1, c2, max_it=30):
    f_hi = phi(a_hi)[0]
    for _ in range(max_it):
        # safeguarded cubic-free interpolation: bisection with a quadratic guess
        denom = 2.0 * (f_hi - f_lo - d_lo * (a_hi - a_lo))
        a = a_lo - d_lo * (a_hi - a_lo) ** 2 / denom if denom > 0 else 0.5 * (a_lo + a_hi)
        lo, hi = min(a_lo, a_hi), max(a_lo, a_hi)
        if not (lo + 0.1 * (hi - lo) <= a <= hi - 0.1 * (hi - lo)):
            a = 0.5 * (a_lo + a_hi)
        fa, ga, da = phi(a)
        if not _decrease_ok(fa, da, a, f0, d0, c1) or fa > f_lo + 1e-6 * abs(f0):
            a_hi, f_hi = a, fa
        else:
            if abs(da) <= -c2 * d0:
                return a, fa, ga
            if da * (a_hi - a_lo) >= 0:
                a_hi, f_hi = a_lo, f_lo
            a_lo, f_lo, d_lo = a, fa, da
    fa, ga, _ = phi(a_lo)
    return a_lo, fa, ga


def _wolfe(f, g, x, d, fx, gx, a1, c1=1e-4, c2=0.1, a_max=1e6, max_it=30):
    cache = {}

    def phi(a):
        if a not in cache:
            xa = x + a * d
            fa = f(xa)
            ga = g(xa)
            cache[a] = (fa, ga, float(ga @ d))
        return cache[a]

    d0 = float(gx @ d)
    a_prev, f_prev, dp_prev = 0.0, fx, d0
    a = a1
    for i in range(max_it):
        fa, ga, da = phi(a)
        if not _decrease_ok(fa, da, a, fx, d0, c1) or (i > 0 and fa > f_prev + 1e-6 * abs(fx)):
            return _zoom(phi, None, a_prev, a, f_prev, dp_prev, fx, d0, c1, c2)
        if abs(da) <= -c2 * d0:
            return a, fa, ga
        if da >= 0:
            return _zoom(phi, None, a, a_prev, fa, da, fx, d0, c1, c2)
        a_prev, f_prev, dp_prev = a, fa, da
        a = min(2.0 * a, a_max)
    return a, fa, ga


@dataclass
class CGResult:
    minimizer: np.ndarray
    minimum: float
    iterations: int
    g_converged: bool


def cg_minimize(f: Callable, g: Callable, x0: np.ndarray, g_abstol: float, max_iter: int = 1000,
                eta: float = 0.4) -> CGResult:
    """Hager-Zhang nonlinear conjugate gradient with a strong-Wolfe line search."""
    x = np.array(x0, dtype=np.float64)
    fx = float(f(x))
    gx = np.asarray(g(x), dtype=np.float64)
    if np.max(np.abs(gx), initial=0.0) <= g_abstol:
        return CGResult(x, fx, 0, True)
    d = -gx
    a = 1.0 / max(np.max(np.abs(gx)), 1e-12)
    gd_prev = None
    for k in range(1, max_iter + 1):
        gd = float(gx @ d)
        if gd >= 0:  # not a descent direction: restart
            d = -gx
            gd = float(gx @ d)
        if gd_prev is not None:
            a = min(max(a * gd_prev / gd, 1e-10), 1e6)
        a, fn, gn = _wolfe(f, g, x, d, fx, gx, a)
        s = a * d
        x = x + s
        y = gn - gx
        if np.max(np.abs(gn)) <= g_abstol:
            return CGResult(x, float(fn), k, True)
        if abs(fn - fx) <= 0.0 and np.max(np.abs(s)) == 0.0:
            return CGResult(x, float(fn), k, False)
        dy = float(d @ y)
        if dy != 0.0:
            beta = float((y - 2.0 * d * (y @ y) / dy) @ gn) / dy
            eta_k = -1.0 / (np.linalg.norm(d) * min(eta, np.linalg.norm(gx)))
            beta = max(beta, eta_k)
        else:
            beta = 0.0
        gd_prev = gd
        d = -gn + beta * d
        fx, gx = float(fn), gn
    return CGResult(x, fx, max_iter, False)


# ---------------------------------------------------------------- occupation optimiser
def occoptr(gamma, C, H, b: api.BTensor, p: Param, freeze_occ: bool = False):
    """src/minimization.jl:100-139.  J_MO, K_MO, H_core come from the device once;
    the CG over gamma runs in the library's native host code (donof_occ_cg, the
    same minimiser as cg_minimize).  Returns (E, nit, success, gamma, n, cj12,
    ck12) and updates p.maxloop like the reference."""
    gamma = np.array(gamma, dtype=np.float64)
    E, nit, ok = -1.0, 0, True
    if p.ndoc > 0 and not freeze_occ:
        J, K, Hc = api.computeJKH_MO(C, H, b, p)
        gamma, E, nit, ok = api.occ_cg(gamma, J, K, Hc, p, p.threshen)
        if nit < 1:
            p.maxloop = p.maxloop + 10
    n, _ = gnof.occupations(gamma, p)
    cj12, ck12 = gnof.coupling(n, p)
    return E, nit, ok, gamma, n, cj12, ck12


# ---------------------------------------------------------------- energy pieces
def lagrange_convergency(elag):
    d = np.abs(elag - elag.T)
    return float(d.sum()), float(d.max())


def ENERGY1r(C, n, H, b: api.BTensor, cj12, ck12, p: Param):
    """src/utils.jl:117-136 (no1 = 0 branch): E via computeE_elec(H, C, n, elag)."""
    elag, Hmat = api.compute_Lagrange2(C, n, H, b, cj12, ck12, p.nalpha, p.nbeta)
    hdiag = np.einsum("mi,mn,ni->i", C, H, C)
    E = float(np.trace(elag[:p.nbf5, :p.nbf5]))
    E += float(np.sum(n[:p.nbeta] * hdiag[:p.nbeta]))
    if not p.HighSpin:
        E += float(np.sum(n[p.nbeta:p.nalpha] * hdiag[p.nbeta:p.nalpha]))
    else:
        E += float(np.sum(0.5 * hdiag[p.nbeta:p.nalpha]))
    E += float(np.sum(n[p.nalpha:p.nbf5] * hdiag[p.nalpha:p.nbf5]))
    sumdiff, maxdiff = lagrange_convergency(elag)
    return E, elag, sumdiff, maxdiff


def order_subspaces(old_C, old_n, elag, H, b: api.BTensor, p: Param):
    """Sort the strong orbitals (with their coupled weak ones) by elag diagonal
    (src/guess.jl:58-106)."""
    C = np.zeros((p.nbf, p.nbf), order="F")
    n = np.zeros(p.nbf5)
    ed = np.diag(elag)
    srt = np.argsort(ed[:p.no1], kind="stable")
    for i in range(p.no1):
        C[:, i] = old_C[:, srt[i]]
    srt = np.argsort(ed[p.no1:p.nbeta], kind="stable")
    C[:, :p.no1] = old_C[:, :p.no1]
    n[:p.no1] = old_n[:p.no1]
    P = p.pair_table()
    for i in range(p.ndoc):
        io = srt[i]
        C[:, p.no1 + i] = old_C[:, p.no1 + io]
        C[:, P[i]] = old_C[:, P[io]]
        n[p.no1 + i] = old_n[p.no1 + io]
        n[P[i]] = old_n[P[io]]
    srt = np.argsort(ed[p.no1 + p.ndoc:p.no1 + p.ndns], kind="stable")
    for i in range(p.nsoc):
        C[:, p.no1 + p.ndoc + i] = old_C[:, p.no1 + p.ndoc + srt[i]]
        n[p.no1 + p.ndoc + i] = old_n[p.no1 + p.ndoc + srt[i]]
    C[:, p.nbf5:] = old_C[:, p.nbf5:]
    cj12, ck12 = gnof.coupling(n, p)
    _, elag, _, _ = ENERGY1r(C, n, H, b, cj12, ck12, p)
    return C, n, elag


@dataclass
class EnergyResult:
    E_elec: float
    E_tot: float
    C: np.ndarray
    n: np.ndarray
    gamma: np.ndarray
    elag: np.ndarray
    iterations: int
    converged: bool
    tot_it_orb: int
    tot_it_occ: int
    history: list = field(default_factory=list)


def energy(H, b: api.BTensor, p: Param, C, gamma=None, E_nuc: float = 0.0, freeze_occ: bool = False,
           maxit: Optional[int] = None, log: Optional[Callable[[dict], None]] = None,
           order: bool = True, native: bool = True, stop_rel_de: float = 0.0) -> EnergyResult:
    """The orbital / occupation alternation of DoNOF.energy (src/energy.jl:140-224)
    for given core Hamiltonian H, device RI tensor b and starting orbitals C
    (the integral and guess set-up of energy.jl:29-105 is outside this path).
    The orbital optimiser runs device resident in the precision of b.

    native=True runs the whole alternation in the library (donof_energy), with
    no interpreter work per iteration; native=False runs the same steps from
    Python, one library call each (the two agree to rounding)."""
    H = np.asfortranarray(H, dtype=np.float64)
    C = np.array(C, dtype=np.float64, order="F")
    gamma = gnof.guess_gamma(p) if gamma is None else np.array(gamma, dtype=np.float64)
    if native:
        C, gamma, n, elag, r, hist = api.energy_loop(H, b, p, C, gamma, maxit=maxit, freeze_occ=freeze_occ,
                                                     order=order, stop_rel_de=stop_rel_de)
        rows = [dict(it=i + 1, nit_orb=int(h[4]), nit_occ=int(h[5]), E=h[0], E_tot=h[0] + E_nuc, E_diff=h[1],
                     max_grad_orb=h[2], norm_grad_occ=h[3]) for i, h in enumerate(hist)]
        if log:
            for row in rows:
                log(row)
        return EnergyResult(r["E_elec"], r["E_elec"] + E_nuc, C, n, gamma, elag, r["iterations"],
                            bool(r["converged"]), r["tot_it_orb"], r["tot_it_occ"], rows)
    n, _ = gnof.occupations(gamma, p)
    cj12, ck12 = gnof.coupling(n, p)
    E_old = 9999.0
    tot_orb = tot_occ = 0
    hist = []
    converged = False
    elag = np.zeros((p.nbf, p.nbf))
    E = E_old
    it = 0
    for it in range(1, (maxit or p.maxit) + 1):
        E_orb, C, nit_orb, _ = api.orbopt(gamma, C, H, b, p)
        E_occ, nit_occ, _, gamma, n, cj12, ck12 = occoptr(gamma, C, H, b, p, freeze_occ)
        if p.occ_method == "Softmax":
            C, gamma = gnof.order_occupations_softmax(C, gamma, p)
        tot_orb += nit_orb
        tot_occ += nit_occ
        E = E_orb
        E_diff = E - E_old
        E_old = E
        _, elag, sumdiff, maxdiff = ENERGY1r(C, n, H, b, cj12, ck12, p)
        n, _ = gnof.occupations(gamma, p)
        cj12, ck12 = gnof.coupling(n, p)
        grad_orb = api.calcorbg(None, n, cj12, ck12, C, H, b, p)
        J, K, Hc = api.computeJKH_MO(C, H, b, p)
        _, grad_occ = api.occ_energy(gamma, J, K, Hc, p)
        row = dict(it=it, nit_orb=nit_orb, nit_occ=nit_occ, E=E, E_tot=E + E_nuc, E_diff=E_diff, maxdiff=maxdiff,
                   max_grad_orb=float(np.max(np.abs(grad_orb))), norm_grad_occ=float(np.linalg.norm(grad_occ)))
        hist.append(row)
        if log:
            log(row)
        if row["max_grad_orb"] < p.threshgorb and row["norm_grad_occ"] < p.threshgocc:
            converged = True
            break
    if order and p.ipnof > 4:
        C, n, elag = order_subspaces(C, n, elag, H, b, p)
    return EnergyResult(E, E + E_nuc, C, n, gamma, elag, it, converged, tot_orb, tot_occ, hist)


def energy_mixed_refined(H, b: api.BTensor, p: Param, C, gamma=None, E_nuc: float = 0.0,
                         maxit: Optional[int] = None, log: Optional[Callable[[dict], None]] = None,
                         mixed_factor: float = 10.0, native: bool = True, mixed_noise: float = 1e-6):
    """The mixed-precision form until its gradients are below mixed_factor times
    the thresholds, or until an outer iteration changes E by no more than
    mixed_noise |E| (the bf16-split energies and gradients carry ~1e-5 relative
    rounding; past that point they would steer the optimiser by their rounding),
    then closing FP64 iterations from its orbitals and occupations until the
    FP64 gradients meet p's thresholds.  Returns (refined result, mixed-phase
    result); b must have been uploaded with precision "mixed" and is left in
    FP64 mode.  The early stop needs the native loop (native=True)."""
    import copy
    pm = copy.copy(p)
    pm.threshgorb = p.threshgorb * mixed_factor
    pm.threshgocc = p.threshgocc * mixed_factor
    b.set_precision("mixed")
    r_mixed = energy(H, b, pm, C, gamma, E_nuc=E_nuc, maxit=maxit, log=log, order=False, native=native,
                     stop_rel_de=mixed_noise if native else 0.0)
    p.maxloop = pm.maxloop
    b.set_precision("fp64")
    r = energy(H, b, p, r_mixed.C, r_mixed.gamma, E_nuc=E_nuc, maxit=maxit, log=log, native=native)
    return r, r_mixed
