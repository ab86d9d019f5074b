"""The library's native occupation layer (donof_occ_energy, donof_occ_cg)
against the oracle's line-by-line restatement (der_CJCKD8 materialised):
energy and gamma-gradient for every GNOF variant (ista 0-5), both occupation
maps, closed and open shells and a core-orbital case; the conjugate-gradient
minimisation reaches the minimum the numpy minimiser finds on the oracle's
functions.  Host code only (no GPU)."""
import numpy as np
import pytest

from oracle import gnof as ognof
from donof_b200 import _lib, api, gnof
from donof_b200.optimize import cg_minimize
from donof_b200.param import Param


def sizes_of(p: Param):
    return ognof.Sizes(nbf=p.nbf, nbeta=p.nbeta, nalpha=p.nalpha, ncwo=p.ncwo, naux=p.nbfaux, no1=p.no1,
                       ista=p.ista, HighSpin=p.HighSpin, h_cut=p.h_cut, occ_method=p.occ_method)

CASES = [dict(nbf=40, nbfaux=9, nbeta=4, nalpha=4, ncwo=3),
         dict(nbf=40, nbfaux=9, nbeta=4, nalpha=6, ncwo=3),
         dict(nbf=60, nbfaux=9, nbeta=5, nalpha=7, ncwo=4),
         dict(nbf=24, nbfaux=9, nbeta=5, nalpha=5, ncwo=-1),
         dict(nbf=50, nbfaux=9, nbeta=6, nalpha=6, ncwo=3, no1=2)]


def _jk(p, seed):
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((p.nbf5, p.nbf5))
    J = np.asfortranarray(np.abs(A @ A.T) / p.nbf5 + 0.01 * rng.standard_normal((p.nbf5, p.nbf5)))
    K = np.asfortranarray(0.3 * J + 0.01 * rng.standard_normal((p.nbf5, p.nbf5)))
    Hc = -np.sort(rng.uniform(0.5, 3.0, p.nbf5))[::-1]
    return J, K, Hc


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("ista", [0, 1, 2, 3, 4, 5])
@pytest.mark.parametrize("occ", ["Softmax", "Trigonometric"])
def test_energy_and_gradient_match_the_oracle(case, ista, occ):
    p = Param(ista=ista, occ_method=occ, **case)
    s = sizes_of(p)
    J, K, Hc = _jk(p, ista + 7 * len(occ))
    rng = np.random.default_rng(ista)
    for _ in range(3):
        gamma = rng.standard_normal(p.nv)
        E, g = api.occ_energy(gamma, J, K, Hc, p)
        E0 = ognof.calcocce(gamma, J, K, Hc, s)
        g0 = ognof.calcoccg(gamma, J, K, Hc, s)
        assert abs(E - E0) <= 1e-12 * max(1.0, abs(E0))
        assert np.max(np.abs(g - g0)) <= 1e-12 * max(1.0, np.max(np.abs(g0)))
        E1, none = api.occ_energy(gamma, J, K, Hc, p, grad=False)
        assert E1 == E and none is None


@pytest.mark.parametrize("occ", ["Softmax", "Trigonometric"])
@pytest.mark.parametrize("case", CASES[:3])
def test_cg_reaches_the_oracle_minimum(case, occ):
    p = Param(occ_method=occ, **case)
    s = sizes_of(p)
    J, K, Hc = _jk(p, 3)
    g0 = gnof.guess_gamma(p)
    x, E, nit, ok = api.occ_cg(g0, J, K, Hc, p, 1e-9, 1000)
    r = cg_minimize(lambda t: ognof.calcocce(t, J, K, Hc, s), lambda t: ognof.calcoccg(t, J, K, Hc, s), g0, 1e-9,
                    1000)
    assert ok and nit > 0
    _, g = api.occ_energy(x, J, K, Hc, p)
    assert np.max(np.abs(g)) <= 1e-9
    if r.g_converged:
        assert abs(E - r.minimum) <= 1e-10 * max(1.0, abs(r.minimum))
        n, _ = ognof.ocupacion(x, s)
        n0, _ = ognof.ocupacion(r.minimizer, s)
        assert np.max(np.abs(n - n0)) <= 1e-6
    else:  # random J/K can leave the Python minimiser short of the test; ours must not be worse
        assert E <= r.minimum + 1e-9 * max(1.0, abs(r.minimum))


def test_converged_start_returns_at_once_and_bad_sizes_raise():
    p = Param(nbf=40, nbfaux=9, nbeta=4, nalpha=4, ncwo=3)
    J, K, Hc = _jk(p, 1)
    x, E, nit, ok = api.occ_cg(gnof.guess_gamma(p), J, K, Hc, p, 1e3, 10)
    assert nit == 0 and ok
    bad = Param(nbf=40, nbfaux=9, nbeta=4, nalpha=4, ncwo=3)
    bad.ista = 7
    with pytest.raises(_lib.DonofError) as e:
        api.occ_energy(np.zeros(p.nv), J, K, Hc, bad)
    assert e.value.status == _lib.ERR_ARG
