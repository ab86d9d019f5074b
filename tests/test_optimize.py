"""CPU tests of the host-side optimisers: the Hager-Zhang CG minimiser that
stands in for Optim.jl's ConjugateGradient, and the occupation minimisation it
performs inside occoptr (src/minimization.jl:100-139), against SciPy's CG."""
import numpy as np
import scipy.optimize

from donof_b200 import Param, gnof
from donof_b200.optimize import cg_minimize
from oracle import gnof as ognof
from oracle import native


def test_cg_quadratic_and_rosenbrock():
    rng = np.random.default_rng(0)
    Q = rng.standard_normal((12, 12))
    A = Q @ Q.T + 12 * np.eye(12)
    bvec = rng.standard_normal(12)
    r = cg_minimize(lambda x: 0.5 * x @ A @ x - bvec @ x, lambda x: A @ x - bvec, np.zeros(12), 1e-8)
    assert r.g_converged and np.max(np.abs(r.minimizer - np.linalg.solve(A, bvec))) < 1e-9

    def f(x):
        return (1 - x[0]) ** 2 + 100 * (x[1] - x[0] ** 2) ** 2

    def g(x):
        return np.array([-2 * (1 - x[0]) - 400 * x[0] * (x[1] - x[0] ** 2), 200 * (x[1] - x[0] ** 2)])

    r = cg_minimize(f, g, np.array([-1.2, 1.0]), 1e-8, max_iter=5000)
    assert r.g_converged and np.max(np.abs(r.minimizer - 1.0)) < 1e-6


def test_cg_already_converged_reports_zero_iterations():
    r = cg_minimize(lambda x: float(x @ x), lambda x: 2 * x, np.zeros(3), 1e-4)
    assert r.iterations == 0 and r.g_converged


def test_occupation_minimum_matches_scipy():
    """Same objective (calcocce/calcoccg at J, K, H_core of a seeded case), two CG codes."""
    for occ in ("Softmax", "Trigonometric"):
        p = Param(nbf=30, nbfaux=40, nbeta=4, nalpha=4, ncwo=3, occ_method=occ)
        s = ognof.Sizes(nbf=30, nbeta=4, nalpha=4, ncwo=3, naux=40, occ_method=occ)
        rng = np.random.default_rng(3)
        b = rng.standard_normal((30, 30, 40)) / np.sqrt(40)
        b = np.asfortranarray(0.5 * (b + b.transpose(1, 0, 2)))
        C = np.asfortranarray(np.linalg.qr(rng.standard_normal((30, 30)))[0])
        A = rng.standard_normal((30, 30))
        H = np.asfortranarray(-np.abs(np.diag(np.arange(30.0))) + 0.05 * (A + A.T))
        J, K, Hc = native.jkh_mo(C, H, b, p.nbf5)
        g0 = gnof.guess_gamma(p)
        r = cg_minimize(lambda x: gnof.calcocce(x, J, K, Hc, p), lambda x: gnof.calcoccg(x, J, K, Hc, p), g0, 1e-9)
        ref = scipy.optimize.minimize(lambda x: ognof.calcocce(x, J, K, Hc, s), g0,
                                      jac=lambda x: ognof.calcoccg(x, J, K, Hc, s), method="CG",
                                      options={"gtol": 1e-9, "norm": np.inf, "maxiter": 5000})
        assert r.g_converged
        assert abs(r.minimum - ref.fun) < 1e-9 * max(1.0, abs(ref.fun))
