"""CPU checks of the oracle itself.

The reference ships no tests or golden vectors and Julia is not available, so
parity with the reference is unpinned: the oracle is checked by (1) a second,
literal einsum restatement of the reference formulas, (2) the identities the
reference code implies (calce == computeE_elec at the same C, finite-
difference orbital and occupation gradients, orthogonality of the rotation,
occupation sum rules), and (3) the committed oracle fixtures (written by the
oracle itself, tests/golden/make_oracle_fixtures.py: they freeze its answers,
they do not come from the reference).
"""
import numpy as np
import pytest
import scipy.linalg

from oracle import gnof, native, orbital


def make_case(nbf=13, naux=29, nbeta=3, ncwo=3, nalpha=None, seed=0, sym=True, ista=0, occ="Softmax"):
    rng = np.random.default_rng(seed)
    nalpha = nbeta if nalpha is None else nalpha
    p = gnof.Sizes(nbf=nbf, nbeta=nbeta, nalpha=nalpha, ncwo=ncwo, naux=naux, ista=ista, occ_method=occ)
    b = rng.standard_normal((nbf, nbf, naux)) / np.sqrt(naux)
    if sym:
        b = 0.5 * (b + b.transpose(1, 0, 2))
    b = np.asfortranarray(b)
    C = np.asfortranarray(np.linalg.qr(rng.standard_normal((nbf, nbf)))[0])
    A = rng.standard_normal((nbf, nbf))
    H = np.asfortranarray(0.5 * (A + A.T) / np.sqrt(nbf))
    if occ == "Softmax":
        gamma = rng.standard_normal(p.nv)
    else:
        gamma = gnof.guess_gamma_trigonometric(p.ndoc, p.ncwo) + 0.3 * rng.standard_normal(p.nv)
    n, dn = gnof.ocupacion(gamma, p)
    cj, ck = gnof.PNOFi_selector(n, p)
    return p, b, C, H, gamma, n, dn, cj, ck


def lagrange_einsum(C, n, H, b, cj12, ck12, nalpha, nbeta):
    """Literal restatement of src/utils.jl:1-59 with einsum."""
    nbf5 = n.shape[0]
    C5 = C[:, :nbf5]
    Hmat = C.T @ (H @ C5)
    tmp = np.einsum("nq,mnl->mql", C5, b)
    bmo = np.einsum("mp,mql->pql", C, tmp)
    elag = np.zeros((C.shape[0], C.shape[0]))
    elag[:, :nbf5] += n[None, :] * Hmat
    if nbeta > 0:
        for rng_ in (np.arange(nbeta), np.arange(nalpha, nbf5)):
            d = bmo[rng_, rng_, :]  # (|rng|, naux)
            elag[:, rng_] += n[rng_][None, :] * np.einsum("abk,bk->ab", bmo[:, rng_, :], d)
    dq = np.einsum("qqk->qk", bmo[:nbf5, :nbf5, :])
    t = cj12 @ dq
    elag[:, :nbf5] += np.einsum("abk,bk->ab", bmo[:, :nbf5, :], t)
    elag[:, :nbf5] -= np.einsum("bq,aqk,bqk->ab", ck12, bmo[:, :nbf5, :], bmo[:nbf5, :nbf5, :])
    return elag, Hmat


def jkh_einsum(C, H, b, nbf5):
    C5 = C[:, :nbf5]
    bpnl = np.einsum("mp,mnl->pnl", C5, b)
    bpql = np.einsum("nq,pnl->pql", C5, bpnl)
    d = np.einsum("ppl->pl", bpql)
    J = d @ d.T
    K = np.einsum("pql,pql->pq", bpql, bpql)
    Hc = np.einsum("mi,mn,ni->i", C5, H, C5)
    return J, K, Hc


def rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("kw", [dict(), dict(sym=False), dict(nbf=24, naux=40, nbeta=5, ncwo=3),
                                dict(nbf=20, naux=17, nbeta=3, nalpha=5, ncwo=3),
                                dict(nbf=16, naux=8, nbeta=0, nalpha=2, ncwo=0)])
def test_lagrange_c_oracle_matches_einsum(kw):
    p, b, C, H, gamma, n, dn, cj, ck = make_case(**kw) if kw.get("nbeta", 3) > 0 else (None,) * 9
    if p is None:
        pytest.skip("ndoc = 0 has no GNOF pairs")
    e1, h1 = native.lagrange2(C, n, H, b, cj, ck, p.nalpha, p.nbeta)
    e2, h2 = lagrange_einsum(C, n, H, b, cj, ck, p.nalpha, p.nbeta)
    assert rel(h1, h2) < 1e-13
    assert rel(e1, e2) < 1e-12
    assert np.all(e1[:, p.nbf5:] == 0.0)


@pytest.mark.parametrize("kw", [dict(), dict(sym=False), dict(nbf=24, naux=40, nbeta=5, ncwo=3)])
def test_jkh_c_oracle_matches_einsum(kw):
    p, b, C, H, *_ = make_case(**kw)
    J1, K1, h1 = native.jkh_mo(C, H, b, p.nbf5)
    J2, K2, h2 = jkh_einsum(C, H, b, p.nbf5)
    assert rel(J1, J2) < 1e-12 and rel(K1, K2) < 1e-12 and rel(h1, h2) < 1e-12


@pytest.mark.parametrize("kw", [dict(), dict(nbf=24, naux=40, nbeta=5, ncwo=3),
                                dict(nbf=20, naux=17, nbeta=3, nalpha=5, ncwo=3)])
def test_calce_equals_e_elec(kw):
    """sum_b elag_bb + n_b H_bb == calce(JKH_MO) at the same C (pnof.jl:1273 vs utils.jl:216)."""
    p, b, C, H, gamma, n, dn, cj, ck = make_case(**kw)
    elag, Hmat = native.lagrange2(C, n, H, b, cj, ck, p.nalpha, p.nbeta)
    J, K, Hc = native.jkh_mo(C, H, b, p.nbf5)
    E1 = gnof.computeE_elec_Hmat(Hmat, n, elag, p)
    E2 = gnof.calce(n, cj, ck, J, K, Hc, p)
    assert abs(E1 - E2) < 1e-11 * max(1.0, abs(E2))
    E3 = gnof.computeE_elec_HC(H, C, n, elag, p)
    assert abs(E3 - E1) < 1e-11 * max(1.0, abs(E1))


def test_orbital_gradient_is_derivative_of_energy():
    """calcorbg(y=0) equals the central finite difference of calce(rotate_orbital(y))."""
    p, b, C, H, gamma, n, dn, cj, ck = make_case(nbf=12, naux=20, nbeta=2, ncwo=3, seed=3)
    g = orbital.calcorbg(None, n, cj, ck, C, H, b, p)
    h = 1e-5
    rng = np.random.default_rng(1)
    for k in rng.choice(p.nvar, size=12, replace=False):
        y = np.zeros(p.nvar)
        y[k] = h
        Ep = gnof.calce(n, cj, ck, *native.jkh_mo(native.rotate(y, C, p.nbf5), H, b, p.nbf5), p)
        y[k] = -h
        Em = gnof.calce(n, cj, ck, *native.jkh_mo(native.rotate(y, C, p.nbf5), H, b, p.nbf5), p)
        fd = (Ep - Em) / (2 * h)
        assert abs(fd - g[k]) < 1e-6 * max(1.0, abs(g[k])), (k, fd, g[k])


@pytest.mark.parametrize("occ,ista,nalpha", [("Softmax", 0, None), ("Softmax", 1, None), ("Softmax", 2, None),
                                             ("Softmax", 3, None), ("Softmax", 4, None), ("Softmax", 5, None),
                                             ("Trigonometric", 0, None), ("Softmax", 0, 5),
                                             ("Trigonometric", 0, 5)])
def test_occupation_gradient_is_derivative_of_energy(occ, ista, nalpha):
    p, b, C, H, gamma, n, dn, cj, ck = make_case(nbf=20, naux=15, nbeta=3, nalpha=nalpha, ncwo=3, seed=5,
                                                 ista=ista, occ=occ)
    J, K, Hc = native.jkh_mo(C, H, b, p.nbf5)
    g = gnof.calcoccg(gamma, J, K, Hc, p)
    h = 1e-6
    for k in range(p.nv):
        e = np.zeros(p.nv)
        e[k] = h
        fd = (gnof.calcocce(gamma + e, J, K, Hc, p) - gnof.calcocce(gamma - e, J, K, Hc, p)) / (2 * h)
        assert abs(fd - g[k]) < 2e-6 * max(1.0, abs(g[k])), (k, fd, g[k])


@pytest.mark.parametrize("occ", ["Softmax", "Trigonometric"])
def test_occupation_sum_rules(occ):
    p, *_ , gamma, n, dn, cj, ck = make_case(nbf=30, naux=5, nbeta=4, ncwo=4, seed=2, occ=occ)
    for i in range(1, p.ndoc + 1):
        ll = p.no1 + p.ndns + (p.ndoc - i)
        idx = ll + p.ndoc * np.arange(p.ncwo)
        assert abs(n[p.no1 + i - 1] + n[idx].sum() - 1.0) < 1e-14
    assert np.all((n > 0) & (n < 1))
    assert abs(2 * n.sum() - 2 * p.ndoc) < 1e-12
    # dn/dgamma by finite differences
    h = 1e-7
    for k in range(p.nv):
        e = np.zeros(p.nv)
        e[k] = h
        fd = (gnof.ocupacion(gamma + e, p)[0] - gnof.ocupacion(gamma - e, p)[0]) / (2 * h)
        if occ == "Softmax":
            # the reference multiplies by n[i] (pnof.jl:1152); with no1 = 0 that is exact
            assert np.max(np.abs(fd - dn[:, k])) < 1e-7
        else:
            assert np.max(np.abs(fd - dn[:, k])) < 1e-7


def test_expm_matches_scipy_and_rotation_is_orthogonal():
    rng = np.random.default_rng(4)
    for scale in (1e-3, 0.3, 4.0, 40.0):
        A = rng.standard_normal((17, 17)) * scale
        assert rel(native.expm(A), scipy.linalg.expm(A)) < 1e-12
    p, b, C, H, *_ = make_case(nbf=15, naux=3, nbeta=2, ncwo=3)
    y = 0.05 * rng.standard_normal(p.nvar)
    Cn = native.rotate(y, C, p.nbf5)
    assert np.max(np.abs(Cn.T @ Cn - np.eye(p.nbf))) < 1e-13


def test_b_symmetrisation_invariance():
    """For symmetric b the Lagrangian is unchanged by b -> b^T(mn) (survey identity 6)."""
    p, b, C, H, gamma, n, dn, cj, ck = make_case()
    e1, _ = native.lagrange2(C, n, H, b, cj, ck, p.nalpha, p.nbeta)
    e2, _ = native.lagrange2(C, n, H, np.asfortranarray(b.transpose(1, 0, 2)), cj, ck, p.nalpha, p.nbeta)
    assert rel(e1, e2) < 1e-13


@pytest.mark.parametrize("sym,nalpha_extra", [(True, 0), (False, 0), (True, 2)])
def test_blas_mirror_matches_the_c_oracle(sym, nalpha_extra):
    """The BLAS mirror (the CPU baseline) computes what the C oracle computes."""
    from oracle import blas_mirror
    p, b, C, H, gamma, n, dn, cj, ck = make_case(nbf=21, naux=33, nbeta=3, ncwo=3, nalpha=3 + nalpha_extra,
                                                 seed=4, sym=sym)
    e1, h1 = native.lagrange2(C, n, H, b, cj, ck, p.nalpha, p.nbeta)
    e2, h2 = blas_mirror.lagrange2(C, n, H, b, cj, ck, p.nalpha, p.nbeta)
    assert np.max(np.abs(e1 - e2)) <= 1e-12 * np.max(np.abs(e1))
    assert np.max(np.abs(h1 - h2)) <= 1e-12 * np.max(np.abs(h1))
    nbf5 = n.shape[0]
    for x1, x2 in zip(native.jkh_mo(C, H, b, nbf5), blas_mirror.jkh_mo(C, H, b, nbf5)):
        assert np.max(np.abs(x1 - x2)) <= 1e-12 * max(1.0, np.max(np.abs(x1)))
    y = np.random.default_rng(3).standard_normal(nbf5 * p.nbf - nbf5 * (nbf5 + 1) // 2) * 0.1
    assert np.max(np.abs(native.rotate(y, C, nbf5) - blas_mirror.rotate(y, C, nbf5))) <= 1e-12
