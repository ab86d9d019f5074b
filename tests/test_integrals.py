"""The integral front end (csrc/ints.cu through donof_b200.integrals), which
replaces GaussianBasis.jl/libcint in compute_integrals (src/integrals.jl:1-49).
No output of the reference or of libcint is available here, so the engine is
checked against published values (the H2 STO-3G integrals of Szabo and
Ostlund, "Modern Quantum Chemistry", section 3.5), closed forms for s
Gaussians, and derivative identities that build p and d integrals from s ones
independently of the Hermite recursions: a normalised p_x primitive is
a^{-1/2} d/dA_x of the normalised s primitive with the same exponent, and the
Cartesian d_xx and d_xy primitives are (d^2/dA_x^2 + 2a)/(a sqrt 3) and
d^2/dA_x dA_y / (a sqrt 3) of it."""
import math

import numpy as np
import pytest
from scipy.special import erf

from donof_b200 import integrals as it

H_STO3G = [(0, np.array([3.42525091, 0.62391373, 0.16885540]), np.array([0.15432897, 0.53532814, 0.44463454]))]
B2A = 1.0 / it.ANGSTROM_TO_BOHR


def atoms_bohr(spec):
    return [it.Atom(s, it.ELEMENTS.index(s) + 1, np.array(x, dtype=float) * B2A) for s, x in spec]


def basis(spec, shells, spherical=True):
    return it.BasisSet("test", atoms_bohr(spec), shells, spherical)


def test_h2_sto3g_matches_szabo_ostlund():
    b = basis([("H", (0, 0, 0)), ("H", (0, 0, 1.4))], {"H": H_STO3G})
    S, T, V = it.one_electron(b)
    assert np.allclose(S, [[1.0, 0.6593], [0.6593, 1.0]], atol=1e-4)
    assert np.allclose(T, [[0.7600, 0.2365], [0.2365, 0.7600]], atol=1e-4)
    assert np.allclose(V, [[-1.8804, -1.1948], [-1.1948, -1.8804]], atol=1e-4)
    I = it.ERI_2e4c(b)
    assert abs(I[0, 0, 0, 0] - 0.7746) < 1e-4
    assert abs(I[0, 0, 1, 1] - 0.5697) < 1e-4
    assert abs(I[1, 0, 0, 0] - 0.4441) < 1e-4
    assert abs(I[1, 0, 1, 0] - 0.2970) < 1e-4
    # eight-fold symmetry of the four-index array
    for perm in [(1, 0, 2, 3), (0, 1, 3, 2), (2, 3, 0, 1)]:
        assert np.array_equal(I, I.transpose(perm))


def test_s_closed_forms():
    """Normalised s primitives a at A and b at B: S = (4ab/p^2)^{3/4} exp(-mu R^2),
    T = mu (3 - 2 mu R^2) S, (a|b) = 2 pi^{5/2} / (ab sqrt(a+b)) N_a N_b F_0(mu R^2)."""
    a, b, R = 0.8, 1.7, 1.3
    bs = basis([("H", (0, 0, 0)), ("He", (0, 0, R))], {"H": [(0, np.array([a]), np.array([1.0]))],
                                                          "He": [(0, np.array([b]), np.array([1.0]))]})
    S, T, _ = it.one_electron(bs)
    p, mu = a + b, a * b / (a + b)
    s_ab = (4 * a * b / p ** 2) ** 0.75 * math.exp(-mu * R * R)
    assert abs(S[0, 1] - s_ab) < 1e-14
    assert abs(T[0, 1] - mu * (3 - 2 * mu * R * R) * s_ab) < 1e-13
    G = it.ERI_2e2c(bs)
    na, nb = (2 * a / math.pi) ** 0.75, (2 * b / math.pi) ** 0.75
    x = mu * R * R
    f0 = 0.5 * math.sqrt(math.pi / x) * erf(math.sqrt(x))
    assert abs(G[0, 1] - 2 * math.pi ** 2.5 / (a * b * math.sqrt(a + b)) * na * nb * f0) < 1e-13
    # the Boys function's large-argument branch (T > 35)
    far = basis([("H", (0, 0, 0)), ("He", (0, 0, 12.0))], {"H": [(0, np.array([a]), np.array([1.0]))],
                                                              "He": [(0, np.array([b]), np.array([1.0]))]})
    x = mu * 144.0
    assert x > 35
    f0 = 0.5 * math.sqrt(math.pi / x)
    assert abs(it.ERI_2e2c(far)[0, 1] - 2 * math.pi ** 2.5 / (a * b * math.sqrt(a + b)) * na * nb * f0) < 1e-14


MIXED = {"H": [(0, np.array([1.3, 0.4]), np.array([0.6, 0.5])), (1, np.array([0.8]), np.array([1.0]))],
         "C": [(0, np.array([7.0, 1.1, 0.3]), np.array([0.2, 0.5, 0.4])), (1, np.array([2.0, 0.5]), np.array([0.4, 0.7])),
               (2, np.array([0.9]), np.array([1.0])), (3, np.array([0.7]), np.array([1.0]))]}
GEOM = [("C", (0.1, -0.2, 0.3)), ("H", (1.2, 0.9, -0.4)), ("H", (-1.0, 0.4, 1.1))]


@pytest.mark.parametrize("spherical", [True, False])
def test_normalisation_symmetry_and_shell_orthogonality(spherical):
    b = basis(GEOM, MIXED, spherical)
    S, T, V = it.one_electron(b)
    for M in (S, T, V):
        assert np.allclose(M, M.T, atol=1e-14)
    if spherical:
        assert np.allclose(np.diag(S), 1.0, atol=1e-13)
        # the components of a spherical shell on one centre are orthonormal
        ao = 0
        for l in b.shell_l:
            n = 2 * l + 1
            assert np.allclose(S[ao:ao + n, ao:ao + n], np.eye(n), atol=1e-13), l
            ao += n
    else:
        # Cartesian components normalised like x^l: the axis components have unit norm
        ao = 0
        for l in b.shell_l:
            n = (l + 1) * (l + 2) // 2
            assert abs(S[ao, ao] - 1.0) < 1e-13 and abs(S[ao + n - 1, ao + n - 1] - 1.0) < 1e-13
            ao += n
    assert np.all(np.linalg.eigvalsh(S) > 0)
    aux = basis(GEOM, MIXED, spherical)
    G = it.ERI_2e2c(aux)
    assert np.allclose(G, G.T, atol=1e-14) and np.all(np.linalg.eigvalsh(G) > 0)
    I = it.ERI_2e3c(b, aux)
    assert np.allclose(I, I.transpose(1, 0, 2), atol=1e-14)


def test_translation_and_rotation_invariance():
    b0 = basis(GEOM, MIXED)
    shift = np.array([0.7, -1.9, 2.5])
    b1 = basis([(s, tuple(np.array(x) + shift)) for s, x in GEOM], MIXED)
    for f in (lambda b: it.one_electron(b), lambda b: (it.ERI_2e2c(b),), lambda b: (it.ERI_2e3c(b, b),)):
        for x, y in zip(f(b0), f(b1)):
            assert np.allclose(x, y, atol=1e-12)
    # a rotation mixes the components of each spherical shell: spectra are invariant
    th = 0.7
    Rz = np.array([[math.cos(th), -math.sin(th), 0], [math.sin(th), math.cos(th), 0], [0, 0, 1]])
    b2 = basis([(s, tuple(Rz @ np.array(x))) for s, x in GEOM], MIXED)
    for x, y in zip(it.one_electron(b0), it.one_electron(b2)):
        assert np.allclose(np.linalg.eigvalsh(x), np.linalg.eigvalsh(y), atol=1e-12)
    assert np.allclose(np.linalg.eigvalsh(it.ERI_2e2c(b0)), np.linalg.eigvalsh(it.ERI_2e2c(b2)), atol=1e-12)


def _fd_case(kind, l_probe, a, h=1e-3):
    """Integrals of the probe shell (one primitive, exponent a, at A) against a
    fixed second function, by the engine and by finite differences of the s
    integrals (Cartesian components)."""
    A = np.array([0.3, -0.4, 0.2])
    other = [("C", (1.1, 0.5, -0.7))]
    oth_sh = {"C": [(1, np.array([0.9]), np.array([1.0]))]}

    def engine(center, l):
        sh = {"He": [(l, np.array([a]), np.array([1.0]))], **oth_sh}
        b = basis([("He", tuple(center))] + other, sh, spherical=False)
        n = (l + 1) * (l + 2) // 2
        if kind == "V":  # the nuclei stay put (only the other atom's): the operator does not move with A
            return it.one_electron(b, nuclei=atoms_bohr(other))[2][:n, n:]
        if kind == "T":
            return it.one_electron(b)[1][:n, n:]
        if kind == "G":
            return it.ERI_2e2c(b)[:n, n:]
        aux = basis(other, {"C": [(2, np.array([1.4]), np.array([1.0]))]}, spherical=False)
        return it.ERI_2e3c(b, aux)[:n, n:, :].reshape(n, -1)

    got = engine(A, l_probe)

    def s_at(dx):
        return engine(A + dx, 0)[0]

    e = np.eye(3) * h
    if l_probe == 1:
        fd = np.array([(s_at(e[k]) - s_at(-e[k])) / (2 * h) for k in range(3)]) / math.sqrt(a)
        return got, fd
    # d: components xx, xy, xz, yy, yz, zz
    s0 = s_at(np.zeros(3))
    rows = []
    for (i, j) in [(0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2)]:
        if i == j:
            d2 = (s_at(e[i]) - 2 * s0 + s_at(-e[i])) / (h * h)
            rows.append((d2 + 2 * a * s0) / (a * math.sqrt(3)))
        else:
            d2 = (s_at(e[i] + e[j]) - s_at(e[i] - e[j]) - s_at(-e[i] + e[j]) + s_at(-e[i] - e[j])) / (4 * h * h)
            rows.append(d2 / (a * math.sqrt(3)))
    return got, np.array(rows)


@pytest.mark.parametrize("kind", ["T", "V", "G", "I3c"])
@pytest.mark.parametrize("l_probe", [1, 2])
def test_p_and_d_integrals_from_derivatives_of_s_integrals(kind, l_probe):
    # central differences: O(h^2) truncation, O(eps / h^k) rounding
    got, fd = _fd_case(kind, l_probe, 0.85, h=1e-4 if l_probe == 1 else 1e-3)
    tol = 1e-8 if l_probe == 1 else 1e-6
    assert np.max(np.abs(got - fd)) <= tol * max(1.0, np.max(np.abs(got))), (got, fd)


def test_basis_text_parser_and_molecule():
    text = """
! comment line
H     0
S   3   1.00
      3.42525091D+00         0.15432897D+00
      0.62391373             0.53532814
      0.16885540             0.44463454
****
O     0
S   1   1.00
      5.0             1.0
SP   2   1.00
      5.0331513              -0.09996723             0.15591627
      1.1695961               0.39951283             0.60768372
****
"""
    sh = it.parse_gbs(text)
    assert [s[0] for s in sh["O"]] == [0, 0, 1]
    assert np.allclose(sh["H"][0][1], [3.42525091, 0.62391373, 0.16885540])
    bset, p = it.molecule("0 1\nO 0 0 0\nH 0 0.757 0.587\nH 0 -0.757 0.587", text, spherical=True)
    assert bset.nbas == 1 + 1 + 3 + 2 and bset.natoms == 3
    assert (p.nalpha, p.nbeta, p.nbf) == (5, 5, 7)
    # compute_E_nuc with the reference's factor 1.88973 (src/utils.jl:299-312)
    r_oh = math.sqrt(0.757 ** 2 + 0.587 ** 2)
    e = 2 * 8 / (r_oh * 1.88973) + 1 / (1.514 * 1.88973)
    assert abs(it.compute_E_nuc(bset) - e) < 1e-12
    with pytest.raises(ValueError):
        it.molecule("Xx 0 0 0", text)


def test_ri_diagonal_is_a_lower_bound():
    """Coulomb-metric fitting: (mn|mn)_RI = sum (mn|P) G^-1_PQ (Q|mn) <= (mn|mn),
    and a richer auxiliary basis brings it closer."""
    b = basis([("H", (0, 0, 0)), ("H", (0, 0, 1.4))], {"H": H_STO3G})
    I4 = it.ERI_2e4c(b)
    prev = None
    for n_et in (3, 6):
        ex = 0.2 * 2.5 ** np.arange(n_et)
        aux_sh = {"H": [(0, np.array([x]), np.array([1.0])) for x in ex] + [(1, np.array([1.0]), np.array([1.0]))]}
        aux = basis([("H", (0, 0, 0)), ("H", (0, 0, 1.4))], aux_sh)
        G = it.ERI_2e2c(aux)
        I3 = it.ERI_2e3c(b, aux).reshape(4, -1)
        ri = I3 @ np.linalg.solve(G, I3.T)
        exact = I4.reshape(4, 4)
        err = np.max(np.abs(ri - exact))
        assert np.all(np.diag(ri) <= np.diag(exact) + 1e-12)
        if prev is not None:
            assert err < prev
        prev = err
    assert prev < 5e-3


def test_invalid_shells_are_refused():
    from donof_b200 import _lib

    good = {"H": H_STO3G}
    with pytest.raises(_lib.DonofError) as e:
        basis([("H", (0, 0, 0))], {"H": [(6, np.array([1.0]), np.array([1.0]))]})
    assert e.value.status == _lib.ERR_ARG
    with pytest.raises(_lib.DonofError):
        basis([("H", (0, 0, 0))], {"H": [(0, np.array([-1.0]), np.array([1.0]))]})
    with pytest.raises(ValueError):
        basis([("C", (0, 0, 0))], good)  # no shells for C
    with pytest.raises(ValueError):
        it.parse_gbs("H 0\nQ 1 1.0\n 1.0 1.0\n****")


def test_compute_integrals_without_ri_returns_the_four_index_array():
    bset, p = it.molecule(f"H 0 0 0\nH 0 0 {1.4 * B2A:.12f}", "H 0\nS 3 1.00\n 3.42525091 0.15432897\n"
                          " 0.62391373 0.53532814\n 0.16885540 0.44463454\n****", spherical=True)
    p.RI = False
    S, T, V, H, I = it.compute_integrals(bset, None, p)
    assert np.allclose(H, T + V) and I.shape == (2, 2, 2, 2)
    assert abs(I[0, 0, 0, 0] - 0.7746) < 1e-4


@pytest.mark.parametrize("spherical_orb", [True, False])
def test_ri_is_exact_when_the_auxiliary_basis_spans_every_product(spherical_orb):
    """On one centre, s(a) s(a) = s(2a), s(a) p(b) = p(a+b) and p(b) p(b) lies in
    the six Cartesian d(2b) functions, so with those as the auxiliary basis the
    RI factorisation sum (mn|P) G^-1_PQ (Q|ls) reproduces (mn|ls) exactly: a
    consistency check of the two-, three- and four-centre integrals together."""
    a, b = 0.9, 0.6
    orb = basis([("He", (0.2, -0.1, 0.3))], {"He": [(0, np.array([a]), np.array([1.0])),
                                                    (1, np.array([b]), np.array([1.0]))]}, spherical_orb)
    aux = basis([("He", (0.2, -0.1, 0.3))], {"He": [(0, np.array([2 * a]), np.array([1.0])),
                                                    (1, np.array([a + b]), np.array([1.0])),
                                                    (2, np.array([2 * b]), np.array([1.0]))]}, spherical=False)
    n = orb.nbas
    I4 = it.ERI_2e4c(orb).reshape(n * n, n * n)
    I3 = it.ERI_2e3c(orb, aux).reshape(n * n, -1)
    G = it.ERI_2e2c(aux)
    ri = I3 @ np.linalg.solve(G, I3.T)
    assert np.max(np.abs(ri - I4)) < 1e-11 * np.max(np.abs(I4))
