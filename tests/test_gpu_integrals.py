"""The integral front end on the B200: the device three-centre kernel against
the host path, and compute_integrals -> Iaux -> the energy loop on H2 against
the exact two-electron energy of the same (RI) Hamiltonian."""
import numpy as np
import pytest

import donof_b200 as d
from donof_b200 import _lib, gnof
from donof_b200 import integrals as it
from donof_b200.guess import guess

from test_integrals import H_STO3G, basis

pytestmark = pytest.mark.gpu

ORB = {"H": [(0, np.array([1.3, 0.4]), np.array([0.6, 0.5])), (1, np.array([0.8]), np.array([1.0]))],
       "C": [(0, np.array([7.0, 1.1, 0.3]), np.array([0.2, 0.5, 0.4])), (1, np.array([2.0, 0.5]), np.array([0.4, 0.7])),
             (2, np.array([0.9, 0.35]), np.array([0.6, 0.5]))]}
AUX = {"H": [(0, np.array([2.0]), np.array([1.0])), (1, np.array([1.1]), np.array([1.0])),
             (2, np.array([0.9]), np.array([1.0]))],
       "C": [(0, np.array([9.0, 1.5]), np.array([0.5, 0.5])), (1, np.array([2.2]), np.array([1.0])),
             (2, np.array([1.2]), np.array([1.0])), (3, np.array([0.8]), np.array([1.0]))]}
GEOM = [("C", (0.1, -0.2, 0.3)), ("H", (1.2, 0.9, -0.4)), ("H", (-1.0, 0.4, 1.1)), ("H", (0.2, -1.5, -0.6))]


@pytest.mark.parametrize("spherical", [True, False])
def test_device_three_centre_matches_host(cuda_ctx, spherical):
    b, aux = basis(GEOM, ORB, spherical), basis(GEOM, AUX, spherical)
    host = it.ERI_2e3c(b, aux)
    dev = it.ERI_2e3c_dev(b, aux, cuda_ctx).cpu().numpy().reshape(host.shape, order="F")
    assert np.max(np.abs(dev - host)) <= 1e-13 * np.max(np.abs(host))


def test_device_three_centre_with_f_orbital_and_g_auxiliary_shells(cuda_ctx):
    b = basis(GEOM, {**ORB, "C": ORB["C"] + [(3, np.array([0.7]), np.array([1.0]))]})
    aux = basis(GEOM, {**AUX, "C": AUX["C"] + [(4, np.array([0.9]), np.array([1.0]))]})
    host = it.ERI_2e3c(b, aux)
    dev = it.ERI_2e3c_dev(b, aux, cuda_ctx).cpu().numpy().reshape(host.shape, order="F")
    assert np.max(np.abs(dev - host)) <= 1e-13 * np.max(np.abs(host))


def test_device_three_centre_refuses_shells_beyond_its_limits(cuda_ctx):
    b = basis(GEOM, {**ORB, "C": ORB["C"] + [(4, np.array([0.7]), np.array([1.0]))]})
    aux = basis(GEOM, AUX)
    with pytest.raises(_lib.DonofError) as e:
        it.ERI_2e3c_dev(b, aux, cuda_ctx)
    assert e.value.status == _lib.ERR_ARG


def _two_electron_exact(h, bmo):
    """Lowest singlet of two electrons in orthonormal orbitals: h one-electron,
    (ij|kl) = sum_P b[i,j,P] b[k,l,P]; the spatial wave function is symmetric."""
    n = h.shape[0]
    eri = np.einsum("ijP,klP->ijkl", bmo, bmo)
    H2 = (np.einsum("ik,jl->ijkl", h, np.eye(n)) + np.einsum("ik,jl->ijkl", np.eye(n), h) +
          eri.transpose(0, 2, 1, 3)).reshape(n * n, n * n)
    sym = []
    for i in range(n):
        for j in range(i, n):
            v = np.zeros((n, n))
            v[i, j] += 1.0
            v[j, i] += 1.0
            sym.append(v.ravel() / np.linalg.norm(v))
    Q = np.array(sym).T
    return float(np.linalg.eigvalsh(Q.T @ H2 @ Q)[0])


def test_h2_energy_from_computed_integrals_is_the_exact_two_electron_energy(cuda_ctx):
    """H2 / STO-3G at 1.4 bohr with an s, p, d auxiliary basis: compute_integrals
    (one-electron matrices, (P|Q), (mn|P) on the device, b = I G^{-1/2} by
    Iaux_gpu).  b agrees with I G^{-1/2} in numpy; JKH_MO on the device at the
    symmetry orbitals (sigma_g, sigma_u, fixed by symmetry in a minimal basis)
    then gives a GNOF energy whose minimum over the occupation is the lowest
    two-electron eigenvalue of the same RI Hamiltonian (GNOF for one pair in two
    orbitals is the Loewdin-Shull functional, exact for two electrons), within
    the RI error of the published full-CI energy (-1.137284 Eh).  DoNOF.energy's
    loop started there ends at orbitals and occupations whose GNOF energy is
    that exact energy; the energy it reports is the orbital step's, taken
    before the iteration's occupation step (src/energy.jl:147-168), so here,
    where the first iteration already meets the gradient thresholds, it lies
    above."""
    R = 1.4 / it.ANGSTROM_TO_BOHR
    atoms, _, _ = it.parse_molecule(f"H 0 0 0\nH 0 0 {R:.12f}")
    bset = it.BasisSet("sto-3g", atoms, {"H": H_STO3G}, spherical=True)
    ex = 0.15 * 2.2 ** np.arange(7)
    aux_sh = {"H": [(0, np.array([x]), np.array([1.0])) for x in ex] +
                   [(1, np.array([0.6]), np.array([1.0])), (1, np.array([2.0]), np.array([1.0])),
                    (2, np.array([1.0]), np.array([1.0]))]}
    aux = it.BasisSet("aux", atoms, aux_sh, spherical=True)
    p = d.Param(nbf=bset.nbas, nbfaux=0, nalpha=1, nbeta=1)
    S, T, V, H, bt = it.compute_integrals(bset, aux, p, cuda_ctx)
    assert p.nbfaux == aux.nbas and bt.naux == aux.nbas
    # b as the library keeps it (read back through the transform with C = 1), against I G^{-1/2}
    G = it.ERI_2e2c(aux)
    w, U = np.linalg.eigh((G + G.T) / 2)
    b_ref = np.einsum("mnQ,QP->mnP", it.ERI_2e3c(bset, aux), (U / np.sqrt(w)) @ U.T)
    J1, K1, _ = d.JKH_MO(np.eye(2), H, bt, 2, 2, aux.nbas)
    assert np.allclose(J1, np.einsum("iiP,jjP->ij", b_ref, b_ref), atol=1e-10)
    assert np.allclose(K1, np.einsum("ijP,ijP->ij", b_ref, b_ref), atol=1e-10)
    # the exact two-electron energy of the same Hamiltonian, in Loewdin-orthogonalised orbitals
    ws, Us = np.linalg.eigh(S)
    X = Us @ np.diag(ws ** -0.5) @ Us.T
    E_exact = _two_electron_exact(X @ H @ X, np.einsum("mi,nj,mnP->ijP", X, X, b_ref))
    assert abs(E_exact + 1.0 / 1.4 - (-1.137284)) < 5e-4
    # GNOF at the symmetry orbitals, minimised over the occupation
    C, gamma = guess(H, p, S)
    J, K, Hc = d.JKH_MO(C, H, bt, 2, 2, aux.nbas)
    Es = []
    for g in np.linspace(-8.0, 0.0, 8001):
        n, _ = gnof.occupations(np.array([g]), p)
        cj, ck = gnof.coupling(n, p)
        Es.append(gnof.calce(n, cj, ck, J, K, Hc, p))
    assert abs(min(Es) - E_exact) < 1e-7, (min(Es), E_exact)
    # the energy loop
    p.threshgorb, p.threshgocc, p.threshen = 1e-6, 1e-6, 1e-10
    C1, g1, n1, _, r, _ = d.api.energy_loop(H, bt, p, C, gamma, maxit=2000)
    assert r["converged"]
    J, K, Hc = d.JKH_MO(C1, H, bt, 2, 2, aux.nbas)
    cj, ck = gnof.coupling(n1, p)
    E_final = gnof.calce(n1, cj, ck, J, K, Hc, p)
    assert abs(E_final - E_exact) < 1e-7, (E_final, E_exact)
    assert r["E_elec"] >= E_final - 1e-9
    bt.free()


def test_compute_integrals_takes_the_auxiliary_basis_as_text(cuda_ctx):
    """The auxiliary basis given as Gaussian94 text is placed on the molecule in
    the orbital basis' form and gives the same RI tensor as the BasisSet."""
    text = ("H 0\nS 3 1.00\n 3.42525091 0.15432897\n 0.62391373 0.53532814\n 0.16885540 0.44463454\n****\n")
    aux_text = ("H 0\nS 1 1.00\n 1.2 1.0\n****\nH 0\nS 1 1.00\n 0.35 1.0\nP 1 1.00\n 0.9 1.0\n****\n")
    bset, p = it.molecule("H 0 0 0\nH 0 0 0.74", text, spherical=True)
    _, _, _, H, b1 = it.compute_integrals(bset, aux_text, p, cuda_ctx)
    aux = it.BasisSet.from_text("aux", aux_text, bset.atoms, True)
    _, _, _, _, b2 = it.compute_integrals(bset, aux, p, cuda_ctx)
    assert b1.naux == aux.nbas == 2 * (1 + 1 + 3)
    J1, K1, _ = d.JKH_MO(np.eye(2), H, b1, 2, 2, b1.naux)
    J2, K2, _ = d.JKH_MO(np.eye(2), H, b2, 2, 2, b2.naux)
    assert np.array_equal(J1, J2) and np.array_equal(K1, K2)
    b1.free()
    b2.free()
