"""CPU tests of the host side: the package's occupation/functional layer (the
library's native host code) against the oracle, the synthetic workloads, and the C ABI library (loads and
exports every symbol the header declares; no compute calls without a GPU)."""
import ctypes as ct
import re
from pathlib import Path

import numpy as np
import pytest

from oracle import gnof as ognof
from donof_b200 import Param, _lib, gnof, workload

ROOT = Path(__file__).resolve().parents[1]


def sizes_of(p: Param):
    return ognof.Sizes(nbf=p.nbf, nbeta=p.nbeta, nalpha=p.nalpha, ncwo=p.ncwo, naux=p.nbfaux, no1=p.no1,
                       ista=p.ista, HighSpin=p.HighSpin, h_cut=p.h_cut, occ_method=p.occ_method)


CASES = [dict(nbf=40, nbfaux=9, nbeta=4, nalpha=4, ncwo=3),
         dict(nbf=40, nbfaux=9, nbeta=4, nalpha=6, ncwo=3),
         dict(nbf=60, nbfaux=9, nbeta=5, nalpha=7, ncwo=4),
         dict(nbf=24, nbfaux=9, nbeta=5, nalpha=5, ncwo=-1)]


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("ista", [0, 1, 2, 3, 4, 5])
@pytest.mark.parametrize("occ", ["Softmax", "Trigonometric"])
def test_gnof_layer_matches_oracle(case, ista, occ):
    p = Param(ista=ista, occ_method=occ, **case)
    s = sizes_of(p)
    rng = np.random.default_rng(ista + 10 * len(occ))
    gamma = gnof.guess_gamma(p) + 0.4 * rng.standard_normal(p.nv)
    n1, dn1 = gnof.occupations(gamma, p)
    n2, dn2 = ognof.ocupacion(gamma, s)
    assert np.array_equal(n1, n2) or np.max(np.abs(n1 - n2)) < 1e-15
    assert np.max(np.abs(dn1 - dn2)) < 1e-15
    cj1, ck1 = gnof.coupling(n1, p)
    cj2, ck2 = ognof.PNOFi_selector(n2, s)
    assert np.max(np.abs(cj1 - cj2)) < 1e-15 and np.max(np.abs(ck1 - ck2)) < 1e-14
    J = rng.standard_normal((p.nbf5, p.nbf5)); J = J + J.T
    K = rng.standard_normal((p.nbf5, p.nbf5)); K = K + K.T
    Hc = rng.standard_normal(p.nbf5)
    assert abs(gnof.calcocce(gamma, J, K, Hc, p) - ognof.calcocce(gamma, J, K, Hc, s)) < 1e-12
    assert np.max(np.abs(gnof.calcoccg(gamma, J, K, Hc, p) - ognof.calcoccg(gamma, J, K, Hc, s))) < 1e-12


def test_guess_and_ordering_match_oracle():
    p = Param(nbf=40, nbfaux=9, nbeta=4, nalpha=4, ncwo=3)
    s = sizes_of(p)
    assert np.array_equal(gnof.guess_gamma(p), ognof.guess_gamma_softmax(p.ndoc, p.ncwo))
    p.occ_method = s.occ_method = "Trigonometric"
    assert np.array_equal(gnof.guess_gamma(p), ognof.guess_gamma_trigonometric(p.ndoc, p.ncwo))
    p.occ_method = s.occ_method = "Softmax"
    rng = np.random.default_rng(0)
    C = np.asfortranarray(rng.standard_normal((40, 40)))
    g = rng.standard_normal(p.nv)
    C1, g1 = gnof.order_occupations_softmax(C, g, p)
    C2, g2 = ognof.order_occupations_softmax(C, g, s)
    assert np.array_equal(C1, C2) and np.array_equal(g1, g2)


def test_param_derived_sizes():
    p = Param(nbf=256, nbfaux=1024, nbeta=16, nalpha=16, ncwo=3)
    assert (p.nbf5, p.nv, p.nvar, p.no0) == (64, 48, 14304, 192)
    w = Param(nbf=24, nbfaux=116, nbeta=5, nalpha=5)  # water cc-pVDZ: ncwo = trunc(19/5) = 3
    assert (w.ncwo, w.nbf5, w.nvar, w.nv) == (3, 20, 270, 15)
    o = Param(nbf=202, nbfaux=974, nbeta=33, nalpha=33, ncwo=5)
    assert (o.nbf5, o.nvar, o.nv) == (198, 20295, 165)


def test_workload_is_seeded_and_shaped():
    a = workload.synthetic(nbf=20, naux=7, nbeta=3, ncwo=3, seed=9)
    b = workload.synthetic(nbf=20, naux=7, nbeta=3, ncwo=3, seed=9)
    assert a.b.shape == (20, 20, 7) and a.b.flags.f_contiguous
    assert np.array_equal(a.b, b.b) and np.array_equal(a.C, b.C)
    assert np.allclose(a.b, a.b.transpose(1, 0, 2))
    assert np.allclose(a.C.T @ a.C, np.eye(20))
    assert np.allclose(a.H, a.H.T)


def header_symbols():
    text = (ROOT / "include" / "donof_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)  # drop comments
    return sorted(set(re.findall(r"\b(donof_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_header_symbol():
    lib = _lib.load()
    syms = header_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(lib, s), f"{s} missing from libdonofb200.so"
    assert set(syms) == set(_lib.SIGNATURES), "ctypes signature table out of sync with the header"
    assert lib.donof_version() >= 1
    assert lib.donof_status_string(_lib.ERR_ARG) == b"invalid argument"


def test_create_without_gpu_reports_an_error():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = _lib.load()
    h = ct.c_void_p()
    st = lib.donof_create(0, ct.byref(h))
    assert st != _lib.OK and not h.value
    assert b"device" in lib.donof_last_error(None)


@pytest.mark.parametrize("occ", ["Softmax", "Trigonometric"])
@pytest.mark.parametrize("case", [dict(nbf=40, nbeta=5, nalpha=5, ncwo=3), dict(nbf=30, nbeta=4, nalpha=6, ncwo=2),
                                  dict(nbf=24, nbeta=3, nalpha=3, ncwo=1)])
def test_n_to_gammas_restart(case, occ):
    """Restart from occupations (src/energy.jl:95-99): n_to_gammas matches the
    oracle's line-by-line restatement of src/utils.jl:539-584, and the gamma it
    gives reproduces the occupations."""
    p = Param(nbfaux=8, occ_method=occ, **case)
    s = ognof.Sizes(nbf=case["nbf"], nbeta=case["nbeta"], nalpha=case["nalpha"], ncwo=case["ncwo"], occ_method=occ)
    rng = np.random.default_rng(3)
    gamma = rng.standard_normal(p.nv)
    if occ == "Trigonometric":
        gamma = np.abs(gamma) % (np.pi / 2)           # the principal branch acos / asin return
    n, _ = gnof.occupations(gamma, p)
    g1 = gnof.n_to_gammas(n, p)
    g0 = (ognof.n_to_gammas_softmax if occ == "Softmax" else ognof.n_to_gammas_trigonometric)(n, s)
    assert np.allclose(g1, g0, rtol=0, atol=1e-13)
    n1, _ = gnof.occupations(g1, p)
    assert np.allclose(n1, n, rtol=0, atol=1e-12)
