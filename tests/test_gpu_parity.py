"""GPU parity of the plain FP64 form against the CPU oracle (<= 1e-10 relative,
max-norm), through the C ABI (host-buffer and device-buffer entry points)."""
from pathlib import Path

import numpy as np
import pytest

from oracle import gnof as ognof
from oracle import native, orbital

import donof_b200 as d
from donof_b200 import Param, _lib, gnof, workload

pytestmark = pytest.mark.gpu
TOL = 1e-10
FIXTURES = Path(__file__).resolve().parent / "golden"  # oracle fixtures (not reference outputs)


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300))


def case(nbf, naux, nbeta, ncwo, nalpha=None, seed=0, sym=True):
    wl = workload.synthetic(nbf=nbf, naux=naux, nbeta=nbeta, ncwo=ncwo, seed=seed)
    p = wl.p
    n, cj, ck = wl.n, wl.cj12, wl.ck12
    if nalpha is not None and nalpha != nbeta:
        p = Param(nbf=nbf, nbfaux=naux, nbeta=nbeta, nalpha=nalpha, ncwo=ncwo)
        gamma = np.random.default_rng(seed + 5).standard_normal(p.nv)
        n, _ = gnof.occupations(gamma, p)
        cj, ck = gnof.coupling(n, p)
    b = wl.b
    if not sym:
        rng = np.random.default_rng(seed + 9)
        b = np.asfortranarray(b + 0.1 * rng.standard_normal(b.shape) / np.sqrt(naux))
    return p, b, wl.C, wl.H, n, np.asfortranarray(cj), np.asfortranarray(ck)


CASES = [
    dict(nbf=13, naux=29, nbeta=3, ncwo=3),                 # odd sizes (8-byte staging path)
    dict(nbf=24, naux=116, nbeta=5, ncwo=3),                # water cc-pVDZ surrogate
    dict(nbf=20, naux=17, nbeta=3, ncwo=3, nalpha=5),       # open shell (nsoc = 2)
    dict(nbf=64, naux=64, nbeta=4, ncwo=15),                # nbf5 == nbf (no0 = 0)
    dict(nbf=96, naux=33, nbeta=6, ncwo=3, sym=False),      # b not symmetric in (m, n)
    dict(nbf=130, naux=1, nbeta=7, ncwo=3),                 # single aux function, nbf not a tile multiple
    dict(nbf=256, naux=1024, nbeta=16, ncwo=3),             # benchmark workload
]


@pytest.mark.parametrize("kw", CASES, ids=lambda k: "-".join(f"{a}{b}" for a, b in k.items()))
def test_lagrange2_fp64_matches_oracle(cuda_ctx, kw):
    p, b, C, H, n, cj, ck = case(**kw)
    bt = d.eris_to_gpu(b, "fp64", cuda_ctx)
    elag, Hmat, E = d.compute_Lagrange2(C, n, H, bt, cj, ck, p.nalpha, p.nbeta, return_energy=True)
    e_ref, h_ref = native.lagrange2(C, n, H, b, cj, ck, p.nalpha, p.nbeta)
    assert rel(Hmat, h_ref) <= TOL
    assert rel(elag, e_ref) <= TOL
    assert np.all(elag[:, p.nbf5:] == 0.0)
    E_ref = orbital.e_elec(h_ref, n, e_ref, p.nbf5)
    assert abs(E - E_ref) <= TOL * max(1.0, abs(E_ref))
    bt.free()


@pytest.mark.parametrize("kw", CASES, ids=lambda k: "-".join(f"{a}{b}" for a, b in k.items()))
def test_jkh_mo_fp64_matches_oracle(cuda_ctx, kw):
    p, b, C, H, n, cj, ck = case(**kw)
    bt = d.eris_to_gpu(b, "fp64", cuda_ctx)
    J, K, Hc = d.JKH_MO(C, H, bt, p.nbf, p.nbf5, p.nbfaux)
    J0, K0, H0 = native.jkh_mo(C, H, b, p.nbf5)
    assert rel(J, J0) <= TOL and rel(K, K0) <= TOL and rel(Hc, H0) <= TOL
    bt.free()


@pytest.mark.parametrize("nbf,nbf5,scale", [(13, 12, 0.02), (24, 20, 0.0), (24, 20, 0.5), (256, 64, 0.01),
                                            (256, 64, 0.2), (100, 100, 0.3), (64, 8, 3.0)])
def test_rotate_matches_oracle(cuda_ctx, nbf, nbf5, scale):
    rng = np.random.default_rng(nbf + nbf5)
    C = np.asfortranarray(np.linalg.qr(rng.standard_normal((nbf, nbf)))[0])
    nvar = nbf5 * nbf - nbf5 * (nbf5 + 1) // 2
    y = scale * rng.standard_normal(nvar)
    p = Param(nbf=nbf, nbfaux=1, nbeta=1, nalpha=1, ncwo=nbf5 - 1)
    assert p.nbf5 == nbf5
    Cn = d.rotate_orbital(y, C, p, cuda_ctx)
    C0 = native.rotate(y, C, nbf5)
    assert rel(Cn, C0) <= TOL
    assert np.max(np.abs(Cn.T @ Cn - np.eye(nbf))) < 1e-12


def test_orbgrad_matches_oracle(cuda_ctx):
    p, b, C, H, n, cj, ck = case(nbf=40, naux=50, nbeta=4, ncwo=3, seed=3)
    s = ognof.Sizes(nbf=p.nbf, nbeta=p.nbeta, nalpha=p.nalpha, ncwo=p.ncwo, naux=p.nbfaux)
    bt = d.eris_to_gpu(b, "fp64", cuda_ctx)
    g0 = orbital.calcorbg(None, n, cj, ck, C, H, b, s)
    assert rel(d.calcorbg(None, n, cj, ck, C, H, bt, p), g0) <= TOL
    y = 0.01 * np.random.default_rng(1).standard_normal(p.nvar)
    g1 = orbital.calcorbg(y, n, cj, ck, C, H, b, s)
    assert rel(d.calcorbg(y, n, cj, ck, C, H, bt, p), g1) <= TOL
    bt.free()


@pytest.mark.parametrize("method", ["ADAM", "ADABelief", "YOGI", "Demon"])
def test_orbopt_matches_oracle_loop(cuda_ctx, method):
    p, b, C, H, n, cj, ck = case(nbf=48, naux=60, nbeta=4, ncwo=3, seed=4)
    s = ognof.Sizes(nbf=p.nbf, nbeta=p.nbeta, nalpha=p.nalpha, ncwo=p.ncwo, naux=p.nbfaux)
    bt = d.eris_to_gpu(b, "fp64", cuda_ctx)
    gamma = np.random.default_rng(4).standard_normal(p.nv)
    p.occ_method = "Softmax"
    n, _ = gnof.occupations(gamma, p)
    cj, ck = gnof.coupling(n, p)
    p.alpha, p.maxloop = 0.01, 6
    E, C1, nit, ok = d.orbopt(gamma, C, H, bt, p, method)
    E0, C0, nit0, ok0, a0, ml0 = orbital.orbopt(method, n, cj, ck, C, H, b, s, 0.01, 6, p.threshgorb)
    assert (nit, ok) == (nit0, ok0)
    assert abs(E - E0) <= TOL * max(1.0, abs(E0))
    assert rel(C1, C0) <= 1e-9
    assert (p.alpha, p.maxloop) == (a0, ml0)
    bt.free()


def test_device_entry_points_match_host(cuda_ctx):
    import torch

    p, b, C, H, n, cj, ck = case(nbf=64, naux=40, nbeta=4, ncwo=3, seed=8)
    bt = d.eris_to_gpu(b, "fp64", cuda_ctx)
    e_h, h_h, E_h = d.compute_Lagrange2(C, n, H, bt, cj, ck, p.nalpha, p.nbeta, return_energy=True)
    tC, tH, tn, tcj, tck = (d.to_device(x) for x in (C, H, n, cj, ck))
    el = torch.zeros(p.nbf, p.nbf, dtype=torch.float64, device="cuda")
    hm = torch.zeros(p.nbf5, p.nbf, dtype=torch.float64, device="cuda")
    E = torch.zeros(1, dtype=torch.float64, device="cuda")
    d.compute_Lagrange2_dev(tC, tn, tH, bt, tcj, tck, p.nalpha, p.nbeta, el, hm, E)
    torch.cuda.synchronize()
    assert np.array_equal(d.from_device(el), e_h)
    assert np.array_equal(d.from_device(hm), h_h)
    # attach a device-resident b (no copy) and compare again
    tb = d.to_device(b)
    bt2 = d.eris_to_gpu(tb, "fp64", cuda_ctx)
    e2, h2 = d.compute_Lagrange2(C, n, H, bt2, cj, ck, p.nalpha, p.nbeta)
    assert np.array_equal(e2, e_h)
    bt.free()
    bt2.free()


def test_page_locked_caller_arrays_match_pageable(cuda_ctx):
    """Caller arrays in page-locked memory are DMA'd directly (no staging copy):
    rotate_orbital and compute_Lagrange2 give the same bits as with ordinary
    arrays, for inputs and outputs, mixed pinned and pageable in one call."""
    p, b, C, H, n, cj, ck = case(nbf=64, naux=40, nbeta=4, ncwo=3, seed=11)
    bt = d.eris_to_gpu(b, "fp64", cuda_ctx)
    y = 0.02 * np.random.default_rng(2).standard_normal(p.nvar)

    def pinned(a):
        h = d.host_pinned(a.shape)
        h[...] = a
        return h

    C1 = d.rotate_orbital(y, C, p, cuda_ctx)
    e1, h1, E1 = d.compute_Lagrange2(C1, n, H, bt, cj, ck, p.nalpha, p.nbeta, return_energy=True)
    Cp = d.host_pinned(C.shape)
    d.rotate_orbital(pinned(y), pinned(C), p, cuda_ctx, out=Cp)
    assert np.array_equal(Cp, C1)
    ep, hp = d.host_pinned((p.nbf, p.nbf)), d.host_pinned((p.nbf, p.nbf5))
    _, _, Ep = d.compute_Lagrange2(Cp, pinned(n), H, bt, pinned(cj), ck, p.nalpha, p.nbeta, return_energy=True,
                                   out=(ep, hp))
    assert np.array_equal(ep, e1) and np.array_equal(hp, h1) and Ep == E1
    with pytest.raises(ValueError):
        d.compute_Lagrange2(C, n, H, bt, cj, ck, p.nalpha, p.nbeta, out=(np.zeros((p.nbf, p.nbf)), hp))
    with pytest.raises(ValueError):
        d.rotate_orbital(y, Cp, p, cuda_ctx, out=Cp)
    bt.free()


def test_energy_identity_at_full_size(cuda_ctx):
    """Size-independent check at the benchmark size: computeE_elec(Lagrangian) ==
    calce(JKH_MO) at the same C, both from the device."""
    wl = workload.synthetic(nbf=256, naux=1024, nbeta=16, ncwo=3, seed=21)
    p = wl.p
    bt = d.eris_to_gpu(wl.b, "fp64", cuda_ctx)
    _, _, E = d.compute_Lagrange2(wl.C, wl.n, wl.H, bt, wl.cj12, wl.ck12, p.nalpha, p.nbeta, return_energy=True)
    J, K, Hc = d.JKH_MO(wl.C, wl.H, bt, p.nbf, p.nbf5, p.nbfaux)
    E2 = gnof.calce(wl.n, wl.cj12, wl.ck12, J, K, Hc, p)
    assert abs(E - E2) <= TOL * max(1.0, abs(E2))
    bt.free()


@pytest.mark.parametrize("name", ["water_surrogate", "open_shell_small"])
def test_oracle_fixtures(cuda_ctx, name):
    """The CUDA path against the committed fixtures written by the oracle
    (tests/golden/make_oracle_fixtures.py); the reference itself could not be
    run, so these pin the oracle's answers, not the reference's."""
    g = np.load(FIXTURES / f"{name}.npz")
    nbf, naux, nbeta, nalpha, ncwo, seed = (int(g[k]) for k in ("nbf", "naux", "nbeta", "nalpha", "ncwo", "seed"))
    wl = workload.synthetic(nbf=nbf, naux=naux, nbeta=nbeta, ncwo=ncwo, seed=seed)
    bt = d.eris_to_gpu(wl.b, "fp64", cuda_ctx)
    elag, Hmat, E = d.compute_Lagrange2(wl.C, g["n"], wl.H, bt, g["cj12"], g["ck12"], nalpha, nbeta,
                                        return_energy=True)
    assert rel(elag, g["elag"]) <= TOL and rel(Hmat, g["Hmat"]) <= TOL
    assert abs(E - float(g["E"])) <= TOL * max(1.0, abs(float(g["E"])))
    p = Param(nbf=nbf, nbfaux=naux, nbeta=nbeta, nalpha=nalpha, ncwo=ncwo)
    J, K, Hc = d.JKH_MO(wl.C, wl.H, bt, nbf, p.nbf5, naux)
    assert rel(J, g["J"]) <= TOL and rel(K, g["K"]) <= TOL and rel(Hc, g["Hcore"]) <= TOL
    assert rel(d.rotate_orbital(g["y"], wl.C, p, cuda_ctx), g["Crot"]) <= TOL
    bt.free()


def test_invalid_arguments_raise(cuda_ctx):
    p, b, C, H, n, cj, ck = case(nbf=16, naux=4, nbeta=2, ncwo=3)
    bt = d.eris_to_gpu(b, "fp64", cuda_ctx)
    with pytest.raises(_lib.DonofError) as e:
        d.compute_Lagrange2(C, n, H, bt, cj, ck, p.nalpha + 20, p.nbeta)
    assert e.value.status == _lib.ERR_ARG
    with pytest.raises(_lib.DonofError) as e:
        d.JKH_MO(C, H, bt, p.nbf, p.nbf + 1, p.nbfaux)
    assert e.value.status == _lib.ERR_ARG
    out = np.zeros((p.nbf, p.nbf), order="F")
    hm = np.zeros((p.nbf, p.nbf5), order="F")
    with pytest.raises(_lib.DonofError) as e:  # mixed form needs a job uploaded for it
        d.compute_Lagrange2_dev(C, n, H, bt, cj, ck, p.nalpha, p.nbeta, out, hm, precision="mixed")
    assert e.value.status == _lib.ERR_ARG and "bf16 split" in str(e.value)
    bt.free()
