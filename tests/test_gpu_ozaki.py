"""The FP64 form with its first contraction on the tensor cores (int8 digit
slices of b and C5, exact int32 products, FP64 recombination; ozaki.cu).

Bounds stated here: the contraction itself is within T1_TOL = 1e-12 of the
largest |tmp| of the FP64 GEMM (7 slices of 7 bits: the dropped digit
products and the truncation residual are ~1e-13 of it), and everything
downstream keeps the FP64 form's 1e-10 parity with the oracle.
"""
import copy

import numpy as np
import pytest

from oracle import native, orbital

import donof_b200 as d
from donof_b200 import _lib, workload

from test_gpu_parity import CASES, TOL, case, rel

pytestmark = pytest.mark.gpu
T1_TOL = 1e-12


@pytest.fixture(autouse=True)
def _needs_cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _t1_pair(ctx, b, C, nbf5):
    """tmp of the DMMA GEMM and of the tensor-core form for the same job."""
    import torch

    nbf, _, naux = b.shape
    bt = d.eris_to_gpu(b, "fp64", ctx)
    tC = d.to_device(C)
    ref = torch.empty(nbf * nbf5 * naux, dtype=torch.float64, device="cuda")
    out = torch.empty_like(ref)
    torch.cuda.synchronize()
    d.t1_dev(tC, bt, nbf5, ref)
    ctx.synchronize()
    base = bt.device_bytes()
    bt.set_fp64_tc(True)
    assert bt.fp64_tc
    slices = bt.device_bytes() - base
    d.t1_dev(tC, bt, nbf5, out)
    ctx.synchronize()
    bt.free()
    return ref.cpu().numpy(), out.cpu().numpy(), slices


@pytest.mark.parametrize("nbf,naux,nbf5,sym", [
    (13, 29, 12, True),      # odd sizes: one partial tile in m, n and q
    (24, 116, 20, True),     # water cc-pVDZ surrogate
    (64, 64, 64, True),      # nbf5 == nbf
    (96, 33, 40, False),     # b not symmetric in (m, n)
    (130, 1, 70, True),      # one aux function; m and n cross a 128 tile by 2
    (202, 97, 198, True),    # n-octane shape: 4 q tiles, C5 stages streamed
    (300, 24, 70, True),     # three n chunks, two q tiles
    (256, 1024, 64, True),   # benchmark workload (C5 resident)
])
def test_t1_matches_the_fp64_gemm(cuda_ctx, nbf, naux, nbf5, sym):
    rng = np.random.default_rng(nbf * 7 + naux)
    b = workload.make_b(nbf, naux, rng)
    if not sym:
        b = np.asfortranarray(b + 0.1 * rng.standard_normal(b.shape) / np.sqrt(naux))
    C = np.asfortranarray(np.linalg.qr(rng.standard_normal((nbf, nbf)))[0])
    ref, out, slices = _t1_pair(cuda_ctx, b, C, nbf5)
    assert rel(out, ref) <= T1_TOL
    # and against the host: tmp_l = b_l C5
    tmp = np.einsum("mnl,nq->lqm", b, C[:, :nbf5]).reshape(-1)
    assert rel(out, tmp) <= T1_TOL
    ldn = (nbf + 15) // 16 * 16
    assert slices >= 7 * naux * nbf * ldn


def test_t1_rows_of_very_different_size(cuda_ctx):
    """Every row of b has its own power-of-two scale: rows 1e-9 and 1e+6 times
    the rest, and an all-zero row, keep their relative accuracy."""
    nbf, naux, nbf5 = 48, 20, 16
    rng = np.random.default_rng(3)
    b = workload.make_b(nbf, naux, rng).copy(order="F")
    b[5, :, :] *= 1e-9
    b[:, 5, :] *= 1e-9
    b[9, :, :] *= 1e6
    b[:, 9, :] *= 1e6
    b[11, :, :] = 0.0
    b[:, 11, :] = 0.0
    C = np.asfortranarray(np.linalg.qr(rng.standard_normal((nbf, nbf)))[0])
    ref, out, _ = _t1_pair(cuda_ctx, b, C, nbf5)
    ref = ref.reshape(naux, nbf5, nbf)
    out = out.reshape(naux, nbf5, nbf)
    for m in range(nbf):
        scale = np.max(np.abs(b[m]))
        if scale == 0.0:
            assert np.all(out[:, :, m] == 0.0)
            continue
        err = np.max(np.abs(out[:, :, m] - ref[:, :, m]))
        assert err <= T1_TOL * scale * np.sqrt(nbf)


@pytest.mark.parametrize("kw", CASES, ids=lambda k: "-".join(f"{a}{b}" for a, b in k.items()))
def test_lagrange2_and_jkh_mo_on_the_tensor_cores_match_the_oracle(cuda_ctx, kw):
    p, b, C, H, n, cj, ck = case(**kw)
    bt = d.eris_to_gpu(b, "fp64", cuda_ctx)
    bt.set_fp64_tc(True)
    elag, Hmat, E = d.compute_Lagrange2(C, n, H, bt, cj, ck, p.nalpha, p.nbeta, return_energy=True)
    e_ref, h_ref = native.lagrange2(C, n, H, b, cj, ck, p.nalpha, p.nbeta)
    assert rel(Hmat, h_ref) <= TOL
    assert rel(elag, e_ref) <= TOL
    assert np.all(elag[:, p.nbf5:] == 0.0)
    E_ref = orbital.e_elec(h_ref, n, e_ref, p.nbf5)
    assert abs(E - E_ref) <= TOL * max(1.0, abs(E_ref))
    J, K, Hc = d.JKH_MO(C, H, bt, p.nbf, p.nbf5, p.nbfaux)
    J0, K0, H0 = native.jkh_mo(C, H, b, p.nbf5)
    assert rel(J, J0) <= TOL and rel(K, K0) <= TOL and rel(Hc, H0) <= TOL
    bt.free()


def test_orbital_optimiser_on_the_tensor_cores_matches_the_fp64_gemm(cuda_ctx):
    """The captured optimiser loop (graph) picks up the switch both ways."""
    wl = workload.molecule_like(nbf=96, naux=384, nbeta=8, ncwo=3, seed=5, two_e_scale=0.2)
    p = wl.p
    bt = d.eris_to_gpu(wl.b, "fp64", cuda_ctx)
    runs = []
    for tc in (False, True, False):
        bt.set_fp64_tc(tc)
        E, C, nit, ok = d.orbopt(wl.gamma, wl.C, wl.H, bt, copy.deepcopy(p), "ADAM")
        runs.append((E, C, nit))
    bt.free()
    (E0, C0, n0), (E1, C1, n1), (E2, C2, n2) = runs
    assert E2 == E0 and n2 == n0 and np.array_equal(C2, C0)   # switching back restores the GEMM path exactly
    assert n1 == n0
    assert abs(E1 - E0) <= TOL * abs(E0)
    assert rel(C1, C0) <= 1e-8


def test_a_wait_that_runs_out_returns_timeout_and_the_context_recovers():
    ctx = d.Context(0, torch_stream=False)
    try:
        wl = workload.synthetic(nbf=64, naux=40, nbeta=4, ncwo=3, seed=5)
        p = wl.p
        bt = d.eris_to_gpu(wl.b, "fp64", ctx)
        bt.set_fp64_tc(True)
        call = lambda: d.compute_Lagrange2(wl.C, wl.n, wl.H, bt, wl.cj12, wl.ck12, p.nalpha, p.nbeta)
        before = call()
        ctx.set_wait_limit(1)
        try:
            with pytest.raises(_lib.DonofError) as e:
                call()
        finally:
            ctx.set_wait_limit(0)
        assert e.value.status == _lib.ERR_TIMEOUT
        after = call()
        for a, b in zip(before, after):
            np.testing.assert_array_equal(a, b)
        bt.free()
    finally:
        ctx.close()


def test_disabling_frees_the_slices(cuda_ctx):
    wl = workload.synthetic(nbf=32, naux=16, nbeta=3, ncwo=3, seed=2)
    bt = d.eris_to_gpu(wl.b, "fp64", cuda_ctx)
    base = bt.device_bytes()
    bt.set_fp64_tc(True)
    assert bt.device_bytes() > base
    bt.set_fp64_tc(False)
    assert not bt.fp64_tc
    assert bt.device_bytes() == base
    bt.free()
