"""GPU checks of the mixed-precision form (bf16 hi/lo split products on
tcgen05, FP32 accumulation) against the plain FP64 form.

The tolerance is the one of the split representation, not of FP64: b and
every operand are stored as two bf16 numbers (16 significant bits), so each
contraction carries a relative error of order 1e-5 of its largest output;
the tests bound the max-norm relative error by 2e-4 (T1 / b_pq / J / K /
elag) and the energy by 1e-5 relative.  Shapes beyond the fused kernel
(nbf5 > 64 or nbf > 256) exercise the general-shape pipeline.
"""
import ctypes as ct

import numpy as np
import pytest

import donof_b200 as d
from donof_b200 import _lib, workload

pytestmark = pytest.mark.gpu
TOL = 2e-4


def rel(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


SIZES = [
    dict(nbf=24, naux=116, nbeta=5, ncwo=3),      # water surrogate: nbf5 = 20, one 64-wide box
    dict(nbf=64, naux=40, nbeta=4, ncwo=3),       # nbf5 = 16
    dict(nbf=130, naux=70, nbeta=8, ncwo=3),      # three boxes, nbf not a multiple of 32
    dict(nbf=256, naux=1024, nbeta=16, ncwo=3),   # benchmark workload
    # general-shape pipeline (nbf5 > 64 or nbf > 256)
    dict(nbf=96, naux=60, nbeta=20, ncwo=3),      # nbf5 = 80: one row tile
    dict(nbf=202, naux=120, nbeta=33, ncwo=5),    # n-octane shape, nbf5 = 198: two row tiles
    dict(nbf=300, naux=40, nbeta=20, ncwo=3),     # nbf > 256: two column tiles in T1 and Y
    dict(nbf=330, naux=24, nbeta=65, ncwo=3),     # nbf5 = 260 > 256: two column tiles in T2
]


def ids(k):
    return f"nbf{k['nbf']}-naux{k['naux']}"


@pytest.fixture(scope="module")
def jobs(cuda_ctx):
    made = {}

    def get(kw):
        key = tuple(sorted(kw.items()))
        if key not in made:
            wl = workload.synthetic(**kw, seed=17)
            made[key] = (wl, d.eris_to_gpu(wl.b, "mixed", cuda_ctx))
        return made[key]

    yield get
    for wl, bt in made.values():
        bt.free()


def error_flag(bt):
    f = ct.c_int(-1)
    bt.ctx.check(bt.ctx.lib.donof_job_error_flag(bt.handle, ct.byref(f)))
    return f.value


@pytest.mark.parametrize("kw", SIZES, ids=ids)
def test_mixed_first_transform(jobs, kw):
    import torch

    wl, bt = jobs(kw)
    p = wl.p
    tC = d.to_device(wl.C)
    out = torch.zeros(p.nbfaux, p.nbf5, p.nbf, dtype=torch.float32, device="cuda")
    bt.ctx.check(bt.ctx.lib.donof_mixed_tmp_dev(bt.handle, tC.data_ptr(), p.nbf5, out.data_ptr()))
    torch.cuda.synchronize()
    assert error_flag(bt) == 0
    tmp = out.double().cpu().numpy()                       # [l, q, m]
    ref = np.einsum("mnl,nq->lqm", wl.b, wl.C[:, :p.nbf5])
    assert rel(tmp, ref) <= TOL


@pytest.mark.parametrize("kw", SIZES, ids=ids)
def test_mixed_jkh_mo_matches_fp64(jobs, kw):
    wl, bt = jobs(kw)
    p = wl.p
    import torch
    tC, tH = d.to_device(wl.C), d.to_device(wl.H)
    outs = {}
    for prec in ("fp64", "mixed"):
        J = torch.zeros(p.nbf5, p.nbf5, dtype=torch.float64, device="cuda")
        K = torch.zeros_like(J)
        Hc = torch.zeros(p.nbf5, dtype=torch.float64, device="cuda")
        d.JKH_MO_dev(tC, tH, bt, p.nbf5, J, K, Hc, precision=prec)
        torch.cuda.synchronize()
        outs[prec] = (d.from_device(J), d.from_device(K), Hc.cpu().numpy())
    assert error_flag(bt) == 0
    (J0, K0, H0), (J1, K1, H1) = outs["fp64"], outs["mixed"]
    assert rel(J1, J0) <= TOL and rel(K1, K0) <= TOL
    assert rel(H1, H0) <= 1e-12


@pytest.mark.parametrize("kw", SIZES, ids=ids)
def test_mixed_lagrangian_matches_fp64(jobs, kw):
    import torch

    wl, bt = jobs(kw)
    p = wl.p
    tC, tH, tn, tcj, tck = (d.to_device(x) for x in (wl.C, wl.H, wl.n, wl.cj12, wl.ck12))
    res = {}
    for prec in ("fp64", "mixed"):
        el = torch.zeros(p.nbf, p.nbf, dtype=torch.float64, device="cuda")
        hm = torch.zeros(p.nbf5, p.nbf, dtype=torch.float64, device="cuda")
        E = torch.zeros(1, dtype=torch.float64, device="cuda")
        d.compute_Lagrange2_dev(tC, tn, tH, bt, tcj, tck, p.nalpha, p.nbeta, el, hm, E, precision=prec)
        torch.cuda.synchronize()
        res[prec] = (d.from_device(el), d.from_device(hm), float(E))
    assert error_flag(bt) == 0
    (e0, h0, E0), (e1, h1, E1) = res["fp64"], res["mixed"]
    assert rel(h1, h0) <= 1e-12                # H_mat stays FP64
    assert rel(e1, e0) <= TOL
    assert np.all(e1[:, p.nbf5:] == 0.0)
    assert abs(E1 - E0) <= 1e-5 * abs(E0)


def test_mixed_rejects_bad_nbf5(cuda_ctx):
    import torch

    wl = workload.synthetic(nbf=40, naux=4, nbeta=4, ncwo=3, seed=1)
    bt = d.eris_to_gpu(wl.b, "mixed", cuda_ctx)
    tC = d.to_device(wl.C)
    out = torch.zeros(64 * 41 * 4, dtype=torch.float32, device="cuda")
    for bad in (0, 41):
        st = bt.ctx.lib.donof_mixed_tmp_dev(bt.handle, tC.data_ptr(), bad, out.data_ptr())
        assert st == _lib.ERR_ARG
    bt.free()


@pytest.mark.parametrize("kw", [SIZES[1], SIZES[4]], ids=ids)
def test_cta_limit_gives_the_same_lagrangian(cuda_ctx, kw):
    """A context limited to a few CTAs (a served job's share of the SMs) runs
    the same arithmetic; only the order of the partial sums changes."""
    import torch

    wl = workload.synthetic(**kw, seed=23)
    p = wl.p
    res = {}
    for limit in (0, 8):
        ctx = d.Context(0)
        ctx.set_cta_limit(limit)
        bt = d.eris_to_gpu(wl.b, "mixed", ctx)
        tC, tH, tn, tcj, tck = (d.to_device(x) for x in (wl.C, wl.H, wl.n, wl.cj12, wl.ck12))
        for prec in ("fp64", "mixed"):
            el = torch.zeros(p.nbf, p.nbf, dtype=torch.float64, device="cuda")
            hm = torch.zeros(p.nbf5, p.nbf, dtype=torch.float64, device="cuda")
            E = torch.zeros(1, dtype=torch.float64, device="cuda")
            d.compute_Lagrange2_dev(tC, tn, tH, bt, tcj, tck, p.nalpha, p.nbeta, el, hm, E, precision=prec)
            torch.cuda.synchronize()
            res[(limit, prec)] = d.from_device(el)
        assert error_flag(bt) == 0
        bt.free()
        ctx.close()
    assert rel(res[(8, "fp64")], res[(0, "fp64")]) <= 1e-12
    assert rel(res[(8, "mixed")], res[(0, "mixed")]) <= 1e-5  # FP32 partial sums in another order
