"""Failure detection on the GPU, without a fault or a hang.

Every wait in the library's kernels is bounded.  A tiny wait budget
(donof_set_wait_limit) makes the waits run out on purpose: the kernels stop,
drain what they have in flight, free their tensor memory and record the
failure in the context's failure words; the call returns DONOF_ERR_TIMEOUT
and the context stays usable (the next call with the normal budget gives the
same result as before the failure).  Host-side failures: a RI tensor holding
a NaN or an infinity is refused, a job larger than the server's memory budget
is refused, and queued and running server jobs can be cancelled.
"""
import copy
import threading
import time

import numpy as np
import pytest

import donof_b200 as d
from donof_b200 import _lib, workload

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _needs_cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


@pytest.fixture
def ctx():
    c = d.Context(0, torch_stream=False)
    yield c
    c.close()


def _lagrangian(wl, bt):
    p = wl.p
    return d.compute_Lagrange2(wl.C, wl.n, wl.H, bt, wl.cj12, wl.ck12, p.nalpha, p.nbeta, return_energy=True)


def _fails_then_recovers(ctx, call, what):
    before = call()
    ctx.set_wait_limit(1)  # one cycle: every wait that is not already complete runs out
    try:
        with pytest.raises(_lib.DonofError) as e:
            call()
    finally:
        ctx.set_wait_limit(0)
    assert e.value.status == _lib.ERR_TIMEOUT
    assert what in str(e.value)
    assert ctx.error_flags() == 0  # the failing call read and cleared the words
    after = call()
    for a, b in zip(before, after):
        np.testing.assert_array_equal(np.asarray(a), np.asarray(b))


@pytest.mark.parametrize("precision,kw", [
    ("fp64", dict(nbf=96, naux=64, nbeta=8, ncwo=3)),     # cooperative FP64 tail: grid barrier
    ("mixed", dict(nbf=64, naux=40, nbeta=4, ncwo=3)),    # fused tcgen05 kernel: mbarrier waits
    ("mixed", dict(nbf=96, naux=60, nbeta=20, ncwo=3)),   # general tcgen05 pipeline (nbf5 = 80)
], ids=["fp64-tail", "mixed-fused", "mixed-general"])
def test_a_wait_that_runs_out_returns_timeout_and_the_context_recovers(ctx, precision, kw):
    wl = workload.synthetic(**kw, seed=5)
    bt = d.eris_to_gpu(wl.b, precision, ctx)
    try:
        _fails_then_recovers(ctx, lambda: _lagrangian(wl, bt),
                             "grid-barrier" if precision == "fp64" else "mbarrier")
    finally:
        bt.free()


def test_rotation_barrier_timeout_returns_timeout_and_the_context_recovers(ctx):
    wl = workload.synthetic(nbf=96, naux=8, nbeta=8, ncwo=3, seed=6)
    p = wl.p
    y = np.random.default_rng(1).standard_normal(p.nbf5 * p.nbf - p.nbf5 * (p.nbf5 + 1) // 2) * 0.05
    _fails_then_recovers(ctx, lambda: (d.rotate_orbital(y, wl.C, p, ctx),), "grid-barrier")


def test_job_error_flag_reports_a_failure_of_a_device_entry_point(ctx):
    """The _dev entry points only enqueue work: their caller reads the flag."""
    import ctypes as ct
    import torch

    wl = workload.synthetic(nbf=64, naux=40, nbeta=4, ncwo=3, seed=8)
    p = wl.p
    bt = d.eris_to_gpu(wl.b, "mixed", ctx)
    try:
        dev = {k: d.to_device(getattr(wl, k)) for k in ("C", "n", "H", "cj12", "ck12")}
        elag = torch.zeros((p.nbf, p.nbf), dtype=torch.float64, device="cuda")
        Hmat = torch.zeros((p.nbf5, p.nbf), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()  # the inputs were made on torch's stream, the call runs on the context's
        flag = ct.c_int()
        ctx.set_wait_limit(1)
        ctx.check(ctx.lib.donof_lagrange2_dev(bt.handle, dev["C"].data_ptr(), dev["n"].data_ptr(),
                                              dev["H"].data_ptr(), dev["cj12"].data_ptr(), dev["ck12"].data_ptr(),
                                              p.nbf5, p.nalpha, p.nbeta, elag.data_ptr(), Hmat.data_ptr(), None))
        ctx.set_wait_limit(0)
        ctx.check(ctx.lib.donof_job_error_flag(bt.handle, ct.byref(flag)))
        assert flag.value == 1
        ctx.check(ctx.lib.donof_job_error_flag(bt.handle, ct.byref(flag)))
        assert flag.value == 0  # cleared by the read
    finally:
        ctx.set_wait_limit(0)
        bt.free()


@pytest.mark.parametrize("bad", [np.nan, np.inf, -np.inf])
def test_a_b_tensor_with_nan_or_infinity_is_refused(ctx, bad):
    wl = workload.synthetic(nbf=24, naux=16, nbeta=3, ncwo=3, seed=9)
    b = np.array(wl.b, order="F")
    b[3, 5, 7] = bad
    for prec in ("fp64", "mixed"):
        with pytest.raises(_lib.DonofError) as e:
            d.eris_to_gpu(b, prec, ctx)
        assert e.value.status == _lib.ERR_ARG and "NaN or an infinity" in str(e.value)
    # attaching a device tensor is checked the same way
    import ctypes as ct
    t = d.to_device(b)
    h = ct.c_void_p()
    st = ctx.lib.donof_b_attach(ctx.handle, t.data_ptr(), wl.p.nbf, wl.p.nbfaux, _lib.PREC_FP64, ct.byref(h))
    assert st == _lib.ERR_ARG and not h.value
    assert ctx.error_flags() == 0
    # and a finite tensor still goes through
    d.eris_to_gpu(wl.b, "fp64", ctx).free()


def _native_request(wl, maxit=2000):
    from donof_b200.serve import Request
    return Request(H=wl.H, b=wl.b, C=wl.C, p=copy.deepcopy(wl.p), gamma=wl.gamma, precision="fp64", maxit=maxit)


def _slow_job(seed):
    wl = workload.molecule_like(nbf=48, naux=116, nbeta=10, ncwo=3, seed=seed, two_e_scale=0.2)
    wl.p.threshgorb = wl.p.threshgocc = 1e-12  # never met: the job runs until cancelled
    wl.p.threshen = 1e-10
    return wl


def test_native_server_refuses_a_job_beyond_its_budget():
    from donof_b200.serve import NativeServer
    wl = workload.molecule_like(nbf=48, naux=116, nbeta=10, ncwo=3, seed=3)
    with NativeServer(budget_bytes=1 << 20, max_inflight=1) as srv:
        with pytest.raises(_lib.DonofError) as e:
            srv.submit(_native_request(wl))
        assert e.value.status == _lib.ERR_ARG


def test_native_server_cancels_queued_and_running_jobs():
    from donof_b200.serve import NativeServer
    with NativeServer(max_inflight=1) as srv:
        t_run = srv.submit(_native_request(_slow_job(21)))
        t_queued = srv.submit(_native_request(_slow_job(22)))
        srv.cancel(t_queued)
        r_q = srv.wait(t_queued)
        assert r_q.error == "cancelled"
        srv.cancel(t_run)  # stops at its next outer iteration
        r_r = srv.wait(t_run)
        assert r_r.error == "cancelled"
        # the server goes on serving: the next job runs to its end
        wl = workload.molecule_like(nbf=24, naux=58, nbeta=5, ncwo=3, seed=23, two_e_scale=0.2)
        wl.p.threshgorb = wl.p.threshgocc = 1e-4
        r = srv.wait(srv.submit(_native_request(wl, maxit=20)))
        assert r.error is None and r.iterations > 0 and np.isfinite(r.E_elec)


def test_native_server_destroy_releases_a_blocked_waiter():
    from donof_b200.serve import NativeServer
    srv = NativeServer(max_inflight=1)
    t_run = srv.submit(_native_request(_slow_job(31)))
    t_queued = srv.submit(_native_request(_slow_job(32)))
    got = {}
    th = threading.Thread(target=lambda: got.setdefault("r", srv.wait(t_queued)))
    th.start()
    time.sleep(1.0)     # the waiter is blocked inside donof_server_wait by now
    srv.cancel(t_run)   # so that destroy does not wait for a long job
    srv.close()         # cancels the queued job; the waiter returns its cancelled result
    th.join(60)
    assert not th.is_alive()
    assert got["r"].error == "cancelled"


def test_eigensolver_barrier_timeout_returns_timeout_and_recovers(ctx):
    """The Jacobi eigensolver of Iaux waits on bounded grid barriers: a one-cycle
    budget makes them run out; Iaux returns DONOF_ERR_TIMEOUT and the next call
    gives the same b as before.  naux = 200 gives 100 x 101 / 2 rotation pairs
    per round, so the solver runs on 20 CTAs and its barriers really wait (one
    CTA alone never waits)."""
    import torch
    rng = np.random.default_rng(3)
    nbf, naux = 8, 200
    Q, _ = np.linalg.qr(rng.standard_normal((naux, naux)))
    G = np.asfortranarray((Q * np.linspace(0.5, 2.0, naux)) @ Q.T)
    I = np.asfortranarray(rng.standard_normal((nbf, nbf, naux)))

    def download(bt):
        C = d.to_device(np.asfortranarray(np.eye(nbf)))
        out = torch.zeros(nbf * nbf * naux, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()  # the fill runs on torch's stream, the transform on the context's
        d.transform_dev(C, bt, nbf, out=out)
        ctx.synchronize()
        return out.cpu().numpy()

    b0 = d.Iaux_gpu(G, I, "fp64", ctx)
    before = download(b0)
    b0.free()
    ctx.set_wait_limit(1)
    try:
        with pytest.raises(_lib.DonofError) as e:
            d.Iaux_gpu(G, I, "fp64", ctx)
    finally:
        ctx.set_wait_limit(0)
    assert e.value.status == _lib.ERR_TIMEOUT
    b1 = d.Iaux_gpu(G, I, "fp64", ctx)
    np.testing.assert_array_equal(download(b1), before)
    b1.free()


def test_grouped_mixed_kernel_timeout_returns_timeout_and_recovers(ctx):
    """The grouped mixed Lagrangian of a batch (one launch over every job's CTA
    range) with a one-cycle wait budget: DONOF_ERR_TIMEOUT, then the same
    result as before with the normal budget."""
    import torch
    jobs = [workload.synthetic(nbf=48, naux=60, nbeta=4, ncwo=3, seed=s) for s in (1, 2)]
    bts = [d.eris_to_gpu(wl.b, "mixed", ctx) for wl in jobs]
    batch = d.Batch(bts, [wl.p for wl in jobs], ctx)
    batch.set_precision("mixed")
    dev = [{k: d.to_device(getattr(wl, k)) for k in ("C", "n", "H", "cj12", "ck12")} for wl in jobs]
    elag = [torch.zeros(wl.p.nbf, wl.p.nbf, dtype=torch.float64, device="cuda") for wl in jobs]
    hmat = [torch.zeros(wl.p.nbf5, wl.p.nbf, dtype=torch.float64, device="cuda") for wl in jobs]
    torch.cuda.synchronize()  # torch's copies and fills before the context's stream reads them
    call = lambda: batch.lagrange2([x["n"] for x in dev], [x["cj12"] for x in dev], [x["ck12"] for x in dev],
                                   [x["H"] for x in dev], [x["C"] for x in dev], elag, hmat)
    before = call()
    ctx.set_wait_limit(1)
    try:
        with pytest.raises(_lib.DonofError) as e:
            call()
    finally:
        ctx.set_wait_limit(0)
    assert e.value.status == _lib.ERR_TIMEOUT
    assert call() == before
    batch.free()
    for bt in bts:
        bt.free()
