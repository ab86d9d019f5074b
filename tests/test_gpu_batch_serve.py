"""Continuous batching at the step level (donof_batch_serve): the batch's jobs
are slots; requests of a slot's shape take it when it frees, every outer
iteration advances all running requests as grouped launches, and each request
gives bit-for-bit what donof_energy gives it alone -- whatever it shares the
batch with and whenever it arrives."""
import copy
import threading
import time

import numpy as np
import pytest

from oracle import gnof as ognof

import donof_b200 as d
from donof_b200 import _lib, workload

pytestmark = pytest.mark.gpu

SHAPES = [dict(nbf=24, naux=96, nbeta=5, ncwo=3), dict(nbf=40, naux=80, nbeta=4, ncwo=3)]


def _requests(count_per_shape, seed0=10):
    out = []
    for k in range(count_per_shape):
        for s, shape in enumerate(SHAPES):
            wl = workload.molecule_like(**shape, seed=seed0 + 10 * k + s)
            wl.p.threshgorb, wl.p.threshgocc, wl.p.threshen = 1e-5, 1e-5, 1e-9
            out.append((wl, ognof.guess_gamma_softmax(wl.p.nbeta, wl.p.ncwo)))
    return out


def _alone(wl, bt, g):
    C1, g1, n1, _, r1, _ = d.api.energy_loop(wl.H, bt, copy.deepcopy(wl.p), wl.C, g, maxit=1000)
    return C1, g1, n1, r1


def _check(q, tickets, reqs, bts):
    for t, (wl, g), bt in zip(tickets, reqs, bts):
        C, gamma, n, r = q.wait(t)
        C1, g1, n1, r1 = _alone(wl, bt, g)
        assert r["converged"]
        assert r == r1, (t, r, r1)
        assert np.array_equal(C, C1) and np.array_equal(gamma, g1) and np.array_equal(n, n1), t


def test_more_requests_than_slots_each_as_alone(cuda_ctx):
    """Two slots (one per shape), six requests: the slots are refilled as requests
    converge, and every request ends bit-for-bit as it does alone."""
    reqs = _requests(3)
    bts = [d.eris_to_gpu(wl.b, "fp64", cuda_ctx) for wl, _ in reqs]
    batch = d.Batch(bts[:2], [copy.deepcopy(reqs[0][0].p), copy.deepcopy(reqs[1][0].p)], cuda_ctx)
    q = d.BatchQueue()
    tickets = [q.push(bt, wl.H, wl.C, g, copy.deepcopy(wl.p), maxit=1000) for (wl, g), bt in zip(reqs, bts)]
    q.close()
    batch.serve(q)
    _check(q, tickets, reqs, bts)
    batch.free()
    q.free()
    for bt in bts:
        bt.free()


def test_requests_pushed_while_serving(cuda_ctx):
    """Requests that arrive while the batch runs join at the next outer iteration."""
    reqs = _requests(2, seed0=40)
    bts = [d.eris_to_gpu(wl.b, "fp64", cuda_ctx) for wl, _ in reqs]
    batch = d.Batch(bts[:2] + bts[:2], [copy.deepcopy(reqs[j % 2][0].p) for j in range(4)], cuda_ctx)
    q = d.BatchQueue()
    err = []

    def run():
        try:
            batch.serve(q)
        except Exception as e:  # pragma: no cover - reported below
            err.append(e)

    th = threading.Thread(target=run)
    th.start()
    tickets = []
    for (wl, g), bt in zip(reqs, bts):
        tickets.append(q.push(bt, wl.H, wl.C, g, copy.deepcopy(wl.p), maxit=1000))
        time.sleep(0.05)
    q.close()
    th.join(120)
    assert not th.is_alive() and not err
    _check(q, tickets, reqs, bts)
    batch.free()
    q.free()
    for bt in bts:
        bt.free()


def test_a_request_that_fits_no_slot_is_refused(cuda_ctx):
    reqs = _requests(1, seed0=70)
    bts = [d.eris_to_gpu(wl.b, "fp64", cuda_ctx) for wl, _ in reqs]
    batch = d.Batch(bts[:1], [copy.deepcopy(reqs[0][0].p)], cuda_ctx)  # a slot of the first shape only
    q = d.BatchQueue()
    t_ok = q.push(bts[0], reqs[0][0].H, reqs[0][0].C, reqs[0][1], copy.deepcopy(reqs[0][0].p), maxit=1000)
    t_bad = q.push(bts[1], reqs[1][0].H, reqs[1][0].C, reqs[1][1], copy.deepcopy(reqs[1][0].p), maxit=1000)
    q.close()
    batch.serve(q)
    with pytest.raises(_lib.DonofError) as e:
        q.wait(t_bad)
    assert e.value.status == _lib.ERR_ARG
    assert q.wait(t_ok)[3]["converged"]
    batch.free()
    q.free()
    for bt in bts:
        bt.free()
