"""Continuous batching on the GPU: jobs of different basis sizes and precisions
give the same energies when run one at a time and when they share the device
(each on its own stream, admitted while the others run)."""
import numpy as np
import pytest

from donof_b200 import workload
from donof_b200.serve import Request, Server

pytestmark = pytest.mark.gpu

JOBS = [
    (dict(nbf=20, naux=30, nbeta=3, ncwo=3), 2, "fp64"),
    (dict(nbf=28, naux=44, nbeta=4, ncwo=3), 3, "fp64"),
    (dict(nbf=24, naux=40, nbeta=3, ncwo=3), 4, "mixed"),
    (dict(nbf=20, naux=30, nbeta=3, ncwo=3), 2, "mixed_refined"),
]


def _requests():
    out = []
    for i, (cfg, seed, prec) in enumerate(JOBS):
        wl = workload.molecule_like(**cfg, seed=seed)
        p = wl.p
        p.threshgorb, p.threshgocc, p.threshen = 1e-4, 1e-4, 1e-8
        out.append(Request(H=wl.H, b=wl.b, C=wl.C, p=p, gamma=wl.gamma, precision=prec, maxit=400, tag=i))
    return out


def test_results_alone_equal_results_in_the_mix():
    alone = []
    with Server(max_inflight=1) as s:
        for r in _requests():
            alone.append(s.wait(s.submit(r), timeout=600))
    with Server(max_inflight=len(JOBS)) as s:
        tickets = [s.submit(r) for r in _requests()]
        mix = [s.wait(t, timeout=600) for t in tickets]
    for a, m in zip(alone, mix):
        assert a.error is None and m.error is None, (a.error, m.error)
        assert a.converged and m.converged
        assert abs(a.E_elec - m.E_elec) <= 1e-10 * max(1.0, abs(a.E_elec))
        assert np.max(np.abs(a.n - m.n)) <= 1e-8
    # the jobs did share the device: some ran while others were in flight
    spans = sorted((m.t_start, m.t_done) for m in mix)
    assert any(spans[i + 1][0] < spans[i][1] for i in range(len(spans) - 1))
