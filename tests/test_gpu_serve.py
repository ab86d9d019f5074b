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


def test_native_server_matches_sequential_fp64(cuda_ctx):
    """donof_server_*: jobs of different sizes served natively (8 workers) give
    the FP64 energies of running each job alone, and report every job done."""
    import copy
    import donof_b200 as d
    from donof_b200.optimize import energy
    from donof_b200.serve import NativeServer, Request

    shapes = [(24, 58, 5, 3), (34, 80, 5, 5), (48, 116, 10, 3), (24, 58, 5, 3), (40, 90, 6, 3)]
    wls = [workload.molecule_like(nbf=a, naux=b, nbeta=c, ncwo=e, seed=40 + i, two_e_scale=0.2)
           for i, (a, b, c, e) in enumerate(shapes)]
    for wl in wls:
        wl.p.threshgorb = wl.p.threshgocc = 1e-5
        wl.p.threshen = 1e-6
    alone = []
    for wl in wls:
        bt = d.eris_to_gpu(wl.b, "fp64", cuda_ctx)
        alone.append(energy(wl.H, bt, copy.deepcopy(wl.p), wl.C, wl.gamma, maxit=500))
        bt.free()
    with NativeServer(max_inflight=8) as srv:
        tickets = [srv.submit(Request(H=wl.H, b=wl.b, C=wl.C, p=copy.deepcopy(wl.p), gamma=wl.gamma,
                                      precision="fp64", maxit=500)) for wl in wls]
        served = [srv.wait(t) for t in tickets]
    for a, s in zip(alone, served):
        assert s.error is None, s.error
        assert s.converged == a.converged
        assert abs(s.E_elec - a.E_elec) <= 1e-10 * max(1.0, abs(a.E_elec))
        assert np.max(np.abs(s.n - a.n)) <= 1e-8


def test_grouped_server_gives_each_job_its_alone_result():
    """Small FP64 jobs that wait together start as one group (donof_batch_energy:
    their gradient steps advance with grouped launches); each job's energy,
    occupations and orbitals are bit-for-bit those of the job served alone."""
    import copy

    shapes = [(24, 58, 5, 3), (34, 80, 5, 5), (48, 116, 10, 3), (24, 58, 5, 3), (40, 90, 6, 3)]
    wls = [workload.molecule_like(nbf=a, naux=b, nbeta=c, ncwo=e, seed=60 + i, two_e_scale=0.2)
           for i, (a, b, c, e) in enumerate(shapes)]
    for wl in wls:
        wl.p.threshgorb = wl.p.threshgocc = 1e-5
        wl.p.threshen = 1e-6
    req = lambda wl, i: Request(H=wl.H, b=wl.b, C=wl.C, p=copy.deepcopy(wl.p), gamma=wl.gamma, precision="auto",
                                maxit=500, tag=i)
    with Server(max_inflight=1) as s:
        alone = [s.wait(s.submit(req(wl, i)), timeout=600) for i, wl in enumerate(wls)]
    with Server(max_inflight=1, group_max=8) as s:
        tickets = [s.submit(req(wl, i)) for i, wl in enumerate(wls)]
        grouped = [s.wait(t, timeout=600) for t in tickets]
    # the first job took the slot alone; the others waited and ran as one group
    starts = [g.t_start for g in grouped]
    assert len(set(starts[1:])) == 1 and starts[1] > starts[0]
    for a, g in zip(alone, grouped):
        assert a.error is None and g.error is None, (a.error, g.error)
        assert a.converged and g.converged
        assert g.E_elec == a.E_elec and g.iterations == a.iterations
        assert np.array_equal(g.n, a.n) and np.array_equal(g.C, a.C)


def test_continuous_server_gives_each_job_its_alone_result():
    """continuous_slots: FP64 jobs of one shape share a batch whose slots are
    refilled as jobs converge (donof_batch_serve), jobs of other shapes run in
    their own batches, mixed jobs on their own streams; each FP64 job's energy,
    occupations and orbitals are bit-for-bit those it gets served alone."""
    import copy

    shapes = [(24, 58, 5, 3), (34, 80, 5, 5), (24, 58, 5, 3), (24, 58, 5, 3), (34, 80, 5, 5), (24, 58, 5, 3)]
    wls = [workload.molecule_like(nbf=a, naux=b, nbeta=c, ncwo=e, seed=80 + i, two_e_scale=0.2)
           for i, (a, b, c, e) in enumerate(shapes)]
    for wl in wls:
        wl.p.threshgorb = wl.p.threshgocc = 1e-5
        wl.p.threshen = 1e-6
    req = lambda wl, i, prec="fp64": Request(H=wl.H, b=wl.b, C=wl.C, p=copy.deepcopy(wl.p), gamma=wl.gamma,
                                             precision=prec, maxit=500, tag=i)
    with Server(max_inflight=1) as s:
        alone = [s.wait(s.submit(req(wl, i)), timeout=600) for i, wl in enumerate(wls)]
    mixed = workload.molecule_like(nbf=24, naux=40, nbeta=3, ncwo=3, seed=4)
    mixed.p.threshgorb, mixed.p.threshgocc, mixed.p.threshen = 1e-4, 1e-4, 1e-8
    with Server(max_inflight=2, continuous_slots=2) as s:
        tickets = [s.submit(req(wl, i)) for i, wl in enumerate(wls)]
        tm = s.submit(req(mixed, 99, "mixed_refined"))
        served = [s.wait(t, timeout=600) for t in tickets]
        rm = s.wait(tm, timeout=600)
    assert rm.error is None and rm.converged
    for a, g in zip(alone, served):
        assert a.error is None and g.error is None, (a.error, g.error)
        assert a.converged and g.converged
        assert g.E_elec == a.E_elec and g.iterations == a.iterations
        assert np.array_equal(g.n, a.n) and np.array_equal(g.C, a.C)
