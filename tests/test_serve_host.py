"""Host-side tests of the continuous-batching server: admission by memory budget
and slots, no starvation of a large job, and the submit/poll/wait plumbing with
a fake executor (no GPU)."""
import threading
import time

import numpy as np
import pytest

from donof_b200.param import Param
from donof_b200.serve import Admission, Request, Result, Server, footprint, percentiles


def test_admission_fits_budget_and_slots():
    a = Admission(budget_bytes=100, max_inflight=2)
    for t, nb in ((1, 60), (2, 30), (3, 30)):
        a.push(t, nb)
    assert [t for t, _ in a.take()] == [1, 2]      # third: no slot left
    a.release(60)
    assert [t for t, _ in a.take()] == [3]
    assert a.used == 60 and a.inflight == 2


def test_admission_first_fit_then_head_protected():
    a = Admission(budget_bytes=100, max_inflight=8, max_bypass=2)
    a.push(1, 90)
    assert [t for t, _ in a.take()] == [1]
    a.push(2, 50)                                    # head: does not fit beside job 1
    for t in (3, 4, 5):
        a.push(t, 5)
    started = [t for t, _ in a.take()]
    assert started == [3, 4]                         # two small jobs pass the head, then it is protected
    a.release(90)
    assert [t for t, _ in a.take()] == [2, 5]


def test_admission_rejects_oversize():
    a = Admission(budget_bytes=10)
    with pytest.raises(ValueError):
        a.push(1, 11)


def test_footprint_grows_with_precision_and_size():
    f64 = footprint(64, 128, 16, "fp64")
    mix = footprint(64, 128, 16, "mixed")
    assert mix > f64 > 8 * 64 * 64 * 128
    assert footprint(128, 128, 16, "fp64") > f64


def _req(nbf, tag):
    p = Param(nbf=nbf, nbfaux=8, nbeta=2, nalpha=2, ncwo=1)
    return Request(H=np.eye(nbf), b=np.zeros((nbf, nbf, 8)), C=np.eye(nbf), p=p, tag=tag)


def test_server_overlaps_and_returns_every_ticket():
    live, peak = [0], [0]
    lock = threading.Lock()

    def fake(req, device):
        with lock:
            live[0] += 1
            peak[0] = max(peak[0], live[0])
        time.sleep(0.05)
        with lock:
            live[0] -= 1
        return Result(ticket=-1, E_elec=float(req.p.nbf), converged=True)

    with Server(budget_bytes=10**12, max_inflight=3, executor=fake) as s:
        tickets = [s.submit(_req(8 + i, tag=i)) for i in range(7)]
        res = [s.wait(t, timeout=10) for t in tickets]
    assert [r.E_elec for r in res] == [8.0 + i for i in range(7)]
    assert [r.tag for r in res] == list(range(7))
    assert peak[0] == 3                                  # jobs ran side by side, never more than the slots
    assert all(r.latency >= 0.05 for r in res)
    q = percentiles([r.latency for r in res])
    assert q["p50"] <= q["p99"]


def test_server_reports_a_failing_job_and_goes_on():
    def fake(req, device):
        if req.tag == "bad":
            raise RuntimeError("boom")
        return Result(ticket=-1, E_elec=1.0)

    with Server(budget_bytes=10**12, executor=fake) as s:
        t1 = s.submit(_req(8, "bad"))
        t2 = s.submit(_req(8, "good"))
        r1, r2 = s.wait(t1, 5), s.wait(t2, 5)
    assert r1.error and "boom" in r1.error
    assert r2.error is None and r2.E_elec == 1.0


def test_cta_share_splits_the_sms_between_inflight_jobs():
    from donof_b200.serve import cta_share
    assert cta_share(1, 148) == 0            # one job: all SMs
    assert cta_share(8, 148) == 37           # about two jobs per SM
    assert cta_share(32, 148) == 16          # never fewer than 16 CTAs


def test_auto_precision_picks_mixed_for_large_transforms_only():
    from donof_b200.serve import resolve_precision, footprint
    assert resolve_precision("auto", 48, 40, 232) == "fp64"
    assert resolve_precision("auto", 202, 198, 974) == "mixed_refined"
    assert resolve_precision("fp64", 202, 198, 974) == "fp64"
    # the mixed footprint includes the bf16 split and, beyond the fused kernel's
    # shapes, the general pipeline's scratch
    assert footprint(202, 974, 198, "mixed_refined") > footprint(202, 974, 198, "fp64")


def test_take_group_collects_eligible_jobs_behind_an_eligible_head():
    a = Admission(budget_bytes=100, max_inflight=2)
    for t, nb in [(1, 10), (2, 30), (3, 10), (4, 10), (5, 10)]:
        a.push(t, nb)
    small = lambda t: t != 2                           # ticket 2 is not groupable
    g = a.take_group(small, max_group=3, scale=2.0)
    assert [t for t, _ in g] == [1, 3, 4]              # in arrival order, 2 left in the queue
    assert [nb for _, nb in g] == [20, 20, 20]         # each job's bytes times the scale
    assert a.inflight == 1 and a.used == 60
    assert [t for t, _ in a.queue] == [2, 5]
    assert a.take_group(small, max_group=3) == []      # head (2) not eligible: no group passes it
    assert [t for t, _ in a.take()] == [2]             # the single-job path takes the head
    a.release_group(60)
    assert a.inflight == 1 and a.used == 30
    assert a.take_group(small, max_group=3) == []      # one eligible job left: below min_group


def test_server_runs_small_fp64_jobs_as_groups_and_the_rest_alone():
    groups, singles = [], []

    def fake_group(reqs, device):
        groups.append([r.tag for r in reqs])
        time.sleep(0.05)
        return [Result(ticket=-1, E_elec=float(r.p.nbf), converged=True) for r in reqs]

    def fake(req, device):
        singles.append(req.tag)
        time.sleep(0.1)  # the other jobs queue up meanwhile
        return Result(ticket=-1, E_elec=float(req.p.nbf), converged=True)

    with Server(budget_bytes=10**12, max_inflight=1, executor=fake, group_max=4,
                group_executor=fake_group) as s:
        # the first job takes the only slot; the next five wait and then start as groups
        tickets = [s.submit(_req(8 + i, tag=i)) for i in range(6)]
        res = [s.wait(t, timeout=10) for t in tickets]
    assert [r.E_elec for r in res] == [8.0 + i for i in range(6)]
    assert [r.tag for r in res] == list(range(6))
    assert sum(len(g) for g in groups) + len(singles) == 6
    assert any(len(g) >= 2 for g in groups)
    assert all(len(g) <= 4 for g in groups)


def test_take_group_counts_a_passed_over_head_and_stops_at_max_bypass():
    a = Admission(budget_bytes=100, max_inflight=8, max_bypass=2)
    a.push(1, 40)                                      # eligible head that does not fit (2 x 40 > room)
    for t in range(2, 10):
        a.push(t, 5)
    a.used = 30                                        # 70 bytes free
    every = lambda t: True
    g1 = a.take_group(every, max_group=2)
    assert [t for t, _ in g1] == [2, 3]                # the head is passed over once
    g2 = a.take_group(every, max_group=2)
    assert [t for t, _ in g2] == [4, 5]                # twice
    assert a.take_group(every, max_group=2) == []      # max_bypass reached: the head waits for memory
    assert a.take() == []                              # and take() does not pass it either
    a.used = 0
    a.inflight = 0
    g = a.take_group(every, max_group=2)
    assert g[0][0] == 1                                # the head goes first once it fits
    assert a._head_bypassed == 0


def test_cancel_of_a_queued_job_returns_a_cancelled_result_and_frees_its_place():
    started = []
    gate = threading.Event()

    def fake(req, device):
        started.append(req.tag)
        gate.wait(5)
        return Result(ticket=-1, E_elec=1.0, converged=True)

    with Server(budget_bytes=10**12, max_inflight=1, executor=fake) as s:
        t1 = s.submit(_req(8, tag="running"))
        t2 = s.submit(_req(8, tag="queued"))
        t3 = s.submit(_req(8, tag="next"))
        assert s.cancel(t2) is True
        r2 = s.wait(t2, timeout=1)
        assert r2.error == "cancelled" and r2.tag == "queued"
        assert s.cancel(t1) is False                   # already running: not cancelled here
        gate.set()
        r1, r3 = s.wait(t1, timeout=10), s.wait(t3, timeout=10)
    assert r1.error is None and r3.error is None
    assert started == ["running", "next"]              # the cancelled job never ran


def test_server_refuses_a_job_larger_than_its_budget():
    with Server(budget_bytes=1000, max_inflight=1, executor=lambda r, d: Result(ticket=-1)) as s:
        with pytest.raises(ValueError, match="budget"):
            s.submit(_req(16, tag=0))


def test_a_failing_job_reports_its_error_and_the_server_goes_on():
    def fake(req, device):
        if req.tag == "bad":
            raise RuntimeError("b holds a NaN or an infinity")
        return Result(ticket=-1, E_elec=2.0, converged=True)

    with Server(budget_bytes=10**12, max_inflight=2, executor=fake) as s:
        tb, tg = s.submit(_req(8, tag="bad")), s.submit(_req(8, tag="good"))
        rb, rg = s.wait(tb, timeout=10), s.wait(tg, timeout=10)
    assert "NaN" in rb.error and rg.error is None and rg.E_elec == 2.0


def test_fp64_tensor_core_policy_and_footprint():
    from donof_b200.serve import FP64_TC_MIN_NBF, footprint, use_fp64_tc
    assert not use_fp64_tc(None, FP64_TC_MIN_NBF - 1) and use_fp64_tc(None, FP64_TC_MIN_NBF)
    assert use_fp64_tc(True, 24) and not use_fp64_tc(False, 512)
    # the digit slices: 7 bytes per element of b with rows padded to 16 bytes, plus the row scales
    extra = footprint(202, 974, 198, "fp64", True) - footprint(202, 974, 198, "fp64")
    assert extra == 7 * 202 * 208 * 974 + 8 * 202 * 974
