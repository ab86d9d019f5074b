"""The aux-index split of the RI hot path across ranks, on the CPU: two gloo
ranks (127.0.0.1) each hold a contiguous slice of b; the oracle's Lagrangian
and J/K terms of each slice, summed with shard.sum_over_ranks (a real gloo
all-reduce), equal the oracle's values for the whole tensor."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]

from donof_b200 import shard  # noqa: E402


def test_aux_slices_cover_the_range_contiguously_and_evenly():
    for naux, world in ((10, 3), (1024, 8), (7, 7), (974, 4), (5, 1)):
        sl = shard.aux_slices(naux, world)
        assert sl[0][0] == 0 and sl[-1][1] == naux
        assert all(a[1] == b[0] for a, b in zip(sl, sl[1:]))
        sizes = [l1 - l0 for l0, l1 in sl]
        assert max(sizes) - min(sizes) <= 1 and min(sizes) >= 1
    with pytest.raises(ValueError):
        shard.aux_slices(1, 2)


def test_local_slice_is_the_rank_block_in_julia_layout():
    b = np.asfortranarray(np.arange(3 * 3 * 7, dtype=np.float64).reshape(3, 3, 7, order="F"))
    parts = [shard.local_slice(b, r, 3) for r in range(3)]
    assert all(p.flags.f_contiguous for p in parts)
    assert np.array_equal(np.concatenate(parts, axis=2), b)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    sys.path[:0] = [str(ROOT), str(ROOT / "donof.jl_b200")]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    from donof_b200 import shard, workload
    from oracle import blas_mirror

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        wl = workload.synthetic(nbf=20, naux=37, nbeta=3, ncwo=3, seed=13)
        p = wl.p
        b_r = shard.local_slice(wl.b, rank, world)
        elag_r, Hmat = blas_mirror.lagrange2(wl.C, wl.n, wl.H, b_r, wl.cj12, wl.ck12, p.nalpha, p.nbeta)
        own = np.zeros_like(elag_r)
        own[:, :p.nbf5] = Hmat * wl.n[None, :]
        G = torch.from_numpy(np.ascontiguousarray(elag_r - own))   # this slice's two-electron terms
        shard.sum_over_ranks(G)
        J, K, Hc = (torch.from_numpy(np.ascontiguousarray(x)) for x in blas_mirror.jkh_mo(wl.C, wl.H, b_r, p.nbf5))
        shard.sum_over_ranks(J)
        shard.sum_over_ranks(K)
        out.put((rank, (G.numpy() + own), J.numpy(), K.numpy(), Hc.numpy()))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_gloo_ranks_sum_their_slices_to_the_whole_tensor_result():
    from donof_b200 import workload
    from oracle import native

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    res = sorted((q.get(timeout=100) for _ in procs), key=lambda r: r[0])
    for pr in procs:
        pr.join(timeout=30)
        assert pr.exitcode == 0
    wl = workload.synthetic(nbf=20, naux=37, nbeta=3, ncwo=3, seed=13)
    p = wl.p
    elag, _ = native.lagrange2(wl.C, wl.n, wl.H, wl.b, wl.cj12, wl.ck12, p.nalpha, p.nbeta)
    J, K, Hc = native.jkh_mo(wl.C, wl.H, wl.b, p.nbf5)
    for rank, el, Jr, Kr, Hcr in res:
        assert np.max(np.abs(el - elag)) <= 1e-12 * np.max(np.abs(elag))
        assert np.max(np.abs(Jr - J)) <= 1e-12 * np.max(np.abs(J))
        assert np.max(np.abs(Kr - K)) <= 1e-12 * np.max(np.abs(K))
        assert np.max(np.abs(Hcr - Hc)) <= 1e-13
