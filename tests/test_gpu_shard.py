"""The aux-index split on the GPU: the library's partial Lagrangians of the
slices of b, summed and finished, equal the Lagrangian of the whole tensor
(<= 1e-10 relative), and so do the summed J_MO / K_MO.  The slices run one
after the other on one device (no kernel waits on another rank), with the sum
taken on the device as the all-reduce between GPUs would take it."""
import numpy as np
import pytest
import torch

import donof_b200 as d
from donof_b200 import shard, workload

pytestmark = pytest.mark.gpu
TOL = 1e-10


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("kw,world", [
    (dict(nbf=48, naux=96, nbeta=4, ncwo=3), 2),
    (dict(nbf=130, naux=70, nbeta=8, ncwo=3), 3),
    (dict(nbf=256, naux=1024, nbeta=16, ncwo=3), 4),
])
def test_slices_sum_to_the_whole_tensor_lagrangian(cuda_ctx, kw, world):
    wl = workload.synthetic(**kw, seed=21)
    p = wl.p
    full = d.eris_to_gpu(wl.b, "fp64", cuda_ctx)
    elag_ref, Hmat_ref, E_ref = d.compute_Lagrange2(wl.C, wl.n, wl.H, full, wl.cj12, wl.ck12, p.nalpha, p.nbeta,
                                                    return_energy=True)
    J_ref, K_ref, Hc_ref = d.JKH_MO(wl.C, wl.H, full, p.nbf, p.nbf5, p.nbfaux)
    full.free()
    C, n, H, cj, ck = (d.to_device(x) for x in (wl.C, wl.n, wl.H, wl.cj12, wl.ck12))
    Ysum = torch.zeros((p.nbf5, p.nbf), dtype=torch.float64, device="cuda")
    Jsum = torch.zeros((p.nbf5, p.nbf5), dtype=torch.float64, device="cuda")
    Ksum = torch.zeros_like(Jsum)
    slices = []
    for r in range(world):
        bt = d.eris_to_gpu(shard.local_slice(wl.b, r, world), "fp64", cuda_ctx)
        slices.append(bt)
        Y = torch.empty_like(Ysum)
        cuda_ctx.check(cuda_ctx.lib.donof_lagrange2_partial_dev(bt.handle, C.data_ptr(), n.data_ptr(), cj.data_ptr(),
                                                                ck.data_ptr(), p.nbf5, p.nalpha, p.nbeta,
                                                                Y.data_ptr()))
        J = torch.empty_like(Jsum)
        K = torch.empty_like(Jsum)
        Hc = torch.empty(p.nbf5, dtype=torch.float64, device="cuda")
        d.api.JKH_MO_dev(C, H, bt, p.nbf5, J, K, Hc)
        cuda_ctx.synchronize()
        Ysum += Y
        Jsum += J
        Ksum += K
    torch.cuda.synchronize()
    elag = torch.empty((p.nbf, p.nbf), dtype=torch.float64, device="cuda")
    Hmat = torch.empty((p.nbf5, p.nbf), dtype=torch.float64, device="cuda")
    E = torch.empty(1, dtype=torch.float64, device="cuda")
    cuda_ctx.check(cuda_ctx.lib.donof_lagrange2_finish_dev(slices[0].handle, C.data_ptr(), n.data_ptr(), H.data_ptr(),
                                                           p.nbf5, Ysum.data_ptr(), elag.data_ptr(), Hmat.data_ptr(),
                                                           E.data_ptr()))
    cuda_ctx.synchronize()
    assert rel(d.from_device(elag), elag_ref) <= TOL
    assert rel(d.from_device(Hmat), Hmat_ref) <= TOL
    assert abs(float(E) - E_ref) <= TOL * abs(E_ref)
    assert rel(d.from_device(Jsum), J_ref) <= TOL and rel(d.from_device(Ksum), K_ref) <= TOL
    assert rel(d.from_device(Hc), Hc_ref) <= TOL
    for bt in slices:
        bt.free()


def test_single_rank_sharded_call_is_the_plain_call(cuda_ctx):
    """shard.compute_Lagrange2 / shard.JKH_MO with one rank (no process group)."""
    wl = workload.synthetic(nbf=64, naux=80, nbeta=4, ncwo=3, seed=22)
    p = wl.p
    bt = d.eris_to_gpu(wl.b, "fp64", cuda_ctx)
    elag_ref, Hmat_ref, E_ref = d.compute_Lagrange2(wl.C, wl.n, wl.H, bt, wl.cj12, wl.ck12, p.nalpha, p.nbeta,
                                                    return_energy=True)
    C, n, H, cj, ck = (d.to_device(x) for x in (wl.C, wl.n, wl.H, wl.cj12, wl.ck12))
    torch.cuda.synchronize()
    elag, Hmat, E = shard.compute_Lagrange2(C, n, H, bt, cj, ck, p.nalpha, p.nbeta)
    assert rel(d.from_device(elag), elag_ref) <= TOL and abs(float(E) - E_ref) <= TOL * abs(E_ref)
    J, K, Hc = shard.JKH_MO(C, H, bt, p.nbf5)
    J_ref, K_ref, _ = d.JKH_MO(wl.C, wl.H, bt, p.nbf, p.nbf5, p.nbfaux)
    assert rel(d.from_device(J), J_ref) <= TOL and rel(d.from_device(K), K_ref) <= TOL
    bt.free()
