"""The RI hot path with the aux index split across GPUs (one process per GPU).

b[m, n, l] is cut into contiguous slices of l, one per rank; every elag,
J_MO and K_MO term of the reference (src/utils.jl:39-55,
src/integrals.jl:162-166) is a sum over l, so a rank computes its slice's
part and one all-reduce per call sums the parts:

  compute_Lagrange2   Y_r = sum_{l in slice r} tmp_l W_l  (nbf x nbf5 FP64,
                      donof_lagrange2_partial_dev); all-reduce Y; elag, H_mat,
                      E_elec from the summed Y (donof_lagrange2_finish_dev)
  JKH_MO              J_r, K_r of the slice (donof_jkh_mo_dev); all-reduce J, K

The orbitals, occupations, H and the optimiser state are the same on every
rank.  The collective is torch.distributed's all_reduce (NCCL between GPUs);
the partial and finishing steps are the library's kernels.
"""
from __future__ import annotations

from typing import Callable, List, Optional, Tuple

import numpy as np


def aux_slices(naux: int, world: int) -> List[Tuple[int, int]]:
    """Contiguous [l0, l1) slices of the aux index, one per rank, sizes within one."""
    if world < 1 or naux < world:
        raise ValueError(f"cannot split {naux} aux indices over {world} ranks")
    base, extra = divmod(naux, world)
    out, l0 = [], 0
    for r in range(world):
        l1 = l0 + base + (1 if r < extra else 0)
        out.append((l0, l1))
        l0 = l1
    return out


def local_slice(b, rank: int, world: int):
    """This rank's slice b[:, :, l0:l1] (Julia layout, Fortran order)."""
    l0, l1 = aux_slices(b.shape[2], world)[rank]
    return np.asfortranarray(b[:, :, l0:l1])


def sum_over_ranks(x, group=None, all_reduce: Optional[Callable] = None):
    """All-reduce (sum) of a tensor in place; all_reduce(x, group) may be given
    (a test's stand-in), else torch.distributed's; a single rank is a no-op."""
    if all_reduce is not None:
        all_reduce(x, group)
        return x
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(x, op=dist.ReduceOp.SUM, group=group)
    return x


def compute_Lagrange2(C, n, H, b_slice, cj12, ck12, nalpha: int, nbeta: int, group=None,
                      all_reduce: Optional[Callable] = None):
    """compute_Lagrange2 of the whole tensor from this rank's slice (a BTensor
    holding b[:, :, l0:l1]); device arrays in and out (torch CUDA tensors in
    the column-major layout of ``api.to_device``).  Returns (elag, H_mat, E)."""
    import torch

    from . import api

    ctx = b_slice.ctx
    nbf, nbf5 = b_slice.nbf, int(n.shape[0])
    Y = torch.empty((nbf5, nbf), dtype=torch.float64, device=C.device)
    elag = torch.empty((nbf, nbf), dtype=torch.float64, device=C.device)
    Hmat = torch.empty((nbf5, nbf), dtype=torch.float64, device=C.device)
    E = torch.empty(1, dtype=torch.float64, device=C.device)
    ctx.check(ctx.lib.donof_lagrange2_partial_dev(b_slice.handle, api._ptr(C), api._ptr(n), api._ptr(cj12),
                                                  api._ptr(ck12), nbf5, int(nalpha), int(nbeta), api._ptr(Y)))
    ctx.synchronize()  # the collective runs on torch's stream
    sum_over_ranks(Y, group, all_reduce)
    torch.cuda.current_stream(C.device).synchronize()
    ctx.check(ctx.lib.donof_lagrange2_finish_dev(b_slice.handle, api._ptr(C), api._ptr(n), api._ptr(H), nbf5,
                                                 api._ptr(Y), api._ptr(elag), api._ptr(Hmat), api._ptr(E)))
    ctx.synchronize()
    return elag, Hmat, E


def JKH_MO(C, H, b_slice, nbf5: int, group=None, all_reduce: Optional[Callable] = None):
    """J_MO, K_MO (summed over the ranks' slices) and H_core, device arrays."""
    import torch

    from . import api

    ctx = b_slice.ctx
    J = torch.empty((nbf5, nbf5), dtype=torch.float64, device=C.device)
    K = torch.empty((nbf5, nbf5), dtype=torch.float64, device=C.device)
    Hc = torch.empty(nbf5, dtype=torch.float64, device=C.device)
    api.JKH_MO_dev(C, H, b_slice, nbf5, J, K, Hc)
    ctx.synchronize()
    sum_over_ranks(J, group, all_reduce)
    sum_over_ranks(K, group, all_reduce)
    return J, K, Hc
