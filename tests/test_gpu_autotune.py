"""GPU checks of the GEMM autotuner: the first FP64 Lagrangian of a new shape
tunes its GEMMs (three-index transforms and the Y product), and the chosen
configurations give the same result in every later call."""
import numpy as np
import pytest

import donof_b200 as d
from donof_b200 import _lib, workload

pytestmark = pytest.mark.gpu


def test_first_call_tunes_and_later_calls_repeat(cuda_ctx):
    lib = _lib.load()
    wl = workload.synthetic(nbf=72, naux=50, nbeta=6, ncwo=3, seed=11)
    p = wl.p
    bt = d.eris_to_gpu(wl.b, "fp64", cuda_ctx)
    before = lib.donof_autotune_entries()
    e1, h1 = d.compute_Lagrange2(wl.C, wl.n, wl.H, bt, wl.cj12, wl.ck12, p.nalpha, p.nbeta)
    after = lib.donof_autotune_entries()
    assert after >= before + 3
    e2, h2 = d.compute_Lagrange2(wl.C, wl.n, wl.H, bt, wl.cj12, wl.ck12, p.nalpha, p.nbeta)
    assert lib.donof_autotune_entries() == after
    assert np.array_equal(e1, e2) and np.array_equal(h1, h2)
    bt.free()
