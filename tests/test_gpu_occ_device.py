"""The occupation solver on the GPU (donof_occ_cg_dev: occoptr's conjugate
gradient run by one CTA) against the library's host solver, which the oracle
pins (tests/test_occ_native.py): the energy and gradient of one evaluation for
every GNOF variant (ista 0-5), both occupation maps, closed and open shells and
a core-orbital case (<= 1e-12 relative), the minimisation reaching the same
minimum, and the energy loop with the occupation step on the device against
the loop with it on the host."""
import ctypes as ct

import numpy as np
import pytest
import torch

import donof_b200 as d
from donof_b200 import _lib, api, gnof, workload
from donof_b200.param import Param

pytestmark = pytest.mark.gpu

CASES = [dict(nbf=40, nbfaux=9, nbeta=4, nalpha=4, ncwo=3),
         dict(nbf=40, nbfaux=9, nbeta=4, nalpha=6, ncwo=3),
         dict(nbf=60, nbfaux=9, nbeta=5, nalpha=7, ncwo=4),
         dict(nbf=24, nbfaux=9, nbeta=5, nalpha=5, ncwo=-1),
         dict(nbf=50, nbfaux=9, nbeta=6, nalpha=6, ncwo=3, no1=2),
         dict(nbf=202, nbfaux=9, nbeta=33, nalpha=33, ncwo=5)]


def _jk(p, seed):
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((p.nbf5, p.nbf5))
    J = np.asfortranarray(np.abs(A @ A.T) / p.nbf5 + 0.01 * rng.standard_normal((p.nbf5, p.nbf5)))
    K = np.asfortranarray(0.3 * J + 0.01 * rng.standard_normal((p.nbf5, p.nbf5)))
    Hc = -np.sort(rng.uniform(0.5, 3.0, p.nbf5))[::-1]
    return J, K, Hc


def device_cg(ctx, p, J, K, Hc, gamma, tol, max_iter):
    prm = api._occ_params(p)
    tJ, tK = d.to_device(J), d.to_device(K)
    tH = torch.from_numpy(np.ascontiguousarray(Hc)).cuda()
    tg = torch.from_numpy(np.array(gamma, dtype=np.float64)).cuda()
    res = torch.zeros(3 + p.nv, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    ctx.check(ctx.lib.donof_occ_cg_dev(ctx.handle, ct.byref(prm), tJ.data_ptr(), tK.data_ptr(), tH.data_ptr(),
                                       tg.data_ptr(), float(tol), int(max_iter), res.data_ptr()))
    ctx.synchronize()
    r = res.cpu().numpy()
    return tg.cpu().numpy(), r[0], int(r[1]), bool(r[2]), r[3:]


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("ista", [0, 1, 2, 3, 4, 5])
@pytest.mark.parametrize("occ", ["Softmax", "Trigonometric"])
def test_one_evaluation_matches_the_host_layer(cuda_ctx, case, ista, occ):
    p = Param(ista=ista, occ_method=occ, **case)
    J, K, Hc = _jk(p, ista + 7 * len(occ))
    gamma = np.random.default_rng(ista).standard_normal(p.nv)
    # max_iter = 0: the solver evaluates at gamma and returns
    g_out, E, nit, _, grad = device_cg(cuda_ctx, p, J, K, Hc, gamma, 0.0, 0)
    E0, g0 = api.occ_energy(gamma, J, K, Hc, p)
    assert nit == 0 and np.array_equal(g_out, gamma)
    # the device sums in another order (and with fused multiply-adds): rounding only
    assert abs(E - E0) <= 1e-11 * max(1.0, abs(E0))
    assert np.max(np.abs(grad - g0)) <= 1e-11 * max(1.0, np.max(np.abs(g0)))


@pytest.mark.parametrize("occ", ["Softmax", "Trigonometric"])
@pytest.mark.parametrize("case", CASES[:3] + CASES[5:])
def test_minimisation_reaches_the_host_minimum(cuda_ctx, case, occ):
    p = Param(occ_method=occ, **case)
    J, K, Hc = _jk(p, 3)
    g0 = gnof.guess_gamma(p)
    # g_abstol 1e-8: on these random J/K the CG is slow near 1e-9, where the energy
    # differences of a line search reach the rounding of E
    x_h, E_h, nit_h, ok_h = api.occ_cg(g0, J, K, Hc, p, 1e-8, 2000)
    x_d, E_d, nit_d, ok_d, grad = device_cg(cuda_ctx, p, J, K, Hc, g0, 1e-8, 2000)
    # the iteration counts differ (a long CG path turns on rounding), the minimum does not
    assert ok_d and nit_d > 0 and np.max(np.abs(grad)) <= 1e-8, (ok_d, nit_d, np.max(np.abs(grad)), nit_h)
    _, g_chk = api.occ_energy(x_d, J, K, Hc, p)      # the returned gradient is the host's at gamma
    assert np.max(np.abs(g_chk - grad)) <= 1e-11
    if ok_h:
        # both stop at max|g| <= 1e-8 on an ill-conditioned surface: the energies agree
        # to what that leaves (second order in the gradient), the occupations closely
        assert abs(E_d - E_h) <= 1e-8 * max(1.0, abs(E_h))
        n_d, _ = gnof.occupations(x_d, p)
        n_h, _ = gnof.occupations(x_h, p)
        assert np.max(np.abs(n_d - n_h)) <= 1e-4
    # the same call gives the same result (fixed-order sums)
    x2, E2, nit2, _, _ = device_cg(cuda_ctx, p, J, K, Hc, g0, 1e-8, 2000)
    assert E2 == E_d and nit2 == nit_d and np.array_equal(x2, x_d)


@pytest.mark.parametrize("occ", ["Softmax", "Trigonometric"])
def test_energy_loop_with_the_device_occupation_step(cuda_ctx, occ):
    """donof_energy with occoptr's CG on the device against the host CG: the
    first orbital optimisation is the same, the first occupation step reaches
    the same minimum (in a different number of CG iterations: the path turns on
    rounding), and the converged energies agree to what the thresholds leave."""
    from donof_b200.optimize import energy
    wl = workload.molecule_like(nbf=48, naux=116, nbeta=6, ncwo=3, seed=12, occ_method=occ, two_e_scale=0.3)
    out = {}
    for dev in (False, True):
        p = workload.molecule_like(nbf=48, naux=116, nbeta=6, ncwo=3, seed=12, occ_method=occ, two_e_scale=0.3).p
        p.threshgorb, p.threshgocc, p.threshen = 1e-6, 1e-6, 1e-10
        p.occ_device = dev
        b = d.eris_to_gpu(wl.b, "fp64", cuda_ctx)
        out[dev] = energy(wl.H, b, p, wl.C, wl.gamma, maxit=1000)
        b.free()
    rh, rd = out[False], out[True]
    assert rh.converged and rd.converged
    h0, h1 = rh.history[0], rd.history[0]
    assert h0["nit_orb"] == h1["nit_orb"] and h1["E"] == h0["E"]
    assert abs(h1["norm_grad_occ"] - h0["norm_grad_occ"]) <= 1e-6
    assert abs(rd.E_elec - rh.E_elec) <= 1e-7
    assert np.max(np.abs(rd.n - rh.n)) <= 1e-5
