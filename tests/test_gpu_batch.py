"""Grouped multi-job path (donof_batch_*): several molecules of different sizes
advance together, one grouped launch per stage of a gradient step.

Checks, through the C ABI:
  * the grouped Lagrangian of every job against the CPU oracle (<= 1e-10) and
    against the single-job FP64 path;
  * the grouped optimiser loop against each job optimised alone with
    donof_orbopt_dev: bit-for-bit the same (every product sums in the same
    order, the Lagrangian GEMM with the same split of its K range), so the
    same iteration counts, stopping decisions, step back-off, energies and
    orbitals; and against the oracle's loop;
  * a job's result is bit-for-bit the same alone (a batch of one) and in the
    mix, whatever else the batch holds;
  * the batched energy loop against donof_energy for each job alone (the same
    alternation, bit-for-bit) and against the oracle's energy loop.
"""
import numpy as np
import pytest

from oracle import gnof as ognof
from oracle import native, orbital

import donof_b200 as d

from test_gpu_parity import case, rel

pytestmark = pytest.mark.gpu
TOL = 1e-10

# water-cluster and alkane surrogates of different sizes, an open shell, odd sizes
SHAPES = [
    dict(nbf=24, naux=116, nbeta=5, ncwo=3, seed=1),
    dict(nbf=48, naux=232, nbeta=10, ncwo=1, seed=2),
    dict(nbf=13, naux=29, nbeta=3, ncwo=3, seed=3),
    dict(nbf=20, naux=17, nbeta=3, ncwo=3, nalpha=5, seed=4),
    dict(nbf=96, naux=120, nbeta=6, ncwo=3, seed=5),
    dict(nbf=72, naux=348, nbeta=15, ncwo=3, seed=6),
    dict(nbf=128, naux=200, nbeta=16, ncwo=3, seed=7),      # nbf5 = 64: the fused mixed kernel's largest
    dict(nbf=40, naux=64, nbeta=5, ncwo=2, seed=8),         # odd nbf5 = 15 with even nbf
]


def device_inputs(cases):
    import torch  # noqa: F401

    out = []
    for p, b, C, H, n, cj, ck in cases:
        out.append(dict(p=p, b=b, C=C, H=H, n=n, cj=cj, ck=ck, tC=d.to_device(C), tH=d.to_device(H),
                        tn=d.to_device(n), tcj=d.to_device(cj), tck=d.to_device(ck)))
    return out


def make_batch(ctx, inputs):
    bts = [d.eris_to_gpu(x["b"], "fp64", ctx) for x in inputs]
    return d.Batch(bts, [x["p"] for x in inputs], ctx), bts


def test_batch_lagrange2_matches_oracle_and_single_job(cuda_ctx):
    import torch

    inputs = device_inputs([case(**kw) for kw in SHAPES])
    batch, bts = make_batch(cuda_ctx, inputs)
    elag = [torch.zeros(x["p"].nbf, x["p"].nbf, dtype=torch.float64, device="cuda") for x in inputs]
    hmat = [torch.zeros(x["p"].nbf5, x["p"].nbf, dtype=torch.float64, device="cuda") for x in inputs]
    E = batch.lagrange2([x["tn"] for x in inputs], [x["tcj"] for x in inputs], [x["tck"] for x in inputs],
                        [x["tH"] for x in inputs], [x["tC"] for x in inputs], elag, hmat)
    torch.cuda.synchronize()
    for j, x in enumerate(inputs):
        p = x["p"]
        e_ref, h_ref = native.lagrange2(x["C"], x["n"], x["H"], x["b"], x["cj"], x["ck"], p.nalpha, p.nbeta)
        e, h = d.from_device(elag[j]), d.from_device(hmat[j])
        assert rel(h, h_ref) <= TOL, j
        assert rel(e, e_ref) <= TOL, j
        assert np.all(e[:, p.nbf5:] == 0.0)
        E_ref = orbital.e_elec(h_ref, x["n"], e_ref, p.nbf5)
        assert abs(E[j] - E_ref) <= TOL * max(1.0, abs(E_ref)), j
        # the single-job FP64 path at the same C
        e1, h1, E1 = d.compute_Lagrange2(x["C"], x["n"], x["H"], bts[j], x["cj"], x["ck"], p.nalpha, p.nbeta,
                                         return_energy=True)
        assert np.array_equal(h, h1), j
        assert np.array_equal(e, e1), j
        assert E[j] == E1, j
    batch.free()
    for b in bts:
        b.free()


def run_alone(ctx, x, method, alpha, maxloop, thresh):
    bt = d.eris_to_gpu(x["b"], "fp64", ctx)
    C = x["tC"].clone()
    E, nit, ok, a, ml = d.orbopt_dev(method, x["tn"], x["tcj"], x["tck"], x["tH"], C, bt, x["p"], alpha, maxloop,
                                     thresh)
    bt.free()
    return E, nit, ok, a, ml, d.from_device(C)


@pytest.mark.parametrize("method", ["ADAM", "Demon"])
def test_batch_orbopt_matches_each_job_alone(cuda_ctx, method):
    inputs = device_inputs([case(**kw) for kw in SHAPES])
    batch, bts = make_batch(cuda_ctx, inputs)
    k = len(inputs)
    # different step sizes, loop lengths and thresholds per job: the jobs stop at
    # different iterations, some on the gradient rule, some on maxloop
    alpha = [0.01, 0.02, 0.01, 0.005, 0.01, 0.02, 0.01, 0.02]
    maxloop = [6, 9, 3, 12, 5, 8, 7, 4]
    thresh = [1e-4, 1e-1, 1e-4, 1.0, 1e-4, 1e-4, 1e-4, 1e-4]
    assert len(alpha) == k
    Cs = [x["tC"].clone() for x in inputs]
    res = batch.orbopt(method, [x["tn"] for x in inputs], [x["tcj"] for x in inputs], [x["tck"] for x in inputs],
                       [x["tH"] for x in inputs], Cs, alpha, maxloop, thresh)
    for j, x in enumerate(inputs):
        E0, nit0, ok0, a0, ml0, C0 = run_alone(cuda_ctx, x, method, alpha[j], maxloop[j], thresh[j])
        assert res[j] == (E0, nit0, ok0, a0, ml0), (j, res[j], (E0, nit0, ok0, a0, ml0))
        assert np.array_equal(d.from_device(Cs[j]), C0), j
    batch.free()
    for b in bts:
        b.free()


def test_batch_orbopt_matches_oracle_loop(cuda_ctx):
    kws = [SHAPES[0], SHAPES[2], dict(nbf=48, naux=60, nbeta=4, ncwo=3, seed=4)]
    inputs = device_inputs([case(**kw) for kw in kws])
    batch, bts = make_batch(cuda_ctx, inputs)
    Cs = [x["tC"].clone() for x in inputs]
    res = batch.orbopt("YOGI", [x["tn"] for x in inputs], [x["tcj"] for x in inputs], [x["tck"] for x in inputs],
                       [x["tH"] for x in inputs], Cs, [0.01] * 3, [6] * 3, [1e-4] * 3)
    for j, x in enumerate(inputs):
        p = x["p"]
        s = ognof.Sizes(nbf=p.nbf, nbeta=p.nbeta, nalpha=p.nalpha, ncwo=p.ncwo, naux=p.nbfaux)
        E0, C0, nit0, ok0, a0, ml0 = orbital.orbopt("YOGI", x["n"], x["cj"], x["ck"], x["C"], x["H"], x["b"], s,
                                                    0.01, 6, 1e-4)
        E, nit, ok, a, ml = res[j]
        assert (nit, ok, a, ml) == (nit0, ok0, a0, ml0), j
        assert abs(E - E0) <= TOL * max(1.0, abs(E0)), j
        assert rel(d.from_device(Cs[j]), C0) <= 1e-9, j
    batch.free()
    for b in bts:
        b.free()


def test_batch_result_same_alone_and_in_the_mix(cuda_ctx):
    inputs = device_inputs([case(**kw) for kw in SHAPES])
    target = 4  # nbf 96
    args = lambda xs: ([x["tn"] for x in xs], [x["tcj"] for x in xs], [x["tck"] for x in xs], [x["tH"] for x in xs])
    one, bt1 = make_batch(cuda_ctx, [inputs[target]])
    C1 = [inputs[target]["tC"].clone()]
    r1 = one.orbopt("ADAM", *args([inputs[target]]), C1, [0.01], [7], [1e-4])
    mix, btm = make_batch(cuda_ctx, inputs)
    Cm = [x["tC"].clone() for x in inputs]
    rm = mix.orbopt("ADAM", *args(inputs), Cm, [0.01] * len(inputs), [7] * len(inputs), [1e-4] * len(inputs))
    assert r1[0] == rm[target]
    assert np.array_equal(d.from_device(C1[0]), d.from_device(Cm[target]))
    # a second call of the same batch (graph replayed) gives the same again
    Cm2 = [x["tC"].clone() for x in inputs]
    rm2 = mix.orbopt("ADAM", *args(inputs), Cm2, [0.01] * len(inputs), [7] * len(inputs), [1e-4] * len(inputs))
    assert rm2 == rm
    assert all(np.array_equal(d.from_device(a), d.from_device(b)) for a, b in zip(Cm, Cm2))
    for o in (one, mix):
        o.free()
    for b in bt1 + btm:
        b.free()


def test_batch_energy_matches_each_job_alone(cuda_ctx):
    """donof_batch_energy: DoNOF.energy's alternation for several molecules, the
    orbital optimisation of all of them grouped per outer iteration.  Each job
    takes exactly the steps donof_energy takes for it alone (same iterations,
    bit-for-bit the same energy, orbitals and occupations), and a job that
    converges early leaves the later grouped calls."""
    from donof_b200 import workload
    from oracle import driver

    shapes = [dict(nbf=24, naux=96, nbeta=5, ncwo=3, seed=3), dict(nbf=40, naux=80, nbeta=4, ncwo=3, seed=4),
              dict(nbf=20, naux=30, nbeta=3, ncwo=3, seed=2), dict(nbf=48, naux=96, nbeta=4, ncwo=3, seed=5)]
    wls = [workload.molecule_like(**kw) for kw in shapes]
    for wl in wls:
        wl.p.threshgorb, wl.p.threshgocc, wl.p.threshen = 1e-5, 1e-5, 1e-9
    g0 = [ognof.guess_gamma_softmax(wl.p.nbeta, wl.p.ncwo) for wl in wls]
    bts = [d.eris_to_gpu(wl.b, "fp64", cuda_ctx) for wl in wls]
    batch = d.Batch(bts, [wl.p for wl in wls], cuda_ctx)
    res = batch.energy([wl.H for wl in wls], [wl.C for wl in wls], g0, maxit=1000)
    its = []
    for j, (kw, wl) in enumerate(zip(shapes, wls)):
        C, gamma, n, r = res[j]
        assert r["converged"], j
        p = workload.molecule_like(**kw).p
        p.threshgorb, p.threshgocc, p.threshen = 1e-5, 1e-5, 1e-9
        C1, g1, n1, _, r1, _ = d.api.energy_loop(wl.H, bts[j], p, wl.C, g0[j], maxit=1000)
        assert r == r1, (j, r, r1)
        assert np.array_equal(C, C1) and np.array_equal(gamma, g1) and np.array_equal(n, n1), j
        its.append(r["iterations"])
    assert len(set(its)) > 1, "the jobs should need different numbers of outer iterations"
    # the smallest case against the oracle's energy loop
    s = ognof.Sizes(nbf=20, nbeta=3, nalpha=3, ncwo=3, naux=30)
    E0, _, _, _, conv0 = driver.energy(wls[2].H, wls[2].b, s, wls[2].C, g0[2], threshgorb=1e-5, threshgocc=1e-5,
                                       threshen=1e-9, maxit=1000)
    assert conv0 and abs(res[2][3]["E_elec"] - E0) <= 1e-7
    batch.free()
    for b in bts:
        b.free()


def test_batch_orbopt_leaves_out_jobs_with_maxloop_zero(cuda_ctx):
    inputs = device_inputs([case(**kw) for kw in SHAPES[:3]])
    batch, bts = make_batch(cuda_ctx, inputs)
    Cs = [x["tC"].clone() for x in inputs]
    res = batch.orbopt("ADAM", [x["tn"] for x in inputs], [x["tcj"] for x in inputs], [x["tck"] for x in inputs],
                       [x["tH"] for x in inputs], Cs, [0.01, 0.01, 0.02], [5, 0, 4], [1e-4] * 3)
    assert res[1][1] == 0 and res[1][3:] == (0.01, 0)  # untouched
    assert np.array_equal(d.from_device(Cs[1]), inputs[1]["C"])
    for j in (0, 2):
        E0, nit0, ok0, a0, ml0, C0 = run_alone(cuda_ctx, inputs[j], "ADAM", [0.01, 0.01, 0.02][j], [5, 0, 4][j], 1e-4)
        assert res[j] == (E0, nit0, ok0, a0, ml0), j
    batch.free()
    for b in bts:
        b.free()


def test_batch_energy_variants_match_each_job_alone(cuda_ctx):
    """The batched energy loop for trigonometric occupations, an open shell and
    another GNOF variant (ista 1), with the ADABelief orbital optimiser: every
    job bit-for-bit what donof_energy gives it alone."""
    import copy

    from donof_b200 import Param, workload
    from donof_b200.gnof import guess_gamma

    def job(kw, seed, **over):
        wl = workload.molecule_like(**kw, seed=seed, two_e_scale=0.2)
        p = Param(nbf=kw["nbf"], nbfaux=kw["naux"], nbeta=kw["nbeta"], nalpha=over.pop("nalpha", kw["nbeta"]),
                  ncwo=kw["ncwo"], **over)
        p.orb_method = "ADABelief"
        p.threshgorb = p.threshgocc = 1e-5
        p.threshen = 1e-9
        return wl, p, guess_gamma(p)

    jobs = [job(dict(nbf=28, naux=60, nbeta=4, ncwo=3), 11, occ_method="Trigonometric"),
            job(dict(nbf=30, naux=64, nbeta=4, ncwo=3), 12, nalpha=6),
            job(dict(nbf=24, naux=50, nbeta=3, ncwo=3), 13, ista=1)]
    bts = [d.eris_to_gpu(wl.b, "fp64", cuda_ctx) for wl, _, _ in jobs]
    batch = d.Batch(bts, [copy.deepcopy(p) for _, p, _ in jobs], cuda_ctx)
    res = batch.energy([wl.H for wl, _, _ in jobs], [wl.C for wl, _, _ in jobs], [g for _, _, g in jobs], maxit=500)
    for j, ((wl, p, g), bt) in enumerate(zip(jobs, bts)):
        C, gamma, n, r = res[j]
        C1, g1, n1, _, r1, _ = d.api.energy_loop(wl.H, bt, copy.deepcopy(p), wl.C, g, maxit=500)
        assert r == r1, (j, r, r1)
        assert np.array_equal(C, C1) and np.array_equal(gamma, g1) and np.array_equal(n, n1), j
    batch.free()
    for b in bts:
        b.free()


MIXED_TOL = 2e-4  # the mixed form's bound on elag (max-norm relative; tests/test_gpu_mixed.py)


def test_mixed_batch_lagrangian_matches_each_job_and_the_oracle(cuda_ctx):
    """donof_batch_set_precision(MIXED): the fused tcgen05 kernel of every job in
    one grouped launch, each job on its own CTA range, then the grouped FP64
    tail.  Against the single-job mixed Lagrangian (the same products, Y
    partials summed over other CTA ranges: FP32 rounding apart) and against the
    FP64 oracle (the mixed form's tolerance)."""
    import torch

    inputs = device_inputs([case(**kw) for kw in SHAPES])
    bts = [d.eris_to_gpu(x["b"], "mixed", cuda_ctx) for x in inputs]
    batch = d.Batch(bts, [x["p"] for x in inputs], cuda_ctx)
    batch.set_precision("mixed")
    elag = [torch.zeros(x["p"].nbf, x["p"].nbf, dtype=torch.float64, device="cuda") for x in inputs]
    hmat = [torch.zeros(x["p"].nbf5, x["p"].nbf, dtype=torch.float64, device="cuda") for x in inputs]
    E = batch.lagrange2([x["tn"] for x in inputs], [x["tcj"] for x in inputs], [x["tck"] for x in inputs],
                        [x["tH"] for x in inputs], [x["tC"] for x in inputs], elag, hmat)
    torch.cuda.synchronize()
    for j, x in enumerate(inputs):
        p = x["p"]
        e_ref, h_ref = native.lagrange2(x["C"], x["n"], x["H"], x["b"], x["cj"], x["ck"], p.nalpha, p.nbeta)
        e, h = d.from_device(elag[j]), d.from_device(hmat[j])
        assert rel(h, h_ref) <= TOL, j          # H_mat stays FP64
        assert rel(e, e_ref) <= MIXED_TOL, j
        assert np.all(e[:, p.nbf5:] == 0.0)
        bts[j].set_precision("mixed")
        e1, h1, E1 = d.compute_Lagrange2(x["C"], x["n"], x["H"], bts[j], x["cj"], x["ck"], p.nalpha, p.nbeta,
                                         return_energy=True)
        assert rel(e, e1) <= 1e-5, j
        # energies: the mixed form's bound (1e-5 relative, as tests/test_gpu_mixed.py states)
        assert abs(E[j] - E1) <= 1e-5 * max(1.0, abs(E1)), j
        E_ref = orbital.e_elec(h_ref, x["n"], e_ref, p.nbf5)
        assert abs(E[j] - E_ref) <= 1e-5 * max(1.0, abs(E_ref)), j
    # back to FP64: the grouped FP64 path again, bit-for-bit the single-job FP64 result
    batch.set_precision("fp64")
    E64 = batch.lagrange2([x["tn"] for x in inputs], [x["tcj"] for x in inputs], [x["tck"] for x in inputs],
                          [x["tH"] for x in inputs], [x["tC"] for x in inputs], elag, hmat)
    for j, x in enumerate(inputs):
        p = x["p"]
        bts[j].set_precision("fp64")
        _, _, E1 = d.compute_Lagrange2(x["C"], x["n"], x["H"], bts[j], x["cj"], x["ck"], p.nalpha, p.nbeta,
                                       return_energy=True)
        assert E64[j] == E1, j
    batch.free()


def test_mixed_batch_orbital_optimiser_runs_every_job(cuda_ctx):
    """The grouped optimiser loop on the mixed Lagrangian: every job's energy
    within the mixed form's rounding of the FP64 batch's, and the same stopping
    behaviour (iterations within a few steps)."""
    import copy

    import torch

    inputs = device_inputs([case(**kw) for kw in SHAPES[:4]])
    bts = [d.eris_to_gpu(x["b"], "mixed", cuda_ctx) for x in inputs]
    out = {}
    for prec in ("fp64", "mixed"):
        batch = d.Batch(bts, [x["p"] for x in inputs], cuda_ctx)
        batch.set_precision(prec)
        Cs = [x["tC"].clone() for x in inputs]
        res = batch.orbopt("ADAM", [x["tn"] for x in inputs], [x["tcj"] for x in inputs],
                           [x["tck"] for x in inputs], [x["tH"] for x in inputs], Cs,
                           [0.01] * len(inputs), [20] * len(inputs), [1e-12] * len(inputs))
        torch.cuda.synchronize()
        out[prec] = res
        batch.free()
    for j in range(len(inputs)):
        E64, nit64 = out["fp64"][j][0], out["fp64"][j][1]
        Em, nitm = out["mixed"][j][0], out["mixed"][j][1]
        assert nitm > 0 and np.isfinite(Em)
        assert abs(Em - E64) <= 1e-4 * max(1.0, abs(E64)), (j, Em, E64)
