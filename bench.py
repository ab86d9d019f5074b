#!/usr/bin/env python
"""Benchmark of the GNOF orbital-gradient step (the per-iteration RI hot path).

One step = one iteration of the orbital optimiser loop of DoNOF.jl
(src/minimization.jl:387-422): AMSGrad-style update of the rotation y,
C <- C exp(Y(y)), compute_Lagrange2 (three-index transform + Lagrangian),
computeE_elec and the packed orbital gradient.

Workload (synthetic; the reference publishes no data set and no basis data
or integral engine exists here): nbf = 256, naux = 1024, nbf5 = 64
(ndoc = 16, ncwo = 3), b ~ N(0, 1/sqrt(naux)) symmetrised, C = Q of a seeded
QR, softmax occupations from N(0,1) logits, GNOF coefficients.  b (512 MiB
FP64) exceeds the 126 MB L2, so no flush is needed between steps.

  value   device-resident loop (donof_orbopt_dev, inputs in HBM)
  e2e     the reference-facing host-buffer calls per step (donof_rotate +
          donof_lagrange2 with host arrays, optimiser update on the host),
          as DoNOF.jl's loop drives its GPU plugin
          (e2e.latency_ms: p50/p99 of the per-step times of that loop)
  energies  converged GNOF energies/s of the FP64 form and of the mixed form
          with closing FP64 iterations, from the same start, on a molecule-
          shaped surrogate (nbf = 96, naux = 384), with |dE| between them
  serving  converged energies/s of a seeded Poisson stream of jobs of different
          sizes, served with continuous batching (and with small FP64 jobs
          started as grouped batches), against the plain FP64 form serving the
          same stream one job at a time; p50/p99 latency; |dE|
  batched  job orbital-gradient steps/s of 64 uneven water-cluster surrogates
          advanced together (one grouped launch per stage of a step, the loop as
          one captured graph) against the same jobs one after the other
  batched_energies  converged energies/s of 16 molecule surrogates through the
          batched energy loop against donof_energy per job (|dE| = 0: the
          grouped path is bit-for-bit the single-job one)
  --impl reference   the CPU restatement of the reference path on the same
          workload: the reference contraction order as threaded FP64 BLAS GEMMs
          on all host threads (oracle/blas_mirror.py), with the scalar C/OpenMP
          oracle beside it

Multi-GPU: the optimiser loop of one job does not shard without a collective
per step; --gpus N runs N independent replicas (one job per GPU, weak scaling).
"""
from __future__ import annotations

import argparse
import ctypes as ct
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path[:0] = [str(ROOT), str(ROOT / "donof.jl_b200")]

METRIC = "GNOF orbital-gradient steps/s"
UNIT = "steps/s"
WORKLOAD = dict(nbf=256, naux=1024, nbeta=16, ncwo=3)
SEED = 1234


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--method", default="ADAM")
    ap.add_argument("--no-fp64-tc", action="store_true",
                    help="FP64 form with its first contraction on the DMMA GEMM instead of the tensor cores "
                         "(int8 digit slices, exact integer products)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-energies", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--profile-case", nargs="?", const="synthetic256",
                    choices=["synthetic256", "octane600", "batch64", "batch8", "ints3c", "pipeline"],
                    help="run the mixed and FP64 Lagrangian and the rotation three times each and exit (the "
                         "cases the committed ncu captures use): the benchmark workload, or an n-octane-shaped "
                         "job (nbf 202, nbf5 198, naux 600) on the general-shape mixed pipeline; batch64: three "
                         "grouped orbital steps of the 64-job water-cluster batch; batch8: the same for its first 8 "
                         "jobs; ints3c: the integral front end's three-centre kernel on a cc-pVDZ-sized synthetic "
                         "basis of (H2O)_8 (nbf 192, naux 512), three launches, timed against the host path; "
                         "pipeline: that molecule from its basis to 20 outer iterations of the energy loop "
                         "(integrals, RI tensor, guess, loop), timed by stage")
    return ap.parse_args()


def config(args, world):
    return {"workload": "synthetic-256 GNOF orbital step (nbf=256, naux=1024, nbf5=64)",
            "nbf": WORKLOAD["nbf"], "naux": WORKLOAD["naux"], "nbf5": 64, "ndoc": 16, "ncwo": 3,
            "orb_method": args.method, "precision": args.precision,
            "fp64_t1": ("DMMA GEMM" if getattr(args, "no_fp64_tc", False) else
                        "tensor cores: 7 int8 digit slices of b and C5, exact int32 products, FP64 recombination"),
            "parallelism": f"replicas x{world}", "l2": "inputs > L2 (b = 512 MiB FP64)"}


class ClockSampler:
    """nvidia-smi samples (200 ms) of SM clock and throttle reasons during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def wait_samples(self, k: int, timeout: float = 3.0):
        """Block until k more samples have arrived (so the sampled window brackets
        a short timed region on both sides)."""
        if not self.proc:
            return
        want = len(self.lines) + k
        t0 = time.time()
        while len(self.lines) < want and time.time() - t0 < timeout:
            time.sleep(0.02)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                smax = float(parts[1])
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower() in ("active", "1"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_dgemm_tflops(torch, dev):
    """FP64 tensor-core ceiling for the plain form: cuBLAS DGEMM 8192^3, best of 5
    (the driver's peak file carries HBM and BF16 figures only)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    for _ in range(2):
        torch.matmul(a, b)
    best = 1e30
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        torch.cuda.synchronize()
        best = min(best, s.elapsed_time(e) / 1e3)
    del a, b
    return 2.0 * n ** 3 / best / 1e12


def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text())
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "fallback": True}


def traffic_from_profiles(kernel_key):
    """DRAM bytes per launch of the transform from the committed ncu summary, if present."""
    p = ROOT / "profiles" / "traffic.json"
    if p.exists():
        try:
            return json.loads(p.read_text()).get(kernel_key)
        except Exception:
            return None
    return None


def max_over_ranks(t, dist, device=None):
    """The largest of the ranks' values (a multi-GPU run takes as long as its
    slowest rank); t itself with a single process."""
    if dist is None:
        return t
    import torch
    tt = torch.tensor([float(t)], dtype=torch.float64, device=device)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    return float(tt.item())


class HostAdam:
    """The optimiser's host side per step: calcorbg's packing of 4 (elag - elag^T),
    row-wise over i < nbf5, j > i (src/pnof.jl:1395-1403), and the AMSGrad form of
    ADAM (src/minimization.jl:406-412), in arrays allocated once (``alloc``
    makes them, e.g. page-locked).  The returned y is overwritten by the next
    step."""

    def __init__(self, nbf, nbf5, alpha=0.01, beta1=0.5, beta2=0.9, alloc=np.zeros):
        iu = np.triu_indices(nbf, 1)
        sel = iu[0] < nbf5
        self.ij = (iu[0][sel] + nbf * iu[1][sel]).astype(np.intp)  # elag[i, j], column-major
        self.ji = (iu[1][sel] + nbf * iu[0][sel]).astype(np.intp)  # elag[j, i]
        nvar = self.ij.shape[0]
        self.m, self.v, self.vmax, self.g, self.t = (np.zeros(nvar) for _ in range(5))
        self.y = alloc(nvar)
        self.alpha, self.beta1, self.beta2, self.i = alpha, beta1, beta2, 0

    def reset(self):
        for a in (self.m, self.v, self.vmax):
            a[:] = 0.0
        self.i = 0

    def step(self, elag):
        g, t, m, v, y = self.g, self.t, self.m, self.v, self.y
        b1, b2 = self.beta1, self.beta2
        self.i += 1
        f = elag.ravel(order="F")
        np.take(f, self.ij, out=g)
        np.take(f, self.ji, out=t)
        np.subtract(g, t, out=g)
        np.multiply(g, 4.0, out=g)
        np.multiply(m, b1, out=m)
        np.multiply(g, 1.0 - b1, out=t)
        np.add(m, t, out=m)
        np.multiply(v, b2, out=v)
        np.multiply(g, g, out=t)
        np.multiply(t, 1.0 - b2, out=t)
        np.add(v, t, out=v)
        np.multiply(v, 1.0 / (1.0 - b2 ** self.i), out=t)
        np.maximum(self.vmax, t, out=self.vmax)
        np.add(self.vmax, 1e-16, out=t)
        np.sqrt(t, out=t)
        np.multiply(m, 1.0 / (1.0 - b1 ** self.i), out=y)
        np.divide(y, t, out=y)
        np.multiply(y, -self.alpha, out=y)
        return y


def run_cpu_steps(wl, steps, budget_s, threads=None, impl="blas"):
    """Orbital steps on the CPU (FP64): host update + rotate + Lagrangian, with
    impl "blas" (oracle/blas_mirror.py: the reference contraction order as
    threaded BLAS GEMMs) or "port" (the scalar C/OpenMP oracle)."""
    if impl == "blas":
        from oracle import blas_mirror as native
    else:
        from oracle import native

        if threads:
            native.set_threads(threads)
    p = wl.p
    C = wl.C.copy(order="F")
    elag, _ = native.lagrange2(C, wl.n, wl.H, wl.b, wl.cj12, wl.ck12, p.nalpha, p.nbeta)
    adam = HostAdam(p.nbf, p.nbf5)
    done = 0
    t0 = time.perf_counter()
    for i in range(1, steps + 1):
        y = adam.step(elag)
        C = native.rotate(y, C, p.nbf5)
        elag, Hmat = native.lagrange2(C, wl.n, wl.H, wl.b, wl.cj12, wl.ck12, p.nalpha, p.nbeta)
        done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    return done, dt, (native.threads() if impl == "blas" else native.num_threads())


def reference_arm(args, rank, world):
    from donof_b200 import workload

    if rank != 0:
        return None
    # the inputs' occupations and couplings from the oracle's restatement, so that
    # this arm runs nothing of the library
    from oracle import gnof as ognof

    def sizes(p):
        return ognof.Sizes(nbf=p.nbf, nbeta=p.nbeta, nalpha=p.nalpha, ncwo=p.ncwo, naux=p.nbfaux, no1=p.no1,
                           ista=p.ista, HighSpin=p.HighSpin, h_cut=p.h_cut, occ_method=p.occ_method)

    layer = (lambda g, p: ognof.ocupacion(g, sizes(p)), lambda n, p: ognof.PNOFi_selector(n, sizes(p)))
    wl = workload.synthetic(**WORKLOAD, seed=SEED, layer=layer)
    run_cpu_steps(wl, max(1, min(args.warmup, 1)), 60.0)  # warm caches / thread pool
    done, dt, cores = run_cpu_steps(wl, args.steps, 150.0)
    v = done / dt
    pdone, pdt, pcores = run_cpu_steps(wl, 3, 20.0, impl="port")
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * dt / done, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": config(args, world),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"{done} of {args.steps} orbital steps: rotate_orbital + compute_Lagrange2 "
                                       "in the reference contraction order as threaded FP64 BLAS GEMMs "
                                       "(oracle/blas_mirror.py; the reference's Tullio loops cannot run here)",
                             "scalar_port": {"value": pdone / pdt, "unit": UNIT, "cores": pcores,
                                             "sample": f"{pdone} orbital steps on the scalar C/OpenMP oracle"}},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    return line


ENERGY_CASE = dict(nbf=96, naux=384, nbeta=8, ncwo=3)
# the n-octane shape (nbf 202, nbf5 198, naux 974) with a weak two-electron part
# (scale 0.05): one GNOF minimum, so that FP64 and mixed + refinement from the
# same start must meet it (at 0.1-0.2 this surrogate has several minima -- the
# pairings of the weak orbitals -- and the two paths can end in different ones)
ENERGY_OCTANE = dict(nbf=202, naux=974, nbeta=33, ncwo=5)


def energies_case(d, torch, ctx, shape, scale, seed):
    from donof_b200 import workload
    from donof_b200.optimize import energy, energy_mixed_refined
    from donof_b200.serve import use_fp64_tc
    out = {"workload": f"molecule-like surrogate (nbf={shape['nbf']}, naux={shape['naux']}, nbeta={shape['nbeta']}, "
                       f"ncwo={shape['ncwo']}, two_e_scale={scale}, seed {seed}), max|g_orb|, |g_occ| < 1e-6",
           "unit": "energies/s",
           "fp64_t1": "tensor cores" if use_fp64_tc(None, shape["nbf"]) else "DMMA GEMM"}
    res = {}
    for form in ("fp64", "mixed_refined"):
        wl = workload.molecule_like(**shape, seed=seed, two_e_scale=scale)
        p = wl.p
        p.threshgorb = p.threshgocc = 1e-6
        p.threshen = 1e-10  # occupations solved tightly each iteration: both forms reach the same minimum
        b = d.eris_to_gpu(wl.b, "fp64" if form == "fp64" else "mixed", ctx)
        if use_fp64_tc(None, p.nbf):
            b.set_fp64_tc(True)   # both forms' FP64 iterations, as the server runs them
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        if form == "fp64":
            r = energy(wl.H, b, p, wl.C, wl.gamma, maxit=1500)
            extra = {}
        else:
            r, rm = energy_mixed_refined(wl.H, b, p, wl.C, wl.gamma, maxit=1500)
            extra = {"mixed_outer_iterations": rm.iterations, "mixed_orbital_steps": rm.tot_it_orb}
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        b.free()
        res[form] = r
        out[form] = {"value": 1.0 / dt, "seconds": dt, "E_elec": r.E_elec, "converged": r.converged,
                     "outer_iterations": r.iterations, "orbital_steps": r.tot_it_orb,
                     "occupation_cg_iterations": r.tot_it_occ, **extra}
    out["abs_dE_Eh"] = abs(res["mixed_refined"].E_elec - res["fp64"].E_elec)
    out["within_1uEh"] = out["abs_dE_Eh"] <= 1e-6
    out["speedup"] = out["mixed_refined"]["value"] / out["fp64"]["value"]
    return out


def energies_bench(d, torch, ctx):
    """Converged GNOF energies/s of the FP64 form and of the mixed form with
    closing FP64 iterations, from the same start, on molecule-shaped surrogates
    with a single well-defined minimum, with the energy difference between the
    two results: an nbf = 96 case and the n-octane shape (config 2's sizes)."""
    out = energies_case(d, torch, ctx, ENERGY_CASE, 0.2, 5)
    out["n_octane"] = energies_case(d, torch, ctx, ENERGY_OCTANE, 0.05, 104)
    return out


# Served stream (shapes of the reference's serving workload: water clusters
# (H2O)_k and linear alkanes CnH2n+2 in cc-pVDZ with a JK-fit set, as molecule-
# shaped surrogates): (nbf, naux, nbeta, ncwo).
SERVE_SHAPES = [(24 * k, 116 * k, 5 * k, 3) for k in (1, 2, 3, 4)] + \
               [(24 * n + 10, int(4.8 * (24 * n + 10)), 4 * n + 1, 5) for n in (1, 2, 3)]
SERVE_LARGE = (202, 974, 33, 5)   # n-octane shape
SERVE = dict(jobs=64, large=4, rate_per_s=20.0, seed=7, thresh=1e-5, threshen=1e-6, inflight=8,
             group_max=16, continuous_slots=8)  # threshen = thresh / 10
# the n-octane-sized jobs (the ones auto runs mixed + closing FP64): a weak
# two-electron part (one GNOF minimum) and gradients to 1e-6, where the energy is
# pinned well below 1 uEh (at 1e-5 two FP64 paths still differ by ~1e-5 Eh)
SERVE_LARGE_JOB = dict(two_e_scale=0.05, thresh=1e-6, threshen=1e-7)


def serving_bench(d, torch):
    """Converged energies/s of a seeded Poisson stream of jobs of different
    sizes: served with continuous batching (auto precision: the mixed form with
    closing FP64 iterations where it pays off), and by the plain FP64 form
    serving the same stream one job at a time; per-job |dE| between the two."""
    import copy
    from donof_b200 import workload
    from donof_b200.serve import Request, Server, resolve_precision, use_fp64_tc
    rng = np.random.default_rng(SERVE["seed"])
    shapes = [SERVE_SHAPES[i] for i in rng.integers(len(SERVE_SHAPES), size=SERVE["jobs"])]
    for pos in rng.choice(len(shapes) + SERVE["large"], size=SERVE["large"], replace=False):
        shapes.insert(int(pos), SERVE_LARGE)
    gaps = rng.exponential(1.0 / SERVE["rate_per_s"], size=len(shapes))
    arrivals = np.cumsum(gaps) - gaps[0]
    jobs = []
    for j, (nbf, naux, nbeta, ncwo) in enumerate(shapes):
        large = (nbf, naux, nbeta, ncwo) == SERVE_LARGE
        wl = workload.molecule_like(nbf=nbf, naux=naux, nbeta=nbeta, ncwo=ncwo, seed=100 + j,
                                    two_e_scale=SERVE_LARGE_JOB["two_e_scale"] if large else 0.2)
        wl.p.threshgorb = wl.p.threshgocc = SERVE_LARGE_JOB["thresh"] if large else SERVE["thresh"]
        wl.p.threshen = SERVE_LARGE_JOB["threshen"] if large else SERVE["threshen"]
        jobs.append(wl)

    # tune every shape's GEMMs and load the kernels before either arm is timed
    ctx = d.Context(0)
    for shp in sorted(set(shapes)):
        wl = jobs[shapes.index(shp)]
        p = wl.p
        prec = resolve_precision("auto", p.nbf, p.nbf5, p.nbfaux)
        b = d.eris_to_gpu(wl.b, "fp64" if prec == "fp64" else "mixed", ctx)
        if use_fp64_tc(None, p.nbf):
            b.set_fp64_tc(True)
        for form in (("fp64",) if prec == "fp64" else ("fp64", "mixed")):
            b.set_precision(form)
            d.compute_Lagrange2(wl.C, wl.n, wl.H, b, wl.cj12, wl.ck12, p.nalpha, p.nbeta)
            d.JKH_MO(wl.C, wl.H, b, p.nbf, p.nbf5, p.nbfaux)
        b.free()
    ctx.close()

    def run(precision, inflight, group_max=0, rate_scale=1.0, continuous=0):
        with Server(max_inflight=inflight, group_max=group_max, continuous_slots=continuous) as srv:
            t0 = time.perf_counter()
            tickets = []
            for wl, t_arr in zip(jobs, arrivals * rate_scale):
                delay = t0 + t_arr - time.perf_counter()
                if delay > 0:
                    time.sleep(delay)
                tickets.append(srv.submit(Request(H=wl.H, b=wl.b, C=wl.C, p=copy.deepcopy(wl.p), gamma=wl.gamma,
                                                  precision=precision, maxit=1000)))
            res = [srv.wait(t) for t in tickets]
            span = max(r.t_done for r in res) - t0
        lat = np.array([r.latency for r in res])
        return res, {"value": len(res) / span, "seconds": span, "converged": int(sum(r.converged for r in res)),
                     "errors": [r.error for r in res if r.error][:2],
                     "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))}}

    ref, seq = run("fp64", 1)
    res, served = run("auto", SERVE["inflight"])
    res_g, served_g = run("auto", SERVE["inflight"], group_max=SERVE["group_max"])
    res_c, served_c = run("auto", SERVE["inflight"], continuous=SERVE["continuous_slots"])
    # the arrival rate swept: the same stream twice as fast, and all requests at once
    sweep = [{"rate_per_s": SERVE["rate_per_s"], "value": served["value"], "latency_s": served["latency_s"]}]
    for scale, label in ((0.5, 2 * SERVE["rate_per_s"]), (0.0, "all at t=0")):
        _, sv = run("auto", SERVE["inflight"], rate_scale=scale)
        sweep.append({"rate_per_s": label, "value": sv["value"], "latency_s": sv["latency_s"],
                      "speedup_vs_fp64_one_at_a_time": sv["value"] / seq["value"]})
    dE = np.array([abs(a.E_elec - b.E_elec) for a, b in zip(res, ref)])
    dE_g = np.array([abs(a.E_elec - b.E_elec) for a, b in zip(res_g, ref)])
    dE_c = np.array([abs(a.E_elec - b.E_elec) for a, b in zip(res_c, ref)])
    return {"unit": "energies/s",
            "workload": f"{len(jobs)} jobs, Poisson arrivals at {SERVE['rate_per_s']:g}/s (seed {SERVE['seed']}): "
                        "molecule-shaped surrogates of (H2O)_k k=1..4, CnH2n+2 n=1..3 and "
                        f"{SERVE['large']} n-octane-sized jobs (nbf 24-202); max|g_orb|, |g_occ| < "
                        f"{SERVE['thresh']:g} ({SERVE_LARGE_JOB['thresh']:g} for the n-octane-sized jobs, "
                        f"two_e_scale {SERVE_LARGE_JOB['two_e_scale']})",
            "fp64_t1": "tensor cores for nbf >= 128 (both arms), DMMA GEMM below",
            "served": {**served, "precision": "auto (mixed + closing FP64 for nbf*nbf5*naux >= 2e7, else FP64)",
                       "max_inflight": SERVE["inflight"]},
            "served_grouped": {**served_g, "group_max": SERVE["group_max"],
                               "path": "as served, and the FP64 jobs waiting when a slot frees start together as one "
                                       "grouped batch (donof_batch_energy)",
                               "abs_dE_Eh_vs_fp64": {"max": float(dE_g.max()), "median": float(np.median(dE_g)),
                                                     "within_1uEh": int(np.sum(dE_g <= 1e-6))}},
            "served_continuous": {**served_c, "slots_per_shape": SERVE["continuous_slots"],
                                  "path": "as served, and the FP64 jobs of each shape share one batch whose slots are "
                                          "refilled as jobs converge (donof_batch_serve: every outer iteration "
                                          "advances all running jobs of the shape as grouped launches)",
                                  "abs_dE_Eh_vs_fp64": {"max": float(dE_c.max()), "median": float(np.median(dE_c)),
                                                        "within_1uEh": int(np.sum(dE_c <= 1e-6))}},
            "speedup_continuous": served_c["value"] / seq["value"],
            "served_rate_sweep": sweep,
            "fp64_one_at_a_time": seq,
            "speedup": served["value"] / seq["value"],
            "speedup_grouped": served_g["value"] / seq["value"],
            "abs_dE_Eh": {"max": float(dE.max()), "median": float(np.median(dE)),
                          "within_1uEh": int(np.sum(dE <= 1e-6)), "of": len(dE)}}


BATCH = dict(count=64, kmax=8, seed=11)


def batched_mixed_bench(d, torch, ctx, steps, warmup, method):
    """The jobs of the water-cluster batch that fit the fused mixed kernel
    ((H2O)_k with k <= 3: nbf <= 72, nbf5 <= 60) advanced together, the grouped
    step with the FP64 Lagrangian against the grouped step with the mixed one
    (donof_batch_set_precision: every job's fused tcgen05 kernel in one grouped
    launch)."""
    from donof_b200 import workload
    jobs = [(j, k, wl) for j, (k, wl) in enumerate(workload.water_clusters(**BATCH)) if k <= 3]
    bts, ins = [], []
    for j, k, wl in jobs:
        tb = workload.b_device(wl.p.nbf, wl.p.nbfaux, seed=BATCH["seed"] * 7919 + j)
        bts.append(d.eris_to_gpu(tb, "mixed", ctx))
        ins.append(dict(p=wl.p, C=d.to_device(wl.C), H=d.to_device(wl.H), n=d.to_device(wl.n),
                        cj=d.to_device(wl.cj12), ck=d.to_device(wl.ck12)))
    nj = len(jobs)
    cols = lambda key: [x[key] for x in ins]
    out = {"workload": f"the {nj} jobs of the 64-job water-cluster batch with k <= 3 (nbf 24-72, nbf5 20-60), "
                       f"{steps} orbital steps each", "unit": "job orbital-gradient steps/s"}
    Es = {}
    for prec in ("fp64", "mixed"):
        batch = d.Batch(bts, [x["p"] for x in ins], ctx)
        batch.set_precision(prec)

        def grouped(ml):
            Cs = [x["C"].clone() for x in ins]
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            res = batch.orbopt(method, cols("n"), cols("cj"), cols("ck"), cols("H"), Cs, [0.01] * nj, [ml] * nj,
                               [0.0] * nj)
            e1.record()
            torch.cuda.synchronize()
            return e0.elapsed_time(e1) / 1e3, res

        grouped(warmup)
        tg, res = grouped(steps)
        Es[prec] = [r[0] for r in res]
        out[prec] = {"value": nj * steps / tg, "ms_per_step": 1e3 * tg / steps}
        batch.free()
    out["mixed"]["path"] = "donof_batch_orbopt with donof_batch_set_precision(MIXED)"
    out["speedup_mixed_vs_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    out["max_rel_dE_mixed_vs_fp64"] = max(abs(a - b) / max(1.0, abs(b)) for a, b in zip(Es["mixed"], Es["fp64"]))
    for b in bts:
        b.free()
    return out


def batched_bench(d, torch, ctx, steps, warmup, method, sequential_arm=True, spec=None):
    """Orbital-gradient steps/s of a batch of uneven jobs advanced together (one
    grouped launch per stage of a step, the loop as one captured graph) against
    the same jobs run one after the other through the single-job device loop:
    64 water-cluster surrogates (H2O)_k, k uniform in 1..8 (nbf 24-192), FP64."""
    from donof_b200 import workload
    spec = spec or BATCH
    jobs = workload.water_clusters(**spec)
    bts, ins = [], []
    for j, (k, wl) in enumerate(jobs):
        tb = workload.b_device(wl.p.nbf, wl.p.nbfaux, seed=spec["seed"] * 7919 + j)
        bts.append(d.eris_to_gpu(tb, "fp64", ctx))
        ins.append(dict(p=wl.p, C=d.to_device(wl.C), H=d.to_device(wl.H), n=d.to_device(wl.n),
                        cj=d.to_device(wl.cj12), ck=d.to_device(wl.ck12)))
    nj = len(jobs)
    batch = d.Batch(bts, [x["p"] for x in ins], ctx)
    cols = lambda key: [x[key] for x in ins]

    def grouped(ml):
        Cs = [x["C"].clone() for x in ins]
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = d.launch_count()
        e0.record()
        res = batch.orbopt(method, cols("n"), cols("cj"), cols("ck"), cols("H"), Cs, [0.01] * nj, [ml] * nj,
                           [0.0] * nj)
        e1.record()
        torch.cuda.synchronize()
        assert all(r[1] == ml for r in res), "every job takes exactly maxloop steps"
        return e0.elapsed_time(e1) / 1e3, d.launch_count() - l0, res

    grouped(warmup)  # autotune + capture
    tg, lg, res_g = grouped(steps)

    def sequential(ml):
        Cs = [x["C"].clone() for x in ins]
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        res = [d.orbopt_dev(method, x["n"], x["cj"], x["ck"], x["H"], C, bt, x["p"], 0.01, ml, 0.0)
               for x, C, bt in zip(ins, Cs, bts)]
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3, res

    if not sequential_arm:
        batch.free()
        for b in bts:
            b.free()
        return {"grouped_ms_per_step": 1e3 * tg / steps, "launches_per_step": lg / steps}
    sequential(warmup)
    ts, res_s = sequential(steps)
    dE = max(abs(a[0] - b[0]) / max(1.0, abs(b[0])) for a, b in zip(res_g, res_s))
    out = {"workload": f"{nj} water-cluster surrogates (H2O)_k, k ~ U{{1..{spec['kmax']}}} (nbf 24-192, naux 116k, "
                       f"nbf5 20k), FP64, {steps} orbital steps each",
           "ks": [k for k, _ in jobs], "unit": "job orbital-gradient steps/s",
           "grouped": {"value": nj * steps / tg, "ms_per_step": 1e3 * tg / steps, "launches_per_step": lg / steps,
                       "path": "donof_batch_orbopt (grouped persistent GEMMs + grouped cooperative kernels, "
                               "one graph)"},
           "sequential": {"value": nj * steps / ts, "ms_per_round": 1e3 * ts / steps,
                          "path": "donof_orbopt_dev per job, one after the other"},
           "speedup": ts / tg, "max_rel_dE_grouped_vs_sequential": dE,
           "device_bytes": batch.device_bytes()}
    batch.free()
    for b in bts:
        b.free()
    return out


BATCH_E = dict(count=16, kmax=4, seed=13, thresh=1e-6)


def batched_energies_bench(d, torch, ctx):
    """Converged GNOF energies/s of a batch of water-cluster-shaped molecules
    (k uniform in 1..4: nbf 24-96), FP64: every job's energy loop with the
    orbital optimisations of all running jobs grouped per outer iteration
    (donof_batch_energy), against the same jobs through donof_energy one after
    the other; both from the same start to the same thresholds."""
    from donof_b200 import workload
    from donof_b200.gnof import guess_gamma
    rng = np.random.default_rng(BATCH_E["seed"])
    ks = [int(k) for k in rng.integers(1, BATCH_E["kmax"] + 1, size=BATCH_E["count"])]
    th = BATCH_E["thresh"]

    def make(j, k):
        wl = workload.molecule_like(nbf=24 * k, naux=116 * k, nbeta=5 * k, ncwo=3, seed=BATCH_E["seed"] * 100 + j,
                                    two_e_scale=0.2)
        wl.p.threshgorb = wl.p.threshgocc = th
        wl.p.threshen = th / 1e4
        return wl

    wls = [make(j, k) for j, k in enumerate(ks)]
    g0 = [guess_gamma(wl.p) for wl in wls]
    bts = [d.eris_to_gpu(wl.b, "fp64", ctx) for wl in wls]
    fresh = lambda: [make(j, k).p for j, k in enumerate(ks)]
    # warm-up (autotuning, graph capture, scratch) of both arms
    batch = d.Batch(bts, fresh(), ctx)
    batch.energy([wl.H for wl in wls], [wl.C for wl in wls], g0, maxit=1)
    for wl, bt, p, g in zip(wls, bts, fresh(), g0):
        d.api.energy_loop(wl.H, bt, p, wl.C, g, maxit=1)
    torch.cuda.synchronize()
    batch.params = fresh()
    t0 = time.perf_counter()
    rb = batch.energy([wl.H for wl in wls], [wl.C for wl in wls], g0, maxit=1000)
    tb = time.perf_counter() - t0
    t0 = time.perf_counter()
    rs = [d.api.energy_loop(wl.H, bt, p, wl.C, g, maxit=1000)[4] for wl, bt, p, g in zip(wls, bts, fresh(), g0)]
    ts = time.perf_counter() - t0
    dEs = sorted(abs(a[3]["E_elec"] - b["E_elec"]) for a, b in zip(rb, rs))
    out = {"workload": f"{len(ks)} water-cluster-shaped molecule surrogates (H2O)_k, k ~ U{{1..{BATCH_E['kmax']}}} "
                       f"(nbf 24-96, naux 116k), FP64, max|g_orb|, |g_occ| < {th}",
           "ks": ks, "unit": "energies/s",
           "grouped": {"value": len(ks) / tb, "seconds": tb, "converged": sum(r[3]["converged"] for r in rb),
                       "outer_iterations": [r[3]["iterations"] for r in rb],
                       "path": "donof_batch_energy (orbital loops of all running jobs grouped per outer iteration)"},
           "sequential": {"value": len(ks) / ts, "seconds": ts, "converged": sum(r["converged"] for r in rs),
                          "path": "donof_energy per job, one after the other"},
           "speedup": ts / tb, "abs_dE_Eh": {"median": dEs[len(dEs) // 2], "max": dEs[-1],
                                              "within_1uEh": sum(x <= 1e-6 for x in dEs)}}
    batch.free()
    for b in bts:
        b.free()
    return out


def profile_case(d, torch, wl, ctx):
    """Three calls each of the mixed and FP64 Lagrangian and of the rotation, then
    three of the FP64 Lagrangian with its first contraction on the tensor cores."""
    import numpy as np
    p = wl.p
    bt = d.eris_to_gpu(wl.b, "mixed", ctx)
    tC, tH, tn, tcj, tck = (d.to_device(x) for x in (wl.C, wl.H, wl.n, wl.cj12, wl.ck12))
    y = torch.from_numpy(0.003 * np.random.default_rng(0).standard_normal(p.nvar)).cuda()
    Cn = torch.empty_like(tC)
    el = torch.zeros(p.nbf, p.nbf, dtype=torch.float64, device="cuda")
    hm = torch.zeros(p.nbf5, p.nbf, dtype=torch.float64, device="cuda")
    E = torch.zeros(1, dtype=torch.float64, device="cuda")
    for _ in range(3):
        d.compute_Lagrange2_dev(tC, tn, tH, bt, tcj, tck, p.nalpha, p.nbeta, el, hm, E, precision="mixed")
        d.compute_Lagrange2_dev(tC, tn, tH, bt, tcj, tck, p.nalpha, p.nbeta, el, hm, E, precision="fp64")
        d.rotate_orbital_dev(y, tC, Cn, p.nbf, p.nbf5, ctx)
    bt.set_fp64_tc(True)
    for _ in range(3):
        d.compute_Lagrange2_dev(tC, tn, tH, bt, tcj, tck, p.nalpha, p.nbeta, el, hm, E, precision="fp64")
    torch.cuda.synchronize()
    bt.free()


def ints3c_case(d, torch, workload, device):
    """(mn|P) of the integral front end on the device (three launches, CUDA
    events on the context's stream) and on the host threads, same basis."""
    import numpy as np
    from donof_b200 import integrals as it

    ctx = d.Context(device)
    orb, aux = workload.water_cluster_bases(8)
    ms = []
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        out = it.ERI_2e3c_dev(orb, aux, ctx)
        e1.record()
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    t = time.perf_counter()
    host = it.ERI_2e3c(orb, aux)
    th = time.perf_counter() - t
    dev = out.cpu().numpy().reshape(host.shape, order="F")
    return {"case": "ints3c", "nbf": orb.nbas, "naux": aux.nbas, "device_ms": ms, "host_ms": th * 1e3,
            "host_threads": os.cpu_count(), "max_rel_diff": float(np.max(np.abs(dev - host)) / np.max(np.abs(host)))}


def pipeline_case(d, torch, workload, device, outer=20):
    """A molecule through the whole path: integrals (one-electron and (P|Q) on
    the host, (mn|P) on the device), b = I G^{-1/2} on the device (Iaux), the
    core-Hamiltonian guess, then `outer` iterations of the FP64 energy loop
    (first contraction on the tensor cores), each stage timed."""
    from donof_b200 import integrals as it
    from donof_b200.guess import guess

    ctx = d.Context(device)
    orb, aux = workload.water_cluster_bases(8)
    ne = sum(a.Z for a in orb.atoms)
    p = d.Param(nbf=orb.nbas, nbfaux=0, nalpha=ne // 2, nbeta=ne // 2)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    S, T, V, H, bt = it.compute_integrals(orb, aux, p, ctx)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    bt.set_fp64_tc(True)
    C, gamma = guess(H, p, S)
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    _, _, _, _, r, hist = d.api.energy_loop(H, bt, p, C, gamma, maxit=outer)
    t3 = time.perf_counter()
    out = {"case": "pipeline", "workload": "synthetic cc-pVDZ-sized basis on (H2O)_8", "nbf": orb.nbas,
           "naux": aux.nbas, "nbf5": p.nbf5, "electrons": ne, "integrals_and_iaux_s": t1 - t0,
           "digit_split_and_guess_s": t2 - t1, "energy_loop_s": t3 - t2, "outer_iterations": r["iterations"],
           "orbital_steps": r["tot_it_orb"], "E_elec": r["E_elec"], "converged": bool(r["converged"])}
    bt.free()
    return out


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        backend = "nccl" if args.impl == "ours" else "gloo"
        if backend == "nccl":
            import torch
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))

    if args.impl == "reference":
        line = reference_arm(args, rank, world)
        if line is not None:
            print(json.dumps(line), flush=True)
        if dist is not None:
            dist.destroy_process_group()
        return

    import torch
    import donof_b200 as d
    from donof_b200 import workload

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if args.profile_case == "ints3c":
        print(json.dumps(ints3c_case(d, torch, workload, local)), flush=True)
        return
    if args.profile_case == "pipeline":
        print(json.dumps(pipeline_case(d, torch, workload, local)), flush=True)
        return
    wl = workload.synthetic(**WORKLOAD, seed=SEED)
    p = wl.p
    ctx = d.Context(local)
    if args.profile_case in ("batch64", "batch8"):
        spec = dict(BATCH, count=8) if args.profile_case == "batch8" else BATCH
        print(json.dumps(batched_bench(d, torch, ctx, 3, 1, args.method, sequential_arm=False, spec=spec)), flush=True)
        return
    if args.profile_case:
        if args.profile_case == "octane600":
            wl = workload.synthetic(nbf=202, naux=600, nbeta=33, ncwo=5, seed=SEED)
        profile_case(d, torch, wl, ctx)
        return
    bt = d.eris_to_gpu(wl.b, "mixed", ctx)   # FP64 b and its bf16 split: both forms are timed
    bt.set_precision(args.precision)
    if not args.no_fp64_tc:
        bt.set_fp64_tc(True)                  # and b's int8 digit slices for the FP64 form's T1
    tC0, tH, tn, tcj, tck = (d.to_device(x, dev) for x in (wl.C, wl.H, wl.n, wl.cj12, wl.ck12))

    def barrier():
        if dist is not None:
            dist.barrier()

    # ---- device-resident optimiser loop: warm-up, then exactly K steps
    tC = tC0.clone()
    d.orbopt_dev(args.method, tn, tcj, tck, tH, tC, bt, p, 0.01, args.warmup, 0.0)
    tC.copy_(tC0)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    l0 = d.launch_count()
    with ClockSampler(local) as clk:
        clk.wait_samples(2)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        E, nit, ok, _, _ = d.orbopt_dev(args.method, tn, tcj, tck, tH, tC, bt, p, 0.01, args.steps, 0.0)
        ev1.record()
        torch.cuda.synchronize()
        clk.wait_samples(1)
    launches = d.launch_count() - l0
    barrier()
    t = ev0.elapsed_time(ev1) / 1e3
    assert nit == args.steps, (nit, args.steps)
    t = max_over_ranks(t, dist, dev)
    value = world * args.steps / t

    # ---- the other form's device loop on the same workload (same step count)
    other = "mixed" if args.precision == "fp64" else "fp64"
    bt.set_precision(other)
    tC.copy_(tC0)
    d.orbopt_dev(args.method, tn, tcj, tck, tH, tC, bt, p, 0.01, args.warmup, 0.0)
    tC.copy_(tC0)
    torch.cuda.synchronize()
    barrier()
    ev0.record()
    _, nit2, _, _, _ = d.orbopt_dev(args.method, tn, tcj, tck, tH, tC, bt, p, 0.01, args.steps, 0.0)
    ev1.record()
    torch.cuda.synchronize()
    t2 = ev0.elapsed_time(ev1) / 1e3
    t2 = max_over_ranks(t2, dist, dev)
    other_form = {"precision": other, "value": world * nit2 / t2, "unit": UNIT, "ms_per_step": 1e3 * t2 / nit2}
    bt.set_precision(args.precision)
    tC.copy_(tC0)

    # ---- the FP64 form with its first contraction on the DMMA GEMM (same step count)
    fp64_gemm = None
    if bt.fp64_tc:
        bt.set_fp64_tc(False)
        bt.set_precision("fp64")
        d.orbopt_dev(args.method, tn, tcj, tck, tH, tC, bt, p, 0.01, args.warmup, 0.0)
        tC.copy_(tC0)
        torch.cuda.synchronize()
        barrier()
        ev0.record()
        E3, nit3, _, _, _ = d.orbopt_dev(args.method, tn, tcj, tck, tH, tC, bt, p, 0.01, args.steps, 0.0)
        ev1.record()
        torch.cuda.synchronize()
        t3 = max_over_ranks(ev0.elapsed_time(ev1) / 1e3, dist, dev)
        fp64_gemm = {"value": world * nit3 / t3, "unit": UNIT, "ms_per_step": 1e3 * t3 / nit3,
                     "t1": "DMMA GEMM (mma.sync f64)", "final_E": E3,
                     "abs_dE_vs_tensor_cores": abs(E3 - E)}
        bt.set_fp64_tc(True)
        bt.set_precision(args.precision)
        tC.copy_(tC0)

    # ---- roofline of the dominant kernel, timed by the library's events on the launching stream
    nbf, naux, nbf5 = p.nbf, p.nbfaux, p.nbf5
    lib = ctx.lib
    ctx.check(lib.donof_profile_enable(ctx.handle, 1))
    el = torch.zeros(nbf, nbf, dtype=torch.float64, device=dev)
    hm = torch.zeros(nbf5, nbf, dtype=torch.float64, device=dev)
    Eb = torch.zeros(1, dtype=torch.float64, device=dev)
    durs = []
    for r in range(13):
        d.compute_Lagrange2_dev(tC, tn, tH, bt, tcj, tck, p.nalpha, p.nbeta, el, hm, Eb)
        ms = ct.c_float()
        ctx.check(lib.donof_profile_last_ms(ctx.handle, ct.byref(ms)))
        if r >= 3:
            durs.append(ms.value / 1e3)
    ctx.check(lib.donof_profile_enable(ctx.handle, 0))
    tr = statistics.mean(durs)
    peaks = load_peaks()
    if args.precision == "fp64" and bt.fp64_tc:
        ldn = (nbf + 15) // 16 * 16
        byts = 7.0 * nbf * ldn * naux + 8.0 * nbf * nbf5 * naux
        macs = 28.0 * nbf * nbf * nbf5 * naux
        roof = {"bound": "hbm", "achieved": byts / tr / 1e9, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": byts / tr / 1e9 / peaks["hbm_gbs"], "traffic": traffic_from_profiles("t1_oz"),
                "kernel": "ozaki_t1_kernel (T1 tmp_l = b_l C5 on tcgen05 kind::i8: 28 digit products, "
                          "int32 TMEM accumulators, FP64 recombination)",
                "algorithmic": f"int8 slices of b read once + tmp written = 7*nbf*ldn*naux + 8*nbf*nbf5*naux "
                               f"= {byts:.4e} bytes per launch",
                "int8_tops": 2.0 * macs / tr / 1e12, "fp64_equivalent_tflops": 2.0 * nbf * nbf * nbf5 * naux / tr / 1e12,
                "ms": tr * 1e3,
                "peak_source": "MEASURED_PEAKS.json hbm_gbs, of measured" + (" (fallback)" if peaks.get("fallback") else "")}
    elif args.precision == "fp64":
        flops = 2.0 * nbf * nbf * nbf5 * naux
        peak = measured_dgemm_tflops(torch, dev)
        roof = {"bound": "tensor", "achieved": flops / tr / 1e12, "peak": peak, "unit": "TFLOP/s",
                "frac": flops / tr / 1e12 / peak, "traffic": traffic_from_profiles("t1_f64"),
                "kernel": "gemm_f64 T1 (DMMA; tile shape and grid form chosen by the autotuner): tmp_l = b_l C5, batched over naux",
                "algorithmic": f"2*nbf^2*nbf5*naux = {flops:.4e} FLOP per launch", "ms": tr * 1e3,
                "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (FP64 tensor pipe); of measured"}
    else:
        byts = 4.0 * nbf * nbf * naux
        # MMA work actually issued per launch: T1 (hi and lo b), T2, Y (hi and lo tmp), M = 128 rows
        flops = naux * (2 * 2.0 * 128 * nbf * nbf + 2.0 * 128 * 128 * nbf + 2 * 2.0 * 128 * nbf * 64)
        roof = {"bound": "hbm", "achieved": byts / tr / 1e9, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": byts / tr / 1e9 / peaks["hbm_gbs"], "traffic": traffic_from_profiles("lag_mixed"),
                "kernel": "lag_mixed_kernel (fused T1, T2, W, Y on tcgen05, bf16 hi/lo)",
                "algorithmic": f"b_hi + b_lo read once = 4*nbf^2*naux = {byts:.4e} bytes per launch",
                "tensor_tflops": flops / tr / 1e12, "ms": tr * 1e3,
                "peak_source": "MEASURED_PEAKS.json hbm_gbs, of measured" + (" (fallback)" if peaks.get("fallback") else "")}

    # ---- end to end through the host-buffer C ABI (what a DoNOF.jl loop does per step)
    e2e = None
    if not args.no_e2e:
        # the caller's arrays in page-locked host memory, as a DoNOF.jl loop
        # would hold them pinned: the entry points DMA them with no staging copy
        def pinned_copy(a):
            h = d.host_pinned(a.shape)
            h[...] = a
            return h

        Hh, nh, cjh, ckh = (pinned_copy(a) for a in (wl.H, wl.n, wl.cj12, wl.ck12))
        Cs = [pinned_copy(wl.C), d.host_pinned(wl.C.shape)]
        elag, Hm = d.host_pinned((nbf, nbf)), d.host_pinned((nbf, nbf5))
        # the host side of each iteration (gradient packing, AMSGrad update) in the
        # library's compiled helper, as a compiled Julia loop would run it
        adam = d.OrbStepHost(nbf, nbf5, "ADAM", alpha=0.01, maxloop=p.maxloop, alloc=d.host_pinned)

        def host_step(k):
            # one iteration of src/minimization.jl:387-422: update, rotate, Lagrangian + energy
            y = adam.step(elag)
            d.rotate_orbital(y, Cs[k % 2], p, ctx, out=Cs[(k + 1) % 2])
            d.compute_Lagrange2(Cs[(k + 1) % 2], nh, Hh, bt, cjh, ckh, p.nalpha, p.nbeta, return_energy=True,
                                out=(elag, Hm))

        def start():
            Cs[0][...] = wl.C
            adam.reset()
            d.compute_Lagrange2(Cs[0], nh, Hh, bt, cjh, ckh, p.nalpha, p.nbeta, out=(elag, Hm))

        start()
        for k in range(args.warmup):
            host_step(k)
        start()
        torch.cuda.synchronize()
        barrier()
        evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
        evs[0].record()
        for i in range(1, args.steps + 1):
            host_step(i - 1)
            evs[i].record()
        torch.cuda.synchronize()
        te = evs[0].elapsed_time(evs[-1]) / 1e3
        per_step = [evs[i - 1].elapsed_time(evs[i]) for i in range(1, args.steps + 1)]
        te = max_over_ranks(te, dist, dev)
        nn, n55 = nbf * nbf, nbf5 * nbf5
        h2d = 8 * (p.nvar + nn) + 8 * (nn + nn + nbf5 + 2 * n55)
        d2h = 8 * nn + 8 * (nn + nbf * nbf5 + 1)
        e2e = {"value": world * args.steps / te, "unit": UNIT, "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h,
               "path": "donof_rotate + donof_lagrange2 (page-locked host buffers), "
                       "host update by donof_orb_step_host",
               "latency_ms": {"p50": float(np.percentile(per_step, 50)), "p99": float(np.percentile(per_step, 99)),
                              "per": "orbital step through the host-buffer C ABI"}}

    energies = None
    if rank == 0 and world == 1 and not args.no_energies:
        energies = energies_bench(d, torch, ctx)
    serving = None
    if rank == 0 and world == 1 and not args.no_serving:
        serving = serving_bench(d, torch)

    batched = batched_e = None
    if rank == 0 and world == 1 and not args.no_batched:
        batched = batched_bench(d, torch, ctx, args.steps, args.warmup, args.method)
        batched["mixed_subset"] = batched_mixed_bench(d, torch, ctx, args.steps, args.warmup, args.method)
        batched_e = batched_energies_bench(d, torch, ctx)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        run_cpu_steps(wl, 1, 20.0)  # warm the thread pool
        done, dt, cores = run_cpu_steps(wl, 20, 15.0)
        pdone, pdt, pcores = run_cpu_steps(wl, 6, 15.0, impl="port")
        cpu = {"value": done / dt, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"{done} orbital steps of the same workload: rotate_orbital + compute_Lagrange2 in the "
                         "reference contraction order as threaded FP64 BLAS GEMMs (oracle/blas_mirror.py)",
               "scalar_port": {"value": pdone / pdt, "unit": UNIT, "cores": pcores,
                               "sample": f"{pdone} orbital steps on the scalar C/OpenMP oracle"}}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": "f64" if args.precision == "fp64" else "bf16x2-split+f64", "data": "synthetic",
                "config": config(args, world), "roofline": roof, "cpu_baseline": cpu, "e2e": e2e,
                "gpu_launches": int(launches), "clocks": clk.summary(), "final_E": E,
                "other_form": other_form, "fp64_dmma_t1": fp64_gemm}
        if energies is not None:
            line["energies"] = energies
        if serving is not None:
            line["serving"] = serving
        if batched is not None:
            line["batched"] = batched
            line["batched_energies"] = batched_e
        print(json.dumps(line), flush=True)
    bt.free()
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
