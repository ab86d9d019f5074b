"""Writes the oracle fixtures of this folder from the CPU oracle.

These are NOT reference outputs: the reference (Julia) cannot run here and
ships no fixtures or golden vectors, so these vectors come from the oracle
restatement (itself pinned only by identities and a second restatement,
tests/test_oracle.py).  Parity against the reference stays unpinned; the
fixtures freeze the oracle's answers so that a change to either side shows.
Inputs are regenerated from the seed by donof_b200.workload (numpy PCG64),
so only sizes, seed and outputs are stored.

    python tests/golden/make_oracle_fixtures.py
"""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path[:0] = [str(ROOT), str(ROOT / "donof.jl_b200")]

from donof_b200 import workload  # noqa: E402
from oracle import gnof, native  # noqa: E402

CASES = {
    "water_surrogate": dict(nbf=24, naux=116, nbeta=5, ncwo=3, seed=11),
    "open_shell_small": dict(nbf=30, naux=41, nbeta=3, ncwo=3, seed=12, nalpha=5),
}


def make(name, nbf, naux, nbeta, ncwo, seed, nalpha=None):
    kw = {}
    wl = workload.synthetic(nbf=nbf, naux=naux, nbeta=nbeta, ncwo=ncwo, seed=seed)
    p = wl.p
    if nalpha is not None:
        # open shell: same b/C/H, occupations of an nalpha > nbeta system
        from donof_b200 import Param, gnof as pg
        p = Param(nbf=nbf, nbfaux=naux, nbeta=nbeta, nalpha=nalpha, ncwo=ncwo)
        rng = np.random.default_rng(seed + 1)
        gamma = rng.standard_normal(p.nv)
        n, _ = pg.occupations(gamma, p)
        cj, ck = pg.coupling(n, p)
        kw = dict(gamma=gamma)
    else:
        n, cj, ck = wl.n, wl.cj12, wl.ck12
        kw = dict(gamma=wl.gamma)
    elag, Hmat = native.lagrange2(wl.C, n, wl.H, wl.b, cj, ck, p.nalpha, p.nbeta)
    J, K, Hc = native.jkh_mo(wl.C, wl.H, wl.b, p.nbf5)
    rng = np.random.default_rng(seed + 2)
    y = 0.02 * rng.standard_normal(p.nvar)
    Crot = native.rotate(y, wl.C, p.nbf5)
    s = gnof.Sizes(nbf=nbf, nbeta=p.nbeta, nalpha=p.nalpha, ncwo=ncwo, naux=naux)
    E = gnof.computeE_elec_Hmat(Hmat, n, elag, s)
    np.savez_compressed(Path(__file__).with_name(f"{name}.npz"), nbf=nbf, naux=naux, nbeta=p.nbeta,
                        nalpha=p.nalpha, ncwo=ncwo, seed=seed, n=n, cj12=cj, ck12=ck, elag=elag, Hmat=Hmat,
                        J=J, K=K, Hcore=Hc, y=y, Crot=Crot, E=E, **kw)


if __name__ == "__main__":
    for name, kw in CASES.items():
        make(name, **kw)
        print("wrote", name)
