"""Seeded synthetic inputs with the shapes and value distributions of the
benchmark workloads (the reference publishes no data set for this path and
no integral engine or basis data is available, so every workload is
synthetic):

  b[m,n,l] ~ N(0, 1/sqrt(naux)) symmetrised in (m, n)  -- the RI tensor
  C        = Q of the QR of a seeded N(0,1) nbf x nbf matrix
  H        = seeded symmetric N(0,1)/sqrt(nbf) matrix
  gamma    ~ N(0,1) softmax parameters, pairs then sorted by
             order_occupations_softmax (which also permutes C)
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import gnof
from .param import Param


@dataclass
class Workload:
    p: Param
    b: np.ndarray      # (nbf, nbf, naux), Fortran order (Julia layout)
    C: np.ndarray      # (nbf, nbf), Fortran order
    H: np.ndarray
    gamma: np.ndarray
    n: np.ndarray
    cj12: np.ndarray
    ck12: np.ndarray


def make_b(nbf: int, naux: int, rng: np.random.Generator) -> np.ndarray:
    # generated as (l, n, m) in C order, i.e. b[m, n, l] in Julia's column-major order
    raw = rng.standard_normal((naux, nbf, nbf)) * (1.0 / np.sqrt(naux))
    raw += raw.transpose(0, 2, 1)
    raw *= 0.5
    return raw.T  # Fortran-ordered view with shape (nbf, nbf, naux)


def synthetic(nbf: int = 256, naux: int = 1024, nbeta: int = 16, ncwo: int = 3, seed: int = 1234,
              occ_method: str = "Softmax", with_b: bool = True, layer=None, **param_kw) -> Workload:
    """layer: (occupations, coupling) functions of (gamma | n, Param) giving n and
    cj12/ck12 (default: this package's, i.e. the library's native host code)."""
    occupations, coupling = layer or (gnof.occupations, gnof.coupling)
    rng = np.random.default_rng(seed)
    p = Param(nbf=nbf, nbfaux=naux, nalpha=nbeta, nbeta=nbeta, ncwo=ncwo, occ_method=occ_method, **param_kw)
    if p.nbf5 > nbf:
        raise ValueError(f"nbf5 = {p.nbf5} exceeds nbf = {nbf}")
    b = make_b(nbf, naux, rng) if with_b else None
    Q, _ = np.linalg.qr(rng.standard_normal((nbf, nbf)))
    C = np.asfortranarray(Q)
    A = rng.standard_normal((nbf, nbf))
    H = np.asfortranarray((A + A.T) * (0.5 / np.sqrt(nbf)))
    gamma = rng.standard_normal(p.nv)
    if occ_method == "Softmax":
        C, gamma = gnof.order_occupations_softmax(C, gamma, p)
    n, _ = occupations(gamma, p)
    cj12, ck12 = coupling(n, p)
    return Workload(p, b, C, H, gamma, n, np.asfortranarray(cj12), np.asfortranarray(ck12))


def molecule_like(nbf: int = 256, naux: int = 1024, nbeta: int = 16, ncwo: int = 3, seed: int = 1234,
                  two_e_scale: float = 0.5, occ_method: str = "Softmax", **param_kw) -> Workload:
    """Seeded inputs with a molecule-like energy landscape for full optimisations:
    H = Q diag(eps) Q^T with nbeta bound levels in [-3, -0.8] Eh and the rest in
    [0.1, 2.5] Eh, b ~ N(0, two_e_scale/sqrt(naux)) symmetrised (a two-electron part
    weaker than the one-electron one), starting orbitals close to those of H, and
    the reference's initial gamma (src/guess.jl:200-213).  The purely random
    workload of ``synthetic`` has an occupation landscape with several stationary
    points, which makes converged energies depend on the optimiser's path."""
    rng = np.random.default_rng(seed)
    p = Param(nbf=nbf, nbfaux=naux, nalpha=nbeta, nbeta=nbeta, ncwo=ncwo, occ_method=occ_method, **param_kw)
    Q, _ = np.linalg.qr(rng.standard_normal((nbf, nbf)))
    eps = np.sort(np.concatenate([-np.linspace(3.0, 0.8, nbeta), np.linspace(0.1, 2.5, nbf - nbeta)]))
    H = np.asfortranarray((Q * eps) @ Q.T)
    raw = rng.standard_normal((naux, nbf, nbf)) * (two_e_scale / np.sqrt(naux))
    raw += raw.transpose(0, 2, 1)
    raw *= 0.5
    b = raw.T
    C = np.asfortranarray(np.linalg.qr(Q + 0.05 * rng.standard_normal((nbf, nbf)))[0])
    gamma = gnof.guess_gamma(p)
    n, _ = gnof.occupations(gamma, p)
    cj12, ck12 = gnof.coupling(n, p)
    return Workload(p, b, C, H, gamma, n, np.asfortranarray(cj12), np.asfortranarray(ck12))


def b_device(nbf: int, naux: int, seed: int, device="cuda"):
    """The RI tensor of ``make_b``'s distribution generated on the GPU (seeded
    torch generator): a CUDA tensor of shape (naux, nbf, nbf) holding b[m, n, l]
    in Julia's column-major order, for workloads too large to build on the host."""
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    raw = torch.randn((naux, nbf, nbf), generator=g, device=device, dtype=torch.float64) * (1.0 / np.sqrt(naux))
    raw += raw.transpose(1, 2).clone()
    raw *= 0.5
    return raw.contiguous()


def water_clusters(count: int = 64, kmax: int = 8, seed: int = 11) -> list:
    """Shapes of a batch of (H2O)_k clusters, k uniform in 1..kmax (seeded), as
    molecule-shaped surrogates of cc-pVDZ with its JK-fit set: nbf = 24k,
    naux = 116k, nbeta = 5k, ncwo = 3 (nbf5 = 20k).  b is not built here
    (``b_device``); each entry is (k, Workload without b)."""
    rng = np.random.default_rng(seed)
    ks = rng.integers(1, kmax + 1, size=count)
    return [(int(k), synthetic(nbf=24 * int(k), naux=116 * int(k), nbeta=5 * int(k), ncwo=3,
                               seed=seed * 1000 + j, with_b=False)) for j, k in enumerate(ks)]


# Named workloads (sizes of the molecule-shaped surrogates: nbf, naux, nbeta, ncwo)
CONFIGS = {
    "water-ccpvdz-surrogate": dict(nbf=24, naux=116, nbeta=5, ncwo=3),
    "synthetic-256": dict(nbf=256, naux=1024, nbeta=16, ncwo=3),
    "n-octane-ccpvdz-surrogate": dict(nbf=202, naux=974, nbeta=33, ncwo=5),
}


def _et(lo: float, ratio: float, count: int) -> np.ndarray:
    return lo * ratio ** np.arange(count)[::-1]


def water_cluster_bases(k: int = 8, seed: int = 0, spherical: bool = True):
    """A cc-pVDZ-sized synthetic orbital basis and an s-f auxiliary basis on a
    seeded (H2O)_k (the integral front end's workload; no basis-set data ships
    here, so the exponents are even-tempered and the contractions seeded):
    O 3s2p1d + H 2s1p (24 functions per water), auxiliary O 5s3p3d1f + H 3s2p1d
    (64 per water).  Returns (orbital BasisSet, auxiliary BasisSet)."""
    from . import integrals as it

    rng = np.random.default_rng(seed)
    prim = _et(0.25, 3.0, 8)
    c = lambda n: np.abs(rng.standard_normal(n)) + 0.1
    orb = {"O": [(0, prim, c(8)), (0, prim[-3:], c(3)), (0, prim[-1:], np.ones(1)),
                 (1, _et(0.3, 3.5, 3), c(3)), (1, np.array([0.3]), np.ones(1)), (2, np.array([1.2]), np.ones(1))],
           "H": [(0, _et(0.15, 4.0, 3), c(3)), (0, np.array([0.12]), np.ones(1)), (1, np.array([0.7]), np.ones(1))]}
    aux = {"O": [(0, np.array([x]), np.ones(1)) for x in _et(0.3, 4.0, 5)] +
                [(1, np.array([x]), np.ones(1)) for x in _et(0.5, 4.0, 3)] +
                [(2, np.array([x]), np.ones(1)) for x in _et(0.4, 3.0, 3)] + [(3, np.array([1.0]), np.ones(1))],
           "H": [(0, np.array([x]), np.ones(1)) for x in _et(0.3, 5.0, 3)] +
                [(1, np.array([x]), np.ones(1)) for x in _et(0.5, 4.0, 2)] + [(2, np.array([1.0]), np.ones(1))]}
    lines = []
    for _ in range(k):
        o = rng.uniform(-4.0, 4.0, 3)
        lines += [f"O {o[0]} {o[1]} {o[2]}", f"H {o[0]} {o[1] + 0.757} {o[2] + 0.587}",
                  f"H {o[0]} {o[1] - 0.757} {o[2] + 0.587}"]
    atoms, _, _ = it.parse_molecule("\n".join(lines))
    return it.BasisSet("synthetic-dz", atoms, orb, spherical), it.BasisSet("synthetic-dz-jk", atoms, aux, spherical)
