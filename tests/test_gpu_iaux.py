"""b = I G^{-1/2} built on the device (donof_iaux) against the oracle's
restatement of Iaux (src/integrals.jl:68-91): FP64, including a G with
negative eigenvalues (their inverse square roots are zero) and a G whose
lower triangle differs from the upper one (Symmetric(G) reads the upper)."""
import numpy as np
import pytest
import torch

import donof_b200 as d
from oracle import integrals

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _inputs(nbf, naux, seed, negative=0, asym=False):
    rng = np.random.default_rng(seed)
    Q, _ = np.linalg.qr(rng.standard_normal((naux, naux)))
    w = np.linspace(0.5, 4.0, naux)
    if negative:
        w[:negative] = -np.linspace(0.1, 0.3, negative)
    G = (Q * w) @ Q.T
    if asym:
        G = G + np.tril(rng.standard_normal((naux, naux)), -1)  # only the upper triangle counts
    I = rng.standard_normal((nbf, nbf, naux))
    I = 0.5 * (I + I.transpose(1, 0, 2))
    return np.asfortranarray(G), np.asfortranarray(I)


def _download_b(bt, nbf, naux):
    # b_pq = C5^T b_l C5 with C = identity and nbf5 = nbf is b itself (exact in FP64)
    C = d.to_device(np.asfortranarray(np.eye(nbf)))
    out = torch.zeros(nbf * nbf * naux, dtype=torch.float64, device="cuda")
    d.transform_dev(C, bt, nbf, out=out)
    torch.cuda.synchronize()
    return out.cpu().numpy().reshape(nbf, nbf, naux, order="F")


@pytest.mark.parametrize("nbf,naux,negative,asym", [(13, 29, 0, False), (24, 116, 3, False), (40, 64, 0, True),
                                                     (96, 200, 5, True), (16, 1, 0, False), (20, 333, 2, True),
                                                     (24, 1024, 0, False)])
def test_iaux_matches_oracle(cuda_ctx, nbf, naux, negative, asym):
    G, I = _inputs(nbf, naux, nbf + naux, negative, asym)
    bt = d.Iaux_gpu(G, I, "fp64", cuda_ctx)
    b = _download_b(bt, nbf, naux)
    b0 = integrals.iaux(G, I)
    assert rel(b, b0) <= 1e-10
    bt.free()


def test_iaux_feeds_the_lagrangian(cuda_ctx):
    """The job from donof_iaux is a regular RI tensor: the Lagrangian from it equals
    the one from uploading the oracle's b."""
    from donof_b200 import workload
    nbf, naux = 24, 116
    G, I = _inputs(nbf, naux, 7)
    wl = workload.synthetic(nbf=nbf, naux=naux, nbeta=5, ncwo=3, seed=3)
    p = wl.p
    b1 = d.Iaux_gpu(G, I, "fp64", cuda_ctx)
    b2 = d.eris_to_gpu(integrals.iaux(G, I), "fp64", cuda_ctx)
    e1, h1 = d.compute_Lagrange2(wl.C, wl.n, wl.H, b1, wl.cj12, wl.ck12, p.nalpha, p.nbeta)
    e2, h2 = d.compute_Lagrange2(wl.C, wl.n, wl.H, b2, wl.cj12, wl.ck12, p.nalpha, p.nbeta)
    assert rel(e1, e2) <= 1e-10 and rel(h1, h2) <= 1e-12
    b1.free()
    b2.free()


def test_iaux_rejects_bad_shapes(cuda_ctx):
    with pytest.raises(ValueError):
        d.Iaux_gpu(np.eye(5), np.zeros((4, 4, 6)), "fp64", cuda_ctx)


def test_iaux_with_repeated_eigenvalues(cuda_ctx):
    """Degenerate eigenvalues (a multiple of the identity plus a low-rank term):
    G^{-1/2} is unique even though the eigenvectors are not."""
    nbf, naux = 12, 80
    rng = np.random.default_rng(11)
    U = np.linalg.qr(rng.standard_normal((naux, 3)))[0]
    G = np.asfortranarray(2.0 * np.eye(naux) + (U * np.array([1.0, 1.0, 3.0])) @ U.T)
    I = rng.standard_normal((nbf, nbf, naux))
    I = np.asfortranarray(0.5 * (I + I.transpose(1, 0, 2)))
    bt = d.Iaux_gpu(G, I, "fp64", cuda_ctx)
    b = _download_b(bt, nbf, naux)
    assert rel(b, integrals.iaux(G, I)) <= 1e-10
    bt.free()
