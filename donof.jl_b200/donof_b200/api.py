"""Host-side mirror of DoNOF.jl's GPU plugin interface (ext/DoNOFGPUExt.jl),
driving libdonofb200 through its C ABI.

Function names, argument order and meaning follow the reference methods they
replace; arrays are FP64 in Julia (column-major) layout:

  numpy inputs   : Fortran-ordered arrays indexed like Julia, e.g. C[m, p],
                   b[m, n, l] (any order is accepted and converted).
  torch inputs   : CUDA tensors holding the same column-major memory, i.e.
                   with the index order reversed (b as (naux, nbf, nbf)),
                   see ``to_device`` / ``from_device``.

Every call goes to the CUDA library; there is no CPU code path for the hot
contractions, and a missing library raises at import of ``_lib``.
"""
from __future__ import annotations

import ctypes as ct
from typing import Optional

import numpy as np

from . import _lib
from .param import Param

try:  # torch is optional for the host-buffer entry points
    import torch
except Exception:  # pragma: no cover
    torch = None


def _ptr(a) -> int:
    if a is None:
        return None
    if torch is not None and isinstance(a, torch.Tensor):
        if not a.is_cuda or a.dtype != torch.float64 or not a.is_contiguous():
            raise ValueError("device arrays must be contiguous float64 CUDA tensors")
        return a.data_ptr()
    return a.ctypes.data


def _f64(a) -> np.ndarray:
    return np.asfortranarray(np.asarray(a, dtype=np.float64))


def to_device(a: np.ndarray, device="cuda"):
    """Julia-layout numpy array -> CUDA tensor with the same memory order."""
    a = _f64(a)
    return torch.from_numpy(np.ascontiguousarray(a.T)).to(device)


def from_device(t) -> np.ndarray:
    """Inverse of ``to_device``."""
    return np.asfortranarray(t.detach().cpu().numpy().T)


class Context:
    """One libdonofb200 context (device + CUDA stream)."""

    def __init__(self, device: int = 0, torch_stream: bool = True):
        self.lib = _lib.load()
        h = ct.c_void_p()
        _lib.check(self.lib.donof_create(int(device), ct.byref(h)), None)
        self.handle = h
        self.device = device
        if torch_stream and torch is not None and torch.cuda.is_available():
            # share torch's current stream so torch events time the work
            self.set_stream(torch.cuda.current_stream(device).cuda_stream)

    def set_stream(self, stream_handle: int) -> None:
        self.check(self.lib.donof_set_stream(self.handle, ct.c_void_p(stream_handle)))

    def set_cta_limit(self, max_ctas: int) -> None:
        """Most CTAs this context's persistent and cooperative kernels may use
        (0: one per SM)."""
        self.check(self.lib.donof_set_cta_limit(self.handle, int(max_ctas)))

    def check(self, status: int) -> None:
        _lib.check(status, self.handle)

    def error_flags(self) -> int:
        """Failures the context's kernels recorded since the last read (bit mask:
        _lib.FAIL_MBAR, FAIL_BARRIER, FAIL_NONFINITE), cleared by the read;
        synchronises the context stream."""
        f = ct.c_int()
        self.check(self.lib.donof_error_flags(self.handle, ct.byref(f)))
        return f.value

    def set_wait_limit(self, cycles: int) -> None:
        """Cycle budget of every bounded wait in the kernels launched from now
        on (0: the built-in one); a tiny budget drives the failure path."""
        self.check(self.lib.donof_set_wait_limit(self.handle, int(cycles)))

    def synchronize(self) -> None:
        self.check(self.lib.donof_synchronize(self.handle))

    def close(self) -> None:
        """Free every job of this context, then the context itself (a job must
        never outlive its context: the library dereferences it on free)."""
        if getattr(self, "handle", None):
            for job in list(getattr(self, "_jobs", ())):
                job.free()
            self.lib.donof_destroy(self.handle)
            self.handle = None

    def _register(self, job) -> None:
        if not hasattr(self, "_jobs"):
            import weakref
            self._jobs = weakref.WeakSet()
        self._jobs.add(job)

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass


_default_ctx: Optional[Context] = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


class BTensor:
    """The RI tensor b[m, n, l] resident on the device (a libdonofb200 job);
    the counterpart of the CuArray that eris_to_gpu returns."""

    def __init__(self, ctx: Context, handle, nbf: int, naux: int, precision: int, keep=None):
        self.ctx, self.handle, self.nbf, self.naux, self.precision = ctx, handle, nbf, naux, precision
        self._keep = keep  # keeps an attached device tensor alive
        ctx._register(self)

    @property
    def shape(self):
        return (self.nbf, self.nbf, self.naux)

    def set_precision(self, precision) -> None:
        """Switch the precision of the calls that take none explicitly ("fp64" is
        always allowed; "mixed" needs a job uploaded as mixed)."""
        prec = _prec(precision)
        self.ctx.check(self.ctx.lib.donof_job_set_precision(self.handle, prec))
        self.precision = prec

    def set_fp64_tc(self, enable: bool = True) -> None:
        """Run the FP64 form's first contraction (tmp_l = b_l C5) on the tensor
        cores from int8 digit slices of b (made now, 7/8 of b's FP64 size), or
        back on the FP64 GEMM (enable=False frees the slices)."""
        self.ctx.check(self.ctx.lib.donof_job_set_fp64_tc(self.handle, 1 if enable else 0))

    @property
    def fp64_tc(self) -> bool:
        return bool(self.ctx.lib.donof_job_fp64_tc(self.handle))

    def device_bytes(self) -> int:
        return int(self.ctx.lib.donof_job_device_bytes(self.handle))

    def free(self) -> None:
        # the context frees its jobs before it is destroyed; after that the handle is gone
        if self.handle and getattr(self.ctx, "handle", None):
            self.ctx.lib.donof_job_free(self.handle)
        self.handle = None

    def __del__(self):  # pragma: no cover
        try:
            self.free()
        except Exception:
            pass


def _prec(precision) -> int:
    if precision in ("fp64", _lib.PREC_FP64, None):
        return _lib.PREC_FP64
    if precision in ("mixed", _lib.PREC_MIXED):
        return _lib.PREC_MIXED
    raise ValueError(f"unknown precision {precision!r}")


def eris_to_gpu(b, precision="fp64", ctx: Optional[Context] = None) -> BTensor:
    """Upload (numpy) or attach (CUDA tensor) the RI tensor b
    (ext/DoNOFGPUExt.jl:36-50)."""
    ctx = ctx or default_context()
    prec = _prec(precision)
    h = ct.c_void_p()
    if torch is not None and isinstance(b, torch.Tensor):
        naux, nbf, nbf2 = b.shape
        assert nbf == nbf2
        ctx.check(ctx.lib.donof_b_attach(ctx.handle, ct.c_void_p(_ptr(b)), nbf, naux, prec, ct.byref(h)))
        return BTensor(ctx, h, nbf, naux, prec, keep=b)
    b = _f64(b)
    nbf, nbf2, naux = b.shape
    assert nbf == nbf2
    ctx.check(ctx.lib.donof_b_upload(ctx.handle, ct.c_void_p(b.ctypes.data), nbf, naux, prec, ct.byref(h)))
    return BTensor(ctx, h, nbf, naux, prec)


def Iaux_gpu(G, I, precision="fp64", ctx: Optional[Context] = None) -> BTensor:
    """b = I G^{-1/2} built on the device from the two-centre integrals G
    (naux x naux; its upper triangle, Symmetric(G)) and the three-centre
    integrals I (nbf x nbf x naux), kept there as the job's RI tensor
    (Iaux / Iaux_gpu, src/integrals.jl:68-91, ext/DoNOFGPUExt.jl:9-33,
    followed by eris_to_gpu)."""
    ctx = ctx or default_context()
    prec = _prec(precision)
    G = _f64(G)
    I = _f64(I)
    nbf, nbf2, naux = I.shape
    if nbf != nbf2 or G.shape != (naux, naux):
        raise ValueError(f"I must be nbf x nbf x naux and G naux x naux (got {I.shape}, {G.shape})")
    h = ct.c_void_p()
    ctx.check(ctx.lib.donof_iaux(ctx.handle, ct.c_void_p(G.ctypes.data), ct.c_void_p(I.ctypes.data), nbf, naux,
                                 prec, ct.byref(h)))
    return BTensor(ctx, h, nbf, naux, prec)


Iaux = Iaux_gpu


def host_pinned(shape) -> np.ndarray:
    """Zeroed Fortran-ordered FP64 numpy array in page-locked host memory (the
    storage of a pinned torch tensor, kept alive by the array).  The host-buffer
    entry points DMA such arrays directly, without a staging copy."""
    shape = (shape,) if np.isscalar(shape) else tuple(shape)
    t = torch.zeros(int(np.prod(shape)), dtype=torch.float64, pin_memory=True)
    return t.numpy().reshape(shape, order="F")


def _out(out, shape):
    if out is None:
        return np.zeros(shape, order="F")
    if out.shape != shape or out.dtype != np.float64 or not out.flags.f_contiguous:
        raise ValueError(f"output array must be Fortran-ordered float64 of shape {shape}")
    return out


def compute_Lagrange2(C, n, H, b: BTensor, cj12, ck12, nalpha: int, nbeta: int, return_energy=False,
                      out=None):
    """elag, H_mat = compute_Lagrange2(C, n, H, b, cj12, ck12, nalpha, nbeta)
    (src/utils.jl:1-59; ext/DoNOFGPUExt.jl:150-245).  Host arrays in and out;
    ``out=(elag, H_mat)`` writes into caller arrays (page-locked ones from
    ``host_pinned`` skip the staging copy)."""
    C, n, H, cj12, ck12 = _f64(C), _f64(n), _f64(H), _f64(cj12), _f64(ck12)
    nbf, nbf5 = b.nbf, n.shape[0]
    elag = _out(None if out is None else out[0], (nbf, nbf))
    Hmat = _out(None if out is None else out[1], (nbf, nbf5))
    E = np.zeros(1)
    b.ctx.check(b.ctx.lib.donof_lagrange2(b.handle, _ptr(C), _ptr(n), _ptr(H), _ptr(cj12), _ptr(ck12),
                                          nbf5, int(nalpha), int(nbeta), _ptr(elag), _ptr(Hmat), _ptr(E)))
    if return_energy:
        return elag, Hmat, float(E[0])
    return elag, Hmat


def compute_Lagrange2_dev(C, n, H, b: BTensor, cj12, ck12, nalpha: int, nbeta: int, elag, Hmat, E=None,
                          precision=None):
    """Device-pointer form: all arrays are CUDA tensors in Julia layout; only
    enqueues work on the context stream."""
    prec = b.precision if precision is None else _prec(precision)
    nbf5 = n.shape[0]
    b.ctx.check(b.ctx.lib.donof_lagrange2_prec_dev(b.handle, prec, _ptr(C), _ptr(n), _ptr(H), _ptr(cj12),
                                                   _ptr(ck12), nbf5, int(nalpha), int(nbeta), _ptr(elag),
                                                   _ptr(Hmat), _ptr(E)))


def JKH_MO(C, H, b: BTensor, nbf: int, nbf5: int, nbfaux: int):
    """J_MO, K_MO, H_core = JKH_MO(C, H, b, nbf, nbf5, nbfaux)
    (src/integrals.jl:144-172; ext/DoNOFGPUExt.jl:63-94)."""
    if nbf != b.nbf or nbfaux != b.naux:
        raise ValueError("nbf/nbfaux do not match the b tensor")
    C, H = _f64(C), _f64(H)
    J = np.zeros((nbf5, nbf5), order="F")
    K = np.zeros((nbf5, nbf5), order="F")
    Hc = np.zeros(nbf5)
    b.ctx.check(b.ctx.lib.donof_jkh_mo(b.handle, _ptr(C), _ptr(H), int(nbf5), _ptr(J), _ptr(K), _ptr(Hc)))
    return J, K, Hc


def JKH_MO_dev(C, H, b: BTensor, nbf5: int, J, K, Hcore, precision=None):
    prec = b.precision if precision is None else _prec(precision)
    b.ctx.check(b.ctx.lib.donof_jkh_mo_prec_dev(b.handle, prec, _ptr(C), _ptr(H), int(nbf5), _ptr(J), _ptr(K),
                                                _ptr(Hcore)))


def computeJKH_MO(C, H, b: BTensor, p: Param):
    """src/integrals.jl:131-140 (RI branch); ext/DoNOFGPUExt.jl:52-61."""
    return JKH_MO(C, H, b, p.nbf, p.nbf5, p.nbfaux)


def rotate_orbital(y, C, p: Param, ctx: Optional[Context] = None, out=None):
    """C exp(Y(y)) in FP64 (src/utils.jl:499-521; replaces ext/DoNOFGPUExt.jl:355-382).
    ``out`` receives the result when given (it must not be C itself)."""
    ctx = ctx or default_context()
    y, C = _f64(y), _f64(C)
    if y.shape[0] != p.nvar:
        raise ValueError(f"y has {y.shape[0]} entries, nvar = {p.nvar}")
    Cn = _out(out, C.shape)
    if Cn is C:
        raise ValueError("rotate_orbital cannot write its result over C")
    ctx.check(ctx.lib.donof_rotate(ctx.handle, _ptr(y), p.nbf, p.nbf5, _ptr(C), _ptr(Cn)))
    return Cn


def rotate_orbital_dev(y, C, Cnew, nbf: int, nbf5: int, ctx: Optional[Context] = None):
    ctx = ctx or default_context()
    ctx.check(ctx.lib.donof_rotate_dev(ctx.handle, _ptr(y), nbf, nbf5, _ptr(C), _ptr(Cnew)))


def calcorbg(y, n, cj12, ck12, C, H, b: BTensor, p: Param):
    """Packed orbital gradient at y (src/pnof.jl:1389-1407)."""
    n, cj12, ck12, C, H = _f64(n), _f64(cj12), _f64(ck12), _f64(C), _f64(H)
    yv = None if y is None else _f64(y)
    g = np.zeros(p.nvar)
    b.ctx.check(b.ctx.lib.donof_orbgrad(b.handle, _ptr(yv), _ptr(C), _ptr(n), _ptr(H), _ptr(cj12), _ptr(ck12),
                                        p.nbf5, p.nalpha, p.nbeta, _ptr(g)))
    return g


class OrbStepHost:
    """The host side of the reference's optimiser loop (src/minimization.jl:390-412)
    for a caller that drives it through rotate_orbital + compute_Lagrange2:
    ``y = step(elag)`` packs calcorbg's gradient and applies the update of the
    next iteration in compiled code (donof_orb_step_host), keeping m, v, vmax.
    ``alloc`` makes the arrays (e.g. host_pinned, so that y is DMA'd directly);
    y is overwritten by the next step; ``gmax`` holds max|g| of the last one."""

    def __init__(self, nbf: int, nbf5: int, method: str = "ADAM", alpha: float = 0.01, maxloop: int = 10,
                 alloc=np.zeros):
        self.lib = _lib.load()
        self.nbf, self.nbf5, self.method = nbf, nbf5, _lib.ORB_METHODS[method]
        self.alpha, self.maxloop = alpha, maxloop
        nvar = nbf5 * nbf - nbf5 * (nbf5 + 1) // 2
        self.g, self.m, self.v, self.vmax = (np.zeros(nvar) for _ in range(4))
        self.y = alloc(nvar)
        self.it = 0
        self.gmax = ct.c_double()

    def reset(self) -> None:
        for a in (self.m, self.v, self.vmax):
            a[:] = 0.0
        self.it = 0

    def step(self, elag) -> np.ndarray:
        elag = _f64(elag)
        if elag.shape != (self.nbf, self.nbf):
            raise ValueError(f"elag must be {self.nbf} x {self.nbf}")
        self.it += 1
        _lib.check(self.lib.donof_orb_step_host(self.method, self.it, self.maxloop, float(self.alpha), _ptr(elag),
                                                self.nbf, self.nbf5, _ptr(self.g), _ptr(self.m), _ptr(self.v),
                                                _ptr(self.vmax), _ptr(self.y), ct.byref(self.gmax)))
        return self.y


def orbopt(gamma, C, H, b: BTensor, p: Param, method: Optional[str] = None):
    """One orbital-optimiser call, device resident (src/minimization.jl:242-630).
    Returns (E, C, nit, success) and updates p.alpha / p.maxloop like the reference."""
    from . import gnof

    method = method or p.orb_method
    n, _ = gnof.occupations(gamma, p)
    cj12, ck12 = gnof.coupling(n, p)
    Cio = np.array(_f64(C), copy=True, order="F")
    alpha = ct.c_double(p.alpha)
    maxloop = ct.c_int(p.maxloop)
    E = ct.c_double()
    nit = ct.c_int()
    ok = ct.c_int()
    n, cj12, ck12, H = _f64(n), _f64(cj12), _f64(ck12), _f64(H)
    b.ctx.check(b.ctx.lib.donof_orbopt(b.handle, _lib.ORB_METHODS[method], _ptr(n), _ptr(cj12), _ptr(ck12),
                                       _ptr(H), p.nbf5, p.nalpha, p.nbeta, ct.byref(alpha), ct.byref(maxloop),
                                       float(p.threshgorb), _ptr(Cio), ct.byref(E), ct.byref(nit),
                                       ct.byref(ok)))
    p.alpha = alpha.value
    p.maxloop = maxloop.value
    return E.value, Cio, nit.value, bool(ok.value)


def orbopt_dev(method: str, n, cj12, ck12, H, C, b: BTensor, p: Param, alpha: float, maxloop: int,
               threshgorb: float):
    """Device-pointer optimiser call: n, cj12, ck12, H, C are CUDA tensors in
    Julia layout; C is updated in place.  Returns (E, nit, success, alpha, maxloop)."""
    a, ml = ct.c_double(alpha), ct.c_int(maxloop)
    E, nit, ok = ct.c_double(), ct.c_int(), ct.c_int()
    b.ctx.check(b.ctx.lib.donof_orbopt_dev(b.handle, _lib.ORB_METHODS[method], _ptr(n), _ptr(cj12), _ptr(ck12),
                                           _ptr(H), n.shape[0], p.nalpha, p.nbeta, ct.byref(a), ct.byref(ml),
                                           float(threshgorb), _ptr(C), ct.byref(E), ct.byref(nit), ct.byref(ok)))
    return E.value, nit.value, bool(ok.value), a.value, ml.value


class _BatchShape(ct.Structure):
    _fields_ = [("job", ct.c_void_p), ("nbf5", ct.c_int), ("nalpha", ct.c_int), ("nbeta", ct.c_int)]


class _BatchItem(ct.Structure):
    _fields_ = [("n", ct.c_void_p), ("cj12", ct.c_void_p), ("ck12", ct.c_void_p), ("H", ct.c_void_p),
                ("C", ct.c_void_p), ("alpha", ct.c_double), ("maxloop", ct.c_int), ("threshgorb", ct.c_double),
                ("E", ct.c_double), ("nit", ct.c_int), ("success", ct.c_int)]


class Batch:
    """Several jobs optimised together (donof_batch_*): every gradient step of
    all jobs runs as one grouped launch per stage, the loop as one captured
    graph.  ``jobs`` are FP64 BTensors of one context, ``params`` the matching
    Param objects (nbf5, nalpha, nbeta are read).  DoNOF.jl optimises one
    molecule per call; each job here gives what ``orbopt_dev`` gives alone."""

    def __init__(self, jobs, params, ctx: Optional[Context] = None):
        if len(jobs) != len(params) or not jobs:
            raise ValueError("one Param per job, at least one job")
        self.ctx = ctx or jobs[0].ctx
        self.jobs, self.params = list(jobs), list(params)
        shapes = (_BatchShape * len(jobs))()
        for s, b, p in zip(shapes, jobs, params):
            s.job, s.nbf5, s.nalpha, s.nbeta = b.handle.value if hasattr(b.handle, "value") else b.handle, \
                p.nbf5, p.nalpha, p.nbeta
        h = ct.c_void_p()
        self.ctx.check(self.ctx.lib.donof_batch_create(self.ctx.handle, len(jobs), shapes, ct.byref(h)))
        self.handle = h

    def __len__(self):
        return len(self.jobs)

    def device_bytes(self) -> int:
        return int(self.ctx.lib.donof_batch_device_bytes(self.handle))

    def _items(self, n, cj12, ck12, H, C, alpha=None, maxloop=None, threshgorb=None):
        items = (_BatchItem * len(self.jobs))()
        for j, it in enumerate(items):
            it.n, it.cj12, it.ck12, it.H, it.C = (_ptr(x[j]) for x in (n, cj12, ck12, H, C))
            if alpha is not None:
                it.alpha, it.maxloop, it.threshgorb = float(alpha[j]), int(maxloop[j]), float(threshgorb[j])
        return items

    def orbopt(self, method: str, n, cj12, ck12, H, C, alpha, maxloop, threshgorb):
        """Optimiser loop of every job; per-job lists of CUDA tensors (Julia
        layout; C updated in place) and scalars.  Returns one
        (E, nit, success, alpha, maxloop) tuple per job."""
        items = self._items(n, cj12, ck12, H, C, alpha, maxloop, threshgorb)
        self.ctx.check(self.ctx.lib.donof_batch_orbopt(self.handle, _lib.ORB_METHODS[method], items))
        return [(it.E, it.nit, bool(it.success), it.alpha, it.maxloop) for it in items]

    def lagrange2(self, n, cj12, ck12, H, C, elag, Hmat):
        """compute_Lagrange2 of every job at C[j] into elag[j], Hmat[j] (CUDA
        tensors); returns the E_elec of each job."""
        items = self._items(n, cj12, ck12, H, C)
        k = len(self.jobs)
        pe = (ct.c_void_p * k)(*[_ptr(x) for x in elag])
        ph = (ct.c_void_p * k)(*[_ptr(x) for x in Hmat])
        E = (ct.c_double * k)()
        self.ctx.check(self.ctx.lib.donof_batch_lagrange2(self.handle, items, pe, ph, E))
        return list(E)

    def energy(self, Hs, Cs, gammas, maxit: Optional[int] = None, order: bool = True):
        """DoNOF.energy's alternation for every job (donof_batch_energy): each
        outer iteration runs the orbital optimisation of all jobs still going as
        one grouped call.  Host (numpy) H, C, gamma per job; updates each job's
        Param alpha / maxloop.  Returns one (C, gamma, n, result fields) per job."""
        k = len(self.jobs)
        prms = (_EnergyParams * k)()
        for prm, p in zip(prms, self.params):
            prm.occ = _occ_params(p)
            prm.orb_method = _lib.ORB_METHODS[p.orb_method]
            prm.maxit, prm.maxloop, prm.alpha = int(maxit or p.maxit), int(p.maxloop), float(p.alpha)
            prm.threshgorb, prm.threshgocc, prm.threshen = float(p.threshgorb), float(p.threshgocc), float(p.threshen)
            prm.order_subspaces = int(bool(order) and p.ipnof > 4)
            prm.occ_device = int(bool(getattr(p, "occ_device", False)))
        Hf = [_f64(H) for H in Hs]
        Cio = [np.array(_f64(C), copy=True, order="F") for C in Cs]
        gio = [np.array(g, dtype=np.float64, copy=True) for g in gammas]
        ns = [np.zeros(p.nbf5) for p in self.params]
        arr = lambda xs: (ct.c_void_p * k)(*[_ptr(x) for x in xs])
        res = (_EnergyResult * k)()
        self.ctx.check(self.ctx.lib.donof_batch_energy(self.handle, prms, arr(Hf), arr(Cio), arr(gio), arr(ns), res))
        out = []
        for j, p in enumerate(self.params):
            p.alpha, p.maxloop = prms[j].alpha, prms[j].maxloop
            out.append((Cio[j], gio[j], ns[j], {f: getattr(res[j], f) for f, _ in _EnergyResult._fields_}))
        return out

    def set_precision(self, precision) -> None:
        """The form of the batch's Lagrangian: "fp64", or "mixed" (the fused
        tcgen05 kernel for every job in one grouped launch; the jobs uploaded as
        mixed, nbf <= 256, nbf5 <= 64)."""
        self.ctx.check(self.ctx.lib.donof_batch_set_precision(self.handle, _prec(precision)))

    def serve(self, queue: "BatchQueue") -> None:
        """Continuous batching (donof_batch_serve): the batch's jobs are slots of
        their shapes; requests pushed into ``queue`` (also from other threads while
        this runs) take a free slot of their shape, every outer iteration advances
        all running requests as grouped launches, and a request returns as soon as
        it converges.  Returns once the queue is closed and every request has
        finished."""
        self.ctx.check(self.ctx.lib.donof_batch_serve(self.handle, queue.handle))

    def free(self) -> None:
        if getattr(self, "handle", None) and getattr(self.ctx, "handle", None):
            self.ctx.lib.donof_batch_destroy(self.handle)
        self.handle = None

    def __del__(self):  # pragma: no cover
        try:
            self.free()
        except Exception:
            pass


def transform_dev(C, b: BTensor, nbf5: int, out=None, precision=None):
    """b_pq^l = C5^T b_l C5 on the device (out: CUDA tensor or None)."""
    prec = b.precision if precision is None else _prec(precision)
    b.ctx.check(b.ctx.lib.donof_transform_dev(b.handle, prec, _ptr(C), int(nbf5), _ptr(out)))


def t1_dev(C, b: BTensor, nbf5: int, out):
    """tmp[m + nbf*q + nbf*nbf5*l] = sum_n b[m,n,l] C[n,q] of the FP64 form on the
    device (C and out: CUDA tensors; out holds nbf*nbf5*naux doubles)."""
    b.ctx.check(b.ctx.lib.donof_t1_dev(b.handle, _ptr(C), int(nbf5), _ptr(out)))


def launch_count() -> int:
    return int(_lib.load().donof_launch_count())


def orbopt_adam(gamma, C, H, b, p):
    return orbopt(gamma, C, H, b, p, "ADAM")


def orbopt_adabelief(gamma, C, H, b, p):
    return orbopt(gamma, C, H, b, p, "ADABelief")


def orbopt_yogi(gamma, C, H, b, p):
    return orbopt(gamma, C, H, b, p, "YOGI")


def orbopt_demon(gamma, C, H, b, p):
    return orbopt(gamma, C, H, b, p, "Demon")


# ---------------------------------------------------------------- occupation layer (host, native)
class _OccParams(ct.Structure):
    _fields_ = [("nbf5", ct.c_int), ("no1", ct.c_int), ("nbeta", ct.c_int), ("nalpha", ct.c_int),
                ("ncwo", ct.c_int), ("ista", ct.c_int), ("high_spin", ct.c_int), ("occ_method", ct.c_int),
                ("h_cut", ct.c_double)]


def _occ_params(p: Param) -> _OccParams:
    methods = {"Softmax": 0, "Trigonometric": 1}
    if p.occ_method not in methods:
        raise ValueError(f"occupation method {p.occ_method!r} is not supported")
    return _OccParams(p.nbf5, p.no1, p.nbeta, p.nalpha, p.ncwo, p.ista, int(bool(p.HighSpin)),
                      methods[p.occ_method], float(p.h_cut))


def occ_energy(gamma, J_MO, K_MO, H_core, p: Param, grad: bool = True):
    """calcocce (and calcoccg) in the library's native host code: (E, gradient or None)."""
    lib = _lib.load()
    prm = _occ_params(p)
    gamma = np.ascontiguousarray(gamma, dtype=np.float64)
    J, K = _f64(J_MO), _f64(K_MO)
    Hc = np.ascontiguousarray(H_core, dtype=np.float64)
    E = ct.c_double()
    g = np.zeros(p.nv) if grad else None
    _lib.check(lib.donof_occ_energy(ct.byref(prm), _ptr(gamma), _ptr(J), _ptr(K), _ptr(Hc), ct.byref(E),
                                    _ptr(g) if grad else None))
    return E.value, g


class _EnergyParams(ct.Structure):
    _fields_ = [("occ", _OccParams), ("orb_method", ct.c_int), ("maxit", ct.c_int), ("maxloop", ct.c_int),
                ("alpha", ct.c_double), ("threshgorb", ct.c_double), ("threshgocc", ct.c_double),
                ("threshen", ct.c_double), ("order_subspaces", ct.c_int), ("freeze_occ", ct.c_int),
                ("stop_rel_de", ct.c_double), ("occ_device", ct.c_int)]


class _EnergyResult(ct.Structure):
    _fields_ = [("E_elec", ct.c_double), ("iterations", ct.c_int), ("converged", ct.c_int),
                ("tot_it_orb", ct.c_int), ("tot_it_occ", ct.c_int), ("max_grad_orb", ct.c_double),
                ("norm_grad_occ", ct.c_double)]


def energy_loop(H, b: BTensor, p: Param, C, gamma, maxit: Optional[int] = None, freeze_occ: bool = False,
                order: bool = True, stop_rel_de: float = 0.0):
    """DoNOF.energy's orbital / occupation alternation in one native call
    (donof_energy), in the precision b is set to.  Updates p.alpha and
    p.maxloop like the reference.  Returns (C, gamma, n, elag, result fields,
    history rows (E, E_diff, max|g_orb|, |g_occ|, nit_orb, nit_occ))."""
    maxit = int(maxit or p.maxit)
    prm = _EnergyParams(_occ_params(p), _lib.ORB_METHODS[p.orb_method], maxit, int(p.maxloop), float(p.alpha),
                        float(p.threshgorb), float(p.threshgocc), float(p.threshen),
                        int(bool(order) and p.ipnof > 4), int(bool(freeze_occ)), float(stop_rel_de),
                        int(bool(getattr(p, "occ_device", False))))
    Cio = np.array(_f64(C), copy=True, order="F")
    g = np.array(gamma, dtype=np.float64, copy=True)
    n = np.zeros(p.nbf5)
    elag = np.zeros((p.nbf, p.nbf), order="F")
    hist = np.zeros((maxit, 6))
    res = _EnergyResult()
    Hf = _f64(H)  # kept alive across the call
    b.ctx.check(b.ctx.lib.donof_energy(b.handle, ct.byref(prm), _ptr(Hf), _ptr(Cio), _ptr(g), _ptr(n),
                                       _ptr(elag), _ptr(hist), ct.byref(res)))
    p.alpha = prm.alpha
    p.maxloop = prm.maxloop
    out = {f: getattr(res, f) for f, _ in _EnergyResult._fields_}
    return Cio, g, n, elag, out, hist[:res.iterations]


def occ_cg(gamma, J_MO, K_MO, H_core, p: Param, g_abstol: float, max_iter: int = 1000):
    """The conjugate-gradient minimisation of occoptr over gamma in native host
    code: (gamma, E, iterations, converged)."""
    lib = _lib.load()
    prm = _occ_params(p)
    x = np.array(gamma, dtype=np.float64, copy=True)
    J, K = _f64(J_MO), _f64(K_MO)
    Hc = np.ascontiguousarray(H_core, dtype=np.float64)
    E, nit, ok = ct.c_double(), ct.c_int(), ct.c_int()
    _lib.check(lib.donof_occ_cg(ct.byref(prm), _ptr(J), _ptr(K), _ptr(Hc), _ptr(x), float(g_abstol), int(max_iter),
                                ct.byref(E), ct.byref(nit), ct.byref(ok)))
    return x, E.value, nit.value, bool(ok.value)


class _BatchRequest(ct.Structure):
    _fields_ = [("job", ct.c_void_p), ("params", _EnergyParams), ("H", ct.c_void_p), ("C_inout", ct.c_void_p),
                ("gamma_inout", ct.c_void_p), ("n_out", ct.c_void_p)]


class BatchQueue:
    """Requests for ``Batch.serve`` (donof_batch_queue_*).  ``push`` copies the
    inputs into arrays the queue owns until the request is collected."""

    def __init__(self):
        self.lib = _lib.load()
        h = ct.c_void_p()
        _lib.check(self.lib.donof_batch_queue_create(ct.byref(h)), None)
        self.handle = h
        self._keep = {}

    def push(self, b: BTensor, H, C, gamma, p: Param, maxit: Optional[int] = None, order: bool = True) -> int:
        prm = _EnergyParams()
        prm.occ = _occ_params(p)
        prm.orb_method = _lib.ORB_METHODS[p.orb_method]
        prm.maxit, prm.maxloop, prm.alpha = int(maxit or p.maxit), int(p.maxloop), float(p.alpha)
        prm.threshgorb, prm.threshgocc, prm.threshen = float(p.threshgorb), float(p.threshgocc), float(p.threshen)
        prm.order_subspaces = int(bool(order) and p.ipnof > 4)
        prm.occ_device = int(bool(getattr(p, "occ_device", False)))
        Hf = _f64(H)
        Cio = np.array(_f64(C), copy=True, order="F")
        gio = np.array(gamma, dtype=np.float64, copy=True)
        n = np.zeros(p.nbf5)
        req = _BatchRequest(b.handle, prm, _ptr(Hf), _ptr(Cio), _ptr(gio), _ptr(n))
        t = ct.c_ulonglong()
        _lib.check(self.lib.donof_batch_queue_push(self.handle, ct.byref(req), ct.byref(t)), None)
        self._keep[t.value] = (b, Hf, Cio, gio, n)
        return t.value

    def close(self) -> None:
        _lib.check(self.lib.donof_batch_queue_close(self.handle), None)

    def poll(self, ticket: int, wait: bool = False):
        """None while running; else (C, gamma, n, result fields) -- or raises the
        request's error."""
        done, status, res = ct.c_int(), ct.c_int(), _EnergyResult()
        _lib.check(self.lib.donof_batch_queue_poll(self.handle, ct.c_ulonglong(ticket), 1 if wait else 0,
                                                   ct.byref(done), ct.byref(status), ct.byref(res)), None)
        if not done.value:
            return None
        _, _, Cio, gio, n = self._keep[ticket]
        if status.value != 0:
            raise _lib.DonofError(status.value, f"batch request {ticket} failed")
        return Cio, gio, n, {f: getattr(res, f) for f, _ in _EnergyResult._fields_}

    def wait(self, ticket: int):
        return self.poll(ticket, wait=True)

    def free(self) -> None:
        if getattr(self, "handle", None):
            self.lib.donof_batch_queue_destroy(self.handle)
        self.handle = None

    def __del__(self):  # pragma: no cover
        try:
            self.free()
        except Exception:
            pass
