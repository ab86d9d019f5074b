"""ctypes binding of libdonofb200.so (the C ABI declared in include/donof_b200.h).

The library is built in-tree next to this file.  There is no fallback: if the
shared library is missing or a symbol is absent, loading raises.
"""
from __future__ import annotations

import ctypes as ct
import os
from pathlib import Path

LIB_NAME = "libdonofb200.so"
LIB_PATH = Path(__file__).resolve().parent / LIB_NAME

OK = 0
ERR_ARG = 1
ERR_CUDA = 2
ERR_OOM = 3
ERR_STATE = 4
ERR_NOT_CONVERGED = 5
ERR_TIMEOUT = 6

# bits of donof_error_flags
FAIL_MBAR = 1
FAIL_BARRIER = 2
FAIL_NONFINITE = 4

PREC_FP64 = 0
PREC_MIXED = 1

ORB_ADAM = 0
ORB_ADABELIEF = 1
ORB_YOGI = 2
ORB_DEMON = 3
ORB_METHODS = {"ADAM": ORB_ADAM, "ADABelief": ORB_ADABELIEF, "YOGI": ORB_YOGI, "Demon": ORB_DEMON}

_dp = ct.POINTER(ct.c_double)
_ip = ct.POINTER(ct.c_int)
_vp = ct.c_void_p
_i = ct.c_int

# name -> (restype, argtypes); mirrors include/donof_b200.h one to one.
SIGNATURES = {
    "donof_version": (_i, []),
    "donof_status_string": (ct.c_char_p, [_i]),
    "donof_last_error": (ct.c_char_p, [_vp]),
    "donof_create": (_i, [_i, ct.POINTER(_vp)]),
    "donof_destroy": (_i, [_vp]),
    "donof_set_stream": (_i, [_vp, _vp]),
    "donof_get_stream": (_vp, [_vp]),
    "donof_set_cta_limit": (_i, [_vp, _i]),
    "donof_synchronize": (_i, [_vp]),
    "donof_b_upload": (_i, [_vp, _vp, _i, _i, _i, ct.POINTER(_vp)]),
    "donof_b_attach": (_i, [_vp, _vp, _i, _i, _i, ct.POINTER(_vp)]),
    "donof_iaux": (_i, [_vp, _vp, _vp, _i, _i, _i, ct.POINTER(_vp)]),
    "donof_job_free": (_i, [_vp]),
    "donof_job_set_precision": (_i, [_vp, _i]),
    "donof_job_device_bytes": (ct.c_size_t, [_vp]),
    "donof_occupations": (_i, [_vp, _vp, _vp, _vp]),
    "donof_coupling": (_i, [_vp, _vp, _vp, _vp]),
    "donof_occ_energy": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "donof_occ_cg_dev": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, ct.c_double, _i, _vp]),
    "donof_occ_cg": (_i, [_vp, _vp, _vp, _vp, _vp, ct.c_double, _i, _vp, _vp, _vp]),
    "donof_energy": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "donof_server_create": (_i, [_i, ct.c_size_t, _i, ct.POINTER(_vp)]),
    "donof_server_submit": (_i, [_vp, _vp, _vp, _vp, ct.POINTER(ct.c_ulonglong)]),
    "donof_server_poll": (_i, [_vp, ct.c_ulonglong, _vp, _ip]),
    "donof_server_wait": (_i, [_vp, ct.c_ulonglong, _vp]),
    "donof_server_cancel": (_i, [_vp, ct.c_ulonglong]),
    "donof_server_destroy": (_i, [_vp]),
    "donof_lagrange2": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _i, _i, _i, _vp, _vp, _vp]),
    "donof_lagrange2_dev": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _i, _i, _i, _vp, _vp, _vp]),
    "donof_lagrange2_prec_dev": (_i, [_vp, _i, _vp, _vp, _vp, _vp, _vp, _i, _i, _i, _vp, _vp, _vp]),
    "donof_lagrange2_noalloc_dev": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _i, _i, _i, _vp, _vp, _vp]),
    "donof_lagrange2_partial_dev": (_i, [_vp, _vp, _vp, _vp, _vp, _i, _i, _i, _vp]),
    "donof_lagrange2_finish_dev": (_i, [_vp, _vp, _vp, _vp, _i, _vp, _vp, _vp, _vp]),
    "donof_jkh_mo": (_i, [_vp, _vp, _vp, _i, _vp, _vp, _vp]),
    "donof_jkh_mo_dev": (_i, [_vp, _vp, _vp, _i, _vp, _vp, _vp]),
    "donof_jkh_mo_prec_dev": (_i, [_vp, _i, _vp, _vp, _i, _vp, _vp, _vp]),
    "donof_rotate": (_i, [_vp, _vp, _i, _i, _vp, _vp]),
    "donof_rotate_dev": (_i, [_vp, _vp, _i, _i, _vp, _vp]),
    "donof_orbgrad": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _i, _i, _i, _vp]),
    "donof_orbopt_dev": (_i, [_vp, _i, _vp, _vp, _vp, _vp, _i, _i, _i, _dp, _ip, ct.c_double, _vp, _dp,
                              _ip, _ip]),
    "donof_transform_dev": (_i, [_vp, _i, _vp, _i, _vp]),
    "donof_launch_count": (ct.c_ulonglong, []),
    "donof_autotune_entries": (_i, []),
    "donof_job_error_flag": (_i, [_vp, _ip]),
    "donof_error_flags": (_i, [_vp, _ip]),
    "donof_set_wait_limit": (_i, [_vp, ct.c_longlong]),
    "donof_profile_enable": (_i, [_vp, _i]),
    "donof_profile_last_ms": (_i, [_vp, ct.POINTER(ct.c_float)]),
    "donof_mixed_tmp_dev": (_i, [_vp, _vp, _i, _vp]),
    "donof_orb_step_host": (_i, [_i, _i, _i, ct.c_double, _vp, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp]),
    # integral front end
    "donof_basis_create": (_i, [_i, _vp, _vp, _vp, _vp, _vp, _i, ct.POINTER(_vp)]),
    "donof_basis_nbf": (_i, [_vp]),
    "donof_basis_free": (_i, [_vp]),
    "donof_int1e": (_i, [_vp, _i, _vp, _vp, _vp, _vp, _vp]),
    "donof_int2c2e": (_i, [_vp, _vp]),
    "donof_int3c2e": (_i, [_vp, _vp, _vp]),
    "donof_int3c2e_dev": (_i, [_vp, _vp, _vp, _vp]),
    "donof_int4c2e": (_i, [_vp, _vp]),
    "donof_job_set_fp64_tc": (_i, [_vp, _i]),
    "donof_job_fp64_tc": (_i, [_vp]),
    "donof_t1_dev": (_i, [_vp, _vp, _i, _vp]),
    "donof_orbopt": (_i, [_vp, _i, _vp, _vp, _vp, _vp, _i, _i, _i, _dp, _ip, ct.c_double, _vp, _dp,
                          _ip, _ip]),
    "donof_batch_create": (_i, [_vp, _i, _vp, ct.POINTER(_vp)]),
    "donof_batch_destroy": (_i, [_vp]),
    "donof_batch_device_bytes": (ct.c_size_t, [_vp]),
    "donof_batch_orbopt": (_i, [_vp, _i, _vp]),
    "donof_batch_lagrange2": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "donof_batch_energy": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "donof_batch_queue_create": (_i, [_vp]),
    "donof_batch_queue_push": (_i, [_vp, _vp, _vp]),
    "donof_batch_queue_close": (_i, [_vp]),
    "donof_batch_queue_poll": (_i, [_vp, ct.c_ulonglong, _i, _vp, _vp, _vp]),
    "donof_batch_queue_destroy": (_i, [_vp]),
    "donof_batch_serve": (_i, [_vp, _vp]),
    "donof_batch_set_precision": (_i, [_vp, _i]),
}


class DonofError(RuntimeError):
    """A libdonofb200 call returned a non-zero status."""

    def __init__(self, status: int, message: str):
        super().__init__(f"libdonofb200 status {status}: {message}")
        self.status = status


_lib = None


def load(path: str | os.PathLike | None = None) -> ct.CDLL:
    """Load libdonofb200.so (once) and declare every exported signature."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path is not None else LIB_PATH
    if not p.exists():
        raise FileNotFoundError(
            f"{p} is missing: build the CUDA library first (python -c 'import __graft_entry__ as g; g.build()')")
    lib = ct.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)  # AttributeError if the symbol is absent
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def check(status: int, ctx=None) -> None:
    if status != OK:
        lib = load()
        msg = lib.donof_last_error(ctx)
        raise DonofError(status, (msg or b"").decode(errors="replace"))
