"""donof_b200 -- B200 (sm_100a) RI hot path of DoNOF.jl's GNOF energy.

The compute path is libdonofb200.so (hand-written CUDA for sm_100a behind a
C ABI, include/donof_b200.h); this package is the host-side mirror of the
reference's GPU-extension interface plus the host occupation layer.
"""
from . import _lib
from .api import (Batch, BatchQueue, BTensor, OrbStepHost, Context, Iaux, Iaux_gpu, JKH_MO, JKH_MO_dev, calcorbg, compute_Lagrange2,
                  compute_Lagrange2_dev, computeJKH_MO, default_context, eris_to_gpu, from_device, host_pinned,
                  launch_count, orbopt, orbopt_adabelief, orbopt_dev, orbopt_adam, orbopt_demon, orbopt_yogi, rotate_orbital,
                  rotate_orbital_dev, t1_dev, to_device, transform_dev)
from .param import Param

__all__ = [
    "Batch", "BatchQueue", "BTensor", "OrbStepHost", "Context", "Iaux", "Iaux_gpu", "JKH_MO", "JKH_MO_dev", "Param", "calcorbg", "compute_Lagrange2",
    "compute_Lagrange2_dev", "computeJKH_MO", "default_context", "eris_to_gpu", "from_device", "host_pinned",
    "launch_count", "orbopt", "orbopt_dev", "transform_dev", "orbopt_adabelief", "orbopt_adam", "orbopt_demon", "orbopt_yogi", "rotate_orbital",
    "rotate_orbital_dev", "t1_dev", "to_device",
]
