"""B200-native ARS(2,2,2) IMEX step for 2-D resistive MHD (sm_100a, FP64).

The product is the shared library ``libmhd_b200.so`` (CUDA kernels + the C ABI of
``include/mhd_b200.h``); this package is its Python mirror:

* :class:`Context` -- one device-resident simulation (set_state / step / run / cfl_dt / divb);
* :class:`Batch` -- many independent simulations of uneven sizes stepped together;
* :class:`Adjoint` -- a differentiable fixed-dt trajectory (hand-written adjoint kernels); its
  torch.autograd binding is :mod:`magnetohydrodynamics_simulator_b200.autograd`;
* :mod:`problems` -- the benchmark initial conditions.
"""
from .capi import (  # noqa: F401
    CT_REFERENCE,
    CT_TRUE_ABS,
    FIELDS,
    LAYOUT_DENSE,
    LAYOUT_PADDED,
    Adjoint,
    Batch,
    Context,
    MHDError,
    ars_gamma,
    device_available,
    load_library,
)
from . import problems  # noqa: F401

__all__ = [
    "Adjoint",
    "Batch",
    "Context",
    "MHDError",
    "FIELDS",
    "LAYOUT_DENSE",
    "LAYOUT_PADDED",
    "CT_REFERENCE",
    "CT_TRUE_ABS",
    "ars_gamma",
    "device_available",
    "load_library",
    "problems",
]
