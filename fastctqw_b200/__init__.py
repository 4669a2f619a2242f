"""fastctqw_b200: continuous-time quantum walks on NVIDIA B200 (sm_100a).

A from-scratch B200 implementation of the hot path of Crinton/FastCTQW: the dense
propagator U = expm(-iHt) by scaling and squaring with Pade approximants, and psi = U psi0.
The package mirrors the reference's Python API (``Ctqw``, ``Operator``, ``State``,
``fastexpm.ExpMat*``); all device work runs in the native library
``lib/libfastctqw_b200.so`` (tcgen05 tensor-core products, HBM-bound norm / LU / matvec
kernels).  There is no CPU fallback.
"""
from . import Ctqw, Operator, State, fastexpm, graphs  # noqa: F401
from ._native import Engine, device_ok  # noqa: F401

__version__ = "0.1.0"
