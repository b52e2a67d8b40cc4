"""mpmsnow_b200 — the implicit MPM snow time step of davidsminor/mpmsnow, rebuilt for NVIDIA B200 (sm_100a).

The product is ``libmpmsnow_b200.so`` (CUDA kernels + the C-ABI of ``include/mpm_gpu.h``); ``mpmsnow_b200.sim``
mirrors the reference's ``MpmSim`` classes over that C-ABI.
"""
from .capi import MpmError  # noqa: F401

__all__ = ["MpmError"]
