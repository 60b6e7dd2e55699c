"""B200 (sm_100a) multiphase Potts segmentation solver for cylindrical micro-CT cores.

A from-scratch GPU implementation of the Chambolle–Cremers–Pock primal-dual
Potts iteration of slavaandrejev/segmentctscans
(potts-model/potts-min-partition.{h,cpp}) behind a C ABI
(include/potts_b200.h, ``libpotts_b200.so``), with a host API mirroring the
reference's ``make_context / upload / potts_min_partition / download``.

The solver names below are resolved on first use, so that importing a
submodule that needs no GPU code (``layout``, ``phantom``) does not load the
native library.
"""
from __future__ import annotations

import importlib

_FROM_LAYOUT = ("CylinderMapping", "get_stride", "prev_stride")
_FROM_POTTS = ("CudaContext", "DeviceField", "PottsError", "PottsResult", "SolveStats", "device_memory", "download",
               "make_context", "potts_min_partition", "reference_tau", "solve", "solve_device", "solve_host",
               "upload")

__all__ = [*_FROM_LAYOUT, *_FROM_POTTS]


def __getattr__(name: str):
    if name in _FROM_LAYOUT:
        return getattr(importlib.import_module(".layout", __name__), name)
    if name in _FROM_POTTS:
        return getattr(importlib.import_module(".potts", __name__), name)
    raise AttributeError(f"module {__name__!r} has no attribute {name!r}")
