"""B200 (sm_100a) multiphase Potts segmentation solver for cylindrical micro-CT cores.

A from-scratch GPU implementation of the Chambolle–Cremers–Pock primal-dual
Potts iteration of slavaandrejev/segmentctscans
(potts-model/potts-min-partition.{h,cpp}) behind a C ABI
(include/potts_b200.h, ``libpotts_b200.so``), with a host API mirroring the
reference's ``make_context / upload / potts_min_partition / download``.
"""
from .layout import CylinderMapping, get_stride, prev_stride  # noqa: F401
from .potts import (  # noqa: F401
    CudaContext,
    DeviceField,
    PottsError,
    PottsResult,
    SolveStats,
    device_memory,
    download,
    make_context,
    potts_min_partition,
    reference_tau,
    solve,
    solve_device,
    solve_host,
    upload,
)

__all__ = [
    "CylinderMapping", "get_stride", "prev_stride", "CudaContext", "DeviceField", "PottsError", "PottsResult",
    "SolveStats", "device_memory", "download", "make_context", "potts_min_partition", "reference_tau", "solve",
    "solve_device", "solve_host", "upload",
]
