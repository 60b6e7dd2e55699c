"""ctypes binding of the native library ``libpotts_b200.so`` (include/potts_b200.h).

The library is built in-tree by ``segmentctscans_b200.build``.  Loading fails
loudly when it is missing: there is no CPU fallback for the solver.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

from .build import LIB_PATH

POTTS_OK, POTTS_EINVAL, POTTS_ENOMEM, POTTS_ECUDA, POTTS_ETIMEOUT, POTTS_ENODEV = range(6)
VARIANT_FUSED, VARIANT_PLAIN = 0, 1
STORE_F32, STORE_BF16, STORE_F16, STORE_F64 = 0, 1, 2, 3
STORAGE = {"f32": STORE_F32, "bf16": STORE_BF16, "f16": STORE_F16, "f64": STORE_F64}
ARITH_EXACT, ARITH_FAST = 0, 1
ARITH = {"exact": ARITH_EXACT, "fast": ARITH_FAST}
MAX_PHASES = 6


class PottsMapping(ctypes.Structure):
    _fields_ = [
        ("n_images", ctypes.c_uint32), ("rows", ctypes.c_uint32), ("cols", ctypes.c_uint32),
        ("nstride", ctypes.c_uint32), ("col_begin", ctypes.c_uint32), ("col_end", ctypes.c_uint32),
        ("start_row", ctypes.POINTER(ctypes.c_uint32)), ("base", ctypes.POINTER(ctypes.c_uint32)),
    ]


class PottsOptions(ctypes.Structure):
    _fields_ = [
        ("variant", ctypes.c_int), ("storage", ctypes.c_int), ("gap_every", ctypes.c_int),
        ("slab_w", ctypes.c_int), ("track_dq", ctypes.c_int), ("sync_monitor", ctypes.c_int),
        ("tile_rows", ctypes.c_int), ("tile_slices", ctypes.c_int), ("segment_cols", ctypes.c_int),
        ("tile_vpt", ctypes.c_int), ("prefetch", ctypes.c_int), ("autotune", ctypes.c_int),
        ("arith", ctypes.c_int), ("stall_plane", ctypes.c_int), ("persistent", ctypes.c_int),
    ]


class PottsStats(ctypes.Structure):
    _fields_ = [
        ("n_slabs", ctypes.c_int), ("slab_w", ctypes.c_int), ("iters", ctypes.c_int),
        ("dq_last", ctypes.c_float), ("solve_ms", ctypes.c_double), ("loop_ms", ctypes.c_double),
        ("loop_launches", ctypes.c_int), ("total_launches", ctypes.c_int), ("state_bytes", ctypes.c_uint64),
        ("dq_trace", ctypes.POINTER(ctypes.c_float)), ("energy_trace", ctypes.POINTER(ctypes.c_double)),
        ("loop_iters", ctypes.c_int),
    ]


class PottsBatchVolume(ctypes.Structure):
    _fields_ = [
        ("map", PottsMapping), ("d_u", ctypes.c_void_p), ("ci", ctypes.POINTER(ctypes.c_float)),
        ("lambda_", ctypes.c_float), ("d_res", ctypes.c_void_p), ("d_labels", ctypes.c_void_p),
        ("d_V", ctypes.c_void_p),
    ]


class PottsBatchInfo(ctypes.Structure):
    _fields_ = [
        ("n_volumes", ctypes.c_int), ("n_work", ctypes.c_int), ("tile_rows", ctypes.c_int),
        ("tile_slices", ctypes.c_int), ("tile_vpt", ctypes.c_int), ("segment_cols", ctypes.c_int),
        ("voxels", ctypes.c_uint64), ("state_bytes", ctypes.c_uint64), ("graph_launches", ctypes.c_int),
        ("autotune_ms", ctypes.c_double), ("persistent", ctypes.c_int),
    ]


class PottsArchiveInfo(ctypes.Structure):
    _fields_ = [
        ("n_images", ctypes.c_uint32), ("rows", ctypes.c_uint32), ("cols", ctypes.c_uint32),
        ("nstride", ctypes.c_uint32), ("col_begin", ctypes.c_uint32), ("col_end", ctypes.c_uint32),
        ("span", ctypes.c_uint64), ("lo", ctypes.c_float), ("hi", ctypes.c_float),
        ("header_bits", ctypes.c_uint64), ("voxels", ctypes.c_uint64), ("total_bytes", ctypes.c_uint64),
    ]


class PottsIoStats(ctypes.Structure):
    _fields_ = [("kernel_ms", ctypes.c_double), ("launches", ctypes.c_int)]


ELEM_F32, ELEM_U16 = 0, 1
ELEMENTS = {"f32": ELEM_F32, "u16": ELEM_U16}

_P = ctypes.c_void_p
_I = ctypes.c_int
_F = ctypes.c_float
_U32 = ctypes.c_uint32
_U64 = ctypes.c_uint64
_FP = ctypes.POINTER(ctypes.c_float)
_MP = ctypes.POINTER(PottsMapping)
_OP = ctypes.POINTER(PottsOptions)
_SP = ctypes.POINTER(PottsStats)

# name -> (restype, argtypes); every entry point declared in include/potts_b200.h
SIGNATURES = {
    "potts_default_options": (None, [_OP]),
    "potts_status_string": (ctypes.c_char_p, [_I]),
    "potts_last_error": (ctypes.c_char_p, []),
    "potts_context_create": (_I, [_I, ctypes.POINTER(_P)]),
    "potts_context_create_on_stream": (_I, [_I, _P, ctypes.POINTER(_P)]),
    "potts_context_destroy": (None, [_P]),
    "potts_context_synchronize": (_I, [_P]),
    "potts_context_launches": (ctypes.c_longlong, [_P]),
    "potts_device_memory": (_I, [_P, ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t)]),
    "potts_field_create": (_I, [_P, _MP, ctypes.POINTER(_P)]),
    "potts_field_upload": (_I, [_P, _MP, _FP, ctypes.POINTER(_P)]),
    "potts_field_download": (_I, [_P, _P, _FP, _U64]),
    "potts_field_data": (_P, [_P]),
    "potts_field_span": (_U64, [_P]),
    "potts_field_destroy": (None, [_P]),
    "potts_min_partition": (_I, [_P, _P, _MP, _I, _FP, _F, _F, _F, _I, _OP, ctypes.POINTER(_P), _SP]),
    "potts_solve_device": (_I, [_P, _MP, _P, _I, _FP, _F, _F, _F, _I, _OP, _P, _P, _P, _P, _SP]),
    "potts_solve_device_f64": (_I, [_P, _MP, _P, _I, _FP, _F, _F, _F, _I, _OP, _P, _P, _P, _P, _SP]),
    "potts_solve_host": (_I, [_P, _MP, _P, _I, _FP, _F, _F, _F, _I, _OP, _P, _P, _SP]),
    "potts_cylinder_mapping": (_U64, [_U32, _U32, ctypes.c_double, ctypes.c_double, ctypes.c_double, _U32,
                                      ctypes.POINTER(_U32), ctypes.POINTER(_U32), ctypes.POINTER(_U32),
                                      ctypes.POINTER(_U32)]),
    "potts_get_stride": (_U32, [_U32]),
    "potts_energies_static": (_I, [_MP, _P, _I, _FP, _F, _P, _P, _P, ctypes.POINTER(ctypes.c_double)]),
    "potts_batch_create": (_I, [_P, _I, ctypes.POINTER(PottsBatchVolume), _I, _F, _F, _I, _OP, ctypes.POINTER(_P)]),
    "potts_batch_run": (_I, [_P, _SP]),
    "potts_batch_get_info": (_I, [_P, ctypes.POINTER(PottsBatchInfo)]),
    "potts_batch_read_dq": (_I, [_P, _FP]),
    "potts_batch_destroy": (None, [_P]),
    "potts_forward_ckpt": (_I, [_P, _MP, _P, _P, _I, _FP, _F, _F, _F, _I, _I, _F, _P,
                                ctypes.POINTER(ctypes.c_double), ctypes.POINTER(_P)]),
    "potts_backward": (_I, [_P, _P, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
    "potts_tape_destroy": (None, [_P]),
    "potts_shard_partition": (_I, [_MP, _I, ctypes.POINTER(_U32)]),
    "potts_shard_bounds": (_I, [_MP, ctypes.POINTER(_U32), _I, _I, ctypes.POINTER(_U32), ctypes.POINTER(_U64)]),
    "potts_shard_create": (_I, [_P, _MP, ctypes.POINTER(_U32), _I, _I, _P, _I, _FP, _F, _F, _F, _OP,
                                ctypes.POINTER(_P)]),
    "potts_shard_link": (_I, [_P, _P]),
    "potts_nccl_unique_id": (_I, [_P]),
    "potts_nccl_comm_create": (_I, [_P, _I, _I, _I, ctypes.POINTER(_P)]),
    "potts_nccl_comm_destroy": (_I, [_P]),
    "potts_shard_set_nccl": (_I, [_P, _P]),
    "potts_shard_solve": (_I, [ctypes.POINTER(_P), _I, _I, ctypes.POINTER(_P), ctypes.POINTER(_P),
                               ctypes.POINTER(_P), _SP]),
    "potts_shard_destroy": (None, [_P]),
    "potts_tv_denoise": (_I, [_P, _MP, _P, _F, _F, _I, _I, _SP]),
    "potts_min_max": (_I, [_P, _MP, _P, _FP, _FP]),
    "potts_min_max_positive": (_I, [_P, _MP, _P, _FP, _FP]),
    "potts_grad_magn": (_I, [_P, _MP, _P, _P]),
    "potts_calc_hist": (_I, [_P, _MP, _P, _F, _F, _U32, _F, _U64, _P, _P]),
    "potts_calc_hist_auto": (_I, [_P, _MP, _P, _U32, _F, _U64, _P, _P, _FP, _FP]),
    "potts_uv_hist_stride": (_U32, [_U32]),
    "potts_uv_hist_span": (_U64, [_U32]),
    "potts_uv_hist": (_I, [_P, _MP, _P, _P, _F, _F, _F, _F, _U32, _P]),
    "potts_uv_hist_auto": (_I, [_P, _MP, _P, _P, _U32, _P, _FP]),
    "potts_archive_read_header": (_I, [_P, _U64, _I, ctypes.POINTER(PottsArchiveInfo), _P, _P]),
    "potts_archive_size": (_I, [_MP, _I, ctypes.POINTER(_U64), ctypes.POINTER(_U64)]),
    "potts_archive_load": (_I, [_P, _P, _U64, _I, _P, _U64, ctypes.POINTER(PottsArchiveInfo),
                                ctypes.POINTER(PottsIoStats)]),
    "potts_archive_save": (_I, [_P, _MP, _I, _P, _F, _F, _P, _U64, ctypes.POINTER(_U64),
                                ctypes.POINTER(PottsIoStats)]),
    "potts_convert_to_fp": (_I, [_P, _MP, _I, _P, _F, _F, _P]),
    "potts_find_intensity_range": (_I, [_P, _MP, _P, ctypes.c_double, ctypes.POINTER(ctypes.c_uint16),
                                        ctypes.POINTER(ctypes.c_uint16), _P]),
    "potts_raw_labels_dims": (_I, [_MP, ctypes.POINTER(_U32), ctypes.POINTER(_U32), ctypes.POINTER(_U32),
                                   ctypes.POINTER(_U32)]),
    "potts_raw_labels": (_I, [_P, _MP, _P, _P]),
    "potts_vtk_labels": (_I, [_P, _MP, _P, _P, _U64, ctypes.POINTER(_U64), ctypes.POINTER(PottsIoStats)]),
    "potts_png_slice": (_I, [_P, _MP, _P, _U32, _P, _U64, ctypes.POINTER(_U64)]),
}
STATIC_MAX_COLS = 16384

_lib = None


class PottsError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{message} (status {status})")
        self.status = status


def lib_path() -> Path:
    return LIB_PATH


def host_lib() -> ctypes.CDLL:
    """Load the library (no CUDA call is made by loading it)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(
                f"native library {LIB_PATH} is missing; build it with `python -m segmentctscans_b200.build`")
        lib = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def check(status: int) -> None:
    if status != POTTS_OK:
        lib = host_lib()
        msg = lib.potts_last_error().decode(errors="replace")
        raise PottsError(status, f"{lib.potts_status_string(status).decode()}: {msg}")


def default_options(**kw) -> PottsOptions:
    o = PottsOptions()
    host_lib().potts_default_options(ctypes.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise TypeError(f"unknown option {k}")
        if k == "storage" and isinstance(v, str):
            if v not in STORAGE:
                raise ValueError(f"unknown storage {v!r}; one of {sorted(STORAGE)}")
            v = STORAGE[v]
        if k == "arith" and isinstance(v, str):
            if v not in ARITH:
                raise ValueError(f"unknown arith {v!r}; one of {sorted(ARITH)}")
            v = ARITH[v]
        setattr(o, k, int(v))
    return o
