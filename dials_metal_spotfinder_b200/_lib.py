"""Loads libspotfinder_b200.so and declares its C ABI (include/spotfinder_b200.h).

The library is built in-tree by ``make -C dials_metal_spotfinder_b200/csrc``
(``__graft_entry__.build()`` runs it). There is no fallback: if the library is
missing this module raises ImportError, and every device entry point raises
DeviceError when no CUDA device is present.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libspotfinder_b200.so")
HEADER_PATH = os.path.join(os.path.dirname(HERE), "include", "spotfinder_b200.h")

# include/spotfinder_b200.h: sf_signal_pixel, sf_pixel, sf_spot, sf_counts.
SIGNAL_PIXEL = np.dtype(
    [("index", "<u4"), ("value", "<u4"), ("background", "<f4"),
     ("population", "<u2"), ("reserved", "<u2")]
)
PIXEL = np.dtype([("frame", "<i4"), ("index", "<u4"), ("value", "<u4")])
SPOT = np.dtype(
    {
        "names": ["bbox", "position", "variance", "intensity",
                  "intensity_variance", "n_signal", "first"],
        "formats": [("<i4", 6), ("<f8", 3), ("<f8", 3), "<f8", "<f8", "<u4", "<u8"],
        "offsets": [0, 24, 48, 72, 80, 88, 96],
        "itemsize": 104,
    }
)
COUNT_NAMES = ("signal_pixels", "groups", "too_small", "too_large", "separated", "accepted")


class BadArgument(ValueError):
    """Status -1: the reference's 'bad argument' return."""


class Overflow(RuntimeError):
    """Status -2: more signal pixels than the list holds."""


class DeviceError(RuntimeError):
    """Status -3: a CUDA or runtime failure."""


class Refused(RuntimeError):
    """Status -4: a labelling input refused (order, range)."""


class GroupOptions(ctypes.Structure):
    _fields_ = [("min_spot_size", ctypes.c_uint64), ("max_spot_size", ctypes.c_uint64),
                ("max_separation", ctypes.c_double), ("two_d", ctypes.c_int32),
                ("reserved", ctypes.c_int32)]


_P = ctypes.c_void_p
_S = ctypes.c_size_t
_I = ctypes.c_int

# name -> (restype, argtypes). Every function the header declares appears
# here; tests/test_abi.py checks the two lists agree and that each symbol is
# exported.
SIGNATURES = {
    "sf_backend": (ctypes.c_char_p, []),
    "sf_available": (_I, []),
    "sf_memory_free": (_S, []),
    "sf_host_alloc": (_P, [_S]),
    "sf_host_free": (None, [_P]),
    "sf_last_error": (ctypes.c_char_p, []),
    "sf_set_device": (_I, [_I]),
    "sf_find_u16": (_I, [_P, _S, _S, _P, _S, ctypes.POINTER(_S)]),
    "sf_find_u32": (_I, [_P, _S, _S, _P, _S, ctypes.POINTER(_S)]),
    "sf_find_u16_noalloc": (_I, [_P, _S, _S, _P, _S, ctypes.POINTER(_S), _P]),
    "sf_profile_stages": (None, [_I]),
    "sf_profile_stages_enabled": (_I, []),
    "sf_last_stage_times": (None, [_P]),
    "sf_labeller_create": (_I, [_S, _S, _P, ctypes.POINTER(_P)]),
    "sf_labeller_destroy": (None, [_P]),
    "sf_labeller_add": (_I, [_P, ctypes.c_int64, _P, _S]),
    "sf_labeller_finish": (_I, [_P]),
    "sf_labeller_counts": (_I, [_P, _P]),
    "sf_labeller_nspots": (_S, [_P]),
    "sf_labeller_npixels": (_S, [_P]),
    "sf_labeller_live": (_S, [_P]),
    "sf_labeller_spots": (_I, [_P, _P, _S]),
    "sf_labeller_pixels": (_I, [_P, _P, _S]),
    "sf_refl_write": (_I, [ctypes.c_char_p, _P, _S, _P, _S, _S, _P]),
    "sf_chunk_bound": (_S, [_S, _S, _I]),
    "sf_chunk_encode": (_I, [_I, _P, _S, _S, _I, _P, _S, ctypes.POINTER(_S)]),
    "sf_chunk_decode": (_I, [_I, _P, _S, _S, _S, _I, _P]),
    "sf_chunk_decode_device": (_I, [_I, _P, _S, _S, _S, _I, _P, _S]),
    "sf_server_create": (_I, [_P, ctypes.POINTER(_P)]),
    "sf_server_destroy": (None, [_P]),
    "sf_server_open": (_I, [_P, _S, _S, _I, _P, ctypes.c_int64, ctypes.POINTER(_I)]),
    "sf_server_set_pixel_mask": (_I, [_P, _I, _P]),
    "sf_server_submit": (_I, [_P, _I, _P, _S, _I, ctypes.c_int64]),
    "sf_server_close": (_I, [_P, _I]),
    "sf_server_stats": (_I, [_P, _I, _P, _P]),
    "sf_server_spots": (_I, [_P, _I, _P, _S, ctypes.POINTER(_S)]),
    "sf_server_pixels": (_I, [_P, _I, _P, _S, ctypes.POINTER(_S)]),
    "sf_server_take": (_I, [_P, _I, _P, _S, ctypes.POINTER(_S), _P, _S, ctypes.POINTER(_S)]),
    "sf_server_signal_counts": (_I, [_P, _I, _P, _S, ctypes.POINTER(_S)]),
    "sf_server_latencies": (_I, [_P, _I, _I, _P, _S, ctypes.POINTER(_S)]),
    "sf_engine_create": (_I, [_I, _I, _P, _P, _P, ctypes.POINTER(_P)]),
    "sf_engine_destroy": (None, [_P]),
    "sf_engine_info": (_I, [_P, _P]),
    "sf_engine_upload": (_I, [_P, _I, _I, _P]),
    "sf_engine_upload_device": (_I, [_P, _I, _I, _P, _S]),
    "sf_engine_upload_chunk": (_I, [_P, _I, _I, _P, _S, _I]),
    "sf_engine_upload_chunks": (_I, [_P, _I, _S, _P, _P, _P, _I]),
    "sf_engine_set_pixel_mask": (_I, [_P, _I, _P]),
    "sf_engine_run": (_I, [_P, _I]),
    "sf_engine_use_graph": (_I, [_P, _I]),
    "sf_engine_synchronize": (_I, [_P]),
    "sf_engine_counts": (_I, [_P, _I, _P]),
    "sf_engine_signal": (_I, [_P, _I, _I, _P, _S, ctypes.POINTER(_S)]),
    "sf_engine_signals": (_I, [_P, _I, _P, _S, _P]),
    "sf_engine_record": (_I, [_P, _I]),
    "sf_engine_elapsed": (_I, [_P, _I, _I, ctypes.POINTER(ctypes.c_float)]),
    "sf_engine_profile": (_I, [_P, _I]),
    "sf_engine_stage_totals": (_I, [_P, _P]),
    "sf_engine_enable_grouping": (_I, [_P, _P, ctypes.c_int64, ctypes.c_uint64]),
    "sf_engine_nseries": (_I, [_P]),
    "sf_engine_series_shape": (_I, [_P, _I, ctypes.POINTER(ctypes.c_int32),
                                    ctypes.POINTER(ctypes.c_int32)]),
    "sf_engine_series_counts": (_I, [_P, _I, _P, ctypes.POINTER(ctypes.c_uint64)]),
    "sf_engine_series_spots": (_I, [_P, _I, _P, _S, ctypes.POINTER(_S)]),
    "sf_engine_series_pixels": (_I, [_P, _I, _P, _S, ctypes.POINTER(_S)]),
    "sf_engine_group_counts": (_I, [_P, _P, ctypes.POINTER(ctypes.c_uint64)]),
    "sf_engine_spots": (_I, [_P, _P, _S, ctypes.POINTER(_S)]),
    "sf_engine_pixels": (_I, [_P, _P, _S, ctypes.POINTER(_S)]),
    "sf_engine_finish": (_I, [_P]),
    "sf_tune": (_I, [_I, _I, _I, _P, _I, _P, _P]),
    "sf_engine_tuning": (_I, [_P, _P]),
}


class ReflOptions(ctypes.Structure):
    _fields_ = [("panel", ctypes.c_uint64), ("id", ctypes.c_int32), ("shoeboxes", ctypes.c_int32),
                ("identifier", ctypes.c_char_p)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("hbm_budget", ctypes.c_uint64), ("slots", ctypes.c_int32),
                ("use_graph", ctypes.c_int32)]


class TuneOptions(ctypes.Structure):
    _fields_ = [("min_frames", ctypes.c_int32), ("max_frames", ctypes.c_int32),
                ("steps", ctypes.c_int32), ("grouping", ctypes.c_int32),
                ("use_cache", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("hbm_budget", ctypes.c_uint64), ("cache_path", ctypes.c_char_p)]


class TuneResult(ctypes.Structure):
    _fields_ = [("frames_per_launch", ctypes.c_int32), ("warps_per_block", ctypes.c_int32),
                ("seg_rows", ctypes.c_int32), ("from_cache", ctypes.c_int32),
                ("candidates", ctypes.c_int32), ("blocks_per_sm", ctypes.c_int32),
                ("seg_ratio", ctypes.c_double), ("us_per_frame", ctypes.c_double)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_ if name != "reserved"}


class EngineConfig(ctypes.Structure):
    _fields_ = [("seg_rows", ctypes.c_int32), ("warps_per_block", ctypes.c_int32),
                ("blocks_per_sm", ctypes.c_int32), ("slots", ctypes.c_int32)]


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is not built; run `make -C {os.path.join(HERE, 'csrc')}` "
            "(there is no CPU fallback)"
        )
    lib = ctypes.CDLL(LIB_PATH)
    for name, (restype, argtypes) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = restype
        fn.argtypes = argtypes
    return lib


lib = _load()


def last_error() -> str:
    msg = lib.sf_last_error()
    return msg.decode() if msg else ""


def raise_for(status: int, what: str) -> None:
    if status == 0:
        return
    if status == -1:
        raise BadArgument(f"{what}: bad argument {last_error()}".rstrip())
    if status == -2:
        raise Overflow(f"{what}: more signal pixels than the list holds")
    if status == -4:
        raise Refused(f"{what}: {last_error()}")
    raise DeviceError(f"{what}: {last_error() or f'status {status}'}")


def require_device() -> None:
    if not lib.sf_available():
        raise DeviceError("no CUDA device is available (the B200 path has no CPU fallback)")
