"""ctypes bindings for the checkers. TEST INFRASTRUCTURE ONLY.

Two libraries, both built by oracle/Makefile:

* ``_build/liboracle.so`` -- the plain-C restatement (sf_oracle.c) of the
  reference's threshold (src/dext.cc:9-225) and grouping
  (src/dials_spots.cc:36-360). Always present once built.
* ``_ref/libref.so`` -- the reference's own dext.cc / dials_spots.cc /
  refl.cc compiled from its sources, plus ``_ref/libref_gpu.so``, its CUDA
  backend. Present where the reference tree was available at build time.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module. The product (dials_metal_spotfinder_b200) never does.
"""

from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libref.so")
REF_GPU_SO = os.path.join(HERE, "_ref", "libref_gpu.so")

# src/signal_pixel.hh:20-26
SIGNAL_PIXEL = np.dtype(
    [("index", "<u4"), ("value", "<u4"), ("background", "<f4"),
     ("population", "<u2"), ("reserved", "<u2")]
)
# src/dials_spots.hh:50-54
PIXEL = np.dtype([("frame", "<i4"), ("index", "<u4"), ("value", "<u4")])
# src/dials_spots.hh:57-79, with the 4 bytes of padding before `first`.
SPOT = np.dtype(
    {
        "names": ["bbox", "position", "variance", "intensity",
                  "intensity_variance", "n_signal", "first"],
        "formats": [("<i4", 6), ("<f8", 3), ("<f8", 3), "<f8", "<f8", "<u4", "<u8"],
        "offsets": [0, 24, 48, 72, 80, 88, 96],
        "itemsize": 104,
    }
)
COUNT_NAMES = ("signal_pixels", "groups", "too_small", "too_large", "separated",
               "accepted")

_P = ctypes.c_void_p
_S = ctypes.c_size_t


def _load(path):
    if not os.path.exists(path):
        return None
    return ctypes.CDLL(path)


def _bind_dext(lib, prefix):
    for t in ("u16", "u32"):
        fn = getattr(lib, f"{prefix}_dext_{t}")
        fn.argtypes = [_P, _S, _S, _P, _S, ctypes.POINTER(_S)]
        fn.restype = ctypes.c_int


_oracle = None
_ref = None
_ref_gpu = None


def oracle_lib():
    global _oracle
    if _oracle is None:
        lib = _load(ORACLE_SO)
        if lib is None:
            raise RuntimeError(f"{ORACLE_SO} is not built; run `make -C oracle oracle`")
        _bind_dext(lib, "sfo")
        lib.sfo_lab_new.argtypes = [_S, _S, _S, _S, ctypes.c_double, ctypes.c_int]
        lib.sfo_lab_new.restype = _P
        lib.sfo_lab_free.argtypes = [_P]
        lib.sfo_lab_add.argtypes = [_P, ctypes.c_int64, _P, _S]
        lib.sfo_lab_add.restype = ctypes.c_int
        lib.sfo_lab_finish.argtypes = [_P]
        lib.sfo_lab_error.argtypes = [_P]
        lib.sfo_lab_error.restype = ctypes.c_char_p
        for name in ("nspots", "npixels", "live"):
            fn = getattr(lib, f"sfo_lab_{name}")
            fn.argtypes = [_P]
            fn.restype = _S
        lib.sfo_lab_spots.argtypes = [_P]
        lib.sfo_lab_spots.restype = _P
        lib.sfo_lab_pixels.argtypes = [_P]
        lib.sfo_lab_pixels.restype = _P
        lib.sfo_lab_counts.argtypes = [_P, _P]
        lib.sfo_spot_size.restype = _S
        assert lib.sfo_spot_size() == SPOT.itemsize
        _oracle = lib
    return _oracle


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref_lib():
    global _ref
    if _ref is None:
        lib = _load(REF_SO)
        if lib is None:
            raise RuntimeError(f"{REF_SO} is not built (needs the reference tree)")
        _bind_dext(lib, "ref")
        lib.ref_last_error.restype = ctypes.c_char_p
        lib.ref_make_frame.argtypes = [_S, _S, ctypes.c_uint64, ctypes.c_double,
                                       ctypes.c_int, _P]
        lib.ref_labeller_new.argtypes = [_S, _S, _S, _S, ctypes.c_double, ctypes.c_int]
        lib.ref_labeller_new.restype = _P
        lib.ref_labeller_free.argtypes = [_P]
        lib.ref_labeller_add.argtypes = [_P, ctypes.c_int64, _P, _S]
        lib.ref_labeller_finish.argtypes = [_P]
        for name in ("nspots", "npixels", "live"):
            fn = getattr(lib, f"ref_labeller_{name}")
            fn.argtypes = [_P]
            fn.restype = _S
        lib.ref_labeller_spots.argtypes = [_P, _P, _S]
        lib.ref_labeller_pixels.argtypes = [_P, _P, _S]
        lib.ref_labeller_counts.argtypes = [_P, _P]
        lib.ref_spot_size.restype = _S
        lib.ref_refl_write.argtypes = [ctypes.c_char_p, _P, _S, ctypes.c_char_p, ctypes.c_int,
                                       ctypes.c_int]
        assert lib.ref_spot_size() == SPOT.itemsize
        _ref = lib
    return _ref


def ref_gpu_lib():
    global _ref_gpu
    if _ref_gpu is None:
        lib = _load(REF_GPU_SO)
        if lib is None:
            raise RuntimeError(f"{REF_GPU_SO} is not built (needs the reference tree)")
        lib.refgpu_find_u16.argtypes = [_P, _S, _S, _P, _S, ctypes.POINTER(_S)]
        lib.refgpu_find_u16.restype = ctypes.c_int
        lib.refgpu_last_error.restype = ctypes.c_char_p
        lib.refgpu_host_alloc.argtypes = [_S]
        lib.refgpu_host_alloc.restype = _P
        lib.refgpu_host_free.argtypes = [_P]
        _ref_gpu = lib
    return _ref_gpu


def _run_dext(fn, image: np.ndarray, capacity: int | None = None):
    image = np.ascontiguousarray(image)
    h, w = image.shape
    if capacity is None:
        capacity = h * w
    out = np.zeros(max(capacity, 1), dtype=SIGNAL_PIXEL)
    found = _S(0)
    status = fn(image.ctypes.data, h, w, out.ctypes.data, capacity, ctypes.byref(found))
    if status != 0:
        return status, out[:0], found.value
    return 0, out[: found.value].copy(), found.value


def dext(image: np.ndarray, capacity: int | None = None, use_ref: bool = False):
    """Threshold one frame. Returns (status, signal pixels, count)."""
    lib = ref_lib() if use_ref else oracle_lib()
    prefix = "ref" if use_ref else "sfo"
    kind = {np.dtype(np.uint16): "u16", np.dtype(np.uint32): "u32"}[image.dtype]
    return _run_dext(getattr(lib, f"{prefix}_dext_{kind}"), image, capacity)


def make_frame(height: int, width: int, seed: int, background: float,
               with_mask: bool) -> np.ndarray:
    """The reference's own device-test frame (tests/synthetic_frame.hh:93-157)."""
    out = np.zeros((height, width), dtype=np.uint16)
    ref_lib().ref_make_frame(height, width, seed, background, int(with_mask),
                             out.ctypes.data)
    return out


@dataclass
class Grouped:
    spots: np.ndarray
    pixels: np.ndarray
    counts: dict
    live: int


class Labeller:
    """The oracle's (or the reference's) grouping, mirroring
    dials_spots::Labeller (src/dials_spots.hh:108-126)."""

    def __init__(self, height, width, min_spot_size=3, max_spot_size=1000,
                 max_separation=2.0, two_d=False, use_ref=False):
        self.use_ref = use_ref
        self.lib = ref_lib() if use_ref else oracle_lib()
        new = self.lib.ref_labeller_new if use_ref else self.lib.sfo_lab_new
        self.handle = new(height, width, min_spot_size, max_spot_size,
                          max_separation, int(two_d))
        if not self.handle:
            raise RuntimeError("invalid labeller options")
        self.width = width

    def __del__(self):
        if getattr(self, "handle", None):
            (self.lib.ref_labeller_free if self.use_ref else self.lib.sfo_lab_free)(self.handle)
            self.handle = None

    def add(self, frame: int, signal: np.ndarray) -> None:
        signal = np.ascontiguousarray(signal, dtype=SIGNAL_PIXEL)
        if self.use_ref:
            status = self.lib.ref_labeller_add(self.handle, frame, signal.ctypes.data, len(signal))
            if status != 0:
                raise RuntimeError(self.lib.ref_last_error().decode())
        else:
            status = self.lib.sfo_lab_add(self.handle, frame, signal.ctypes.data, len(signal))
            if status != 0:
                raise RuntimeError(self.lib.sfo_lab_error(self.handle).decode())

    def finish(self) -> None:
        (self.lib.ref_labeller_finish if self.use_ref else self.lib.sfo_lab_finish)(self.handle)

    def result(self) -> Grouped:
        lib = self.lib
        if self.use_ref:
            ns = lib.ref_labeller_nspots(self.handle)
            npx = lib.ref_labeller_npixels(self.handle)
            spots = np.zeros(ns, dtype=SPOT)
            pixels = np.zeros(npx, dtype=PIXEL)
            if ns:
                lib.ref_labeller_spots(self.handle, spots.ctypes.data, ns)
            if npx:
                lib.ref_labeller_pixels(self.handle, pixels.ctypes.data, npx)
            counts = np.zeros(6, dtype=np.uint64)
            lib.ref_labeller_counts(self.handle, counts.ctypes.data)
            live = lib.ref_labeller_live(self.handle)
        else:
            ns = lib.sfo_lab_nspots(self.handle)
            npx = lib.sfo_lab_npixels(self.handle)
            spots = np.zeros(ns, dtype=SPOT)
            pixels = np.zeros(npx, dtype=PIXEL)
            if ns:
                ctypes.memmove(spots.ctypes.data, lib.sfo_lab_spots(self.handle), ns * SPOT.itemsize)
            if npx:
                ctypes.memmove(pixels.ctypes.data, lib.sfo_lab_pixels(self.handle), npx * PIXEL.itemsize)
            counts = np.zeros(6, dtype=np.uint64)
            lib.sfo_lab_counts(self.handle, counts.ctypes.data)
            live = lib.sfo_lab_live(self.handle)
        return Grouped(spots, pixels, dict(zip(COUNT_NAMES, (int(c) for c in counts))), int(live))

    def write_refl(self, path: str, identifier: str = "", shoeboxes: bool = True,
                   experiment_id: int = 0) -> None:
        if not self.use_ref:
            raise RuntimeError("only the reference labeller writes .refl files")
        status = self.lib.ref_refl_write(path.encode(), self.handle, self.width,
                                         identifier.encode(), int(shoeboxes), experiment_id)
        if status != 0:
            raise RuntimeError(self.lib.ref_last_error().decode())


def group(frames_signal, height, width, frame_numbers=None, use_ref=False, **options) -> Grouped:
    """Run a whole series of signal lists through a labeller and finish."""
    lab = Labeller(height, width, use_ref=use_ref, **options)
    numbers = range(len(frames_signal)) if frame_numbers is None else frame_numbers
    for z, signal in zip(numbers, frames_signal):
        lab.add(int(z), signal)
    lab.finish()
    return lab.result()
