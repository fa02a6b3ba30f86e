#!/usr/bin/env python3
"""Writes the golden fixtures in this directory from the reference's own code.

Needs oracle/_ref/libref.so, which oracle/Makefile compiles from the
reference's src/dext.cc, src/dials_spots.cc and src/refl.cc and its
tests/synthetic_frame.hh (``make -C oracle ref``; only possible where the
reference tree is present). The fixtures are committed so that the tests can
run anywhere without it.

    python tests/golden/make_golden.py

Fixtures:
  threshold_u16.npz  the reference device-test frame set (test_dext_gpu.cc:
                     155-176: exact tile, under one tile, ragged, ragged
                     masked, dark, module, entirely masked), each with the
                     reference dext<uint16_t> output.
  threshold_u32.npz  two 32-bit frames with bright planted spots (sums of
                     squares past 2^32) and both 32-bit sentinels, with the
                     reference dext<uint32_t> output.
  small_series.npz   the 256 x 384 x 12 small configuration (seeded), the
                     reference threshold of every frame, and the reference
                     Labeller's spots, pixels and counts in 3D and in 2D.
  refl_small.refl    the reference refl::write of the 3D small-series spots
                     with shoeboxes, identifier "golden".
  refl_small_2d.refl the same for the 2D grouping, no identifier.
  refl_small_noshoebox.refl  the 3D spots without the shoebox column, id 3.
"""

from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from dials_metal_spotfinder_b200 import synth  # noqa: E402  (numpy only)

# (name, height, width, seed, background, with_mask): test_dext_gpu.cc:155-167
FRAME_SET = [
    ("exact tile", 32, 32, 1, 12.0, False),
    ("under one tile", 19, 27, 2, 8.0, False),
    ("ragged", 200, 301, 3, 15.0, False),
    ("ragged, masked", 200, 301, 4, 15.0, True),
    ("dark", 128, 128, 5, 1.0, False),
    ("module", 512, 1030, 6, 20.0, True),
]


def pack_list(arrays):
    offsets = np.zeros(len(arrays) + 1, np.int64)
    for i, a in enumerate(arrays):
        offsets[i + 1] = offsets[i] + len(a)
    flat = np.concatenate(arrays) if arrays else np.zeros(0)
    return flat, offsets


def threshold_u16():
    frames, names = [], []
    for name, h, w, seed, bg, mask in FRAME_SET:
        frames.append(O.make_frame(h, w, seed, bg, mask))
        names.append(name)
    frames.append(np.full((64, 64), 0xFFFF, np.uint16))
    names.append("entirely masked")
    outs = []
    for img in frames:
        status, sig, _ = O.dext(img, use_ref=True)
        assert status == 0
        outs.append(sig)
    data = {}
    for i, (img, sig) in enumerate(zip(frames, outs)):
        data[f"frame{i}"] = img
        data[f"signal{i}"] = sig.view(np.uint8).reshape(-1, 16) if len(sig) else np.zeros((0, 16), np.uint8)
    data["names"] = np.array(names)
    np.savez_compressed(os.path.join(HERE, "threshold_u16.npz"), **data)
    print("threshold_u16:", [len(s) for s in outs])


def threshold_u32():
    rng = np.random.default_rng(0x32B17)
    frames = []
    for h, w in ((96, 130), (160, 200)):
        img = rng.poisson(4.0, (h, w)).astype(np.uint32)
        for _ in range(6):
            y, x = rng.integers(2, h - 2), rng.integers(2, w - 2)
            peak = int(rng.integers(200000, 2000000))
            img[y - 1:y + 2, x - 1:x + 2] += np.uint32(peak // 4)
            img[y, x] += np.uint32(peak)
        img[0, 0] = 0xFFFFFFFF
        img[h // 2, :] = 0xFFFFFFFE
        img[5, w - 1] = 0xFFFFFFFF
        frames.append(img)
    data = {}
    for i, img in enumerate(frames):
        status, sig, _ = O.dext(img, use_ref=True)
        assert status == 0
        data[f"frame{i}"] = img
        data[f"signal{i}"] = sig.view(np.uint8).reshape(-1, 16)
        print("threshold_u32 frame", i, len(sig))
    np.savez_compressed(os.path.join(HERE, "threshold_u32.npz"), **data)


def small_series():
    series = synth.small()
    stack = series.frames_array(0, series.frames)
    signals = []
    for img in stack:
        status, sig, _ = O.dext(img, use_ref=True)
        assert status == 0
        signals.append(sig)
    data = {"frames": stack}
    flat, offsets = pack_list(signals)
    data["signal"] = flat.view(np.uint8).reshape(-1, 16)
    data["signal_offsets"] = offsets
    for mode, two_d in (("3d", False), ("2d", True)):
        lab = O.Labeller(*stack.shape[1:], two_d=two_d, use_ref=True)
        for z, sig in enumerate(signals):
            lab.add(z, sig)
        lab.finish()
        res = lab.result()
        data[f"spots_{mode}"] = res.spots.view(np.uint8).reshape(-1, 104)
        data[f"pixels_{mode}"] = res.pixels.view(np.uint8).reshape(-1, 12)
        data[f"counts_{mode}"] = np.array([res.counts[k] for k in O.COUNT_NAMES], np.uint64)
        print("small_series", mode, len(res.spots), res.counts)
        if mode == "3d":
            lab.write_refl(os.path.join(HERE, "refl_small.refl"), identifier="golden")
    np.savez_compressed(os.path.join(HERE, "small_series.npz"), **data)


def refl_variants():
    """refl::write with the other option branches: 2D spots with an empty
    identifier map, and 3D spots without shoeboxes under experiment id 3."""
    g = np.load(os.path.join(HERE, "small_series.npz"))
    h, w = g["frames"].shape[1:]
    signals = [np.ascontiguousarray(g["signal"][a:b]).view(O.SIGNAL_PIXEL).reshape(-1)
               for a, b in zip(g["signal_offsets"][:-1], g["signal_offsets"][1:])]
    for name, two_d, ident, ident_id, shoeboxes in (
            ("refl_small_2d.refl", True, "", 0, True),
            ("refl_small_noshoebox.refl", False, "golden-3", 3, False)):
        lab = O.Labeller(h, w, two_d=two_d, use_ref=True)
        for z, sig in enumerate(signals):
            lab.add(z, sig)
        lab.finish()
        lab.write_refl(os.path.join(HERE, name), identifier=ident, shoeboxes=shoeboxes,
                       experiment_id=ident_id)
        print(name, len(lab.result().spots))


if __name__ == "__main__":
    if not O.ref_available():
        sys.exit("oracle/_ref/libref.so is missing: run `make -C oracle ref` where the "
                 "reference tree is present")
    if sys.argv[1:] == ["refl"]:
        refl_variants()
        sys.exit(0)
    threshold_u16()
    threshold_u32()
    small_series()
    refl_variants()
