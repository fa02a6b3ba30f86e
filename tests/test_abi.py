"""The C-ABI library loads and exports every function include/*.h declares.
CPU only: no compute call is made."""

import ctypes
import os
import re
import subprocess

from conftest import ROOT

HEADER_DIR = os.path.join(ROOT, "include")


def declared_c_functions():
    names = set()
    for fname in os.listdir(HEADER_DIR):
        if not fname.endswith(".h"):
            continue
        text = open(os.path.join(HEADER_DIR, fname)).read()
        names.update(re.findall(r"^SF_API[^;(]*?\b(sf_\w+)\s*\(", text, flags=re.M))
    return names


def test_library_loads_and_exports_every_declared_symbol():
    from dials_metal_spotfinder_b200 import _lib
    declared = declared_c_functions()
    assert declared, "no declarations found"
    for name in declared:
        assert hasattr(_lib.lib, name), f"{name} is declared but not exported"


def test_binding_table_matches_header():
    from dials_metal_spotfinder_b200 import _lib
    assert set(_lib.SIGNATURES) == declared_c_functions()


def test_only_the_c_abi_is_exported():
    from dials_metal_spotfinder_b200 import _lib
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    assert exported, "nothing exported"
    stray = {s for s in exported if not s.startswith("sf_")}
    assert not stray, f"unexpected exports: {sorted(stray)[:10]}"


def test_record_layouts_match_the_reference():
    from dials_metal_spotfinder_b200 import PIXEL, SIGNAL_PIXEL, SPOT
    assert SIGNAL_PIXEL.itemsize == 16
    assert PIXEL.itemsize == 12
    assert SPOT.itemsize == 104
    assert SPOT.fields["first"][1] == 96


def test_no_device_means_a_loud_failure_not_a_fallback():
    import dials_metal_spotfinder_b200 as sf
    if sf.available():
        return
    import numpy as np
    import pytest
    with pytest.raises(sf.DeviceError):
        sf.find(np.zeros((8, 8), np.uint16))
