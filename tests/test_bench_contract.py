"""bench.py's own arm on the CPU, with the engine and the device calls
replaced by fakes: the JSON line it prints carries every key of the
benchmark contract, with values of the right kinds. Nothing here is a
measurement; the numbers come from the fakes."""

import contextlib
import io
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


class FakeHostBuffer:
    def __init__(self, shape, dtype):
        self.array = np.zeros(shape, dtype)

    def close(self):
        self.array = None


def fake_engine(sf):
    class FakeEngine:
        def __init__(self, shapes, dtype, slots=2, **kw):
            self.shapes = shapes
            self.accepted = 0

        def enable_grouping(self, **kw):
            pass

        def info(self):
            return {"seg_rows": 0, "slots": 2}

        def tuning(self):
            return {"frames_per_launch": len(self.shapes), "warps_per_block": 4,
                    "seg_rows": 100, "from_cache": False}

        def upload(self, slot, frame, image):
            assert image.shape == self.shapes[frame]

        def upload_chunks(self, slot, chunks, frames=None, algorithm="bslz4"):
            assert len(chunks) == len(self.shapes)

        def upload_chunk(self, slot, frame, chunk, algorithm="bslz4"):
            assert 0 <= frame < len(self.shapes)

        def synchronize(self):
            pass

        def run(self, slot):
            self.accepted += 1000

        def group_counts(self):
            return {"accepted": self.accepted, "groups": 1}, 0

        def record(self, i):
            pass

        def elapsed_ms(self, a, b):
            return 8.0

        def profile(self, on):
            pass

        def stage_totals(self):
            return {"threshold_ms": 2.0, "place_ms": 0.2, "group_ms": 4.0, "runs": 2}

        def counts(self, slot):
            return np.full(len(self.shapes), 1000, np.uint32)

        def use_graph(self, on):
            pass

        def close(self):
            pass

        def _records(self, n, dtype, out):
            if out is None:
                return np.zeros(n, dtype)
            out[:n] = np.zeros(n, dtype)
            return out[:n]

        def spots(self, series=0, out=None):
            return self._records(7, sf.SPOT, out)

        def pixels(self, series=0, out=None):
            return self._records(40, sf.PIXEL, out)

    return FakeEngine


def test_bench_line_has_the_contract_keys(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    import dials_metal_spotfinder_b200 as sf
    import dials_metal_spotfinder_b200.engine as engine
    from dials_metal_spotfinder_b200 import _lib

    for var in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(var, raising=False)
    monkeypatch.setattr(engine, "Engine", fake_engine(sf))
    monkeypatch.setattr(sf, "HostBuffer", FakeHostBuffer)
    monkeypatch.setattr(sf, "find", lambda image, out=None: np.zeros(0, sf.SIGNAL_PIXEL))
    monkeypatch.setattr(_lib, "raise_for", lambda status, what: None)
    monkeypatch.setattr(bench, "reference_gpu_form", lambda frame: {"unavailable": "fake"})
    monkeypatch.setattr(bench, "parity_check", lambda pool, F: {"status": "fake"})
    monkeypatch.setattr(bench, "make_pool",
                        lambda n: [np.zeros(bench.SHAPE, np.uint16) for _ in range(n)])
    monkeypatch.setattr(sys, "argv", ["bench.py", "--steps", "2", "--warmup", "3", "--no-cpu",
                                      "--serve-seconds", "0", "--no-4m", "--e2e-steps", "2",
                                      "--pool", "2", "--no-tune", "--no-u32", "--no-stills"])
    out = io.StringIO()
    with contextlib.redirect_stdout(out):
        bench.main()
    lines = [ln for ln in out.getvalue().splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
                "roofline", "clocks", "gpu_launches", "e2e", "cpu_baseline", "parity"):
        assert key in d, key
    assert d["n_gpus"] == 1 and d["steps"] == 2 and d["warmup"] == 3
    assert d["higher_is_better"] is True and d["scaling"] == "weak"
    assert "workload" in d["config"]
    assert d["value"] > 0 and d["ms_per_step"] > 0
    r = d["roofline"]
    for key in ("bound", "achieved", "peak", "unit", "frac", "traffic"):
        assert key in r, key
    assert r["bound"] == "hbm" and r["unit"] == "GB/s"
    assert abs(r["frac"] - r["achieved"] / r["peak"]) < 1e-12
    e = d["e2e"]
    for key in ("value", "unit", "h2d_bytes_per_step", "d2h_bytes_per_step"):
        assert key in e, key
    assert e["h2d_bytes_per_step"] == bench.DEFAULT_FRAMES * bench.SHAPE[0] * bench.SHAPE[1] * 2
    assert e["d2h_bytes_per_step"] == 7 * sf.SPOT.itemsize + 40 * sf.PIXEL.itemsize
    assert d["gpu_launches"] > 0 and d["gpu_launches"] % d["steps"] == 0
    assert d["gpixels_per_s"] > 0 and d["pipeline_bytes"]["per_frame"] > 0
    c = d["e2e_chunks"]
    assert c["value"] > 0 and 0 < c["h2d_bytes_per_step"] < e["h2d_bytes_per_step"]
