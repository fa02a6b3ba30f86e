"""bench.py runs the serving replay in a process of its own
(`serving_process`): the child's last JSON line becomes the `serving`
entry, marked with where it ran, and a child that fails or prints nothing
gives an `error` entry instead of stopping the bench. The child is faked
here; nothing runs on a device."""

import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    sys.path.insert(0, ROOT)
    import bench
    return bench


class _Done:
    def __init__(self, rc, out, err=""):
        self.returncode, self.stdout, self.stderr = rc, out, err


def test_child_line_becomes_the_entry(monkeypatch):
    bench = _bench()
    seen = {}

    def fake_run(cmd, **kw):
        seen["cmd"] = cmd
        line = json.dumps({"seconds": 60.0, "served": [{"dropped": 0}]})
        return _Done(0, "warming up\n" + line + "\n")

    monkeypatch.setattr(subprocess, "run", fake_run)
    out = bench.serving_process(60.0, 10.0)
    assert out["seconds"] == 60.0 and out["served"] == [{"dropped": 0}]
    assert out["process"] == "a process of its own"
    cmd = seen["cmd"]
    assert cmd[0] == sys.executable and cmd[1].endswith("bench.py")
    assert "--serve-child" in cmd
    assert cmd[cmd.index("--serve-seconds") + 1] == "60.0"
    assert cmd[cmd.index("--plain-seconds") + 1] == "10.0"


def test_failed_child_gives_an_error_entry(monkeypatch):
    bench = _bench()
    monkeypatch.setattr(subprocess, "run",
                        lambda cmd, **kw: _Done(1, "", "Traceback\nRuntimeError: no device\n"))
    out = bench.serving_process(1.0, 0.0)
    assert "error" in out and "exited 1" in out["error"] and "no device" in out["error"]


def test_silent_child_gives_an_error_entry(monkeypatch):
    bench = _bench()
    monkeypatch.setattr(subprocess, "run", lambda cmd, **kw: _Done(0, "no json here\n"))
    assert "error" in bench.serving_process(1.0, 0.0)


def test_hung_child_gives_an_error_entry(monkeypatch):
    bench = _bench()

    def hang(cmd, **kw):
        raise subprocess.TimeoutExpired(cmd, kw.get("timeout", 0))

    monkeypatch.setattr(subprocess, "run", hang)
    assert bench.serving_process(1.0, 0.0) == {"error": "the serving process did not finish"}


def test_child_makes_its_frames_on_one_thread(monkeypatch):
    """The child's frames come from make_pool(threads=False): the same
    frames as the threaded pool, made without a thread pool."""
    bench = _bench()
    import concurrent.futures as cf

    class NoPool:
        def __init__(self, *a, **kw):
            raise AssertionError("the one-thread pool must not start threads")

    synth = bench.load_synth()
    monkeypatch.setattr(synth, "eiger_16m", lambda frames, dtype=None: synth.small())
    monkeypatch.setattr(cf, "ThreadPoolExecutor", NoPool)
    pool = bench.make_pool(3, threads=False)
    assert len(pool) == 3 and pool[0].shape == synth.SMALL
