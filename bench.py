#!/usr/bin/env python3
"""Benchmark of the spot-finder hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--batch F] [--pool P]

Workload: Eiger2-16M-shaped uint16 frames (4362 x 4148, slow x fast), seeded
synthetic data with module gaps, a Poisson ring background and 6000 Gaussian
reflections per frame. One step is one batch of F frames (default 16) through
the batched engine: the fused threshold kernel and the ordered compaction,
frames resident in HBM, two slots of distinct frames alternating. Every batch
is 580 MB, well over the 126 MB L2, so each step re-reads its frames from HBM.

Prints one JSON line (rank 0). `value` is frames/s over the timed steps from
CUDA events on the engine's stream (max over ranks); `e2e` is the same metric
through the public API from pinned host frames, with the host-to-device copy
of the frames and the device-to-host read of the signal lists inside the
timed region; `roofline` is the threshold kernel's algorithmic bytes per
launch over its event-timed launch duration; `cpu_baseline` is the
reference's own CPU code (dext.cc + dials_spots.cc, compiled from the
reference sources) on a bounded sample, all host cores.

--impl reference times that reference CPU path alone as the bench's reference
arm, on the same workload, metric and unit.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "16M uint16 frames/s (threshold+3D label), % HBM roofline; p99 frame latency"
UNIT = "frames/s"
SHAPE = (4362, 4148)
L2_BYTES = 126 * 1024 * 1024
# both arms name the workload the same way
WORKLOAD = "Eiger2-16M-shaped uint16 frames, 4362x4148, threshold + 3D grouping + spot pass"
# frames per step when the autotuner does not choose (its range is 8-32; it
# has chosen 32 on these frames), and the reference arm's step
DEFAULT_FRAMES = 32


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--batch", type=int, default=0,
                    help="frames per launch; 0: the autotuner's choice (8 to 32)")
    # Distinct consecutive frames of one series, cycled. With grouping in the
    # step the cycle must be longer than any reflection's extent in z (about
    # ten frames here): a reflection present at both ends of a short cycle
    # would be joined across the wrap into a streak that never closes.
    ap.add_argument("--pool", type=int, default=32, help="distinct synthetic frames")
    ap.add_argument("--e2e-steps", type=int, default=16)
    ap.add_argument("--cpu-frames", type=int, default=8)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--serve-seconds", type=float, default=60.0,
                    help="length of the two-stream serving replay (0: skip)")
    ap.add_argument("--plain-seconds", type=float, default=10.0,
                    help="length of the plain per-frame replay of the same streams")
    ap.add_argument("--no-4m", action="store_true")
    ap.add_argument("--no-u32", action="store_true")
    ap.add_argument("--no-stills", action="store_true")
    ap.add_argument("--serve-child", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--no-parity", action="store_true",
                    help="skip the check of one step's output against the oracle")
    ap.add_argument("--no-tune", action="store_true",
                    help="skip the autotuner (frames per launch 16 unless --batch)")
    return ap.parse_args()


# -- ranks ------------------------------------------------------------------

class Ranks:
    """One process per GPU under torchrun; replicas only (no data exchange on
    the path), so the process group carries nothing but barriers and the
    max-over-ranks of the timings."""

    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime

            import torch.distributed as dist
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=300))
            self.dist = dist

    def barrier(self):
        if self.world > 1:
            self.dist.barrier()

    def max(self, v: float) -> float:
        if self.world == 1:
            return v
        import torch
        t = torch.tensor([v], dtype=torch.float64)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, v: float) -> float:
        if self.world == 1:
            return v
        import torch
        t = torch.tensor([v], dtype=torch.float64)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.world > 1:
            self.dist.destroy_process_group()


# -- clocks -----------------------------------------------------------------

REASONS = {0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap",
           0x8: "hw_slowdown", 0x10: "sync_boost", 0x20: "sw_thermal_slowdown",
           0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown",
           0x100: "display_clock_setting"}


class ClockSampler:
    def __init__(self, device: int):
        self.device = device
        self.samples = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device),
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 4:
                try:
                    self.samples.append((float(parts[0]), float(parts[1]),
                                         float(parts[2]), int(parts[3], 16)))
                except ValueError:
                    pass

    def __exit__(self, *exc):
        time.sleep(0.3)
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        busy = [s for s in self.samples if not (s[3] & 0x1)] or self.samples
        mask = 0
        for s in busy:
            mask |= s[3]
        return {"sm_mhz": statistics.median(s[0] for s in busy),
                "sm_max_mhz": max(s[1] for s in busy),
                "power_w_max": max(s[2] for s in busy),
                "samples": len(busy),
                "reasons": [name for bit, name in REASONS.items() if mask & bit and bit != 0x1]}


# -- data -------------------------------------------------------------------

def load_synth():
    """The synthetic-series module on its own, without importing the package
    (whose import maps the product library): the reference arm must run with
    nothing of the product loaded."""
    import importlib.util
    name = "_spotfinder_synth"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(
        name, os.path.join(ROOT, "dials_metal_spotfinder_b200", "synth.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def make_pool(n: int, dtype=np.uint16, threads: bool = True):
    """n synthetic 16M frames, made on host threads unless `threads` is
    false. The serving replay's process makes them on one thread: in a
    process whose frames were made on 16 threads, the replay's server saw
    stalls of 70-100 ms that dropped frames, and kept seeing them after the
    frames were freed; the same replay after one-thread generation dropped
    none. What in that process's state causes it was not found."""
    series = load_synth().eiger_16m(frames=max(n, 3), dtype=dtype)
    if not threads:
        return [series.frame(f) for f in range(n)]
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(min(16, os.cpu_count() or 1)) as ex:
        return list(ex.map(series.frame, range(n)))


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def recorded_traffic():
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


# -- the reference CPU path -------------------------------------------------

def cpu_reference(frames, threads):
    """The reference's dext<uint16_t> on `threads` workers over frames already
    in memory, and its Labeller fed in frame order on this thread, as
    src/find_spots.cc:472-591 does without the HDF5 read and decompression.
    Uses oracle/_ref (the reference's own sources) where built, else the C
    restatement. Returns (seconds, kind)."""
    from concurrent.futures import ThreadPoolExecutor

    from oracle import oracle as O
    use_ref = O.ref_available()
    h, w = frames[0].shape
    t0 = time.perf_counter()
    lab = O.Labeller(h, w, use_ref=use_ref)
    with ThreadPoolExecutor(threads) as pool:
        for z, (status, sig, _) in enumerate(pool.map(lambda im: O.dext(im, use_ref=use_ref),
                                                      frames)):
            lab.add(z, sig)
    lab.finish()
    return time.perf_counter() - t0, ("reference" if use_ref else "port")


# -- arms -------------------------------------------------------------------

def mapped_libraries():
    """The shared objects of this repository mapped into the process."""
    found = set()
    try:
        with open("/proc/self/maps") as fh:
            for line in fh:
                path = line.split()[-1] if len(line.split()) >= 6 else ""
                if path.endswith(".so") and os.path.realpath(path).startswith(
                        os.path.realpath(ROOT)):
                    found.add(os.path.relpath(os.path.realpath(path), os.path.realpath(ROOT)))
    except OSError:
        pass
    return sorted(found)


def run_reference_arm(args, ranks):
    if ranks.rank != 0:
        return
    threads = os.cpu_count() or 1
    # the same frames per step as the product arm (--batch fixes both arms;
    # otherwise its autotuner picks, 32 on these frames)
    n = args.batch or DEFAULT_FRAMES
    frames = make_pool(n)
    for _ in range(max(0, min(args.warmup, 1))):
        cpu_reference(frames[:2], threads)
    times = []
    for _ in range(max(1, args.steps)):
        dt, kind = cpu_reference(frames, threads)
        times.append(dt)
        if sum(times) > 120:
            break
    value = n * len(times) / sum(times)
    print(json.dumps({
        "mapped_libraries": mapped_libraries(),
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": len(times), "warmup": args.warmup,
        "ms_per_step": 1000 * sum(times) / len(times), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u16/f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "frames_per_step": n, "shape": list(SHAPE),
                   "where": "the reference's dext.cc + dials_spots.cc on the host cores"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                         "sample": f"{n} frames of 4362x4148 per step"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }), flush=True)


def run_ours(args, ranks):
    import dials_metal_spotfinder_b200 as sf
    from dials_metal_spotfinder_b200 import _lib
    from dials_metal_spotfinder_b200.engine import Engine

    _lib.raise_for(_lib.lib.sf_set_device(ranks.local), "sf_set_device")
    pool = make_pool(args.pool)
    frame_bytes = SHAPE[0] * SHAPE[1] * 2
    # frames per launch, warps per block and task height from the autotuner
    # (a timed search, or its tuner file when this device has one)
    tuning = None
    if not args.no_tune:
        from dials_metal_spotfinder_b200.tune import tune
        t0 = time.perf_counter()
        tuning = tune(pool[:16], min_frames=8, max_frames=32)
        tuning["seconds"] = time.perf_counter() - t0
    F = args.batch or (tuning["frames_per_launch"] if tuning else DEFAULT_FRAMES)
    eng = Engine([SHAPE] * F, np.uint16, slots=2)
    eng.enable_grouping(first_frame=0)
    info = eng.info()
    engine_tuning = eng.tuning()
    for s in range(2):
        for f in range(F):
            eng.upload(s, f, pool[(s * F + f) % len(pool)])
    eng.synchronize()

    # warm-up
    for i in range(args.warmup):
        eng.run(i % 2)
    eng.synchronize()

    # timed: resident frames, the whole step (threshold, ordered compaction,
    # 3D grouping and the spot pass) on the device; a step's threshold
    # overlaps the previous step's grouping
    accepted0 = eng.group_counts()[0]["accepted"]
    ranks.barrier()
    with ClockSampler(ranks.local) as clocks:
        eng.record(0)
        for i in range(args.steps):
            eng.run(i % 2)
        eng.record(1)
        eng.synchronize()
    ms = eng.elapsed_ms(0, 1)
    spots_per_frame = (eng.group_counts()[0]["accepted"] - accepted0) / (F * args.steps)
    ranks.barrier()
    ms_max = ranks.max(ms)

    # the stages one by one: the same steps with per-stage events, each step
    # kept apart from the next so that every kernel times alone
    eng.profile(True)
    for i in range(args.steps):
        eng.run(i % 2)
    eng.synchronize()
    stage = eng.stage_totals()
    eng.profile(False)
    counts = [eng.counts(s) for s in range(2)]
    nsig_per_step = [int(c.sum()) for c in counts]
    group_counts, live = eng.group_counts()
    frames_total = ranks.sum(F * args.steps)
    value = frames_total / (ms_max / 1000.0)

    # the same steps replayed from CUDA graphs
    eng.use_graph(True)
    for i in range(2):
        eng.run(i % 2)
    eng.synchronize()
    eng.record(2)
    for i in range(args.steps):
        eng.run(i % 2)
    eng.record(3)
    eng.synchronize()
    graph_ms = ranks.max(eng.elapsed_ms(2, 3))
    eng.use_graph(False)

    # roofline of the threshold kernel: algorithmic bytes per launch (one read
    # of every frame plus one 16-byte record per signal pixel) over the
    # kernel's average event-timed duration
    alg_bytes = statistics.mean(F * frame_bytes + 16 * n for n in nsig_per_step)
    thr_ms = stage["threshold_ms"] / max(stage["runs"], 1)
    achieved = alg_bytes / (thr_ms / 1000.0) / 1e9
    peak, peak_kind = measured_peaks()
    traffic = recorded_traffic().get(f"threshold_u16_{SHAPE[0]}x{SHAPE[1]}_per_frame")

    # e2e: pinned host frames -> device -> the finished spots and their
    # pixels back into pinned host memory, every step. Pipelined the way a
    # user drives the engine: step i+1's frames stream in on the copy engine
    # while step i computes and its results come back on the other direction
    # of the link.
    e2e = e2e_chunks = None
    if args.e2e_steps > 0:
        hb = [sf.HostBuffer(SHAPE, np.uint16) for _ in range(F)]
        for f in range(F):
            hb[f].array[:] = pool[f % len(pool)]

        def e2e_upload(slot):
            for f in range(F):
                eng.upload(slot, f, hb[f].array)

        # result buffers sized from one untimed step
        e2e_upload(0)
        eng.run(0)
        n_spots, n_pix = len(eng.spots()), len(eng.pixels())
        spot_buf = sf.HostBuffer((2 * n_spots + (1 << 16),), sf.SPOT)
        pix_buf = sf.HostBuffer((2 * n_pix + (1 << 20),), sf.PIXEL)
        d2h = []

        def e2e_read():
            sp = eng.spots(out=spot_buf.array)
            px = eng.pixels(out=pix_buf.array)
            d2h.append(sp.nbytes + px.nbytes)

        eng.synchronize()
        ranks.barrier()
        t0 = time.perf_counter()
        e2e_upload(0)
        eng.run(0)
        for i in range(1, args.e2e_steps):
            e2e_upload(i % 2)
            e2e_read()          # step i-1, overlapping step i's upload
            eng.run(i % 2)
        e2e_read()
        eng.synchronize()
        dt = ranks.max(time.perf_counter() - t0)
        e2e = {"value": ranks.sum(F * args.e2e_steps) / dt, "unit": UNIT,
               "h2d_bytes_per_step": F * frame_bytes,
               "d2h_bytes_per_step": int(statistics.mean(d2h)),
               "timer": "host wall clock, synchronised at both ends",
               "form": "Engine.upload from pinned host frames, run, spots/pixels into "
                       "pinned host arrays; step i+1 uploads while step i computes and "
                       "reads back"}

        # the same with the frames as the detector writes them, bslz4 chunks:
        # only the compressed bytes cross PCIe, and the engine decodes them
        from dials_metal_spotfinder_b200 import chunk as C
        cb = []
        for f in range(F):
            c = C.encode(pool[f % len(pool)], "bslz4")
            b = sf.HostBuffer((len(c),), np.uint8)
            b.array[:] = c
            cb.append(b)
        chunk_bytes = sum(len(b.array) for b in cb)

        def chunk_upload(slot):
            eng.upload_chunks(slot, [b.array for b in cb])

        def chunk_upload_each(slot):
            for f in range(F):
                eng.upload_chunk(slot, f, cb[f].array)

        def timed_chunks(upload):
            upload(0)
            eng.run(0)
            e2e_read()
            eng.synchronize()
            d2h.clear()
            ranks.barrier()
            t0 = time.perf_counter()
            upload(0)
            eng.run(0)
            for i in range(1, args.e2e_steps):
                upload(i % 2)
                e2e_read()
                eng.run(i % 2)
            e2e_read()
            eng.synchronize()
            return ranks.max(time.perf_counter() - t0)

        dt = timed_chunks(chunk_upload)
        e2e_chunks = {"value": ranks.sum(F * args.e2e_steps) / dt, "unit": UNIT,
                      "h2d_bytes_per_step": chunk_bytes,
                      "d2h_bytes_per_step": int(statistics.mean(d2h)),
                      "timer": "host wall clock, synchronised at both ends",
                      "form": "Engine.upload_chunks of bslz4 chunks from pinned host memory "
                              "(framing checked on host threads, decoded on the device), "
                              "run, spots/pixels into pinned host arrays; pipelined as e2e"}
        # the same steps with the chunks handed over one call each
        # (upload_chunk), their framing walked on the calling thread: what
        # the batched call's parallel framing walk is worth, in one run
        dt_each = timed_chunks(chunk_upload_each)
        e2e_chunks["one_call_per_chunk"] = {
            "value": ranks.sum(F * args.e2e_steps) / dt_each, "unit": UNIT,
            "form": "Engine.upload_chunk per frame, otherwise as above"}
        for b in hb + cb + [spot_buf, pix_buf]:
            b.close()

    # the plain per-frame GPU form, the same frame through sf_find_u16
    plain = None
    if ranks.rank == 0:
        hb0 = sf.HostBuffer(SHAPE, np.uint16)
        hb0.array[:] = pool[0]
        sig0 = sf.HostBuffer((SHAPE[0] * SHAPE[1] * 2 // 16,), sf.SIGNAL_PIXEL)
        for _ in range(2):
            sf.find(hb0.array, out=sig0.array)
        t0 = time.perf_counter()
        nplain = 10
        for _ in range(nplain):
            sf.find(hb0.array, out=sig0.array)
        plain = {"value": nplain / (time.perf_counter() - t0), "unit": UNIT,
                 "form": "sf_find_u16, one frame per call, pinned host frame and "
                         "pinned signal list"}
        hb0.close()
        sig0.close()

    ref_gpu = None
    if ranks.rank == 0:
        ref_gpu = reference_gpu_form(pool[0])

    four_m = None
    if ranks.rank == 0 and not args.no_4m:
        four_m = batched_vs_plain_4m()

    u32 = None
    if ranks.rank == 0 and not args.no_u32:
        u32 = u32_16m(args.steps)

    stills = None
    if ranks.rank == 0 and not args.no_stills:
        stills = stills_uneven()

    served = None
    if ranks.rank == 0 and args.serve_seconds > 0:
        served = serving_process(args.serve_seconds, args.plain_seconds)

    cpu = None
    if ranks.rank == 0 and ranks.world == 1 and not args.no_cpu:
        n = max(2, args.cpu_frames)
        frames = [pool[i % len(pool)] for i in range(n)]
        threads = os.cpu_count() or 1
        dt, kind = cpu_reference(frames, threads)
        cpu = {"value": n / dt, "unit": UNIT, "cores": threads, "kind": kind,
               "sample": f"{n} frames of 4362x4148, threshold on {threads} threads "
                         "and 3D grouping on one, as the reference CLI runs them"}

    # threshold; placement reduce, scan, copy; grouping: setup, gather, link,
    # keep_table, flatten, mark, compact, count, rank, scatter, accept (small
    # and large components), write, carry, finalize, and 5 scans of 3
    # launches
    launches_per_step = 1 + 3 + (16 + 5 * 3)
    # the whole pipeline's algorithmic bytes per frame: one read of the
    # frame, the signal list written and read back by the grouping, the
    # spot rows written
    sig_per_frame = statistics.mean(nsig_per_step) / F
    pipe_bytes = frame_bytes + 32 * sig_per_frame + 104 * spots_per_frame
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ranks.world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u16 pixels, u32 sums, f32 tests, f64 spots", "data": "synthetic",
        "config": {"workload": WORKLOAD, "shape": list(SHAPE),
                   "frames_per_step": F, "slots": 2, "distinct_frames": len(pool),
                   "where": "the batched engine on the device",
                   "l2": f"inputs larger than L2 ({F * frame_bytes / 1e6:.0f} MB per step)",
                   "parallelism": f"replicas x{ranks.world}",
                   "engine": info},
        "tuning": {"search": tuning, "engine": engine_tuning},
        "graph_replay": {"value": frames_total / (graph_ms / 1000.0), "unit": UNIT,
                         "ms_per_step": graph_ms / args.steps},
        "grouping": {"spots_per_frame": spots_per_frame,
                     "counts": group_counts, "live": live},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "kernel": "threshold_kernel<uint16_t>",
                     "kernel_ms_per_launch": thr_ms,
                     "algorithmic_bytes_per_launch": alg_bytes,
                     "traffic": (traffic * F if traffic else None)},
        "stage_ms_per_step": {"threshold": thr_ms,
                              "placement": stage["place_ms"] / max(stage["runs"], 1),
                              "grouping": stage["group_ms"] / max(stage["runs"], 1)},
        "signal_pixels_per_frame": sig_per_frame,
        "gpixels_per_s": value * SHAPE[0] * SHAPE[1] / 1e9,
        "pipeline_bytes": {"per_frame": pipe_bytes,
                           "achieved_gbs": value * pipe_bytes / 1e9,
                           "frac": value * pipe_bytes / 1e9 / peak, "peak_kind": peak_kind,
                           "counted": "frame read + 32 B per signal pixel (list written, "
                                      "read by the grouping) + 104 B per spot row"},
        "clocks": clocks.summary(),
        "gpu_launches": launches_per_step * args.steps,
        "e2e": e2e,
        "e2e_chunks": e2e_chunks,
        "plain_gpu": plain,
        "reference_gpu": ref_gpu,
        "batched_vs_plain_4m": four_m,
        "u32_16m": u32,
        "stills_uneven": stills,
        "latency": ({"frame_to_mask_p99_ms": {
                        name: r["frame_to_mask_ms"]["p99"]
                        for name, r in zip(("4m_500hz", "16m_100hz"), served["served"])},
                     "frame_to_spot_p99_ms": {
                        name: r["frame_to_spot_ms"]["p99"]
                        for name, r in zip(("4m_500hz", "16m_100hz"), served["served"])},
                     "source": "serving"} if served else None),
        "serving": served,
        "cpu_baseline": cpu,
    }
    eng.close()
    # the step's output checked against the oracle, outside every timed region
    line["parity"] = parity_check(pool, F) if ranks.rank == 0 and not args.no_parity else None
    if ranks.rank == 0:
        print(json.dumps(line), flush=True)


def parity_check(pool, F):
    """Two steps of the timed form -- the same engine configuration (F frames
    per run, two slots, 3D grouping with components carried between runs) on
    the bench's first 2F frames, then finish -- against the oracle's dext +
    Labeller on the same frames: every signal list of the second step, every
    spot field and pixel, and the counts. Returns "ok" or what differed."""
    from concurrent.futures import ThreadPoolExecutor

    from dials_metal_spotfinder_b200.engine import Engine
    from oracle import oracle as O
    frames = [pool[i % len(pool)] for i in range(2 * F)]
    spots, pixels = [], []
    with Engine([SHAPE] * F, np.uint16, slots=2) as eng:
        eng.enable_grouping(first_frame=0)
        for b in range(2):
            for f in range(F):
                eng.upload(b, f, frames[b * F + f])
            eng.run(b)
            spots.append(eng.spots())
            pixels.append(eng.pixels())
        lists = [eng.signal(1, f) for f in range(F)]
        eng.finish()
        spots.append(eng.spots())
        pixels.append(eng.pixels())
        counts, _ = eng.group_counts()
    spots, pixels = np.concatenate(spots), np.concatenate(pixels)
    with ThreadPoolExecutor(os.cpu_count() or 1) as ex:
        want_lists = [sig for _, sig, _ in ex.map(O.dext, frames)]
    want = O.group(want_lists, *SHAPE)
    out = {"frames": 2 * F, "spots": len(spots), "pixels": len(pixels),
           "against": "oracle dext + Labeller (C restatement of src/dext.cc, "
                      "src/dials_spots.cc)"}
    bad = [f for f in range(F) if lists[f].tobytes() != want_lists[F + f].tobytes()]
    if bad:
        out["status"] = f"signal lists differ on frames {bad}"
    elif counts != want.counts:
        out["status"] = f"counts differ: {counts} vs {want.counts}"
    elif len(spots) != len(want.spots) or any(
            np.ascontiguousarray(spots[k]).tobytes() !=
            np.ascontiguousarray(want.spots[k]).tobytes() for k in want.spots.dtype.names):
        out["status"] = "spot fields differ"
    elif pixels.tobytes() != want.pixels.tobytes():
        out["status"] = "pixels differ"
    else:
        out["status"] = "ok"
    return out


def batched_vs_plain_4m(steps: int = 12):
    """4M-shaped frames (2162 x 2068), the batched engine (16 frames per
    launch) against the plain per-frame form (sf_find_u16, one frame per
    call), like for like: both fed from the same page-locked host frames,
    both returning their results to page-locked host memory, both timed on
    the host wall clock over the same work.

    threshold: the signal lists only -- batched: upload 16 frames, run
    without grouping, read the 16 lists (one call), step i+1's upload
    overlapping step i's run and read; plain: sf_find_u16 per frame.
    grouped: threshold + 3D grouping, the finished spots and their pixels
    returned -- batched: the engine with grouping; plain: sf_find_u16 per
    frame then the device labeller's add (sf_labeller_add), the reference
    CLI's per-frame order (src/find_spots.cc:243-264,550-591)."""
    import dials_metal_spotfinder_b200 as sf
    from dials_metal_spotfinder_b200.engine import Engine
    from dials_metal_spotfinder_b200.labeller import Labeller
    series = load_synth().eiger_4m(frames=32)
    pool = [series.frame(f) for f in range(32)]
    shape = pool[0].shape
    F = 16
    cap = shape[0] * shape[1] * 2 // 16
    hb = [sf.HostBuffer(shape, np.uint16) for _ in range(32)]
    for f in range(32):
        hb[f].array[:] = pool[f]
    lists = sf.HostBuffer((F * cap,), sf.SIGNAL_PIXEL)
    one = sf.HostBuffer((cap,), sf.SIGNAL_PIXEL)
    spot_buf = sf.HostBuffer((1 << 18,), sf.SPOT)
    pix_buf = sf.HostBuffer((1 << 22,), sf.PIXEL)
    out = {"workload": "4M-shaped uint16 frames, 2162x2068", "unit": UNIT,
           "timer": "host wall clock, synchronised at both ends",
           "input": "page-locked host frames, 32 distinct, cycled",
           "batched_form": "engine, 16 frames per launch, two slots, step i+1 uploading "
                           "while step i runs and reads back",
           "plain_form": "sf_find_u16 per frame (upload, threshold, list back), one call "
                         "after another"}

    def batched(grouping):
        with Engine([shape] * F, np.uint16, slots=2) as eng:
            if grouping:
                eng.enable_grouping(first_frame=0)

            def upload(i):
                for f in range(F):
                    eng.upload(i % 2, f, hb[(i * F + f) % 32].array)

            def read(i):
                if grouping:
                    eng.spots(out=spot_buf.array)
                    eng.pixels(out=pix_buf.array)
                else:
                    eng.signals(i % 2, out=lists.array)

            for rep in range(2):  # the first pass warms up
                eng.synchronize()
                t0 = time.perf_counter()
                upload(0)
                eng.run(0)
                for i in range(1, steps):
                    upload(i)
                    read(i - 1)
                    eng.run(i % 2)
                read(steps - 1)
                eng.synchronize()
                dt = time.perf_counter() - t0
            return F * steps / dt

    def plain(grouping):
        n = F * steps
        lab = Labeller(*shape) if grouping else None
        for rep in range(2):
            t0 = time.perf_counter()
            for i in range(n):
                sig = sf.find(hb[i % 32].array, out=one.array)
                if grouping:
                    lab.add(rep * n + i, sig)
            if grouping:  # the spots and pixels found so far, to the host
                lab.spots()
                lab.pixels()
            dt = time.perf_counter() - t0
        if lab:
            lab.close()
        return n / dt

    try:
        for name, grouping in (("threshold", False), ("grouped", True)):
            b, p = batched(grouping), plain(grouping)
            out[name] = {"batched": b, "plain": p, "ratio": b / p}
    finally:
        for b in hb + [lists, one, spot_buf, pix_buf]:
            b.close()
    return out


def stills_uneven(frames_per_series: int = 500):
    """Uneven batched stills: four series of panel sizes 1028x1062,
    2068x2162, 3110x3269 and 4148x4362 (fast x slow) interleaved in the same
    launches, four frames of each per launch, 2D grouping (each frame on its
    own), frames resident, CUDA events; `frames_per_series` frames of each
    series in all. Spot density 0.5 per 1000 px^2 as the stills
    configuration has it."""
    from dials_metal_spotfinder_b200.engine import Engine
    synth = load_synth()
    per = 4
    shapes = [tuple(s) for s in synth.STILL_SHAPES]
    pools = [[synth.still(s, frames=8).frame(f) for f in range(8)] for s in shapes]
    layout = [k for k in range(len(shapes)) for _ in range(per)]
    steps = max(1, frames_per_series // per)
    with Engine([shapes[k] for k in layout], np.uint16, slots=2) as eng:
        eng.enable_grouping(first_frame=0, two_d=True)
        for s in range(2):
            for f, k in enumerate(layout):
                eng.upload(s, f, pools[k][(s * per + f % per) % 8])
        eng.synchronize()
        for i in range(3):
            eng.run(i % 2)
        eng.synchronize()
        eng.record(0)
        for i in range(steps):
            eng.run(i % 2)
        eng.record(1)
        eng.synchronize()
        ms = eng.elapsed_ms(0, 1)
        spots = sum(eng.group_counts(k)[0]["accepted"] for k in range(eng.nseries()))
    frames = steps * len(layout)
    px = steps * per * sum(h * w for h, w in shapes)
    return {"workload": "uneven stills: 1028x1062, 2068x2162, 3110x3269, 4148x4362 uint16, "
                        "interleaved, 2D grouping", "unit": UNIT,
            "value": frames / (ms / 1e3), "frames_per_step": len(layout),
            "frames_per_series": steps * per, "gpixels_per_s": px / (ms / 1e3) / 1e9,
            "ms_per_step": ms / steps, "spots": spots,
            "form": "batched engine, resident frames (8 distinct per series, cycled), "
                    "CUDA events"}


def u32_16m(steps: int):
    """The 16M uint32 variant (intensities up to 2e6): threshold + 3D
    grouping through the batched engine, frames resident, CUDA events as the
    headline's; the uint32 threshold kernel's roofline beside it."""
    from dials_metal_spotfinder_b200.engine import Engine
    F = 16
    pool = make_pool(24, np.uint32)
    shape = pool[0].shape
    frame_bytes = shape[0] * shape[1] * 4
    with Engine([shape] * F, np.uint32, slots=2) as eng:
        eng.enable_grouping(first_frame=0)
        for s in range(2):
            for f in range(F):
                eng.upload(s, f, pool[(s * F + f) % len(pool)])
        eng.synchronize()
        for i in range(3):
            eng.run(i % 2)
        eng.synchronize()
        eng.record(0)
        for i in range(steps):
            eng.run(i % 2)
        eng.record(1)
        eng.synchronize()
        ms = eng.elapsed_ms(0, 1)
        eng.profile(True)
        for i in range(steps):
            eng.run(i % 2)
        eng.synchronize()
        stage = eng.stage_totals()
        eng.profile(False)
        nsig = [int(eng.counts(s).sum()) for s in range(2)]
    alg = statistics.mean(F * frame_bytes + 16 * n for n in nsig)
    thr_ms = stage["threshold_ms"] / max(stage["runs"], 1)
    peak, peak_kind = measured_peaks()
    achieved = alg / (thr_ms / 1e3) / 1e9
    return {"workload": "Eiger2-16M-shaped uint32 frames, 4362x4148, intensities up to 2e6, "
                        "batched engine, threshold + 3D grouping",
            "value": F * steps / (ms / 1e3), "unit": UNIT, "frames_per_step": F,
            "ms_per_step": ms / steps, "signal_pixels_per_frame": statistics.mean(nsig) / F,
            "stage_ms_per_step": {"threshold": thr_ms,
                                  "placement": stage["place_ms"] / max(stage["runs"], 1),
                                  "grouping": stage["group_ms"] / max(stage["runs"], 1)},
            "roofline": {"bound": "hbm", "kernel": "threshold_kernel<uint32_t>",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "kernel_ms_per_launch": thr_ms, "algorithmic_bytes_per_launch": alg}}


def serving(seconds: float, plain_seconds: float, pool16):
    """Two live streams on one device through the serving loop, frames as
    bitshuffle/LZ4 chunks decoded on the device: 4M at 500 Hz and 16M at
    100 Hz. Then the plain per-frame form (host decode, sf_find_u16,
    labeller) on the same streams for plain_seconds."""
    from dials_metal_spotfinder_b200 import chunk as C
    from dials_metal_spotfinder_b200.serve import Stream, drive, drive_plain
    # distinct frames cycled, longer than any reflection's z extent
    n = min(24, len(pool16))
    s4 = load_synth().eiger_4m(frames=n)
    c4 = [C.encode(s4.frame(f), "bslz4") for f in range(n)]
    c16 = [C.encode(f, "bslz4") for f in pool16[:n]]
    raw4 = s4.height * s4.width * 2
    raw16 = pool16[0].nbytes

    def streams(sec):
        return [Stream((s4.height, s4.width), c4, rate_hz=500.0, frames=max(1, int(500 * sec))),
                Stream(pool16[0].shape, c16, rate_hz=100.0, frames=max(1, int(100 * sec)))]
    out = {"streams": "4M (2162x2068) at 500 Hz and 16M (4362x4148) at 100 Hz, bslz4 chunks",
           "compression": {"4m": raw4 / statistics.mean(len(c) for c in c4),
                           "16m": raw16 / statistics.mean(len(c) for c in c16)},
           "seconds": seconds, "served": drive(streams(seconds))}
    if plain_seconds > 0:
        out["plain_seconds"] = plain_seconds
        out["plain"] = drive_plain(streams(plain_seconds))
    return out


def serving_process(seconds: float, plain_seconds: float):
    """`serving` in a Python process of its own, as a detector's server runs:
    this process has by then held several engines, gigabytes of page-locked
    buffers and thread pools, none of which a server shares a process with.
    The child makes the same 16M frames from the same seeds."""
    cmd = [sys.executable, os.path.abspath(__file__), "--serve-child",
           "--serve-seconds", str(seconds), "--plain-seconds", str(plain_seconds)]
    try:
        r = subprocess.run(cmd, capture_output=True, text=True,
                           timeout=seconds + plain_seconds + 900)
    except subprocess.TimeoutExpired:
        return {"error": "the serving process did not finish"}
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    if r.returncode != 0 or not lines:
        tail = (r.stderr.strip().splitlines() or ["no output"])[-1]
        return {"error": f"the serving process exited {r.returncode}: {tail}"}
    out = json.loads(lines[-1])
    out["process"] = "a process of its own"
    return out


def reference_gpu_form(frame):
    """The reference's own CUDA backend (src/dext_cuda.cu via its gpu::find),
    built for sm_100a from the reference sources, on the same frame."""
    try:
        import ctypes

        from oracle import oracle as O
        lib = O.ref_gpu_lib()
    except Exception as exc:  # not built where the reference tree was absent
        return {"unavailable": str(exc)}
    import dials_metal_spotfinder_b200 as sf
    lib.refgpu_quiet()
    hb = sf.HostBuffer(frame.shape, np.uint16)
    hb.array[:] = frame
    cap = frame.size * 2 // 16
    out = np.empty(cap, sf.SIGNAL_PIXEL)
    found = ctypes.c_size_t(0)
    for _ in range(2):
        lib.refgpu_find_u16(hb.array.ctypes.data, frame.shape[0], frame.shape[1],
                            out.ctypes.data, cap, ctypes.byref(found))
    n = 10
    t0 = time.perf_counter()
    for _ in range(n):
        st = lib.refgpu_find_u16(hb.array.ctypes.data, frame.shape[0], frame.shape[1],
                                 out.ctypes.data, cap, ctypes.byref(found))
    dt = time.perf_counter() - t0
    hb.close()
    return {"value": n / dt, "unit": UNIT, "status": st, "signal_pixels": found.value,
            "form": "reference src/dext_cuda.cu gpu::find, one frame per call, sm_100a"}


def main():
    args = parse()
    if args.serve_child:
        pool = make_pool(24, threads=False)
        print(json.dumps(serving(args.serve_seconds, args.plain_seconds, pool)), flush=True)
        return
    ranks = Ranks()
    try:
        if args.impl == "reference":
            run_reference_arm(args, ranks)
        else:
            run_ours(args, ranks)
    finally:
        ranks.close()


if __name__ == "__main__":
    main()
