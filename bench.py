#!/usr/bin/env python
"""Benchmark of the B200 macroblock engine on the 1080p High-profile workload.

Workload (one "step"): a seeded synthetic 1920x1080 4:2:0 clip of 120 frames (sum of four
gratings + blurred noise, +-24 px quarter-sample global motion, 12 moving textured rectangles),
encoded as ragdoll transcode cuts it -- 8 independent 15-frame GOPs (IDR + 14 P), High profile
decisions (8x8 transform), fixed QP 26 -- with the 8 GOPs analysed side by side in one persistent
launch. The device step covers analysis, reconstruction, deblocking and border extension of all
120 frames; the learned form's step also runs the candidate network and the coarse motion pass.

The default line is the learned form against the plain (Balanced) form:
value:  frames/s of the learned form's device step (network, coarse motion, persistent analysis
        launch; sources resident in HBM).
e2e:    frames/s of the learned form through the public encoder (rg_encoder_set_form, then
        rg_encoder_submit / _collect): host->device copy of every frame from pinned host memory,
        the launches, device->host copy of every macroblock record, and the CABAC access units of
        all 120 pictures written on the host cores -- two waves in flight.
bd_rate_vs_plain_pct: Bjontegaard delta rate of the learned form against the plain form (bits at
        equal luma PSNR over QP 22 / 26 / 30 / 34, every access unit written); `rd` the points.
plain:  the plain form's device frames/s, its e2e through the same encoder (and the analysis-only
        host-buffer call), its HBM roofline, and the parity of its bitstream with the oracle.
--impl reference: the CPU restatement of ragdoll's encoder (the oracle) on the same workload
        sample, GOP-parallel across the host cores (parallel_gop_map semantics).
--workload batched: the batched-streams configuration instead (64 streams of four sizes, a QP
        per stream; aggregate frames/s and per-frame latency percentiles; see run_batched).

Multi-GPU (torchrun): every rank encodes its own 120-frame clip (weak scaling, no collective on
the data path); the timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

W, H, FRAMES, GOP, QP = 1920, 1080, 120, 15, 26
MOTION, RECTS = 24.0, 12
METRIC = "1080p H.264 encode frames/s: learned vs plain GPU, equal PSNR, \u22642% bit cost"
UNIT = "frames/s"
BYTES_PER_FRAME = 7.5 * W * H  # source 1.5 + reference 1.5 + recon 1.5 + deblock read/write 3.0 (x W*H)
# DRAM bytes per picture of pipeline_kernel measured by ncu (dram__bytes_read + write) on a launch
# of 8 streams x 4 pictures of this workload: 490.2 MB / 32 (scaled to a launch by its pictures).
TRAFFIC_PER_FRAME = 490.2e6 / 32


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def bench_config(world: int, mode: str = "pipelined") -> dict:
    """The workload both arms report (the engine arm and --impl reference)."""
    return {"workload": "1080p High QP26 Balanced, 120 frames = 8 GOPs x 15 (IDR + 14 P) side by side",
            "mode": mode, "width": W, "height": H, "frames_per_gpu": FRAMES, "gop": GOP, "qp": QP,
            "profile": "high", "motion_px": MOTION, "rects": RECTS, "parallelism": f"replicas x{world}",
            "l2": "inputs larger than L2 (373 MB source clip per GPU)"}


def clip_seed(rank: int) -> int:
    """Each rank encodes its own clip (replicas, weak scaling): distinct content per GPU."""
    return 2000 + 97 * rank


def max_over_ranks(x: float, dist, device) -> float:
    """The slowest rank's time (every multi-GPU number is the max over ranks)."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def make_clip(seed: int, frames: int = FRAMES):
    from ragdoll_b200.synth import grating_clip
    return grating_clip(W, H, frames, seed=seed, motion=MOTION, rects=RECTS)


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while the timed region runs."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        rows = []
        for line in Path(self.path).read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 8:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[0]) for r in rows if r[0].replace(".", "").isdigit()]
        smax = float(rows[0][1]) if rows[0][1].replace(".", "").isdigit() else None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[4 + k].lower() == "active"})
        loaded = [s for s in sm if smax and s > 0.5 * smax] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": smax,
                "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------------------------------------------
def oracle_gops(clip, gops: int, frames_per_gop: int, threads: int, keep: bool = False):
    """Encodes `gops` GOPs of the clip with the oracle on `threads` host threads. Returns the
    seconds taken and (keep=True) each GOP's access units."""
    sys.path.insert(0, str(ROOT / "tests"))
    from oracle_lib import OracleEncoder

    work = list(range(gops))
    lock = threading.Lock()
    aus = [None] * gops

    def worker():
        while True:
            with lock:
                if not work:
                    return
                g = work.pop(0)
            enc = OracleEncoder(W, H, QP, profile=2, keyint=GOP)
            out = []
            for i in range(frames_per_gop):
                au, _ = enc.encode(clip[g * GOP + i])
                if keep:
                    out.append(au)
            aus[g] = out

    t0 = time.perf_counter()
    ts = [threading.Thread(target=worker) for _ in range(min(threads, gops))]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    return time.perf_counter() - t0, aus


def oracle_sample(clip, gops: int, cores: int) -> dict:
    """The CPU figures beside the GPU numbers: the oracle encoding the whole step (every GOP, all
    its pictures) GOP-parallel on the host cores, the same for one GOP on one thread, and the
    integer work the oracle's decisions evaluate per frame (pixel differences of every SAD / SSD /
    SATD). Also returns the oracle's access units of the step (key "aus", [g][f]) for the parity
    check of the GPU's bitstream."""
    sys.path.insert(0, str(ROOT / "tests"))
    from oracle_lib import pixel_ops
    pixel_ops(reset=True)
    t, aus = oracle_gops(clip, gops, GOP, cores, keep=True)
    ops = pixel_ops(reset=True)
    t1, _ = oracle_gops(clip, 1, GOP, 1)
    return {"value": round(gops * GOP / t, 3), "unit": UNIT, "cores": min(cores, gops), "host_cores": cores,
            "kind": "port", "single_thread": round(GOP / t1, 3),
            "oracle_pixel_ops_per_frame": round(ops / (gops * GOP)),
            "sample": f"the whole step: {gops} GOPs x {GOP} frames (IDR + {GOP - 1} P), one oracle encoder per "
                      f"GOP on {min(cores, gops)} threads ({cores} host cores; one thread per GOP); "
                      f"single_thread: 1 GOP x {GOP} frames on one thread",
            "aus": aus}


def bitstream_digest(aus_by_gop) -> str:
    """SHA-256 of the GOPs' access units, GOP by GOP in display order."""
    import hashlib
    h = hashlib.sha256()
    for g in aus_by_gop:
        for au in g:
            h.update(au)
    return h.hexdigest()


BATCH_SIZES = [(320, 240), (640, 360), (1280, 720), (1920, 1080)]
BATCH_STREAMS, BATCH_FRAMES, BATCH_WAVE = 16, 30, 10


def run_batched(args, rank, world, local):
    """--workload batched: measure_batched's line."""
    if rank != 0:
        return
    line = measure_batched(args, local)
    print(json.dumps(line), flush=True)


def measure_batched(args, local):
    """The batched-streams configuration: 64 concurrent streams, 16 each at 320x240, 640x360,
    1280x720 and 1920x1080, 30 frames each (one GOP: IDR + 29 P) from independent seeds, Main
    profile (CABAC), a QP drawn uniformly from 20..36 per stream, Balanced analysis. One encoder
    per size; each step's 30 pictures of every stream of all four submitted as one group
    (rg_encoder_submit_group: one persistent, graph-captured launch over the four contexts), each
    encoder's access units written on its own host threads as the launch finishes them, two steps
    in flight; each size's launch
    shape (warps per SM, segment length) picked by ragdoll_b200.autotune on its first wave before
    timing (--no-autotune: library defaults; the group launch takes the largest size's). Beside it,
    the four encoders each with their own launches over waves of 10 pictures, driven from four host
    threads. A step is the
    whole encode of the 1920 pictures: host frames in (pinned), access units out.
    Reports the aggregate frames/s and the per-frame latency percentiles (a picture's latency: its
    wave's submit to its access unit written)."""
    import torch

    from ragdoll_b200.encoder import H264Encoder
    from ragdoll_b200.engine import RG_FRAME_IDR, RG_FRAME_P, RG_PROFILE_MAIN
    from ragdoll_b200.synth import grating_clip

    torch.cuda.set_device(local)
    rng = np.random.default_rng(4)
    cores = os.cpu_count() or 1
    areas = [w * h for w, h in BATCH_SIZES]
    jobs = []
    for k, (w, h) in enumerate(BATCH_SIZES):
        cw, ch = (w + 1) // 2, (h + 1) // 2
        fb = w * h + 2 * cw * ch
        host = torch.empty((BATCH_STREAMS, BATCH_FRAMES, fb), dtype=torch.uint8).pin_memory()
        hn = host.numpy()
        for s in range(BATCH_STREAMS):
            clip = grating_clip(w, h, BATCH_FRAMES, seed=4000 + 100 * k + s, motion=8.0, rects=6)
            for f, (y, u, v) in enumerate(clip):
                hn[s, f] = np.concatenate([y.reshape(-1), u.reshape(-1), v.reshape(-1)])
        qps = [int(q) for q in rng.integers(20, 37, BATCH_STREAMS)]
        threads = max(2, round(cores * areas[k] / sum(areas)))
        enc = H264Encoder(w, h, 26, profile=RG_PROFILE_MAIN, keyint=BATCH_FRAMES, streams=BATCH_STREAMS,
                          max_frames=BATCH_WAVE, device=local, threads=threads)
        for s, q in enumerate(qps):
            enc.set_stream_qp(s, q)
        frames = [[(hn[s, f, :w * h].reshape(h, w), hn[s, f, w * h:w * h + cw * ch].reshape(ch, cw),
                    hn[s, f, w * h + cw * ch:].reshape(ch, cw)) for s in range(BATCH_STREAMS)]
                  for f in range(BATCH_FRAMES)]
        tuning = None
        if args.autotune:
            # the launch shape of this size, timed on its first wave (outside the timed region)
            from ragdoll_b200.autotune import autotune_pipeline
            kinds = [[RG_FRAME_IDR if f == 0 else RG_FRAME_P] * BATCH_STREAMS for f in range(BATCH_WAVE)]
            tuning, _ = autotune_pipeline(w, h, 26, RG_PROFILE_MAIN, frames[:BATCH_WAVE], kinds, device=local)
            enc.set_pipeline_tuning(**tuning)
        jobs.append({"size": f"{w}x{h}", "enc": enc, "frames": frames, "host": host, "qps": qps,
                     "threads": threads, "tuning": tuning})

    def encode_all(job, out):
        enc, frames, lat, nbytes = job["enc"], job["frames"], [], 0
        waves = [frames[i:i + BATCH_WAVE] for i in range(0, BATCH_FRAMES, BATCH_WAVE)]
        t0 = time.perf_counter()
        for i, wave in enumerate(waves):
            enc.submit(wave)
            if i:
                nbytes += sum(len(au) for row in enc.collect() for au in row)
                lat.append(enc.latencies().reshape(-1))
        nbytes += sum(len(au) for row in enc.collect() for au in row)
        lat.append(enc.latencies().reshape(-1))
        out[job["size"]] = (time.perf_counter() - t0, np.concatenate(lat), nbytes)

    def step():
        out = {}
        ts = [threading.Thread(target=encode_all, args=(j, out)) for j in jobs]
        t0 = time.perf_counter()
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        return time.perf_counter() - t0, out

    for _ in range(max(args.warmup, 1)):      # every stream continues with a new GOP each step
        step()
    clocks = ClockSampler(local)
    clocks.start()
    walls, lats, per = [], [], {}
    for _ in range(args.steps):
        wall, out = step()
        walls.append(wall)
        lats.append(np.concatenate([out[j["size"]][1] for j in jobs]))
        for j in jobs:
            t, _, nb = out[j["size"]]
            per.setdefault(j["size"], []).append((t, nb))
    pictures = len(BATCH_SIZES) * BATCH_STREAMS * BATCH_FRAMES
    wall = statistics.median(walls)
    lat = np.concatenate(lats)

    # the configuration as specified: all 64 streams analysed by ONE persistent launch
    # (rg_encoder_submit_group: the four sizes' contexts in one graph-captured group launch), each
    # encoder's pictures written on its own pool as the launch finishes them, the four collected
    # from four threads. One wave per step of all 30 pictures of every stream (a group launch over
    # a third of a GOP pays its ramps three times), submitted continuously with two in flight.
    for j in jobs:
        j["enc"].close()
    encs = []
    for j, (w, h) in zip(jobs, BATCH_SIZES):
        e = H264Encoder(w, h, 26, profile=RG_PROFILE_MAIN, keyint=BATCH_FRAMES, streams=BATCH_STREAMS,
                        max_frames=BATCH_FRAMES, device=local, threads=j["threads"])
        for s_, q in enumerate(j["qps"]):
            e.set_stream_qp(s_, q)
        if j["tuning"]:
            e.set_pipeline_tuning(**j["tuning"])
        encs.append(e)

    def group_run(n):
        lat_g, nbytes = [], [0]

        def collect_all():
            outs = [None] * len(encs)

            def one_enc(k):
                outs[k] = encs[k].collect()
            ts = [threading.Thread(target=one_enc, args=(k,)) for k in range(len(encs))]
            for t in ts:
                t.start()
            for t in ts:
                t.join()
            for e, o in zip(encs, outs):
                lat_g.append(e.latencies().reshape(-1))
                nbytes[0] += sum(len(au) for row in o for au in row)
        t0 = time.perf_counter()
        for k in range(n):
            H264Encoder.submit_group(encs, [j["frames"] for j in jobs])
            if k:
                collect_all()
        collect_all()
        return time.perf_counter() - t0, np.concatenate(lat_g), nbytes[0]

    group_run(max(args.warmup, 1))
    gw, g_lat, gb = group_run(args.steps)
    clk = clocks.stop()
    g_walls, g_bytes = [gw / args.steps], [gb / args.steps]
    g_wall = statistics.median(g_walls)
    one = batched_one_launch(args, local, jobs)
    line = {
        "metric": "batched streams: aggregate encode frames/s (64 streams of mixed size, one GPU)",
        "value": round(pictures / g_wall, 2), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": max(args.warmup, 1),
        "ms_per_step": round(1000 * g_wall, 3), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "path": "rg_encoder_submit_group per step (all 30 pictures of the 64 streams, two steps in flight): host "
                "frames in, ONE persistent group launch over the four sizes' contexts (a CUDA graph per shape), "
                "each picture's records out as the launch finishes it, CABAC on the host",
        "latency_ms": {"p50": round(float(np.percentile(g_lat, 50)), 2), "p99": round(float(np.percentile(g_lat, 99)), 2),
                       "max": round(float(g_lat.max()), 2),
                       "definition": "a wave's submit to the picture's access unit written"},
        "bitstream_bytes_per_step": int(statistics.median(g_bytes)),
        "per_size_encoders": {"frames_per_s": round(pictures / wall, 2), "ms_per_step": round(1000 * wall, 3),
                              "latency_ms": {"p50": round(float(np.percentile(lat, 50)), 2),
                                             "p99": round(float(np.percentile(lat, 99)), 2)},
                              "path": "the four encoders each with its own launches, driven from four host threads"},
        "dtype": "u8/int32", "data": "synthetic (seeded gratings, +-8 px global motion, 6 moving rectangles, independent seed per stream)",
        "config": {"workload": "batched streams: 16 x 320x240, 16 x 640x360, 16 x 1280x720, 16 x 1920x1080, "
                               "30 frames each (one GOP), Main CABAC, QP U[20,36] per stream, Balanced",
                   "encoders": "one per size; each step (30 pictures of all 64 streams) submitted as one group, "
                               "one launch, two steps in flight; the four collected from four host threads; "
                               "per_size_encoders: waves of 10 pictures, each encoder its own launches",
                   "host_threads": {j["size"]: j["threads"] for j in jobs},
                   "launch_shape": {j["size"]: j["tuning"] or "library defaults" for j in jobs}},
        "per_size": {k: {"frames_per_s": round(BATCH_STREAMS * BATCH_FRAMES / statistics.median(t for t, _ in v), 1),
                         "bitstream_bytes": int(statistics.median(nb for _, nb in v))} for k, v in per.items()},
        "one_launch": one,
        "clocks": clk,
        # per timed step of the headline path: one group launch plus each context's error hand-off
        "gpu_launches": args.steps * (1 + len(jobs)),
    }
    for e in encs:
        e.close()
    return line


def batched_one_launch(args, local, jobs):
    """The batched configuration's analysis with the sources resident on the device: all 64 streams'
    30 pictures in ONE persistent launch (rg_analyse_gops_group over one context per size, the
    sizes' work lists merged), against the four contexts' own launches queued together on their four
    CUDA streams. Device time with CUDA events; analysis, reconstruction and deblocking only (no
    copies, no bitstream)."""
    import torch

    from ragdoll_b200.engine import RG_FRAME_IDR, RG_FRAME_P, RG_PROFILE_MAIN, Engine
    engs, planes, kinds, sy, suv, keep = [], [], [], [], [], []
    for j, (w, h) in zip(jobs, BATCH_SIZES):
        cw, ch = (w + 1) // 2, (h + 1) // 2
        dev = j["host"].to(f"cuda:{local}")
        keep.append(dev)
        e = Engine(w, h, 26, profile=RG_PROFILE_MAIN, num_streams=BATCH_STREAMS, device=local, max_frames=BATCH_FRAMES)
        for s, q in enumerate(j["qps"]):
            e.set_stream_qp(s, q)
        if j["tuning"]:
            e.set_pipeline_tuning(**j["tuning"])
        p, k = [], []
        for f in range(BATCH_FRAMES):
            for s in range(BATCH_STREAMS):
                b = dev[s, f].data_ptr()
                p += [b, b + w * h, b + w * h + cw * ch]
                k.append(RG_FRAME_IDR if f == 0 else RG_FRAME_P)
        engs.append(e)
        planes.append(p)
        kinds.append(k)
        sy.append(w)
        suv.append(cw)
    st = torch.cuda.ExternalStream(engs[0].cuda_stream, device=f"cuda:{local}")

    def group():
        Engine.analyse_gops_group(engs, planes, sy, suv, kinds, BATCH_FRAMES)

    def separate():
        for e, p, k, a, b in zip(engs, planes, kinds, sy, suv):
            e.analyse_gops_device(p, a, b, k, BATCH_FRAMES)

    out = {}
    steps = max(1, min(args.steps, 4))
    for name, fn in (("one_launch", group), ("launch_per_size", separate)):
        for _ in range(max(args.warmup, 3)):   # the work order settles (observed reach) and the graphs are captured
            fn()
        for e in engs:
            e.sync()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        for _ in range(steps):
            fn()
        if name == "launch_per_size":   # the last of the four streams to finish ends the step
            for e in engs[1:]:
                ev = torch.cuda.Event()
                ev.record(torch.cuda.ExternalStream(e.cuda_stream, device=f"cuda:{local}"))
                st.wait_event(ev)
        b.record(st)
        b.synchronize()
        for e in engs:
            e.sync()
        ms = a.elapsed_time(b) / steps
        out[name] = {"frames_per_s": round(len(jobs) * BATCH_STREAMS * BATCH_FRAMES / (ms / 1000), 1),
                     "ms_per_step": round(ms, 3), "wall_ms_per_step": round((time.perf_counter() - t0) * 1000 / steps, 3)}
    out["steps"] = steps
    import ctypes
    from ragdoll_b200.engine import lib
    cap, lau = ctypes.c_int64(), ctypes.c_int64()
    lib().rg_group_graph_counts(engs[0].h, ctypes.byref(cap), ctypes.byref(lau))
    out["one_launch"]["cuda_graph"] = {"captures": cap.value, "graph_launches": lau.value}
    out["what"] = ("device step of all 1920 pictures (64 streams x 30) with sources resident: one "
                   "rg_analyse_gops_group launch (a CUDA graph replayed per call) vs the four contexts' "
                   "launches on four streams")
    for e in engs:
        e.close()
    return out


def run_reference(args, rank, world):
    """CPU arm: the oracle (C++ restatement of ragdoll's Balanced encoder) on the host cores, each
    step the whole workload -- 8 GOPs x 15 pictures, one oracle encoder per GOP (parallel_gop_map
    semantics: as many threads as GOPs, up to the host's cores)."""
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    gops = FRAMES // GOP
    clip = make_clip(2000, FRAMES)
    sys.path.insert(0, str(ROOT / "tests"))
    from oracle_lib import pixel_ops
    for _ in range(args.warmup):
        oracle_gops(clip, gops, 1, cores)
    pixel_ops(reset=True)
    times = [oracle_gops(clip, gops, GOP, cores)[0] for _ in range(args.steps)]
    ops = pixel_ops(reset=True)
    t = statistics.median(times)
    value = gops * GOP / t
    t1, _ = oracle_gops(clip, 1, GOP, 1)
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1000 * t, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8/int32", "data": "synthetic (seeded gratings with global motion and moving rectangles, 1080p 8-bit 4:2:0)",
        "config": bench_config(world),
        "cpu_baseline": {"value": round(value, 3), "unit": UNIT, "cores": min(cores, gops), "host_cores": cores,
                         "kind": "port", "single_thread": round(GOP / t1, 3),
                         "oracle_pixel_ops_per_frame": round(ops / (args.steps * gops * GOP)),
                         "sample": f"each step the whole workload: {gops} GOPs x {GOP} frames, one oracle encoder per "
                                   f"GOP on {min(cores, gops)} threads ({cores} host cores); single_thread: 1 GOP "
                                   f"x {GOP} frames on one thread"},
        "e2e": {"value": round(value, 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


LEARNED_METRIC = METRIC
QPS = (22, 26, 30, 34)
CNN_FLOP_PER_MB = 2 * (22 * 22 * 32 * 18 + 20 * 20 * 32 * 288 + 18 * 18 * 32 * 288)  # 24x24 crop, three 3x3 convs


def bd_rate(r1, p1, r2, p2) -> float:
    """Bjontegaard delta rate (%) of curve 2 against curve 1: mean log-rate difference over the PSNR
    range both cover, each curve interpolated piecewise-cubically (monotone) in PSNR."""
    from scipy.interpolate import PchipInterpolator
    p1, p2, l1, l2 = map(np.asarray, (p1, p2, np.log10(r1), np.log10(r2)))
    o1, o2 = np.argsort(p1), np.argsort(p2)
    lo, hi = max(p1.min(), p2.min()), min(p1.max(), p2.max())
    if hi <= lo:
        return float("nan")
    xs = np.linspace(lo, hi, 401)
    d = PchipInterpolator(p2[o2], l2[o2])(xs) - PchipInterpolator(p1[o1], l1[o1])(xs)
    return float((10 ** (np.trapezoid(d, xs) / (hi - lo)) - 1) * 100)


def run_learned(args, rank, world, local):
    """The learned form against the plain and full-search forms on the 1080p workload (8 GOPs x 15,
    High profile): device frames/s of each form at QP 26 (one persistent launch of the 120 pictures;
    the learned form's network inference included), then bits and luma PSNR of every form at QP 22,
    26, 30 and 34 (records written by the host CABAC writer, reconstructions compared with the
    source) and the Bjontegaard delta rates. `no_net` is the learned form with fixed candidates
    instead of the network's (the coarse motion vectors kept): what the network gains."""
    import torch

    from ragdoll_b200.engine import (HINT_DTYPE, RG_FORM_FULLSEARCH, RG_FORM_LEARNED, RG_FORM_PLAIN, RG_FRAME_IDR,
                                     RG_FRAME_P, RG_PROFILE_HIGH, BitstreamWriter, Engine)
    from ragdoll_b200.learned import WEIGHTS, CandidateNet, hints_for, prior_hints
    if rank != 0:
        return
    torch.cuda.set_device(local)
    gops = FRAMES // GOP
    clip = make_clip(clip_seed(0), FRAMES)
    cw, ch = (W + 1) // 2, (H + 1) // 2
    fbytes = W * H + 2 * cw * ch
    host = np.empty((FRAMES, fbytes), np.uint8)
    for i, (y, u, v) in enumerate(clip):
        host[i] = np.concatenate([y.reshape(-1), u.reshape(-1), v.reshape(-1)])
    dev = torch.from_numpy(host).to(f"cuda:{local}")
    base = dev.data_ptr()

    def planes(i):
        p = base + i * fbytes
        return [p, p + W * H, p + W * H + cw * ch]

    net = CandidateNet.trained(local)
    idx = [g * GOP + f for g in range(gops) for f in range(GOP)]
    prev = [i if i % GOP == 0 else i - 1 for i in idx]
    hints, _ = hints_for(net, [base + i * fbytes for i in idx], [base + i * fbytes for i in prev], W, H, W)
    hint_of = {i: hints[k] for k, i in enumerate(idx)}
    n_mb = ((W + 15) // 16) * ((H + 15) // 16)
    # the network's candidates replaced by fixed ones; the coarse motion vectors kept
    fixed = prior_hints(n_mb)
    prior_of = {}
    torch.cuda.synchronize()
    for i in idx:
        h = hint_of[i].cpu().numpy().view(HINT_DTYPE).copy()
        for field in ("part_mask", "mv_off", "i4_mask"):
            h[field] = fixed[field]
        prior_of[i] = torch.from_numpy(h.view(np.uint8)).to(f"cuda:{local}")
    # one partition type per macroblock: the network's best against 16x16 always
    net.set_hint_policy(1)
    hints1, _ = hints_for(net, [base + i * fbytes for i in idx], [base + i * fbytes for i in prev], W, H, W)
    net.set_hint_policy()
    hint1_of = {i: hints1[k] for k, i in enumerate(idx)}
    fixed1 = prior_hints(n_mb, part_order=(0,))
    prior1_of = {}
    torch.cuda.synchronize()
    for i in idx:
        h = hint1_of[i].cpu().numpy().view(HINT_DTYPE).copy()
        for field in ("part_mask", "mv_off", "i4_mask"):
            h[field] = fixed1[field]
        prior1_of[i] = torch.from_numpy(h.view(np.uint8)).to(f"cuda:{local}")
    forms = {"plain": RG_FORM_PLAIN, "fullsearch": RG_FORM_FULLSEARCH, "learned": RG_FORM_LEARNED,
             "no_net": RG_FORM_LEARNED, "learned_top1": RG_FORM_LEARNED, "no_net_top1": RG_FORM_LEARNED}
    hints_by_form = {"learned": hint_of, "no_net": prior_of, "learned_top1": hint1_of, "no_net_top1": prior1_of}
    torch.cuda.synchronize()

    # network inference alone: the 120 pictures' hints
    st = torch.cuda.Stream(device=local)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(2):
        net.predict_hints([base + i * fbytes for i in idx], [base + i * fbytes for i in prev], W, H, W,
                          [h.data_ptr() for h in hints], None, st.cuda_stream)
    e0.record(st)
    reps = 5
    for _ in range(reps):
        net.predict_hints([base + i * fbytes for i in idx], [base + i * fbytes for i in prev], W, H, W,
                          [h.data_ptr() for h in hints], None, st.cuda_stream)
    e1.record(st)
    e1.synchronize()
    net.check(st.cuda_stream)
    cnn_ms = e0.elapsed_time(e1) / reps

    # 1. speed at QP 26: persistent launches, sources resident
    speed = {}
    for name, form in forms.items():
        if name.startswith("no_net"):
            continue
        eng = Engine(W, H, QP, profile=RG_PROFILE_HIGH, num_streams=gops, device=local, max_frames=GOP)
        if form != RG_FORM_PLAIN:
            eng.set_analysis_form(form, 32)
        if form == RG_FORM_LEARNED:
            net.set_hint_policy(1 if name == "learned_top1" else 3)
            eng.set_hint_net(net)   # each launch first runs the network on its own sources
        stream = torch.cuda.ExternalStream(eng.cuda_stream, device=f"cuda:{local}")
        ptrs, kinds = [], []
        for f in range(GOP):
            for g in range(gops):
                ptrs += planes(g * GOP + f)
                kinds.append(RG_FRAME_IDR if f == 0 else RG_FRAME_P)
        steps = args.steps if form != RG_FORM_FULLSEARCH else max(1, min(args.steps, 3))
        for _ in range(max(args.warmup, 1)):
            eng.analyse_gops_device(ptrs, W, cw, kinds, GOP)
        eng.sync()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(steps):
            eng.analyse_gops_device(ptrs, W, cw, kinds, GOP)
        b.record(stream)
        b.synchronize()
        eng.sync()
        ms = a.elapsed_time(b) / steps
        speed[name] = {"frames_per_s": round(FRAMES / (ms / 1000), 2), "ms_per_step": round(ms, 3), "steps": steps}
        eng.close()

    net.set_hint_policy()

    # 2. rate and distortion at four QPs (per-picture calls; every access unit written)
    rd = {name: {} for name in forms}
    for qp in QPS:
        for name, form in forms.items():
            eng = Engine(W, H, qp, profile=RG_PROFILE_HIGH, num_streams=gops, device=local)
            if form != RG_FORM_PLAIN:
                eng.set_analysis_form(form, 32)
            writers = [BitstreamWriter(W, H, qp, profile=RG_PROFILE_HIGH) for _ in range(gops)]
            bits, psnr = 0, []
            for f in range(GOP):
                kind = RG_FRAME_IDR if f == 0 else RG_FRAME_P
                ptrs = []
                for g in range(gops):
                    ptrs += planes(g * GOP + f)
                if name in hints_by_form:
                    eng.set_hints_device([hints_by_form[name][g * GOP + f].data_ptr() for g in range(gops)])
                eng.analyse_device(ptrs, W, cw, [kind] * gops)
                recs = eng.records()
                for g in range(gops):
                    bits += 8 * len(writers[g].picture(recs[g], kind))
                    y = eng.recon_coded(g)[0][:H, :W].astype(np.int32)
                    mse = float(np.mean((y - clip[g * GOP + f][0].astype(np.int32)) ** 2))
                    psnr.append(10 * np.log10(255.0 ** 2 / max(mse, 1e-9)))
            rd[name][qp] = {"kbits": round(bits / 1000, 1), "psnr_y": round(float(np.mean(psnr)), 4)}
            eng.close()

    def curve(name):
        return [rd[name][q]["kbits"] for q in QPS], [rd[name][q]["psnr_y"] for q in QPS]

    bd = {}
    for a, b in (("plain", "learned"), ("fullsearch", "learned"), ("plain", "fullsearch"), ("fullsearch", "no_net"),
                 ("no_net", "learned"), ("no_net_top1", "learned_top1"), ("plain", "learned_top1")):
        ra, pa = curve(a)
        rb, pb = curve(b)
        bd[f"{b}_vs_{a}"] = round(bd_rate(ra, pa, rb, pb), 3)
    tflops = n_mb * FRAMES * CNN_FLOP_PER_MB / (cnn_ms / 1000) / 1e12
    peaks = {}
    try:
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except Exception:
        pass
    peak = peaks.get("bf16_tflops", 1590.0)
    line = {
        "metric": LEARNED_METRIC, "value": speed["learned"]["frames_per_s"], "unit": UNIT, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": speed["learned"]["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "bf16 network / u8,int32 analysis",
        "data": "synthetic (seeded gratings with global motion and moving rectangles, 1080p 8-bit 4:2:0)",
        "config": {**bench_config(1), "workload": "1080p High, 120 frames = 8 GOPs x 15, QP 26 for speed; QP 22/26/30/34 "
                                                 "for rate and PSNR; +-32 integer search of the search forms",
                   "network_weights": WEIGHTS.name},
        "speed": speed,
        "learned_over_plain": round(speed["learned"]["frames_per_s"] / speed["plain"]["frames_per_s"], 4),
        "learned_over_fullsearch": round(speed["learned"]["frames_per_s"] / speed["fullsearch"]["frames_per_s"], 4),
        "bd_rate_pct": bd, "rd": rd,
        "network": {"ms_per_120_pictures": round(cnn_ms, 3), "tflops": round(tflops, 1),
                    "roofline": {"bound": "tensor", "achieved": round(tflops, 1), "peak": peak, "unit": "TFLOP/s",
                                 "frac": round(tflops / peak, 4),
                                 "flop_per_mb": CNN_FLOP_PER_MB, "kernel": "cnn_infer_kernel"}},
    }
    print(json.dumps(line), flush=True)


def run_4k(args, rank, world, local):
    """The 4K configuration: 8 streams of 3840x2160 (+-48 px global motion, 24 rectangles), High
    profile, QP 28, the learned form with a +-64 integer search -- its network run by the engine on
    each call's sources, then one persistent launch of all streams' pictures -- and SSIM / MS-SSIM of
    every reconstructed picture against its source in batched launches. One GOP (IDR + 14 P) per
    stream per step (the configuration's 60 frames are four such steps)."""
    import torch

    from ragdoll_b200.engine import (RG_FORM_LEARNED, RG_FRAME_IDR, RG_FRAME_P, RG_PROFILE_HIGH, Engine,
                                     ssim_batch_device)
    from ragdoll_b200.learned import CandidateNet
    from ragdoll_b200.synth import grating_clip
    if rank != 0:
        return
    torch.cuda.set_device(local)
    w4, h4, S, F, qp = 3840, 2160, 8, GOP, 28
    cw, ch = w4 // 2, h4 // 2
    fbytes = w4 * h4 + 2 * cw * ch
    dev = torch.empty((S, F, fbytes), dtype=torch.uint8, device=f"cuda:{local}")
    for s_ in range(S):
        for f, (y, u, v) in enumerate(grating_clip(w4, h4, F, seed=5000 + s_, motion=48.0, rects=24)):
            dev[s_, f] = torch.from_numpy(np.concatenate([y.reshape(-1), u.reshape(-1), v.reshape(-1)]))
    base = dev.data_ptr()

    def pic(s_, f):
        p = base + (s_ * F + f) * fbytes
        return [p, p + w4 * h4, p + w4 * h4 + cw * ch]

    net = CandidateNet.trained(local)
    eng = Engine(w4, h4, qp, profile=RG_PROFILE_HIGH, num_streams=S, device=local, max_frames=F)
    eng.set_analysis_form(RG_FORM_LEARNED, 64)
    eng.set_hint_net(net)
    ptrs, kinds = [], []
    for f in range(F):
        for s_ in range(S):
            ptrs += pic(s_, f)
            kinds.append(RG_FRAME_IDR if f == 0 else RG_FRAME_P)
    stream = torch.cuda.ExternalStream(eng.cuda_stream, device=f"cuda:{local}")
    for _ in range(max(args.warmup, 1)):
        eng.analyse_gops_device(ptrs, w4, cw, kinds, F)
    eng.sync()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    steps = max(1, min(args.steps, 4))
    a.record(stream)
    for _ in range(steps):
        eng.analyse_gops_device(ptrs, w4, cw, kinds, F)
    b.record(stream)
    b.synchronize()
    eng.sync()
    ms = a.elapsed_time(b) / steps
    # SSIM / MS-SSIM: the final reconstruction of every stream against its source, and the batched
    # throughput over all S x F pictures of a step (each against the next picture of its stream)
    recon = torch.stack([torch.from_numpy(np.ascontiguousarray(eng.recon(s_)[0])) for s_ in range(S)]).to(f"cuda:{local}")
    fin, fin_ms = ssim_batch_device([recon[s_].data_ptr() for s_ in range(S)], [pic(s_, F - 1)[0] for s_ in range(S)],
                                    w4, h4, w4, w4, device=local)
    pa = [pic(s_, f)[0] for s_ in range(S) for f in range(F)]
    pb = [pic(s_, (f + 1) % F)[0] for s_ in range(S) for f in range(F)]
    qs = torch.cuda.Stream(device=local)
    ssim_batch_device(pa, pb, w4, h4, w4, w4, device=local, stream=qs.cuda_stream)
    q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    q0.record(qs)
    ssim_batch_device(pa, pb, w4, h4, w4, w4, device=local, stream=qs.cuda_stream)
    q1.record(qs)
    q1.synchronize()
    line = {"metric": "4K learned + batched: encode frames/s (8 streams of 3840x2160, one GPU)",
            "value": round(S * F / (ms / 1000), 2), "unit": UNIT, "n_gpus": 1, "steps": steps, "warmup": max(args.warmup, 1),
            "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16 network / u8,int32 analysis",
            "data": "synthetic (seeded gratings, +-48 px global motion, 24 moving rectangles, 3840x2160 8-bit 4:2:0)",
            "config": {"workload": "8 streams x 3840x2160, one GOP (IDR + 14 P) each per step, High, QP 28, learned form, "
                                   "+-64 integer search, network and analysis launches on one stream",
                       "l2": "inputs larger than L2"},
            "ssim_final": [round(float(x), 6) for x in fin], "ms_ssim_final": [round(float(x), 6) for x in fin_ms],
            "ssim_batch": {"pairs": len(pa), "ms": round(q0.elapsed_time(q1), 3)}}
    print(json.dumps(line), flush=True)
    eng.close()


# ------------------------------------------------------------------------------------------------
def rd_point(eng_factory, clip, planes, gops, qp, hints_of=None):
    """Bits and mean luma PSNR of the 8 GOPs x 15 at one QP: per-picture calls of one engine, every
    access unit written by the host CABAC writer, reconstructions compared with the source."""
    from ragdoll_b200.engine import RG_FRAME_IDR, RG_FRAME_P, RG_PROFILE_HIGH, BitstreamWriter
    eng = eng_factory(qp)
    writers = [BitstreamWriter(W, H, qp, profile=RG_PROFILE_HIGH) for _ in range(gops)]
    cw = (W + 1) // 2
    bits, psnr = 0, []
    for f in range(GOP):
        kind = RG_FRAME_IDR if f == 0 else RG_FRAME_P
        ptrs = []
        for g in range(gops):
            ptrs += planes(g * GOP + f)
        if hints_of is not None:
            eng.set_hints_device([hints_of[g * GOP + f].data_ptr() for g in range(gops)])
        eng.analyse_device(ptrs, W, cw, [kind] * gops)
        recs = eng.records()
        for g in range(gops):
            bits += 8 * len(writers[g].picture(recs[g], kind))
            y = eng.recon_coded(g)[0][:H, :W].astype(np.int32)
            mse = float(np.mean((y - clip[g * GOP + f][0].astype(np.int32)) ** 2))
            psnr.append(10 * np.log10(255.0 ** 2 / max(mse, 1e-9)))
    eng.close()
    return {"kbits": round(bits / 1000, 1), "psnr_y": round(float(np.mean(psnr)), 4)}


def measure_learned(args, local, dist, base, fbytes, planes, gops, frames_host, clip, rank, barrier):
    """The learned form on the step's workload: device frames/s of the whole learned step (network
    and coarse-motion launches, then the persistent analysis launch, one stream), the network alone
    and the analysis alone (hints computed beforehand); end to end through the public encoder
    (rg_encoder_set_form); on rank 0 the rate and PSNR of the plain and learned forms at QP 22 / 26
    / 30 / 34 and the Bjontegaard delta rate of the learned form against the plain one."""
    import torch

    from ragdoll_b200.encoder import H264Encoder
    from ragdoll_b200.engine import (RG_FORM_FULLSEARCH, RG_FORM_LEARNED, RG_FORM_PLAIN, RG_FRAME_IDR, RG_FRAME_P,
                                     RG_PROFILE_HIGH, Engine)
    from ragdoll_b200.learned import WEIGHTS, CandidateNet, hints_for
    cw = (W + 1) // 2
    net = CandidateNet.trained(local)
    ptrs, kinds = [], []
    for f in range(GOP):
        for g in range(gops):
            ptrs += planes(g * GOP + f)
            kinds.append(RG_FRAME_IDR if f == 0 else RG_FRAME_P)
    idx = [g * GOP + f for f in range(GOP) for g in range(gops)]          # the call's [f][s] order
    prev = [i if i % GOP == 0 else i - 1 for i in idx]
    cur_p, prev_p = [base + i * fbytes for i in idx], [base + i * fbytes for i in prev]

    def learned_engine(qp, with_net=True):
        e = Engine(W, H, qp, profile=RG_PROFILE_HIGH, num_streams=gops, device=local, max_frames=GOP)
        e.set_analysis_form(RG_FORM_LEARNED, 32)
        if with_net:
            e.set_hint_net(net)
        return e

    def timed(stream, fn, steps):
        for _ in range(max(args.warmup, 1)):
            fn()
        torch.cuda.synchronize()
        barrier()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(steps):
            fn()
        b.record(stream)
        b.synchronize()
        torch.cuda.synchronize()
        barrier()
        return max_over_ranks(a.elapsed_time(b) / steps, dist, f"cuda:{local}")

    # 1. the learned step: network + coarse motion + analysis, one stream
    eng = learned_engine(QP)
    st = torch.cuda.ExternalStream(eng.cuda_stream, device=f"cuda:{local}")
    steps = max(1, min(args.steps, 8))
    clocks = ClockSampler(local)
    clocks.start()
    step_ms = timed(st, lambda: eng.analyse_gops_device(ptrs, W, cw, kinds, GOP), steps)
    clk = clocks.stop()
    eng.close()
    # 2. the network (and coarse pass) alone, and 3. the analysis alone with those hints
    hints, _ = hints_for(net, cur_p, prev_p, W, H, W, device=local)
    hs = torch.cuda.Stream(device=local)

    def predict():
        net.predict_hints(cur_p, prev_p, W, H, W, [h.data_ptr() for h in hints], None, hs.cuda_stream)
    net.set_coarse_range(0)
    cnn_ms = timed(hs, predict, steps)
    net.set_coarse_range(32)
    net_ms = timed(hs, predict, steps)
    net.check(hs.cuda_stream)
    eng = learned_engine(QP, with_net=False)
    st = torch.cuda.ExternalStream(eng.cuda_stream, device=f"cuda:{local}")
    hp = [h.data_ptr() for h in hints]

    def analysis():
        eng.set_hints_device(hp)
        eng.analyse_gops_device(ptrs, W, cw, kinds, GOP)
    ana_ms = timed(st, analysis, steps)
    eng.close()
    # the same step with one partition type per macroblock (hint policy top-1), and the full-search
    # form (the learned form's fallback and judge)
    net.set_hint_policy(1)
    eng = learned_engine(QP)
    st = torch.cuda.ExternalStream(eng.cuda_stream, device=f"cuda:{local}")
    top1_ms = timed(st, lambda: eng.analyse_gops_device(ptrs, W, cw, kinds, GOP), steps)
    eng.close()
    hints1, _ = hints_for(net, cur_p, prev_p, W, H, W, device=local)
    net.set_hint_policy()
    eng = Engine(W, H, QP, profile=RG_PROFILE_HIGH, num_streams=gops, device=local, max_frames=GOP)
    eng.set_analysis_form(RG_FORM_FULLSEARCH, 32)
    st = torch.cuda.ExternalStream(eng.cuda_stream, device=f"cuda:{local}")
    fs_ms = timed(st, lambda: eng.analyse_gops_device(ptrs, W, cw, kinds, GOP), max(1, min(steps, 3)))
    eng.close()
    # 4. end to end: host frames in, access units out, through the public encoder
    local_world = int(os.environ.get("LOCAL_WORLD_SIZE", "1"))
    enc = H264Encoder(W, H, QP, profile=RG_PROFILE_HIGH, keyint=GOP, streams=gops, max_frames=GOP, device=local,
                      threads=max(2, (os.cpu_count() or 1) // max(local_world, 1)))
    enc.set_form(RG_FORM_LEARNED, 32, net)
    for _ in range(2):
        enc.new_gops()
        enc.submit(frames_host)
    enc.collect()
    enc.collect()
    barrier()
    t0 = time.perf_counter()
    out_bytes = 0
    for k in range(steps):
        enc.new_gops()
        enc.submit(frames_host)
        if k:
            out_bytes += sum(len(au) for row in enc.collect() for au in row)
    out_bytes += sum(len(au) for row in enc.collect() for au in row)
    e2e_ms = max_over_ranks((time.perf_counter() - t0) * 1000 / steps, dist, f"cuda:{local}")
    rec_bytes = enc.record_bytes()
    enc.close()
    out = {"record_bytes_per_step": rec_bytes, "step_ms": step_ms, "cnn_ms": cnn_ms, "network_ms": net_ms, "analysis_ms": ana_ms, "e2e_ms": e2e_ms, "steps": steps,
           "top1_ms": top1_ms, "fullsearch_ms": fs_ms,
           "clocks": clk, "bitstream_bytes_per_step": round(out_bytes / steps), "weights": WEIGHTS.name}
    # 5. rate and distortion (rank 0, outside the timed regions)
    if rank == 0:
        def plain_engine(qp):
            e = Engine(W, H, qp, profile=RG_PROFILE_HIGH, num_streams=gops, device=local)
            e.set_analysis_form(RG_FORM_PLAIN, 32)
            return e
        def fs_engine(qp):
            e = Engine(W, H, qp, profile=RG_PROFILE_HIGH, num_streams=gops, device=local)
            e.set_analysis_form(RG_FORM_FULLSEARCH, 32)
            return e
        by_pic = {i: hints[k] for k, i in enumerate(idx)}
        by_pic1 = {i: hints1[k] for k, i in enumerate(idx)}
        rd = {"plain": {}, "learned": {}, "learned_top1": {}, "fullsearch": {}}
        for qp in QPS:
            rd["plain"][qp] = rd_point(plain_engine, clip, planes, gops, qp)
            # the hints do not depend on the QP: the same ones serve every QP
            rd["learned"][qp] = rd_point(lambda q: learned_engine(q, with_net=False), clip, planes, gops, qp, by_pic)
            rd["learned_top1"][qp] = rd_point(lambda q: learned_engine(q, with_net=False), clip, planes, gops, qp,
                                              by_pic1)
            rd["fullsearch"][qp] = rd_point(fs_engine, clip, planes, gops, qp)

        def curve(name):
            return [rd[name][q]["kbits"] for q in QPS], [rd[name][q]["psnr_y"] for q in QPS]
        out["rd"] = rd
        out["bd_rate_vs_plain_pct"] = round(bd_rate(*curve("plain"), *curve("learned")), 3)
        out["bd_rates_pct"] = {f"{b}_vs_{a}": round(bd_rate(*curve(a), *curve(b)), 3)
                               for a, b in (("plain", "learned_top1"), ("fullsearch", "learned"),
                                            ("fullsearch", "learned_top1"), ("plain", "fullsearch"))}
    net.close()
    return out


# ------------------------------------------------------------------------------------------------
def run_engine(args, rank, world, local):
    import torch

    from ragdoll_b200.engine import RG_FRAME_IDR, RG_FRAME_P, RG_PROFILE_HIGH, Engine

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    gops = FRAMES // GOP
    clip = make_clip(clip_seed(rank), FRAMES)
    # source clip resident in HBM: one contiguous buffer per frame (Y | U | V)
    cw, ch = (W + 1) // 2, (H + 1) // 2
    fbytes = W * H + 2 * cw * ch
    host = np.empty((FRAMES, fbytes), np.uint8)
    for i, (y, u, v) in enumerate(clip):
        host[i, :W * H] = y.reshape(-1)
        host[i, W * H:W * H + cw * ch] = u.reshape(-1)
        host[i, W * H + cw * ch:] = v.reshape(-1)
    dev = torch.from_numpy(host).to(f"cuda:{local}")
    base = dev.data_ptr()

    def planes(i):
        p = base + i * fbytes
        return [p, p + W * H, p + W * H + cw * ch]

    eng = Engine(W, H, QP, profile=RG_PROFILE_HIGH, num_streams=gops, device=local, max_frames=GOP)
    eng.set_pipeline_tuning(lag=args.lag, seg=args.seg, grid=args.grid, deblock_sms=args.deblock_sms,
                            intra_sms=args.intra_sms)
    stream = torch.cuda.ExternalStream(eng.cuda_stream, device=f"cuda:{local}")
    torch.cuda.synchronize()
    gop_ptrs, gop_kinds = [], []
    for i in range(GOP):
        for g in range(gops):
            gop_ptrs += planes(g * GOP + i)
            gop_kinds.append(RG_FRAME_IDR if i == 0 else RG_FRAME_P)
    # end-to-end inputs and outputs in pinned host memory, allocated once (the public host-buffer
    # API copies from / to them every step)
    pinned = torch.from_numpy(host).pin_memory()
    ph = pinned.numpy()

    def host_planes(i):
        return (ph[i, :W * H].reshape(H, W), ph[i, W * H:W * H + cw * ch].reshape(ch, cw),
                ph[i, W * H + cw * ch:].reshape(ch, cw))

    frames_host = [[host_planes(g * GOP + i) for g in range(gops)] for i in range(GOP)]
    kinds_host = [[RG_FRAME_IDR if i == 0 else RG_FRAME_P] * gops for i in range(GOP)]
    from ragdoll_b200.engine import RECORD_DTYPE
    rec_pinned = [torch.empty(GOP * gops * eng.n_mb * RECORD_DTYPE.itemsize, dtype=torch.uint8).pin_memory()
                  for _ in range(2)]
    rec_host = [r.numpy().view(RECORD_DTYPE).reshape(GOP, gops, eng.n_mb) for r in rec_pinned]
    e2e_calls = [0]

    if args.mode == "pipelined":
        def device_step():
            eng.analyse_gops_device(gop_ptrs, W, cw, gop_kinds, GOP)

        def host_step():
            # asynchronous host-buffer calls: copy-in of this step and copy-out of the last one
            # overlap the launches; records land in alternating pinned buffers
            eng.analyse_gops_async(frames_host, kinds_host, rec_host[e2e_calls[0] % 2])
            e2e_calls[0] += 1
    else:
        def device_step():
            for i in range(GOP):
                ptrs = []
                for g in range(gops):
                    ptrs += planes(g * GOP + i)
                eng.analyse_device(ptrs, W, cw, [RG_FRAME_IDR if i == 0 else RG_FRAME_P] * gops)

        def host_step():
            for i in range(GOP):
                eng.analyse(frames_host[i], [RG_FRAME_IDR if i == 0 else RG_FRAME_P] * gops)

    def barrier():
        if dist is not None:
            dist.barrier()


    # warm-up
    for _ in range(args.warmup):
        device_step()
    eng.sync()
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        device_step()
    ev1.record(stream)
    ev1.synchronize()
    eng.sync()
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    dev_ms = max_over_ranks(ev0.elapsed_time(ev1) / args.steps, dist, f"cuda:{local}")

    # the analysis alone through the host-buffer C ABI (records copied back every batch)
    host_step()
    eng.sync()
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        host_step()
    eng.sync()
    torch.cuda.synchronize()
    ana_ms = max_over_ranks((time.perf_counter() - t0) * 1000 / args.steps, dist, f"cuda:{local}")

    # end to end: the whole encode through the public encoder, host frames in, access units out
    from ragdoll_b200.encoder import H264Encoder
    # the host cores shared among the ranks of this node (one writer pool per rank)
    local_world = int(os.environ.get("LOCAL_WORLD_SIZE", str(world)))
    enc_threads = max(2, (os.cpu_count() or 1) // max(local_world, 1))
    enc = H264Encoder(W, H, QP, profile=RG_PROFILE_HIGH, keyint=GOP, streams=gops, max_frames=GOP,
                      device=local, threads=enc_threads)
    # every wave is the workload's 8 GOP chunks, each coded as by a fresh encoder per chunk (the
    # pipeline's own shape: IDR with idr_pic_id 0, then 14 P pictures)
    for _ in range(2):                         # both wave slots once
        enc.new_gops()
        enc.submit(frames_host)
    enc.collect()
    enc.collect()
    barrier()
    t0 = time.perf_counter()
    out_bytes = 0
    for k in range(args.steps):
        enc.new_gops()
        enc.submit(frames_host)
        if k:
            out_bytes += sum(len(au) for row in enc.collect() for au in row)
    last_aus = enc.collect()
    out_bytes += sum(len(au) for row in last_aus for au in row)
    e2e_ms = max_over_ranks((time.perf_counter() - t0) * 1000 / args.steps, dist, f"cuda:{local}")
    enc_threads = enc.threads
    rec_bytes = enc.record_bytes()
    # the same with compact records written by the launch into mapped host memory (opt-in), for
    # comparison
    enc.set_record_compaction(96)
    for _ in range(2):
        enc.new_gops()
        enc.submit(frames_host)
    enc.collect()
    enc.collect()
    barrier()
    t0 = time.perf_counter()
    for k in range(args.steps):
        enc.new_gops()
        enc.submit(frames_host)
        if k:
            enc.collect()
    enc.collect()
    e2e_compact_ms = max_over_ranks((time.perf_counter() - t0) * 1000 / args.steps, dist, f"cuda:{local}")
    compact_bytes = enc.record_bytes()
    enc.close()

    # the learned form on the same workload (the headline of the line)
    learned = measure_learned(args, local, dist, base, fbytes, planes, gops, frames_host, clip, rank, barrier)

    # SSIM and MS-SSIM of 120 luma plane pairs in one batched call (shared launches over every
    # pair and pyramid level); the pairs are pictures of the step's clip (their values do not change
    # the work). Algorithmic bytes per 1080p pair: both planes read at the five levels, and four
    # decimations reading one level and writing the next: ~5.98 W H.
    from ragdoll_b200.engine import ssim_batch_device
    qstream = torch.cuda.Stream(device=local)
    pa = [base + i * fbytes for i in range(FRAMES)]
    pb = [base + ((i + 1) % FRAMES) * fbytes for i in range(FRAMES)]
    ssim_batch_device(pa, pb, W, H, W, W, device=local, stream=qstream.cuda_stream)
    q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    q_reps = 3
    tq = time.perf_counter()
    q0.record(qstream)
    for _ in range(q_reps):
        ssim_batch_device(pa, pb, W, H, W, W, device=local, stream=qstream.cuda_stream)
    q1.record(qstream)
    q1.synchronize()
    q_wall_ms = (time.perf_counter() - tq) * 1000 / q_reps
    q_ms = q0.elapsed_time(q1) / q_reps
    lv = sum(4.0 ** -k for k in range(5))
    q_bytes = FRAMES * W * H * (2 * lv + 2 * (lv - 4.0 ** -4) + 2 * (lv - 1))

    # per-launch duration of the dominant kernel
    steps_per_frame = (eng.mb_w - 1) + 2 * (eng.mb_h - 1) + 1 + 3
    if args.mode == "pipelined":
        kernel_name, launches_per_step = "pipeline_kernel", 1
        launch_ms = dev_ms
        bytes_per_launch = BYTES_PER_FRAME * FRAMES
    else:
        kernel_name, launches_per_step = "wavefront_step_kernel", GOP * (steps_per_frame + 1)
        launch_ms = dev_ms / launches_per_step
        bytes_per_launch = BYTES_PER_FRAME * gops / (steps_per_frame + 1)

    frames_total = FRAMES * world
    value = frames_total / (dev_ms / 1000)
    e2e = frames_total / (e2e_ms / 1000)
    peaks = {}
    try:
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except Exception:
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    achieved = bytes_per_launch / (launch_ms / 1000) / 1e9
    # kernels of this library per timed step: the pipelined launch and the one-thread kernel that
    # hands its error word to the host; per-diagonal mode: the diagonal steps and the padding
    launches = args.steps * (2 if args.mode == "pipelined" else launches_per_step)

    cpu, parity = None, None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # outside the timed regions: the oracle encodes the same step, which is both the CPU
        # baseline and the parity check of the step's bitstream (every access unit of every GOP)
        cpu = oracle_sample(clip, gops, os.cpu_count() or 1)
        want = bitstream_digest(cpu.pop("aus"))
        got = bitstream_digest([[last_aus[f][g] for f in range(GOP)] for g in range(gops)])
        parity = {"bitstream_equals_oracle": got == want, "sha256": got,
                  "checked": f"every access unit of the last timed e2e step ({gops} GOPs x {GOP} pictures)"}

    if rank == 0:
        l_value = frames_total / (learned["step_ms"] / 1000)
        l_e2e = frames_total / (learned["e2e_ms"] / 1000)
        l_ana = bytes_per_launch / (learned["analysis_ms"] / 1000) / 1e9 if args.mode == "pipelined" else None
        n_mb = eng.n_mb
        cnn_tflops = n_mb * FRAMES * CNN_FLOP_PER_MB / (learned["cnn_ms"] / 1000) / 1e12
        tpeak = peaks.get("bf16_tflops", 1590.0)
        plain = {
            "value": round(value, 2), "ms_per_step": round(dev_ms, 3), "steps": args.steps,
            "e2e": {"value": round(e2e, 2), "unit": UNIT, "h2d_bytes_per_step": FRAMES * fbytes,
                    "d2h_bytes_per_step": rec_bytes, "bitstream_bytes_per_step": round(out_bytes / args.steps),
                    "host_threads": enc_threads,
                    "path": "rg_encoder_submit/collect: copy in, persistent launch, each picture's records "
                            "copied out as the launch finishes it, CABAC on the host"},
            "e2e_compact_records": {"value": round(frames_total / (e2e_compact_ms / 1000), 2), "unit": UNIT,
                                    "d2h_bytes_per_step": compact_bytes,
                                    "path": "the same with rg_set_record_compaction(96): compact records written "
                                            "by the launch into mapped host memory"},
            "e2e_analysis": {"value": round(frames_total / (ana_ms / 1000), 2), "unit": UNIT,
                             "path": "rg_analyse_gops_async: copy in, persistent launch, records out"},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 5),
                         "traffic": round(TRAFFIC_PER_FRAME * FRAMES) if args.mode == "pipelined" else None,
                         "kernel": kernel_name, "launch_ms": round(launch_ms, 5),
                         "bytes_per_launch": round(bytes_per_launch)},
            "parity": parity, "clocks": clk, "gpu_launches": launches,
        }
        line = {
            "metric": METRIC, "value": round(l_value, 2), "unit": UNIT, "n_gpus": world, "steps": learned["steps"],
            "warmup": max(args.warmup, 1), "ms_per_step": round(learned["step_ms"], 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "bf16 network / u8,int32 analysis",
            "data": "synthetic (seeded gratings with global motion and moving rectangles, 1080p 8-bit 4:2:0)",
            "config": bench_config(world, args.mode),
            "form": {"headline": "learned: network hints, coarse motion, +-2 windows, full search +-32 fallback",
                     "network_weights": learned["weights"], "compared_with": "plain (ragdoll's Balanced decisions)"},
            "e2e": {"value": round(l_e2e, 2), "unit": UNIT, "h2d_bytes_per_step": FRAMES * fbytes,
                    "d2h_bytes_per_step": learned["record_bytes_per_step"],
                    "bitstream_bytes_per_step": learned["bitstream_bytes_per_step"], "host_threads": enc_threads,
                    "path": "rg_encoder_set_form(learned) + submit/collect: copy in, network and coarse-motion "
                            "launches, persistent analysis launch, records out, CABAC on the host"},
            "learned_over_plain": {"device": round(l_value / value, 4), "e2e": round(l_e2e / e2e, 4)},
            "bd_rate_vs_plain_pct": learned.get("bd_rate_vs_plain_pct"),
            "forms_frames_per_s": {"plain": round(value, 2), "learned": round(l_value, 2),
                                   "learned_top1": round(frames_total / (learned["top1_ms"] / 1000), 2),
                                   "fullsearch": round(frames_total / (learned["fullsearch_ms"] / 1000), 2)},
            "bd_rates_pct": learned.get("bd_rates_pct"),
            "rd": learned.get("rd"),
            "target": "learned >= 3x plain frames/s at <= +2 % bits for equal PSNR (QP 22/26/30/34)",
            "learned_breakdown_ms": {"step": round(learned["step_ms"], 3), "network": round(learned["cnn_ms"], 3),
                                     "network_and_coarse_motion": round(learned["network_ms"], 3),
                                     "analysis_with_hints": round(learned["analysis_ms"], 3)},
            "roofline": {"bound": "hbm", "achieved": round(l_ana, 2) if l_ana else None, "peak": peak, "unit": "GB/s",
                         "frac": round(l_ana / peak, 5) if l_ana else None, "traffic": None,
                         "kernel": "pipeline_kernel (learned form)", "launch_ms": round(learned["analysis_ms"], 4),
                         "bytes_per_launch": round(bytes_per_launch)},
            "roofline_network": {"bound": "tensor", "achieved": round(cnn_tflops, 1), "peak": tpeak, "unit": "TFLOP/s",
                                 "frac": round(cnn_tflops / tpeak, 4), "kernel": "cnn_infer_kernel",
                                 "flop_per_launch": n_mb * FRAMES * CNN_FLOP_PER_MB,
                                 "launch_ms": round(learned["cnn_ms"], 4)},
            "plain": plain,
            "quality": {"what": "SSIM + 5-scale MS-SSIM of 120 1080p luma plane pairs, one rg_ssim_batch_device call",
                        "ms_device": round(q_ms, 3), "ms_call": round(q_wall_ms, 3),
                        "pairs_per_s": round(FRAMES / (q_ms / 1000), 1),
                        "roofline": {"bound": "hbm", "achieved": round(q_bytes / (q_ms / 1000) / 1e9, 1), "peak": peak,
                                     "unit": "GB/s", "frac": round(q_bytes / (q_ms / 1000) / 1e9 / peak, 4),
                                     "bytes_per_call": round(q_bytes)}},
            "cpu_baseline": cpu,
            "parity": parity,
            "clocks": learned["clocks"],
            # kernels of this library per timed learned step: the network, the coarse motion pass,
            # the persistent analysis launch and the one-thread error hand-off
            "gpu_launches": 4 * learned["steps"],
        }
        if world == 1 and args.batched:
            # the batched-streams configuration (64 streams of four sizes), two timed steps, beside
            # the 1080p numbers: its own untimed region, after the 1080p work is done
            b_args = argparse.Namespace(**vars(args))
            b_args.steps, b_args.warmup = 2, 1
            bl = measure_batched(b_args, local)
            line["batched"] = {k: bl[k] for k in ("metric", "value", "unit", "ms_per_step", "steps", "path",
                                                  "latency_ms", "per_size_encoders", "one_launch", "per_size",
                                                  "config", "clocks", "gpu_launches")}
        print(json.dumps(line), flush=True)
    eng.close()
    if dist is not None:
        dist.destroy_process_group()


def run_profile_case_cnn(args, local):
    """Small case for ncu of the network kernel: the hints of 8 pictures of the 1080p clip (65 280
    macroblocks a launch of cnn_infer_kernel): twice without the coarse motion pass, twice with it."""
    import torch

    from ragdoll_b200.learned import CandidateNet, hints_for
    torch.cuda.set_device(local)
    clip = make_clip(2000, 9)
    luma = torch.from_numpy(np.stack([fr[0] for fr in clip])).to(f"cuda:{local}")
    net = CandidateNet.trained(local)
    ptrs = [luma[i].data_ptr() for i in range(1, 9)]
    prev = [luma[i - 1].data_ptr() for i in range(1, 9)]
    times = {}
    for coarse in (0, 32):   # the network alone, then with the coarse motion pass after it
        net.set_coarse_range(coarse)
        times[coarse] = []
        for _ in range(2):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            hints_for(net, ptrs, prev, W, H, W)
            e1.record()
            e1.synchronize()
            times[coarse].append(round(e0.elapsed_time(e1), 3))
    net.check()
    print(json.dumps({"profile_case": "network hints of 8 1080p pictures", "ms_network": times[0],
                      "ms_network_and_coarse_motion": times[32]}), flush=True)


def run_profile_case_learned(args, local):
    """Launch list of the learned step (ncu, one metric): two learned steps of the default workload
    (8 GOPs x 15 of 1080p) -- the network, the coarse motion pass and the persistent analysis
    launch each time."""
    import torch

    from ragdoll_b200.engine import RG_FORM_LEARNED, RG_FRAME_IDR, RG_FRAME_P, RG_PROFILE_HIGH, Engine
    from ragdoll_b200.learned import CandidateNet
    torch.cuda.set_device(local)
    gops = FRAMES // GOP
    clip = make_clip(clip_seed(0), FRAMES)
    cw, ch = (W + 1) // 2, (H + 1) // 2
    fbytes = W * H + 2 * cw * ch
    host = np.stack([np.concatenate([p.reshape(-1) for p in fr]) for fr in clip])
    dev = torch.from_numpy(host).to(f"cuda:{local}")
    base = dev.data_ptr()
    net = CandidateNet.trained(local)
    eng = Engine(W, H, QP, profile=RG_PROFILE_HIGH, num_streams=gops, device=local, max_frames=GOP)
    eng.set_analysis_form(RG_FORM_LEARNED, 32)
    eng.set_hint_net(net)
    ptrs, kinds = [], []
    for f in range(GOP):
        for g in range(gops):
            p = base + (g * GOP + f) * fbytes
            ptrs += [p, p + W * H, p + W * H + cw * ch]
            kinds.append(RG_FRAME_IDR if f == 0 else RG_FRAME_P)
    times = []
    stream = torch.cuda.ExternalStream(eng.cuda_stream, device=f"cuda:{local}")
    for _ in range(2):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        eng.analyse_gops_device(ptrs, W, cw, kinds, GOP)
        e1.record(stream)
        e1.synchronize()
        times.append(round(e0.elapsed_time(e1), 3))
    eng.sync()
    eng.close()
    print(json.dumps({"profile_case": "learned step, 1080p 8 GOPs x 15", "ms": times}), flush=True)


def run_profile_case(args, local):
    """Small case for ncu: one IDR batch and one P batch of the 8-GOP 1080p workload (16 frames),
    with the device time of each batch -- per anti-diagonal launches, or (pipelined) the first
    --profile-frames pictures (IDR, P, ...) of the 8 GOPs in one persistent launch."""
    import torch

    from ragdoll_b200.engine import RG_FRAME_IDR, RG_FRAME_P, RG_PROFILE_HIGH, Engine

    torch.cuda.set_device(local)
    gops = FRAMES // GOP
    clip = make_clip(2000, GOP + 1)
    # GOP g reads frames (g, g+1) of one short clip: distinct content per GOP, 16 frames in total
    cw, ch = (W + 1) // 2, (H + 1) // 2
    fbytes = W * H + 2 * cw * ch
    host = np.empty((len(clip), fbytes), np.uint8)
    for i, (y, u, v) in enumerate(clip):
        host[i] = np.concatenate([y.reshape(-1), u.reshape(-1), v.reshape(-1)])
    dev = torch.from_numpy(host).to(f"cuda:{local}")
    base = dev.data_ptr()
    if args.profile_case == "pipelined":
        nf = args.profile_frames
        eng = Engine(W, H, QP, profile=RG_PROFILE_HIGH, num_streams=gops, device=local, max_frames=nf)
        eng.set_pipeline_tuning(lag=args.lag, seg=args.seg, grid=args.grid, deblock_sms=args.deblock_sms,
                                intra_sms=args.intra_sms)
        if args.profile_form == "learned":   # the learned form, its network run by each launch
            from ragdoll_b200.engine import RG_FORM_LEARNED
            from ragdoll_b200.learned import CandidateNet
            net = CandidateNet.trained(local)
            eng.set_analysis_form(RG_FORM_LEARNED, 32)
            eng.set_hint_net(net)
        stream = torch.cuda.ExternalStream(eng.cuda_stream, device=f"cuda:{local}")
        ptrs, kinds = [], []
        for f in range(nf):
            for g in range(gops):
                p = base + (g + f) * fbytes
                ptrs += [p, p + W * H, p + W * H + cw * ch]
                kinds.append(RG_FRAME_IDR if f == 0 else RG_FRAME_P)
        torch.cuda.synchronize()
        times = []
        for _ in range(2):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            eng.analyse_gops_device(ptrs, W, cw, kinds, nf)
            e1.record(stream)
            e1.synchronize()
            eng.sync()
            times.append(e0.elapsed_time(e1))
        print(json.dumps({"profile_case": f"1080p High QP26, 8 streams x {nf} pictures (IDR, then P), one pipelined "
                                          f"launch, {args.profile_form} form",
                          "launch_ms": [round(t, 3) for t in times]}), flush=True)
        eng.close()
        return
    eng = Engine(W, H, QP, profile=RG_PROFILE_HIGH, num_streams=gops, device=local)
    stream = torch.cuda.ExternalStream(eng.cuda_stream, device=f"cuda:{local}")
    torch.cuda.synchronize()
    times = []
    for f in range(2):
        ptrs = []
        for g in range(gops):
            p = base + (g + f) * fbytes
            ptrs += [p, p + W * H, p + W * H + cw * ch]
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        eng.analyse_device(ptrs, W, cw, [RG_FRAME_IDR if f == 0 else RG_FRAME_P] * gops)
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    recs = eng.records()
    kinds = np.bincount(recs["mb_type"].reshape(-1), minlength=4).tolist()
    print(json.dumps({"profile_case": "1080p High QP26, 8 streams, IDR batch then P batch",
                      "idr_batch_ms": round(times[0], 3), "p_batch_ms": round(times[1], 3),
                      "launches_per_batch": eng.mb_w - 1 + 2 * (eng.mb_h - 1) + 1 + 3 + 1,
                      "p_mb_types[skip,p16,i16,i4]": kinds}), flush=True)
    eng.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=16)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", dest="batched", action="store_false",
                    help="leave the batched-streams measurement out of the 1080p line")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="batched workload: keep the library's default launch shape for every size")
    ap.add_argument("--workload", default="1080p", choices=["1080p", "batched", "learned", "4k"],
                    help="the 1080p 8-GOP workload, or the batched-streams configuration (64 mixed-size streams)")
    ap.add_argument("--mode", default="pipelined", choices=["pipelined", "wavefront"],
                    help="one persistent launch for all 15 pictures of the 8 GOPs, or one launch per anti-diagonal")
    ap.add_argument("--profile-case", nargs="?", const="wavefront", default=None,
                    choices=["wavefront", "pipelined", "cnn", "learned"],
                    help="a small slice of the workload (the ncu capture case)")
    ap.add_argument("--profile-form", default="plain", choices=["plain", "learned"],
                    help="analysis form of --profile-case pipelined")
    ap.add_argument("--profile-frames", type=int, default=3, choices=range(1, 9),
                    help="pictures per stream of the pipelined profile case")
    ap.add_argument("--grid", type=int, default=0,
                    help="pipelined mode: resident warps (0 = default)")
    ap.add_argument("--deblock-sms", type=int, default=0,
                    help="pipelined mode: SMs taking deblocking segments first (0 = default, -1 = one mixed queue)")
    ap.add_argument("--intra-sms", type=int, default=0,
                    help="pipelined mode: SMs taking IDR-picture analysis first (0 = default, -1 = none)")
    ap.add_argument("--lag", type=int, default=0,
                    help="pipelined mode: macroblock-times between consecutive pictures in the work order (0 = default)")
    ap.add_argument("--seg", type=int, default=0,
                    help="pipelined mode: macroblocks per work segment (0 = default)")
    args = ap.parse_args()
    rank, world, local = dist_env()
    if args.profile_case == "learned":
        run_profile_case_learned(args, local)
        return
    if args.profile_case == "cnn":
        run_profile_case_cnn(args, local)
        return
    if args.profile_case:
        run_profile_case(args, local)
        return
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.workload == "batched":
        run_batched(args, rank, world, local)
        return
    if args.workload == "learned":
        run_learned(args, rank, world, local)
        return
    if args.workload == "4k":
        run_4k(args, rank, world, local)
        return
    run_engine(args, rank, world, local)


if __name__ == "__main__":
    main()
