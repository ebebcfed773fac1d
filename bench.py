#!/usr/bin/env python
"""Benchmark of the laser Doppler path on the full-size workload (1024^2 x 64 M0 images/s).

Workload (the reference's headline configuration): 1024x1024 frames of 12-bit values packed
2 pixels / 3 bytes, windows of T = 64 frames every 16 frames, fs = 67 kHz, top-4 SVD clutter
removal, single-FFT Fresnel propagation (z = 0.25 m, 852 nm, 12 um), M0/M1/M2 over 4-33 kHz
(bins 4..31).  A step reconstructs `--batch` consecutive windows of a device frame ring that is
larger than L2 (403 MB), so no L2 flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--form plain|chosen]

One process per GPU (torchrun for N > 1): every rank reconstructs its own independent stream
(replicas; the path has no cross-GPU exchange), timing is the max over ranks of CUDA-event time.
Rank 0 prints one JSON line.  `--impl reference` times the CPU restatement of the path (the
reference has no CPU implementation of its own) on the host cores.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import pathlib
import statistics
import subprocess
import threading
import time

ROOT = pathlib.Path(__file__).resolve().parent
H = W = 1024
T, HOP, FS = 64, 16, 67e3
Z0, Z1 = 4, 32                  # 4-33 kHz at df = fs/T = 1046.875 Hz
RANK_CLUTTER = 4
RING_FRAMES = 256               # 403 MB of packed frames (> 126 MB L2)
METRIC = "1024²×64 M0 images/s and p99 frame-to-image latency, chosen vs plain form"
E2E_STEPS = 200                 # end-to-end steps timed (p99 over this many latency samples)
DTYPE = {"chosen": "u12 frames; i8 Gram and f16 hi+lo band DFT on tcgen05 tensor cores (f32 accumulate); "
                   "f32 FFTs and moments; f64 top-r eigenpairs",
         "plain": "u12 frames; f32 Gram, band DFT, FFTs and moments; f64 top-r eigenpairs"}
WORKLOAD = "config1: 1024x1024 12-bit packed, T=64 hop=16, fs=67kHz, top-4 SVD clutter filter, Fresnel z=0.25m, M0/M1/M2 4-33kHz"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--form", default="both", choices=["both", "plain", "chosen"],
                    help="both: the chosen form (the headline) and the plain form on the same ring and steps; "
                         "chosen: tensor-core Gram and band DFT only; plain: all-FP32 kernels only")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the config-2 error, config-3 and config-4 legs of the default run")
    ap.add_argument("--batch", type=int, default=8, help="windows per step")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--af-nz", type=int, default=Z1 - Z0, help="autofocus workload: band planes of the spectrum")
    ap.add_argument("--af-no-pipeline", action="store_true", help="autofocus workload: skip the pipeline leg")
    ap.add_argument("--workload", default="config1", choices=["config1", "batched", "serve", "autofocus"],
                    help="config1: the headline line; batched: 16 uneven acquisitions in one graph launch; "
                         "serve: Poisson-arriving camera streams on the streaming server; autofocus: the "
                         "Shack-Hartmann pass on one config-1 spectrum and its cost inside the pipeline")
    return ap.parse_args()


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_table(name="ncu_traffic_config1.txt"):
    """Per-window (per-launch) DRAM bytes of each stage from a committed ncu summary, if present."""
    p = ROOT / "profiles" / name
    out = {}
    if p.exists():
        for line in p.read_text().splitlines():
            parts = line.split()
            if len(parts) == 2 and not line.startswith("#"):
                try:
                    out[parts[0]] = float(parts[1])
                except ValueError:
                    pass
    return out


def algorithmic_bytes_per_window(nmom=3):
    P, nz = H * W, Z1 - Z0
    packed = 1.5 * P * T
    return {
        "covariance": packed,
        "eigen_filter": 2 * 8 * T * T,
        "band_dft": packed + 8 * P * nz,
        "fft_rows": 2 * 8 * P * nz,
        "fft_cols_moments": 8 * P * nz + 4 * P * nmom,
        "band_dft_rows": packed + 8 * P * nz,
    }


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    def __init__(self, index: int):
        self.index, self.rows, self.proc = index, [], None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in self.rows for n, v in zip(names, r[5:9]) if v.strip().lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def max_over_ranks(value: float, world: int, device=None) -> float:
    """The largest `value` over all ranks (device-timed milliseconds); identity on one rank."""
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(world: int, steps: int, units_per_step: int, ms: float) -> float:
    """Whole-job units per second: every rank processed steps x units_per_step in (max) `ms`."""
    return world * steps * units_per_step / (ms / 1000.0)


def cpu_config1(frames_u16, steps, warmup):
    """The FP32 C++/OpenMP restatement of the path (oracle/cpu_path.cc) on one config-1 window per
    step, all host threads: (windows/s, seconds per window, threads)."""
    from oracle import cpu_path as CP
    from oracle import oracle as O
    cfg = O.PathConfig(H, W, T, HOP, Z0, Z1, fs=FS, z=0.25, clutter_rank=RANK_CLUTTER)
    packed = O.pack12(frames_u16.reshape(-1)).reshape(T, -1)
    for _ in range(max(1, warmup)):
        CP.window(packed, cfg)
    t0 = time.perf_counter()
    for _ in range(steps):
        CP.window(packed, cfg)
    dt = (time.perf_counter() - t0) / steps
    return 1.0 / dt, dt, CP.threads()


def cpu_config0(steps=10):
    """Config 0 (512^2 uint16, T = 32 hop 32, angular spectrum z = 0.30 m, M0/M1/M2 6-18 kHz, no
    clutter filter) on the FP32 C++ restatement, all host threads: images/s."""
    from oracle import cpu_path as CP
    from oracle import oracle as O
    from oracle import synth as S
    frames = S.Interferograms(S.config0(32)).frames(0, 32)
    z0, z1 = O.band_bins(6e3, 18e3, 37e3, 32)
    cfg = O.PathConfig(512, 512, 32, 32, z0, z1, fs=37e3, z=0.30, propagation="angular_spectrum")
    CP.window(frames, cfg, packed=False)
    t0 = time.perf_counter()
    for _ in range(steps):
        CP.window(frames, cfg, packed=False)
    return steps / (time.perf_counter() - t0)


def run_reference(args, rank, world):
    """The reference has no host implementation of the path and its GPU sources cannot be built
    here (they need fetched libraries), so the reference arm times the FP32 C++/OpenMP restatement
    of its algorithm (oracle/cpu_path.cc) on the host cores, rank 0 only: one full config-1 window
    per step, plus config 0's images/s."""
    if rank != 0:
        return
    from oracle import cpu_path as CP
    from oracle import synth as S
    CP.build()
    frames = S.Interferograms(S.config1(T)).frames(0, T)
    v, dt, threads = cpu_config1(frames, args.steps, args.warmup)
    c0 = cpu_config0()
    sample = (f"1 full config-1 window (64 x 1024^2 Mono12p) per step, FP32 C++/OpenMP restatement "
              f"(oracle/cpu_path.cc), {threads} threads, {dt:.3f} s per window")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(v, 4), "unit": "images/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1000 * dt, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 Jacobi)", "data": "synthetic",
        "config": {"workload": WORKLOAD, "windows_per_step": 1, "device": "cpu"},
        "cpu_baseline": {"value": round(v, 4), "unit": "images/s", "cores": threads, "kind": "port",
                         "sample": sample},
        "config0_images_per_s": round(c0, 3),
        "config0": "512^2 uint16, T=32 hop 32, fs 37 kHz, angular spectrum z=0.30 m, M0/M1/M2 6-18 kHz",
        "e2e": {"value": round(v, 4), "unit": "images/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def run_batched(args, local, steps=None):
    """Sixteen seeded acquisitions of uneven frame size (256^2 .. 1536 x 1024), window length
    (32/64/128), z and fs: every acquisition's windows in ONE graph launch (chosen form, schedule
    picked by the autotuner) against per-acquisition launches of the plain form."""
    import torch
    from holoflow_b200 import pipeline as pl
    from holoflow_b200 import synth as sy
    from holoflow_b200.multi import Multi
    dev = torch.device("cuda", local)
    torch.cuda.set_device(local)
    steps = steps or args.steps
    acqs = sy.config3_acquisitions()
    WIN = 2  # windows per acquisition per step
    rings, nfr, outs = [], [], []
    for a in acqs:
        n = a.frames + (WIN - 1) * a.hop
        fr = sy.DeviceInterferograms(a.scene, device=dev).frames(0, n)
        rings.append(pl.pack12(fr.reshape(-1)))
        nfr.append(n)
        outs.append(torch.empty((WIN, 3, a.scene.height, a.scene.width), dtype=torch.float32, device=dev))
        del fr
    first = [0] * len(acqs)

    def cfg(a, form):
        return pl.PipelineConfig(height=a.scene.height, width=a.scene.width, frames=a.frames, hop=a.hop,
                                 z_begin=a.z_begin, z_end=a.z_end, fs=a.scene.fs, z=a.z, clutter_rank=4,
                                 form=form, max_batch=WIN)

    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # per-acquisition launches, plain form
    plans = [pl.Pipeline(cfg(a, 0)) for a in acqs]
    for _ in range(args.warmup):
        for p, r, n, o in zip(plans, rings, nfr, outs):
            p.run(r, n, 0, WIN, out=o)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(steps):
        for p, r, n, o in zip(plans, rings, nfr, outs):
            p.run(r, n, 0, WIN, out=o)
    e1.record(stream)
    torch.cuda.synchronize()
    plain_ms = e0.elapsed_time(e1) / steps
    for p in plans:
        p.close()
    del plans
    # one graph launch, chosen form, tuned schedule
    m = Multi([cfg(a, 1) for a in acqs])
    streams, tuned_ms = m.tune(rings, nfr, first, outs, reps=3)
    schedule = m.schedule()
    for _ in range(args.warmup):
        m.exec(rings, nfr, first, outs)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(steps):
        m.exec(rings, nfr, first, outs)
    e1.record(stream)
    torch.cuda.synchronize()
    graph_ms = e0.elapsed_time(e1) / steps
    m.close()
    nwin = WIN * len(acqs)
    return {
        "metric": "uneven acquisitions: windows/s, one graph launch (chosen) vs per-acquisition launches (plain)",
        "value": round(nwin / (graph_ms / 1000.0), 2), "unit": "windows/s", "n_gpus": 1, "steps": steps,
        "warmup": args.warmup, "ms_per_step": round(graph_ms, 4), "higher_is_better": True,
        "baseline_plain_per_acquisition": {"value": round(nwin / (plain_ms / 1000.0), 2), "ms_per_step":
                                           round(plain_ms, 4)},
        "speedup_vs_plain_per_acquisition": round(plain_ms / graph_ms, 3),
        "schedule": {"branches": schedule["branches"],
                     "assignment": "largest-first" if schedule["largest_first"] else "round-robin",
                     "fused_segment_passes": bool(schedule["fused"]),
                     "seg_tiles": schedule["seg_tiles"] or "max", "band_ctas": schedule["band_ctas"] or "all",
                     "tuned_ms": round(tuned_ms, 4)},
        "config": {"workload": "config3: 16 seeded acquisitions, sizes 256^2..1536x1024, T 32/64/128 hop T/4, "
                               "z 0.15-0.40 m, fs 37/67 kHz, top-4 clutter filter, Fresnel, M0/M1/M2",
                   "windows_per_step": nwin,
                   "acquisitions": [[a.scene.height, a.scene.width, a.frames, a.z_end - a.z_begin] for a in acqs]},
        "dtype": DTYPE["chosen"], "data": "synthetic (device-generated interferograms, seeded)",
    }


def run_serve(args, local, form, seed=1004, life=120):
    """Config 4: camera streams arrive by a Poisson process in time (4 open at the start, then a mean
    gap of ARRIVAL_GAP_S until 12 have come), each with its own frame size (512^2 .. 1536 x 1024), 12-bit packed input,
    (T, hop) of (64, 16) or (128, 32), z and fs; a stream leaves after 120 windows.  Each round every
    open stream pushes one batch worth of new frames from pinned host memory once its previous batch
    has been delivered, and the server gives every stream with ready windows and a free output
    buffer one batch.  No round waits for the device: completions are polled, a stream's two
    pinned output buffers alternate, and arrivals are admitted while other batches run.  Reported:
    sustained frames/s and windows/s and the p50 / p99 frame-to-image latency (push of a window's
    last frame to its images in host memory)."""
    import random

    import numpy as np
    import torch
    from holoflow_b200 import pipeline as pl
    from holoflow_b200 import synth as sy
    from holoflow_b200.server import Server
    dev = torch.device("cuda", local)
    torch.cuda.set_device(local)
    rng = random.Random(seed)
    sizes = [(512, 512), (768, 768), (1024, 1024), (1024, 1536)]
    pools = {}

    def pool(H, W):  # 64 distinct packed frames per size, pinned host
        if (H, W) not in pools:
            fr = sy.DeviceInterferograms(sy.Scene(H, W, 67e3, int(0.85 * min(H, W)), 0.25, seed=2000 + H + W),
                                         device=dev).frames(0, 64)
            pools[(H, W)] = pl.pack12(fr.reshape(-1)).view(64, -1).cpu().pin_memory()
        return pools[(H, W)]

    def new_stream(k):
        H, W = sizes[rng.randrange(len(sizes))]
        T, hop = [(64, 16), (128, 32)][rng.randrange(2)]
        fs = rng.uniform(10e3, 67e3)
        z0, z1 = sy.band_bins(4e3, min(33e3, fs / 2 - 1e3), fs, T)
        cfg = pl.PipelineConfig(height=H, width=W, frames=T, hop=hop, z_begin=max(z0, 1), z_end=z1, fs=fs,
                                z=rng.uniform(0.15, 0.40), clutter_rank=4, form=form, max_batch=4)
        return {"cfg": cfg, "pool": pool(H, W), "pos": 0, "done": 0, "issued": [], "total": 0,
                "out": [torch.empty((4, 3, H, W), dtype=torch.float32, pin_memory=True) for _ in range(2)]}

    LIFE = life  # windows per stream
    srv = Server(max_streams=24, hbm_reserve_bytes=8 << 30)
    waiting = [new_stream(k) for k in range(12)]
    # arrival times: 4 streams at the start, then a Poisson process of mean gap ARRIVAL_GAP_S
    at, arrive = 0.0, []
    for k in range(12):
        if k >= 4:
            at += rng.expovariate(1.0 / ARRIVAL_GAP_S)
        arrive.append(at)
    open_, frames_done, windows_done, refused = {}, 0, 0, 0
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    t0.record()
    start = time.perf_counter()
    rnd = 0
    while (waiting or open_) and time.perf_counter() - start < 120.0:
        # arrivals whose time has come are admitted while the device has room; the others wait
        now = time.perf_counter() - start
        while waiting and arrive[12 - len(waiting)] <= now:
            st = waiting[0]
            cfg = st["cfg"]
            sid = srv.open(cfg, cfg.frames + 6 * cfg.max_batch * cfg.hop)
            if sid is None:
                refused += 1
                break
            waiting.pop(0)
            open_[sid] = st
        for sid, st in open_.items():
            cfg = st["cfg"]
            # one batch in the system per stream: the next batch's frames are pushed once the
            # previous batch has been delivered (a closed loop per stream, no global barrier)
            if st["issued"] or srv.ready(sid) > 0 or st["total"] >= LIFE:
                continue
            need = (cfg.frames - cfg.hop) if st["pos"] == 0 else 0
            left = need + cfg.hop * cfg.max_batch
            while left > 0:  # the pool holds 64 frames: wrap around it
                off = st["pos"] % 64
                k = min(left, 64 - off)
                srv.push(sid, st["pool"][off:], k)
                st["pos"] += k
                left -= k
        outs = {}
        for sid, st in open_.items():
            used = {b for b, _, _ in st["issued"]}
            free = [b for b in (0, 1) if b not in used]
            if free and st["total"] < LIFE:
                outs[sid] = st["out"][free[0]]
        done = srv.step(outs)
        for sid, n in done.items():
            st = open_[sid]
            b = 0 if outs[sid] is st["out"][0] else 1
            st["total"] += n
            st["issued"].append((b, n, st["total"]))
        delivered = srv.poll()
        for sid, st in open_.items():
            while st["issued"] and delivered.get(sid, 0) >= st["issued"][0][2]:
                _, n, _ = st["issued"].pop(0)
                st["done"] += n
                windows_done += n
                frames_done += n * st["cfg"].hop
        for sid in [s_ for s_, st in open_.items() if st["done"] >= LIFE]:
            srv.close(sid)
            del open_[sid]
        if not done:
            time.sleep(50e-6)  # nothing issued this round: yield the host core instead of spinning
        rnd += 1
    t1.record()
    torch.cuda.synchronize()
    secs = t0.elapsed_time(t1) / 1000.0
    lat = np.array(srv.latencies())
    srv.close_all()
    return {"frames_per_s": round(frames_done / secs, 1), "windows_per_s": round(windows_done / secs, 2),
            "latency_ms_p50": round(float(np.percentile(lat, 50)), 3) if lat.size else None,
            "latency_ms_p99": round(float(np.percentile(lat, 99)), 3) if lat.size else None,
            "windows": int(windows_done), "latency_samples": int(lat.size), "rounds": rnd,
            "admission_deferrals": refused, "seconds": round(secs, 3)}


ARRIVAL_GAP_S = 0.05  # mean gap between stream arrivals in the serving workload

AF_NB, AF_ORDERS = 5, (4, 5, 6, 7, 8, 9, 10)
AF_LAM, AF_DX, AF_Z = 852e-9, 12e-6, 0.25


def autofocus_planes(nz, side, device, seed=11):
    """Band planes of one spectrum seen through an aberration: per plane, seeded point scatterers
    in the Fresnel image plane, conj(lens) IFFT(points) exp(i (3 Z4 + 1.5 Z5 - Z6)), complex64 on
    the device."""
    import torch
    g = torch.Generator(device="cpu").manual_seed(seed)
    k = math.pi / (AF_LAM * AF_Z)
    c = (torch.arange(side, dtype=torch.float64) - side / 2.0) * AF_DX
    lens = torch.polar(torch.ones(side, side, dtype=torch.float64), k * (c[None, :] ** 2 + c[:, None] ** 2))
    u = (torch.arange(side, dtype=torch.float64) - (side - 1) / 2.0) / (side / 2.0)
    x, y = u[None, :], u[:, None]
    phi = 3.0 * math.sqrt(3.0) * (2.0 * (x * x + y * y) - 1.0) + 1.5 * 2.0 * math.sqrt(6.0) * x * y \
        - math.sqrt(6.0) * (x * x - y * y)
    ab = torch.conj(lens) * torch.polar(torch.ones_like(phi), phi)
    out = torch.empty((nz, side, side), dtype=torch.complex64, device=device)
    for i in range(nz):
        pts = torch.zeros(side, side, dtype=torch.complex128)
        idx = torch.randint(side // 4, 3 * side // 4, (12, 2), generator=g)
        pts[idx[:, 0], idx[:, 1]] = torch.polar(1.0 + torch.rand(12, generator=g, dtype=torch.float64),
                                                2 * math.pi * torch.rand(12, generator=g, dtype=torch.float64))
        out[i] = (ab * torch.fft.ifft2(pts) * side).to(torch.complex64).to(device)
    return out


def run_autofocus(args, local):
    """One Shack-Hartmann pass (measure + correct) on one config-1 spectrum, its per-call split and
    the roofline of its dominant kernel, the oracle on the host beside it, and the pipeline's
    windows/s with autofocus on and off."""
    import torch
    import holoflow_b200 as hf
    from holoflow_b200 import autofocus as af
    from holoflow_b200 import pipeline as pl
    from holoflow_b200 import synth as sy

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    nz, side, s = args.af_nz, H, H // AF_NB
    planes = autofocus_planes(nz, side, dev)
    out = torch.empty_like(planes)
    op = af.Autofocus(nz, side, side, AF_NB, AF_LAM, AF_DX, AF_Z, indexes=AF_ORDERS)
    stfd = af.ShortTimeFresnel(planes.shape, (s, s), (s, s), AF_LAM, AF_DX, AF_DX, AF_Z, phase_ref="global",
                               output="mean_magnitude", fftshift_windows=True)
    slopes = af.ShackHartmannSlopes(AF_NB, AF_NB, s, s, AF_LAM, AF_DX, AF_DX, AF_Z)
    m0 = stfd(planes)
    sl = slopes(m0)
    phase = torch.zeros((side, side), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream()

    def timed(fn, k):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(k):
            fn()
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / k

    lib = hf.lib()
    lib.hf_reset_launch_count()
    with ClockSampler(local) as clk:
        ms = timed(lambda: op(planes, out=out), args.steps)
        launches = lib.hf_launch_count() // (args.warmup + args.steps)
        split = {"short_time_fresnel_mean": timed(lambda: stfd(planes, out=m0), args.steps),
                 "slopes": timed(lambda: slopes(m0), args.steps),
                 "correct_phase": timed(lambda: af.correct_phase(planes, phase, out=out), args.steps)}
    split["zernike_fit_and_phase"] = max(0.0, ms - sum(split.values()))
    P, Pw = side * side, AF_NB * AF_NB * s * s
    algo = {"short_time_fresnel_mean": 8 * nz * P + 2 * 8 * nz * Pw + 4 * Pw,
            "correct_phase": 2 * 8 * nz * P + 4 * P}
    dom = max(("short_time_fresnel_mean", "correct_phase"), key=lambda k: split[k])
    peak, peak_kind = peaks()
    achieved = algo[dom] / (split[dom] / 1000.0) / 1e9
    tr = traffic_table("ncu_traffic_autofocus.txt").get(dom) if nz == Z1 - Z0 else None
    roof = {"kernel": dom, "bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "peak_kind": peak_kind,
            "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": tr,
            "algorithmic_bytes_per_launch": algo[dom], "ms_per_launch": round(split[dom], 4),
            "calls_ms": {k: round(v, 4) for k, v in split.items()}}

    # the pipeline on config-1 windows with the pass on every window (chosen form), and without
    def pipeline_rate(orders):
        B = 8
        cfg = pl.PipelineConfig(height=H, width=W, frames=T, hop=HOP, z_begin=Z0, z_end=Z1, fs=FS, z=AF_Z,
                                lam=AF_LAM, pitch=AF_DX, clutter_rank=RANK_CLUTTER, max_batch=B,
                                form=hf.HF_FORM_CHOSEN, autofocus_nb_subaps=AF_NB if orders else 0,
                                autofocus_orders=orders)
        gen = sy.DeviceInterferograms(sy.config1_scene(acquisition=0), device=dev)
        packed = pl.pack12(gen.frames(0, 64).reshape(-1)).view(64, cfg.frame_bytes)
        ring = torch.cat([packed] * (RING_FRAMES // 64)).reshape(-1).contiguous()
        pipe = pl.Pipeline(cfg)
        res = torch.empty((B, *pipe.out_shape), dtype=torch.float32, device=dev)
        step = [0]

        def run():
            pipe.run(ring, RING_FRAMES, (step[0] * B * HOP) % RING_FRAMES, B, out=res)
            step[0] += 1
        t = timed(run, max(4, args.steps // 2))
        pipe.timing(True)
        run()
        torch.cuda.synchronize()
        stages = {k: round(v[0], 3) for k, v in pipe.stage_times().items() if v[0] > 0}
        pipe.timing(False)
        pipe.close()
        return B / (t / 1000.0), t, stages

    on, on_ms, on_st = pipeline_rate(AF_ORDERS) if not args.af_no_pipeline else (0.0, 0.0, {})
    off, off_ms, off_st = pipeline_rate(()) if not args.af_no_pipeline else (0.0, 0.0, {})

    cpu = None
    if not args.no_cpu:
        from oracle import shack as SH
        host = planes.cpu().numpy()
        cfg = SH.AutofocusConfig(AF_NB, AF_LAM, AF_DX, AF_Z, list(AF_ORDERS))
        SH.autofocus(host[:2], cfg)  # warm-up (imports, FFT plans) on a 2-plane sample
        t0 = time.perf_counter()
        SH.autofocus(host, cfg)
        dt = time.perf_counter() - t0
        cpu = {"value": round(1.0 / dt, 4), "unit": "passes/s", "cores": 1, "kind": "port",
               "sample": f"one full pass over the same {nz} x {side}^2 spectrum (oracle/shack.py, NumPy)"}

    print(json.dumps({
        "metric": "Shack-Hartmann autofocus passes/s on one spectrum", "value": round(1000.0 / ms, 2),
        "unit": "passes/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded point scatterers behind a defocus + astigmatism aberration)",
        "config": {"workload": f"config1 spectrum: {nz} x {side}x{side} complex64 band planes, nb_subaps={AF_NB} "
                               f"({s}x{s} sub-apertures), Noll {list(AF_ORDERS)}, lambda 852 nm, 12 um, z 0.25 m; "
                               "measure (short-time Fresnel + band mean, slopes, fit, phase) + correct",
                   "l2": "inputs (1.9 GB of planes per pass) larger than L2"},
        "gpu_launches": launches, "roofline": roof, "cpu_baseline": cpu,
        "pipeline_config1_chosen": {"autofocus_on_windows_per_s": round(on, 1), "ms_per_8_windows_on": round(on_ms, 3),
                                    "autofocus_off_windows_per_s": round(off, 1),
                                    "ms_per_8_windows_off": round(off_ms, 3),
                                    "stages_ms_per_8_windows_on": on_st, "stages_ms_per_8_windows_off": off_st},
        "clocks": clk.summary()}), flush=True)


def serve_pair(args, local):
    """Config 4 for both forms: an untimed warm-up of each (loads every kernel module and builds
    every table once, so neither timed run pays the process's first-use costs), then the timed
    runs on the same seeded streams."""
    for f in (1, 0):
        run_serve(args, local, f, life=8)
    res = {f: run_serve(args, local, 1 if f == "chosen" else 0) for f in ("chosen", "plain")}
    return {
        "metric": "streaming server: sustained frames/s and p50/p99 frame-to-image latency, chosen vs plain",
        "value": res["chosen"]["frames_per_s"], "unit": "frames/s", "n_gpus": 1, "higher_is_better": True,
        "chosen": res["chosen"], "plain": res["plain"],
        "chosen_over_plain_frames_per_s": round(res["chosen"]["frames_per_s"] / res["plain"]["frames_per_s"], 3),
        "config": {"workload": "config4: 12 Poisson-arriving streams (4 at start, then a mean gap of 50 ms), 512^2.."
                               "1536x1024 12-bit packed, (T, hop) (64,16)/(128,32), fs 10-67 kHz, z 0.15-0.40 m, "
                               "top-4 clutter filter, 120 windows per stream, 8 GiB free-HBM reserve"},
        "dtype": DTYPE["chosen"], "data": "synthetic (device-generated interferograms, seeded)"}


def config1_cfg(form, B):
    from holoflow_b200 import pipeline as pl
    return pl.PipelineConfig(height=H, width=W, frames=T, hop=HOP, z_begin=Z0, z_end=Z1, fs=FS, z=0.25,
                             clutter_rank=RANK_CLUTTER, max_batch=B, form=form)


def measure_form(args, world, dev, local, form, packed, e2e_on=True):
    """One numeric form on the config-1 workload: device-resident windows/s over exactly K timed
    steps (the camera stream's ring filled before timing), per-stage times, the dominant stage's
    roofline, then the end-to-end leg through the camera-stream API.  Returns the numbers and the
    images of the last timed step's first window (its frames are generated frames 0..63 in order)."""
    import torch
    import torch.distributed as dist
    import holoflow_b200 as hf
    from holoflow_b200 import pipeline as pl

    B = args.batch
    cfg = config1_cfg(form, B)
    fb = cfg.frame_bytes
    pipe = pl.Pipeline(cfg)
    nmom = pipe.out_shape[0]
    out = torch.empty((B, *pipe.out_shape), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream()

    # device-resident input: every frame of the warm-up and timed steps is in the camera stream's
    # ring before timing starts (the stream overlaps the next batch's eigen phase with this one)
    nsteps = args.warmup + args.steps
    total_frames = (T - HOP) + nsteps * B * HOP
    cam_dev = pl.CameraStream(pipe, total_frames)
    reps = (total_frames + 63) // 64
    src = torch.cat([packed] * reps)[:total_frames].contiguous()
    cam_dev.push(src, total_frames)
    del src
    torch.cuda.synchronize()

    def step():
        n = cam_dev.process(B, out)
        assert n == B

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    pipe.timing(True)
    lib = hf.lib()
    lib.hf_reset_launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
    launches = lib.hf_launch_count()
    ms = e0.elapsed_time(e1)
    stages = {k: v for k, v in pipe.stage_times().items() if v[0] > 0}
    pipe.timing(False)
    window0 = out[0].cpu().numpy().copy()
    cam_dev.close()
    ms = max_over_ranks(ms, world, dev)
    res = {"value": round(aggregate_rate(world, args.steps, B, ms), 2), "ms_per_step": round(ms / args.steps, 4),
           "gpu_launches": int(launches), "clocks": clk.summary(),
           "stages_ms_per_step": {k: round(v[0] / max(args.steps, 1), 4) for k, v in stages.items()}}

    # roofline of the dominant stage on the critical path (the next batch's eigen phase runs on a
    # side stream): algorithmic bytes of that stage for the step's windows / its CUDA-event time
    peak, peak_kind = peaks()
    algo = algorithmic_bytes_per_window(nmom)
    crit = {k: v for k, v in stages.items() if k != "eigen_filter"}
    dom = max(crit, key=lambda k: crit[k][0]) if crit else None
    if dom:
        per_launch_ms = stages[dom][0] / max(args.steps, 1)
        bytes_launch = algo.get(dom, 0.0) * B
        achieved = bytes_launch / (per_launch_ms / 1000.0) / 1e9
        tr = traffic_table().get(dom) if form == 1 else None
        res["roofline"] = {"kernel": dom, "bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                           "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
                           "traffic": (tr * B) if tr else None, "algorithmic_bytes_per_launch": bytes_launch,
                           "ms_per_launch": round(per_launch_ms, 4),
                           "stage_note": "eigen_filter of the next batch runs on a side stream, overlapped"}

    if e2e_on:
        res["e2e"] = measure_e2e(args, world, dev, pipe, packed, fb, nmom)
    pipe.close()
    return res, window0


def measure_e2e(args, world, dev, pipe, packed, fb, nmom):
    """End to end through the camera-stream API: pinned host frames in, pinned host moments out.

    Throughput leg: each step pushes one step of new frames (B*hop) on a copy stream, reconstructs
    B windows on the compute stream and copies their images to the host on the camera stream's copy
    stream.  Frames are pushed PUSH_AHEAD steps before they are reconstructed (the lookahead Gram
    pass of step s reads step s+1's frames), so step s's H2D, step s-2's compute and step s-3's D2H
    overlap.  The timed region holds exactly K pushes, K reconstructions and K output copies, with
    K = max(--steps, 200) so that the latency percentiles rest on enough samples.
    Unloaded-latency leg: one step at a time (push, reconstruct, copy out, wait), 200 steps: the
    frame-to-image latency of a step that meets an idle device."""
    import torch
    import torch.distributed as dist
    from holoflow_b200 import pipeline as pl
    B = args.batch
    K = max(args.steps, E2E_STEPS)
    stream = torch.cuda.current_stream()
    PUSH_AHEAD = 2
    nstep_frames = B * HOP
    host_frames = torch.empty(nstep_frames * fb, dtype=torch.uint8, pin_memory=True)
    reps = (nstep_frames + 63) // 64
    host_frames.view(nstep_frames, fb).copy_(torch.cat([packed] * reps)[:nstep_frames].cpu())
    host_out = [torch.empty((B, *pipe.out_shape), dtype=torch.float32, pin_memory=True) for _ in range(2)]
    h2d = torch.cuda.Stream(device=dev)
    tstream = torch.cuda.Stream(device=dev)
    cam = pl.CameraStream(pipe, (T - HOP) + (PUSH_AHEAD + 2) * nstep_frames)
    pushed_at = {}

    def push_step(j):
        ev = torch.cuda.Event(enable_timing=True)
        ev.record(h2d)
        pushed_at[j] = ev
        cam.push(host_frames, nstep_frames, stream=h2d)

    cam.push(host_frames, T - HOP, stream=h2d)  # prefill: the first window needs T - hop older frames
    for j in range(PUSH_AHEAD):
        push_step(j)
    total = args.warmup + K
    lat = []
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for s in range(total):
        if s == args.warmup:
            torch.cuda.synchronize()
            if world > 1:
                dist.barrier()
            f0.record(stream)
            h2d.wait_event(f0)
        push_step(s + PUSH_AHEAD)
        n = cam.process(B, host_out[s % 2], stream=stream, async_copy=True)
        assert n == B
        cam.output_wait(tstream)
        b = torch.cuda.Event(enable_timing=True)
        b.record(tstream)
        if s >= args.warmup:
            lat.append((pushed_at[s], b))
    cam.output_wait(stream)
    f1.record(stream)
    torch.cuda.synchronize()
    ems = max_over_ranks(f0.elapsed_time(f1), world, dev)
    cam.close()

    def pct(v, q):
        v = sorted(v)
        return v[min(len(v) - 1, int(round(q * (len(v) - 1))))]

    step_lat = [a.elapsed_time(b) for a, b in lat]
    # unloaded latency: nothing queued ahead of a step
    cam = pl.CameraStream(pipe, (T - HOP) + 2 * nstep_frames)
    cam.push(host_frames, T - HOP, stream=h2d)
    idle = []
    for s in range(args.warmup + E2E_STEPS):
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        a.record(h2d)
        cam.push(host_frames, nstep_frames, stream=h2d)
        cam.process(B, host_out[0], stream=stream, async_copy=True)
        cam.output_wait(tstream)
        b = torch.cuda.Event(enable_timing=True)
        b.record(tstream)
        torch.cuda.synchronize()
        if s >= args.warmup:
            idle.append(a.elapsed_time(b))
    cam.close()
    return {"value": round(aggregate_rate(world, K, B, ems), 2), "unit": "images/s",
            "h2d_bytes_per_step": nstep_frames * fb, "d2h_bytes_per_step": B * nmom * H * W * 4,
            "steps": K, "ms_per_step": round(ems / K, 4),
            "latency_ms_p50": round(pct(step_lat, 0.5), 3), "latency_ms_p99": round(pct(step_lat, 0.99), 3),
            "latency_definition": "start of the H2D push of a step's new frames (pinned host) to its "
                                  "moment images in pinned host memory; frames are pushed 2 steps ahead "
                                  "(H2D, compute and D2H of different steps overlap)",
            "unloaded_latency_ms_p50": round(pct(idle, 0.5), 3), "unloaded_latency_ms_p99": round(pct(idle, 0.99), 3),
            "unloaded_latency_definition": f"{E2E_STEPS} steps one at a time on an idle device: push of B*hop "
                                           "new frames, reconstruction of B windows, images in pinned host memory"}


def config2_errors(dev, oracle_mod):
    """Config 2 as stated: 1024^2 x 64 frames with a rank-2 global clutter at SCR 0, -20, -40 dB
    (device-generated), top-4 clutter removal; each form's M0/M1/M2 relative L2 error against the
    FP64 oracle, which is the checker here and runs outside any timed region."""
    import numpy as np
    import torch
    import holoflow_b200 as hf
    from holoflow_b200 import pipeline as pl
    from holoflow_b200 import synth as sy
    O = oracle_mod
    out = {}
    ocfg = O.PathConfig(H, W, T, HOP, Z0, Z1, fs=FS, z=0.25, clutter_rank=RANK_CLUTTER)
    for scr in (0.0, -20.0, -40.0):
        fr = sy.DeviceInterferograms(sy.config2_scene(scr), device=dev).frames(0, T)
        ring = pl.pack12(fr.reshape(-1))
        host = fr.cpu().numpy().view(np.uint16)
        exp = O.reconstruct_window(host, ocfg)
        row = {}
        for name, form in (("chosen", hf.HF_FORM_CHOSEN), ("plain", hf.HF_FORM_PLAIN)):
            p = pl.Pipeline(config1_cfg(form, 1))
            got = p.run(ring, T, 0, 1).cpu().numpy()[0]
            p.close()
            row[name] = [float("%.3e" % O.rel_l2(got[m], exp[m])) for m in range(3)]
        out[f"{scr:+.0f}dB"] = row
        del fr, ring
    return out


def main():
    args = parse()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.workload == "batched":
        if rank == 0:
            print(json.dumps(run_batched(args, local)), flush=True)
        return None
    if args.workload == "autofocus":
        return run_autofocus(args, local) if rank == 0 else None
    if args.workload == "serve":
        if rank == 0:
            print(json.dumps(serve_pair(args, local)), flush=True)
        return None

    import numpy as np
    import torch
    import torch.distributed as dist
    import holoflow_b200 as hf
    from holoflow_b200 import pipeline as pl
    from holoflow_b200 import synth as sy

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)

    B = args.batch
    # synthetic frames: 64 distinct frames generated on the device, tiled over the ring
    gen = sy.DeviceInterferograms(sy.config1_scene(acquisition=rank), device=dev)
    base = gen.frames(0, 64)
    packed = pl.pack12(base.reshape(-1)).view(64, config1_cfg(1, B).frame_bytes)
    base_host = base.cpu().numpy().view(np.uint16).copy()
    del base, gen

    forms = ["chosen", "plain"] if args.form == "both" else [args.form]
    results, windows = {}, {}
    for f in forms:
        code = hf.HF_FORM_CHOSEN if f == "chosen" else hf.HF_FORM_PLAIN
        results[f], windows[f] = measure_form(args, world, dev, local, code, packed, e2e_on=not args.no_e2e)
    head = forms[0]
    r = results[head]

    # the FP64 oracle as the checker (outside every timed region, rank 0 at N = 1): moment errors
    # of the last timed step's first window, and the CPU baseline timed on the same window
    cpu, merr, cfg2 = None, None, None
    if rank == 0 and world == 1 and not args.no_cpu:
        from oracle import oracle as O
        ocfg = O.PathConfig(H, W, T, HOP, Z0, Z1, fs=FS, z=0.25, clutter_rank=RANK_CLUTTER)
        exp = O.reconstruct_window(base_host, ocfg)
        merr = {f: [float("%.3e" % O.rel_l2(windows[f][m], exp[m])) for m in range(3)] for f in forms}
        from oracle import cpu_path as CP
        CP.build()
        v, dt, threads = cpu_config1(base_host, 5, 1)
        cpu = {"value": round(v, 4), "unit": "images/s", "cores": threads, "kind": "port",
               "sample": "5 full config-1 windows (64 x 1024^2 Mono12p, the bench's own frames), FP32 C++/OpenMP "
                         "restatement of the path (oracle/cpu_path.cc), %.3f s per window" % dt,
               "config0_images_per_s": round(cpu_config0(), 3)}
        if not args.no_extra:
            cfg2 = config2_errors(dev, O)

    extra = {}
    if rank == 0 and world == 1 and not args.no_extra and args.form == "both":
        torch.cuda.empty_cache()
        extra["config3_batched"] = run_batched(args, local, steps=min(args.steps, 10))
        torch.cuda.empty_cache()
        extra["config4_serve"] = serve_pair(args, local)

    if rank == 0:
        line = {
            "metric": METRIC, "value": r["value"], "unit": "images/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": DTYPE[head],
            "data": "synthetic (device-generated interferograms, seeded)",
            "config": {"workload": WORKLOAD, "form": head, "windows_per_step": B, "ring_frames": RING_FRAMES,
                       "l2": "inputs larger than L2 (403 MB frame ring + 235 MB band planes per window)",
                       "parallelism": f"replicas x{world}"},
            "gpu_launches": r["gpu_launches"], "roofline": r.get("roofline"), "cpu_baseline": cpu,
            "e2e": r.get("e2e"), "clocks": r["clocks"], "stages_ms_per_step": r["stages_ms_per_step"],
        }
        if "plain" in results and head != "plain":
            p = results["plain"]
            line["plain"] = {"value": p["value"], "ms_per_step": p["ms_per_step"], "dtype": DTYPE["plain"],
                             "stages_ms_per_step": p["stages_ms_per_step"], "roofline": p.get("roofline"),
                             "e2e": p.get("e2e"), "clocks": p["clocks"], "gpu_launches": p["gpu_launches"]}
            line["chosen_over_plain"] = round(r["value"] / p["value"], 3)
            if r.get("e2e") and p.get("e2e"):
                line["chosen_over_plain_e2e"] = round(r["e2e"]["value"] / p["e2e"]["value"], 3)
        if merr:
            line["moment_error"] = {"metric": "relative L2 of M0/M1/M2 vs the FP64 oracle, last timed step's "
                                              "first window", **merr}
        if cfg2:
            line["config2_moment_error"] = {"workload": "config2: config 1 + rank-2 global clutter, 1024^2 x 64, "
                                                        "top-4 removal; relative L2 of M0/M1/M2 vs FP64 oracle",
                                            **cfg2}
        line.update(extra)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
