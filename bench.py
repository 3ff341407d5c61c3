#!/usr/bin/env python
"""Benchmark of the reconstruction path on B200.

Default workload (one GPU), `recon_4k`: the seeded 4096 x 4096 x 41-tilt
series (-60..60 step 3, thickness 1200, 500 ellipsoids + 40 beads scaled to
4k, Poisson noise at 50 e-/px).  The line's value is SART on it (15
iterations, 5 subsets, relaxation 1/subsets, FP32); a "step" is one full
reconstruction of the series.  Sub-records on the same frames: `wbp` (the
metric's WBP half, FP32), `precision` (FP16 and BF16 storage of WBP and SART
beside FP32, with their error against the FP64 oracle) and `reference_cuda`
(the reference's own CUDA Recon, built from its sources, against this
library's reference-shaped entry points on a band of rows).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

Metric: GVoxel*tilt/s = Nx * ny * Nz * T of the output grid per second (the
same count for WBP and SART; SART's iterations are work inside a step).

* value    : device-resident (projections already in HBM), CUDA events on the
             launching stream, max over ranks.  Inputs (2.75 GB of projections,
             80.5 GB of volume) exceed the 126 MB L2.
* e2e      : the same through the host API (at3r_run_host): pinned host
             frames in, host volume frames out, copies inside the timed region
             (--e2e-steps of them).
* roofline : the kernel with the largest device time, its algorithmic bytes
             per launch / its mean launch time (CUDA events around every
             launch on its stream, during one instrumented step), against the
             measured HBM copy bandwidth; plus its on-chip (L1/shared) figure.
* cpu_baseline : the FP32 C++ port of the same math (oracle/, OpenMP) on the
             host cores, on a sample of the series' slices.
* error    : the volume's two middle slices against the FP64 oracle.

With --impl reference the same workload is timed on the host cores by the
FP32 port, rank 0 only (the reference's Recon has no CPU implementation).
N > 1: torchrun, one process per GPU, each rank reconstructs its own series
(weak scaling, no collective on the data path); the sub-records are N = 1 only.
Other workloads: --workload sart_1k | wbp_512 | wbp_4k | sart_4k | batch_uneven |
serve_mix | stack_4k | thick_4k (and profiling cases, see workload()).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "GVoxel·tilt/s (WBP, SART) + p50/p99 series latency vs plain FP32 at stated err"
UNIT = "GVoxel·tilt/s"


def workload(name: str, seed_offset: int = 0) -> dict:
    from aretomo3_b200 import synth
    if name == "sart_1k":
        c = synth.sart_1k(seed=2 + seed_offset)
        c.update(method="sart", relax=0.3, label="SART 1024x1024x61 tilts, thickness 300, 15 iterations, 5 subsets, "
                                                 "relaxation 0.3, Poisson 50 e-/px")
    elif name == "sart_1k_small":
        # profiling case: the same shape per slice, 128 rows (volume 157 MB > L2)
        c = synth.sart_1k(seed=2 + seed_offset)
        c.update(ny=128, method="sart", relax=0.3,
                 label="SART 1024x128x61 tilts, thickness 300, 15 iterations, 5 subsets, relaxation 0.3")
    elif name == "sart_1k_ref_relax":
        c = synth.sart_1k(seed=2 + seed_offset)
        c.update(method="sart", relax=0.0, label="SART 1024x1024x61 tilts, thickness 300, 15 iterations, 5 subsets, "
                                                 "relaxation 1/subsets")
    elif name == "wbp_512":
        c = synth.wbp_small(seed=1 + seed_offset)
        c.update(method="wbp", label="WBP 512x512x41 tilts, thickness 128, Gaussian noise 0.1 x mean")
    elif name == "wbp_4k":
        c = synth.precision_4k(seed=3 + seed_offset)
        c.update(method="wbp", label="WBP 4096x4096x41 tilts, thickness 1200")
    elif name == "sart_4k_rows":
        # tuning case: the 4k geometry per slice, 256 rows
        c = synth.precision_4k(seed=3 + seed_offset)
        c.update(ny=256, method="sart", relax=0.0,
                 label="SART 4096x256x41 tilts, thickness 1200, 15 iterations, 5 subsets")
    elif name == "wbp_4k_rows":
        c = synth.precision_4k(seed=3 + seed_offset)
        c.update(ny=256, method="wbp", label="WBP 4096x256x41 tilts, thickness 1200")
    elif name == "sart_4k_rows64":
        # profiling case of the default series: 64 rows (volume 1.26 GB > L2)
        c = synth.precision_4k(seed=3 + seed_offset)
        c.update(ny=64, method="sart", relax=0.0,
                 label="SART 4096x64x41 tilts, thickness 1200, 15 iterations, 5 subsets")
    elif name == "sart_4k":
        c = synth.precision_4k(seed=3 + seed_offset)
        c.update(method="sart", relax=0.0, label="SART 4096x4096x41 tilts, thickness 1200, 15 iterations, 5 subsets")
    elif name == "recon_4k":
        # the 4096 x 4096 x 41 series both halves of the metric are quoted on:
        # SART is the line's value, WBP / the 16-bit forms / the reference's own
        # CUDA Recon are sub-records on the same frames
        c = synth.precision_4k(seed=3 + seed_offset)
        c.update(method="sart", relax=0.0, with_wbp=True, with_precision=True, with_reference_cuda=True,
                 label="SART 4096x4096x41 tilts (-60..60 step 3), thickness 1200, 15 iterations, 5 subsets, "
                       "relaxation 1/subsets; 500 ellipsoids + 40 beads, Poisson 50 e-/px",
                 wbp_label="WBP 4096x4096x41 tilts (-60..60 step 3), thickness 1200, same frames")
    else:
        raise SystemExit(f"unknown workload {name}")
    c["name"] = name
    return c


def units_per_step(c) -> float:
    return float(c["nx"] & ~1) * c["ny"] * c["vol_z"] * len(c["tilts"])


STORAGE = {"f32": 0, "f16": 1, "bf16": 2}


def plan_kwargs(c) -> dict:
    from aretomo3_b200 import recon
    st = STORAGE[c.get("storage", "f32")]
    slab = int(c.get("slab", 0))
    if c["method"] == "sart":
        return dict(method=recon.SART, start_tilt=0, num_tilts=len(c["tilts"]), iterations=c["iters"],
                    subsets=c["subsets"], relax=c.get("relax", 0.0), storage=st, slab_slices=slab)
    return dict(method=recon.WBP, storage=st, slab_slices=slab)


# --- clocks -----------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.gpu)], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["active", "hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names[1:], f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(smax)), "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def profiled_traffic(kernel: str, workload_name: str, storage: str):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    d = json.load(open(p))
    return d.get(f"{workload_name}/{storage}", {}).get(kernel)


# Shared-memory / L1 bytes one work unit of a kernel moves on chip: the back-
# projectors read one 8-byte (p[i], p[i+1]) pair per voxel, tilt and slice;
# the forward projector reads four bilinear taps per ray sample and slice (a
# 16-byte load serves four slices: 16 B per sample-slice, 8 B from the 16-bit
# shadow).
def onchip_bytes_per_unit(kernel: str, storage: str):
    if kernel in ("bp_sart", "bp_wbp_2x"):
        return 8.0
    if kernel == "fp_diff":
        return 16.0 if storage == "f32" else 8.0
    return None


def onchip_roof(kernel: str, d: dict, storage: str, clk: dict):
    """The kernel's algorithmic L1/shared-memory bytes per second against the
    data path's 128 B/clk/SM over 148 SMs at the SM clock sampled during the
    timed region."""
    b = onchip_bytes_per_unit(kernel, storage)
    mhz = clk.get("sm_mhz") or 1965.0
    if b is None or not d["ms"]:
        return None
    achieved = b * d["units"] / (d["ms"] / 1e3) / 1e12
    peak = 148 * 128 * mhz * 1e6 / 1e12
    return {"resource": "L1/shared-memory data path", "bytes_per_unit": b, "achieved": achieved, "peak": peak,
            "unit": "TB/s", "frac": achieved / peak, "sm_mhz": mhz}


# --- CPU side (oracle/ FP32 port): baseline leg and reference arm ------------
def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib  # noqa: E402  (checker / CPU baseline only)
    return oracle_lib


def cpu_port_run(c, frames, y0, y1, threads):
    ol = _oracle()
    if c["method"] == "sart":
        return ol.sart(frames, c["tilts"], c["vol_z"], 0, len(c["tilts"]), c["iters"], c["subsets"],
                       relax=c.get("relax", 0.0), y0=y0, y1=y1, f32=True, threads=threads)
    return ol.wbp(frames, c["tilts"], c["vol_z"], y0=y0, y1=y1, f32=True, threads=threads)


def cpu_sample_slices(c) -> int:
    # about 10-30 s of CPU work on 16 host cores
    if c["method"] == "sart":
        return 48 if c["nx"] <= 1024 else 4
    return 128 if c["nx"] <= 1024 else 8


def cpu_baseline(c, frames, threads) -> dict:
    s = min(cpu_sample_slices(c), c["ny"])
    y0 = (c["ny"] - s) // 2
    t = time.perf_counter()
    cpu_port_run(c, frames, y0, y0 + s, threads)
    dt = time.perf_counter() - t
    units = float(c["nx"] & ~1) * s * c["vol_z"] * len(c["tilts"])
    return {"value": units / dt / 1e9, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{s} of {c['ny']} y-slices of the series ({c['label']}); FP32 C++ port, OpenMP, "
                      f"{dt:.2f} s"}


def error_vs_oracle(c, frames, vol_gpu, n_slices=2, mid=None) -> dict:
    """Relative L2 / max-abs of the GPU volume against the FP64 oracle on a few
    slices (the checker).  `mid`: those slices alone, when the whole volume was
    not copied back."""
    ol = _oracle()
    y0 = c["ny"] // 2
    if c["method"] == "sart":
        ref = ol.sart(frames, c["tilts"], c["vol_z"], 0, len(c["tilts"]), c["iters"], c["subsets"],
                      relax=c.get("relax", 0.0), y0=y0, y1=y0 + n_slices)
    else:
        from aretomo3_b200 import recon
        mode = 1 if c.get("_c2r") == recon.C2R_PACKED else 0
        ref = ol.wbp(frames, c["tilts"], c["vol_z"], y0=y0, y1=y0 + n_slices, c2r_mode=mode)
    got = (mid if mid is not None else vol_gpu[y0:y0 + n_slices]).astype(np.float64)
    return {"rel_l2": float(np.linalg.norm(got - ref) / np.linalg.norm(ref)),
            "max_abs": float(np.abs(got - ref).max()), "slices": n_slices, "against": "FP64 oracle"}


def run_reference_arm(args, c, rank, world):
    if rank != 0:
        return
    from aretomo3_b200 import synth
    frames = synth.make_tilt_series(c["nx"], c["ny"], c["tilts"], c["vol_z"], c["phantom"])
    threads = os.cpu_count() or 1
    # a 4096-wide slice is seconds of work on all host threads: one per step
    s = 1 if c["nx"] > 1024 else min(max(4, cpu_sample_slices(c) // 3), c["ny"])
    y0 = (c["ny"] - s) // 2
    for _ in range(args.warmup):
        cpu_port_run(c, frames, y0, min(y0 + 1, c["ny"]), threads)
    t = time.perf_counter()
    for _ in range(args.steps):
        cpu_port_run(c, frames, y0, y0 + s, threads)
    dt = time.perf_counter() - t
    units = float(c["nx"] & ~1) * s * c["vol_z"] * len(c["tilts"]) * args.steps
    value = units / dt / 1e9
    sample = (f"each step: {s} of {c['ny']} y-slices ({c['label']}); FP32 C++ port of the reference math "
              f"(the reference's Recon is GPU-only), OpenMP on {threads} host threads")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": {"workload": c["label"], "name": c["name"]},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _gpu_index(local_rank: int) -> int:
    cvd = os.environ.get("CUDA_VISIBLE_DEVICES", "")
    if cvd.replace(",", "").isdigit():
        return int(cvd.split(",")[local_rank])
    return local_rank


def measure(c, frames, proj, vol, stream, steps, warmup, e2e_steps, world, gpu_index, instrument=True,
            clocks=True):
    """One plan over the series already in HBM: `warmup` untimed steps, then
    `steps` timed ones (barrier + synchronize on both sides, CUDA events on the
    launching stream, max over ranks), one instrumented step (an event pair
    around every launch) for the per-kernel shares, and `e2e_steps` through the
    host API (pinned frames in, pinned volume frames out, copies inside the
    timed region).  Returns a dict of the measurements; the volume's two middle
    slices are copied back for the error check."""
    import torch
    from aretomo3_b200 import recon, ranks
    T, ny, nx = frames.shape
    Nx, Nz = nx & ~1, c["vol_z"]
    dev = proj.device
    plan = recon.Plan(nx, ny, c["tilts"], Nz, **plan_kwargs(c))
    c["_c2r"] = plan.c2r
    out = {"slab_slices": plan.slab, "c2r": plan.c2r}
    for _ in range(warmup):
        plan.run_device(proj.data_ptr(), vol.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize()
    sampler = ClockSampler(gpu_index) if clocks else None
    if sampler:
        sampler.start()
        time.sleep(0.3)
    ranks.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        plan.run_device(proj.data_ptr(), vol.data_ptr(), stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ranks.barrier()
    ms_total = ranks.max_over_ranks(e0.elapsed_time(e1), device=dev)
    out["clocks"] = sampler.stop() if sampler else None
    out["launches_per_step"] = plan.last_launches
    units = units_per_step(c)
    out["ms_per_step"] = ms_total / steps
    out["value"] = ranks.aggregate_rate(units, steps, world, ms_total) / 1e9
    y_mid = ny // 2
    out["mid"] = vol[y_mid:y_mid + 2].cpu().numpy()
    if instrument:
        # per-kernel device times: one more step with an event pair on the
        # launching stream around every launch (the plan runs one stream while
        # timing is on, so no kernel's events also time another's work)
        plan.set_timing(True)
        torch.cuda.synchronize()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        plan.run_device(proj.data_ptr(), vol.data_ptr(), stream.cuda_stream)
        f1.record(stream)
        torch.cuda.synchronize()
        out["instrumented_ms"] = ranks.max_over_ranks(f0.elapsed_time(f1), device=dev)
        out["kstats"] = plan.kernel_stats()
        plan.set_timing(False)
    if e2e_steps > 0:
        # e2e through the host API: pinned frames in, pinned volume frames out
        # (a ring of frames when the volume would not fit host memory twice)
        big = Nx * Nz * ny * 4 > (8 << 30)
        ring = 64 if big else ny
        pin_in = torch.from_numpy(frames).pin_memory()
        pin_out = torch.empty((ring, Nz, Nx), dtype=torch.float32).pin_memory()
        fin = [pin_in[t].numpy() for t in range(T)]
        fout = [pin_out[y % ring].numpy() for y in range(ny)]
        plan.run_host(fin, fout, stream.cuda_stream)  # warm the host-path buffers
        torch.cuda.synchronize()
        ranks.barrier()
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        for _ in range(e2e_steps):
            plan.run_host(fin, fout, stream.cuda_stream)
        g1.record(stream)
        torch.cuda.synchronize()
        ranks.barrier()
        ms_e2e = ranks.max_over_ranks(g0.elapsed_time(g1), device=dev)
        # the frames the host path wrote last equal the device path's slices
        last = torch.arange(ny - ring, ny)
        dev_tail = vol[ny - ring:].cpu()
        host_ok = bool(torch.equal(pin_out[last % ring], dev_tail))
        out["e2e"] = {"value": ranks.aggregate_rate(units, e2e_steps, world, ms_e2e) / 1e9, "unit": UNIT,
                      "ms_per_step": ms_e2e / e2e_steps, "steps": e2e_steps,
                      "h2d_bytes_per_step": int(frames.nbytes), "d2h_bytes_per_step": int(Nx * Nz * ny * 4),
                      "host_equals_device": host_ok,
                      "host_frames": "one pinned frame per slice" if not big else
                                     f"every slice copied out, into a ring of {ring} pinned frames"}
        del pin_in, pin_out
    plan.close()
    return out


def roofline_of(kstats, c, clk) -> tuple[dict, dict]:
    """Roofline of the kernel with the largest device time in `kstats`, and
    the share table of every kernel."""
    peaks = measured_peaks()
    dname, d = max(kstats.items(), key=lambda kv: kv[1]["ms"])
    per_launch_bytes = d["bytes"] / d["launches"]
    per_launch_ms = d["ms"] / d["launches"]
    achieved = per_launch_bytes / (per_launch_ms / 1e3) / 1e9
    roof = {"bound": "hbm", "kernel": dname, "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
            "frac": achieved / peaks["hbm_gbs"], "peak_source": peaks["source"],
            "traffic": profiled_traffic(dname, c["name"], c["storage"]),
            "bytes_per_launch": per_launch_bytes, "ms_per_launch": per_launch_ms,
            "units_per_s": d["units"] / (d["ms"] / 1e3),
            "onchip": onchip_roof(dname, d, c["storage"], clk or {})}
    tot = max(sum(x["ms"] for x in kstats.values()), 1e-9)
    share = {k: {"launches": v["launches"], "ms": round(v["ms"], 3), "share": round(v["ms"] / tot, 4),
                 "GB_per_s": round(v["bytes"] / max(v["ms"], 1e-9) / 1e6, 1),
                 "Gunits_per_s": round(v["units"] / max(v["ms"], 1e-9) / 1e6, 1)}
             for k, v in kstats.items()}
    return roof, share


def oracle_mid(c, frames, c2r) -> np.ndarray:
    """The FP64 oracle's two middle slices of the series (the checker)."""
    ol = _oracle()
    y0 = c["ny"] // 2
    threads = os.cpu_count() or 1
    if c["method"] == "sart":
        return ol.sart(frames, c["tilts"], c["vol_z"], 0, len(c["tilts"]), c["iters"], c["subsets"],
                       relax=c.get("relax", 0.0), y0=y0, y1=y0 + 2, threads=threads)
    from aretomo3_b200 import recon
    return ol.wbp(frames, c["tilts"], c["vol_z"], y0=y0, y1=y0 + 2, c2r_mode=1 if c2r == recon.C2R_PACKED else 0,
                  threads=threads)


def err_of(got, ref) -> dict:
    g = got.astype(np.float64)
    return {"rel_l2": float(np.linalg.norm(g - ref) / np.linalg.norm(ref)), "max_abs": float(np.abs(g - ref).max()),
            "slices": int(got.shape[0]), "against": "FP64 oracle"}


def reference_cuda(c_sart, c_wbp, frames) -> dict:
    """The reference's own CUDA Recon (CDoWbpRecon::DoIt / CDoSartRecon::DoIt,
    built from its sources for sm_100a into oracle/_ref/ref_recon) against this
    library's reference-shaped entry points (recon.CDoWbpRecon / CDoSartRecon:
    a new plan per call, pageable host frames in and out, as CTiltSeries holds
    them) on a band of rows of the same series (every y-slice is independent):
    wall time of each DoIt (median of three after a warm-up for ours, the
    reference's own timer around its DoIt), and the relative L2 between the two
    volumes."""
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import gen_golden  # noqa: E402  (runs the reference binary)
    from aretomo3_b200 import recon
    if not os.path.exists(gen_golden.REF_BIN):
        return {"unavailable": "oracle/_ref/ref_recon was not built (the reference tree was absent at build time)"}
    out = {}
    for c, rows in ((c_wbp, 256), (c_sart, 32)):
        y0 = c["ny"] // 2 - rows // 2
        band = np.ascontiguousarray(frames[:, y0:y0 + rows, :])
        T, ny, nx = band.shape
        if c["method"] == "sart":
            ref, info = gen_golden.run_reference("sart", band, c["tilts"], c["vol_z"], 0, T, c["iters"], c["subsets"])
        else:
            ref, info = gen_golden.run_reference("wbp", band, c["tilts"], c["vol_z"])
        ts = recon.TiltSeries(band)
        ap = recon.AlignParam(np.asarray(c["tilts"], np.float32))

        def ours():
            if c["method"] == "sart":
                return recon.CDoSartRecon().DoIt(ts, ap, 0, T, c["vol_z"], c["iters"], c["subsets"])
            return recon.CDoWbpRecon().DoIt(ts, ap, c["vol_z"])
        ours()
        times = []
        for _ in range(3):
            t = time.perf_counter()
            vol = ours()
            times.append(time.perf_counter() - t)
        t_ours = float(np.median(times))
        units = float(nx & ~1) * ny * c["vol_z"] * T
        out[c["method"]] = {
            "rows": [int(y0), int(y0 + rows)], "reference_s": info["seconds"], "ours_s": t_ours,
            "reference_value": units / info["seconds"] / 1e9, "ours_value": units / t_ours / 1e9, "unit": UNIT,
            "speedup": info["seconds"] / t_ours,
            "rel_l2_vs_reference": float(np.linalg.norm(vol.astype(np.float64) - ref) /
                                         np.linalg.norm(ref.astype(np.float64)))}
    out["note"] = ("pageable host frames in, host XZ frames out on both sides; the reference's DoIt has no "
                   "relaxation argument (1/subsets), as this workload's SART")
    return out


def run_our_arm(args, c, rank, world, local_rank):
    import torch
    from aretomo3_b200 import synth
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    frames = synth.make_tilt_series(c["nx"], c["ny"], c["tilts"], c["vol_z"], c["phantom"])
    T, ny, nx = frames.shape
    Nx, Nz = nx & ~1, c["vol_z"]
    stream = torch.cuda.current_stream(dev)
    proj = torch.from_numpy(frames).to(dev)
    vol = torch.empty((ny, Nz, Nx), device=dev, dtype=torch.float32)
    gpu_index = _gpu_index(local_rank)
    e2e_steps = args.steps if args.e2e_steps <= 0 else min(args.steps, args.e2e_steps)
    m = measure(c, frames, proj, vol, stream, args.steps, args.warmup, e2e_steps, world, gpu_index)
    clk = m["clocks"]
    sub = {}
    full = rank == 0 and world == 1 and not args.no_cpu_baseline
    if c.get("with_wbp") and world == 1 and not args.primary_only:
        # the metric's WBP half on the same series
        cw = dict(c, method="wbp", name=c["name"] + "_wbp", label=c["wbp_label"])
        w = measure(cw, frames, proj, vol, stream, min(args.steps, 5), 2, min(args.steps, 2), world, gpu_index,
                    clocks=True)
        sub["wbp"] = (cw, w)
    prec = {}
    if c.get("with_precision") and world == 1 and not args.primary_only:
        # the reduced-precision form beside the FP32 path, WBP and SART
        for st in ("f16", "bf16"):
            for meth, base in (("sart", (c, m)), ("wbp", sub.get("wbp"))):
                if base is None:
                    continue
                cc = dict(base[0], storage=st)
                r = measure(cc, frames, proj, vol, stream, min(args.steps, 2 if meth == "sart" else 3), 1, 0,
                            world, gpu_index, instrument=False, clocks=False)
                prec[f"{meth}_{st}"] = (cc, r, base[1])
    if rank != 0:
        return
    roof, share = roofline_of(m["kstats"], c, clk)
    units = units_per_step(c)
    line = {
        "metric": METRIC, "value": m["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": m["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32" if c["storage"] == "f32" else f"{c['storage']}-storage/f32-accumulate",
        "data": "synthetic",
        "config": {"workload": c["label"], "name": c["name"], "storage": c["storage"], "nx": nx, "ny": ny,
                   "tilts": T, "vol_z": Nz, "units_per_step": units, "slab_slices": m["slab_slices"],
                   "step": "one full reconstruction of the series",
                   "l2": f"inputs larger than L2 (projections {frames.nbytes / 1e6:.0f} MB, volume "
                         f"{Nx * Nz * ny * 4 / 1e9:.2f} GB)",
                   "parallelism": f"replicas x{world}"},
        "e2e": m.get("e2e"),
        "gpu_launches": int(m["launches_per_step"] * args.steps),
        "roofline": roof,
        "kernels": share,
        "instrumented": {"ms_per_step": m["instrumented_ms"], "steps": 1,
                         "overhead": m["instrumented_ms"] / m["ms_per_step"] - 1.0,
                         "note": "per-kernel events, one stream; the kernels and roofline come from this step"},
        "clocks": clk,
    }
    refs = {}
    if full:
        threads = os.cpu_count() or 1
        line["cpu_baseline"] = cpu_baseline(c, frames, threads)
        refs["sart" if c["method"] == "sart" else "wbp"] = oracle_mid(c, frames, m["c2r"])
        line["error"] = err_of(m["mid"], refs[c["method"]])
    if "wbp" in sub:
        cw, w = sub["wbp"]
        wroof, wshare = roofline_of(w["kstats"], cw, w["clocks"])
        rec = {"value": w["value"], "unit": UNIT, "ms_per_step": w["ms_per_step"], "steps": min(args.steps, 5),
               "warmup": 2, "workload": cw["label"], "units_per_step": units_per_step(cw),
               "slab_slices": w["slab_slices"], "e2e": w.get("e2e"), "roofline": wroof, "kernels": wshare,
               "gpu_launches": int(w["launches_per_step"] * min(args.steps, 5)), "clocks": w["clocks"]}
        if full:
            refs["wbp"] = oracle_mid(cw, frames, w["c2r"])
            rec["error"] = err_of(w["mid"], refs["wbp"])
            base = dict(cw, storage="f32")
            rec["cpu_baseline"] = cpu_baseline(base, frames, os.cpu_count() or 1)
        line["wbp"] = rec
    if prec:
        pr = {}
        for k, (cc, r, b) in prec.items():
            e = {"value": r["value"], "unit": UNIT, "ms_per_step": r["ms_per_step"],
                 "speedup_vs_f32": r["value"] / b["value"], "storage": cc["storage"],
                 "steps": min(args.steps, 2 if cc["method"] == "sart" else 3), "warmup": 1}
            if cc["method"] in refs:
                e["error"] = err_of(r["mid"], refs[cc["method"]])
                e["error_f32"] = err_of(b["mid"], refs[cc["method"]])
                e["within_1e-3"] = e["error"]["rel_l2"] <= 1e-3
            pr[k] = e
        pr["note"] = ("filtered projections (WBP) or weighted projections and residual (SART) stored as 16-bit "
                      "values with one FP32 scale per (slice, tilt) row; SART also reads a 16-bit shadow of its "
                      "working volume in the forward projection; accumulation FP32; bound 1e-3 relative L2 "
                      "against the FP64 oracle")
        line["precision"] = pr
    if full and c.get("with_reference_cuda") and not args.primary_only:
        cw = sub["wbp"][0] if "wbp" in sub else dict(c, method="wbp")
        line["reference_cuda"] = reference_cuda(c, cw, frames)
    print(json.dumps(line), flush=True)


# --- batched form: many uneven series in one graph launch --------------------
def batch_specs(n, seed=7):
    """Uneven series: nx, ny in {512..2048 step 256}, 31..61 tilts over +-60
    degrees, thickness 128..600."""
    from aretomo3_b200 import synth
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        nx = 512 + 256 * int(rng.integers(0, 7))
        ny = 512 + 256 * int(rng.integers(0, 7))
        nt = int(rng.integers(31, 62))
        vz = int(rng.integers(128, 601))
        ph = synth.Phantom(seed=500 + i, n_ellipsoids=200, n_beads=20)
        out.append(dict(nx=nx, ny=ny, tilts=np.linspace(-60, 60, nt).astype(np.float32), vol_z=vz, phantom=ph))
    return out


def volume_sums(v, chunk=16):
    """Two checksums of a device volume [ny][Nz][Nx]'s bit patterns, slices
    `chunk` at a time: the plain sum of the words, and a position-weighted one
    (each row's sum of word ^ (word >> 11) times the row's index + 1, plus each
    column's sum of words times the column's index + 1), so a moved row or
    column changes it too.  Equal volumes give equal pairs; the pair stands in
    for a copy where memory holds no second volume."""
    import torch
    ny, nz, nx = v.shape
    s1 = torch.zeros((), dtype=torch.int64, device=v.device)
    s2 = torch.zeros((), dtype=torch.int64, device=v.device)
    col_w = torch.arange(1, nx + 1, dtype=torch.int64, device=v.device)
    for y0 in range(0, ny, chunk):
        b = v[y0:y0 + chunk].reshape(-1, nx).view(torch.int32)
        row_w = torch.arange(y0 * nz + 1, y0 * nz + b.shape[0] + 1, dtype=torch.int64, device=v.device)
        s1 += b.sum(dtype=torch.int64)
        s2 += (torch.bitwise_xor(b, b >> 11).sum(dim=1, dtype=torch.int64) * row_w).sum()
        s2 += (b.sum(dim=0, dtype=torch.int64) * col_w).sum()
    return int(s1.item()), int(s2.item())


def run_batch_arm(args):
    import torch
    from aretomo3_b200 import recon, synth
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev)
    specs = batch_specs(args.series)
    st = STORAGE[args.storage]
    # group <= 0: every series resident at once, one graph launch for all; the
    # plans then take slabs of batch_slab slices so that their workspaces fit
    # beside the series and volumes
    group = len(specs) if args.group <= 0 else args.group
    slab = args.batch_slab if group == len(specs) and len(specs) > 16 else 0
    clocks = ClockSampler(0)
    clocks.start()
    tot_units, ms_graph, ms_plain, equal, slabs, launches = 0.0, 0.0, 0.0, True, [], 0
    forms = []
    for g0 in range(0, len(specs), group):
        grp = specs[g0:g0 + group]
        projs, vols, plans = [], [], []
        for c in grp:
            fr = synth.make_tilt_series(c["nx"], c["ny"], c["tilts"], c["vol_z"], c["phantom"])
            projs.append(torch.from_numpy(fr).to(dev))
            del fr
            pl = recon.Plan(c["nx"], c["ny"], c["tilts"], c["vol_z"], method=recon.WBP, storage=st, slab_slices=slab)
            vols.append(torch.empty(pl.volume_shape, device=dev, dtype=torch.float32))
            plans.append(pl)
            tot_units += units_per_step(c)
        for pl, pj, v in zip(plans, projs, vols):
            slabs.append(pl.autotune(pj.data_ptr(), v.data_ptr(), stream.cuda_stream))
        # plain: per-series launches, one after another on one stream
        for _ in range(args.warmup):
            for pl, pj, v in zip(plans, projs, vols):
                pl.run_device(pj.data_ptr(), v.data_ptr(), stream.cuda_stream)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            for pl, pj, v in zip(plans, projs, vols):
                pl.run_device(pj.data_ptr(), v.data_ptr(), stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        ms_plain += e0.elapsed_time(e1)
        launches += sum(pl.last_launches for pl in plans) * args.steps
        ref = [volume_sums(v) for v in vols]
        batch = recon.Batch(plans, [p.data_ptr() for p in projs], [v.data_ptr() for v in vols],
                            branches=args.branches)
        for v in vols:
            v.fill_(float("nan"))
        for _ in range(args.warmup):   # the first run captures the graph
            batch.run(stream.cuda_stream)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            batch.run(stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        ms_graph += e0.elapsed_time(e1)
        equal = equal and all(volume_sums(v) == r for v, r in zip(vols, ref))
        form, mw, mb = batch.mode
        forms.append({"form": form, "waves_ms": mw, "branches_ms": mb})
        batch.close()
        for pl in plans:
            pl.close()
        del projs, vols, ref
        torch.cuda.empty_cache()
    clk = clocks.stop()
    value = tot_units * args.steps / (ms_graph / 1e3) / 1e9
    plain = tot_units * args.steps / (ms_plain / 1e3) / 1e9
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_graph / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if args.storage == "f32" else f"{args.storage}-storage/f32-accumulate",
            "data": "synthetic",
            "config": {"workload": f"batched WBP: {len(specs)} seeded series, nx, ny in 512..2048 step 256, "
                                   f"31..61 tilts over +-60 deg, thickness 128..600; "
                                   + (f"all resident, one CUDA-graph launch for all, {slab}-slice slabs"
                                      if group == len(specs) else
                                      f"groups of {group} resident series, each group one CUDA-graph launch"),
                       "name": "batch_uneven", "storage": args.storage, "series": len(specs),
                       "units_per_step": tot_units,
                       "l2": "inputs larger than L2 (each group holds tens of GB of series and volumes)"},
            "plain_launches": {"value": plain, "unit": UNIT, "ms_per_step": ms_plain / args.steps},
            "speedup_vs_plain": value / plain, "graph_equals_plain": bool(equal),
            "forms": forms,
            "forms_note": ("per group, the form the batch's first run kept after timing one graph launch of each: "
                           "waves = persistent stage kernels over all series, branches = every plan's own "
                           "launches on parallel branches"),
            "autotuned_slabs": {str(k): slabs.count(k) for k in sorted(set(slabs))},
            "compare": "per-series volume checksums (bit-pattern sum and a position-weighted sum), plain vs graph",
            "gpu_launches": int(launches), "clocks": clk}
    print(json.dumps(line), flush=True)


# --- serving form: Poisson arrivals through the request loop ------------------
def serve_pool(n, seed=11):
    """Distinct seeded series the requests draw from: nx, ny in {256..1024
    step 128}, 31..61 tilts over +-60 degrees, thickness 64..300."""
    from aretomo3_b200 import synth
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        nx = 128 * int(rng.integers(2, 9))
        ny = 128 * int(rng.integers(2, 9))
        nt = int(rng.integers(31, 62))
        vz = int(rng.integers(64, 301))
        ph = synth.Phantom(seed=900 + i, n_ellipsoids=150, n_beads=15)
        out.append(dict(nx=nx, ny=ny, tilts=np.linspace(-60, 60, nt).astype(np.float32), vol_z=vz, phantom=ph))
    return out


def serve_once(pool, frames, reqs, arrivals, storage, inflight, budget, out_bufs):
    """Feeds the requests to a server at their arrival times; returns per
    request (latency from arrival, queued) and the makespan."""
    import threading as th
    from aretomo3_b200 import recon
    srv = recon.Server(hbm_budget_bytes=budget, max_inflight=inflight)
    free = list(range(len(out_bufs)))
    cv = th.Condition()
    order = []   # (id, request index, buffer, submit time)
    lat = [None] * len(reqs)
    done_evt = th.Event()

    def waiter():
        k = 0
        while k < len(reqs):
            with cv:
                while k >= len(order):
                    cv.wait()
                rid, i, b, t_sub = order[k]
            _, l, q = srv.wait(rid)
            lat[i] = (t_sub - t0 - arrivals[i] + l, q)
            with cv:
                free.append(b)
                cv.notify_all()
            k += 1
        done_evt.set()

    w = th.Thread(target=waiter, daemon=True)
    t0 = time.perf_counter()
    w.start()
    for i, (pi, sart) in enumerate(reqs):
        c = pool[pi]
        delay = t0 + arrivals[i] - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        with cv:
            while not free:
                cv.wait()
            b = free.pop()
        Nx = c["nx"] & ~1
        out = out_bufs[b][: c["ny"] * c["vol_z"] * Nx].reshape(c["ny"], c["vol_z"], Nx)
        kw = dict(method=1, iterations=10, subsets=5) if sart else dict(method=0)
        rid = srv.submit(frames[pi], c["tilts"], c["vol_z"], out=out, storage=storage, **kw)
        with cv:
            order.append((rid, i, b, time.perf_counter()))
            cv.notify_all()
    done_evt.wait()
    makespan = time.perf_counter() - t0
    srv.close()
    return lat, makespan


def run_serving_arm(args):
    import torch
    from aretomo3_b200 import recon, synth
    torch.cuda.set_device(0)
    pool = serve_pool(args.pool)
    frames = [torch.from_numpy(synth.make_tilt_series(c["nx"], c["ny"], c["tilts"], c["vol_z"], c["phantom"]))
              .pin_memory().numpy() for c in pool]
    rng = np.random.default_rng(12)
    n = args.requests
    reqs = [(int(rng.integers(0, len(pool))), bool(rng.random() < 0.3)) for _ in range(n)]
    arrivals = np.cumsum(rng.exponential(args.interarrival, n))
    arrivals -= arrivals[0]
    vmax = max(c["ny"] * c["vol_z"] * (c["nx"] & ~1) for c in pool)
    out_bufs = [torch.empty(vmax, dtype=torch.float32).pin_memory().numpy() for _ in range(args.out_buffers)]
    units = np.array([units_per_step(pool[pi]) for pi, _ in reqs])
    budget = int(args.hbm_budget_gb * (1 << 30))
    st16 = STORAGE[args.storage]

    def summary(lat, makespan):
        l = np.array([x[0] for x in lat])
        q = np.array([x[1] for x in lat])
        return {"p50_s": float(np.percentile(l, 50)), "p99_s": float(np.percentile(l, 99)),
                "mean_s": float(l.mean()), "max_s": float(l.max()), "queued_p99_s": float(np.percentile(q, 99)),
                "makespan_s": makespan, "GVoxel_tilt_per_s": float(units.sum() / makespan / 1e9),
                "series_per_s": n / makespan}

    # warm: one request of every pool series through each form
    for storage, inflight in ((st16, args.inflight), (STORAGE["f32"], 1)):
        w_reqs = [(i, False) for i in range(len(pool))]
        serve_once(pool, frames, w_reqs, np.zeros(len(pool)), storage, inflight, budget, out_bufs)
    clocks = ClockSampler(0)
    clocks.start()
    res = {}
    zeros = np.zeros(n)
    for name, storage, inflight in (("served", st16, args.inflight), ("plain_fp32", STORAGE["f32"], 1)):
        res[name] = {"arrivals": summary(*serve_once(pool, frames, reqs, arrivals, storage, inflight, budget,
                                                     out_bufs)),
                     "saturated": summary(*serve_once(pool, frames, reqs, zeros, storage, inflight, budget,
                                                      out_bufs))}
    clk = clocks.stop()
    # error against the FP64 oracle on two slices of one WBP and one SART series, each form
    err = {}
    if not args.no_cpu_baseline:
        ol = _oracle()
        k = int(np.argmin([c["nx"] * c["ny"] * c["vol_z"] for c in pool]))
        c = pool[k]
        y0 = c["ny"] // 2
        for meth, kw in (("wbp", dict(method=0)), ("sart", dict(method=1, iterations=10, subsets=5))):
            if meth == "sart":
                ref = ol.sart(frames[k], c["tilts"], c["vol_z"], 0, len(c["tilts"]), 10, 5, y0=y0, y1=y0 + 2)
            else:
                ref = ol.wbp(frames[k], c["tilts"], c["vol_z"], y0=y0, y1=y0 + 2)
            for sname, s in (("served", st16), ("plain_fp32", 0)):
                srv = recon.Server(hbm_budget_bytes=budget, max_inflight=1)
                rid = srv.submit(frames[k], c["tilts"], c["vol_z"], storage=s, **kw)
                vol = srv.wait(rid)[0]
                srv.close()
                got = vol[y0:y0 + 2].astype(np.float64)
                err[f"{meth}_{sname}"] = {"rel_l2": float(np.linalg.norm(got - ref) / np.linalg.norm(ref)),
                                          "max_abs": float(np.abs(got - ref).max())}
    sat = res["served"]["saturated"]["GVoxel_tilt_per_s"]
    line = {"metric": METRIC, "value": sat, "unit": UNIT, "n_gpus": 1, "steps": n, "warmup": len(pool),
            "ms_per_step": res["served"]["saturated"]["makespan_s"] / n * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": f"{args.storage}-storage/f32-accumulate",
            "data": "synthetic",
            "config": {"workload": f"serving: {n} requests over {len(pool)} distinct seeded series (nx, ny in "
                                   f"256..1024 step 128, 31..61 tilts, thickness 64..300), Poisson arrivals "
                                   f"mean {args.interarrival} s (20 s acquisition interval accelerated "
                                   f"{20.0 / args.interarrival:.0f}x), 70% WBP / 30% SART 10 iterations 5 subsets, "
                                   f"{args.storage} storage, {args.inflight} in flight, HBM budget "
                                   f"{args.hbm_budget_gb} GB; host frames in, host volumes out",
                       "name": "serve_mix", "step": "one request"},
            "latency": res["served"]["arrivals"], "saturated": res["served"]["saturated"],
            "plain_fp32": res["plain_fp32"],
            "speedup_vs_plain_fp32": sat / res["plain_fp32"]["saturated"]["GVoxel_tilt_per_s"],
            "p99_below_acquisition_interval": res["served"]["arrivals"]["p99_s"] < 20.0,
            "e2e": {"value": sat, "unit": UNIT, "h2d_bytes_per_step": int(np.mean([frames[pi].nbytes for pi, _ in reqs])),
                    "d2h_bytes_per_step": int(np.mean([4 * pool[pi]["ny"] * pool[pi]["vol_z"] * (pool[pi]["nx"] & ~1)
                                                       for pi, _ in reqs]))},
            "error": err, "clocks": clk}
    print(json.dumps(line), flush=True)


def run_serving_4k_arm(args):
    """Serving at the size of the 4096 x 4096 x 41 series (thickness 1200):
    args.requests requests, 70 % WBP / 30 % SART 10 iterations 5 subsets, in
    16-bit storage (args.storage) against the plain FP32 form served one at a
    time.  Every request reconstructs the seeded series from pinned host
    frames; its volume rows stream into a pinned ring of 64 frames per
    request in flight (an 80.5 GB volume per request does not fit host memory
    twice), so the timing includes every device-to-host copy.  Three
    arrival patterns: all at once (saturated throughput, the sustainable
    arrival rate), Poisson at the 20 s acquisition interval accelerated 100x
    (0.2 s), and Poisson at the real 20 s acquisition interval
    (args.interarrival_slow, args.requests_slow requests), whose p99 is
    stated against that interval."""
    import threading as th
    import torch
    from aretomo3_b200 import recon, synth
    torch.cuda.set_device(0)
    c = synth.precision_4k(seed=3)
    frames = torch.from_numpy(synth.make_tilt_series(c["nx"], c["ny"], c["tilts"], c["vol_z"], c["phantom"])) \
        .pin_memory().numpy()
    T, ny, nx = frames.shape
    Nx, Nz = nx & ~1, c["vol_z"]
    rng = np.random.default_rng(31)
    n = args.requests
    kinds = [bool(rng.random() < 0.3) for _ in range(n)]   # True: SART
    budget = int(args.hbm_budget_gb * (1 << 30))
    rings = [[f for f in torch.empty((64, Nz, Nx), dtype=torch.float32).pin_memory().numpy()]
             for _ in range(args.inflight)]

    def run(arrivals, storage, inflight):
        n = len(arrivals)
        srv = recon.Server(hbm_budget_bytes=budget, max_inflight=inflight)
        free = list(range(len(rings)))
        cv = th.Condition()
        lat = [None] * n
        order = []
        t0 = time.perf_counter()

        def waiter():
            for k in range(n):
                with cv:
                    while k >= len(order):
                        cv.wait()
                    rid, i, b, t_sub = order[k]
                _, l, q = srv.wait(rid)
                lat[i] = (t_sub - t0 - arrivals[i] + l, q)
                with cv:
                    free.append(b)
                    cv.notify_all()

        w = th.Thread(target=waiter, daemon=True)
        w.start()
        for i in range(n):
            delay = t0 + arrivals[i] - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            with cv:
                while not free:
                    cv.wait()
                b = free.pop()
            kw = dict(method=recon.SART, iterations=10, subsets=5) if kinds[i] else dict(method=recon.WBP)
            ring = rings[b]
            rid = srv.submit(frames, c["tilts"], Nz, out_frames=[ring[y % 64] for y in range(ny)],
                             storage=storage, **kw)
            with cv:
                order.append((rid, i, b, time.perf_counter()))
                cv.notify_all()
        w.join()
        makespan = time.perf_counter() - t0
        srv.close()
        l = np.array([x[0] for x in lat])
        q = np.array([x[1] for x in lat])
        return {"p50_s": float(np.percentile(l, 50)), "p99_s": float(np.percentile(l, 99)),
                "mean_s": float(l.mean()), "max_s": float(l.max()), "queued_p99_s": float(np.percentile(q, 99)),
                "makespan_s": makespan, "GVoxel_tilt_per_s": n * units_per_step(c) / makespan / 1e9,
                "series_per_s": n / makespan}

    st16 = STORAGE[args.storage]
    zeros = np.zeros(n)
    run(np.zeros(min(n, 2)), st16, args.inflight)   # warm: plans, kernels, FFT convention
    clocks = ClockSampler(0)
    clocks.start()
    served_sat = run(zeros, st16, args.inflight)
    plain_sat = run(zeros, STORAGE["f32"], 1)
    fast = rng.exponential(0.2, n)
    fast = np.cumsum(fast) - fast[0]
    served_fast = run(fast, st16, args.inflight)
    n_slow = min(n, args.requests_slow)
    slow = rng.exponential(args.interarrival_slow, n_slow)
    slow = np.cumsum(slow) - slow[0]
    served_slow = run(slow, st16, args.inflight)
    clk = clocks.stop()
    sat = served_sat["GVoxel_tilt_per_s"]
    line = {"metric": METRIC, "value": sat, "unit": UNIT, "n_gpus": 1, "steps": n, "warmup": 2,
            "ms_per_step": served_sat["makespan_s"] / n * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": f"{args.storage}-storage/f32-accumulate", "data": "synthetic",
            "config": {"workload": f"serving at 4096x4096x41, thickness 1200: {n} requests, "
                                   f"{sum(kinds)} SART 10 iterations 5 subsets / {n - sum(kinds)} WBP, "
                                   f"{args.storage} storage, {args.inflight} requests active, HBM budget "
                                   f"{args.hbm_budget_gb} GB; pinned host frames in, volume rows streamed into "
                                   f"pinned rings of 64 frames", "name": "serve_4k", "step": "one request"},
            "saturated": served_sat, "plain_fp32_one_at_a_time": plain_sat,
            "speedup_vs_plain_fp32": sat / plain_sat["GVoxel_tilt_per_s"],
            "sustainable_arrival_per_s": served_sat["series_per_s"],
            "poisson_0.2s": served_fast,
            f"poisson_{args.interarrival_slow:g}s": served_slow,
            "p99_below_acquisition_interval": served_slow["p99_s"] < 20.0,
            "e2e": {"value": sat, "unit": UNIT, "h2d_bytes_per_step": int(frames.nbytes),
                    "d2h_bytes_per_step": int(4 * ny * Nz * Nx)},
            "clocks": clk}
    print(json.dumps(line), flush=True)


# --- input stage (aligned + Fourier-binned series) and thickness ------------
STACK_METRIC = "GPixel·tilt/s of raw frames aligned and Fourier-binned (input stage)"
STACK_UNIT = "GPixel·tilt/s"


def stack_workload(name: str, seed: int = 3) -> dict:
    """The 4096 x 4096 x 41 series of the precision workload, aligned as a
    K3-style series: per-tilt shifts of +-20 px, tilt axis 85-87 degrees (x / y
    swapped), seeded random fill; binned by 4 (stack_4k) or measured for
    thickness at binning 20 (thick_4k, pixel size 1)."""
    from aretomo3_b200 import synth
    c = synth.precision_4k(seed=seed)
    rng = np.random.default_rng(seed)
    T = len(c["tilts"])
    c.update(name=name, shifts=rng.uniform(-20, 20, (T, 2)).astype(np.float32),
             axes=rng.uniform(85.0, 87.0, T).astype(np.float32), seed=4242, bin=4.0, pix=1.0)
    if name == "stack_4k":
        c["label"] = ("input stage 4096x4096x41 tilts: shift +-20 px, tilt axis 85-87 deg (x/y swap), random fill, "
                      "Fourier-crop binning 4 -> 1024x1024")
    else:
        c["label"] = ("thickness measurement 4096x4096x41 tilts, pixel size 1: align + bin 20, WBP 204x204, "
                      "plane statistics, edges")
    return c


def stack_bytes_per_tilt(ax, ay, nx, ny, bx, by) -> float:
    """Compulsory DRAM bytes per tilt of the stack's kernels: raw read and
    aligned + mask write (k_corr), mask read (k_fill), aligned read and row
    spectra write (k_bin_r2c), spectra read / cropped write (k_bin_cols),
    cropped read and binned write (k_bin_c2r)."""
    W = ax & ~1
    kx = bx // 2 + 1
    return (4.0 * nx * ny + 4.0 * ax * ay + W * ay) + W * ay + (4.0 * ax * ay + 8.0 * kx * ay) + \
        (8.0 * kx * ay + 8.0 * kx * by) + (8.0 * kx * by + 4.0 * bx * by)


def run_stack_arm(args):
    import torch
    from aretomo3_b200 import recon
    c = stack_workload(args.workload)
    frames = synth_frames(c)
    if args.tilts:
        # a smaller case of the same frames (profiling)
        n = args.tilts
        frames = np.ascontiguousarray(frames[:n])
        c.update(tilts=c["tilts"][:n], shifts=c["shifts"][:n], axes=c["axes"][:n])
        c["label"] += f"; first {n} tilts"
    T, ny, nx = frames.shape
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream()
    if args.workload == "thick_4k":
        return run_thick_arm(args, c, frames)
    st = recon.Stack(nx, ny, T, shifts=c["shifts"], tilt_axes=c["axes"], size_axis=float(c["axes"][0]),
                     seed=c["seed"], bin=c["bin"])
    (ax, ay), (bx, by) = st.aligned_xy, st.binned_xy
    raw = torch.from_numpy(frames).cuda()
    out = torch.empty(st.binned_shape, device="cuda", dtype=torch.float32)
    for _ in range(args.warmup):
        st.run_device(raw.data_ptr(), out.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize()
    clocks = ClockSampler(0)
    clocks.start()
    time.sleep(0.3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        st.run_device(raw.data_ptr(), out.data_ptr(), stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1) / args.steps
    units = float(nx) * ny * T
    dev_out = out.cpu().numpy()
    # e2e through the host entry point: pinned frames in and out
    pin_in = torch.from_numpy(frames).pin_memory()
    pin_out = torch.empty(st.binned_shape, dtype=torch.float32).pin_memory()
    fin = [pin_in[t].numpy() for t in range(T)]
    st.run_host(fin, pin_out.numpy())
    torch.cuda.synchronize()
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    g0.record(stream)
    for _ in range(args.steps):
        st.run_host(fin, pin_out.numpy(), stream.cuda_stream)
    g1.record(stream)
    torch.cuda.synchronize()
    ms_e2e = g0.elapsed_time(g1) / args.steps
    host_ok = bool(np.array_equal(pin_out.numpy(), dev_out))
    # pageable frames, as CTiltSeries holds them
    t = time.perf_counter()
    st.run_host([f for f in frames], np.empty(st.binned_shape, np.float32))
    ms_pageable = (time.perf_counter() - t) * 1e3
    peaks = measured_peaks()
    bpt = stack_bytes_per_tilt(ax, ay, nx, ny, bx, by)
    achieved = bpt * T / (ms / 1e3) / 1e9
    line = {
        "metric": STACK_METRIC, "value": units / (ms / 1e3) / 1e9, "unit": STACK_UNIT, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": c["label"], "name": c["name"], "aligned": [ax, ay], "binned": [bx, by],
                   "l2": "inputs larger than L2 (2.75 GB of frames)"},
        "e2e": {"value": units / (ms_e2e / 1e3) / 1e9, "unit": STACK_UNIT, "ms_per_step": ms_e2e,
                "h2d_bytes_per_step": int(frames.nbytes), "d2h_bytes_per_step": int(4 * T * bx * by),
                "host_equals_device": host_ok, "pageable_ms": ms_pageable},
        "gpu_launches": int(args.steps * 6),
        "roofline": {"bound": "hbm", "kernel": "all stack kernels (k_corr, k_fill, k_fill_mean, k_bin_r2c, "
                                               "k_bin_cols, k_bin_c2r)",
                     "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"], "peak_source": peaks["source"],
                     "traffic": (profiled_traffic("all", "stack_4k", "f32") if c["name"] == "stack_4k" and T == 41
                                 else None),
                     "bytes_per_step": bpt * T},
        "clocks": clk,
    }
    st.close()
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = stack_cpu_baseline(c, frames)
        line["error"] = stack_error(c, frames, dev_out, (ax, ay), (bx, by))
    print(json.dumps(line), flush=True)


def synth_frames(c):
    from aretomo3_b200 import synth
    return synth.make_tilt_series(c["nx"], c["ny"], c["tilts"], c["vol_z"], c["phantom"])


def stack_cpu_baseline(c, frames, n=None):
    """The FP64 oracle's restatement of the stage (the reference's stage is
    GPU-only) on a sample of tilts, one tilt per host thread."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as ol
    threads = os.cpu_count() or 1
    n = n or min(len(c["tilts"]), threads)
    table = np.arange((4096 & ~1) * 4096, dtype=np.int32)[::-1].copy()   # any valid chain table for timing
    t = time.perf_counter()
    ol.stack(frames[:n], shifts=c["shifts"][:n], tilt_axes=c["axes"][:n], size_axis=float(c["axes"][0]),
             table=table, bin=c["bin"], threads=threads)
    dt = time.perf_counter() - t
    units = float(c["nx"]) * c["ny"] * n
    return {"value": units / dt / 1e9, "unit": STACK_UNIT, "cores": threads, "kind": "port",
            "sample": f"{n} of {len(c['tilts'])} tilts, FP64 C++ restatement, one tilt per thread, {dt:.2f} s"}


def stack_error(c, frames, out, aligned_xy, binned_xy, n=2):
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as ol
    from aretomo3_b200 import recon
    T = frames.shape[0]
    st = recon.Stack(c["nx"], c["ny"], T, shifts=c["shifts"], tilt_axes=c["axes"], size_axis=float(c["axes"][0]),
                     seed=c["seed"], bin=c["bin"])
    try:
        table, mode = st.fill_table(), (1 if st.c2r == recon.C2R_PACKED else 0)
    finally:
        st.close()
    ref, _ = ol.stack(frames[:n], shifts=c["shifts"][:n], tilt_axes=c["axes"][:n], size_axis=float(c["axes"][0]),
                      table=table, bin=c["bin"], c2r_mode=mode)
    got = out[:n].astype(np.float64)
    return {"rel_l2": float(np.linalg.norm(got - ref) / np.linalg.norm(ref)), "tilts": n,
            "against": "FP64 oracle (host cos/sin; see tests for the bit-exact pin against the reference)"}


def run_thick_arm(args, c, frames):
    import torch
    from aretomo3_b200 import recon
    T = frames.shape[0]
    ap = recon.AlignParam(tilts=c["tilts"], shifts=c["shifts"], tilt_axes=c["axes"])
    pin = torch.from_numpy(frames).pin_memory()
    ts = recon.TiltSeries(pin.numpy())
    for _ in range(args.warmup):
        recon.CCalcVolThick().DoIt(ts, ap, c["pix"], seed=c["seed"])
    torch.cuda.synchronize()
    t = time.perf_counter()
    for _ in range(args.steps):
        r = recon.CCalcVolThick().DoIt(ts, ap, c["pix"], seed=c["seed"])
    torch.cuda.synchronize()
    ms = (time.perf_counter() - t) / args.steps * 1e3
    units = float(c["nx"]) * c["ny"] * T
    line = {"metric": "thickness measurements/s (CCalcVolThick)", "value": 1e3 / ms, "unit": "series/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": c["label"], "name": c["name"]},
            "e2e": {"value": 1e3 / ms, "unit": "series/s", "h2d_bytes_per_step": int(frames.nbytes),
                    "d2h_bytes_per_step": 4 * (r.result.vol_z - 1)},
            "result": {"edges": list(r.m_aiSampleEdges), "thickness": r.result.thickness,
                       "offset_z": r.result.offset_z, "binning": float(r.m_fBinning)},
            "raw_gpixel_per_s": units / (ms / 1e3) / 1e9}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="recon_4k")
    ap.add_argument("--e2e-steps", type=int, default=3,
                    help="steps of the host-API (e2e) measurement, at most --steps (0: --steps)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--primary-only", action="store_true",
                    help="the line's own measurement only, without the WBP / precision / reference sub-records "
                         "(for profiling runs)")
    ap.add_argument("--storage", default="f32", choices=sorted(STORAGE),
                    help="staged-sinogram storage: f32, or f16 / bf16 with per-tilt scale (FP32 accumulation)")
    ap.add_argument("--slab", type=int, default=0, help="slices per device batch (0: the plan's default)")
    ap.add_argument("--output", default="xzy", choices=["xzy", "xyz"],
                    help="xyz: also time the volume output stage (XY frames, as FlipVol)")
    ap.add_argument("--series", type=int, default=64, help="batch_uneven: number of series")
    ap.add_argument("--group", type=int, default=0,
                    help="batch_uneven: series resident per graph launch (0: all of them, one launch)")
    ap.add_argument("--batch-slab", type=int, default=4,
                    help="batch_uneven with every series resident: slab slices per plan")
    ap.add_argument("--branches", type=int, default=4, help="batch_uneven: parallel graph branches")
    ap.add_argument("--requests", type=int, default=200, help="serve_mix: number of requests")
    ap.add_argument("--pool", type=int, default=16, help="serve_mix: distinct series the requests draw from")
    ap.add_argument("--interarrival", type=float, default=0.2, help="serve_mix: mean Poisson inter-arrival, s")
    ap.add_argument("--interarrival-slow", type=float, default=20.0,
                    help="serve_4k: mean Poisson inter-arrival of the run at the acquisition interval, s")
    ap.add_argument("--requests-slow", type=int, default=6,
                    help="serve_4k: requests of the run at the acquisition interval")
    ap.add_argument("--inflight", type=int, default=4, help="serve_mix: requests on the GPU at once")
    ap.add_argument("--out-buffers", type=int, default=12, help="serve_mix: pinned host volume buffers")
    ap.add_argument("--hbm-budget-gb", type=float, default=150.0, help="serve_mix: HBM admission budget")
    ap.add_argument("--tilts", type=int, default=0, help="stack_4k / thick_4k: first N tilts only (0: all)")
    args = ap.parse_args()
    if args.workload in ("stack_4k", "thick_4k"):
        if args.impl == "reference":
            c = stack_workload(args.workload)
            base = stack_cpu_baseline(c, synth_frames(c))
            print(json.dumps({"impl": "reference", "metric": STACK_METRIC, "value": base["value"], "unit": STACK_UNIT,
                              "n_gpus": 1, "steps": 1, "warmup": 0, "higher_is_better": True, "dtype": "f64",
                              "config": {"workload": c["label"], "name": c["name"]}, "cpu_baseline": base,
                              "e2e": {"value": base["value"], "unit": STACK_UNIT, "h2d_bytes_per_step": 0,
                                      "d2h_bytes_per_step": 0}}), flush=True)
        else:
            run_stack_arm(args)
        return
    if args.impl == "ours" and args.workload == "serve_4k":
        if args.storage == "f32":
            args.storage = "f16"
        run_serving_4k_arm(args)
        return
    if args.impl == "ours" and args.workload in ("batch_uneven", "serve_mix"):
        if args.workload == "batch_uneven":
            run_batch_arm(args)
        else:
            if args.storage == "f32":
                args.storage = "f16"
            run_serving_arm(args)
        return
    from aretomo3_b200 import ranks
    rank, world, local_rank = ranks.rank_env()
    c = workload(args.workload, seed_offset=rank)
    c["storage"] = args.storage
    c["slab"] = args.slab
    if args.storage != "f32":
        c["label"] += f"; {args.storage} storage with per-tilt scale, FP32 accumulation"
    if args.impl == "reference":
        run_reference_arm(args, c, rank, world)
        return
    if world > 1:
        import datetime
        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        run_our_arm(args, c, rank, world, local_rank)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
