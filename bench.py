#!/usr/bin/env python
"""Benchmark of the reconstruction path on B200.

Default workload (one GPU): SART on the seeded 1024 x 1024 x 61-tilt series
(-60..60 step 2, thickness 300, 500 ellipsoids + 40 beads, Poisson noise at
50 e-/px), 15 iterations, 5 subsets, relaxation 0.3.  A "step" is one full
reconstruction of that series.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

Metric: GVoxel*tilt/s = Nx * ny * Nz * T of the output grid per second (the
same count for WBP and SART; SART's iterations are work inside a step).

* value    : device-resident (projections already in HBM), CUDA events on the
             launching stream, max over ranks.  Inputs (256 MB of projections,
             1.26 GB of volume) exceed the 126 MB L2.
* e2e      : the same through the host API (at3r_run_host): pinned host
             frames in, host volume frames out, copies inside the timed region.
* roofline : the kernel with the largest device time, its algorithmic bytes
             per launch / its mean launch time (CUDA events around every
             launch on its stream, during a timed step), against the measured
             HBM copy bandwidth.
* cpu_baseline : the FP32 C++ port of the same math (oracle/, OpenMP over
             y-slices) on the host cores, on a sample of the series' slices.

With --impl reference the same workload is timed on the host cores by the
FP32 port, rank 0 only (the reference's Recon has no CPU implementation).
N > 1: torchrun, one process per GPU, each rank reconstructs its own series
(weak scaling, no collective on the data path).
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
    elif name == "sart_4k":
        c = synth.precision_4k(seed=3 + seed_offset)
        c.update(method="sart", relax=0.0, label="SART 4096x4096x41 tilts, thickness 1200, 15 iterations, 5 subsets")
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
    if c["method"] == "sart":
        return dict(method=recon.SART, start_tilt=0, num_tilts=len(c["tilts"]), iterations=c["iters"],
                    subsets=c["subsets"], relax=c.get("relax", 0.0), storage=st)
    return dict(method=recon.WBP, storage=st)


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


def profiled_traffic(kernel: str, workload_name: str):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    d = json.load(open(p))
    return d.get(workload_name, {}).get(kernel)


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


def error_vs_oracle(c, frames, vol_gpu, n_slices=2) -> dict:
    """Relative L2 / max-abs of the GPU volume against the FP64 oracle on a few
    slices (the checker)."""
    ol = _oracle()
    y0 = c["ny"] // 2
    if c["method"] == "sart":
        ref = ol.sart(frames, c["tilts"], c["vol_z"], 0, len(c["tilts"]), c["iters"], c["subsets"],
                      relax=c.get("relax", 0.0), y0=y0, y1=y0 + n_slices)
    else:
        from aretomo3_b200 import recon
        mode = 1 if c.get("_c2r") == recon.C2R_PACKED else 0
        ref = ol.wbp(frames, c["tilts"], c["vol_z"], y0=y0, y1=y0 + n_slices, c2r_mode=mode)
    got = vol_gpu[y0:y0 + n_slices].astype(np.float64)
    return {"rel_l2": float(np.linalg.norm(got - ref) / np.linalg.norm(ref)),
            "max_abs": float(np.abs(got - ref).max()), "slices": n_slices, "against": "FP64 oracle"}


def run_reference_arm(args, c, rank, world):
    if rank != 0:
        return
    from aretomo3_b200 import synth
    frames = synth.make_tilt_series(c["nx"], c["ny"], c["tilts"], c["vol_z"], c["phantom"])
    threads = os.cpu_count() or 1
    s = min(max(4, cpu_sample_slices(c) // 3), c["ny"])
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


def run_our_arm(args, c, rank, world, local_rank):
    import torch
    from aretomo3_b200 import recon, synth
    dist = world > 1
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    frames = synth.make_tilt_series(c["nx"], c["ny"], c["tilts"], c["vol_z"], c["phantom"])
    T, ny, nx = frames.shape
    Nx, Nz = nx & ~1, c["vol_z"]
    plan = recon.Plan(nx, ny, c["tilts"], Nz, **plan_kwargs(c))
    c["_c2r"] = plan.c2r
    stream = torch.cuda.current_stream(dev)
    proj = torch.from_numpy(frames).to(dev)
    vol = torch.empty((ny, Nz, Nx), device=dev, dtype=torch.float32)

    def barrier():
        if dist:
            torch.distributed.barrier()

    def max_over_ranks(x: float) -> float:
        if not dist:
            return x
        t = torch.tensor([x], device=dev, dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return float(t.item())

    for _ in range(args.warmup):
        plan.run_device(proj.data_ptr(), vol.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize()

    # timed region: device-resident, per-kernel events on the launching stream
    plan.set_timing(True)
    gpu_index = int(os.environ.get("CUDA_VISIBLE_DEVICES", str(local_rank)).split(",")[local_rank]) \
        if os.environ.get("CUDA_VISIBLE_DEVICES", "").replace(",", "").isdigit() else local_rank
    clocks = ClockSampler(gpu_index)
    clocks.start()
    time.sleep(0.3)
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        plan.run_device(proj.data_ptr(), vol.data_ptr(), stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms_total = max_over_ranks(e0.elapsed_time(e1))
    clk = clocks.stop()
    kstats = plan.kernel_stats()   # the last timed step
    launches_per_step = plan.last_launches
    plan.set_timing(False)

    # same steps without per-launch events (overhead of the instrumentation)
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(args.steps):
        plan.run_device(proj.data_ptr(), vol.data_ptr(), stream.cuda_stream)
    f1.record(stream)
    torch.cuda.synchronize()
    ms_plain = max_over_ranks(f0.elapsed_time(f1))
    vol_host = vol.cpu().numpy() if rank == 0 else None

    # e2e through the host API: pinned frames in, pinned volume frames out
    pin_in = torch.from_numpy(frames).pin_memory()
    pin_out = torch.empty((ny, Nz, Nx), dtype=torch.float32).pin_memory()
    fin = [pin_in[t].numpy() for t in range(T)]
    fout = [pin_out[y].numpy() for y in range(ny)]
    plan.run_host(fin, fout, stream.cuda_stream)  # warm the host-path buffers
    torch.cuda.synchronize()
    barrier()
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    g0.record(stream)
    for _ in range(args.steps):
        plan.run_host(fin, fout, stream.cuda_stream)
    g1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms_e2e = max_over_ranks(g0.elapsed_time(g1))
    host_ok = bool(np.array_equal(pin_out.numpy(), vol_host)) if rank == 0 else True

    units = units_per_step(c)
    value = units * args.steps * world / (ms_total / 1e3) / 1e9
    e2e_value = units * args.steps * world / (ms_e2e / 1e3) / 1e9

    if rank != 0:
        return
    # roofline of the dominant kernel
    peaks = measured_peaks()
    dom = max(kstats.items(), key=lambda kv: kv[1]["ms"])
    dname, d = dom
    per_launch_bytes = d["bytes"] / d["launches"]
    per_launch_ms = d["ms"] / d["launches"]
    achieved = per_launch_bytes / (per_launch_ms / 1e3) / 1e9
    roof = {"bound": "hbm", "kernel": dname, "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
            "frac": achieved / peaks["hbm_gbs"], "peak_source": peaks["source"],
            "traffic": profiled_traffic(dname, c["name"]),
            "bytes_per_launch": per_launch_bytes, "ms_per_launch": per_launch_ms,
            "units_per_s": d["units"] / (d["ms"] / 1e3)}
    step_ms = ms_total / args.steps
    kernel_share = {k: {"launches": v["launches"], "ms": round(v["ms"], 3),
                        "share": round(v["ms"] / max(sum(x["ms"] for x in kstats.values()), 1e-9), 4),
                        "GB_per_s": round(v["bytes"] / max(v["ms"], 1e-9) / 1e6, 1),
                        "Gunits_per_s": round(v["units"] / max(v["ms"], 1e-9) / 1e6, 1)}
                    for k, v in kstats.items()}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32" if c["storage"] == "f32" else f"{c['storage']}-storage/f32-accumulate",
        "data": "synthetic",
        "config": {"workload": c["label"], "name": c["name"], "storage": c["storage"], "nx": nx, "ny": ny, "tilts": T, "vol_z": Nz,
                   "units_per_step": units, "slab_slices": plan.geom.slab_slices or "auto",
                   "l2": "inputs larger than L2 (projections 256 MB, volume 1.26 GB at the default workload)",
                   "parallelism": f"replicas x{world}"},
        "e2e": {"value": e2e_value, "unit": UNIT, "ms_per_step": ms_e2e / args.steps,
                "h2d_bytes_per_step": int(frames.nbytes), "d2h_bytes_per_step": int(Nx * Nz * ny * 4),
                "host_equals_device": host_ok},
        "gpu_launches": int(launches_per_step * args.steps),
        "roofline": roof,
        "kernels": kernel_share,
        "timing_overhead": (ms_total - ms_plain) / ms_plain,
        "clocks": clk,
    }
    if not args.no_cpu_baseline and world == 1:
        threads = os.cpu_count() or 1
        line["cpu_baseline"] = cpu_baseline(c, frames, threads)
        line["error"] = error_vs_oracle(c, frames, vol_host)
    print(json.dumps(line), flush=True)
    plan.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="sart_1k")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--storage", default="f32", choices=sorted(STORAGE),
                    help="staged-sinogram storage: f32, or f16 / bf16 with per-tilt scale (FP32 accumulation)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    c = workload(args.workload, seed_offset=rank)
    c["storage"] = args.storage
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
