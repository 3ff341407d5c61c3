"""Times the reference's own CUDA Recon (oracle/_ref/ref_recon, built from the
reference sources for sm_100a) against this implementation's host-path entry
points on the same seeded series, on one GPU.  Test infrastructure: it runs
on a B200 box,

    python tests/golden/time_reference.py > gpurun_out/reference_timing.json

and prints one JSON line per workload: the reference's DoIt wall time (host
frames in, host XZ frames out, its own timer around DoIt), ours through
CDoWbpRecon().DoIt / CDoSartRecon().DoIt with the same inputs (median of
three, after one warm-up), and the relative L2 between the two volumes.
Rows: the 4k series is timed on a band of rows (every y-slice is
independent), and the rate is per output voxel*tilt.
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import gen_golden  # noqa: E402
from gen_golden import ROOT, run_reference  # noqa: E402, F401

from aretomo3_b200 import recon, synth  # noqa: E402


def workloads():
    w = synth.wbp_small()
    yield dict(w, name="wbp_512", mode="wbp")
    s = synth.sart_1k()
    yield dict(s, name="sart_1k", mode="sart", start=0, ntilts=61)
    p = synth.precision_4k()
    yield dict(p, name="wbp_4k_rows", mode="wbp", rows=(1920, 2176))
    yield dict(p, name="sart_4k_rows", mode="sart", start=0, ntilts=41, rows=(2032, 2064))


def ours(c, frames):
    ts = recon.TiltSeries(frames)
    ap = recon.AlignParam(np.asarray(c["tilts"], np.float32))
    if c["mode"] == "wbp":
        return recon.CDoWbpRecon().DoIt(ts, ap, c["vol_z"])
    return recon.CDoSartRecon().DoIt(ts, ap, c["start"], c["ntilts"], c["vol_z"], c["iters"], c["subsets"])


def main():
    if not os.path.exists(gen_golden.REF_BIN):
        print(json.dumps({"unavailable": "oracle/_ref/ref_recon not built"}))
        return
    for c in workloads():
        frames = synth.make_tilt_series(c["nx"], c["ny"], c["tilts"], c["vol_z"], c["phantom"])
        if "rows" in c:
            r0, r1 = c["rows"]
            frames = np.ascontiguousarray(frames[:, r0:r1, :])
        ref, info = run_reference(c["mode"], frames, c["tilts"], c["vol_z"], c.get("start", 0), c.get("ntilts", 0),
                                  c.get("iters", 0), c.get("subsets", 0))
        ours(c, frames)   # warm-up (plan set-up, module load)
        ts = []
        for _ in range(3):
            t = time.perf_counter()
            vol = ours(c, frames)
            ts.append(time.perf_counter() - t)
        t_ours = float(np.median(ts))
        T, ny, nx = frames.shape
        units = float(nx & ~1) * ny * c["vol_z"] * T
        rel = float(np.linalg.norm(vol.astype(np.float64) - ref) / np.linalg.norm(ref.astype(np.float64)))
        print(json.dumps({"workload": c["name"], "shape": [T, ny, nx], "vol_z": c["vol_z"],
                          "reference_s": info["seconds"], "ours_s": t_ours,
                          "reference_GVoxel_tilt_per_s": units / info["seconds"] / 1e9,
                          "ours_GVoxel_tilt_per_s": units / t_ours / 1e9,
                          "speedup": info["seconds"] / t_ours, "rel_l2_vs_reference": rel}), flush=True)


def reproj_workloads():
    """The projection-alignment re-projector on a 1024 x 1024 x 61 binned
    stack, alignment thickness 300, at a low and a high tilt."""
    s = synth.sart_1k()
    for proj in (30, 5):
        yield dict(s, name=f"reproj_1k_t{proj}", proj=proj)


def main_reproj():
    if not os.path.exists(gen_golden.REPROJ_BIN):
        print(json.dumps({"unavailable": "oracle/_ref/ref_reproj not built"}))
        return
    for c in reproj_workloads():
        frames = synth.make_tilt_series(c["nx"], c["ny"], c["tilts"], c["vol_z"], c["phantom"])
        ref, info = gen_golden.run_reference_reproj(frames, c["tilts"], c["vol_z"], c["proj"])
        T, ny, nx = frames.shape
        skip = np.zeros(T, np.uint8)
        skip[c["proj"]] = 1
        calc = recon.CCalcReproj()
        calc.Setup((nx, ny, T), c["vol_z"])
        fr = [frames[t] for t in range(T)]
        calc.DoIt(fr, c["tilts"], skip, c["proj"])   # warm-up
        ts = []
        for _ in range(3):
            t = time.perf_counter()
            got = calc.DoIt(fr, c["tilts"], skip, c["proj"])
            ts.append(time.perf_counter() - t)
        t_ours = float(np.median(ts))
        print(json.dumps({"workload": c["name"], "shape": [T, ny, nx], "vol_z": c["vol_z"], "proj": c["proj"],
                          "reference_s": info["seconds"], "ours_s": t_ours, "speedup": info["seconds"] / t_ours,
                          "bit_identical": bool(np.array_equal(got, ref))}), flush=True)


if __name__ == "__main__":
    main()
    main_reproj()
