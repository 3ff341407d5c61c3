"""Times the reference's own CUDA code for the stages beside reconstruction —
the projection-alignment re-projector (oracle/_ref/ref_reproj), the input
stage and the thickness measurement (oracle/_ref/ref_stack, ref_recon) —
against this implementation's entry points on the same seeded series, on one
GPU.  (The reconstruction itself is timed against the reference's CUDA Recon
by bench.py, in the `reference_cuda` record of its default line.)  Test
infrastructure: it runs on a B200 box,

    python tests/golden/time_reference.py [--only reproj,stack,thick] > reference_timing.json

and prints one JSON line per workload: the reference's wall time (its own
timer), ours through the reference-shaped entry points with the same inputs
(median of three, after one warm-up), and how the results compare.
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


def stack_case():
    """The input stage on the 4096 x 4096 x 41 series of bench.py's stack_4k
    workload: shifts +-20 px, tilt axis 85-87 degrees, random fill, binning 4."""
    p = synth.precision_4k()
    rng = np.random.default_rng(3)
    T = len(p["tilts"])
    return dict(p, name="stack_4k", shifts=rng.uniform(-20, 20, (T, 2)).astype(np.float32),
                axes=rng.uniform(85.0, 87.0, T).astype(np.float32), seed=4242, bin=4.0)


def run_reference_stack_timed(frames, c):
    """oracle/_ref/ref_stack in its timing mode (no copy-out of aligned frames)."""
    import subprocess
    import tempfile
    T, ny, nx = frames.shape
    d = "/dev/shm" if os.path.isdir("/dev/shm") else None
    with tempfile.TemporaryDirectory(dir=d) as td:
        fin, fpar, fout = (os.path.join(td, n) for n in ("in.bin", "par.bin", "out.bin"))
        gen_golden.write_input(fin, frames, c["tilts"])
        with open(fpar, "wb") as f:
            np.array([0, 0], np.int32).tofile(f)
            np.ascontiguousarray(c["shifts"], np.float32).tofile(f)
            np.ascontiguousarray(c["axes"], np.float32).tofile(f)
        r = subprocess.run([gen_golden.STACK_BIN, "stack", fin, fpar, fout, str(c["seed"]), repr(float(c["bin"])),
                            repr(float(c["axes"][0])), "noaligned"], capture_output=True, text=True, check=True)
        info = json.loads([ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1])
        with open(fout, "rb") as f:
            ax, ay, bx, by = np.fromfile(f, dtype=np.int32, count=4)
            binned = np.fromfile(f, dtype=np.float32, count=T * by * bx).reshape(T, by, bx)
    return binned, info


def main_stack():
    if not os.path.exists(gen_golden.STACK_BIN):
        print(json.dumps({"unavailable": "oracle/_ref/ref_stack not built"}))
        return
    c = stack_case()
    frames = synth.make_tilt_series(c["nx"], c["ny"], c["tilts"], c["vol_z"], c["phantom"])
    T, ny, nx = frames.shape
    ref, info = run_reference_stack_timed(frames, c)
    st = recon.Stack(nx, ny, T, shifts=c["shifts"], tilt_axes=c["axes"], size_axis=float(c["axes"][0]),
                     seed=c["seed"], bin=c["bin"])
    try:
        fr = [frames[t] for t in range(T)]
        out = np.empty(st.binned_shape, np.float32)
        st.run_host(fr, out)   # warm-up
        ts = []
        for _ in range(3):
            t = time.perf_counter()
            st.run_host(fr, out)
            ts.append(time.perf_counter() - t)
    finally:
        st.close()
    t_ours = float(np.median(ts))
    err = float(np.linalg.norm(out.astype(np.float64) - ref) / np.linalg.norm(ref.astype(np.float64)))
    print(json.dumps({"workload": c["name"], "shape": [T, ny, nx], "binned": list(ref.shape[1:]),
                      "reference_s": info["seconds"], "ours_s": t_ours, "speedup": info["seconds"] / t_ours,
                      "frames": "pageable host frames on both sides", "rel_l2_vs_reference": err}), flush=True)


def main_thick():
    """CCalcVolThick on the same 4k series (pixel size 1: binning 20): the
    reference's stages (ref_stack at binning 20, ref_recon WBP, ref_stack
    thick) against recon.CCalcVolThick."""
    if not (os.path.exists(gen_golden.STACK_BIN) and os.path.exists(gen_golden.REF_BIN)):
        print(json.dumps({"unavailable": "oracle/_ref/ref_stack or ref_recon not built"}))
        return
    c = stack_case()
    c.update(name="thick_4k", bin=20.0)
    frames = synth.make_tilt_series(c["nx"], c["ny"], c["tilts"], c["vol_z"], c["phantom"])
    T, ny, nx = frames.shape
    binned, info_s = run_reference_stack_timed(frames, c)
    vz = int(binned.shape[2] * 0.8) // 2 * 2
    vol, info_w = gen_golden.run_reference("wbp", binned, c["tilts"], vz)
    t = time.perf_counter()
    _, _, res, info_t = gen_golden.run_reference_thick(gen_golden.flip_vol(vol), np.float32(20.0))
    t_thick_ref = time.perf_counter() - t
    ap = recon.AlignParam(tilts=np.asarray(c["tilts"], np.float32), shifts=c["shifts"], tilt_axes=c["axes"])
    ts_ = recon.TiltSeries(frames)
    recon.CCalcVolThick().DoIt(ts_, ap, 1.0, seed=c["seed"])   # warm-up
    ts = []
    for _ in range(3):
        t = time.perf_counter()
        r = recon.CCalcVolThick().DoIt(ts_, ap, 1.0, seed=c["seed"])
        ts.append(time.perf_counter() - t)
    t_ours = float(np.median(ts))
    t_ref = info_s["seconds"] + info_w["seconds"]
    print(json.dumps({"workload": c["name"], "shape": [T, ny, nx], "reference_s": t_ref,
                      "reference_parts_s": {"stack": info_s["seconds"], "wbp_doit": info_w["seconds"],
                                            "measure_process_wall": t_thick_ref},
                      "ours_s": t_ours, "speedup": t_ref / t_ours,
                      "reference_result": res, "ours_result": [r.result.edges[0], r.result.edges[1],
                                                               r.result.thickness, r.result.offset_z],
                      "frames": "pageable host frames on both sides"}), flush=True)


if __name__ == "__main__":
    import argparse
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", default="reproj,stack,thick")
    parts = set(ap.parse_args().only.split(","))
    if "reproj" in parts:
        main_reproj()
    if "stack" in parts:
        main_stack()
    if "thick" in parts:
        main_thick()
