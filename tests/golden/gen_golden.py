"""Generates the golden fixtures in this directory by running the reference's
own CUDA Recon (AreTomo3 AreTomo/Recon, compiled for sm_100a from the
reference sources by oracle/ref/build_ref.sh into oracle/_ref/ref_recon) on
seeded synthetic tilt series.  It needs a GPU, so it runs on a B200 box:

    python tests/golden/gen_golden.py --out gpurun_out/golden

and the resulting ``*.npz`` files are committed here.  Each fixture holds the
input frames, the tilt angles, the reconstruction parameters and the volume
exactly as ``CDoWbpRecon::DoIt`` / ``CDoSartRecon::DoIt`` returned it (one XZ
slice per y, z flipped).  The ``reproj_*`` fixtures hold, in ``volume``, the
re-projection ``CCalcReproj::DoIt`` returned (AreTomo/ProjAlign, built into
oracle/_ref/ref_reproj), [ny][nx].
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from aretomo3_b200 import synth  # noqa: E402

REF_BIN = os.path.join(ROOT, "oracle", "_ref", "ref_recon")
REPROJ_BIN = os.path.join(ROOT, "oracle", "_ref", "ref_reproj")


def small_phantom(seed, noise_kind=synth.NOISE_GAUSSIAN, noise_param=0.1):
    return synth.Phantom(seed=seed, n_ellipsoids=40, axis_min=3, axis_max=14, n_beads=4,
                         bead_radius=2.0, bead_density=5.0, noise_kind=noise_kind, noise_param=noise_param)


def cases():
    t41 = synth.tilt_range(-60, 60, 3)
    t61 = synth.tilt_range(-60, 60, 2)
    t31 = synth.tilt_range(-60, 60, 4) + np.float32(1.3)  # alpha offset folded in
    c = []
    c.append(dict(name="wbp_128", mode="wbp", nx=128, ny=4, tilts=t41, vol_z=48, phantom=small_phantom(11)))
    c.append(dict(name="wbp_odd97", mode="wbp", nx=97, ny=3, tilts=t31, vol_z=37, phantom=small_phantom(12)))
    c.append(dict(name="wbp_160", mode="wbp", nx=160, ny=2, tilts=t61, vol_z=100, phantom=small_phantom(13)))
    c.append(dict(name="sart_128", mode="sart", nx=128, ny=4, tilts=t41, vol_z=48, phantom=small_phantom(21),
                  start=0, ntilts=41, iters=3, subsets=5))
    c.append(dict(name="sart_odd97", mode="sart", nx=97, ny=3, tilts=t31, vol_z=37, phantom=small_phantom(22),
                  start=3, ntilts=24, iters=2, subsets=4))
    # Two rows of the 512x512x41 WBP series and one row of the 1024x1024x61
    # SART series: every y-slice depends only on its own projection rows, so
    # these equal the corresponding slices of the full reconstructions.
    w = synth.wbp_small()
    c.append(dict(name="wbp_512_rows", mode="wbp", nx=512, ny=512, tilts=w["tilts"], vol_z=128,
                  phantom=w["phantom"], rows=(255, 257)))
    s = synth.sart_1k()
    c.append(dict(name="sart_1k_row", mode="sart", nx=1024, ny=1024, tilts=s["tilts"], vol_z=300,
                  phantom=s["phantom"], start=0, ntilts=61, iters=15, subsets=5, rows=(511, 512)))
    return c


def reproj_cases():
    """Re-projection fixtures: seeded series, the tilt re-projected is marked
    skipped as CProjAlignMain::mCalcReproj does."""
    t41 = synth.tilt_range(-60, 60, 3)
    t31 = synth.tilt_range(-60, 60, 4) + np.float32(0.7)
    c = []
    c.append(dict(name="reproj_128_mid", nx=128, ny=6, tilts=t41, vol_z=48, phantom=small_phantom(31), proj=20))
    c.append(dict(name="reproj_128_high", nx=128, ny=5, tilts=t41, vol_z=64, phantom=small_phantom(32), proj=3))
    c.append(dict(name="reproj_97_end", nx=97, ny=4, tilts=t31, vol_z=37, phantom=small_phantom(33), proj=30))
    return c


def run_reference_reproj(frames, tilts, vol_z, proj):
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        write_input(fin, frames, tilts)
        r = subprocess.run([REPROJ_BIN, fin, fout, str(vol_z), str(proj)], capture_output=True, text=True,
                           check=True)
        line = [ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1]
        with open(fout, "rb") as f:
            nx, ny = np.fromfile(f, dtype=np.int32, count=2)
            out = np.fromfile(f, dtype=np.float32).reshape(ny, nx)
        return out, json.loads(line)


def write_input(path, frames, tilts):
    t, ny, nx = frames.shape
    with open(path, "wb") as f:
        np.array([nx, ny, t], dtype=np.int32).tofile(f)
        np.asarray(tilts, dtype=np.float32).tofile(f)
        np.ascontiguousarray(frames, dtype=np.float32).tofile(f)


def read_output(path):
    with open(path, "rb") as f:
        nx, nz, ny = np.fromfile(f, dtype=np.int32, count=3)
        vol = np.fromfile(f, dtype=np.float32).reshape(ny, nz, nx)
    return vol


def run_reference(mode, frames, tilts, vol_z, start=0, ntilts=0, iters=0, subsets=0):
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        write_input(fin, frames, tilts)
        args = [REF_BIN, mode, fin, fout, str(vol_z)]
        if mode == "sart":
            args += [str(start), str(ntilts), str(iters), str(subsets)]
        r = subprocess.run(args, capture_output=True, text=True, check=True)
        line = [ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1]
        return read_output(fout), json.loads(line)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "tests", "golden"))
    ap.add_argument("--only", default="", help="comma-separated fixture names (default: all)")
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    only = set(filter(None, args.only.split(",")))
    for c in cases():
        if only and c["name"] not in only:
            continue
        frames = synth.make_tilt_series(c["nx"], c["ny"], c["tilts"], c["vol_z"], c["phantom"])
        if "rows" in c:
            r0, r1 = c["rows"]
            frames = np.ascontiguousarray(frames[:, r0:r1, :])
        vol, info = run_reference(c["mode"], frames, c["tilts"], c["vol_z"], c.get("start", 0),
                                  c.get("ntilts", 0), c.get("iters", 0), c.get("subsets", 0))
        meta = {k: v for k, v in c.items() if k not in ("tilts", "phantom")}
        meta["reference_run"] = info
        np.savez_compressed(os.path.join(args.out, c["name"] + ".npz"), frames=frames,
                            tilts=np.asarray(c["tilts"], np.float32), volume=vol,
                            meta=json.dumps(meta))
        print(c["name"], vol.shape, info)
    for c in reproj_cases():
        if only and c["name"] not in only:
            continue
        frames = synth.make_tilt_series(c["nx"], c["ny"], c["tilts"], c["vol_z"], c["phantom"])
        out, info = run_reference_reproj(frames, c["tilts"], c["vol_z"], c["proj"])
        meta = {k: v for k, v in c.items() if k not in ("tilts", "phantom")}
        meta["mode"] = "reproj"
        meta["reference_run"] = info
        np.savez_compressed(os.path.join(args.out, c["name"] + ".npz"), frames=frames,
                            tilts=np.asarray(c["tilts"], np.float32), volume=out, meta=json.dumps(meta))
        print(c["name"], out.shape, info)


if __name__ == "__main__":
    main()
