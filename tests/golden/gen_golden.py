"""Generates the golden fixtures in this directory by running the reference's
own CUDA Recon (AreTomo3 AreTomo/Recon, compiled for sm_100a from the
reference sources by oracle/ref/build_ref.sh into oracle/_ref/ref_recon) on
seeded synthetic tilt series.  It needs a GPU, so it runs on a B200 box:

    python tests/golden/gen_golden.py --out <dir>

and the resulting ``*.npz`` files are committed here.  Each fixture holds the
input frames, the tilt angles, the reconstruction parameters and the volume
exactly as ``CDoWbpRecon::DoIt`` / ``CDoSartRecon::DoIt`` returned it (one XZ
slice per y, z flipped).  The ``reproj_*`` fixtures hold, in ``volume``, the
re-projection ``CCalcReproj::DoIt`` returned (AreTomo/ProjAlign, built into
oracle/_ref/ref_reproj), [ny][nx].  The ``stack_*`` fixtures hold the
reference's aligned (GCorrPatchShift + fill) and Fourier-binned frames and
its random table for a seeded series (oracle/_ref/ref_stack); the
``thick_*`` fixtures hold CCalcVolThick's plane profile and edges, for a given
volume (``thick_post_*``) and for the whole chain on a seeded series
regenerated from its phantom parameters (``thick_full_*``).
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
STACK_BIN = os.path.join(ROOT, "oracle", "_ref", "ref_stack")


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


SHIM_BIN = os.path.join(ROOT, "oracle", "_ref", "shim_recon")


def run_reference(mode, frames, tilts, vol_z, start=0, ntilts=0, iters=0, subsets=0, fill_seed=None, binary=None):
    """fill_seed: the seed the reference's empty-voxel fill table is drawn
    with (the driver's time()); None: the clock, as in the reference.
    binary: another build of the same driver (SHIM_BIN: the drop-in shim's
    CDoWbpRecon / CDoSartRecon over libat3r); default the reference's."""
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        write_input(fin, frames, tilts)
        args = [binary or REF_BIN, mode, fin, fout, str(vol_z)]
        if mode == "sart":
            args += [str(start), str(ntilts), str(iters), str(subsets)]
        env = dict(os.environ)
        if fill_seed is not None:
            env["REF_FILL_SEED"] = str(int(fill_seed))
        r = subprocess.run(args, capture_output=True, text=True, check=True, env=env)
        line = [ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1]
        return read_output(fout), json.loads(line)


def stack_cases():
    """Input-stage fixtures: seeded frames, shifts, tilt axes, local patches."""
    rng = np.random.default_rng(99)
    c = []

    def case(name, nx, ny, T, shift_only, axes, size_axis, bin, P, seed, vol_z=40):
        tilts = synth.tilt_range(-60, 60, 120.0 / max(T - 1, 1))[:T]
        shifts = rng.uniform(-6, 6, size=(T, 2)).astype(np.float32)
        local = None
        if P:
            local = np.zeros((T, 5, P), np.float32)
            local[:, 0, :] = rng.uniform(-0.4 * nx, 0.4 * nx, size=(T, P))
            local[:, 1, :] = rng.uniform(-0.4 * ny, 0.4 * ny, size=(T, P))
            local[:, 2:4, :] = rng.uniform(-3, 3, size=(T, 2, P))
            local[:, 4, :] = 1.0
            local[:, 4, 0] = 0.5   # a patch the reference skips
        c.append(dict(name=name, nx=nx, ny=ny, tilts=tilts, vol_z=vol_z, phantom=small_phantom(40 + len(c)),
                      shifts=shifts, axes=np.asarray(axes, np.float32), shift_only=shift_only,
                      size_axis=float(size_axis), bin=float(bin), local=local, seed=seed))
    case("stack_shift_128", 128, 96, 5, 1, np.zeros(5), 0.0, 1.0, 0, 12345)
    case("stack_rot_bin2", 128, 128, 5, 0, rng.uniform(2, 8, 5), 5.0, 2.0, 0, 777)
    case("stack_swap_local", 160, 120, 4, 0, rng.uniform(84, 88, 4), 86.0, 2.5, 4, 4242)
    case("stack_odd_bin3", 131, 97, 3, 0, rng.uniform(1, 2, 3), 1.5, 3.0, 0, 31337)
    return c


def run_reference_stack(frames, tilts, c):
    with tempfile.TemporaryDirectory() as td:
        fin, fpar, fout = (os.path.join(td, n) for n in ("in.bin", "par.bin", "out.bin"))
        write_input(fin, frames, tilts)
        T = frames.shape[0]
        P = 0 if c["local"] is None else c["local"].shape[2]
        with open(fpar, "wb") as f:
            np.array([P, c["shift_only"]], np.int32).tofile(f)
            np.ascontiguousarray(c["shifts"], np.float32).tofile(f)
            np.ascontiguousarray(c["axes"], np.float32).reshape(T).tofile(f)
            if P:
                np.ascontiguousarray(c["local"], np.float32).tofile(f)
        r = subprocess.run([STACK_BIN, "stack", fin, fpar, fout, str(c["seed"]), repr(c["bin"]), repr(c["size_axis"])],
                           capture_output=True, text=True, check=True)
        line = [ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1]
        with open(fout, "rb") as f:
            ax, ay, bx, by = np.fromfile(f, dtype=np.int32, count=4)
            aligned = np.fromfile(f, dtype=np.float32, count=T * ay * ax).reshape(T, ay, ax)
            binned = np.fromfile(f, dtype=np.float32, count=T * by * bx).reshape(T, by, bx)
            n = int(np.fromfile(f, dtype=np.int32, count=1)[0])
            table = np.fromfile(f, dtype=np.int32, count=n)
        return aligned, binned, table, json.loads(line)


def run_reference_thick(vol_xyz, bin):
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "vol.bin"), os.path.join(td, "out.bin")
        nz, ny, nx = vol_xyz.shape
        with open(fin, "wb") as f:
            np.array([nx, ny, nz], np.int32).tofile(f)
            np.ascontiguousarray(vol_xyz, np.float32).tofile(f)
        r = subprocess.run([STACK_BIN, "thick", fin, fout, repr(float(bin))], capture_output=True, text=True,
                           check=True)
        line = [ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1]
        with open(fout, "rb") as f:
            hdr = np.fromfile(f, dtype=np.int32, count=5)
            n = int(hdr[0])
            raw = np.fromfile(f, dtype=np.float32, count=n)
            smooth = np.fromfile(f, dtype=np.float32, count=n)
        return raw, smooth, [int(v) for v in hdr[1:]], json.loads(line)


def flip_vol(vol_xzy):
    """CTiltSeries::FlipVol(true): XZ frames [ny][Nz][Nx] -> XY frames [Nz][ny][Nx], z reversed."""
    return np.ascontiguousarray(vol_xzy.transpose(1, 0, 2)[::-1])


def thick_post_volume(seed=5, nx=64, ny=48, nz=100, z0=30, z1=70):
    """A flipped volume [Nz][ny][Nx]: weak noise everywhere, a textured slab in z in [z0, z1)."""
    rng = np.random.default_rng(seed)
    v = rng.normal(0.0, 0.05, size=(nz, ny, nx)).astype(np.float32)
    v[z0:z1] += rng.normal(0.3, 1.0, size=(z1 - z0, ny, nx)).astype(np.float32)
    v += np.linspace(0, 0.2, nx, dtype=np.float32)[None, None, :]
    return v


def thick_full_case():
    """CCalcVolThick on a seeded 1024 x 1024 x 41 series of a 300-pixel slab
    (pixel size 1: binning 20), small shifts, a 1.5-degree tilt axis."""
    rng = np.random.default_rng(2024)
    T = 41
    return dict(name="thick_full_1k", nx=1024, ny=1024, tilts=synth.tilt_range(-60, 60, 3), vol_z=300,
                phantom_seed=77, shifts=rng.uniform(-5, 5, size=(T, 2)).astype(np.float32),
                axes=np.full(T, 1.5, np.float32) + rng.uniform(-0.2, 0.2, T).astype(np.float32), pix=1.0, seed=90210)


def thick_full_phantom(seed):
    return synth.Phantom(seed=seed, n_ellipsoids=300, n_beads=20)


def gen_stack_and_thick(out_dir, only):
    for c in stack_cases():
        if only and c["name"] not in only:
            continue
        frames = synth.make_tilt_series(c["nx"], c["ny"], c["tilts"], c["vol_z"], c["phantom"])
        aligned, binned, table, info = run_reference_stack(frames, c["tilts"], c)
        meta = {k: v for k, v in c.items() if k in ("name", "nx", "ny", "shift_only", "size_axis", "bin", "seed")}
        meta["mode"] = "stack"
        meta["reference_run"] = info
        extra = {} if c["local"] is None else {"local": c["local"]}
        np.savez_compressed(os.path.join(out_dir, c["name"] + ".npz"), frames=frames,
                            tilts=np.asarray(c["tilts"], np.float32), shifts=c["shifts"], axes=c["axes"],
                            aligned=aligned, binned=binned, table=table, meta=json.dumps(meta), **extra)
        print(c["name"], aligned.shape, binned.shape, info)
    if not only or "thick_post_slab" in only:
        v = thick_post_volume()
        raw, smooth, res, info = run_reference_thick(v, 20.0)
        np.savez_compressed(os.path.join(out_dir, "thick_post_slab.npz"), vol_xyz=v, profile=raw,
                            smoothed=smooth, result=np.asarray(res, np.int32),
                            meta=json.dumps({"mode": "thick_post", "bin": 20.0, "reference_run": info}))
        print("thick_post_slab", res, info)
    c = thick_full_case()
    if not only or c["name"] in only:
        frames = synth.make_tilt_series(c["nx"], c["ny"], c["tilts"], c["vol_z"], thick_full_phantom(c["phantom_seed"]))
        binv = max(20.0 / c["pix"], 20.0)
        sc = dict(shifts=c["shifts"], axes=c["axes"], shift_only=0, size_axis=float(c["axes"][0]), bin=binv,
                  local=None, seed=c["seed"])
        _, binned, _, info_s = run_reference_stack(frames, c["tilts"], sc)
        bx = binned.shape[2]
        vz = int(bx * 0.8) // 2 * 2
        vol, info_w = run_reference("wbp", binned, c["tilts"], vz)
        raw, smooth, res, info_t = run_reference_thick(flip_vol(vol), np.float32(binv))
        meta = {"mode": "thick_full", "nx": c["nx"], "ny": c["ny"], "vol_z": c["vol_z"],
                "phantom": {"seed": c["phantom_seed"], "n_ellipsoids": 300, "n_beads": 20}, "pix": c["pix"],
                "seed": c["seed"], "bin": binv, "wbp_vol_z": vz,
                "reference_run": {"stack": info_s, "wbp": info_w, "thick": info_t}}
        np.savez_compressed(os.path.join(out_dir, c["name"] + ".npz"), tilts=np.asarray(c["tilts"], np.float32),
                            shifts=c["shifts"], axes=c["axes"], binned=binned, volume=vol, profile=raw,
                            smoothed=smooth, result=np.asarray(res, np.int32), meta=json.dumps(meta))
        print(c["name"], binned.shape, vol.shape, res, info_t)


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
    gen_stack_and_thick(args.out, only)


if __name__ == "__main__":
    main()
