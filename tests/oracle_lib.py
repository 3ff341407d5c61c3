"""ctypes binding of the CPU oracle (oracle/liboracle.so) for the tests.
Test infrastructure only."""
from __future__ import annotations

import ctypes
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
_lib = None
P = ctypes.c_void_p


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(ROOT, "oracle", "liboracle.so")
        if not os.path.exists(path):
            import subprocess
            subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "-s"], check=True)
        _lib = ctypes.CDLL(path)
        _lib.oracle_sart_f64.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_int, P, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                         ctypes.c_int, ctypes.c_int, P, P, ctypes.c_int]
        _lib.oracle_sart_f32.argtypes = _lib.oracle_sart_f64.argtypes
        _lib.oracle_set_fill_table.argtypes = [P, ctypes.c_int]
    return _lib


def _p(a):
    return a.ctypes.data_as(P)


def wbp(frames, tilts, vol_z, y0=0, y1=None, c2r_mode=0, f32=False, threads=os.cpu_count()):
    frames = np.ascontiguousarray(frames, np.float32)
    tilts = np.ascontiguousarray(tilts, np.float32)
    t, ny, nx = frames.shape
    y1 = ny if y1 is None else y1
    out = np.zeros((y1 - y0, vol_z, nx & ~1), np.float32 if f32 else np.float64)
    L = lib()
    L.oracle_set_c2r_mode(int(c2r_mode))
    fn = L.oracle_wbp_f32 if f32 else L.oracle_wbp_f64
    rc = fn(_p(frames), nx, ny, t, _p(tilts), vol_z, y0, y1, _p(out), threads)
    if rc != 0:
        raise ValueError(f"oracle wbp rc={rc}")
    return out


def sart(frames, tilts, vol_z, start, ntilts, iters, subsets, relax=0.0, y0=0, y1=None, f32=False,
         threads=os.cpu_count(), rfactor=False, fill_table=None):
    """fill_table: the random table of the empty-voxel fill (Nx * vol_z
    entries, as a device plan drew it); None: empty voxels take the mean."""
    frames = np.ascontiguousarray(frames, np.float32)
    tilts = np.ascontiguousarray(tilts, np.float32)
    t, ny, nx = frames.shape
    y1 = ny if y1 is None else y1
    out = np.zeros((y1 - y0, vol_z, nx & ~1), np.float32 if f32 else np.float64)
    rf = np.zeros(2 * max(iters, 1), np.float64)
    L = lib()
    if fill_table is None:
        L.oracle_set_fill_table(None, 0)
    else:
        tab = np.ascontiguousarray(fill_table, np.int32)
        L.oracle_set_fill_table(_p(tab), int(tab.size))
    fn = L.oracle_sart_f32 if f32 else L.oracle_sart_f64
    rc = fn(_p(frames), nx, ny, t, _p(tilts), vol_z, start, ntilts, iters, subsets, relax, y0, y1, _p(out),
            _p(rf), threads)
    L.oracle_set_fill_table(None, 0)
    if rc != 0:
        raise ValueError(f"oracle sart rc={rc}")
    return (out, rf[: 2 * iters].reshape(iters, 2)) if rfactor else out


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def load_golden(name):
    import json
    z = np.load(os.path.join(ROOT, "tests", "golden", name + ".npz"))
    return z["frames"], z["tilts"], z["volume"], json.loads(str(z["meta"]))


def reproj_range(tilts, proj_idx, skip=None):
    tilts = np.ascontiguousarray(tilts, np.float32)
    sk = None if skip is None else np.ascontiguousarray(skip, np.uint8)
    rng = np.zeros(2, np.int32)
    rc = lib().oracle_reproj_range(_p(tilts), _p(sk) if sk is not None else None, tilts.size, int(proj_idx),
                                   _p(rng))
    if rc != 0:
        raise ValueError(f"oracle reproj range rc={rc}")
    return int(rng[0]), int(rng[1])


def reproj(frames, tilts, proj_idx, vol_z, skip=None, threads=os.cpu_count()):
    """Re-projection of tilt proj_idx (FP32 restatement of CCalcReproj + GReproj)."""
    frames = np.ascontiguousarray(frames, np.float32)
    tilts = np.ascontiguousarray(tilts, np.float32)
    t, ny, nx = frames.shape
    sk = None if skip is None else np.ascontiguousarray(skip, np.uint8)
    out = np.zeros((ny, nx), np.float32)
    rc = lib().oracle_reproj_f32(_p(frames), nx, ny, t, _p(tilts), _p(sk) if sk is not None else None,
                                 int(proj_idx), int(vol_z), _p(out), threads)
    if rc != 0:
        raise ValueError(f"oracle reproj rc={rc}")
    return out


# --- input stage and thickness ------------------------------------------------

def stack_sizes(nx, ny, correct=True, size_axis=0.0, bin=1.0):
    s = np.zeros(4, np.int32)
    if lib().oracle_stack_sizes(int(nx), int(ny), int(bool(correct)), ctypes.c_float(size_axis),
                                ctypes.c_float(bin), _p(s)) != 0:
        raise ValueError("oracle stack sizes")
    return (int(s[0]), int(s[1])), (int(s[2]), int(s[3]))


def stack(raw, correct=True, shifts=None, tilt_axes=None, size_axis=0.0, local_params=None, rand_fill=True,
          table=None, bin=1.0, c2r_mode=0, threads=os.cpu_count()):
    """FP64 restatement of the input stage; returns (binned [T][by][bx] f64,
    aligned-and-filled [T][ay][ax] f32)."""
    raw = np.ascontiguousarray(raw, np.float32)
    T, ny, nx = raw.shape
    (ax, ay), (bx, by) = stack_sizes(nx, ny, correct, size_axis, bin)
    out = np.zeros((T, by, bx), np.float64)
    aligned = np.zeros((T, ay, ax), np.float32)
    keep = []

    def arr(a, dt):
        if a is None:
            return None
        a = np.ascontiguousarray(a, dt)
        keep.append(a)
        return _p(a)
    P = 0 if local_params is None else int(np.asarray(local_params).shape[2])
    L = lib()
    L.oracle_set_c2r_mode(int(c2r_mode))
    rc = L.oracle_stack_f64(_p(raw), nx, ny, T, int(bool(correct)), arr(shifts, np.float32),
                            arr(tilt_axes, np.float32), ctypes.c_float(size_axis), P, arr(local_params, np.float32),
                            int(bool(rand_fill)), arr(table, np.int32), ctypes.c_float(bin), _p(out), _p(aligned),
                            int(threads))
    if rc != 0:
        raise ValueError(f"oracle stack rc={rc}")
    return out, aligned


def stack_fill(img, W, table):
    img = np.ascontiguousarray(img, np.float32).copy()
    ay, ax = img.shape
    t = np.ascontiguousarray(table, np.int32)
    if lib().oracle_stack_fill_f32(_p(img), int(W), ax, ay, _p(t)) != 0:
        raise ValueError("oracle fill")
    return img


def thickness_profile(vol):
    """vol [ny][vol_z][Nx] float32 -> plane standard deviations (vol_z - 1)."""
    vol = np.ascontiguousarray(vol, np.float32)
    ny, nz, nx = vol.shape
    out = np.zeros(nz - 1, np.float32)
    if lib().oracle_thickness_profile(_p(vol), nx, ny, nz, _p(out)) != 0:
        raise ValueError("oracle thickness profile")
    return out


def thickness_edges(profile, bin):
    """-> (smoothed profile, (low edge, high edge, thickness, z offset))."""
    p = np.ascontiguousarray(profile, np.float32)
    sm = np.zeros_like(p)
    r = np.zeros(4, np.int32)
    if lib().oracle_thickness_edges(_p(p), p.size, ctypes.c_float(bin), _p(sm), _p(r)) != 0:
        raise ValueError("oracle thickness edges")
    return sm, tuple(int(v) for v in r)


def load_npz(name):
    """A fixture's arrays and its decoded meta."""
    import json
    z = np.load(os.path.join(ROOT, "tests", "golden", name + ".npz"))
    d = {k: z[k] for k in z.files if k != "meta"}
    return d, json.loads(str(z["meta"]))


def golden_exists(name):
    return os.path.exists(os.path.join(ROOT, "tests", "golden", name + ".npz"))


def flip_vol(vol_xzy):
    """CTiltSeries::FlipVol(true): XZ frames [ny][Nz][Nx] -> XY frames [Nz][ny][Nx], z reversed."""
    return np.ascontiguousarray(np.asarray(vol_xzy).transpose(1, 0, 2)[::-1])


def unflip_vol(vol_xyz):
    """Inverse of flip_vol."""
    return np.ascontiguousarray(np.asarray(vol_xyz)[::-1].transpose(1, 0, 2))
