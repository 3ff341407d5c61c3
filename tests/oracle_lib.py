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
         threads=os.cpu_count(), rfactor=False):
    frames = np.ascontiguousarray(frames, np.float32)
    tilts = np.ascontiguousarray(tilts, np.float32)
    t, ny, nx = frames.shape
    y1 = ny if y1 is None else y1
    out = np.zeros((y1 - y0, vol_z, nx & ~1), np.float32 if f32 else np.float64)
    rf = np.zeros(2 * max(iters, 1), np.float64)
    L = lib()
    fn = L.oracle_sart_f32 if f32 else L.oracle_sart_f64
    rc = fn(_p(frames), nx, ny, t, _p(tilts), vol_z, start, ntilts, iters, subsets, relax, y0, y1, _p(out),
            _p(rf), threads)
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
