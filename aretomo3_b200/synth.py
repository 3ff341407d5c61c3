"""Seeded synthetic tilt series (ellipsoid + gold-bead phantoms, analytic
projection, Gaussian or Poisson noise) for tests and benchmarks.

The generator is C++ (``csrc/synth.cpp``) so that a seed yields the same bytes
on every machine and thread count.  The workloads below are the standard
shapes: a 512x512x41 WBP series, a 1024x1024x61 SART series, the 4096x4096x41
precision series, and the uneven batch used by the batched launch.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

from ._lib import load_library


class _PhantomSpec(ctypes.Structure):
    _fields_ = [
        ("seed", ctypes.c_uint64),
        ("vol_x", ctypes.c_int), ("vol_y", ctypes.c_int), ("vol_z", ctypes.c_int),
        ("n_ellipsoids", ctypes.c_int),
        ("axis_min", ctypes.c_float), ("axis_max", ctypes.c_float),
        ("dens_min", ctypes.c_float), ("dens_max", ctypes.c_float),
        ("n_beads", ctypes.c_int),
        ("bead_radius", ctypes.c_float), ("bead_density", ctypes.c_float),
        ("noise_kind", ctypes.c_int),
        ("noise_param", ctypes.c_float),
    ]


NOISE_NONE, NOISE_GAUSSIAN, NOISE_POISSON = 0, 1, 2


@dataclass
class Phantom:
    seed: int
    n_ellipsoids: int = 200
    axis_min: float = 5.0
    axis_max: float = 40.0
    dens_min: float = 0.2
    dens_max: float = 1.0
    n_beads: int = 20
    bead_radius: float = 4.0
    bead_density: float = 5.0
    noise_kind: int = NOISE_GAUSSIAN
    noise_param: float = 0.1


def tilt_range(lo: float, hi: float, step: float) -> np.ndarray:
    n = int(round((hi - lo) / step)) + 1
    return (lo + step * np.arange(n)).astype(np.float32)


def make_tilt_series(nx: int, ny: int, tilts_deg, thickness: int, phantom: Phantom) -> np.ndarray:
    """Returns frames[T][ny][nx] float32 of the phantom projected at tilts_deg."""
    lib = load_library("libat3r_synth.so")
    lib.at3r_synth_tilt_series.restype = ctypes.c_int
    tilts = np.ascontiguousarray(np.asarray(tilts_deg, dtype=np.float32))
    out = np.empty((tilts.size, ny, nx), dtype=np.float32)
    sp = _PhantomSpec(
        phantom.seed, nx & ~1, ny, thickness, phantom.n_ellipsoids,
        phantom.axis_min, phantom.axis_max, phantom.dens_min, phantom.dens_max,
        phantom.n_beads, phantom.bead_radius, phantom.bead_density,
        phantom.noise_kind, phantom.noise_param)
    rc = lib.at3r_synth_tilt_series(
        ctypes.byref(sp), tilts.ctypes.data_as(ctypes.c_void_p), ctypes.c_int(tilts.size),
        ctypes.c_int(nx), ctypes.c_int(ny), out.ctypes.data_as(ctypes.c_void_p))
    if rc != 0:
        raise ValueError(f"at3r_synth_tilt_series failed ({rc})")
    return out


# Standard workloads --------------------------------------------------------

def wbp_small(seed: int = 1):
    """512x512 projections, 41 tilts (-60..60 step 3), thickness 128, 200
    ellipsoids + 20 beads, Gaussian noise sigma = 0.1 x mean."""
    tilts = tilt_range(-60, 60, 3)
    ph = Phantom(seed=seed, n_ellipsoids=200, n_beads=20, noise_kind=NOISE_GAUSSIAN, noise_param=0.1)
    return dict(nx=512, ny=512, tilts=tilts, vol_z=128, phantom=ph)


def sart_1k(seed: int = 2):
    """1024x1024 projections, 61 tilts (-60..60 step 2), thickness 300, 500
    ellipsoids + 40 beads, Poisson noise at 50 e-/px; 15 iterations, 5 subsets."""
    tilts = tilt_range(-60, 60, 2)
    ph = Phantom(seed=seed, n_ellipsoids=500, n_beads=40, noise_kind=NOISE_POISSON, noise_param=50.0)
    return dict(nx=1024, ny=1024, tilts=tilts, vol_z=300, phantom=ph, iters=15, subsets=5)


def precision_4k(seed: int = 3):
    """4096x4096 projections, 41 tilts (-60..60 step 3), thickness 1200; the
    phantom of the 1k series scaled by 4 in every length."""
    tilts = tilt_range(-60, 60, 3)
    ph = Phantom(seed=seed, n_ellipsoids=500, axis_min=20.0, axis_max=160.0, n_beads=40,
                 bead_radius=16.0, noise_kind=NOISE_POISSON, noise_param=50.0)
    return dict(nx=4096, ny=4096, tilts=tilts, vol_z=1200, phantom=ph, iters=15, subsets=5)
