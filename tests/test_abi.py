"""CPU checks of the C ABI: the library loads, exports every function that
include/at3r.h declares, and rejects invalid geometry before touching a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

from oracle_lib import ROOT


def declared_functions():
    src = open(os.path.join(ROOT, "include", "at3r.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(at3r_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_the_entry_points():
    names = declared_functions()
    for n in ("at3r_plan_create", "at3r_plan_destroy", "at3r_run_device", "at3r_run_host", "at3r_status_str"):
        assert n in names


def test_library_exports_every_declared_function():
    from aretomo3_b200 import recon
    L = recon.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing


def test_status_strings():
    from aretomo3_b200 import recon
    L = recon.lib()
    for s in range(7):
        assert L.at3r_status_str(s)
    assert L.at3r_status_str(0) == b"ok"


@pytest.mark.parametrize("kw", [
    dict(nx=2),                                   # too narrow
    dict(vol_z=1),                                # too thin
    dict(method=7),                               # unknown method
    dict(method=1, subsets=0, iterations=1),      # SART without subsets
    dict(method=1, start_tilt=8, num_tilts=8),    # tilt range outside the series
])
def test_invalid_geometry_is_rejected_without_gpu(kw):
    from aretomo3_b200 import recon
    args = dict(nx=64, ny=4, vol_z=16, method=0, subsets=1)
    args.update(kw)
    tilts = np.linspace(-60, 60, 11).astype(np.float32)
    with pytest.raises(recon.ReconError) as ei:
        recon.Plan(args.pop("nx"), args.pop("ny"), tilts, args.pop("vol_z"), **args)
    assert ei.value.status == 1  # AT3R_ERR_INVALID_ARGUMENT


def test_valid_geometry_without_gpu_reports_no_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from aretomo3_b200 import recon
    with pytest.raises(recon.ReconError) as ei:
        recon.Plan(64, 4, np.linspace(-60, 60, 11), 16)
    assert ei.value.status == 6  # AT3R_ERR_NO_DEVICE


def test_estimate_bytes_without_gpu():
    from aretomo3_b200 import recon
    tilts = np.linspace(-60, 60, 41)
    small = recon.estimate_bytes(256, 64, tilts, 64)
    assert small > 0
    assert recon.estimate_bytes(512, 64, tilts, 128) > small
    # a 4k series holds at least its two host-path slab buffers and the slab workspace
    big = recon.estimate_bytes(4096, 4096, tilts, 1200, method=recon.SART, storage=recon.STORE_F16)
    assert big > 2 * 8 * 4096 * 1200 * 4
    assert recon.estimate_bytes(0, 64, tilts, 64) == 0


def test_reproj_range_matches_oracle_without_gpu():
    """The product's tilt-range choice (CCalcReproj::mFindProjRange) equals
    the oracle's on random tilt sets, skip flags and projection indices."""
    import oracle_lib as ol
    from aretomo3_b200 import recon
    rng = np.random.default_rng(0)
    for _ in range(200):
        T = int(rng.integers(3, 70))
        tilts = np.sort(rng.uniform(rng.uniform(-70, -20), rng.uniform(20, 70), T)).astype(np.float32)
        p = int(rng.integers(0, T))
        skip = (rng.random(T) < 0.15).astype(np.uint8)
        skip[p] = 1
        assert recon.reproj_range(tilts, p, skip) == ol.reproj_range(tilts, p, skip)


@pytest.mark.parametrize("kw", [
    dict(nx=1),                                   # too narrow
    dict(bin=0.5),                                # binning below 1
    dict(local_params=None, num_patches=3),       # patches without parameters
])
def test_invalid_stack_geometry_is_rejected_without_gpu(kw):
    from aretomo3_b200 import recon
    g, keep = recon._stack_geom(64, 48, 3, seed=0)
    for k, v in kw.items():
        setattr(g, k, v if not isinstance(v, float) else float(v))
    h = ctypes.c_void_p()
    rc = recon.lib().at3r_stack_create(ctypes.byref(g), ctypes.byref(h))
    assert rc == 1 and not h.value   # AT3R_ERR_INVALID_ARGUMENT, nothing created


def test_invalid_thickness_arguments_are_rejected_without_gpu():
    from aretomo3_b200 import recon
    g, keep = recon._stack_geom(64, 48, 3, seed=0)
    tilts = np.zeros(3, np.float32)
    frames = [np.zeros((48, 64), np.float32) for _ in range(3)]
    P = ctypes.c_void_p * 3
    r = recon.ThicknessResult()
    L = recon.lib()
    # pixel size 0
    assert L.at3r_thickness_host(ctypes.byref(g), tilts.ctypes.data, 0.0, P(*[f.ctypes.data for f in frames]),
                                 None, None, 0, ctypes.byref(r), None) == 1
    # a missing frame
    assert L.at3r_thickness_host(ctypes.byref(g), tilts.ctypes.data, 1.0, P(frames[0].ctypes.data, None, None),
                                 None, None, 0, ctypes.byref(r), None) == 1


def test_stack_without_gpu_reports_no_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from aretomo3_b200 import recon
    with pytest.raises(recon.ReconError) as ei:
        recon.Stack(64, 48, 3, seed=0)
    assert ei.value.status == 6  # AT3R_ERR_NO_DEVICE


def test_corr_tomo_stack_mirror_refuses_paths_that_are_not_built():
    from aretomo3_b200 import recon
    c = recon.CCorrTomoStack()
    with pytest.raises(NotImplementedError):
        c.Set2(2.0, False, True)       # real-space binning (GBinImage2D)
    with pytest.raises(NotImplementedError):
        c.Set3(False, False, True)     # R-weighted corrected stack


def test_thickness_pixel_size_follows_the_reference_arithmetic():
    from aretomo3_b200 import recon
    # 4096 x 4096 at 1 A, binning 20 -> 204 x 204: (1 * 4096/204) / 20
    assert recon.thickness_pixel_size(1.0, 4096, 4096, 1.5, 204, 20.0) == np.float32(
        np.float32(np.float32(4096) / np.float32(204)) / np.float32(20))
    # an axis near 90 degrees sizes y by the raw x
    assert recon.thickness_pixel_size(0.8, 5760, 4092, 86.0, 286, 25.0) == np.float32(
        np.float32(np.float32(0.8) * (np.float32(5760) / np.float32(286))) / np.float32(25))
