"""The no-allocation SART entry point (at3r_sart_device_noalloc) against the
plan-based one (at3r_plan_create + at3r_run_device), through the C ABI.

at3r_sart_device_noalloc serves callers that cannot allocate device memory
while they reconstruct (an application whose allocator already holds the
device's memory, or a pipeline whose other in-flight work a cudaMalloc or
cudaFree would stall): its scratch is a fixed 16 MiB array inside the
library.  Two calls in a row — a larger series, then a smaller one, so the
second reuses scratch the first left behind — must each match the plan-based
result within the tests' FP32 tolerance.  This file is collected last and
also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-4  # relative L2, as the other FP32 parity tests


def _noalloc(L):
    fn = L.at3r_sart_device_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                   ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_void_p,
                   ctypes.c_void_p]
    return fn


def _series(nx, ny, tilts, vol_z, seed):
    from aretomo3_b200 import synth
    ph = synth.Phantom(seed=seed, n_ellipsoids=80, axis_min=3, axis_max=20, n_beads=6, bead_radius=3,
                       noise_kind=synth.NOISE_POISSON, noise_param=50.0)
    return synth.make_tilt_series(nx, ny, tilts, vol_z, ph)


def test_noalloc_sart_matches_plan_path_twice():
    import torch
    assert torch.cuda.is_available(), "needs a CUDA device"
    from aretomo3_b200 import recon
    L = recon.lib()
    fn = _noalloc(L)
    cases = [
        # (nx, ny, tilts, vol_z, start, num, iters, subsets, relax): the first needs several slabs of scratch
        (1024, 96, np.linspace(-60, 60, 61).astype(np.float32), 300, 0, 61, 4, 5, 0.0),
        (256, 9, np.linspace(-57, 62, 31).astype(np.float32), 64, 3, 25, 3, 4, 0.3),
    ]
    stream = torch.cuda.current_stream()
    for i, (nx, ny, tilts, vz, start, num, iters, subsets, relax) in enumerate(cases):
        frames = _series(nx, ny, tilts, vz, seed=100 + i)
        proj = torch.from_numpy(frames).cuda()
        ref, plan = recon.reconstruct_device(proj, tilts, vz, method=recon.SART, start_tilt=start, num_tilts=num,
                                             iterations=iters, subsets=subsets, relax=relax)
        out = torch.full_like(ref, float("nan"))
        rc = fn(proj.data_ptr(), nx, ny, tilts.size, tilts.ctypes.data, vz, start, num, iters, subsets, relax,
                out.data_ptr(), stream.cuda_stream)
        assert rc == 0, L.at3r_last_error().decode()
        torch.cuda.synchronize()
        a, b = out.cpu().numpy().astype(np.float64), ref.cpu().numpy().astype(np.float64)
        err = np.linalg.norm(a - b) / np.linalg.norm(b)
        print(f"call {i + 1}: rel-L2 no-allocation vs plan path {err:.3e}")
        assert np.isfinite(a).all()
        assert err < TOL
        plan.close()


def test_noalloc_rejects_series_beyond_scratch():
    import torch
    from aretomo3_b200 import recon
    L = recon.lib()
    fn = _noalloc(L)
    tilts = np.linspace(-60, 60, 61).astype(np.float32)
    nx = 40000  # 2 * 61 * 40000 floats per slice > 16 MiB
    dummy = torch.empty(8, device="cuda")
    rc = fn(dummy.data_ptr(), nx, 1, tilts.size, tilts.ctypes.data, 64, 0, 61, 1, 5, 0.0, dummy.data_ptr(), None)
    assert rc == 5  # AT3R_ERR_TOO_LARGE, before any kernel runs
    assert b"16 MiB" in L.at3r_last_error()
