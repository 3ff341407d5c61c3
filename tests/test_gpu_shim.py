"""The C++ drop-in, compiled against the reference's own headers: the shim
(integration/at3r_recon_shim.cpp) defines MAR::CDoWbpRecon and
MAR::CDoSartRecon (AreTomo/Recon/CReconInc.h:259-306) over libat3r and is
linked with the reference's own CTiltSeries / CAlignParam / Recon objects in
place of CDoWbpRecon.cpp and CDoSartRecon.cpp (oracle/ref/build_ref.sh ->
oracle/_ref/shim_recon).  The same driver (oracle/ref/ref_driver.cpp) runs the
shim build and the reference build on the same series: the volumes, frames
as the reference's DoIt returns them, agree within the FP32 bar (1e-4
relative L2).
"""
import os
import sys

import numpy as np
import pytest

from oracle_lib import ROOT, rel_l2

pytestmark = pytest.mark.gpu

sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
import gen_golden  # noqa: E402

TOL = 1e-4


def _need_bins():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    for b in (gen_golden.REF_BIN, gen_golden.SHIM_BIN):
        if not os.path.exists(b):
            pytest.skip(f"{os.path.basename(b)} not built (reference tree absent at build time)")


def _series(nx, ny, tilts, vol_z, seed):
    from aretomo3_b200 import synth
    ph = synth.Phantom(seed=seed, n_ellipsoids=60, axis_min=3, axis_max=20, n_beads=6, bead_radius=3,
                       noise_kind=synth.NOISE_POISSON, noise_param=50.0)
    return synth.make_tilt_series(nx, ny, tilts, vol_z, ph)


@pytest.mark.parametrize("mode,nx,ny,vol_z", [("wbp", 512, 6, 128), ("wbp", 301, 3, 77), ("sart", 256, 5, 96),
                                               ("sart", 97, 3, 37)])
def test_shim_equals_reference(mode, nx, ny, vol_z):
    _need_bins()
    tilts = (np.linspace(-60, 60, 41) + 0.7).astype(np.float32)
    f = _series(nx, ny, tilts, vol_z, seed=nx + vol_z)
    args = (mode, f, tilts, vol_z) + ((2, 35, 4, 5) if mode == "sart" else ())
    ref, info_r = gen_golden.run_reference(*args, fill_seed=11)
    got, info_s = gen_golden.run_reference(*args, fill_seed=11, binary=gen_golden.SHIM_BIN)
    assert got.shape == ref.shape == (ny, vol_z, nx & ~1)
    err = rel_l2(got, ref)
    print(f"shim {mode} {nx}x{ny}x41 Nz {vol_z}: rel-L2 vs reference {err:.3e}; DoIt {info_s['seconds']:.4f} s "
          f"vs reference {info_r['seconds']:.4f} s")
    assert info_s["cuda"] == "no error"
    assert err < TOL


def test_shim_fill_equals_reference():
    """NaN pixels make both builds fill -1e30 voxels; with time() fixed, the
    shim's fill (seeded by at3r_geom_init from time(0), as the reference seeds
    GGenRandoms) picks the same voxels."""
    _need_bins()
    tilts = np.linspace(-60, 60, 41).astype(np.float32)
    f = _series(160, 3, tilts, 48, seed=5)
    rng = np.random.default_rng(5)
    f[rng.random(f.shape) < 2e-4] = np.float32(np.nan)
    args = ("sart", f, tilts, 48, 0, 41, 3, 5)
    ref, _ = gen_golden.run_reference(*args, fill_seed=31337)
    got, _ = gen_golden.run_reference(*args, fill_seed=31337, binary=gen_golden.SHIM_BIN)
    assert (ref > -1e10).all() and (got > -1e10).all()
    err = rel_l2(got, ref)
    print(f"shim SART with filled voxels: rel-L2 vs reference {err:.3e}")
    assert err < TOL
