"""GPU: the back-projection's window staging by bulk asynchronous copies (the
AT3R_BP_BULK_STAGING=1 plan option, FP32 storage) stages the same values as
the load path, so WBP and SART volumes are bit-identical either way —
including tiles whose windows reach past the detector edge (those rows take
the load path) and widths that are not a multiple of 4 (the option is off
there)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _series(nx, ny, tilts, vol_z, seed):
    from aretomo3_b200 import synth
    ph = synth.Phantom(seed=seed, n_ellipsoids=40, axis_min=3, axis_max=16, n_beads=4, bead_radius=3)
    return synth.make_tilt_series(nx, ny, tilts, vol_z, ph)


def _run(frames, tilts, vol_z, bulk, **kw):
    from aretomo3_b200 import recon
    old = os.environ.get("AT3R_BP_BULK_STAGING")
    os.environ["AT3R_BP_BULK_STAGING"] = "1" if bulk else "0"
    try:
        T, ny, nx = frames.shape
        plan = recon.Plan(nx, ny, tilts, vol_z, **kw)
    finally:
        if old is None:
            del os.environ["AT3R_BP_BULK_STAGING"]
        else:
            os.environ["AT3R_BP_BULK_STAGING"] = old
    try:
        vol = np.empty(plan.volume_shape, np.float32)
        plan.run_host([frames[t] for t in range(T)], [vol[y] for y in range(ny)])
        return vol, plan.flags_seen()
    finally:
        plan.close()


@pytest.mark.parametrize("nx,lim", [(256, 60), (512, 72), (258, 60)])
@pytest.mark.parametrize("mode", ["wbp", "sart"])
def test_bulk_staging_equals_load_path(nx, lim, mode):
    import torch
    assert torch.cuda.is_available()
    from aretomo3_b200 import recon
    tilts = np.linspace(-lim, lim, 37).astype(np.float32)
    f = _series(nx, 6, tilts, 64, seed=nx + lim)
    kw = dict(method=recon.WBP) if mode == "wbp" else dict(method=recon.SART, iterations=3, subsets=4)
    a, _ = _run(f, tilts, 64, False, **kw)
    b, seen = _run(f, tilts, 64, True, **kw)
    assert not seen & 16, "a bulk staging wait ran out"
    assert np.array_equal(a, b)
