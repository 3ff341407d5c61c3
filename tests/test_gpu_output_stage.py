"""GPU: the volume output stage.  The XY-frame volume equals
CTiltSeries::FlipVol(bFlip) (DataUtil/CTiltSeries.cpp:286-305) applied to the
XZ frames the reconstruction returns: frame (flip ? Nz-1-zr : zr) holds row zr
of every XZ frame."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def flipvol(vol_xzy, flip):
    """FlipVol restated on a [ny][Nz][Nx] array: new frame index from the old
    row index, flipped when bFlip."""
    ny, nz, nx = vol_xzy.shape
    out = np.empty((nz, ny, nx), vol_xzy.dtype)
    for zr in range(nz):
        out[nz - 1 - zr if flip else zr] = vol_xzy[:, zr, :]
    return out


def _series(nx, ny, tilts, vol_z, seed):
    from aretomo3_b200 import synth
    ph = synth.Phantom(seed=seed, n_ellipsoids=30, axis_min=3, axis_max=15, n_beads=3, bead_radius=3)
    return synth.make_tilt_series(nx, ny, tilts, vol_z, ph)


@pytest.mark.parametrize("flip", [True, False])
@pytest.mark.parametrize("method", ["wbp", "sart"])
def test_run_host_xyz_equals_flipvol(flip, method):
    from aretomo3_b200 import recon
    tilts = np.linspace(-57, 60, 37).astype(np.float32)
    nx, ny, vz = 201, 27, 48
    frames = _series(nx, ny, tilts, vz, seed=77)
    kw = dict(method=recon.SART, iterations=2, subsets=3) if method == "sart" else dict(method=recon.WBP)
    plan = recon.Plan(nx, ny, tilts, vz, slab_slices=8, **kw)   # several slabs
    try:
        vol = np.empty(plan.volume_shape, np.float32)
        plan.run_host([frames[t] for t in range(frames.shape[0])], [vol[y] for y in range(ny)])
        xyz = plan.run_host_xyz([frames[t] for t in range(frames.shape[0])], flip=flip)
    finally:
        plan.close()
    assert np.array_equal(xyz, flipvol(vol, flip))


@pytest.mark.parametrize("flip", [True, False])
def test_volume_xyz_device(flip):
    import torch
    from aretomo3_b200 import recon
    g = torch.Generator().manual_seed(5)
    vol = torch.randn((13, 40, 66), generator=g).cuda()
    out = recon.volume_xyz(vol, flip=flip)
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), flipvol(vol.cpu().numpy(), flip))
