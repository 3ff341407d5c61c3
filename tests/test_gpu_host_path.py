"""GPU: the host path.  Pageable caller frames go through the pinned staging
ring (64 MB slots, pieces split across slots), pinned ones are copied
directly; both give the device path's volume bit for bit, in XZ frames and in
XY frames, with several slabs in flight and with one slab."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _series(nx, ny, tilts, vol_z, seed):
    from aretomo3_b200 import synth
    ph = synth.Phantom(seed=seed, n_ellipsoids=60, axis_min=4, axis_max=30, n_beads=6, bead_radius=3)
    return synth.make_tilt_series(nx, ny, tilts, vol_z, ph)


@pytest.mark.parametrize("slab", [0, 16])
def test_pageable_and_pinned_equal_device(slab):
    import torch
    from aretomo3_b200 import recon
    tilts = np.linspace(-60, 60, 41).astype(np.float32)
    nx, ny, vz = 1024, 96, 300          # volume 118 MB: two and more output slots
    frames = _series(nx, ny, tilts, vz, seed=31)
    plan = recon.Plan(nx, ny, tilts, vz, method=recon.WBP, slab_slices=slab)
    try:
        proj = torch.from_numpy(frames).cuda()
        vdev = torch.empty(plan.volume_shape, device="cuda")
        plan.run_device(proj.data_ptr(), vdev.data_ptr(), torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        ref = vdev.cpu().numpy()
        T = frames.shape[0]
        # pageable in and out
        vol = np.empty(plan.volume_shape, np.float32)
        plan.run_host([frames[t] for t in range(T)], [vol[y] for y in range(ny)])
        assert np.array_equal(vol, ref)
        # pinned in and out
        pin_in = torch.from_numpy(frames).pin_memory().numpy()
        pin_out = torch.empty(plan.volume_shape).pin_memory().numpy()
        plan.run_host([pin_in[t] for t in range(T)], [pin_out[y] for y in range(ny)])
        assert np.array_equal(pin_out, ref)
        # XY frames, pageable and pinned
        want = np.ascontiguousarray(np.transpose(ref, (1, 0, 2))[::-1])   # FlipVol(1)
        assert np.array_equal(plan.run_host_xyz([frames[t] for t in range(T)], flip=True), want)
        pin_xyz = torch.empty((vz, ny, nx)).pin_memory().numpy()
        plan.run_host_xyz([pin_in[t] for t in range(T)], out=pin_xyz, flip=True)
        assert np.array_equal(pin_xyz, want)
    finally:
        plan.close()
