"""GPU: the projection-alignment re-projector against the reference's own
CCalcReproj + GReproj (fixtures it produced, and live runs of
oracle/_ref/ref_reproj when present): the same FP32 operations in the same
order, so the images agree bit for bit; device and host entry points agree;
invalid arguments are refused."""
import os
import sys

import numpy as np
import pytest

from oracle_lib import ROOT, load_golden, rel_l2

pytestmark = pytest.mark.gpu
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "ref_reproj")


def _ours(frames, tilts, proj, vol_z):
    from aretomo3_b200 import recon
    T, ny, nx = frames.shape
    skip = np.zeros(T, np.uint8)
    skip[proj] = 1
    c = recon.CCalcReproj()
    c.Setup((nx, ny, T), vol_z)
    return c.DoIt([frames[t] for t in range(T)], tilts, skip, proj)


@pytest.mark.parametrize("name", ["reproj_128_mid", "reproj_128_high", "reproj_97_end"])
def test_reproj_equals_reference_fixture(name):
    frames, tilts, ref, meta = load_golden(name)
    got = _ours(frames, tilts, meta["proj"], meta["vol_z"])
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("nx,ny,vz,T,proj", [(512, 48, 128, 41, 25), (1024, 16, 300, 61, 2), (301, 9, 77, 35, 34)])
def test_reproj_equals_live_reference(nx, ny, vz, T, proj):
    if not os.path.exists(REF_BIN):
        pytest.skip("oracle/_ref/ref_reproj not built")
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import gen_golden
    from aretomo3_b200 import synth
    tilts = np.linspace(-61, 59, T).astype(np.float32)
    frames = synth.make_tilt_series(nx, ny, tilts, vz, gen_golden.small_phantom(7 + proj))
    ref, _ = gen_golden.run_reference_reproj(frames, tilts, vz, proj)
    got = _ours(frames, tilts, proj, vz)
    assert np.array_equal(got, ref), rel_l2(got[ref > -1e29], ref[ref > -1e29])


def test_reproj_device_equals_host():
    import torch
    from aretomo3_b200 import recon
    frames, tilts, _, meta = load_golden("reproj_128_mid")
    skip = np.zeros(tilts.size, np.uint8)
    skip[meta["proj"]] = 1
    dev = recon.reproj_device(torch.from_numpy(frames).cuda(), tilts, meta["proj"], meta["vol_z"], skip)
    torch.cuda.synchronize()
    assert np.array_equal(dev.cpu().numpy(), _ours(frames, tilts, meta["proj"], meta["vol_z"]))


def test_reproj_invalid_arguments():
    from aretomo3_b200 import recon
    frames = np.zeros((5, 4, 32), np.float32)
    tilts = np.linspace(-20, 20, 5).astype(np.float32)
    c = recon.CCalcReproj()
    c.Setup((32, 4, 5), 16)
    with pytest.raises(recon.ReconError) as e:
        c.DoIt([frames[t] for t in range(5)], tilts, None, 7)   # projection index outside the series
    assert e.value.status == 1
