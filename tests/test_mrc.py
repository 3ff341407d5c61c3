"""CPU checks of the volume file (at3r_mrc_write, CAsyncSaveVol::mSaveVol's
MRC): the header fields and frames, and byte equality with the file the
reference's own writer (LibSrc/Mrcfile CSaveMrc, built into
oracle/_ref/ref_mrc) produces for the same volume.  Host code only: no GPU."""
import os
import subprocess

import numpy as np
import pytest

from oracle_lib import ROOT

REF_MRC = os.path.join(ROOT, "oracle", "_ref", "ref_mrc")


def _volume(nz=7, ny=5, nx=9, seed=0):
    return np.random.default_rng(seed).standard_normal((nz, ny, nx)).astype(np.float32)


def test_header_and_frames(tmp_path):
    from aretomo3_b200 import recon
    vol = _volume()
    path = str(tmp_path / "vol.mrc")
    recon.save_mrc(path, vol, 1.25)
    b = open(path, "rb").read()
    nz, ny, nx = vol.shape
    assert len(b) == 1024 + vol.nbytes
    h = np.frombuffer(b[:1024], np.int32)
    hf = np.frombuffer(b[:1024], np.float32)
    assert list(h[:4]) == [nx, ny, nz, 2]
    assert list(h[7:10]) == [nx, ny, nz]
    assert list(hf[10:13]) == [np.float32(nx * 1.25), np.float32(ny * 1.25), np.float32(nz * 1.25)]
    assert list(hf[13:16]) == [90.0, 90.0, 90.0]
    assert list(h[16:19]) == [1, 2, 3]
    assert list(hf[19:22]) == [0.0, 0.0, 0.0] and h[23] == 0          # no statistics, no extended header
    assert b[104:108] == b"AGAR" and h[27] == 20140
    assert np.frombuffer(b[96:98], np.int16)[0] == -16224
    assert b[208:212] == b"MAP\x00" and b[212:216] == b"DD\x00\x00"
    assert np.array_equal(np.frombuffer(b[1024:], np.float32).reshape(vol.shape), vol)


@pytest.mark.parametrize("shape", [(7, 5, 9), (1, 64, 48), (33, 17, 3)])
def test_equals_reference_writer(tmp_path, shape):
    if not os.path.exists(REF_MRC):
        pytest.skip("oracle/_ref/ref_mrc not built")
    from aretomo3_b200 import recon
    vol = _volume(*shape, seed=sum(shape))
    nz, ny, nx = vol.shape
    fin = str(tmp_path / "in.bin")
    with open(fin, "wb") as f:
        np.array([nx, ny, nz], np.int32).tofile(f)
        np.array([0.87], np.float32).tofile(f)
        np.linspace(-60, 60, nz).astype(np.float32).tofile(f)
        vol.tofile(f)
    ref, ours = str(tmp_path / "ref.mrc"), str(tmp_path / "ours.mrc")
    subprocess.run([REF_MRC, fin, ref], check=True, capture_output=True)
    recon.save_mrc(ours, [vol[z] for z in range(nz)], 0.87)
    assert open(ours, "rb").read() == open(ref, "rb").read()


def test_unwritable_path_is_an_io_error(tmp_path):
    from aretomo3_b200 import recon
    with pytest.raises(recon.ReconError) as ei:
        recon.save_mrc(str(tmp_path / "missing" / "vol.mrc"), _volume(), 1.0)
    assert ei.value.status == 7   # AT3R_ERR_IO
