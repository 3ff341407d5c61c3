"""CPU checks of the oracle: against the reference's own outputs (golden
fixtures produced by tests/golden/gen_golden.py from the reference's CUDA
Recon) and against known answers."""
import ctypes
import glob
import os

import numpy as np
import pytest

import oracle_lib as ol
from oracle_lib import P, lib, load_golden, rel_l2, sart, wbp

GOLDEN = sorted(n for n in (os.path.basename(f)[:-4] for f in glob.glob(os.path.join(os.path.dirname(__file__),
                                                                                  "golden", "*.npz")))
                if not n.startswith(("reproj_", "stack_", "thick_")))

# FP64 oracle vs the reference's FP32 CUDA result: the reference accumulates in
# FP32 (and SART iterates 15 times), so the two agree to ~1e-6 relative L2.
GOLDEN_TOL = 1e-5


@pytest.mark.parametrize("name", GOLDEN)
def test_oracle_matches_reference_golden(name):
    frames, tilts, ref, meta = load_golden(name)
    if meta["mode"] == "wbp":
        out = wbp(frames, tilts, meta["vol_z"])
    else:
        out = sart(frames, tilts, meta["vol_z"], meta["start"], meta["ntilts"], meta["iters"], meta["subsets"])
    assert out.shape == ref.shape
    assert rel_l2(out, ref) < GOLDEN_TOL


@pytest.mark.parametrize("n", [2, 6, 16, 48, 96, 97, 128, 300, 599, 1200, 1198, 4096])
def test_fft_matches_numpy(n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    xi = np.empty(2 * n)
    xi[0::2], xi[1::2] = x.real, x.imag
    for sign, ref in ((-1, np.fft.fft(x)), (1, np.fft.ifft(x) * n)):
        o = np.empty(2 * n)
        assert lib().oracle_fft_f64(xi.ctypes.data_as(P), n, sign, o.ctypes.data_as(P)) == 0
        y = o[0::2] + 1j * o[1::2]
        assert np.abs(y - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max())


def test_rweight_transfer_function_known_values():
    n = 512
    h = np.empty(n // 2 + 1)
    lib().oracle_rweight_filter_f64(n, h.ctypes.data_as(P))
    assert h[0] == 0.0
    # Nyquist: (1/N) * 2 * 0.5 * (0.55 - 0.45) = 0.1 / N  (AreTomo/Recon/GRWeight.cu:19-20)
    assert abs(h[n // 2] - 0.1 / n) < 1e-9 / n
    # the ramp rises then the window rolls off
    assert np.argmax(h) not in (0, n // 2)


def test_rweight_row_is_circular_convolution():
    n = 96
    rng = np.random.default_rng(3)
    row = rng.standard_normal(n)
    out = np.empty(n)
    lib().oracle_rweight_row_f64(row.ctypes.data_as(P), n, out.ctypes.data_as(P))
    h = np.empty(n // 2 + 1)
    lib().oracle_rweight_filter_f64(n, h.ctypes.data_as(P))
    ref = np.fft.irfft(np.fft.rfft(row) * h, n) * n
    assert np.abs(out - ref).max() < 1e-12


@pytest.mark.parametrize("nx,nz", [(64, 32), (48, 21), (96, 37)])
def test_fourier_crop_decimates_band_limited_image(nx, nz):
    X = np.arange(2 * nx)[None, :]
    Z = np.arange(2 * nz)[:, None]
    a, b = 5, 3
    g = np.cos(2 * np.pi * (a * X / (2 * nx) + b * Z / (2 * nz))) + 0.25
    f = np.empty((nz, nx))
    lib().oracle_set_c2r_mode(0)
    assert lib().oracle_fourier_crop_f64(np.ascontiguousarray(g).ctypes.data_as(P), nx, nz, f.ctypes.data_as(P)) == 0
    assert np.abs(f - g[::2, ::2]).max() < 1e-12


@pytest.mark.parametrize("mode", [0, 1])
def test_c2r_conventions(mode):
    """mode 0 drops the imaginary DC/Nyquist parts; mode 1 (half-length
    packing) adds -(Im X0 + Im XN/2) to even and (Im X0 - Im XN/2) to odd
    samples."""
    n = 32
    rng = np.random.default_rng(5)
    X = rng.standard_normal(n // 2 + 1) + 1j * rng.standard_normal(n // 2 + 1)
    xi = np.empty(2 * (n // 2 + 1))
    xi[0::2], xi[1::2] = X.real, X.imag
    out = np.empty(n)
    lib().oracle_set_c2r_mode(mode)
    lib().oracle_c2r_f64(xi.ctypes.data_as(P), n, out.ctypes.data_as(P))
    lib().oracle_set_c2r_mode(0)
    ref = np.fft.irfft(X, n) * n
    if mode == 1:
        b, d = X[0].imag, X[n // 2].imag
        ref[0::2] += -(b + d)
        ref[1::2] += (b - d)
    assert np.abs(out - ref).max() < 1e-12


def test_sart_constant_projections_give_constant_volume():
    """Projections equal to Nz / cos(theta) weight to 1 everywhere; the first
    back-projection then writes 1 into every voxel any ray reaches, and the
    consistent data leave the residual at zero."""
    nx, ny, nz = 64, 2, 16
    tilts = np.linspace(-30, 30, 7).astype(np.float32)
    cs = np.empty(2 * tilts.size, np.float32)
    lib().oracle_cos_sin(tilts.ctypes.data_as(P), tilts.size, cs.ctypes.data_as(P))
    frames = np.empty((tilts.size, ny, nx), np.float32)
    for t in range(tilts.size):
        frames[t] = np.float32(nz) / cs[2 * t]
    out = sart(frames, tilts, nz, 0, tilts.size, 0, 1)
    inner = out[:, 2:-2, 16:-16]
    assert np.allclose(inner, 1.0, atol=1e-6)


def test_sart_residual_decreases_on_consistent_data():
    from aretomo3_b200 import synth
    tilts = synth.tilt_range(-60, 60, 4)
    ph = synth.Phantom(seed=9, n_ellipsoids=20, axis_min=3, axis_max=10, n_beads=2, bead_radius=2,
                       noise_kind=synth.NOISE_NONE)
    frames = synth.make_tilt_series(96, 2, tilts, 32, ph)
    _, rf = sart(frames, tilts, 32, 0, tilts.size, 6, 5, rfactor=True)
    r = rf[:, 0] / rf[:, 1]
    assert np.all(np.diff(r) < 0), r


def test_sart_rejects_tilt_range_outside_series():
    frames, tilts, _, meta = load_golden("sart_odd97")
    with pytest.raises(ValueError):
        sart(frames, tilts, meta["vol_z"], 20, 24, 1, 4)
    with pytest.raises(ValueError):
        sart(frames, tilts, meta["vol_z"], 0, 24, 1, 0)


def test_fp32_port_close_to_fp64():
    frames, tilts, ref, meta = load_golden("wbp_128")
    a = wbp(frames, tilts, meta["vol_z"], f32=True)
    assert rel_l2(a, ref) < 1e-4
    frames, tilts, ref, meta = load_golden("sart_128")
    a = sart(frames, tilts, meta["vol_z"], meta["start"], meta["ntilts"], meta["iters"], meta["subsets"], f32=True)
    assert rel_l2(a, ref) < 1e-4


# --- projection-alignment re-projection (AreTomo/ProjAlign) -----------------
@pytest.mark.parametrize("name", ["reproj_128_mid", "reproj_128_high", "reproj_97_end"])
def test_reproj_oracle_matches_reference_fixture(name):
    frames, tilts, ref, meta = load_golden(name)
    skip = np.zeros(tilts.size, np.uint8)
    skip[meta["proj"]] = 1
    got = ol.reproj(frames, tilts, meta["proj"], meta["vol_z"], skip)
    valid = ref > -1e29
    assert np.array_equal(valid, got > -1e29)    # the same rays pass the 80 % coverage rule
    # host cosf/sinf may differ from the device's in the last bit, which can
    # move a nearest-neighbour sample; the bound allows for that
    assert ol.rel_l2(got[valid], ref[valid]) < 1e-4
