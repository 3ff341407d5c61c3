"""GPU parity for missing-value inputs: the reference's "empty" rules.

The reference treats a projection value at or below -1e10 as missing: the
back-projections skip a lerped sample <= -1e10 (AreTomo/Recon/GBackProj.cu:
43-45, GBackProjWbp.cu:44-46), the forward projection skips a bilinear sample
< -1e10 and writes -1e30 for a ray with none (GForProj.cu:49-75), the SART
residual is 0 where the raw or the forward projection is below -1e10
(GDiffProj.cu:17-20), a SART update at or below -1e10 writes -1e30 (GBackProj.cu:
52-58), and after SART every -1e30 voxel is filled from a random chain
(CTomoSart.cpp:88, MaUtil/GFillEmpty2D.cu:7-143, table of GGenRandoms.cu).

Inputs: seeded series with -1e30 wedges (the empty corners an aligned, rotated
frame has), isolated -1e30 pixels, and pixels whose weighted value lies
just above -1e10 (they are summed, and drive the SART residual below -5e9);
for WBP, spikes whose filtered centre falls below -1e10;
NaN pixels make the reference's SART write -1e30 voxels (a NaN sum fails its
"> -1e10" test), which exercises the forward projection's per-sample path and
the fill.  Each case checks which of the library's guarded paths the run took
(at3r_plan_flags_seen) and compares with the reference's own CUDA Recon run
live (oracle/_ref/ref_recon, with the fill's seed fixed through its time()) and
with the FP64 oracle.

Tolerances (relative L2 over the volume): FP32 1e-4 against the reference and
the FP64 oracle; FP16 / BF16 storage 1e-3 against the FP64 oracle.
"""
import os
import sys

import numpy as np
import pytest

from oracle_lib import ROOT, rel_l2, sart, wbp

pytestmark = pytest.mark.gpu

REF_BIN = os.path.join(ROOT, "oracle", "_ref", "ref_recon")
TOL32 = 1e-4

SEEN_VOL_EMPTY, SEEN_RAW_LOW, SEEN_DIFF_LOW, SEEN_FILL_MEAN = 1, 2, 4, 8


@pytest.fixture(scope="module")
def R():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    from aretomo3_b200 import recon
    return recon


def run_reference(*a, **k):
    if not os.path.exists(REF_BIN):
        pytest.skip("reference binary oracle/_ref/ref_recon not built")
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import gen_golden
    return gen_golden.run_reference(*a, **k)[0]


def cos_table(tilts):
    return np.cos(np.float32(0.017453) * np.asarray(tilts, np.float32)).astype(np.float32)


def missing_series(nx, ny, tilts, vol_z, seed, near=True):
    """A phantom series with -1e30 wedges on the left of every frame (0 to
    nx/8 columns, growing with the tilt), 0.2 % isolated pixels at -1e30 and,
    with `near`, 0.05 % pixels whose weighted value (x cos / vol_z) is -7e9."""
    from aretomo3_b200 import synth
    ph = synth.Phantom(seed=seed, n_ellipsoids=40, axis_min=3, axis_max=14, n_beads=4, bead_radius=2,
                       noise_kind=synth.NOISE_POISSON, noise_param=50.0)
    f = synth.make_tilt_series(nx, ny, tilts, vol_z, ph)
    rng = np.random.default_rng(seed)
    T = len(tilts)
    c = cos_table(tilts)
    for t in range(T):
        w = int(round(abs(float(tilts[t])) / 60.0 * nx / 8))
        f[t, :, :w] = np.float32(-1e30)
    m = rng.random(f.shape) < 0.002
    f[m] = np.float32(-1e30)
    if near:
        m2 = (rng.random(f.shape) < 0.0005) & ~m
        for t in range(T):
            f[t][m2[t]] = np.float32(-7e9 * vol_z / c[t])
    return np.ascontiguousarray(f)


def plan_run(R, frames, tilts, vol_z, **kw):
    """Host-path run through a plan; returns (volume, flags seen)."""
    T, ny, nx = frames.shape
    plan = R.Plan(nx, ny, tilts, vol_z, **kw)
    try:
        vol = np.empty(plan.volume_shape, np.float32)
        plan.run_host([frames[t] for t in range(T)], [vol[y] for y in range(ny)])
        return vol, plan.flags_seen(), (plan.fill_table() if kw.get("method") == R.SART else None)
    finally:
        plan.close()


TILTS = np.linspace(-60, 60, 41).astype(np.float32)


def test_sart_missing_values_vs_reference(R):
    """SART over -1e30 wedges, isolated missing pixels and near-threshold
    values: the back-projection's per-sample path (staged values <= -5e9) and
    the residual rule; against the live reference and the FP64 oracle."""
    f = missing_series(256, 5, TILTS, 64, seed=71)
    kw = dict(method=R.SART, iterations=4, subsets=5, fill_seed=1234)
    vol, seen, _ = plan_run(R, f, TILTS, 64, **kw)
    assert seen & SEEN_RAW_LOW and seen & SEEN_DIFF_LOW, seen
    assert np.isfinite(vol).all() and vol.min() >= 0.0
    ref = run_reference("sart", f, TILTS, 64, 0, 41, 4, 5, fill_seed=1234)
    err = rel_l2(vol, ref)
    o64 = sart(f, TILTS, 64, 0, 41, 4, 5)
    err64 = rel_l2(vol, o64)
    print(f"SART missing values: rel-L2 vs reference {err:.3e}, vs FP64 oracle {err64:.3e}, flags {seen}")
    assert err < TOL32 and err64 < TOL32


@pytest.mark.parametrize("storage,near,tol", [("f16", False, 1e-3), ("bf16", True, 1e-3)])
def test_sart_missing_values_16bit_vs_oracle(R, storage, near, tol):
    """The 16-bit forms store a missing value as NaN (read back as -1e30).  A
    row is stored relative to its largest magnitude, so FP16 (5 exponent
    bits) cannot hold a row whose -7e9 near-threshold value sits beside
    ordinary values of order 1 (they fall below FP16's smallest subnormal,
    2^-24 of the scale); BF16 (8 exponent bits) can.  FP16 is checked on the
    missing values alone."""
    f = missing_series(256, 5, TILTS, 64, seed=72, near=near)
    st = R.STORE_F16 if storage == "f16" else R.STORE_BF16
    vol, seen, _ = plan_run(R, f, TILTS, 64, method=R.SART, iterations=4, subsets=5, storage=st)
    assert seen & SEEN_RAW_LOW and (seen & SEEN_DIFF_LOW or not near), seen
    o64 = sart(f, TILTS, 64, 0, 41, 4, 5)
    err = rel_l2(vol, o64)
    print(f"SART missing values {storage}: rel-L2 vs FP64 oracle {err:.3e}")
    assert np.isfinite(vol).all()
    assert err < tol


def spike_series(nx, ny, tilts, vol_z, seed, amp=-1e11):
    """A phantom series with 0.05 % pixels whose weighted value (x cos /
    vol_z) is `amp`.  The R-weight filter turns such a spike into a centre
    below -1e10 (skipped by the back-projection) flanked by lobes of order
    1e10 of both signs, far from the threshold at rounding level, so the
    skip decisions are robust to FFT rounding.  (A -1e30 value would spread
    through the whole filtered row at a level where the FFT's rounding, not
    the data, decides each sign; the reference never back-projects such rows:
    the input stage fills empty pixels first.)"""
    from aretomo3_b200 import synth
    ph = synth.Phantom(seed=seed, n_ellipsoids=40, axis_min=3, axis_max=14, n_beads=4, bead_radius=2)
    # the phantom at 1e8 (ordinary filtered values 1e6..1e8), so that a row
    # holding a spike's 1e10 lobes keeps its ordinary values in FP16 too
    f = synth.make_tilt_series(nx, ny, tilts, vol_z, ph) * np.float32(1e8)
    rng = np.random.default_rng(seed)
    c = cos_table(tilts)
    m = rng.random(f.shape) < 0.0005
    for t in range(len(tilts)):
        f[t][m[t]] = np.float32(amp * vol_z / c[t])
    return np.ascontiguousarray(f)


def test_wbp_missing_values_vs_reference(R):
    """WBP with filtered values below -1e10: the 2x-grid back-projection's
    per-sample path; against the live reference and the FP64 oracle."""
    f = spike_series(256, 4, TILTS, 64, seed=73)
    vol, seen, _ = plan_run(R, f, TILTS, 64, method=R.WBP)
    assert seen & SEEN_RAW_LOW, seen
    ref = run_reference("wbp", f, TILTS, 64)
    o64 = wbp(f, TILTS, 64)
    err, err64 = rel_l2(vol, ref), rel_l2(vol, o64)
    print(f"WBP missing values: rel-L2 vs reference {err:.3e}, vs FP64 oracle {err64:.3e}")
    assert err < TOL32 and err64 < TOL32


@pytest.mark.parametrize("storage,tol", [("f16", 1e-3), ("bf16", 2e-3)])
def test_wbp_missing_values_16bit_vs_oracle(R, storage, tol):
    """BF16 (8-bit mantissa) stays near 1.1e-3 here, as it does on ordinary
    WBP series (about 1.4e-3 at 4096 x 1200): it is held to 2e-3."""
    f = spike_series(256, 4, TILTS, 64, seed=74)
    st = R.STORE_F16 if storage == "f16" else R.STORE_BF16
    vol, seen, _ = plan_run(R, f, TILTS, 64, method=R.WBP, storage=st)
    assert seen & SEEN_RAW_LOW, seen
    o64 = wbp(f, TILTS, 64)
    err = rel_l2(vol, o64)
    print(f"WBP missing values {storage}: rel-L2 vs FP64 oracle {err:.3e}")
    assert err < tol


def nan_series(nx, ny, tilts, vol_z, seed, frac):
    from aretomo3_b200 import synth
    ph = synth.Phantom(seed=seed, n_ellipsoids=40, axis_min=3, axis_max=14, n_beads=4, bead_radius=2)
    f = synth.make_tilt_series(nx, ny, tilts, vol_z, ph)
    rng = np.random.default_rng(seed)
    f[rng.random(f.shape) < frac] = np.float32(np.nan)
    return np.ascontiguousarray(f)


def test_sart_empty_voxels_filled_as_reference(R):
    """NaN pixels: voxels whose sum takes one become -1e30 (as in the
    reference), the forward projection then tests every sample, and the fill
    replaces each -1e30 voxel with the voxel its random chain reaches.  With
    the fill's seed fixed on both sides the volume (filled voxels included)
    equals the reference's within the FP32 bar, and the FP64 oracle driven by
    the same table agrees."""
    f = nan_series(192, 4, TILTS, 48, seed=81, frac=2e-4)
    vol, seen, table = plan_run(R, f, TILTS, 48, method=R.SART, iterations=3, subsets=5, fill_seed=777)
    assert seen & SEEN_VOL_EMPTY, seen
    assert np.isfinite(vol).all() and (vol > -1e10).all()
    ref = run_reference("sart", f, TILTS, 48, 0, 41, 3, 5, fill_seed=777)
    assert (ref > -1e10).all()
    err = rel_l2(vol, ref)
    o64 = sart(f, TILTS, 48, 0, 41, 3, 5, fill_table=table)
    err64 = rel_l2(vol, o64)
    print(f"SART with empty voxels: rel-L2 vs reference {err:.3e}, vs FP64 oracle {err64:.3e}, flags {seen}")
    assert err < TOL32 and err64 < TOL32
    # a different seed fills from other voxels
    vol2, _, _ = plan_run(R, f, TILTS, 48, method=R.SART, iterations=3, subsets=5, fill_seed=778)
    assert not np.array_equal(vol, vol2)


def test_sart_fill_falls_back_to_mean_as_reference(R):
    """Nearly every voxel empty: most chains run 100 links without finding a
    value and take the slice mean, summed as the reference's 512-thread block
    sums it."""
    # a voxel's samples touch about 82 pixels: 4 % NaN pixels leave ~3 % of
    # the voxels non-empty, so ~3 % of the chains find nothing in 100 links
    f = nan_series(128, 3, TILTS, 40, seed=82, frac=0.04)
    vol, seen, table = plan_run(R, f, TILTS, 40, method=R.SART, iterations=1, subsets=5, fill_seed=99)
    assert seen & SEEN_VOL_EMPTY and seen & SEEN_FILL_MEAN, seen
    ref = run_reference("sart", f, TILTS, 40, 0, 41, 1, 5, fill_seed=99)
    err = rel_l2(vol, ref)
    o64 = sart(f, TILTS, 40, 0, 41, 1, 5, fill_table=table)
    err64 = rel_l2(vol, o64)
    print(f"SART fill by mean: rel-L2 vs reference {err:.3e}, vs FP64 oracle {err64:.3e}")
    assert err < TOL32 and err64 < TOL32


def test_sart_over_relaxed_update_writes_empty_voxels(R):
    """A relaxation above 1 (an at3r_geom option; the reference fixes 1/subsets)
    can drive an update below -1e10, which writes -1e30 and is filled; the
    FP64 oracle with the same table agrees."""
    # a central band of near-threshold pixels in every tilt: the voxels near
    # the tilt axis see it in every tilt, so their residual mean is about -7e9
    f = missing_series(160, 3, TILTS, 48, seed=75, near=False)
    c = cos_table(TILTS)
    for t in range(TILTS.size):
        f[t, :, 76:84] = np.float32(-7e9 * 48 / c[t])
    vol, seen, table = plan_run(R, f, TILTS, 48, method=R.SART, iterations=3, subsets=5, relax=3.0,
                                fill_seed=4242)
    o64 = sart(f, TILTS, 48, 0, 41, 3, 5, relax=3.0, fill_table=table)
    err = rel_l2(vol, o64)
    print(f"SART relax 3: flags {seen}, rel-L2 vs FP64 oracle {err:.3e}")
    assert seen & SEEN_VOL_EMPTY, seen
    assert (vol > -1e10).all()
    assert err < TOL32


def test_fill_table_is_the_reference_draw(R):
    """The plan's table follows GGenRandoms: entries in [0, Nx*Nz), a fixed
    function of the seed."""
    tilts = TILTS[:5]
    a = R.Plan(64, 2, tilts, 16, method=R.SART, iterations=1, subsets=1, fill_seed=5)
    b = R.Plan(64, 2, tilts, 16, method=R.SART, iterations=1, subsets=1, fill_seed=5)
    c = R.Plan(64, 2, tilts, 16, method=R.SART, iterations=1, subsets=1, fill_seed=6)
    ta, tb, tc = a.fill_table(), b.fill_table(), c.fill_table()
    for p in (a, b, c):
        p.close()
    assert ta.min() >= 0 and ta.max() < 64 * 16
    assert np.array_equal(ta, tb) and not np.array_equal(ta, tc)
