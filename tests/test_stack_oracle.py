"""CPU checks of the input-stage and thickness oracle (AreTomo/Correct
CCorrTomoStack with Fourier cropping, AreTomo/Recon/CCalcVolThick): known
answers, and the reference's own outputs (fixtures from oracle/_ref/ref_stack,
tests/golden/gen_golden.py)."""
import numpy as np
import pytest

import oracle_lib as ol

STACK_FIXTURES = ["stack_shift_128", "stack_rot_bin2", "stack_swap_local", "stack_odd_bin3"]


def test_sizes_known_answers():
    # CCorrectUtil::CalcAlignedSize swaps x/y past |sin| > 0.707; GetBinnedImgSize truncates, then rounds to even
    assert ol.stack_sizes(4096, 4096, True, 0.0, 20.0) == ((4096, 4096), (204, 204))
    assert ol.stack_sizes(4096, 3000, True, 85.0, 2.0) == ((3000, 4096), (1500, 2048))
    assert ol.stack_sizes(4096, 3000, True, 44.0, 2.0) == ((4096, 3000), (2048, 1500))
    assert ol.stack_sizes(4096, 3000, False, 85.0, 2.0) == ((4096, 3000), (2048, 1500))
    assert ol.stack_sizes(97, 64, True, 0.0, 1.0) == ((97, 64), (97, 64))
    assert ol.stack_sizes(1023, 1023, True, 0.0, 3.0) == ((1023, 1023), (340, 340))


def test_zero_alignment_takes_the_next_pixel():
    # GCorrPatchShift.cu:72-100: centre + 0.5, back by W/2, then + nx/2 and +0.5
    # before the int() truncation: with no shift or rotation pixel X reads X+1
    rng = np.random.default_rng(0)
    raw = rng.standard_normal((1, 12, 16)).astype(np.float32)
    _, al = ol.stack(raw, rand_fill=False)
    assert np.array_equal(al[0, :-1, :-1], raw[0, 1:, 1:])
    assert np.all(al[0, -1, :] < -1e29) and np.all(al[0, :, -1] < -1e29)


def test_shift_moves_the_sampling_point():
    rng = np.random.default_rng(1)
    raw = rng.standard_normal((1, 20, 24)).astype(np.float32)
    _, al = ol.stack(raw, shifts=np.array([[3.0, -2.0]], np.float32), rand_fill=False)
    # X reads X + 1 + 3, Y reads Y + 1 - 2
    assert np.array_equal(al[0, 1:15, 0:18], raw[0, 0:14, 4:22])


def test_fill_takes_values_from_nonempty_pixels_or_the_mean():
    rng = np.random.default_rng(2)
    ay, ax = 10, 12
    img = rng.standard_normal((ay, ax)).astype(np.float32)
    img[:3, :4] = -1e30
    W = ax
    table = rng.integers(0, W * ay, size=W * ay).astype(np.int32)
    out = ol.stack_fill(img, W, table)
    keep = img > -1e10
    assert np.array_equal(out[keep], img[keep])
    assert np.all(np.isin(out[~keep], img[keep]))
    # a chain that only meets empty pixels ends at the mean of the non-empty ones
    t2 = table.copy()
    t2[:] = 0                       # every chain starts at pixel 0, which is empty and points to itself
    out2 = ol.stack_fill(img, W, t2)
    mean = np.float32(img[keep].astype(np.float64).mean())
    assert np.allclose(out2[~keep], mean, rtol=1e-6)


def test_binning_keeps_constants_and_band_limited_cosines():
    ax, ay, T = 60, 48, 1
    x = np.arange(ax)[None, :]
    y = np.arange(ay)[:, None]
    img = (1.5 + np.cos(2 * np.pi * 3 * x / ax) * np.cos(2 * np.pi * 2 * y / ay)).astype(np.float32)
    out, _ = ol.stack(img[None], correct=False, bin=2.0)
    bx, by = 30, 24
    xb = np.arange(bx)[None, :]
    yb = np.arange(by)[:, None]
    ref = 1.5 + np.cos(2 * np.pi * 3 * xb / bx) * np.cos(2 * np.pi * 2 * yb / by)
    assert out.shape == (T, by, bx)
    assert np.abs(out[0] - ref).max() < 1e-5


def _oracle_for_fixture(d, meta, c2r_mode):
    return ol.stack(d["frames"], correct=True, shifts=d["shifts"],
                    tilt_axes=None if meta["shift_only"] else d["axes"], size_axis=meta["size_axis"],
                    local_params=d.get("local"), rand_fill=True, table=d["table"], bin=meta["bin"],
                    c2r_mode=c2r_mode)


@pytest.mark.parametrize("name", STACK_FIXTURES)
def test_stack_oracle_matches_reference(name):
    if not ol.golden_exists(name):
        pytest.skip("fixture not generated")
    d, meta = ol.load_npz(name)
    best = None
    for mode in (0, 1):   # the C2R convention the reference's cuFFT picked for this size
        out, al = _oracle_for_fixture(d, meta, mode)
        err = ol.rel_l2(out, d["binned"])
        best = err if best is None else min(best, err)
    ref_al = d["aligned"]
    T, ay, ax = al.shape
    W = ax & ~1
    if ax != W:
        # the driver unpads with CPad2D::Unpad, which packs rows of W = ax - 1
        # values for an odd width
        ref_al = ref_al.reshape(T, -1)[:, :ay * W].reshape(T, ay, W)
    same = np.mean(al[:, :, :W] == ref_al[:, :, :W])
    # FP32 coordinates in the reference's operation order: equal pixels, up to
    # host / device cos, sin, exp differences at rounding boundaries
    assert same >= (1.0 if meta["shift_only"] else 0.999)
    assert best < 1e-5


def test_thickness_oracle_matches_reference_on_a_given_volume():
    if not ol.golden_exists("thick_post_slab"):
        pytest.skip("fixture not generated")
    d, meta = ol.load_npz("thick_post_slab")
    prof = ol.thickness_profile(ol.unflip_vol(d["vol_xyz"]))
    assert np.array_equal(prof, d["profile"])
    sm, res = ol.thickness_edges(prof, meta["bin"])
    assert np.array_equal(sm, d["smoothed"])
    assert list(res) == list(d["result"])


def test_thickness_oracle_matches_reference_chain():
    if not ol.golden_exists("thick_full_1k"):
        pytest.skip("fixture not generated")
    d, meta = ol.load_npz("thick_full_1k")
    prof = ol.thickness_profile(d["volume"])
    assert np.array_equal(prof, d["profile"])
    _, res = ol.thickness_edges(prof, meta["bin"])
    assert list(res) == list(d["result"])


def test_thickness_edges_known_answer():
    # a step profile: low outside [30, 70), high inside; bins 20
    n = 100
    p = np.full(n, 0.1, np.float32)
    p[30:70] = 1.0
    sm, res = ol.thickness_edges(p, 20.0)
    lo, hi, thick, off = res
    assert 20 * 20 <= lo <= 32 * 20 and 66 * 20 <= hi <= 80 * 20
    assert thick == hi - lo and off == (lo + hi) // 2 - int(50 * 20.0)


def test_odd_width_covers_one_column_less():
    # GCorrPatchShift / GFillEmpty2D cover (padX/2 - 1) * 2 columns: ax - 1 for an odd ax;
    # the last column is 0 here (the reference leaves it unwritten)
    rng = np.random.default_rng(4)
    raw = rng.standard_normal((2, 14, 17)).astype(np.float32)
    table = rng.integers(0, 16 * 14, size=16 * 14).astype(np.int32)
    _, al = ol.stack(raw, shifts=np.zeros((2, 2), np.float32), table=table)
    assert al.shape == (2, 14, 17)
    assert np.all(al[:, :, 16] == 0.0)
    assert np.all(al[:, :, :16] > -1e10)     # every covered pixel filled


def test_bin_only_equal_sizes_is_a_copy():
    rng = np.random.default_rng(5)
    raw = rng.standard_normal((2, 20, 30)).astype(np.float32)
    out, _ = ol.stack(raw, correct=False, rand_fill=False, bin=1.0)
    assert np.array_equal(out.astype(np.float32), raw)
