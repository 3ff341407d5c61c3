"""GPU: the input stage (at3r_stack: aligned + Fourier-binned tilt series,
CCorrTomoStack / CBinStack::DoFFT) and the thickness measurement
(at3r_thickness: CCalcVolThick) against the reference's own outputs
(fixtures from oracle/_ref/ref_stack) and the FP64 oracle."""
import numpy as np
import pytest

import oracle_lib as ol
from aretomo3_b200 import recon, synth

pytestmark = pytest.mark.gpu

STACK_FIXTURES = ["stack_shift_128", "stack_rot_bin2", "stack_swap_local", "stack_odd_bin3"]
# FP32 binning (shared-memory FFTs) against FP64 and against cuFFT
BIN_TOL = 1e-5


def _stack_for(d, meta):
    T, ny, nx = d["frames"].shape
    return recon.Stack(nx, ny, T, shifts=d["shifts"], tilt_axes=None if meta["shift_only"] else d["axes"],
                       size_axis=meta["size_axis"], local_params=d.get("local"), rand_fill=True, seed=meta["seed"],
                       bin=meta["bin"])


@pytest.mark.parametrize("name", STACK_FIXTURES)
def test_random_table_equals_reference(name):
    if not ol.golden_exists(name):
        pytest.skip("fixture not generated")
    d, meta = ol.load_npz(name)
    st = _stack_for(d, meta)
    try:
        assert np.array_equal(st.fill_table(), d["table"])
    finally:
        st.close()


@pytest.mark.parametrize("name", STACK_FIXTURES)
def test_stack_equals_reference(name):
    if not ol.golden_exists(name):
        pytest.skip("fixture not generated")
    d, meta = ol.load_npz(name)
    st = _stack_for(d, meta)
    try:
        out = st.run_host([f for f in d["frames"]])
        assert out.shape == d["binned"].shape
        if meta["bin"] == 1.0:
            # no Fourier crop: the aligned, filled frames themselves, bit for bit
            assert np.array_equal(out, d["aligned"])
        else:
            assert ol.rel_l2(out, d["binned"]) < BIN_TOL
        # and against the FP64 oracle driven by the same table
        ref, _ = ol.stack(d["frames"], shifts=d["shifts"], tilt_axes=None if meta["shift_only"] else d["axes"],
                          size_axis=meta["size_axis"], local_params=d.get("local"), table=st.fill_table(),
                          bin=meta["bin"], c2r_mode=_mode(st))
        assert ol.rel_l2(out, ref) < BIN_TOL
    finally:
        st.close()


def _mode(st):
    """The oracle's C2R mode for the convention the stack resolved."""
    return 1 if st.c2r == recon.C2R_PACKED else 0


def test_aligned_frames_equal_live_reference_at_4k():
    # at 4096^2 the coordinates are large enough that a different rounding of
    # the rotation picks another raw pixel for ~1 pixel in 10^5: every aligned
    # pixel (fill included) must be the reference kernel's
    import os
    if not os.path.exists(os.path.join(ol.ROOT, "oracle", "_ref", "ref_stack")):
        pytest.skip("oracle/_ref/ref_stack not built")
    import sys
    sys.path.insert(0, os.path.join(ol.ROOT, "tests", "golden"))
    import gen_golden
    rng = np.random.default_rng(3)
    T = 2
    frames = synth.make_tilt_series(4096, 4096, synth.tilt_range(-3, 3, 6), 300,
                                    synth.Phantom(seed=9, n_ellipsoids=150, axis_min=20.0, axis_max=160.0, n_beads=10))
    c = dict(shifts=rng.uniform(-20, 20, (T, 2)).astype(np.float32),
             axes=rng.uniform(85.0, 87.0, T).astype(np.float32), shift_only=0, bin=1.0, local=None, seed=4242)
    c["size_axis"] = float(c["axes"][0])
    al_ref, _, table_ref, _ = gen_golden.run_reference_stack(frames, synth.tilt_range(-3, 3, 6), c)
    st = recon.Stack(4096, 4096, T, shifts=c["shifts"], tilt_axes=c["axes"], size_axis=c["size_axis"], seed=4242,
                     bin=1.0)
    try:
        assert np.array_equal(st.fill_table(), table_ref)
        out = st.run_host([f for f in frames])
    finally:
        st.close()
    assert np.array_equal(out, al_ref)


def test_device_path_equals_host_path():
    import torch
    rng = np.random.default_rng(5)
    T, ny, nx = 6, 200, 256
    frames = rng.standard_normal((T, ny, nx)).astype(np.float32)
    kw = dict(shifts=rng.uniform(-9, 9, (T, 2)), tilt_axes=rng.uniform(-4, 4, T), size_axis=1.0, seed=11, bin=3.0)
    st = recon.Stack(nx, ny, T, **kw)
    try:
        host = st.run_host([f for f in frames])
        raw = torch.from_numpy(frames).cuda()
        out = torch.empty(st.binned_shape, device="cuda", dtype=torch.float32)
        st.run_device(raw.data_ptr(), out.data_ptr(), torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy(), host)
    finally:
        st.close()


def test_host_pipeline_over_several_chunks():
    # 64 MB frames: the host path moves four tilts per chunk, double-buffered,
    # through the pinned staging slots (pageable frames) or directly (pinned)
    import torch
    rng = np.random.default_rng(15)
    T, ny, nx = 9, 4096, 4096
    frames = rng.standard_normal((T, ny, nx), dtype=np.float32)
    st = recon.Stack(nx, ny, T, shifts=rng.uniform(-9, 9, (T, 2)), tilt_axes=rng.uniform(85, 87, T), size_axis=86.0,
                     seed=2, bin=4.0)
    try:
        raw = torch.from_numpy(frames).cuda()
        out = torch.empty(st.binned_shape, device="cuda", dtype=torch.float32)
        st.run_device(raw.data_ptr(), out.data_ptr(), torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        dev = out.cpu().numpy()
        assert np.array_equal(st.run_host([f for f in frames]), dev)
        pin_in = torch.from_numpy(frames).pin_memory()
        pin_out = torch.empty(st.binned_shape, dtype=torch.float32).pin_memory()
        st.run_host([pin_in[t].numpy() for t in range(T)], pin_out.numpy())
        assert np.array_equal(pin_out.numpy(), dev)
        mixed = np.empty(st.binned_shape, np.float32)
        st.run_host([pin_in[t].numpy() for t in range(T)], mixed)
        assert np.array_equal(mixed, dev)
    finally:
        st.close()


@pytest.mark.parametrize("nx,ny,T,bin,axes", [(1000, 1022, 5, 4.0, (-3.0, 3.0)), (1024, 768, 4, 2.0, (85.0, 87.0)),
                                              (510, 498, 3, 1.7, (0.0, 0.0)), (1000, 1022, 4, 4.0, (0.0, 0.0))])
def test_stack_matches_oracle_larger(nx, ny, T, bin, axes):
    # 1022 = 2 x 7 x 73: Bluestein column FFT; 85-87 degrees: x / y swapped.
    # Without rotation the FP32 sampling coordinates are exact and the result
    # meets the FP32 bound.  With rotation the oracle's cos / sin come from the
    # host's libm and the kernel's from CUDA's cosf / sinf (as the reference's
    # do), which can differ in the last bit; the few pixels whose coordinate
    # sits at a rounding boundary then pick a neighbour.  The aligned frames
    # themselves are pinned bit for bit against the reference's own kernels
    # by the stack_* fixtures.
    rng = np.random.default_rng(nx + ny)
    frames = synth.make_tilt_series(nx, ny, synth.tilt_range(-30, 30, 60.0 / max(T - 1, 1))[:T], 200,
                                    synth.Phantom(seed=nx, n_ellipsoids=120, n_beads=8))
    shifts = rng.uniform(-20, 20, (T, 2)).astype(np.float32)
    ax = rng.uniform(axes[0], axes[1], T).astype(np.float32)
    st = recon.Stack(nx, ny, T, shifts=shifts, tilt_axes=ax, size_axis=float(ax[0]), seed=3, bin=bin)
    try:
        out = st.run_host([f for f in frames])
        ref, _ = ol.stack(frames, shifts=shifts, tilt_axes=ax, size_axis=float(ax[0]), table=st.fill_table(),
                          bin=bin, c2r_mode=_mode(st))
        assert ol.rel_l2(out, ref) < (BIN_TOL if axes == (0.0, 0.0) else 2e-4)
    finally:
        st.close()


def test_bin_only_matches_oracle():
    rng = np.random.default_rng(8)
    frames = rng.standard_normal((3, 300, 412)).astype(np.float32)
    out = recon.CBinStack.DoFFT(recon.TiltSeries(frames), 3.3).frames
    ref, _ = ol.stack(frames, correct=False, rand_fill=False, bin=3.3)
    assert out.shape == ref.shape
    assert ol.rel_l2(out, ref) < BIN_TOL


def test_corr_tomo_stack_mirror_matches_stack():
    rng = np.random.default_rng(9)
    T, ny, nx = 4, 160, 192
    frames = rng.standard_normal((T, ny, nx)).astype(np.float32)
    ap = recon.AlignParam(tilts=np.linspace(-30, 30, T).astype(np.float32),
                          shifts=rng.uniform(-5, 5, (T, 2)).astype(np.float32),
                          tilt_axes=rng.uniform(-3, 3, T).astype(np.float32))
    c = recon.CCorrTomoStack()
    c.Set0(recon.TiltSeries(frames))
    c.Set1(0, float(ap.tilt_axes[0]))
    c.Set2(2.0, True, True)
    c.Set3(False, False, False)
    c.Set4(True)
    got = c.DoIt(ap, seed=21).frames
    st = recon.Stack(nx, ny, T, shifts=ap.shifts, tilt_axes=ap.tilt_axes, size_axis=float(ap.tilt_axes[0]), seed=21,
                     bin=2.0)
    try:
        assert np.array_equal(got, st.run_host([f for f in frames]))
    finally:
        st.close()
    bx, by = c.GetBinning()
    assert bx == np.float32(2.0) and by == np.float32(2.0)


def test_invalid_stack_arguments_are_refused():
    with pytest.raises(recon.ReconError):
        recon.Stack(1, 64, 3)
    with pytest.raises(recon.ReconError):
        recon.Stack(64, 64, 3, bin=0.5)
    with pytest.raises(recon.ReconError):
        recon.Stack(64, 64, 3, bin=100.0)   # binned frame below 2 x 2


def test_thickness_full_chain_equals_reference():
    if not ol.golden_exists("thick_full_1k"):
        pytest.skip("fixture not generated")
    d, meta = ol.load_npz("thick_full_1k")
    ph = meta["phantom"]
    frames = synth.make_tilt_series(meta["nx"], meta["ny"], d["tilts"], meta["vol_z"],
                                    synth.Phantom(seed=ph["seed"], n_ellipsoids=ph["n_ellipsoids"],
                                                  n_beads=ph["n_beads"]))
    ap = recon.AlignParam(tilts=d["tilts"], shifts=d["shifts"], tilt_axes=d["axes"])
    c = recon.CCalcVolThick().DoIt(recon.TiltSeries(frames), ap, meta["pix"], seed=meta["seed"])
    r = c.result
    assert r.vol_z == meta["wbp_vol_z"]
    assert (r.binned_xy[0], r.binned_xy[1]) == (d["binned"].shape[2], d["binned"].shape[1])
    assert ol.rel_l2(c.profile, d["profile"]) < 1e-4
    assert [r.edges[0], r.edges[1], r.thickness, r.offset_z] == list(d["result"])
    assert c.GetThickness(False) == float(d["result"][2])


def test_thickness_post_processing_equals_oracle_on_the_same_volume():
    # the pipeline's own stages run through the public entry points; the
    # thickness entry point's profile and edges must equal the oracle's
    # measurement of that volume
    import torch
    rng = np.random.default_rng(12)
    T, ny, nx = 31, 600, 640
    tilts = synth.tilt_range(-60, 60, 4)
    frames = synth.make_tilt_series(nx, ny, tilts, 200, synth.Phantom(seed=4, n_ellipsoids=150, n_beads=10))
    shifts = rng.uniform(-4, 4, (T, 2)).astype(np.float32)
    axes = np.full(T, 0.8, np.float32)
    ap = recon.AlignParam(tilts=tilts, shifts=shifts, tilt_axes=axes)
    c = recon.CCalcVolThick().DoIt(recon.TiltSeries(frames), ap, 1.0, seed=8)
    r = c.result
    st = recon.Stack(nx, ny, T, shifts=shifts, tilt_axes=axes, size_axis=float(axes[0]), seed=8, bin=r.binning)
    try:
        binned = st.run_host([f for f in frames])
    finally:
        st.close()
    vol_t, plan = recon.reconstruct_device(torch.from_numpy(binned).cuda(), tilts, r.vol_z)
    torch.cuda.synchronize()
    vol = vol_t.cpu().numpy()
    plan.close()
    prof = ol.thickness_profile(vol)
    assert np.abs(prof - c.profile).max() <= 2e-7 * max(1.0, float(np.abs(prof).max()))
    sm, res = ol.thickness_edges(c.profile, r.binning)
    assert np.array_equal(sm, c.profile_smoothed)
    assert list(res) == [r.edges[0], r.edges[1], r.thickness, r.offset_z]


@pytest.mark.parametrize("method", [recon.WBP, recon.SART])
def test_recon_series_keeps_the_binned_series_on_the_device(method):
    # CAreTomoMain::mRecon's data flow (aligned, binned, reconstructed) with the
    # binned series kept on the device equals the two host-path stages
    rng = np.random.default_rng(21)
    T, ny, nx = 11, 256, 320
    tilts = synth.tilt_range(-60, 60, 12)
    frames = synth.make_tilt_series(nx, ny, tilts, 80, synth.Phantom(seed=6, n_ellipsoids=60, n_beads=6))
    ap = recon.AlignParam(tilts=tilts, shifts=rng.uniform(-6, 6, (T, 2)).astype(np.float32),
                          tilt_axes=rng.uniform(-2, 2, T).astype(np.float32))
    kw = dict(iterations=3, subsets=4) if method == recon.SART else {}
    got = recon.recon_series(recon.TiltSeries(frames), ap, 48, at_bin=2.0, method=method, seed=5, **kw)
    st = recon.Stack(nx, ny, T, shifts=ap.shifts, tilt_axes=ap.tilt_axes, size_axis=float(ap.tilt_axes[0]), seed=5,
                     bin=2.0)
    try:
        binned = st.run_host([f for f in frames])
    finally:
        st.close()
    if method == recon.WBP:
        ref = recon.CDoWbpRecon().DoIt(recon.TiltSeries(binned), ap, 48)
    else:
        ref = recon.CDoSartRecon().DoIt(recon.TiltSeries(binned), ap, 0, T, 48, 3, 4)
    assert got.shape == ref.shape
    assert np.array_equal(got, ref)
