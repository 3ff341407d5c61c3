"""GPU: the batched form (one CUDA graph over several plans) and the slab
autotuner give exactly the per-series plain results."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _series(nx, ny, tilts, vol_z, seed):
    from aretomo3_b200 import synth
    ph = synth.Phantom(seed=seed, n_ellipsoids=30, axis_min=3, axis_max=15, n_beads=3, bead_radius=3)
    return synth.make_tilt_series(nx, ny, tilts, vol_z, ph)


def test_batch_graph_equals_plain_launches():
    import torch
    from aretomo3_b200 import recon
    rng = np.random.default_rng(4)
    cases = []
    for i in range(7):
        nx = int(rng.choice([128, 192, 256, 320]))
        ny = int(rng.integers(3, 12))
        nt = int(rng.integers(21, 42))
        vz = int(rng.integers(32, 100))
        tilts = np.linspace(-60, 60, nt).astype(np.float32)
        sart = i % 3 == 2
        cases.append((nx, ny, tilts, vz, sart))
    plans, projs, vols, refs = [], [], [], []
    for i, (nx, ny, tilts, vz, sart) in enumerate(cases):
        frames = torch.from_numpy(_series(nx, ny, tilts, vz, seed=50 + i)).cuda()
        kw = dict(method=recon.SART, iterations=3, subsets=4) if sart else dict(method=recon.WBP)
        ref, p0 = recon.reconstruct_device(frames, tilts, vz, **kw)
        torch.cuda.synchronize()
        refs.append(ref.cpu().numpy())
        p0.close()
        plan = recon.Plan(nx, ny, tilts, vz, **kw)
        vol = torch.full(plan.volume_shape, float("nan"), device="cuda")
        plans.append(plan)
        projs.append(frames)
        vols.append(vol)
    batch = recon.Batch(plans, [p.data_ptr() for p in projs], [v.data_ptr() for v in vols], branches=3)
    for _ in range(2):   # capture, then replay
        for v in vols:
            v.fill_(float("nan"))
        batch.run(torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        for v, r in zip(vols, refs):
            assert np.array_equal(v.cpu().numpy(), r)
    batch.close()


def test_autotuned_slab_keeps_results():
    import torch
    from aretomo3_b200 import recon
    tilts = np.linspace(-60, 60, 41).astype(np.float32)
    for kw in (dict(method=recon.WBP), dict(method=recon.SART, iterations=2, subsets=5)):
        frames = torch.from_numpy(_series(256, 40, tilts, 64, seed=9)).cuda()
        ref, p0 = recon.reconstruct_device(frames, tilts, 64, **kw)
        torch.cuda.synchronize()
        plan = recon.Plan(256, 40, tilts, 64, **kw)
        out = torch.empty(plan.volume_shape, device="cuda")
        s = torch.cuda.current_stream().cuda_stream
        chosen = plan.autotune(frames.data_ptr(), out.data_ptr(), s)
        assert 1 <= chosen <= 40 and plan.slab == chosen
        out.fill_(float("nan"))
        plan.run_device(frames.data_ptr(), out.data_ptr(), s)
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy(), ref.cpu().numpy())
        plan.close()
        p0.close()


@pytest.mark.parametrize("storage,mode", [(0, "waves"), (1, "waves"), (0, "auto")])
def test_wbp_wave_batch_equals_plain_launches(storage, mode):
    """WBP series of one storage type run as waves of persistent stage
    kernels (one slab of every series per wave, each stage one launch whose
    CTAs pull blocks across all series); uneven sizes and slab counts, so
    series drop out of later waves.  Bit-identical to per-series launches."""
    import torch
    from aretomo3_b200 import recon
    rng = np.random.default_rng(8)
    plans, projs, vols, refs = [], [], [], []
    for i in range(9):
        nx = int(rng.choice([96, 128, 190, 256, 322]))
        ny = int(rng.integers(2, 17))
        nt = int(rng.integers(17, 45))
        vz = int(rng.integers(24, 101))
        slab = int(rng.choice([0, 3, 4, 8]))
        tilts = np.linspace(-58, 61, nt).astype(np.float32)
        frames = torch.from_numpy(_series(nx, ny, tilts, vz, seed=70 + i)).cuda()
        kw = dict(method=recon.WBP, storage=storage, slab_slices=slab)
        ref, p0 = recon.reconstruct_device(frames, tilts, vz, **kw)
        torch.cuda.synchronize()
        refs.append(ref.cpu().numpy())
        p0.close()
        plan = recon.Plan(nx, ny, tilts, vz, **kw)
        plans.append(plan)
        projs.append(frames)
        vols.append(torch.full(plan.volume_shape, float("nan"), device="cuda"))
    batch = recon.Batch(plans, [p.data_ptr() for p in projs], [v.data_ptr() for v in vols], mode=mode)
    for _ in range(2):   # capture (for "auto": both forms, timed), then replay
        for v in vols:
            v.fill_(float("nan"))
        batch.run(torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        for v, r in zip(vols, refs):
            assert np.array_equal(v.cpu().numpy(), r)
    form, ms_w, ms_b = batch.mode
    if mode == "waves":
        assert form == "waves"
    else:
        assert form in ("waves", "branches") and ms_w > 0 and ms_b > 0
    batch.close()
    for p in plans:
        p.close()
