"""GPU: the serving loop.  A series gives the same volume whether it runs
alone or in a concurrent mix of WBP and SART requests of different sizes and
storage forms; admission keeps the admitted bytes within the HBM budget; a
series larger than the budget is refused at submission."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _series(nx, ny, tilts, vol_z, seed):
    from aretomo3_b200 import synth
    ph = synth.Phantom(seed=seed, n_ellipsoids=30, axis_min=3, axis_max=15, n_beads=3, bead_radius=3)
    return synth.make_tilt_series(nx, ny, tilts, vol_z, ph)


def _mix(n, seed):
    from aretomo3_b200 import recon
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        nx = int(rng.choice([128, 160, 256, 322]))
        ny = int(rng.integers(2, 40))
        nt = int(rng.integers(15, 45))
        vz = int(rng.integers(24, 96))
        tilts = np.linspace(-58, 61, nt).astype(np.float32)
        if i % 3 == 1:
            kw = dict(method=recon.SART, iterations=3, subsets=int(rng.integers(1, 6)))
        else:
            kw = dict(method=recon.WBP)
        kw["storage"] = int(rng.choice([recon.STORE_F32, recon.STORE_F16, recon.STORE_BF16]))
        out.append((_series(nx, ny, tilts, vz, seed=100 + i), tilts, vz, kw))
    return out


def _alone(frames, tilts, vz, kw):
    from aretomo3_b200 import recon
    T, ny, nx = frames.shape
    plan = recon.Plan(nx, ny, tilts, vz, **kw)
    try:
        vol = np.empty(plan.volume_shape, np.float32)
        plan.run_host([frames[t] for t in range(T)], [vol[y] for y in range(ny)])
        return vol
    finally:
        plan.close()


def test_same_alone_and_in_the_mix():
    from aretomo3_b200 import recon
    mix = _mix(12, seed=21)
    alone = [_alone(*m) for m in mix]
    srv = recon.Server(max_inflight=4)
    try:
        ids = [srv.submit(f, t, vz, **kw) for f, t, vz, kw in mix]
        for rid, ref in zip(ids, alone):
            vol, lat, queued = srv.wait(rid)
            assert 0.0 <= queued <= lat
            assert np.array_equal(vol, ref)
    finally:
        srv.close()


def test_budget_bounds_admission_and_refuses_oversize():
    from aretomo3_b200 import recon
    mix = _mix(6, seed=22)
    need = [recon.estimate_bytes(f.shape[2], f.shape[1], t, vz, **kw) for f, t, vz, kw in mix]
    alone = [_alone(*m) for m in mix]
    budget = 2 * max(need) + (1 << 20)   # about two requests at a time
    srv = recon.Server(hbm_budget_bytes=budget, max_inflight=4)
    try:
        big = np.zeros((41, 8, 4098), np.float32)   # 8 rows of a 4098-wide series, 1200 thick
        assert recon.estimate_bytes(4098, 8, np.linspace(-60, 60, 41), 1200, method=recon.SART) > budget
        with pytest.raises(recon.ReconError) as e:
            srv.submit(big, np.linspace(-60, 60, 41), 1200, method=recon.SART, iterations=2)
        assert e.value.status == 5   # AT3R_ERR_TOO_LARGE
        ids = [srv.submit(f, t, vz, **kw) for f, t, vz, kw in mix]
        peak = 0
        for rid, ref in zip(ids, alone):
            peak = max(peak, srv.in_use_bytes)
            vol, lat, queued = srv.wait(rid)
            assert np.array_equal(vol, ref)
        assert peak <= budget
        assert srv.in_use_bytes == 0
    finally:
        srv.close()
