"""Host-side helpers of bench.py that need no GPU: the volume checksums the
batched-form comparison relies on when no second copy of the volumes fits,
and the uneven series of the batched workload."""
import os
import sys

import numpy as np
import torch

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def test_volume_sums_equal_for_equal_volumes_and_differ_for_one_bit():
    rng = np.random.default_rng(3)
    a = torch.from_numpy(rng.standard_normal((37, 5, 9)).astype(np.float32))
    b = a.clone()
    assert bench.volume_sums(a, chunk=4) == bench.volume_sums(b, chunk=16)
    # one flipped bit anywhere changes the pair
    for idx in [(0, 0, 0), (36, 4, 8), (17, 2, 3)]:
        c = a.clone()
        w = c.view(torch.int32)
        w[idx] ^= 1 << 7
        assert bench.volume_sums(c) != bench.volume_sums(a)
    # moved words keep the plain sum but not the position-weighted one
    d = a.clone()
    d[0, 0, 0], d[0, 0, 1] = a[0, 0, 1].item(), a[0, 0, 0].item()
    assert bench.volume_sums(d)[0] == bench.volume_sums(a)[0]
    assert bench.volume_sums(d)[1] != bench.volume_sums(a)[1]
    e = a.clone()
    e[3], e[4] = a[4].clone(), a[3].clone()
    assert bench.volume_sums(e)[0] == bench.volume_sums(a)[0]
    assert bench.volume_sums(e)[1] != bench.volume_sums(a)[1]


def test_volume_sums_see_nan_markers():
    a = torch.zeros((4, 3, 3), dtype=torch.float32)
    b = a.clone()
    b[2, 1, 1] = float("nan")
    assert bench.volume_sums(a) != bench.volume_sums(b)


def test_batch_specs_are_the_stated_uneven_series():
    specs = bench.batch_specs(64)
    assert len(specs) == 64
    for c in specs:
        assert 512 <= c["nx"] <= 2048 and c["nx"] % 256 == 0
        assert 512 <= c["ny"] <= 2048 and c["ny"] % 256 == 0
        assert 31 <= len(c["tilts"]) <= 61
        assert 128 <= c["vol_z"] <= 600
    assert bench.batch_specs(64)[5]["nx"] == specs[5]["nx"]   # seeded
