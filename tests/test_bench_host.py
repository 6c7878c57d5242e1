"""Host-side pieces of bench.py, on CPU: the byte models behind the roofline
fractions and the end-state fingerprint of the ensemble check."""
import numpy as np
import torch

import bench as B


def test_algorithmic_bytes_of_the_roofline_workload():
    # 6M catchments, 200k paths, 977,336 levees, 7k reservoirs: 206.7 B per catchment
    b = B.algorithmic_bytes(6_000_000, 200_000, 977_336, 7_000, True)
    assert b == 1_240_345_376.0
    assert abs(b / 6_000_000 - 206.72) < 0.01
    # plain physics: 172 B per catchment, the paths and levees do not count
    assert B.algorithmic_bytes(60_000, 5, 5, 5, False) == 172.0 * 60_000


def test_fp64_algorithmic_bytes_per_catchment():
    assert B.fp64_algorithmic_bytes(1, 0, 0, 0) == 343.0
    assert B.fp64_algorithmic_bytes(0, 1, 1, 1) == 296.0 + 28.0 + 72.0


def test_bit_sums_see_one_flipped_bit_and_split_members():
    rng = np.random.default_rng(2)
    x = torch.as_tensor(rng.standard_normal((1000, 4)))            # fp64 [N, M]
    y = torch.as_tensor(rng.standard_normal((1000, 4)).astype(np.float32))
    sx, sy = B._bit_sums(x), B._bit_sums(y)
    assert sx.shape == (4,) and sy.shape == (4,)
    for m in range(4):                                             # [N] equals its column
        assert int(B._bit_sums(x[:, m].contiguous())) == int(sx[m])
        assert int(B._bit_sums(y[:, m].contiguous())) == int(sy[m])
    x2 = x.clone()
    x2[17, 2] = np.nextafter(float(x2[17, 2]), np.inf)             # one ulp
    s2 = B._bit_sums(x2)
    assert int(s2[2]) != int(sx[2]) and torch.equal(s2[[0, 1, 3]], sx[[0, 1, 3]])
    y2 = y.clone()
    y2[5, 0] = -y2[5, 0]                                           # a sign bit
    assert int(B._bit_sums(y2)[0]) != int(sy[0])
