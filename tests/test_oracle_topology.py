"""The oracle's network-generation helpers (oracle/topology.py, C in
oracle/cmf_oracle.c) equal the product's (cmfb200.topology, libcmfb200) bit
for bit, so a process that builds a workload through the oracle -- the
reference arm of bench.py, which must not load the product library -- routes
the identical network."""
import ctypes

import numpy as np

from cmfb200 import synthetic as syn, topology as T
from oracle import topology as OT


def test_helpers_equal_product_helpers():
    rng = np.random.default_rng(3)
    n = 5000
    idx = np.arange(n)
    dn = np.minimum(idx + rng.integers(1, 50, size=n), n - 1)
    mouth = rng.random(n) < 0.05
    dn[mouth] = idx[mouth]
    dn[-1] = n - 1
    dn = dn.astype(np.int32)
    v = rng.uniform(1, 100, size=n)
    np.testing.assert_array_equal(OT.accumulate_upstream(dn, v), T.accumulate_upstream(dn, v))
    np.testing.assert_array_equal(OT.accumulate_downstream(dn, v), T.accumulate_downstream(dn, v))
    elev = rng.uniform(0, 500, size=n).astype(np.float32)
    hgt = rng.uniform(0.5, 15, size=n).astype(np.float32)
    np.testing.assert_array_equal(OT.init_river_depth(elev, hgt, dn), T.init_river_depth(elev, hgt, dn))


def test_generated_networks_equal():
    spec = syn.NetworkSpec(20_000, seed=4, bifurcation_paths=300, levee_fraction=0.2,
                           reservoirs=20)
    a = syn.generate(spec)
    b = syn.generate(spec, topo=OT)
    assert a.fields.keys() == b.fields.keys()
    for k in a.fields:
        np.testing.assert_array_equal(a.fields[k], b.fields[k], err_msg=k)


def test_helpers_take_large_arrays():
    """Arrays of a few MB live in separately mapped memory at addresses above
    4 GiB; the helpers must pass them as full 64-bit pointers (the reference
    arm of bench.py builds the 6M-catchment network through them)."""
    rng = np.random.default_rng(7)
    n = 1_500_000
    idx = np.arange(n)
    dn = np.minimum(idx + rng.integers(1, 200, size=n), n - 1).astype(np.int32)
    dn[-1] = n - 1
    v = rng.uniform(1, 100, size=n)
    # a bare Python int would be passed as a 32-bit C int
    assert isinstance(OT._p(v), ctypes.c_void_p) and OT._p(v).value == v.ctypes.data
    np.testing.assert_array_equal(OT.accumulate_upstream(dn, v), T.accumulate_upstream(dn, v))
    elev = rng.uniform(0, 500, size=n).astype(np.float32)
    hgt = rng.uniform(0.5, 15, size=n).astype(np.float32)
    np.testing.assert_array_equal(OT.init_river_depth(elev, hgt, dn), T.init_river_depth(elev, hgt, dn))
