"""Parameter files with the reference's field names and axes
(cmfgpu/params/schema.py:14-140): NetCDF classic written and read back bit
for bit, axis and rank checks, and the container detection that rejects a
NETCDF4 (HDF5) file with the conversion to use."""
import numpy as np
import pytest

from cmfb200 import synthetic as syn
from cmfb200.model import InputProxy
from cmfb200 import params as PR


def _net():
    return syn.generate(syn.NetworkSpec(3000, seed=9, bifurcation_paths=60, levee_fraction=0.2,
                                        reservoirs=8))


def test_netcdf_classic_round_trip(tmp_path):
    net = _net()
    path = tmp_path / "parameters.nc"
    PR.write_parameters(path, net.fields)
    back = InputProxy.from_nc(str(path))
    known = [k for k in net.fields if k in PR.FIELD_DIMS]
    assert set(known) <= set(back)
    for k in known:
        a, b = np.asarray(net.fields[k]), back[k]
        assert a.shape == b.shape, k
        np.testing.assert_array_equal(b, a, err_msg=k)
    # the axes in the file are the reference's names
    from scipy.io import netcdf_file
    with netcdf_file(str(path), "r", mmap=False) as nc:
        assert nc.variables["flood_depth_table"].dimensions == ("catchment", "flood_level")
        assert nc.variables["bifurcation_width"].dimensions == ("bifurcation_path",
                                                                "bifurcation_level")
        assert nc.variables["levee_crown_height"].dimensions == ("levee",)
        assert nc.dimensions["catchment"] == net.num_catchments


def test_npz_and_axis_checks(tmp_path):
    net = _net()
    np.savez(tmp_path / "p.npz", **net.fields)
    back = PR.read_parameters(tmp_path / "p.npz")
    np.testing.assert_array_equal(back["river_width"], net.fields["river_width"])
    bad = dict(net.fields)
    bad["river_width"] = bad["river_width"][:-1]
    with pytest.raises(ValueError, match="catchment"):
        PR.check_fields(bad)
    bad = dict(net.fields)
    bad["flood_depth_table"] = bad["flood_depth_table"][:, 0]
    with pytest.raises(ValueError, match="rank"):
        PR.check_fields(bad)
    bad = {k: v for k, v in net.fields.items() if k != "downstream_id"}
    with pytest.raises(ValueError, match="missing"):
        PR.check_fields(bad)


def test_hdf5_container_is_rejected_with_the_conversion(tmp_path):
    p = tmp_path / "parameters.nc"
    p.write_bytes(b"\x89HDF\r\n\x1a\n" + b"\0" * 64)
    with pytest.raises(ValueError, match="nccopy"):
        PR.read_parameters(p)
