"""The C ABI of libcmfb200: loads without a GPU, exports every declared
symbol, and the ctypes view layout matches the C struct field by field."""
import ctypes

from cmfb200 import _lib


def test_library_loads_and_abi_version():
    h = _lib.lib()
    assert h.cmf_abi_version() == _lib.ABI_VERSION
    assert h.cmf_status_string(_lib.CMF_ERR_ARG) == b"invalid argument"


def test_every_declared_symbol_is_exported():
    h = _lib.lib()
    names = _lib.declared_symbols()
    assert "cmf_step_interval" in names and "cmf_plan_create" in names
    missing = [n for n in names if not hasattr(h, n)]
    assert not missing, missing


def test_view_layout_matches_c():
    h = _lib.lib()
    cap = 128
    offs = (ctypes.c_int64 * cap)()
    n = h.cmf_view_field_offsets(offs, cap)
    fields = [f[0] for f in _lib.CmfView._fields_]
    assert n == len(fields)
    for i, name in enumerate(fields):
        assert getattr(_lib.CmfView, name).offset == offs[i], name
    assert h.cmf_view_size() == ctypes.sizeof(_lib.CmfView)


def test_workspace_size_and_argument_errors():
    h = _lib.lib()
    v = _lib.CmfView()
    v.abi_version = _lib.ABI_VERSION
    v.num_catchments = 1000
    v.num_members = 1
    v.num_flood_levels = 10
    size = ctypes.c_size_t(0)
    assert h.cmf_workspace_size(ctypes.byref(v), ctypes.byref(size)) == 0
    # two flux arrays + two storage buffers at least
    assert size.value >= 1000 * (4 + 4 + 8 + 8)
    # plan creation rejects a view without tensors (no kernel is launched)
    plan = ctypes.c_void_p()
    assert h.cmf_plan_create(ctypes.byref(v), ctypes.byref(plan)) == _lib.CMF_ERR_ARG
    v.abi_version = 999
    assert h.cmf_plan_create(ctypes.byref(v), ctypes.byref(plan)) == _lib.CMF_ERR_ARG
    assert h.cmf_step_interval(None, None, 86400.0, 0) == _lib.CMF_ERR_ARG
    # the plan setters refuse a null plan without touching a device
    assert h.cmf_plan_set_persistent(None, 1) == _lib.CMF_ERR_ARG
    assert h.cmf_plan_set_persistent(None, 0) == _lib.CMF_ERR_ARG
    assert h.cmf_plan_set_member_tile(None, 2) == _lib.CMF_ERR_ARG
    assert h.cmf_probe_barrier_timeout(None, None, None, 10) == _lib.CMF_ERR_ARG
