"""Import pieces of the reference Python package in THIS container only.

The reference (`cmfgpu`) needs `hydroforge`, `netCDF4` and `cftime`, none of
which exist here.  For generating golden vectors we load individual reference
files directly and satisfy those imports with inert stand-ins (a module whose
every attribute is a do-nothing class).  Only the numba/numpy functions and
plain property bodies of the reference are executed; nothing of hydroforge is
emulated.  Used by make_topology_golden.py; never imported by tests at run
time (the reference tree does not exist on the GPU box).
"""
from __future__ import annotations

import importlib.abc
import importlib.machinery
import importlib.util
import os
import sys
import types

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", ".."))
from oracle.refroot import reference_root  # noqa: E402

_root = reference_root()
if _root is None:
    raise RuntimeError("the reference checkout is not available (set CMF_REFERENCE_ROOT)")
REF = str(_root)
STUBBED = ("hydroforge", "netCDF4", "cftime")


class _Inert:
    def __init__(self, *a, **k):
        pass

    def __call__(self, *a, **k):
        # used as a decorator factory: hand the decorated object back
        if len(a) == 1 and not k and (callable(a[0]) or hasattr(a[0], "__get__")):
            return a[0]
        return self

    def __getattr__(self, k):
        return _Inert()

    def __class_getitem__(cls, k):
        return cls


class _InertModule(types.ModuleType):
    def __getattr__(self, k):
        if k.startswith("__"):
            raise AttributeError(k)
        return type(k, (_Inert,), {})


class _Finder(importlib.abc.MetaPathFinder, importlib.abc.Loader):
    def find_spec(self, name, path, target=None):
        if name.split(".")[0] in STUBBED:
            return importlib.machinery.ModuleSpec(name, self, is_package=True)
        return None

    def create_module(self, spec):
        m = _InertModule(spec.name)
        m.__path__ = []
        return m

    def exec_module(self, module):
        pass


def install() -> None:
    if not any(isinstance(f, _Finder) for f in sys.meta_path):
        sys.meta_path.insert(0, _Finder())
    for name, sub in (("cmfgpu", "cmfgpu"), ("cmfgpu.params", "cmfgpu/params"),
                      ("cmfgpu.modules", "cmfgpu/modules")):
        if name not in sys.modules:
            m = types.ModuleType(name)
            m.__path__ = [os.path.join(REF, sub)]
            sys.modules[name] = m
    # schema.py builds tables from hydroforge at import; utils.py only needs
    # its name to exist.
    if "cmfgpu.params.schema" not in sys.modules:
        m = types.ModuleType("cmfgpu.params.schema")
        m.PARAMETER_MODULE_FIELDS = {}
        sys.modules["cmfgpu.params.schema"] = m


def load(name: str, relpath: str):
    install()
    if name in sys.modules and hasattr(sys.modules[name], "__file__"):
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(REF, relpath))
    m = importlib.util.module_from_spec(spec)
    sys.modules[name] = m
    spec.loader.exec_module(m)
    return m
