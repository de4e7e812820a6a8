"""The C-ABI library loads and exports every entry point include/csd_capi.h
declares (no compute calls: runs without a GPU)."""
import ctypes
import os
import re

from csdecomp_b200 import _capi

HEADER = os.path.join(os.path.dirname(__file__), "..", "include", "csd_capi.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(csd_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_the_binding_table():
    assert sorted(_capi.EXPORTS) == declared_functions()


def test_library_exports_all_symbols():
    lib = ctypes.CDLL(_capi.LIB_PATH)
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_version_and_pure_host_helpers():
    assert _capi.lib().csd_version() >= 10000
    assert _capi.lib().csd_num_samples_unadaptive(0.01, 0.05, 0.5) == 2397


def test_batch_shape_counts_match_the_python_names():
    from csdecomp_b200.api import BatchedEdgeInflator
    ns, nc = ctypes.c_int32(-1), ctypes.c_int32(-1)
    _capi.lib().csd_batch_shape_counts(ctypes.byref(ns), ctypes.byref(nc))
    assert ns.value == len(BatchedEdgeInflator.SAMPLE_VARIANTS)
    assert nc.value == len(BatchedEdgeInflator.CHECK_ITEM_CAPS)
