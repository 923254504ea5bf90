"""The C-ABI library: builds for sm_100a, loads, and exports every symbol include/hgx.h declares.
No compute call is made here (CPU only)."""
import ctypes
import os
import re

import pytest

from hypergraphrewritingengine_b200 import api, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    text = open(os.path.join(ROOT, "include", "hgx.h")).read()
    return sorted(set(re.findall(r"HGX_API\s+[\w\s\*]+?\b(hgx_\w+)\s*\(", text)))


def test_header_declarations_are_listed():
    assert _declared() == sorted(api.EXPORTS)


def test_library_exports_every_declared_symbol():
    build.build()
    lib = ctypes.CDLL(build.LIB)
    for name in _declared():
        assert hasattr(lib, name), name


def test_library_is_built_for_sm100a():
    build.build()
    data = open(build.LIB, "rb").read()
    assert b"sm_100a" in data


def test_no_device_fails_loudly():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    L = api.load_library()
    h = ctypes.c_void_p()
    st = L.hgx_engine_create(0, ctypes.byref(h))
    assert st == api.HGX_ERR_NO_DEVICE
    assert b"no CUDA device" in L.hgx_last_error()


def test_rule_builder_limits_match_reference():
    with pytest.raises(ValueError):
        api.make_rule(0).lhs([0, 32])
    with pytest.raises(ValueError):
        api.make_rule(0).lhs(list(range(17)))
    b = api.make_rule(0)
    for _ in range(16):
        b.lhs([0, 1])
    with pytest.raises(ValueError):
        b.lhs([0, 1])
    r = api.make_rule(3).lhs([0, 1]).lhs([0, 2]).rhs([0, 2]).rhs([0, 3]).build()
    assert r.index == 3 and r.new_var_mask() == 1 << 3


def test_blob_encodings():
    b = api.encode_rules([([[0, 1], [1, 2]], [[0, 1], [1, 2], [2, 0]])])
    assert b.tolist() == [1, 2, 2, 0, 1, 2, 1, 2, 3, 2, 0, 1, 2, 1, 2, 2, 2, 0]
    r = api.encode_roots([[[1, 2], [2, 3]]])
    assert r.tolist() == [1, 2, 2, 1, 2, 2, 2, 3]
