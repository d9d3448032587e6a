"""The C-ABI library loads and exports every entry point include/vfray.h
declares (no GPU needed: nothing is called that touches the device)."""
import os
import re

import vfray_b200 as vb
from vfray_b200 import _lib

from tests.conftest import ROOT


def declared():
    names = []
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            src = open(os.path.join(ROOT, "include", fn)).read()
            names += re.findall(r"VFR_API\s+[\w\s\*]*?\b(vfr_\w+)\s*\(", src)
    return names


def test_every_declared_symbol_is_exported():
    lib = vb.load()
    names = declared()
    assert len(names) >= 30
    for n in names:
        assert hasattr(lib, n), n


def test_binding_covers_the_header():
    assert set(declared()) <= set(_lib.SIGNATURES)


def test_status_strings():
    lib = vb.load()
    for rc in range(0, -10, -1):
        s = lib.vfr_status_string(rc).decode()
        assert s and s != "unknown status"


def test_missing_library_fails_loudly(tmp_path):
    import pytest

    old = _lib._LIB
    try:
        _lib._LIB = None
        with pytest.raises(ImportError):
            _lib.load(str(tmp_path / "nope.so"))
    finally:
        _lib._LIB = old


def test_checked_build_alone_has_its_test_hook():
    """The checked build (-DVFR_CHECKED) is built beside the product library
    and exports the same entry points plus its test hook, which the product
    library does not have."""
    import ctypes

    path = os.path.join(ROOT, "vfray_b200", "libvfray_b200_checked.so")
    assert os.path.exists(path), "build it with `make -C vfray_b200 checked`"
    checked = ctypes.CDLL(path)
    for n in declared():
        assert hasattr(checked, n), n
    assert hasattr(checked, "vfr_checked_set_id")
    assert not hasattr(vb.load(), "vfr_checked_set_id")
