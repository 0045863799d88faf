"""The C-ABI library loads on a machine without a GPU and exports every
function that include/*.h declares (no compute calls here)."""
import ctypes
import os
import re

import pytest

from molecular2_b200 import engine

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if not f.endswith(".h"):
            continue
        txt = open(os.path.join(inc, f)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(jk_\w+)\s*\(", txt, re.M):
            names.add(m.group(1))
    return names


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("jk_create", "jk_destroy", "jk_last_error", "jk_direct", "jk_schwarz"):
        assert must in names


def test_library_exports_every_declared_symbol():
    if not os.path.exists(engine.LIBPATH):
        pytest.fail("libm2jk.so not built (python -m molecular2_b200.build)")
    lib = ctypes.CDLL(engine.LIBPATH)
    missing = [n for n in sorted(declared_functions()) if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_signatures_cover_header():
    assert declared_functions() <= set(engine.SIGNATURES), declared_functions() - set(engine.SIGNATURES)


def test_create_without_device_fails_cleanly():
    """On a host without a GPU jk_create must return an error, not crash."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from molecular2_b200 import geometry
    from molecular2_b200.basis import BasisSet
    b = BasisSet(geometry.water(), "cc-pvdz")
    with pytest.raises(engine.JKError):
        engine.IntegralEngine(b)
