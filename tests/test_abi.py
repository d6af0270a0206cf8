"""The C ABI library loads and exports what include/cellweave_b200.h declares (CPU)."""
import ctypes
import os
import re

import pytest

from cellweave_b200 import _lib, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    text = open(os.path.join(ROOT, "include", "cellweave_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cw_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def library():
    build.build()
    return ctypes.CDLL(_lib.LIB_PATH)


def test_every_declared_symbol_is_exported(library):
    names = declared()
    assert len(names) > 40
    missing = [n for n in names if not hasattr(library, n)]
    assert not missing, missing


def test_the_binding_covers_every_declared_symbol():
    assert sorted(set(declared()) - set(_lib.SIGNATURES)) == []


def test_the_integration_guide_maps_every_declared_symbol():
    guide = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    assert [n for n in declared() if not re.search(r"\b%s\b" % n, guide)] == []


def test_without_a_device_calls_fail_loudly():
    import cellweave_b200 as cw
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(cw.CudaError):
        cw.ScalarField.new(8, 8, 0.2)


def test_version_and_error_string(library):
    L = _lib.lib()
    assert L.cw_version() >= 1
    assert isinstance(L.cw_last_error(), bytes)
