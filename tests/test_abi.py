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


def test_a_c_caller_compiles_links_and_calls_without_a_device(tmp_path, library):
    # the header is plain C (what a Rust `extern "C"` block, cgo or a C
    # caller binds): compiled as C99 with every warning an error, linked
    # against the library, and run for the calls that need no device
    import shutil
    import subprocess
    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    src = tmp_path / "caller.c"
    src.write_text(
        '#include <stdio.h>\n#include "cellweave_b200.h"\n'
        "int main(void) {\n"
        "    cw_lattice lat = 0;\n"
        "    uint32_t w = 0, h = 8, d = 1, cap = 4;\n"
        "    int rc = cw_lattice_create(1, &w, &h, &d, &cap, 10.0, &lat);\n"
        '    printf("%d %d %d\\n", cw_version(), rc, lat == 0);\n'
        '    return cw_last_error()[0] == 0;\n'
        "}\n")
    exe = tmp_path / "caller"
    libdir = os.path.dirname(_lib.LIB_PATH)
    libname = os.path.basename(_lib.LIB_PATH)[3:-3]
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
                    str(src), "-L", libdir, "-l" + libname, "-Wl,-rpath," + libdir, "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0, out.stderr
    version, rc, null = (int(v) for v in out.stdout.split())
    # a zero width is refused (CW_ERR_CONFIG) where there is a device, the
    # call fails as CW_ERR_CUDA where there is none; either way no handle
    # and a message (the exit status above)
    assert version == 1 and rc in (1, 5) and null == 1
