"""The C-ABI library loads here (no GPU) and exports every entry point that
include/sgmas.h declares; the Python binding knows all of them."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "sgmas.h")


def declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(sgmas_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def libpath():
    from sgmas import build
    return build.build()


def test_header_lists_entry_points():
    names = declared()
    assert "sgmas_pcg_solve" in names and "sgmas_mas_assemble" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol(libpath):
    out = subprocess.run(["nm", "-D", "--defined-only", libpath], capture_output=True, text=True, check=True).stdout
    exported = set(line.split()[-1] for line in out.splitlines() if line.strip())
    missing = [n for n in declared() if n not in exported]
    assert not missing, missing


def test_library_loads_without_gpu(libpath):
    import ctypes
    L = ctypes.CDLL(libpath)
    for n in declared():
        assert hasattr(L, n), n


def test_binding_covers_header(libpath):
    import sgmas
    assert sorted(sgmas.EXPORTS) == declared()


def test_create_fails_cleanly_without_gpu(libpath):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import sgmas
    with pytest.raises(sgmas.SgmasError):
        sgmas.Context(0)
