"""The C ABI library loads without a GPU and exports every function that
include/mat3d_b200.h declares.  No compute call is made.  CPU only."""
import ctypes
import os
import re

import pytest

import mat3d_b200 as m3d

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    txt = open(os.path.join(ROOT, "include", "mat3d_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(m3d(?:2d|rec)?_[a-z_0-9]+)\s*\(", txt)))


@pytest.mark.skipif(not os.path.exists(m3d.LIB_PATH), reason="library not built")
def test_exports():
    L = ctypes.CDLL(m3d.LIB_PATH)
    names = declared()
    assert len(names) >= 14
    for n in names:
        assert hasattr(L, n), n
    assert set(m3d.EXPORTS) == set(names)


@pytest.mark.skipif(not os.path.exists(m3d.LIB_PATH), reason="library not built")
def test_status_strings_and_version():
    L = m3d.load_library()
    assert L.m3d_abi_version() == 2
    assert L.m3d_status_string(0) == b"ok"
    assert b"iteration cap" in L.m3d_status_string(4)


def test_missing_library_fails_loudly(tmp_path):
    with pytest.raises(ImportError):
        m3d.load_library(str(tmp_path / "nope.so"))
