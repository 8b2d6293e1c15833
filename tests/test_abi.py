"""The C-ABI library loads without a GPU and exports every symbol include/*.h declares."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    inc = os.path.join(ROOT, "include")
    for fn in os.listdir(inc):
        if not fn.endswith(".h"):
            continue
        src = open(os.path.join(inc, fn)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"//[^\n]*", "", src)
        for m in re.finditer(r"\b(?:int|const char\s*\*|void)\s+(ats_\w+)\s*\(", src):
            names.add(m.group(1))
    return names


def test_library_exports_declared_symbols(ats):
    lib = ctypes.CDLL(ats.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 25 and "ats_last_error" in names
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_host_only_calls_work_without_gpu(ats):
    pos, faces = ats.grid_mesh(8)
    assert pos.shape == (64, 3) and faces.shape == (98, 3)
    assert ats.lib().ats_last_error() is not None


def test_invalid_arguments_report_errors(ats):
    import pytest
    with pytest.raises(ats.AtsError) as e:
        ats.grid_mesh(1)
    assert e.value.status == ats.ATS_ERR_INVALID
    assert b"n >= 2" in ats.lib().ats_last_error()
