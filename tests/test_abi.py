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


def test_autotune_cache_file_round_trip(ats, tmp_path):
    """The autotuning cache's text file: load merges valid entries, save writes them
    back, a malformed file is rejected whole (no GPU involved)."""
    import pytest
    ats.autotune_cache_clear()
    assert ats.autotune_cache_size() == 0
    src = tmp_path / "tune.txt"
    src.write_text("ats-autotune 2\n"
                   "NVIDIA_B200|148|v22|i6|c4|s7|b11 1 64 0 2 0 1\n"
                   "NVIDIA_B200|148|v18|i0|c4|s6|b10 1 128 0 0 0 0\n")
    ats.autotune_cache_load(str(src))
    assert ats.autotune_cache_size() == 2
    out = tmp_path / "out.txt"
    ats.autotune_cache_save(str(out))
    assert sorted(out.read_text().splitlines()) == sorted(src.read_text().splitlines())
    for bad in ("ats-autotune 1\nk 1 64 0 0 0\n",               # older version
                "ats-autotune 2\nk 3 64 0 0 0 0\n",             # lanes per vertex not 1, 2, 4, 8
                "ats-autotune 2\nk 1 64 0 3 0 0\n",             # list form out of range
                "ats-autotune 2\nk 1 64 0 0 0 2\n",             # persisting flag not 0 or 1
                "ats-autotune 2\nk 1 64\n"):                    # short line
        f = tmp_path / "bad.txt"
        f.write_text(bad)
        with pytest.raises(ats.AtsError) as e:
            ats.autotune_cache_load(str(f))
        assert e.value.status == ats.ATS_ERR_INVALID
        assert ats.autotune_cache_size() == 2
    with pytest.raises(ats.AtsError):
        ats.autotune_cache_load(str(tmp_path / "missing.txt"))
    with pytest.raises(ats.AtsError) as e:
        ats.autotune_cache_save(str(tmp_path))  # a directory
    assert e.value.status == ats.ATS_ERR_INVALID
    ats.autotune_cache_clear()
    assert ats.autotune_cache_size() == 0
