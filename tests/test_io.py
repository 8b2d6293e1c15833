"""On-disk formats: OBJ export and the checksummed binary cloth state (host only)."""
import numpy as np
import pytest


def test_obj_write_read_roundtrip(ats, tmp_path):
    pos, faces = ats.grid_mesh(9, ats.GRID_ALTERNATING)
    pos = pos + np.float32(0.125)
    p = str(tmp_path / "frame.obj")
    ats.obj_write(p, pos, faces)
    p2, f2 = ats.obj_read(p)
    assert np.array_equal(f2, faces)
    assert np.array_equal(p2, pos)


def test_state_roundtrip_and_checks(ats, tmp_path):
    rng = np.random.RandomState(0)
    x = rng.standard_normal((1000, 3)).astype(np.float32)
    v = rng.standard_normal((1000, 3)).astype(np.float32)
    p = str(tmp_path / "s.bin")
    ats.state_write(p, x, v, frame=42)
    x2, v2, fr = ats.state_read(p)
    assert fr == 42 and np.array_equal(x, x2) and np.array_equal(v, v2)
    raw = bytearray(open(p, "rb").read())
    assert raw[:4] == b"ATSS" and len(raw) == 16 + 24 * 1000 + 8
    raw[100] ^= 1
    open(p, "wb").write(bytes(raw))
    with pytest.raises(ats.AtsError, match="checksum"):
        ats.state_read(p)
    open(p, "wb").write(bytes(raw[:50]))
    with pytest.raises(ats.AtsError, match="truncated"):
        ats.state_read(p)
    open(p, "wb").write(b"NOPE" + bytes(20))
    with pytest.raises(ats.AtsError, match="not a cloth state"):
        ats.state_read(p)


def test_obj_polygons_become_triangle_fans(ats, tmp_path):
    # a quad, a pentagon with texture/normal indices, a negative (relative) index face
    # and a degenerate triangle that is dropped
    p = tmp_path / "poly.obj"
    p.write_text("v 0 0 0\nv 1 0 0\nv 1 0 1\nv 0 0 1\nv 2 0 0\nv 2 0 1\n"
                 "f 1 2 3 4\nf 2/1/1 5/2/1 6/3/1 3/4/1 1/5/1\nf -1 -2 -3\nf 1 1 2\n")
    pos, faces = ats.obj_read(str(p))
    assert pos.shape == (6, 3)
    expect = [[0, 1, 2], [0, 2, 3], [1, 4, 5], [1, 5, 2], [1, 2, 0], [5, 4, 3]]
    assert faces.tolist() == expect
