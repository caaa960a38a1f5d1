"""PFM and CVTRaw files as cvt writes and reads them (PFMSaver / PFMLoader, CVTRawSaver /
CVTRawLoader), through the library's host I/O.  No GPU needed."""
import struct

import numpy as np
import pytest


@pytest.fixture(scope="module")
def io(native):
    from cvt_b200 import imageio

    return imageio


def test_pfm_grey_layout_and_round_trip(io, tmp_path):
    a = np.arange(15, dtype=np.float32).reshape(3, 5) * np.float32(0.25)
    p = tmp_path / "d.pfm"
    io.save_pfm(p, a)
    raw = p.read_bytes()
    hdr = b"Pf\n5 3\n-1.0\n"
    assert raw[:len(hdr)] == hdr
    body = np.frombuffer(raw[len(hdr):], "<f4").reshape(3, 5)
    assert (body == a[::-1]).all()   # rows bottom to top
    assert (io.load_pfm(p) == a).all()


def test_pfm_rgba_drops_alpha_and_loads_opaque(io, tmp_path):
    rng = np.random.default_rng(0)
    a = rng.standard_normal((4, 6, 4)).astype(np.float32)
    p = tmp_path / "n.pfm"
    io.save_pfm(p, a)
    raw = p.read_bytes()
    assert raw.startswith(b"PF\n6 4\n-1.0\n")
    assert len(raw) == len(b"PF\n6 4\n-1.0\n") + 4 * 6 * 3 * 4
    b = io.load_pfm(p)
    assert (b[..., :3] == a[..., :3]).all() and (b[..., 3] == 1.0).all()


def test_pfm_big_endian_and_comments(io, tmp_path):
    a = np.array([[1.5, -2.0], [3.25, 1e-20]], np.float32)
    p = tmp_path / "be.pfm"
    p.write_bytes(b"# written elsewhere\nPf\n# size\n2 2\n1.0\n" + a[::-1].astype(">f4").tobytes())
    assert (io.load_pfm(p) == a).all()


def test_pfm_errors(io, tmp_path):
    from cvt_b200 import StereoError

    p = tmp_path / "bad.pfm"
    p.write_bytes(b"P6\n2 2\n255\n")
    with pytest.raises(StereoError, match="Unknown PFM type"):
        io.load_pfm(p)
    p.write_bytes(b"Pf\n4 4\n-1.0\n" + b"\0" * 20)
    with pytest.raises(StereoError, match="not enough data"):
        io.load_pfm(p)
    with pytest.raises(StereoError):
        io.load_pfm(tmp_path / "missing.pfm")


@pytest.mark.parametrize("kind", ["gray", "rgba8", "rgbaf", "flow"])
def test_cvtraw_layout_and_round_trip(io, tmp_path, kind):
    rng = np.random.default_rng(1)
    a = {"gray": rng.random((5, 7), np.float32), "rgba8": rng.integers(0, 256, (5, 7, 4), dtype=np.uint8),
         "rgbaf": rng.standard_normal((5, 7, 4)).astype(np.float32),
         "flow": rng.standard_normal((5, 7, 2)).astype(np.float32)}[kind]
    fid = {"gray": 4, "rgba8": 9, "rgbaf": 12, "flow": 8}[kind]
    p = tmp_path / "x.cvtraw"
    io.save_cvtraw(p, a)
    raw = p.read_bytes()
    assert struct.unpack("<4I", raw[:16]) == (7, 5, a.strides[0], fid)
    assert raw[16:] == a.tobytes()
    b = io.load_cvtraw(p)
    assert b.dtype == a.dtype and b.shape == a.shape and (b.view(np.uint8) == a.view(np.uint8)).all()


def test_cvtraw_padded_stride_loads(io, tmp_path):
    a = np.arange(24, dtype=np.float32).reshape(4, 6)
    padded = np.zeros((4, 8), np.float32)
    padded[:, :6] = a
    p = tmp_path / "pad.cvtraw"
    p.write_bytes(struct.pack("<4I", 6, 4, 32, 4) + padded.tobytes())
    assert (io.load_cvtraw(p) == a).all()


def test_round_trips_of_random_shapes_and_values(io, tmp_path):
    """Hypothesis draws shapes (1x1 upwards, odd sizes) and values (NaN, infinities, signed
    zeros and subnormals included): CVTRaw keeps every bit of every format; PFM keeps every bit
    of its float channels (alpha reads back as 1)."""
    from hypothesis import HealthCheck, given, settings
    from hypothesis import strategies as st

    floats = st.floats(width=32, allow_nan=True, allow_infinity=True, allow_subnormal=True)

    @settings(max_examples=60, deadline=None, suppress_health_check=[HealthCheck.function_scoped_fixture])
    @given(h=st.integers(1, 9), w=st.integers(1, 11), kind=st.sampled_from(["gray", "rgba8", "rgbaf", "flow"]),
           data=st.data())
    def check(h, w, kind, data):
        ch = {"gray": 1, "rgba8": 4, "rgbaf": 4, "flow": 2}[kind]
        n = h * w * ch
        if kind == "rgba8":
            vals = data.draw(st.lists(st.integers(0, 255), min_size=n, max_size=n))
            a = np.array(vals, np.uint8)
        else:
            a = np.array(data.draw(st.lists(floats, min_size=n, max_size=n)), np.float32)
        a = a.reshape((h, w) if ch == 1 else (h, w, ch))
        p = tmp_path / "r.cvtraw"
        io.save_cvtraw(p, a)
        b = io.load_cvtraw(p)
        assert b.shape == a.shape and (b.view(np.uint8) == a.view(np.uint8)).all()
        if kind in ("gray", "rgbaf"):
            q = tmp_path / "r.pfm"
            io.save_pfm(q, a)
            c = io.load_pfm(q)
            got = c if kind == "gray" else c[..., :3]
            want = a if kind == "gray" else a[..., :3]
            assert (got.view(np.uint32) == want.view(np.uint32)).all()
            if kind == "rgbaf":
                assert (c[..., 3] == 1.0).all()

    check()
