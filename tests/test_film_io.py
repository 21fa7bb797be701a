"""aur_film_write: OpenEXR (uncompressed scanline, half or float RGBA) and PFM, read back by
an independent reader of the published file layouts."""
import struct

import numpy as np
import pytest

from aurora_b200 import _abi


def read_exr(path):
    """Minimal reader of single-part, uncompressed scanline OpenEXR files."""
    b = open(path, "rb").read()
    assert struct.unpack_from("<i", b, 0)[0] == 20000630
    assert struct.unpack_from("<i", b, 4)[0] & 0xff == 2
    pos, attrs = 8, {}
    while b[pos] != 0:
        end = b.index(b"\0", pos); name = b[pos:end].decode(); pos = end + 1
        end = b.index(b"\0", pos); typ = b[pos:end].decode(); pos = end + 1
        size = struct.unpack_from("<i", b, pos)[0]; pos += 4
        attrs[name] = (typ, b[pos:pos + size]); pos += size
    pos += 1
    chans, q = [], 0
    raw = attrs["channels"][1]
    while raw[q] != 0:
        end = raw.index(b"\0", q); cname = raw[q:end].decode(); q = end + 1
        ptype = struct.unpack_from("<i", raw, q)[0]; q += 16
        chans.append((cname, ptype))
    assert attrs["compression"][1] == b"\0"
    x0, y0, x1, y1 = struct.unpack("<4i", attrs["dataWindow"][1])
    w, h = x1 - x0 + 1, y1 - y0 + 1
    offsets = struct.unpack_from(f"<{h}Q", b, pos)
    out = {c: np.zeros((h, w), np.float32) for c, _ in chans}
    for off in offsets:
        y, size = struct.unpack_from("<ii", b, off)
        p = off + 8
        for c, t in chans:
            dt = np.float16 if t == 1 else np.float32
            n = w * np.dtype(dt).itemsize
            out[c][y - y0] = np.frombuffer(b[p:p + n], dt).astype(np.float32)
            p += n
        assert p - off - 8 == size
    return np.stack([out["R"], out["G"], out["B"], out["A"]], -1), attrs


def read_pfm(path):
    b = open(path, "rb").read()
    parts = b.split(b"\n", 3)
    assert parts[0] == b"PF"
    w, h = map(int, parts[1].split())
    assert float(parts[2]) < 0
    return np.frombuffer(parts[3], "<f4").reshape(h, w, 3)[::-1]


@pytest.fixture
def film():
    f = np.random.default_rng(4).uniform(0, 20, (17, 23, 4)).astype(np.float32)
    f[..., 3] = np.random.default_rng(5).uniform(0, 1, (17, 23))
    return f


def test_exr_half_and_float(tmp_path, film):
    import aurora_b200 as ab
    for fmt, conv in ((_abi.FILM_EXR_HALF, lambda a: a.astype(np.float16).astype(np.float32)),
                      (_abi.FILM_EXR_FLOAT, lambda a: a)):
        p = str(tmp_path / f"f{fmt}.exr")
        ab.write_film(p, film, fmt)
        got, attrs = read_exr(p)
        assert attrs["lineOrder"][1] == b"\0" and struct.unpack("<f", attrs["pixelAspectRatio"][1])[0] == 1.0
        np.testing.assert_array_equal(got, conv(film))


def test_pfm(tmp_path, film):
    import aurora_b200 as ab
    p = str(tmp_path / "f.pfm")
    ab.write_film(p, film, _abi.FILM_PFM)
    np.testing.assert_array_equal(read_pfm(p), film[..., :3])


def test_film_write_errors(tmp_path, film):
    import aurora_b200 as ab
    with pytest.raises(_abi.AuroraError) as e:
        ab.write_film(str(tmp_path / "no" / "dir.exr"), film)
    assert e.value.status == _abi.ERR_IO
    with pytest.raises(_abi.AuroraError) as e:
        ab.write_film(str(tmp_path / "x.exr"), film, 7)
    assert e.value.status == _abi.ERR_INVALID_ARG
