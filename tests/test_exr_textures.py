"""OpenEXR textures in scene files (Texture2D reads them through OpenEXR): scanline files
with HALF / FLOAT channels and NONE, RLE, ZIPS or ZIP compression, written here by an
independent encoder of the published file layout, read back by the library's loader."""
import json
import os
import struct
import zlib

import numpy as np
import pytest

from aurora_b200 import _abi, scenes
from test_scene_file import write_obj, write_single

NONE, RLE, ZIPS, ZIP = 0, 1, 2, 3


def _predict_interleave(raw: bytes) -> bytes:
    n = len(raw)
    t = bytearray(n)
    t[0:(n + 1) // 2] = raw[0::2]
    t[(n + 1) // 2:] = raw[1::2]
    out = bytearray(n)
    prev = 0
    for i in range(n):
        out[i] = t[i] if i == 0 else (t[i] - prev + 128 + 256) & 0xff
        prev = t[i]
    return bytes(out)


def _rle(data: bytes) -> bytes:
    out = bytearray()
    i, n = 0, len(data)
    while i < n:
        run = 1
        while i + run < n and run < 128 and data[i + run] == data[i]:
            run += 1
        if run >= 3:
            out += struct.pack("b", run - 1) + data[i:i + 1]
            i += run
        else:
            j = i
            while j < n and j - i < 127 and not (j + 2 < n and data[j] == data[j + 1] == data[j + 2]):
                j += 1
            out += struct.pack("b", -(j - i)) + data[i:j]
            i = j
    return bytes(out)


def write_exr(path, rgb, comp=NONE, ptype=1, channels="BGR", y_order_reversed=False):
    """rgb (H, W, 3) float32; ptype 1 HALF, 2 FLOAT; channels written in name order."""
    h, w, _ = rgb.shape
    names = sorted(channels)
    idx = {"R": 0, "G": 1, "B": 2}
    hdr = bytearray(struct.pack("<ii", 20000630, 2))

    def attr(name, typ, val):
        hdr.extend(name.encode() + b"\0" + typ.encode() + b"\0" + struct.pack("<i", len(val)) + val)
    ch = b"".join(nm.encode() + b"\0" + struct.pack("<iB3xii", ptype, 0, 1, 1) for nm in names) + b"\0"
    attr("channels", "chlist", ch)
    attr("compression", "compression", bytes([comp]))
    attr("dataWindow", "box2i", struct.pack("<4i", 0, 0, w - 1, h - 1))
    attr("displayWindow", "box2i", struct.pack("<4i", 0, 0, w - 1, h - 1))
    attr("lineOrder", "lineOrder", bytes([1 if y_order_reversed else 0]))
    attr("pixelAspectRatio", "float", struct.pack("<f", 1.0))
    attr("screenWindowCenter", "v2f", struct.pack("<ff", 0, 0))
    attr("screenWindowWidth", "float", struct.pack("<f", 1.0))
    hdr.append(0)
    lines = 16 if comp == ZIP else 1
    dt = np.float16 if ptype == 1 else np.float32
    chunks = []
    for y0 in range(0, h, lines):
        raw = b"".join(np.ascontiguousarray(rgb[y, :, idx[nm]]).astype(dt).tobytes()
                       for y in range(y0, min(h, y0 + lines)) for nm in names)
        if comp == NONE:
            data = raw
        elif comp == RLE:
            data = _rle(_predict_interleave(raw))
        else:
            data = zlib.compress(_predict_interleave(raw))
        if len(data) >= len(raw):
            data = raw                                   # stored raw when compression does not pay
        chunks.append((y0, data))
    if y_order_reversed:
        chunks = chunks[::-1]
    table_at = len(hdr)
    body = bytearray()
    offsets = []
    pos = table_at + 8 * len(chunks)
    for y0, data in chunks:
        offsets.append(pos + len(body))
        body += struct.pack("<ii", y0, len(data)) + data
    with open(path, "wb") as f:
        f.write(bytes(hdr) + b"".join(struct.pack("<Q", o) for o in offsets) + bytes(body))


def _load_texture(tmp_path, name):
    v, f = scenes.quad((-1, -1, 0), (1, -1, 0), (1, 1, 0), (-1, 1, 0))
    write_obj(str(tmp_path / "q.obj"), v, f, normals=np.tile([0, 0, 1.0], (4, 1)))
    shaders = {"tex": {"attributetype": "color", "type": "texture2DShader", "texturename": name}}
    mats = {"m": {"type": "matteMaterial", "color": "tex"}}
    data, _, _ = scenes.load_scene_file(write_single(str(tmp_path), "q.obj", 0, materials=mats, shaders=shaders))
    return data.textures[0]


@pytest.mark.parametrize("comp", [NONE, RLE, ZIPS, ZIP], ids=["none", "rle", "zips", "zip"])
@pytest.mark.parametrize("ptype", [1, 2], ids=["half", "float"])
def test_exr_texture_round_trip(tmp_path, comp, ptype):
    r = np.random.default_rng(comp * 7 + ptype)
    rgb = r.uniform(0, 4, (37, 29, 3)).astype(np.float32)
    rgb[5:20, 3:9] = 0.5                                 # runs for RLE
    write_exr(str(tmp_path / "t.exr"), rgb, comp, ptype)
    got = _load_texture(tmp_path, "t.exr")
    want = rgb.astype(np.float16).astype(np.float32) if ptype == 1 else rgb
    np.testing.assert_array_equal(got, want)


def test_exr_missing_channels_and_decreasing_order(tmp_path):
    rgb = np.random.default_rng(3).uniform(0, 1, (20, 16, 3)).astype(np.float32)
    write_exr(str(tmp_path / "t.exr"), rgb, ZIP, 2, channels="RG", y_order_reversed=True)
    got = _load_texture(tmp_path, "t.exr")
    np.testing.assert_array_equal(got[..., :2], rgb[..., :2])
    assert np.all(got[..., 2] == 0.0)


def test_film_writer_output_is_a_texture(tmp_path):
    """What aur_film_write writes (uncompressed half RGBA) reads back as a texture."""
    import aurora_b200 as ab
    film = np.random.default_rng(5).uniform(0, 3, (11, 13, 4)).astype(np.float32)
    ab.write_film(str(tmp_path / "f.exr"), film, _abi.FILM_EXR_HALF)
    got = _load_texture(tmp_path, "f.exr")
    np.testing.assert_array_equal(got, film[..., :3].astype(np.float16).astype(np.float32))


def test_exr_errors(tmp_path):
    rgb = np.zeros((4, 4, 3), np.float32)
    write_exr(str(tmp_path / "piz.exr"), rgb, ZIP, 1)
    b = bytearray(open(tmp_path / "piz.exr", "rb").read())
    at = b.index(b"compression\0compression\0") + len(b"compression\0compression\0") + 4
    b[at] = 4                                            # PIZ
    open(tmp_path / "piz.exr", "wb").write(bytes(b))
    with pytest.raises(_abi.AuroraError) as e:
        _load_texture(tmp_path, "piz.exr")
    assert e.value.status == _abi.ERR_UNSUPPORTED
    write_exr(str(tmp_path / "cut.exr"), rgb, ZIPS, 1)
    whole = open(tmp_path / "cut.exr", "rb").read()
    open(tmp_path / "cut.exr", "wb").write(whole[:len(whole) - 5])
    with pytest.raises(_abi.AuroraError) as e:
        _load_texture(tmp_path, "cut.exr")
    assert e.value.status == _abi.ERR_PARSE
    with pytest.raises(_abi.AuroraError) as e:
        _load_texture(tmp_path, "missing.exr")
    assert e.value.status == _abi.ERR_IO
