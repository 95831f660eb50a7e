"""The PNG of a frame (fae_call "encode_png", ffb_encode_png): RGBA8 with
the config and the render's numbers in tEXt chunks under the reference's
keys and formats (src/png_metadata.rs:144-183; the reference's own test,
python/tests/test_render.py:44-49, looks for Config, Iterations,
IterationsPerThread and RenderTime).  Encoding needs no GPU; the decoder
here checks every chunk's CRC and undoes every filter type."""

import hashlib
import json
import struct
import zlib

import numpy as np
import pytest

from ffb200 import synthetic


def decode(png):
    assert png[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat, text, hdr = 8, b"", {}, None
    while pos < len(png):
        n, = struct.unpack(">I", png[pos:pos + 4])
        kind = png[pos + 4:pos + 8]
        data = png[pos + 8:pos + 8 + n]
        crc, = struct.unpack(">I", png[pos + 8 + n:pos + 12 + n])
        assert zlib.crc32(kind + data) & 0xFFFFFFFF == crc, kind
        if kind == b"IHDR":
            hdr = struct.unpack(">IIBBBBB", data)
        elif kind == b"tEXt":
            k, v = data.split(b"\0", 1)
            text[k.decode("latin-1")] = v.decode("latin-1")
        elif kind == b"IDAT":
            idat += data
        pos += 12 + n
        if kind == b"IEND":
            break
    w, h, depth, ctype, _, _, _ = hdr
    assert (depth, ctype) == (8, 6)
    raw = zlib.decompress(idat)
    stride = w * 4
    out = np.zeros((h, stride), np.uint8)
    prev = np.zeros(stride, np.int32)
    for y in range(h):
        f = raw[y * (stride + 1)]
        line = np.frombuffer(raw, np.uint8, stride, y * (stride + 1) + 1).astype(np.int32)
        cur = np.zeros(stride, np.int32)
        for i in range(stride):
            a = cur[i - 4] if i >= 4 else 0
            b = prev[i]
            c = prev[i - 4] if i >= 4 else 0
            if f == 0: p = 0
            elif f == 1: p = a
            elif f == 2: p = b
            elif f == 3: p = (a + b) // 2
            else:
                pa, pb, pc = abs(b - c), abs(a - c), abs(a + b - 2 * c)
                p = a if pa <= pb and pa <= pc else (b if pb <= pc else c)
            cur[i] = (line[i] + p) & 0xFF
        out[y] = cur
        prev = cur
    return w, h, out.reshape(h, w, 4), text


def frame(w, h, seed=0):
    return np.random.default_rng(seed).integers(0, 256, (h, w, 4), dtype=np.uint8)


def test_encode_png_round_trip_and_metadata(native):
    cfg = synthetic.plain_flame(1)
    cfg["background_color"] = [0.1, 0.5, 1.0]
    text_cfg = json.dumps(cfg)
    img = frame(37, 23)
    png = native.encode_png(text_cfg, img, 37, 23, iterations=1234567, ms=98.765, iterations_per_thread=1024)
    w, h, px, text = decode(png)
    assert (w, h) == (37, 23)
    assert np.array_equal(px, img)
    for key in ("Config", "Iterations", "IterationsPerThread", "RenderTime"):
        assert key in text, key
    assert text["Config"] == text_cfg
    assert text["ConfigChecksum"] == "sha256:" + hashlib.sha256(text_cfg.encode()).hexdigest()
    assert text["Iterations"] == "1234567"
    assert text["IterationsPerThread"] == "1024"
    assert text["RenderTime"] == "98.77ms"
    assert text["Resolution"] == "37x23"
    assert text["BackgroundColor"] == "0.1,0.5,1"
    assert text["Exposure"] == "1" and text["Gamma"] == "4"
    assert text["SpeedFactor"] == "0.50"
    assert text["RenderMode"] == "2D" and text["Projection"] == "N/A"
    assert text["ShaderVariations"] == "3"
    keys = list(text)
    assert keys[:3] == ["Software", "GitHash", "Branch"] and keys[-1] == "ShaderVariations"


def test_fae_call_encode_png(native):
    from ffb200 import Module
    m = Module()
    cfg = json.dumps(synthetic.sierpinski())
    img = frame(16, 9, 1)
    out, info = m.call({"fn": "encode_png", "config": cfg, "width": 16, "height": 9, "iterations": 10, "ms": 1.0,
                        "iterations_per_thread": 256}, img.tobytes())
    w, h, px, text = decode(out)
    assert np.array_equal(px, img) and text["IterationsPerThread"] == "256"
    assert info is None


def test_encode_png_errors(native):
    with pytest.raises(native.EngineError, match="RGBA"):
        native.encode_png(json.dumps(synthetic.sierpinski()), b"\0" * 10, 4, 4)
    with pytest.raises(native.EngineError, match="config"):
        native.encode_png("{}", frame(2, 2), 2, 2)
    from ffb200 import Module
    with pytest.raises(native.EngineError, match="RGBA"):
        Module().call({"fn": "encode_png", "config": json.dumps(synthetic.sierpinski()), "width": 4, "height": 4}, b"\0" * 10)


@pytest.mark.gpu
def test_rendered_frame_saves_as_png(tmp_path):
    from ffb200 import Engine
    image = Engine().render(synthetic.plain_flame(2), 64, 48, iterations=1_000_000)
    path = tmp_path / "f.png"
    image.save(str(path))
    w, h, px, text = decode(path.read_bytes())
    assert (w, h) == (64, 48)
    assert np.array_equal(px, image.array())
    assert int(text["Iterations"]) == image.info["iterations"]
