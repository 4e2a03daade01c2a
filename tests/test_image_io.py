"""The image files and the mean radiance (the reference's image class, src/image.ixx:93-203), on the CPU.

* A PFM written by the library is read back by the oracle's reader (the format ImageCompare consumes) as the same
  float32 values, rows in the right order.
* A PNG with the books' bytes decodes (zlib, any PNG reader) to to_byte of every channel: gamma 2, clamped to 0.999,
  times 256 truncated (image.ixx to_byte), checked at the thresholds.
* The mean radiance is image::mean_radiance's: the pixels folded in order, times 1 / count, channels averaged.
* What the reference refuses, refused here: an unknown extension, an exposure on the books' bytes, an exposure beyond
  24 stops (renderer.cu:1204-1220).
"""
import math
import struct
import zlib

import numpy as np
import pytest

pytestmark = pytest.mark.filterwarnings("ignore:invalid value encountered")

import raytracing_b200 as rt
from oracle import binding as oracle


def _decode_png(path):
    data = open(path, "rb").read()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    at = 8
    chunks = {}
    idat = b""
    while at < len(data):
        (n,) = struct.unpack(">I", data[at:at + 4])
        kind = data[at + 4:at + 8]
        body = data[at + 8:at + 8 + n]
        (crc,) = struct.unpack(">I", data[at + 8 + n:at + 12 + n])
        assert crc == zlib.crc32(kind + body) & 0xFFFFFFFF, kind
        if kind == b"IDAT":
            idat += body
        else:
            chunks[kind] = body
        at += 12 + n
    w, h, depth, color, _, _, _ = struct.unpack(">IIBBBBB", chunks[b"IHDR"])
    assert (depth, color) == (8, 2) and b"IEND" in chunks
    raw = zlib.decompress(idat)
    rows = np.frombuffer(raw, dtype=np.uint8).reshape(h, 1 + 3 * w)
    assert np.all(rows[:, 0] == 0)
    return rows[:, 1:].reshape(h, w, 3)


def _books_byte(v):
    g = math.sqrt(v) if v > 0 else 0.0  # NaN is not above 0
    g = min(max(g, 0.0), 0.999)
    return int(256 * g)


def _image(h=37, w=53, seed=1):
    rng = np.random.default_rng(seed)
    px = rng.exponential(0.4, size=(h, w, 3))
    edge = [0.0, -1.0, 0.998001, 0.998002, 1.0, 15.0, 1e-300, (255 / 256) ** 2, (254.5 / 256) ** 2, np.nan, np.inf]
    px.reshape(-1)[: len(edge)] = edge
    return px


def test_pfm_round_trips_through_the_oracles_reader(tmp_path):
    px = _image()
    px[~np.isfinite(px)] = 0.5
    path = tmp_path / "a.PFM"
    rt.save_image(str(path), px)
    back = oracle.load_pfm(str(path))
    assert np.array_equal(back, px.astype(np.float32).astype(np.float64))
    head = open(path, "rb").read(20)
    assert head.startswith(b"PF\n53 37\n-1.0\n")


def test_png_holds_the_books_bytes(tmp_path):
    px = _image()
    path = tmp_path / "a.png"
    rt.save_image(str(path), px)
    got = _decode_png(path)
    want = np.vectorize(_books_byte, otypes=[np.uint8])(px)
    assert np.array_equal(got, want)
    # (255/256)^2 is exactly byte 255's threshold, (254.5/256)^2 the middle of byte 254, NaN and -1 give 0
    assert got.reshape(-1)[7] == 255 and got.reshape(-1)[8] == 254 and got.reshape(-1)[9] == 0


def test_png_of_a_large_image_spans_several_deflate_blocks(tmp_path):
    px = _image(h=300, w=257, seed=2)  # 231,600 raw bytes: four stored blocks
    path = tmp_path / "big.png"
    rt.save_image(str(path), px)
    assert np.array_equal(_decode_png(path), np.vectorize(_books_byte, otypes=[np.uint8])(px))


def test_mean_radiance_is_the_references_fold():
    px = _image()
    px[~np.isfinite(px)] = 0.25
    flat = px.reshape(-1, 3)
    sums = [0.0, 0.0, 0.0]
    for r, g, b in flat:
        sums[0] += r
        sums[1] += g
        sums[2] += b
    inv = 1 / flat.shape[0]
    want = (inv * sums[0] + inv * sums[1] + inv * sums[2]) / 3
    assert rt.mean_radiance(px) == want


def test_refusals(tmp_path):
    px = _image()
    with pytest.raises(ValueError):
        rt.save_image(str(tmp_path / "a.jpg"), px)
    with pytest.raises(ValueError):
        rt.save_image(str(tmp_path / "a.png"), px, tone="books", exposure=1.0)
    with pytest.raises(ValueError):
        rt.save_image(str(tmp_path / "a.png"), px, tone="agx", exposure=24.5)
    with pytest.raises(ValueError):
        rt.save_image(str(tmp_path / "a.png"), px, tone="agx", exposure=float("nan"))
