"""libggb_image_io.so, the PNG files of the upstream src/image_io.h API on zlib
(no GPU): png_save output decoded by an independent reader, png_load_rgba on
files of every colour type, bit depth, filter and interlace mode written by an
independent writer, and the error returns (NULL / -1 with a message)."""
import os
import struct
import zlib

import numpy as np
import pytest

import ggb_api
import pngfile


@pytest.fixture(scope="module")
def io():
    assert os.path.exists(ggb_api.IMAGE_IO_LIB), "build the library first (__graft_entry__.build())"
    return ggb_api.ImageIO()


@pytest.mark.parametrize("shape", [(1, 1, 3), (5, 7, 4), (33, 64, 3), (64, 33, 4)])
def test_save_round_trip(io, tmp_path, shape):
    rng = np.random.default_rng(sum(shape))
    # smooth plus noise, so that every filter type wins on some row
    y, x = np.mgrid[0:shape[0], 0:shape[1]]
    img = ((x[..., None] * 3 + y[..., None] * 5 + rng.integers(0, 4, shape)) % 256).astype(np.uint8)
    img[shape[0] // 2:] = rng.integers(0, 256, img[shape[0] // 2:].shape)
    f = str(tmp_path / "a.png")
    assert io.save(f, img) == 0
    got, kinds = pngfile.decode(open(f, "rb").read())
    assert kinds[0] == b"IHDR" and kinds[-1] == b"IEND" and b"IDAT" in kinds
    np.testing.assert_array_equal(got, img)
    back = io.load(f)
    ref = np.concatenate([img, np.full(shape[:2] + (1,), 255, np.uint8)], 2) if shape[2] == 3 else img
    np.testing.assert_array_equal(back, ref.astype(np.float32) / np.float32(255))


def test_save_large_image_spans_several_idat_chunks(io, tmp_path):
    img = np.random.default_rng(3).integers(0, 256, (400, 600, 4), dtype=np.uint8)
    f = str(tmp_path / "big.png")
    assert io.save(f, img) == 0
    got, kinds = pngfile.decode(open(f, "rb").read())
    assert kinds.count(b"IDAT") > 1
    np.testing.assert_array_equal(got, img)


def _expected_rgba(s, ctype, depth, palette=None, palpha=None, key=None):
    """What a reader must return (uint8 RGBA) for samples s (h, w, ch)."""
    s = s.astype(np.int64)
    if depth == 16:
        to8 = (s * 255 + 32767) // 65535
    else:
        to8 = s * 255 // ((1 << depth) - 1)
    h, w = s.shape[:2]
    out = np.zeros((h, w, 4), np.int64)
    if ctype == 0:
        out[..., :3] = to8[..., :1]
        out[..., 3] = 255 if key is None else np.where(s[..., 0] == key[0], 0, 255)
    elif ctype == 2:
        out[..., :3] = to8
        out[..., 3] = 255 if key is None else np.where((s == np.array(key)).all(-1), 0, 255)
    elif ctype == 3:
        pal = np.concatenate([np.asarray(palette), np.asarray(palpha)[:, None]], 1)
        out = pal[s[..., 0]]
    elif ctype == 4:
        out[..., :3] = to8[..., :1]
        out[..., 3] = to8[..., 1]
    else:
        out = to8
    return out.astype(np.uint8)


CASES = [(0, d) for d in (1, 2, 4, 8, 16)] + [(2, 8), (2, 16), (3, 1), (3, 2), (3, 4), (3, 8), (4, 8), (4, 16),
                                               (6, 8), (6, 16)]


@pytest.mark.parametrize("interlace", [0, 1])
@pytest.mark.parametrize("ctype,depth", CASES)
def test_load_every_format(io, tmp_path, ctype, depth, interlace):
    rng = np.random.default_rng(ctype * 100 + depth * 2 + interlace)
    h, w = 13, 19                      # odd sizes: partial bytes, every Adam7 pass non-empty
    ch = pngfile.CHANNELS[ctype]
    top = (1 << depth) - 1
    kw = {}
    palette = palpha = key = None
    if ctype == 3:
        npal = min(top + 1, 40)
        s = rng.integers(0, npal, (h, w, 1))
        palette = rng.integers(0, 256, (npal, 3))
        palpha = np.full(npal, 255)
        palpha[: npal // 2] = rng.integers(0, 256, npal // 2)
        kw = dict(palette=palette, trns=bytes(palpha[: npal // 2].astype(np.uint8)))
    else:
        s = rng.integers(0, top + 1, (h, w, ch))
        if ctype in (0, 2):
            key = [int(v) for v in s[3, 4]]
            kw = dict(trns=struct.pack(">" + "H" * ch, *key))
    data = pngfile.encode(s, ctype, depth, interlace=interlace, **kw)
    f = tmp_path / "in.png"
    f.write_bytes(data)
    got = io.load(str(f))
    exp = _expected_rgba(s, ctype, depth, palette, palpha, key)
    np.testing.assert_array_equal(got, exp.astype(np.float32) / np.float32(255))


def test_ancillary_chunks_are_skipped_even_when_damaged(io, tmp_path):
    s = np.random.default_rng(1).integers(0, 256, (4, 6, 4))
    bad = pngfile.chunk(b"tEXt", b"Comment\x00x")
    bad = bad[:-1] + bytes([bad[-1] ^ 1])
    data = pngfile.encode(s, 6, 8, extra=[(b"gAMA", struct.pack(">I", 45455))])
    data = data[:33] + bad + data[33:]
    f = tmp_path / "anc.png"
    f.write_bytes(data)
    np.testing.assert_array_equal(io.load(str(f)), s.astype(np.float32) / np.float32(255))


def _corrupt_idat_crc(data):
    i = data.index(b"IDAT")
    n, = struct.unpack(">I", data[i - 4:i])
    j = i + 4 + n
    return data[:j] + bytes([data[j] ^ 0xff]) + data[j + 1:]


def test_load_errors_return_null_with_a_message(io, tmp_path, capfd):
    s = np.random.default_rng(2).integers(0, 256, (8, 8, 3))
    good = pngfile.encode(s, 2, 8)
    four = pngfile.encode(s[:4], 2, 8)
    bad = {   # file name: (contents, reason printed)
        "missing.png": (None, "cannot open"),
        "text.png": (b"not a png at all", "not a PNG"),
        "truncated.png": (good[: len(good) // 2], "truncated"),
        "crc.png": (_corrupt_idat_crc(good), "CRC"),
        "critical.png": (good[:33] + pngfile.chunk(b"ABCD", b"xx") + good[33:], "critical"),
        "short.png": (pngfile.SIG + pngfile.chunk(b"IHDR", struct.pack(">IIBBBBB", 8, 8, 8, 2, 0, 0, 0)) + four[33:],
                      "not enough image data"),
        "nopal.png": (pngfile.encode(np.zeros((2, 2, 1), np.int64), 3, 8), "PLTE"),
        "badfilter.png": (pngfile.SIG + pngfile.chunk(b"IHDR", struct.pack(">IIBBBBB", 1, 1, 8, 0, 0, 0, 0))
                          + pngfile.chunk(b"IDAT", zlib.compress(b"\x07\x00")) + pngfile.chunk(b"IEND", b""),
                          "filter"),
    }
    for name, (data, reason) in bad.items():
        f = tmp_path / name
        if data is not None:
            f.write_bytes(data)
        assert io.load(str(f)) is None, name
        err = capfd.readouterr().err
        assert err.startswith(str(f) + ": ") and reason in err, (name, err)


def test_save_errors_leave_no_file(io, tmp_path, capfd):
    f = tmp_path / "x.png"
    assert io.lib.png_save(os.fsencode(str(f)), 4, 4, 2, np.zeros(32, np.uint8).ctypes.data) == -1
    assert io.lib.png_save(os.fsencode(str(f)), 0, 4, 3, np.zeros(48, np.uint8).ctypes.data) == -1
    assert not f.exists()
    assert io.save(str(tmp_path / "nodir" / "x.png"), np.zeros((2, 2, 3), np.uint8)) == -1
    err = capfd.readouterr().err
    assert err.count("x.png: ") == 3


def test_strip_written_as_the_driver_input(tmp_path):
    """`python ggb_inputs.py OUT.png [seed]` writes the seeded benchmark strip
    as an 8-bit RGBA PNG equal to ggb_inputs.strip() rounded to bytes."""
    import subprocess
    import sys

    import ggb_inputs
    f = tmp_path / "strip.png"
    script = os.path.join(os.path.dirname(ggb_api.__file__), "ggb_inputs.py")
    p = subprocess.run([sys.executable, script, str(f), "3"], capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr
    got, _ = pngfile.decode(f.read_bytes())
    want = np.round(ggb_inputs.strip(3) * 255).astype(np.uint8)
    np.testing.assert_array_equal(got, want)
