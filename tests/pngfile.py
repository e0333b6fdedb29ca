"""A small, independent PNG encoder / decoder in Python (zlib + struct), used
only to check libggb_image_io.so: it writes files of every colour type, bit
depth, filter and interlace mode for the reader, and reads the writer's output.
Follows the PNG specification (chunk layout, filters 0-4, Adam7)."""
import struct
import zlib

import numpy as np

SIG = b"\x89PNG\r\n\x1a\n"
ADAM7 = [(0, 0, 8, 8), (4, 0, 8, 8), (0, 4, 4, 8), (2, 0, 4, 4), (0, 2, 2, 4), (1, 0, 2, 2), (0, 1, 1, 2)]
CHANNELS = {0: 1, 2: 3, 3: 1, 4: 2, 6: 4}


def chunk(kind, data):
    return struct.pack(">I", len(data)) + kind + data + struct.pack(">I", zlib.crc32(kind + data) & 0xffffffff)


def _paeth(a, b, c):
    p = a + b - c
    pa, pb, pc = abs(p - a), abs(p - b), abs(p - c)
    return a if pa <= pb and pa <= pc else (b if pb <= pc else c)


def _filter(t, cur, prev, bpp):
    out = bytearray(len(cur))
    for i in range(len(cur)):
        a = cur[i - bpp] if i >= bpp else 0
        b = prev[i] if prev is not None else 0
        c = prev[i - bpp] if prev is not None and i >= bpp else 0
        p = (0, a, b, (a + b) >> 1, _paeth(a, b, c))[t]
        out[i] = (cur[i] - p) & 255
    return bytes(out)


def _unfilter(t, cur, prev, bpp):
    out = bytearray(cur)
    for i in range(len(out)):
        a = out[i - bpp] if i >= bpp else 0
        b = prev[i] if prev is not None else 0
        c = prev[i - bpp] if prev is not None and i >= bpp else 0
        p = (0, a, b, (a + b) >> 1, _paeth(a, b, c))[t]
        out[i] = (out[i] + p) & 255
    return bytes(out)


def _pack_row(samples, depth):
    """samples: 1-D int array of one scanline's samples at `depth` bits."""
    if depth == 8:
        return bytes(np.asarray(samples, np.uint8))
    if depth == 16:
        return np.asarray(samples, ">u2").tobytes()
    per = 8 // depth
    out = bytearray((len(samples) + per - 1) // per)
    for i, v in enumerate(samples):
        out[i // per] |= int(v) << (8 - depth - (i % per) * depth)
    return bytes(out)


def encode(samples, ctype, depth, interlace=0, palette=None, trns=None, filters=(0, 1, 2, 3, 4), idat_split=3,
           extra=()):
    """samples: uint array (h, w, channels) at `depth` bits.  Rows take the
    filter types in `filters` in turn; IDAT is cut into `idat_split` chunks."""
    h, w, ch = samples.shape
    assert ch == CHANNELS[ctype]
    bits = ch * depth
    bpp = max(1, bits // 8)
    raw = bytearray()
    passes = ADAM7 if interlace else [(0, 0, 1, 1)]
    k = 0
    for x0, y0, dx, dy in passes:
        sub = samples[y0::dy, x0::dx]
        if sub.size == 0:
            continue
        prev = None
        for row in sub:
            cur = _pack_row(row.reshape(-1), depth)
            t = filters[k % len(filters)]
            k += 1
            raw += bytes([t]) + _filter(t, cur, prev, bpp)
            prev = cur
    z = zlib.compress(bytes(raw), 6)
    parts = [z[i * len(z) // idat_split:(i + 1) * len(z) // idat_split] for i in range(idat_split)]
    out = SIG + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, depth, ctype, 0, 0, interlace))
    for kind, data in extra:
        out += chunk(kind, data)
    if palette is not None:
        out += chunk(b"PLTE", bytes(np.asarray(palette, np.uint8).reshape(-1)))
    if trns is not None:
        out += chunk(b"tRNS", trns)
    for p in parts:
        out += chunk(b"IDAT", p)
    return out + chunk(b"IEND", b"")


def decode(data):
    """Decode a non-interlaced 8-bit RGB / RGBA file (what png_save writes),
    checking every chunk CRC.  Returns (uint8 array (h, w, ch), chunk types)."""
    assert data[:8] == SIG
    pos, kinds, idat, hdr = 8, [], b"", None
    while pos < len(data):
        n, = struct.unpack(">I", data[pos:pos + 4])
        kind, body = data[pos + 4:pos + 8], data[pos + 8:pos + 8 + n]
        crc, = struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])
        assert crc == zlib.crc32(kind + body) & 0xffffffff, kind
        kinds.append(kind)
        if kind == b"IHDR":
            hdr = struct.unpack(">IIBBBBB", body)
        elif kind == b"IDAT":
            idat += body
        pos += 12 + n
    w, h, depth, ctype, comp, filt, inter = hdr
    assert depth == 8 and ctype in (2, 6) and comp == filt == inter == 0
    ch = CHANNELS[ctype]
    raw = zlib.decompress(idat)
    rb = w * ch
    assert len(raw) == h * (rb + 1)
    rows, prev = [], None
    for y in range(h):
        t, cur = raw[y * (rb + 1)], raw[y * (rb + 1) + 1:(y + 1) * (rb + 1)]
        assert t <= 4
        prev = _unfilter(t, cur, prev, ch)
        rows.append(np.frombuffer(prev, np.uint8))
    return np.stack(rows).reshape(h, w, ch), kinds
