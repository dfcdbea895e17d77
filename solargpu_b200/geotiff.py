"""Single-band 32-bit float GeoTIFF rasters: the heightmap the CLI reads and
the irradiance raster it writes (the reference does both with libtiff,
src/geotiff_io.cpp:50-185; libtiff is not part of this build, so the codec is
written here in numpy + zlib).

Read: classic TIFF, either byte order, strips or tiles, no compression,
LZW (5) or Deflate (8, 32946), predictor none (1), horizontal (2) or
floating point (3); 32-bit IEEE float samples only, one sample a pixel (the
reference rejects anything else with the same message).  The GeoTIFF tags
33550 (pixel scale), 33922 (tie points), 34735 (geo keys), 34736 (geo
doubles), 34737 (geo ASCII) and 42113 (GDAL no-data) are kept in TiffMeta.

Write: as the reference's write_tiff: image tags, the input's compression
(when it is one of the above) and rows-per-strip, the five GeoTIFF tags of
the input, scanline (strip) layout, no predictor.  Tiles and predictors can
also be written (tests use them to check the reader).
"""
from __future__ import annotations

import dataclasses
import struct
import zlib

import numpy as np

COMPRESSION_NONE, COMPRESSION_LZW, COMPRESSION_DEFLATE, COMPRESSION_ADOBE_DEFLATE = 1, 5, 8, 32946

_TYPES = {1: ("B", 1), 2: ("s", 1), 3: ("H", 2), 4: ("I", 4), 6: ("b", 1), 7: ("B", 1), 8: ("h", 2),
          9: ("i", 4), 11: ("f", 4), 12: ("d", 8), 16: ("Q", 8)}


@dataclasses.dataclass
class TiffMeta:
    """Image and GeoTIFF tags of one raster (include/geotiff_io.h:15-27)."""
    w: int = 0
    h: int = 0
    compression: int = COMPRESSION_NONE
    rows_per_strip: int = 0
    tiepoints: list = dataclasses.field(default_factory=list)    # 33922
    pixel_scale: list = dataclasses.field(default_factory=list)  # 33550
    geo_keys: list = dataclasses.field(default_factory=list)     # 34735
    geo_doubles: list = dataclasses.field(default_factory=list)  # 34736
    geo_ascii: str = ""                                          # 34737
    nodata: str = ""                                             # 42113 (read only, as the reference)


class TiffError(ValueError):
    pass


# ---------------------------------------------------------------- LZW (TIFF flavour: MSB-first, early change)

def lzw_decode(data: bytes) -> bytes:
    out = bytearray()
    table = [bytes([i]) for i in range(256)] + [b"", b""]
    width, pos, nbits, prev = 9, 0, len(data) * 8, None
    while pos + width <= nbits:
        byte, bit = divmod(pos, 8)
        chunk = int.from_bytes(data[byte:byte + 4].ljust(4, b"\0"), "big")
        code = (chunk >> (32 - bit - width)) & ((1 << width) - 1)
        pos += width
        if code == 257:
            break
        if code == 256:
            table = table[:258]
            width, prev = 9, None
            continue
        if prev is None:
            entry = table[code]
        elif code < len(table):
            entry = table[code]
            table.append(prev + entry[:1])
        else:
            entry = prev + prev[:1]
            table.append(entry)
        out += entry
        prev = entry
        if len(table) + 1 >= (1 << width) and width < 12:
            width += 1
    return bytes(out)


def lzw_encode(data: bytes) -> bytes:
    out, acc, nacc = bytearray(), 0, 0

    def put(code, width):
        nonlocal acc, nacc
        acc = (acc << width) | code
        nacc += width
        while nacc >= 8:
            nacc -= 8
            out.append((acc >> nacc) & 0xFF)
        acc &= (1 << nacc) - 1

    table, nxt, width = {bytes([i]): i for i in range(256)}, 258, 9
    put(256, width)
    w = b""
    for c in data:
        wc = w + bytes([c])
        if wc in table:
            w = wc
            continue
        put(table[w], width)
        table[wc] = nxt
        nxt += 1
        if nxt >= (1 << width) and width < 12:   # the reader widens one code later
            width += 1
        if nxt >= 4093:                       # table full: start over
            put(256, width)
            table, nxt, width = {bytes([i]): i for i in range(256)}, 258, 9
        w = bytes([c])
    if w:
        put(table[w], width)
        nxt += 1
        if nxt >= (1 << width) and width < 12:   # the reader widens one code later
            width += 1
    put(257, width)
    if nacc:
        out.append((acc << (8 - nacc)) & 0xFF)
    return bytes(out)


# ---------------------------------------------------------------- predictors (per row of a strip or tile)

def _undo_predictor(buf: bytes, predictor: int, width: int, rows: int, order: str) -> np.ndarray:
    """Decoded bytes of rows x width float32 samples -> float32 [rows][width]."""
    if predictor == 1:
        return np.frombuffer(buf, dtype=order + "f4", count=rows * width).reshape(rows, width)
    if predictor == 2:   # horizontal differencing of the 32-bit words
        u = np.frombuffer(buf, dtype=order + "u4", count=rows * width).reshape(rows, width)
        return np.cumsum(u, axis=1, dtype=np.uint32).view(np.float32).reshape(rows, width)
    if predictor == 3:   # floating point: byte planes, most significant first, byte-wise differencing
        b = np.frombuffer(buf, dtype=np.uint8, count=rows * width * 4).reshape(rows, width * 4)
        b = np.cumsum(b, axis=1, dtype=np.uint8)
        planes = b.reshape(rows, 4, width).transpose(0, 2, 1)        # [rows][width][4], MSB first
        return np.ascontiguousarray(planes).view(">f4").reshape(rows, width).astype(np.float32)
    raise TiffError(f"unsupported predictor {predictor}")


def _apply_predictor(a: np.ndarray, predictor: int) -> bytes:
    """float32 [rows][width] -> bytes before compression (little endian)."""
    if predictor == 1:
        return a.astype("<f4").tobytes()
    if predictor == 2:
        u = a.astype("<f4").view("<u4")
        d = u.copy()
        d[:, 1:] = u[:, 1:] - u[:, :-1]
        return d.astype("<u4").tobytes()
    if predictor == 3:
        rows, width = a.shape
        planes = a.astype(">f4").view(np.uint8).reshape(rows, width, 4).transpose(0, 2, 1).reshape(rows, width * 4)
        d = planes.copy()
        d[:, 1:] = planes[:, 1:] - planes[:, :-1]
        return d.tobytes()
    raise TiffError(f"unsupported predictor {predictor}")


def _decompress(data: bytes, compression: int) -> bytes:
    if compression == COMPRESSION_NONE:
        return data
    if compression == COMPRESSION_LZW:
        return lzw_decode(data)
    if compression in (COMPRESSION_DEFLATE, COMPRESSION_ADOBE_DEFLATE):
        return zlib.decompress(data)
    raise TiffError(f"unsupported compression {compression}")


def _compress(data: bytes, compression: int) -> bytes:
    if compression == COMPRESSION_NONE:
        return data
    if compression == COMPRESSION_LZW:
        return lzw_encode(data)
    if compression in (COMPRESSION_DEFLATE, COMPRESSION_ADOBE_DEFLATE):
        return zlib.compress(data, 6)
    raise TiffError(f"unsupported compression {compression}")


# ---------------------------------------------------------------- reading

def _read_ifd(raw: bytes, order: str) -> dict:
    (off,) = struct.unpack_from(order + "I", raw, 4)
    (n,) = struct.unpack_from(order + "H", raw, off)
    tags = {}
    for i in range(n):
        tag, typ, cnt, val = struct.unpack_from(order + "HHI4s", raw, off + 2 + 12 * i)
        if typ not in _TYPES:
            continue
        fmt, size = _TYPES[typ]
        nbytes = size * cnt
        data = val if nbytes <= 4 else raw[struct.unpack(order + "I", val)[0]:][:nbytes]
        if typ == 2:
            tags[tag] = data[:cnt].split(b"\0", 1)[0].decode("latin-1")
        else:
            tags[tag] = list(struct.unpack(order + fmt * cnt, data[:nbytes]))
    return tags


def read_tiff(path: str) -> tuple[np.ndarray, TiffMeta]:
    """The raster as float32 [h][w] (row-major, as the reference's
    read_tiff) and its tags."""
    with open(path, "rb") as f:
        raw = f.read()
    if raw[:4] == b"II*\0":
        order = "<"
    elif raw[:4] == b"MM\0*":
        order = ">"
    else:
        raise TiffError(f"{path}: not a classic TIFF file")
    t = _read_ifd(raw, order)

    def one(tag, default=None):
        v = t.get(tag)
        return v[0] if v else default

    meta = TiffMeta(w=one(256, 0), h=one(257, 0), compression=one(259, COMPRESSION_NONE))
    bps, fmt, spp = one(258, 1), one(339, 1), one(277, 1)
    if bps != 32 or fmt != 3:
        raise TiffError(f"Expected 32-bit float TIFF, got bps={bps} fmt={fmt} ({path})")
    if spp != 1 or one(284, 1) != 1:
        raise TiffError(f"{path}: {spp} samples a pixel (one band expected)")
    predictor = one(317, 1)
    meta.rows_per_strip = one(278, meta.h) or meta.h
    meta.tiepoints = list(t.get(33922, []))
    meta.pixel_scale = list(t.get(33550, []))
    meta.geo_keys = list(t.get(34735, []))
    meta.geo_doubles = list(t.get(34736, []))
    meta.geo_ascii = t.get(34737, "") if isinstance(t.get(34737, ""), str) else ""
    meta.nodata = t.get(42113, "") if isinstance(t.get(42113, ""), str) else ""
    W, H = meta.w, meta.h
    out = np.empty((H, W), np.float32)
    if 322 in t:   # tiles
        tw, th = one(322), one(323)
        offs, cnts = t[324], t[325]
        across = (W + tw - 1) // tw
        for i, (o, c) in enumerate(zip(offs, cnts)):
            ty, tx = divmod(i, across)
            y0, x0 = ty * th, tx * tw
            if y0 >= H:
                break
            tile = _undo_predictor(_decompress(raw[o:o + c], meta.compression), predictor, tw, th, order)
            out[y0:min(H, y0 + th), x0:min(W, x0 + tw)] = tile[:min(th, H - y0), :min(tw, W - x0)]
    else:
        offs, cnts = t[273], t[279]
        rps = meta.rows_per_strip
        for i, (o, c) in enumerate(zip(offs, cnts)):
            y0 = i * rps
            rows = min(rps, H - y0)
            if rows <= 0:
                break
            out[y0:y0 + rows] = _undo_predictor(_decompress(raw[o:o + c], meta.compression), predictor, W, rows,
                                                order)
    return out, meta


# ---------------------------------------------------------------- writing

def write_tiff(path: str, data: np.ndarray, meta: TiffMeta, tile: int = 0, predictor: int = 1) -> None:
    """Writes data (meta.h x meta.w float32, row-major) with meta's
    compression and rows-per-strip and its five GeoTIFF tags, as the
    reference's write_tiff (src/geotiff_io.cpp:157-185); tile > 0 writes
    tiles of that side instead of strips."""
    H, W = meta.h, meta.w
    a = np.asarray(data, np.float32).reshape(-1)[:H * W].reshape(H, W)
    comp = meta.compression if meta.compression in (COMPRESSION_NONE, COMPRESSION_LZW, COMPRESSION_DEFLATE,
                                                    COMPRESSION_ADOBE_DEFLATE) else COMPRESSION_NONE
    blocks = []
    if tile:
        for y0 in range(0, H, tile):
            for x0 in range(0, W, tile):
                b = np.zeros((tile, tile), np.float32)
                part = a[y0:y0 + tile, x0:x0 + tile]
                b[:part.shape[0], :part.shape[1]] = part
                blocks.append(_compress(_apply_predictor(b, predictor), comp))
    else:
        rps = meta.rows_per_strip if 0 < meta.rows_per_strip <= H else H
        for y0 in range(0, H, rps):
            blocks.append(_compress(_apply_predictor(a[y0:y0 + rps], predictor), comp))
    entries = {256: (4, [W]), 257: (4, [H]), 258: (3, [32]), 259: (3, [comp]), 262: (3, [1]), 277: (3, [1]),
               284: (3, [1]), 339: (3, [3])}
    if predictor != 1:
        entries[317] = (3, [predictor])
    if tile:
        entries[322] = (4, [tile])
        entries[323] = (4, [tile])
    else:
        entries[278] = (4, [meta.rows_per_strip if 0 < meta.rows_per_strip <= H else H])
    if meta.pixel_scale:
        entries[33550] = (12, list(meta.pixel_scale))
    if meta.tiepoints:
        entries[33922] = (12, list(meta.tiepoints))
    if meta.geo_keys:
        entries[34735] = (3, list(meta.geo_keys))
    if meta.geo_doubles:
        entries[34736] = (12, list(meta.geo_doubles))
    if meta.geo_ascii:
        entries[34737] = (2, meta.geo_ascii)
    off_tag, cnt_tag = (324, 325) if tile else (273, 279)
    entries[off_tag] = (4, [0] * len(blocks))
    entries[cnt_tag] = (4, [len(b) for b in blocks])
    # layout: header, pixel blocks, out-of-line tag values, IFD
    body = bytearray(b"II*\0" + b"\0\0\0\0")
    offsets = []
    for b in blocks:
        offsets.append(len(body))
        body += b
        if len(body) & 1:
            body += b"\0"
    entries[off_tag] = (4, offsets)
    packed = {}
    for tag, (typ, vals) in sorted(entries.items()):
        if typ == 2:
            payload = vals.encode("latin-1") + b"\0"
            cnt = len(payload)
        else:
            fmt, _ = _TYPES[typ]
            payload = struct.pack("<" + fmt * len(vals), *vals)
            cnt = len(vals)
        if len(payload) <= 4:
            packed[tag] = (typ, cnt, payload.ljust(4, b"\0"))
        else:
            packed[tag] = (typ, cnt, struct.pack("<I", len(body)))
            body += payload
            if len(body) & 1:
                body += b"\0"
    ifd = len(body)
    struct.pack_into("<I", body, 4, ifd)
    body += struct.pack("<H", len(packed))
    for tag in sorted(packed):
        typ, cnt, val = packed[tag]
        body += struct.pack("<HHI", tag, typ, cnt) + val
    body += b"\0\0\0\0"
    with open(path, "wb") as f:
        f.write(bytes(body))


def read_tmy_series(path: str, n: int = 8760) -> np.ndarray:
    """The first n whitespace-separated values of a TMY series file
    (src/main.cpp:30-40)."""
    with open(path) as f:
        vals = np.array(f.read().split()[:n], dtype=np.float32)
    if vals.size < n:
        raise ValueError(f"{path}: {vals.size} values, {n} needed")
    return vals
