"""PNG files of tone-mapped films (Renderer.cpp:94-105 writes the colour buffer with
stbi_write_png after flipping it vertically). An 8-bit RGBA, non-interlaced PNG written with the
standard library's zlib; read_png reads the same kind of file back."""
import struct
import zlib

import numpy as np


def _chunk(kind, data):
    body = kind + data
    return struct.pack(">I", len(data)) + body + struct.pack(">I", zlib.crc32(body) & 0xFFFFFFFF)


def write_png(path, rgba, flip=True):
    """rgba: (H, W, 4) uint8, row 0 = the film's first row. flip puts the film's last row at the
    top of the image, as the reference's output does."""
    img = np.ascontiguousarray(rgba, np.uint8)
    if img.ndim != 3 or img.shape[2] != 4:
        raise ValueError("expected an (H, W, 4) uint8 image")
    if flip:
        img = img[::-1]
    h, w = img.shape[:2]
    raw = b"".join(b"\x00" + img[y].tobytes() for y in range(h))  # filter type 0 per row
    ihdr = struct.pack(">IIBBBBB", w, h, 8, 6, 0, 0, 0)
    data = b"\x89PNG\r\n\x1a\n" + _chunk(b"IHDR", ihdr) + _chunk(b"IDAT", zlib.compress(raw, 6)) + \
        _chunk(b"IEND", b"")
    with open(path, "wb") as f:
        f.write(data)


def _unfilter(raw, h, w, bpp):
    stride = bpp * w
    out = np.zeros((h, stride), np.uint8)
    prev = np.zeros(stride, np.int32)
    for y in range(h):
        base = y * (stride + 1)
        ft = raw[base]
        line = np.frombuffer(raw, np.uint8, stride, base + 1).astype(np.int32)
        if ft == 0:
            cur = line
        elif ft == 1:  # Sub: running sum per channel
            cur = np.cumsum(line.reshape(w, bpp), axis=0).reshape(-1) & 0xFF
        elif ft == 2:  # Up
            cur = (line + prev) & 0xFF
        else:
            cur = np.zeros(stride, np.int32)
            left = np.zeros(bpp, np.int32)
            upleft = np.zeros(bpp, np.int32)
            for x in range(w):
                sl = slice(x * bpp, (x + 1) * bpp)
                up = prev[sl]
                if ft == 3:  # Average
                    pred = (left + up) // 2
                else:  # Paeth
                    pa, pb, pc = np.abs(up - upleft), np.abs(left - upleft), np.abs(left + up - 2 * upleft)
                    pred = np.where((pa <= pb) & (pa <= pc), left, np.where(pb <= pc, up, upleft))
                v = (line[sl] + pred) & 0xFF
                cur[sl] = v
                left = v
                upleft = up
        out[y] = cur
        prev = cur.astype(np.int32)
    return out


def read_png_any(path):
    """An 8-bit RGB, RGBA or palette non-interlaced PNG as (h, w, 4) uint8 (alpha 255 where the
    file has none), first row = the top of the image (as stbi_load returns it)."""
    with open(path, "rb") as f:
        data = f.read()
    if data[:8] != b"\x89PNG\r\n\x1a\n":
        raise ValueError(f"not a PNG file: {path}")
    pos, idat, w, h, ctype = 8, b"", 0, 0, 6
    palette, trns = None, None
    while pos < len(data):
        n, = struct.unpack(">I", data[pos:pos + 4])
        kind = data[pos + 4:pos + 8]
        body = data[pos + 8:pos + 8 + n]
        if kind == b"IHDR":
            w, h, depth, ctype, _, _, interlace = struct.unpack(">IIBBBBB", body)
            if depth != 8 or ctype not in (2, 3, 6) or interlace != 0:
                raise ValueError("only 8-bit RGB, RGBA or palette non-interlaced PNG files")
        elif kind == b"PLTE":
            palette = np.frombuffer(body, np.uint8).reshape(-1, 3)
        elif kind == b"tRNS":
            trns = np.frombuffer(body, np.uint8)
        elif kind == b"IDAT":
            idat += body
        pos += 12 + n
    bpp = {6: 4, 2: 3, 3: 1}[ctype]
    img = _unfilter(zlib.decompress(idat), h, w, bpp).reshape(h, w, bpp)
    if ctype == 3:
        rgba = np.full((len(palette), 4), 255, np.uint8)
        rgba[:, :3] = palette
        if trns is not None:
            rgba[:len(trns), 3] = trns
        return rgba[img[..., 0]]
    if bpp == 3:
        img = np.concatenate([img, np.full((h, w, 1), 255, np.uint8)], 2)
    return img


def read_png(path):
    """Reads an 8-bit RGBA (or RGB) non-interlaced PNG as written by write_png."""
    return read_png_any(path)
