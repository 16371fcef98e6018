"""A minimal multi-page TIFF writer for the ingest tests (test
infrastructure): classic TIFF in either byte order, strips or tiles,
uncompressed or PackBits, one sample per pixel."""
import struct

import numpy as np


def packbits(data: bytes) -> bytes:
    out = bytearray()
    i, n = 0, len(data)
    while i < n:
        j = i + 1
        while j < n and j - i < 128 and data[j] == data[i]:
            j += 1
        if j - i >= 3:
            out += struct.pack("b", -(j - i - 1)) + data[i:i + 1]
            i = j
            continue
        j = i + 1
        while j < n and j - i < 128 and not (j + 2 < n and data[j] == data[j + 1] == data[j + 2]):
            j += 1
        out += struct.pack("b", j - i - 1) + data[i:j]
        i = j
    return bytes(out)


def write_tiff(path, pages, byteorder="<", tile=None, rows_per_strip=None, compress=False):
    """pages: list of 2-D arrays (height, width) of one dtype."""
    dt = pages[0].dtype
    fmt = 3 if dt.kind == "f" else (2 if dt.kind == "i" else 1)
    bits = dt.itemsize * 8
    bo = byteorder
    body = bytearray()
    ifds = []
    header = 8
    for a in pages:
        H, W = a.shape
        a = a.astype(dt.newbyteorder(bo))
        pieces = []
        if tile:
            th, tw = tile
            for ty in range(0, H, th):
                for tx in range(0, W, tw):
                    t = np.zeros((th, tw), dtype=a.dtype)
                    blk = a[ty:ty + th, tx:tx + tw]
                    t[:blk.shape[0], :blk.shape[1]] = blk
                    pieces.append(t.tobytes())
        else:
            rps = rows_per_strip or H
            for r in range(0, H, rps):
                pieces.append(a[r:r + rps].tobytes())
        offs, cnts = [], []
        for p in pieces:
            if compress:
                p = packbits(p)
            offs.append(header + len(body))
            cnts.append(len(p))
            body += p
            if len(body) % 2:
                body += b"\0"
        ifds.append((H, W, offs, cnts, rows_per_strip or H))
    out = bytearray(b"II" if bo == "<" else b"MM")
    out += struct.pack(bo + "HI", 42, 0)
    out += body
    prev_link = 4
    for (H, W, offs, cnts, rps) in ifds:
        arrays = bytearray()
        entries = []

        def add(tag, typ, vals):
            entries.append((tag, typ, vals))
        add(256, 4, [W])
        add(257, 4, [H])
        add(258, 3, [bits])
        add(259, 3, [32773 if compress else 1])
        add(262, 3, [1])
        if tile:
            add(322, 4, [tile[1]])
            add(323, 4, [tile[0]])
            add(324, 4, offs)
            add(325, 4, cnts)
        else:
            add(273, 4, offs)
            add(278, 4, [rps])
            add(279, 4, cnts)
        add(277, 3, [1])
        add(339, 3, [fmt])
        entries.sort()
        ifd_at = len(out)
        if ifd_at % 2:
            out += b"\0"
            ifd_at += 1
        struct.pack_into(bo + "I", out, prev_link, ifd_at)
        n = len(entries)
        data_at = ifd_at + 2 + 12 * n + 4
        blob = bytearray()
        raw = bytearray(struct.pack(bo + "H", n))
        for tag, typ, vals in entries:
            sz = 2 if typ == 3 else 4
            code = "H" if typ == 3 else "I"
            payload = struct.pack(bo + code * len(vals), *vals)
            if len(payload) <= 4:
                raw += struct.pack(bo + "HHI", tag, typ, len(vals)) + payload.ljust(4, b"\0")
            else:
                raw += struct.pack(bo + "HHII", tag, typ, len(vals), data_at + len(blob))
                blob += payload
        prev_link = ifd_at + 2 + 12 * n
        raw += struct.pack(bo + "I", 0)
        out += raw + blob
    with open(path, "wb") as f:
        f.write(out)
