"""Writer of small Phantom dump files for the reader's tests (test infrastructure).

The reference's own test dump is not in its checkout, so the reader is tested on files written
here from the record layout Phantom uses (read_phantom.jl:36-225 reads the same layout): every
record framed by its 4-byte length; the capture pattern (default int 60769, default real
60878.0, default int 60878, version, default int 690706); a 100-character identifier; eight
header blocks by type (default int, int*1, int*2, int*4, int*8, default real, real*4, real*8);
the number of array blocks, per block (int*8 count, 8 int*4 array counts), then per block and
type the arrays as (16-character tag, values).
"""
import struct

import numpy as np

TYPES = ("def_int", "int8", "int16", "int32", "int64", "def_real", "float32", "float64")


def _rec(b):
    return struct.pack("<i", len(b)) + b + struct.pack("<i", len(b))


def _tag(s):
    return s.encode("ascii").ljust(16)[:16]


def write_dump(path, blocks, header, def_int=np.int32, def_real=np.float64, version=1,
               identifier="FT:Phantom test dump", swap_tail=False):
    """blocks: list of (n, [(tag, array, type name), ...]) -- block 2 is the sinks block;
    header: list of (name, value, type name), names may repeat (per-type arrays).
    swap_tail corrupts the trailing length of the identifier record (reader error path)."""
    di, dr = np.dtype(def_int), np.dtype(def_real)
    dt = {"def_int": di, "def_real": dr, "int8": np.dtype(np.int8), "int16": np.dtype(np.int16),
          "int32": np.dtype(np.int32), "int64": np.dtype(np.int64), "float32": np.dtype(np.float32),
          "float64": np.dtype(np.float64)}
    out = bytearray()
    cap = (np.array(60769, di).tobytes() + np.array(60878.0, dr).tobytes() + np.array(60878, di).tobytes()
           + np.array(version, di).tobytes() + np.array(690706, di).tobytes())
    out += _rec(cap)
    ident = _rec(identifier.encode("ascii").ljust(100)[:100])
    if swap_tail:
        ident = ident[:-4] + struct.pack("<i", 99)
    out += ident
    for t in TYPES:
        items = [(n, v) for n, v, tt in header if tt == t]
        out += _rec(struct.pack("<i", len(items)))
        if items:
            out += _rec(b"".join(_tag(n) for n, _ in items))
            out += _rec(np.array([v for _, v in items], dt[t]).tobytes())
    out += _rec(struct.pack("<i", len(blocks)))
    for n, arrays in blocks:
        nums = [sum(1 for _, _, tt in arrays if tt == t) for t in TYPES]
        out += _rec(struct.pack("<q", n) + struct.pack("<8i", *nums))
    for n, arrays in blocks:
        for t in TYPES:
            for tag, a, tt in arrays:
                if tt != t:
                    continue
                a = np.asarray(a, dt[t])
                assert len(a) == n
                out += _rec(_tag(tag))
                out += _rec(a.tobytes())
    with open(path, "wb") as f:
        f.write(bytes(out))
    return path
