"""HDF5 output of interpolated grids: ``write_GridDataset`` and ``write_GridBundle``
(Partia.jl/src/julia/IO/gridsIO/write_grids.jl:29-215).

File layout, as the reference writes it:

- ``params/<key>``: one scalar dataset per parameter (String, Int, Bool or Float64);
- ``data/names``: the grids' names (fixed-length UTF-8 strings);
- ``data/coord/<x|y|z>`` (PointSamples) or ``data/axes/<x|y|z>`` (StructuredGrid): the shared
  coordinate or axis vectors of the first grid;
- ``data/grids/<i>``: the values of grid i (1-based), Float64.  A StructuredGrid's values are
  column-major, as in Julia, so the HDF5 dimensions are the grid's size reversed (what HDF5.jl
  writes for a Julia array).

No HDF5 library is available to this package, so the container is encoded here directly, with
the HDF5 format's version-2 structures: a version-2 superblock, version-2 object headers, groups
as compact link lists (Link Info, Group Info and Link messages) and contiguous datasets
(Dataspace, Datatype, Fill Value and Data Layout messages); every superblock and object header
carries the format's Jenkins lookup3 checksum.  Metadata come first, then every dataset's values
at 8-byte aligned addresses computed in advance, so values can be streamed to their place in
any order.

Values that live on a CUDA device (torch tensors) are copied to two pinned host buffers in
chunks on a separate stream while the previous chunk is being written: the device-to-host copy
overlaps the file write.
"""
import datetime
import os
import struct

import numpy as np

from ._lib import ArgumentError

UNDEF = 0xFFFFFFFFFFFFFFFF
_SIG = b"\x89HDF\r\n\x1a\n"
_COORDINATE = ("x", "y", "z")
SCHEMA_NAME, SCHEMA_ID = "GridDataset", "GridDataset.v1"
REQUIRED_UNITS = ("umass", "udist", "utime", "umagfd")


# ---- Jenkins lookup3 (hashlittle), the HDF5 metadata checksum ----

def _rot(x, k):
    return ((x << k) | (x >> (32 - k))) & 0xFFFFFFFF


def lookup3(data, initval=0):
    """Bob Jenkins' lookup3 ``hashlittle`` of a byte string (the published 2006 algorithm)."""
    m = 0xFFFFFFFF
    n = len(data)
    a = b = c = (0xDEADBEEF + n + initval) & m
    i = 0
    while n > 12:
        a = (a + int.from_bytes(data[i:i + 4], "little")) & m
        b = (b + int.from_bytes(data[i + 4:i + 8], "little")) & m
        c = (c + int.from_bytes(data[i + 8:i + 12], "little")) & m
        a = (a - c) & m; a ^= _rot(c, 4); c = (c + b) & m
        b = (b - a) & m; b ^= _rot(a, 6); a = (a + c) & m
        c = (c - b) & m; c ^= _rot(b, 8); b = (b + a) & m
        a = (a - c) & m; a ^= _rot(c, 16); c = (c + b) & m
        b = (b - a) & m; b ^= _rot(a, 19); a = (a + c) & m
        c = (c - b) & m; c ^= _rot(b, 4); b = (b + a) & m
        i += 12
        n -= 12
    if n == 0:
        return c
    tail = data[i:i + n] + b"\x00" * (12 - n)
    a = (a + int.from_bytes(tail[0:4], "little")) & m
    b = (b + int.from_bytes(tail[4:8], "little")) & m
    c = (c + int.from_bytes(tail[8:12], "little")) & m
    c ^= b; c = (c - _rot(b, 14)) & m
    a ^= c; a = (a - _rot(c, 11)) & m
    b ^= a; b = (b - _rot(a, 25)) & m
    c ^= b; c = (c - _rot(b, 16)) & m
    a ^= c; a = (a - _rot(c, 4)) & m
    b ^= a; b = (b - _rot(a, 14)) & m
    c ^= b; c = (c - _rot(b, 24)) & m
    return c


# ---- message encoders (HDF5 file format, version-2 object headers) ----

def _msg(mtype, body):
    return struct.pack("<BHB", mtype, len(body), 0) + body


def _dataspace(dims):
    """Dataspace message, version 2: scalar when dims is empty."""
    return _msg(0x01, struct.pack("<BBBB", 2, len(dims), 0, 1 if dims else 0) +
                b"".join(struct.pack("<Q", d) for d in dims))


def _dtype_f64():
    # class 1 (floating point), version 1; little-endian, implied mantissa MSB, sign bit 63;
    # offset 0, precision 64, exponent at 52 (11 bits), mantissa at 0 (52 bits), bias 1023
    return _msg(0x03, struct.pack("<BBBBI", 0x11, 0x20, 63, 0, 8) + struct.pack("<HHBBBBI", 0, 64, 52, 11, 0, 52, 1023))


def _dtype_int(size, signed):
    # class 0 (fixed point), version 1; little-endian, sign flag in bit 3
    return _msg(0x03, struct.pack("<BBBBI", 0x10, 0x08 if signed else 0x00, 0, 0, size) +
                struct.pack("<HH", 0, 8 * size))


def _dtype_str(size):
    # class 3 (string), version 1; null-padded, UTF-8
    return _msg(0x03, struct.pack("<BBBBI", 0x13, 0x01 | (1 << 4), 0, 0, size))


def _fill_value():
    # version 3: space allocated early, fill value written only if one is set (none is)
    return _msg(0x05, struct.pack("<BB", 3, 0x01 | (2 << 2)))


def _layout_contiguous(addr, size):
    return _msg(0x08, struct.pack("<BBQQ", 3, 1, addr, size))


def _link_info():
    # version 0, no creation order: the links are stored compactly in the object header
    return _msg(0x02, struct.pack("<BBQQ", 0, 0, UNDEF, UNDEF))


def _group_info():
    return _msg(0x0A, struct.pack("<BB", 0, 0))


def _link(name, addr):
    nb = name.encode("utf-8")
    if len(nb) > 255:
        raise ArgumentError("HDF5 link name longer than 255 bytes: %r" % name)
    # version 1; flags: 1-byte name length, character set field present (UTF-8); hard link
    return _msg(0x06, struct.pack("<BBBB", 1, 0x10, 1, len(nb)) + nb + struct.pack("<Q", addr))


def _object_header(messages):
    """Version-2 object header: 'OHDR', version 2, 4-byte chunk size, messages, checksum."""
    body = b"".join(messages)
    head = b"OHDR" + struct.pack("<BBI", 2, 0x02, len(body))
    raw = head + body
    return raw + struct.pack("<I", lookup3(raw))


# ---- the file tree and its layout ----

class _Dataset:
    """A contiguous dataset: its datatype message, HDF5 dimensions and a value source (bytes,
    a numpy array, or a torch tensor) whose bytes, in storage order, are the dataset's."""

    def __init__(self, dtype_msg, dims, nbytes, source):
        self.dtype_msg, self.dims, self.nbytes, self.source = dtype_msg, tuple(dims), int(nbytes), source
        self.addr = 0
        self.data_addr = UNDEF

    def header(self):
        return _object_header([_dataspace(self.dims), self.dtype_msg, _fill_value(),
                               _layout_contiguous(self.data_addr, self.nbytes)])


class _Group:
    def __init__(self):
        self.children = []   # (name, node), in insertion order
        self.addr = 0

    def add(self, name, node):
        self.children.append((name, node))
        return node

    def header(self):
        return _object_header([_link_info(), _group_info()] + [_link(n, c.addr) for n, c in self.children])


def _nodes(root):
    out, stack = [], [root]
    while stack:
        node = stack.pop(0)
        out.append(node)
        if isinstance(node, _Group):
            stack.extend(c for _, c in node.children)
    return out


def _scalar(v):
    """A params value as a scalar dataset (String, Bool, Int or Float64, as the reference allows)."""
    if isinstance(v, str):
        b = v.encode("utf-8")
        return _Dataset(_dtype_str(max(len(b), 1)), (), max(len(b), 1), b if b else b"\x00")
    if isinstance(v, (bool, np.bool_)):
        return _Dataset(_dtype_int(1, False), (), 1, struct.pack("<B", 1 if v else 0))
    if isinstance(v, (int, np.integer)):
        return _Dataset(_dtype_int(8, True), (), 8, struct.pack("<q", int(v)))
    if isinstance(v, (float, np.floating)):
        return _Dataset(_dtype_f64(), (), 8, struct.pack("<d", float(v)))
    raise ArgumentError("params values must be String, Int, Bool or Float64, got %s" % type(v).__name__)


def _strings(names):
    bs = [n.encode("utf-8") for n in names]
    size = max([len(b) for b in bs] + [1])
    return _Dataset(_dtype_str(size), (len(bs),), size * len(bs), b"".join(b.ljust(size, b"\x00") for b in bs))


def _is_torch(a):
    return type(a).__module__.startswith("torch")


def _vector(a):
    """A Float64 vector, from numpy or torch (host or device)."""
    if _is_torch(a):
        t = a.detach()
        if t.dtype != __import__("torch").float64:
            raise ArgumentError("grid values must be Float64")
        t = t.contiguous().reshape(-1)
        return _Dataset(_dtype_f64(), (t.numel(),), 8 * t.numel(), t)
    v = np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
    return _Dataset(_dtype_f64(), (v.size,), 8 * v.size, v)


def _column_major(a):
    """A StructuredGrid's values: column-major bytes, HDF5 dimensions reversed (as HDF5.jl)."""
    g = np.asfortranarray(np.asarray(a, dtype=np.float64))
    return _Dataset(_dtype_f64(), tuple(reversed(g.shape)), 8 * g.size, g.T)   # g.T is C-contiguous


def _superblock(eof, root_addr):
    raw = _SIG + struct.pack("<BBBBQQQQ", 2, 8, 8, 0, 0, UNDEF, eof, root_addr)
    return raw + struct.pack("<I", lookup3(raw))


def _layout(root):
    """Addresses: superblock, object headers (breadth first), then 8-byte aligned values."""
    nodes = _nodes(root)
    pos = 48
    for node in nodes:
        node.addr = pos
        pos += len(node.header())   # sizes do not depend on addresses
    for node in nodes:
        if isinstance(node, _Dataset):
            if node.nbytes == 0:
                node.data_addr = UNDEF
                continue
            pos = (pos + 7) & ~7
            node.data_addr = pos
            pos += node.nbytes
    return nodes, pos


CHUNK_BYTES = 32 << 20   # device-to-host staging chunk


def _write_device(f, jobs):
    """Stream CUDA tensors to their file offsets: chunks are copied to two pinned buffers on a
    side stream, and chunk k is written while chunk k + 1 is in flight."""
    import torch
    dev = jobs[0][1].device
    stream = torch.cuda.Stream(device=dev)
    stream.wait_stream(torch.cuda.current_stream(dev))   # the values' producers come first
    bufs = [torch.empty(CHUNK_BYTES, dtype=torch.uint8, pin_memory=True) for _ in range(2)]
    events = [torch.cuda.Event() for _ in range(2)]
    pieces = []
    for addr, t in jobs:
        raw = t.view(torch.uint8)
        for lo in range(0, raw.numel(), CHUNK_BYTES):
            pieces.append((addr + lo, raw[lo:lo + CHUNK_BYTES]))
    pending = None
    for k, (off, src) in enumerate(pieces):
        b = k & 1
        with torch.cuda.stream(stream):
            bufs[b][:src.numel()].copy_(src, non_blocking=True)
            events[b].record(stream)
        if pending is not None:
            pb, poff, pn = pending
            events[pb].synchronize()
            f.seek(poff)
            f.write(memoryview(bufs[pb].numpy()[:pn]))
        pending = (b, off, src.numel())
    if pending is not None:
        pb, poff, pn = pending
        events[pb].synchronize()
        f.seek(poff)
        f.write(memoryview(bufs[pb].numpy()[:pn]))


def _write_file(path, root):
    nodes, eof = _layout(root)
    device_jobs = []
    with open(path, "wb") as f:
        f.write(_superblock(eof, root.addr))
        for node in nodes:
            f.write(node.header())
        for node in nodes:
            if not isinstance(node, _Dataset) or node.nbytes == 0:
                continue
            src = node.source
            if _is_torch(src):
                if src.is_cuda:
                    device_jobs.append((node.data_addr, src))
                    continue
                src = src.numpy()
            f.seek(node.data_addr)
            f.write(src if isinstance(src, (bytes, bytearray)) else memoryview(np.ascontiguousarray(src)).cast("B"))
        if device_jobs:
            _write_device(f, device_jobs)
        f.truncate(eof)


# ---- GridDataset and the writers (write_grids.jl) ----

class GridDataset:
    """A GridBundle with its metadata (Partia.jl/src/julia/Grids/griddataset/GridDataset.jl):
    ``data`` is the bundle, ``params`` a dict of String / Int / Bool / Float64 values."""

    def __init__(self, data, params=None):
        self.data = data
        self.params = dict(params or {})


def _package_version():
    from . import __version__
    return __version__


def file_identifier(operation_name=""):
    """The reference's file identifier (Partia.jl/src/julia/Tools/logging.jl:152-156) with this
    package in place of Partia's version: "FT:Partia:<version> (<operation>): <time>"."""
    now = datetime.datetime.now()
    stamp = now.strftime("%d/%m/%Y %H:%M:%S") + ".%03d" % (now.microsecond // 1000)
    return "FT:Partia:%s (%s): %s" % (_package_version(), operation_name or "CommonOutput", stamp)


def _grid_kind(g):
    from .grids import PointSamples, StructuredGrid
    if isinstance(g, PointSamples):
        return "PointSamples"
    if isinstance(g, StructuredGrid):
        return "StructuredGrid"
    raise ArgumentError("write_GridDataset: no method for %s (PointSamples or StructuredGrid only)"
                        % type(g).__name__)


def write_GridDataset(gd, filename="PRGridDataset.h5"):
    """Write a GridDataset (write_grids.jl:29-68 for PointSamples, 91-139 for StructuredGrid).
    Every grid must share the first grid's coordinate (axis) vectors -- the same objects, as the
    reference's `===` test -- else ArgumentError."""
    grids, names = gd.data.grids, gd.data.names
    if len(grids) == 0:
        raise ArgumentError("write_GridDataset: the dataset holds no grid")
    kind = _grid_kind(grids[0])
    shared = "coor" if kind == "PointSamples" else "axes"
    g1 = grids[0]
    for i, gi in enumerate(grids[1:], start=2):
        if _grid_kind(gi) != kind:
            raise ArgumentError("grid %d is a %s, grid 1 a %s" % (i, type(gi).__name__, type(g1).__name__))
        for d in range(len(getattr(g1, shared))):
            if getattr(gi, shared)[d] is not getattr(g1, shared)[d]:
                raise ArgumentError("%s %s not shared: grid=%d dim=%d" % (kind, shared, i, d + 1))
    root = _Group()
    pg = root.add("params", _Group())
    for k, v in gd.params.items():
        pg.add(str(k), _scalar(v))
    dg = root.add("data", _Group())
    dg.add("names", _strings([str(n) for n in names]))
    cg = dg.add("coord" if kind == "PointSamples" else "axes", _Group())
    for d, vec in enumerate(getattr(g1, shared)):
        cg.add(_COORDINATE[d], _vector(vec))
    gg = dg.add("grids", _Group())
    for i, g in enumerate(grids, start=1):
        gg.add(str(i), _vector(g.grid) if kind == "PointSamples" else _column_major(g.grid))
    _write_file(os.fspath(filename), root)


def write_GridBundle(gb, filename="PRGridDataset.h5", code_units=None, operation_name="", params=None):
    """GridDataset of a GridBundle with the reference's metadata, written by write_GridDataset
    (write_grids.jl:181-215): schema name and id, system kernel, dtype, grid type, the code units
    (umass, udist, utime and umagfd required, else ArgumentError) and a file identifier."""
    code_units = dict(code_units or {})
    missing = tuple(k for k in REQUIRED_UNITS if k not in code_units)
    if missing:
        raise ArgumentError("code_units missing required keys: %s" % (missing,))
    if len(gb.grids) == 0:
        raise ArgumentError("write_GridBundle: the bundle holds no grid")
    import platform
    p = dict(params or {})
    p["schema_name"] = SCHEMA_NAME
    p["schema_id"] = SCHEMA_ID
    p["system_kernel"] = platform.system()
    p["dtype"] = "Float64"
    p["grid_type"] = _grid_kind(gb.grids[0])
    for k, v in code_units.items():
        p[str(k)] = float(v)
    p["file_identifier"] = file_identifier(operation_name)
    write_GridDataset(GridDataset(gb, p), filename)


# ---- reader (read_grids.jl) for files in the subset written above ----

def _read_oh(buf, addr):
    """(messages [(type, body)]) of a version-2 object header, checksum verified."""
    if buf[addr:addr + 4] != b"OHDR" or buf[addr + 4] != 2:
        raise ArgumentError("not a version-2 HDF5 object header at %d" % addr)
    flags = buf[addr + 5]
    pos = addr + 6 + (16 if flags & 0x20 else 0) + (4 if flags & 0x10 else 0)
    w = 1 << (flags & 3)
    size = int.from_bytes(buf[pos:pos + w], "little")
    pos += w
    end = pos + size
    if struct.unpack_from("<I", buf, end)[0] != lookup3(bytes(buf[addr:end])):
        raise ArgumentError("HDF5 object header checksum mismatch at %d" % addr)
    msgs = []
    while pos + 4 <= end:
        mtype, msize, mflags = struct.unpack_from("<BHB", buf, pos)
        pos += 4 + (2 if flags & 0x04 else 0)
        msgs.append((mtype, bytes(buf[pos:pos + msize])))
        pos += msize
    return msgs


def _links(msgs):
    out = {}
    for mtype, body in msgs:
        if mtype != 0x06:
            continue
        fl = body[1]
        p = 2
        ltype = 0
        if fl & 0x08:
            ltype = body[p]; p += 1
        if fl & 0x04:
            p += 8
        if fl & 0x10:
            p += 1
        w = 1 << (fl & 3)
        n = int.from_bytes(body[p:p + w], "little"); p += w
        name = body[p:p + n].decode("utf-8"); p += n
        if ltype != 0:
            raise ArgumentError("HDF5 link %r is not a hard link" % name)
        out[name] = struct.unpack_from("<Q", body, p)[0]
    return out


def _read_dataset(buf, msgs):
    dims, dt, addr, size = None, None, UNDEF, 0
    for mtype, body in msgs:
        if mtype == 0x01:
            rank = body[1]
            dims = struct.unpack_from("<%dQ" % rank, body, 4) if rank else ()
        elif mtype == 0x03:
            cls, bits, size_t = body[0] & 0x0F, body[1], struct.unpack_from("<I", body, 4)[0]
            dt = (cls, size_t, bool(bits & 0x08))
        elif mtype == 0x08:
            if body[0] != 3 or body[1] != 1:
                raise ArgumentError("only contiguous HDF5 datasets are read")
            addr, size = struct.unpack_from("<QQ", body, 2)
    if dims is None or dt is None:
        raise ArgumentError("HDF5 dataset without dataspace or datatype")
    raw = bytes(buf[addr:addr + size]) if addr != UNDEF else b""
    cls, tsize, signed = dt
    count = int(np.prod(dims)) if dims else 1
    if cls == 3:
        vals = [raw[i * tsize:(i + 1) * tsize].rstrip(b"\x00").decode("utf-8") for i in range(count)]
        return vals[0] if not dims else vals
    if cls == 1 and tsize == 8:
        a = np.frombuffer(raw, dtype="<f8", count=count).copy()
    elif cls == 0:
        a = np.frombuffer(raw, dtype=("<i%d" if signed else "<u%d") % tsize, count=count).copy()
        if tsize == 1 and not signed and not dims:
            return bool(a[0])
    else:
        raise ArgumentError("unsupported HDF5 datatype class %d (size %d)" % (cls, tsize))
    if not dims:
        return a[0].item()
    return a.reshape(dims)


def _open_tree(buf):
    if bytes(buf[:8]) != _SIG or buf[8] != 2:
        raise ArgumentError("not an HDF5 file with a version-2 superblock")
    if struct.unpack_from("<I", buf, 44)[0] != lookup3(bytes(buf[:44])):
        raise ArgumentError("HDF5 superblock checksum mismatch")
    root = struct.unpack_from("<Q", buf, 36)[0]

    def node(addr):
        msgs = _read_oh(buf, addr)
        if any(t == 0x02 for t, _ in msgs):   # a group (Link Info message)
            return {k: node(a) for k, a in _links(msgs).items()}
        return _read_dataset(buf, msgs)
    return node(root)


def _ordered_keys(g):
    ks = list(g.keys())
    if set(ks) <= set(_COORDINATE):
        return [c for c in _COORDINATE if c in ks]
    return sorted(ks)


def read_GridDataset(filename="PRGridDataset.h5"):
    """Read a GridDataset written by write_GridDataset (read_grids.jl:29-80): params, names, the
    shared coordinate (axis) vectors and grids 1..L, as PointSamples or StructuredGrid sharing
    those vectors.  Reads the HDF5 subset this module writes."""
    from .grids import GridBundle, PointSamples, StructuredGrid
    with open(os.fspath(filename), "rb") as f:
        buf = memoryview(f.read())
    tree = _open_tree(buf)
    if "params" not in tree:
        raise ArgumentError("Schema error: missing /params")
    if "data" not in tree:
        raise ArgumentError("Schema error: missing /data")
    params = dict(tree["params"])
    if "dtype" not in params:
        raise ArgumentError("params missing :dtype")
    if "grid_type" not in params:
        raise ArgumentError("params missing :grid_type")
    if params["dtype"] != "Float64":
        raise ArgumentError("Unsupported dtype string in params[:dtype]: %s" % params["dtype"])
    data = tree["data"]
    names = list(data["names"])
    gg = data["grids"]
    order = sorted(gg.keys(), key=int)
    if len(names) != len(order):
        raise ArgumentError("names length != number of grids")
    if params["grid_type"] == "PointSamples":
        if "coord" not in data:
            raise ArgumentError("Schema error: missing data/coord")
        coor = tuple(data["coord"][k] for k in _ordered_keys(data["coord"]))
        grids = [PointSamples(gg[k], coor) for k in order]
    elif params["grid_type"] == "StructuredGrid":
        if "axes" not in data:
            raise ArgumentError("Schema error: missing data/axes")
        axes = tuple(data["axes"][k] for k in _ordered_keys(data["axes"]))
        grids = []
        for k in order:
            v = gg[k]
            size = tuple(reversed(v.shape))
            grids.append(StructuredGrid(np.ascontiguousarray(v).reshape(-1).reshape(size, order="F"), axes, size))
    else:
        raise ArgumentError("Unsupported params[:grid_type] = %s" % params["grid_type"])
    for g in grids[1:]:   # one set of vectors, as the reference's reader builds it
        if isinstance(g, PointSamples):
            g.coor = grids[0].coor
        else:
            g.axes = grids[0].axes
    return GridDataset(GridBundle(grids, names), params)
