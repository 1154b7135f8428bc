"""Phantom dump ingest and ParticleIO's adapter to the interpolation input.

  read_phantom            ParticleIO.jl/src/julia/IO/phantomIO/read_phantom.jl:15-320
  ParticleDataFrame       ParticleIO.jl/src/julia/Particles/ParticleDataFrame.jl:18-21
  add_rho                 add_rho! (ParticleIO.jl/src/julia/Particles/add_quantities.jl:294-345)
  build_input             ParticleIO.jl/src/julia/PartiaAdapter/build_input.jl:44-160 (host arrays)
  build_input_device      the same input built on the device: columns uploaded in their stored
                          type (a dump holds h and velocities as real*4) and converted, the density
                          derived from h and the constant mass broadcast by the library's kernels

A Phantom dump is a Fortran sequential unformatted file: every record is framed by a 4-byte
length before and after it.  The records are: the capture pattern (integers 60769, 60878 and
690706, the real 60878 and the format version, which fix the default integer and real
sizes); a 100-character file identifier; eight global-header blocks, one per type (default
integer, int*1, int*2, int*4, int*8, default real, real*4, real*8), each a count, 16-character
names and the values; then the particle arrays: the number of blocks, per block its particle
count and the number of arrays of each type, then per array a 16-character tag and the values.
Block 2 holds the sink particles.  Repeated header names (per-type arrays such as
massoftype) are renamed name, name_2, name_3, ...
"""
import numpy as np

from ._lib import ArgumentError, DimensionMismatch
from .interpolation import InterpolationCatalog, InterpolationInput, M5_spline

CAPTURE_I1, CAPTURE_I2, CAPTURE_I3 = 60769, 60878, 690706


class ParticleDataFrame:
    """Particle columns (name -> 1-D array, all of one length) and the dump's global values."""

    def __init__(self, columns, params):
        self.columns = dict(columns)
        self.params = dict(params)
        lens = {len(v) for v in self.columns.values()}
        if len(lens) > 1:
            raise DimensionMismatch("ParticleDataFrame columns of different lengths: %s" % sorted(lens))

    def names(self):
        return list(self.columns)

    def __getitem__(self, name):
        return self.columns[str(name)]

    def __contains__(self, name):
        return str(name) in self.columns

    def __setitem__(self, name, value):
        self.columns[str(name)] = value

    @property
    def npart(self):
        return len(next(iter(self.columns.values()))) if self.columns else 0

    def select(self, mask):
        return ParticleDataFrame({k: v[mask] for k, v in self.columns.items()}, self.params)


class _Reader:
    def __init__(self, buf):
        self.buf = memoryview(buf)
        self.pos = 0

    def raw(self, n):
        if self.pos + n > len(self.buf):
            raise ArgumentError("truncated Phantom dump (wanted %d bytes at offset %d)" % (n, self.pos))
        b = self.buf[self.pos:self.pos + n]
        self.pos += n
        return b

    def value(self, dtype):
        return np.frombuffer(self.raw(np.dtype(dtype).itemsize), dtype=dtype)[0]

    def record(self, nbytes):
        """One Fortran record of exactly nbytes: the length tags on both sides must agree."""
        head = bytes(self.raw(4))
        data = self.raw(nbytes)
        tail = bytes(self.raw(4))
        if head != tail:
            raise ArgumentError("Fortran tags mismatch.")
        return data


def _dtypes(def_int, def_real):
    return (def_int, np.int8, np.int16, np.int32, np.int64, def_real, np.float32, np.float64)


def _capture_pattern(r):
    """Validates the first record and returns the default integer and real types
    (read_phantom.jl:36-72): int 60769, real 60878, int 60878, version, int 690706.  As in the
    reference, the first integer is tried as int*4 first; with an 8-byte default integer that
    matches the low half of a little-endian 60769, so such a dump fails the following check
    and is refused, as the reference refuses it."""
    r.pos = 0
    head = bytes(r.raw(4))
    def_int, def_real = np.int32, np.float32
    i1 = r.value(def_int)
    if i1 != CAPTURE_I1:
        r.pos -= 4
        def_int = np.int64
        i1 = r.value(def_int)
        if i1 != CAPTURE_I1:
            raise ArgumentError("CapturePatternError: i1 mismatch. Is this a Phantom data file?")
    r1 = r.value(def_real)
    i2 = r.value(def_int)
    if i2 != CAPTURE_I2 or np.float32(i2) != r1:
        r.pos -= 8
        def_real = np.float64
        r1 = r.value(def_real)
        i2 = r.value(def_int)
        if i2 != CAPTURE_I2 or np.float32(i2) != r1:
            raise ArgumentError("CapturePatternError: i2 mismatch. Is this a Phantom data file?")
    version = int(r.value(def_int))
    i3 = r.value(def_int)
    if i3 != CAPTURE_I3:
        raise ArgumentError("CapturePatternError: i3 mismatch. Is this a Phantom data file?")
    if bytes(r.raw(4)) != head:
        raise ArgumentError("CapturePatternError: Fortran tags mismatch. Is this a Phantom data file?")
    return np.dtype(def_int), np.dtype(def_real), version


def _rename_duplicates(keys):
    seen = {}
    out = []
    for k in keys:
        if k not in seen:
            seen[k] = 1
            out.append(k)
        else:
            seen[k] += 1
            out.append("%s_%d" % (k, seen[k]))
    return out


def _header(r, def_int, def_real):
    params = {}
    for dt in _dtypes(def_int, def_real):
        dt = np.dtype(dt)
        nvars = int(np.frombuffer(r.record(4), np.int32)[0])
        if nvars <= 0:
            continue
        keys = bytes(r.record(16 * nvars)).decode("ascii", "replace")
        keys = [keys[16 * i:16 * i + 16].strip() for i in range(nvars)]
        vals = np.frombuffer(r.record(dt.itemsize * nvars), dt)
        for k, v in zip(_rename_duplicates(keys), vals):
            params[k] = v.item()
    return params


def _arrays(r, def_int, def_real):
    nblocks = int(np.frombuffer(r.record(4), np.int32)[0])
    counts, nums = [], []
    for _ in range(nblocks):
        rec = r.record(40)
        counts.append(int(np.frombuffer(rec[:8], np.int64)[0]))
        nums.append(np.frombuffer(rec[8:40], np.int32).copy())
    main, sinks = {}, {}
    dts = _dtypes(def_int, def_real)
    for b in range(nblocks):
        target = sinks if b == 1 else main
        for i, dt in enumerate(dts):
            dt = np.dtype(dt)
            for _ in range(int(nums[b][i])):
                tag = bytes(r.record(16)).decode("ascii", "replace").strip()
                target[tag] = np.frombuffer(r.record(dt.itemsize * counts[b]), dt).copy()
    return main, sinks


def read_phantom(filename, separate_types="sinks", ignore_inactive=True):
    """Read a Phantom dump; returns a list of ParticleDataFrame (read_phantom.jl:273-320).

    separate_types: "sinks" -> [particles, sinks] when the dump has sinks; "all" -> one frame
    per particle type (``itype``) with params["mass"] = massoftype(_k), then the sinks; None ->
    everything in one frame.  ignore_inactive drops particles with h <= 0 (accreted)."""
    with open(filename, "rb") as f:
        r = _Reader(f.read())
    def_int, def_real, version = _capture_pattern(r)
    ident = bytes(r.record(100)).decode("ascii", "replace").strip()
    params = _header(r, def_int, def_real)
    params.update(default_Int=def_int.name, default_Real=def_real.name, file_identifier=ident,
                  COM_coordinate=np.zeros(6), Origin_sink_id=-1, Origin_sink_mass=np.nan, iversion=version)
    main, sinks = _arrays(r, def_int, def_real)
    df = ParticleDataFrame(main, params)
    if ignore_inactive and "h" in df:
        df = df.select(np.asarray(df["h"]) > 0)
    if separate_types == "all" and "itype" in df and len(np.unique(df["itype"])) > 1:
        out = []
        for t in sorted(np.unique(df["itype"])):
            t = int(t)
            key = "massoftype" if t == 1 else "massoftype_%d" % t
            sub = df.select(np.asarray(df["itype"]) == t)
            p = dict(params, mass=params.get(key), itype=t)
            out.append(ParticleDataFrame(sub.columns, p))
        if sinks:
            out.append(ParticleDataFrame(sinks, params))
        return out
    if separate_types in ("sinks", "all") and sinks:
        return [ParticleDataFrame(df.columns, dict(params, mass=None, itype=np.nan)), ParticleDataFrame(sinks, params)]
    cols = dict(df.columns)
    if sinks:
        n0 = df.npart
        ns = len(next(iter(sinks.values())))
        names = list(cols) + [k for k in sinks if k not in cols]
        merged = {}
        for k in names:   # vcat(cols = :union): a column missing from one part is NaN there
            a = cols.get(k)
            b = sinks.get(k)
            dt = np.result_type(*(x.dtype for x in (a, b) if x is not None), np.float32 if (a is None or b is None) else np.int8)
            ca = a.astype(dt) if a is not None else np.full(n0, np.nan, dt)
            cb = b.astype(dt) if b is not None else np.full(ns, np.nan, dt)
            merged[k] = np.concatenate([ca, cb])
        cols = merged
    return [ParticleDataFrame(cols, dict(params, mass=None, itype=None))]


def add_rho(df):
    """add_rho! in 3D (add_quantities.jl:308-345): rho = (m hfact^3) (1/h)^3 for one particle
    mass m = params["mass"] shared by all particles, in that operation order."""
    if "mass" not in df.params or df.params["mass"] is None:
        raise KeyError("Missing required parameter :mass in data.params.")
    m = float(df.params["mass"])
    hfact = float(df.params["hfact"])
    h = np.asarray(df["h"], np.float64)
    mhfactd = m * hfact * hfact * hfact
    invh = 1.0 / h
    df["rho"] = mhfactd * (invh * invh * invh)
    return df


class MassFromColumn:
    """Particle mass from a column of the frame (MassSource.jl)."""

    def __init__(self, name):
        self.name = str(name)


class MassFromParams:
    """One particle mass for all particles from the frame's params (MassSource.jl)."""

    def __init__(self, name):
        self.name = str(name)


def _quantity_columns(scalars, gradients, divergences, curls):
    """Extra columns the catalog needs, in first-use order (build_input.jl:190-219): scalars,
    gradients, then x/y/z components of each divergence and curl vector."""
    names = []
    for n in list(scalars) + list(gradients):
        if n not in names:
            names.append(n)
    for v in list(divergences) + list(curls):
        for c in ("x", "y", "z"):
            if v + c not in names:
                names.append(v + c)
    return tuple(names)


def _check_columns(df, names, mass_from):
    missing = [b for b in ("x", "y", "z", "h", "rho") if b not in df]
    if isinstance(mass_from, MassFromColumn) and mass_from.name not in df and mass_from.name not in missing:
        missing.append(mass_from.name)
    missing += [n for n in names if n not in df and n not in missing]
    if missing:
        raise ArgumentError("Missing columns in ParticleDataFrame: " + ", ".join(missing))
    if isinstance(mass_from, MassFromParams) and mass_from.name not in df.params:
        raise ArgumentError("Missing parameter in ParticleDataFrame.params: %s" % mass_from.name)


def build_input(df, mass_from, scalars=(), gradients=(), divergences=(), curls=(), smoothed_kernel=M5_spline):
    """ParticleIO's build_input on host arrays: float64 copies of x, y, z, m, h, rho and the
    catalog's quantity columns, and the catalog (build_input.jl:44-160)."""
    names = _quantity_columns(scalars, gradients, divergences, curls)
    _check_columns(df, names, mass_from)
    n = df.npart
    m = (np.asarray(df[mass_from.name], np.float64) if isinstance(mass_from, MassFromColumn)
         else np.full(n, float(df.params[mass_from.name])))
    col = lambda k: np.array(df[k], dtype=np.float64)   # noqa: E731  (fresh arrays: LinearBVH! permutes them)
    inp = InterpolationInput(col("x"), col("y"), col("z"), m, col("h"), col("rho"), tuple(col(k) for k in names),
                             smoothed_kernel=smoothed_kernel)
    cat = InterpolationCatalog(names, scalars=scalars, gradients=gradients, divergences=divergences, curls=curls)
    return inp, cat


def build_input_device(df, mass_from, backend, scalars=(), gradients=(), divergences=(), curls=(),
                       smoothed_kernel=M5_spline, rho_from_h=False):
    """The same input as build_input, built on the backend's device: every column is uploaded
    in its stored type (float32 or float64; half the bytes for a dump's real*4 columns) and
    converted to float64 there; a constant mass (MassFromParams) is broadcast on the device,
    and with ``rho_from_h`` the density is derived from h there (add_rho!) instead of read.
    Returns (InterpolationInput of CUDA tensors, InterpolationCatalog)."""
    import torch
    from ._lib import ptr
    names = _quantity_columns(scalars, gradients, divergences, curls)
    if rho_from_h:
        need = [k for k in ("x", "y", "z", "h") if k not in df] + [k for k in names if k not in df and k != "rho"]
        if need:
            raise ArgumentError("Missing columns in ParticleDataFrame: " + ", ".join(need))
        if df.params.get("mass") is None:
            raise KeyError("Missing required parameter :mass in data.params.")
    else:
        _check_columns(df, names, mass_from)
    H = backend.handle
    dev = "cuda:%d" % backend.device
    n = df.npart

    def upload(a):
        a = np.ascontiguousarray(a)
        if a.dtype not in (np.float32, np.float64):
            a = a.astype(np.float64)
        raw = torch.from_numpy(a).to(dev)
        out = torch.empty(n, dtype=torch.float64, device=dev)
        H.check(H.lib.pb_column_to_f64(H.h, raw.data_ptr(), 1 if a.dtype == np.float32 else 0, n, out.data_ptr()),
                "build_input_device")
        return out

    x, y, z, h = (upload(df[k]) for k in ("x", "y", "z", "h"))
    if isinstance(mass_from, MassFromColumn):
        m = upload(df[mass_from.name])
    else:
        m = torch.empty(n, dtype=torch.float64, device=dev)
        H.check(H.lib.pb_fill_f64(H.h, float(df.params[mass_from.name]), n, m.data_ptr()), "build_input_device")
    if rho_from_h:
        rho = torch.empty(n, dtype=torch.float64, device=dev)
        H.check(H.lib.pb_density_from_h(H.h, ptr(h), n, float(df.params["mass"]), float(df.params["hfact"]),
                                        rho.data_ptr()), "build_input_device")
    else:
        rho = upload(df["rho"])
    # a "rho" quantity column is the density itself (derived from h when rho_from_h, as add_rho!
    # followed by build_input gives it)
    quant = tuple(rho.clone() if (k == "rho" and rho_from_h) else upload(df[k]) for k in names)
    inp = InterpolationInput(x, y, z, m, h, rho, quant, smoothed_kernel=smoothed_kernel)
    cat = InterpolationCatalog(names, scalars=scalars, gradients=gradients, divergences=divergences, curls=curls)
    return inp, cat
