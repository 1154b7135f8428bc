"""Generate the small JSON fixtures under tests/golden/ from the reference's own test files.

The reference is Julia and cannot run here, so no reference outputs exist; what its tests
hold for this path are input fixtures and tabulated data.  This script reads them as text
from the reference checkout (its root given as argv[1] or by the PARTIA_REFERENCE environment
variable) and writes:

  grid_interpolation_fixture.json  the 4-particle sets and sample templates of
      Partia.jl/test/grid_interpolation_test_common.jl:17-121
  line_table_samples.json          every 64th node of each Inorm table of
      Partia.jl/src/julia/KernelInterpolation/table/line_integrated_kernel_tables.jl
      (the regenerated tables are checked against these without the reference present)
"""
import json
import math
import os
import re
import sys

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PARTIA_REFERENCE")
if not REF:
    sys.exit("usage: make_fixtures.py <reference checkout root>  (or set PARTIA_REFERENCE)")
OUT = os.path.dirname(os.path.abspath(__file__))


def _body(src, fname):
    i = src.index("function %s(" % fname)
    j = src.index("\nend", i)
    return src[i:j]


def _vec(body, name):
    m = re.search(r"\b%s\s*=\s*Float64\[([^\]]*)\]" % re.escape(name), body)
    return [float(v) for v in m.group(1).split(",")]


def grid_fixture():
    src = open(os.path.join(REF, "Partia.jl/test/grid_interpolation_test_common.jl")).read()
    b = _body(src, "make_grid_interpolation_fixture")
    parts = {k: _vec(b, k) for k in ("x", "y", "z", "h", "rho", "m", "temp", "vx", "vy", "vz")}
    t = _body(src, "make_point_samples_template")
    pts = [_vec(t, k) for k in ("x", "y", "z")]
    lt = _body(src, "make_line_samples_template")
    inv = 1.0 / math.sqrt(2.0)
    blocks = re.findall(r"Float64\[([^\]]*)\]", lt)
    vals = [[inv if v.strip() == "invsqrt2" else float(v) for v in blk.split(",")] for blk in blocks]
    return {"particles": parts, "point_samples": pts, "line_origin": vals[0:3], "line_direction": vals[3:6]}


def table_samples():
    txt = open(os.path.join(REF, "Partia.jl/src/julia/KernelInterpolation/table/line_integrated_kernel_tables.jl")).read()
    out = {}
    for name, body in re.findall(r"const _(\w+)_Inorm = SVector\{4096,Float64\}\(([^)]*)\)", txt, re.S):
        v = [float(s) for s in body.replace("\n", "").split(",") if s.strip()]
        out[name] = {"index": list(range(0, 4096, 64)) + [4095], "value": v[0:4096:64] + [v[4095]]}
    return out


if __name__ == "__main__":
    with open(os.path.join(OUT, "grid_interpolation_fixture.json"), "w") as f:
        json.dump(grid_fixture(), f, indent=1)
    with open(os.path.join(OUT, "line_table_samples.json"), "w") as f:
        json.dump(table_samples(), f, indent=1)
