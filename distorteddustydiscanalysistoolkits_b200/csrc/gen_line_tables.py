"""Regenerate the 4096-point line-integrated (column) SPH kernel tables.

For each 3D kernel w(q) = sigma3 * f(q) with support radius q_max, the table holds

    Inorm(q_perp) = sigma3 * integral_{-inf}^{inf} f(sqrt(q_perp^2 + s^2)) ds

at the nodes q_k = k * q_max / 4095 (k = 0 .. 4095), which is what Partia's
tabulated lookup expects (Partia.jl/src/julia/KernelInterpolation/kernel_function/
line_integrated_kernel.jl:13-19 reads `Q[2]-Q[1]` as the node spacing and
linearly interpolates `Inorm`).  The tables are computed here from the kernel
formulas (Partia.jl/src/julia/KernelInterpolation/kernel_function/kernels/*.jl),
not copied: for q_perp > 0 the substitution s = q_perp*sinh(t) makes the
integrand smooth in t, each piece between the kernel's breakpoints is integrated
with 128-node Gauss-Legendre quadrature, and q_perp = 0 integrates the
piecewise polynomial exactly.

Output: a C header with the initializer macro PB_LINE_INORM_INIT for a
`double [6][4096]` table and the support radii, included by the CUDA library and by the CPU oracle so both use
bit-identical tables.  Run: python gen_line_tables.py <out.h>
"""
import sys

import numpy as np

NTAB = 4096

# kernel id order used across the C ABI: M4, M5, M6, C2, C4, C6
KERNELS = ("M4_spline", "M5_spline", "M6_spline", "C2_Wendland", "C4_Wendland", "C6_Wendland")
QMAX = {"M4_spline": 2.0, "M5_spline": 2.5, "M6_spline": 3.0,
        "C2_Wendland": 2.0, "C4_Wendland": 2.0, "C6_Wendland": 2.0}
SIGMA3 = {"M4_spline": 1.0 / np.pi, "M5_spline": 0.05 / np.pi, "M6_spline": 1.0 / (120.0 * np.pi),
          "C2_Wendland": 21.0 / (16.0 * np.pi), "C4_Wendland": 495.0 / (256.0 * np.pi),
          "C6_Wendland": 1365.0 / (512.0 * np.pi)}
BREAKS = {"M4_spline": (1.0,), "M5_spline": (0.5, 1.5), "M6_spline": (1.0, 2.0),
          "C2_Wendland": (), "C4_Wendland": (), "C6_Wendland": ()}


def shape(name, r):
    """Dimensionless kernel shape f(r) for r >= 0 (vectorised)."""
    r = np.asarray(r, dtype=np.float64)
    out = np.zeros_like(r)
    if name == "M4_spline":
        a = r < 1.0
        b = (r >= 1.0) & (r < 2.0)
        out[a] = 0.25 * (2.0 - r[a]) ** 3 - (1.0 - r[a]) ** 3
        out[b] = 0.25 * (2.0 - r[b]) ** 3
    elif name == "M5_spline":
        a = r < 0.5
        b = (r >= 0.5) & (r < 1.5)
        c = (r >= 1.5) & (r < 2.5)
        out[a] = (2.5 - r[a]) ** 4 - 5.0 * (1.5 - r[a]) ** 4 + 10.0 * (0.5 - r[a]) ** 4
        out[b] = (2.5 - r[b]) ** 4 - 5.0 * (1.5 - r[b]) ** 4
        out[c] = (2.5 - r[c]) ** 4
    elif name == "M6_spline":
        a = r < 1.0
        b = (r >= 1.0) & (r < 2.0)
        c = (r >= 2.0) & (r < 3.0)
        out[a] = (3.0 - r[a]) ** 5 - 6.0 * (2.0 - r[a]) ** 5 + 15.0 * (1.0 - r[a]) ** 5
        out[b] = (3.0 - r[b]) ** 5 - 6.0 * (2.0 - r[b]) ** 5
        out[c] = (3.0 - r[c]) ** 5
    elif name == "C2_Wendland":
        a = r < 2.0
        out[a] = (1.0 - 0.5 * r[a]) ** 4 * (2.0 * r[a] + 1.0)
    elif name == "C4_Wendland":
        a = r < 2.0
        out[a] = (1.0 - 0.5 * r[a]) ** 6 * (35.0 / 12.0 * r[a] ** 2 + 3.0 * r[a] + 1.0)
    elif name == "C6_Wendland":
        a = r < 2.0
        out[a] = (1.0 - 0.5 * r[a]) ** 8 * (4.0 * r[a] ** 3 + 6.25 * r[a] ** 2 + 4.0 * r[a] + 1.0)
    else:
        raise KeyError(name)
    return out


_GL_X, _GL_W = np.polynomial.legendre.leggauss(128)


def _gl(fun, a, b):
    if b <= a:
        return 0.0
    x = 0.5 * (b - a) * _GL_X + 0.5 * (b + a)
    return 0.5 * (b - a) * float(np.dot(_GL_W, fun(x)))


def column_integral(name, q):
    """integral_{-inf}^{inf} f(sqrt(q^2+s^2)) ds (no normalisation)."""
    qmax = QMAX[name]
    if q >= qmax:
        return 0.0
    if q == 0.0:
        knots = [0.0] + [b for b in BREAKS[name] if b < qmax] + [qmax]
        return 2.0 * sum(_gl(lambda s: shape(name, s), knots[i], knots[i + 1]) for i in range(len(knots) - 1))
    # s = q sinh t  =>  r = q cosh t,  ds = q cosh t dt
    tk = [0.0] + [float(np.arccosh(b / q)) for b in BREAKS[name] if b > q] + [float(np.arccosh(qmax / q))]
    tk = sorted(tk)

    def g(t):
        c = np.cosh(t)
        return shape(name, q * c) * q * c

    return 2.0 * sum(_gl(g, tk[i], tk[i + 1]) for i in range(len(tk) - 1))


def tables():
    out = {}
    for name in KERNELS:
        qmax = QMAX[name]
        qs = np.arange(NTAB, dtype=np.float64) * qmax / (NTAB - 1)
        inorm = np.array([SIGMA3[name] * column_integral(name, float(q)) for q in qs])
        inorm[-1] = 0.0
        out[name] = (qs, inorm)
    return out


def write_header(path):
    """Writes PB_LINE_INORM_INIT, an initializer usable for host and device arrays."""
    tabs = tables()
    lines = ["/* Generated by gen_line_tables.py from the kernel formulas; do not edit. */",
             "#pragma once", "#define PB_LINE_NTAB %d" % NTAB,
             "static const double PB_LINE_QMAX[6] = {%s};" % ", ".join(repr(QMAX[k]) for k in KERNELS),
             "#define PB_LINE_INORM_INIT { \\"]
    for name in KERNELS:
        vals = tabs[name][1]
        lines.append("  { /* %s */ \\" % name)
        for i in range(0, NTAB, 4):
            lines.append("    " + ", ".join("%.17e" % v for v in vals[i:i + 4]) + ", \\")
        lines.append("  }, \\")
    lines.append("}")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


if __name__ == "__main__":
    write_header(sys.argv[1] if len(sys.argv) > 1 else "line_tables.h")
