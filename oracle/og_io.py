"""Oracle of the on-disk formats (test infrastructure only): the Fortran edit
descriptors of backup_VOF_write (vofmodules.f90:2033-2059) and output_VOF
(vofmodules.f90:1908-2031) restated in Python with exact decimal arithmetic,
and the two files built from numpy arrays in the reference layout.

Fortran output editing, as the Fortran standard (F2008 10.7.2) defines it:
  Iw      the integer right-justified in w characters;
  Fw.d    fixed point, d digits after the point;
  Ew.d    0.d1..dd with a decimal exponent, E+ee, or +eee without the E
          when |exponent| > 99 (a zero is 0.00..0E+00);
  ESw.dEe one non-zero digit before the point, d after, E and e exponent
          digits;
each rounded to nearest and right-justified in w characters."""
from decimal import ROUND_HALF_EVEN, Decimal

import numpy as np


def _sig(v, nd):
    """(sign, digits, e10): |v| = 0.digits * 10**e10 to nd significant digits."""
    d = Decimal(float(v))
    sign = "-" if d.is_signed() else ""
    d = abs(d)
    if d == 0:
        return sign, "0" * nd, 0
    e10 = d.adjusted() + 1                      # d = 0.xxx * 10**e10
    q = d.scaleb(-e10).quantize(Decimal(1).scaleb(-nd), rounding=ROUND_HALF_EVEN)
    if q >= 1:                                  # rounding carried into a new digit
        e10 += 1
        q = d.scaleb(-e10).quantize(Decimal(1).scaleb(-nd), rounding=ROUND_HALF_EVEN)
    digits = str(q)[2:].ljust(nd, "0")
    return sign, digits, e10


def fortran_i(v, w):
    return str(int(v)).rjust(w)


def fortran_f(v, w, d):
    q = Decimal(float(v)).quantize(Decimal(1).scaleb(-d), rounding=ROUND_HALF_EVEN)
    s = format(q, "f")
    if Decimal(float(v)).is_signed() and not s.startswith("-"):
        s = "-" + s
    return s.rjust(w)


def fortran_e(v, w, d):
    sign, digits, e10 = _sig(v, d)
    ae = abs(e10)
    exp = ("E%s%02d" % ("-" if e10 < 0 else "+", ae)) if ae <= 99 else ("%s%03d" % ("-" if e10 < 0 else "+", ae))
    return (sign + "0." + digits + exp).rjust(w)


def fortran_es(v, w, d, e):
    sign, digits, e10 = _sig(v, d + 1)
    ex = e10 - 1 if float(v) != 0.0 else 0
    return (sign + digits[0] + "." + digits[1:] + "E%s%0*d" % ("-" if ex < 0 else "+", e, abs(ex))).rjust(w)


def backup_text(desc, u, v, w, p, cvof, time, itimestep):
    """The restart file of backup_VOF_write for one rank."""
    g = desc.ng
    lim = (1, desc.nx + 2 * g, 1, desc.ny + 2 * g, 1, desc.nz + 2 * g)
    out = [fortran_es(time, 17, 8, 3) + fortran_i(itimestep, 10) + "".join(fortran_i(a, 10) for a in lim)]
    fl = [np.ascontiguousarray(a).reshape(-1) for a in (u, v, w, p, cvof)]
    for t in range(fl[0].size):
        out.append("".join(fortran_es(a[t], 25, 16, 3) for a in fl))
    return "\n".join(out) + "\n"


B1, B2, B3, B4 = 8.0 / 64, 4.0 / 64, 2.0 / 64, 1.0 / 64


def vtk_text(desc, cvof, coords, fmt, time, index_range=None, filtered=False):
    """output_VOF_VTKSG (fmt 2) / output_VOF_VTKSP (fmt 3) of cvof over the
    Fortran index box index_range (default is..ie+1, js..je+1, ks..ke+1);
    coords: the x, y, z cell centres indexed Fortran-1."""
    g = desc.ng
    r = index_range or (g + 1, g + desc.nx + 1, g + 1, g + desc.ny + 1, g + 1, g + desc.nz + 1)
    x, y, z = coords["x"], coords["y"], coords["z"]
    np_ = (r[1] - r[0] + 1) * (r[3] - r[2] + 1) * (r[5] - r[4] + 1)
    out = ["# vtk DataFile Version 2.0", "grid, time " + fortran_f(time, 16, 8), "ASCII"]
    dims = "DIMENSIONS " + "".join(fortran_i(r[2 * a + 1] - r[2 * a] + 1, 5) for a in range(3))
    if fmt == 3:
        out += ["DATASET STRUCTURED_POINTS", dims,
                "ORIGIN " + "".join(fortran_f(c[r[2 * a] - 1], 16, 8) for a, c in enumerate((x, y, z))),
                "SPACING " + "".join(fortran_f(c[r[2 * a]] - c[r[2 * a] - 1], 16, 8) for a, c in enumerate((x, y, z)))]
    else:
        out += ["DATASET STRUCTURED_GRID", dims, "POINTS " + fortran_i(np_, 17) + " double"]
        for k in range(r[4], r[5] + 1):
            for j in range(r[2], r[3] + 1):
                for i in range(r[0], r[1] + 1):
                    out.append(fortran_e(x[i - 1], 14, 5) + fortran_e(y[j - 1], 14, 5) + fortran_e(z[k - 1], 14, 5))
    out += ["POINT_DATA " + fortran_i(np_, 17), "SCALARS " + "VOF".rjust(20) + " float 1", "LOOKUP_TABLE default"]
    c = cvof   # (k, j, i) with C index = Fortran index - 1

    def at(i, j, k):
        return float(c[k - 1, j - 1, i - 1])

    for k in range(r[4], r[5] + 1):
        for j in range(r[2], r[3] + 1):
            for i in range(r[0], r[1] + 1):
                if filtered:
                    val = (B1 * at(i, j, k)
                           + B2 * (at(i - 1, j, k) + at(i, j - 1, k) + at(i, j, k - 1) + at(i + 1, j, k)
                                   + at(i, j + 1, k) + at(i, j, k + 1))
                           + B3 * (at(i + 1, j + 1, k) + at(i + 1, j - 1, k) + at(i - 1, j + 1, k)
                                   + at(i - 1, j - 1, k) + at(i + 1, j, k + 1) + at(i + 1, j, k - 1)
                                   + at(i - 1, j, k + 1) + at(i - 1, j, k - 1) + at(i, j + 1, k + 1)
                                   + at(i, j + 1, k - 1) + at(i, j - 1, k + 1) + at(i, j - 1, k - 1))
                           + B4 * (at(i + 1, j + 1, k + 1) + at(i + 1, j + 1, k - 1) + at(i + 1, j - 1, k + 1)
                                   + at(i + 1, j - 1, k - 1) + at(i - 1, j + 1, k + 1) + at(i - 1, j + 1, k - 1)
                                   + at(i - 1, j - 1, k + 1) + at(i - 1, j - 1, k - 1)))
                else:
                    val = at(i, j, k)
                out.append(fortran_e(val, 14, 5))
    return "\n".join(out) + "\n"
