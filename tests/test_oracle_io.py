"""The oracle's Fortran edit descriptors (oracle/og_io.py) against strings
worked out by hand from the Fortran standard's output editing rules: the
formats of backup_VOF_write (FORMAT(es17.8e3,7I10), FORMAT(5es25.16e3),
vofmodules.f90:2055-2058) and output_VOF (E14.5, F16.8, I5, I17,
vofmodules.f90:1928-1948)."""
import pytest

from oracle import og_io as io


@pytest.mark.parametrize("v,w,d,e,want", [
    (1.0, 25, 16, 3, "  1.0000000000000000E+000"),
    (-2.5e-7, 25, 16, 3, " -2.4999999999999999E-007"),      # -2.49999999999999988687...e-7
    (0.0, 25, 16, 3, "  0.0000000000000000E+000"),
    (0.1, 25, 16, 3, "  1.0000000000000001E-001"),        # 0.1 = 0.1000000000000000055511...
    (123.456, 17, 8, 3, "  1.23456000E+002"),
    (9.999999999, 17, 8, 3, "  1.00000000E+001"),              # rounding carries into the exponent
    (1e-300, 25, 16, 3, "  1.0000000000000000E-300"),       # 1.00000000000000002505...e-300
])
def test_es(v, w, d, e, want):
    assert io.fortran_es(v, w, d, e) == want


@pytest.mark.parametrize("v,w,d,want", [
    (1.0, 14, 5, "   0.10000E+01"),
    (-0.03125, 14, 5, "  -0.31250E-01"),
    (0.0, 14, 5, "   0.00000E+00"),
    (0.999996, 14, 5, "   0.10000E+01"),
    (0.5, 14, 5, "   0.50000E+00"),
    (1e-120, 14, 5, "    0.10000-119"[-14:]),
    (3.0e15, 14, 5, "   0.30000E+16"),
])
def test_e(v, w, d, want):
    assert io.fortran_e(v, w, d) == want


@pytest.mark.parametrize("v,w,d,want", [
    (0.5, 16, 8, "      0.50000000"),
    (-0.03125, 16, 8, "     -0.03125000"),
    (0.0, 16, 8, "      0.00000000"),
    (12.345678949, 16, 8, "     12.34567895"),
])
def test_f(v, w, d, want):
    assert io.fortran_f(v, w, d) == want


def test_i():
    assert io.fortran_i(42, 5) == "   42" and io.fortran_i(134217728, 17) == "        134217728"


def test_backup_header_and_records(capi, orc):
    d = capi.make_desc((2, 2, 2))
    z = orc.zeros(d)
    txt = io.backup_text(d, z + 1.0, z, z, z, z + 0.5, 0.25, 7).splitlines()
    assert txt[0] == "  2.50000000E-001" + "         7" + "".join(str(v).rjust(10) for v in (1, 6, 1, 6, 1, 6))
    assert len(txt) == 1 + 6 ** 3
    assert txt[1] == ("  1.0000000000000000E+000" + "  0.0000000000000000E+000" * 3 +
                      "  5.0000000000000000E-001")
