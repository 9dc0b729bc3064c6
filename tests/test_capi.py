"""The C-ABI library loads and exports every entry point include/paris_b200.h
declares; the host-side mirror and the descriptor match the header; no GPU
compute is called here."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "paris_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(paris_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol(capi):
    path = capi.lib_path()
    assert os.path.exists(path), "libparis_b200.so not built"
    lib = ctypes.CDLL(path)
    names = header_functions()
    assert len(names) >= 25
    for n in names:
        assert hasattr(lib, n), n
    # the ctypes prototypes cover the header
    assert set(names) <= set(capi.exported_names()) | {"paris_gpu_profile_report"}


def test_descriptor_layout_matches_header(capi, tmp_path):
    """sizeof/offsetof of the C structs (compiled with gcc against the header)
    equal the ctypes mirrors."""
    import subprocess
    fields = {"paris_grid_desc": capi.GridDesc, "paris_solve_opts": capi.SolveOpts,
              "paris_solve_result": capi.SolveResult}
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{ROOT}/include/paris_b200.h"',
             "int main(void) {"]
    for cname, ct in fields.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for fname, _ in ct._fields_:
            lines.append(f'printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-o", str(exe), str(src)], check=True)
    out = dict(l.rsplit(" ", 1) for l in subprocess.run([str(exe)], capture_output=True, text=True,
                                                         check=True).stdout.split("\n") if l)
    for cname, ct in fields.items():
        assert int(out[cname]) == ctypes.sizeof(ct), cname
        for fname, _ in ct._fields_:
            assert int(out[f"{cname}.{fname}"]) == getattr(ct, fname).offset, (cname, fname)


def test_init_without_device_fails_cleanly(capi):
    """Without a usable device the library returns NO_DEVICE (or BAD_ARGS for a
    bad descriptor) instead of crashing."""
    lib = capi.load_library()
    h = ctypes.c_void_p()
    bad = capi.make_desc((2, 16, 16))
    assert lib.paris_gpu_init(ctypes.byref(bad), ctypes.byref(h)) == capi.BAD_ARGS
    d = capi.make_desc((16, 16, 16), device=4096)
    st = lib.paris_gpu_init(ctypes.byref(d), ctypes.byref(h))
    assert st in (capi.NO_DEVICE, capi.BAD_ARGS)
    assert not h.value


def test_descriptor_validation_rules(capi):
    """The checks of paris_gpu_init that run before any device call: at least
    four cells across except Nz = 2 (two-dimensional runs); a periodic volume
    fraction needs a periodic velocity, while a periodic velocity may carry
    dry/wet VOF ghosts (the capillary-wave setup).  Accepted descriptors get
    as far as the device (NO_DEVICE here, OK on a GPU)."""
    lib = capi.load_library()

    def status(d):
        h = ctypes.c_void_p()
        st = lib.paris_gpu_init(ctypes.byref(d), ctypes.byref(h))
        if h.value:
            lib.paris_gpu_finalize(h)
        return st

    accepted = (capi.OK, capi.NO_DEVICE)
    assert status(capi.make_desc((16, 16, 2))) in accepted
    assert status(capi.make_desc((16, 16, 3))) == capi.BAD_ARGS
    assert status(capi.make_desc((16, 2, 16))) == capi.BAD_ARGS
    vb = [capi.VOFBC_PERIODIC, capi.VOFBC_WET, capi.VOFBC_WET, capi.VOFBC_PERIODIC, capi.VOFBC_DRY, capi.VOFBC_DRY]
    assert status(capi.make_desc((32, 96, 2), length=(1.0, 3.0, 0.0625), vofbc=vb)) in accepted
    walls_periodic_vof = capi.make_desc((16, 16, 16), bc="wall", vofbc=[capi.VOFBC_PERIODIC] * 6)
    assert status(walls_periodic_vof) == capi.BAD_ARGS
