"""The C-ABI library loads and exports exactly what include/spectral_gpu.h declares (no GPU needed)."""
import ctypes
import os
import re
import subprocess

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "spectral_gpu.h")


def declared():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^SPX_API\s+[\w\s\*]+?\b(spx_\w+)\s*\(", txt, flags=re.M)))


def test_header_declares_the_binding_list():
    from spectral_rs_b200 import _lib
    assert declared() == sorted(_lib.EXPORTS)


def test_library_exports_every_declared_symbol():
    from spectral_rs_b200 import _lib
    lib = _lib.load()
    for name in declared():
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = sorted(set(re.findall(r"\bT (spx_\w+)", out)))
    assert exported == declared()


def test_params_struct_layout_matches_header(tmp_path):
    # the ctypes mirror must match the C struct field by field: compile the header and compare offsets
    from spectral_rs_b200 import _lib
    names = [f[0] for f in _lib.SpxParams._fields_]
    src = tmp_path / "layout.c"
    src.write_text("#include <stdio.h>\n#include <stddef.h>\n#include \"spectral_gpu.h\"\nint main(void) {\n"
                   + f'  printf("%zu\\n", sizeof(spx_params));\n'
                   + "".join(f'  printf("%zu\\n", offsetof(spx_params, {n}));\n' for n in names)
                   + "  return 0;\n}\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert got[0] == ctypes.sizeof(_lib.SpxParams)
    assert got[1:] == [getattr(_lib.SpxParams, n).offset for n in names]


def test_errors_without_device_are_reported_not_crashing():
    # spx_create on a machine without a usable device must fail with a status, not abort
    from spectral_rs_b200 import _lib
    lib = _lib.load()
    prm = _lib.SpxParams(size_x=24, size_y=12, delta=5, dt=0.1, c=3.0, dens=2, gamma_inj=5.0, n_pass=4)
    ctx = ctypes.c_void_p()
    code = lib.spx_create(ctypes.byref(prm), ctypes.byref(ctx))
    assert code == 1  # 24 is not a power of two: rejected before touching a device
    assert b"power-of-two" in lib.spx_last_error(None)


def test_rust_binding_covers_the_header():
    # INTEGRATION.md's extern "C" blocks declare every entry point of the header, no other
    txt = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    assert sorted(set(re.findall(r"pub fn (spx_\w+)", txt))) == declared()
