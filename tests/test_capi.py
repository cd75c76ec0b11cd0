"""The C ABI library builds, loads and exports exactly what include/ymkh.h
declares (no GPU needed; no kernel is launched here)."""
import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared():
    text = (ROOT / "include" / "ymkh.h").read_text()
    return set(re.findall(r"^\s*(?:int|long long|const char\*)\s+(ymkh_\w+)\s*\(", text, re.M))


def test_header_declares_core_entry_points():
    need = {"ymkh_create", "ymkh_bind_state", "ymkh_init", "ymkh_step", "ymkh_energy", "ymkh_mode_amp",
            "ymkh_destroy", "ymkh_last_error"}
    assert need <= declared()


def test_library_exports_every_declared_symbol(built):
    from kh_simulations_b200 import _lib

    lib = _lib.load()
    nm = subprocess.run(["nm", "-D", "--defined-only", str(_lib.LIB_PATH)], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (ymkh_\w+)", nm))
    missing = declared() - exported
    assert not missing, missing
    for name in declared():
        assert getattr(lib, name) is not None
    assert set(_lib.EXPORTED) <= exported


def test_errors_are_reported_not_raised(built):
    import ctypes as C

    from kh_simulations_b200 import _lib

    lib = _lib.load()
    rc = lib.ymkh_create(None, None, None)
    assert rc == -1
    assert "null" in _lib.last_error()
    rc = lib.ymkh_step(None, 1, None)
    assert rc == -1


def test_struct_layout_matches_header():
    """ctypes mirrors of ymkh_grid / ymkh_params / ymkh_init_params have the C sizes."""
    import ctypes as C
    import tempfile

    from kh_simulations_b200._lib import Grid, InitParams, Params

    src = r'''
#include <stdio.h>
#include "ymkh.h"
int main(void){printf("%zu %zu %zu\n", sizeof(ymkh_grid), sizeof(ymkh_params), sizeof(ymkh_init_params));return 0;}
'''
    with tempfile.TemporaryDirectory() as td:
        c = Path(td) / "s.c"
        c.write_text(src)
        exe = Path(td) / "s"
        subprocess.run(["gcc", "-I", str(ROOT / "include"), str(c), "-o", str(exe)], check=True)
        sizes = list(map(int, subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()))
    assert sizes == [C.sizeof(Grid), C.sizeof(Params), C.sizeof(InitParams)]


def test_c_program_links_every_entry_point(built):
    """A C program that takes the address of every entry point the header
    declares compiles with gcc against include/ymkh.h and links against
    libymkh.so: what a maintainer's shim beside main_ym.cu needs."""
    import re
    import tempfile

    header = (ROOT / "include" / "ymkh.h").read_text()
    names = sorted(set(re.findall(r"^\s*(?:int|long long)\s+(ymkh_\w+)\s*\(", header, flags=re.M)))
    assert len(names) >= 30
    src = "#include <stdio.h>\n#include \"ymkh.h\"\nint main(void){\n  void* fns[] = {\n"
    src += ",\n".join(f"    (void*){n}" for n in names)
    src += "\n  };\n  int n = 0;\n  for (unsigned i = 0; i < sizeof fns / sizeof fns[0]; ++i) n += fns[i] != 0;\n"
    src += "  printf(\"%d\\n\", n);\n  return 0;\n}\n"
    libdir = ROOT / "kh_simulations_b200"
    cuda_lib = Path("/usr/local/cuda/lib64")
    with tempfile.TemporaryDirectory() as td:
        c = Path(td) / "shim.c"
        c.write_text(src)
        exe = Path(td) / "shim"
        cmd = ["gcc", "-I", str(ROOT / "include"), str(c), "-o", str(exe), "-L", str(libdir), "-lymkh",
               f"-Wl,-rpath,{libdir}", "-Wl,--allow-shlib-undefined"]
        if cuda_lib.exists():
            cmd += [f"-Wl,-rpath,{cuda_lib}"]
        subprocess.run(cmd, check=True)
        out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.strip()
    assert int(out) == len(names)
