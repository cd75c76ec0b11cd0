"""div_rn (division by a grid spacing through its correctly rounded
reciprocal and one Markstein correction, used by the Maxwell kernel) is
bit-identical to the IEEE division a / b: checked on the GPU for every grid
spacing the tests and the benchmark use and for random divisors, on random
numerators over 1400 binades, numerators making the quotient land on or one
ulp beside a double, and special values (signed zeros, infinities, NaN).
Quotients below 2^-900 in magnitude are outside its stated range."""
import ctypes as C
import math
import subprocess
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def checker(cuda, tmp_path_factory):
    out = tmp_path_factory.mktemp("divcheck") / "libdivcheck.so"
    cmd = ["nvcc", "-std=c++17", "-O3", "-fmad=false", "-gencode", "arch=compute_100a,code=sm_100a", "-shared",
           "-Xcompiler", "-fPIC", f"-I{ROOT / 'include'}", f"-I{ROOT / 'kh_simulations_b200' / 'csrc'}",
           str(ROOT / "tests" / "kernels" / "div_rn_check.cu"), "-o", str(out)]
    subprocess.run(cmd, check=True, capture_output=True, timeout=300)
    lib = C.CDLL(str(out))
    lib.div_rn_check.argtypes = [C.c_double, C.c_double, C.c_ulonglong, C.c_longlong, C.c_int,
                                 C.POINTER(C.c_ulonglong), C.POINTER(C.c_double)]
    return lib


def _divisors():
    from kh_simulations_b200.config import derive, loads

    from cases import BASE, CASES

    ds = set()
    texts = [CASES[n] for n in CASES]
    texts += [BASE + f"nz_override = {nz}\nnx_override = {nx}\n"
              for nz, nx in [(256, 512), (4096, 8192), (1024, 2048), (128, 256), (2048, 4096), (4, 8)]]
    for t in texts:
        d = derive(loads(t))
        ds.update([d.dx, d.dz])
    rng = np.random.default_rng(11)
    ds.update(float(x) for x in np.exp(rng.uniform(math.log(1e-4), math.log(1e2), 8)))
    return sorted(ds)


@pytest.mark.parametrize("kind", [0, 1, 2, 3])
def test_div_rn_is_the_ieee_quotient(checker, kind):
    n = (1 << 26) if kind < 3 else 12 * 1000
    for j, b in enumerate(_divisors()):
        bad, first = C.c_ulonglong(0), C.c_double(0.0)
        rc = checker.div_rn_check(b, 1.0 / b, 1234567 + 7919 * j, n, kind, C.byref(bad), C.byref(first))
        assert rc == 0
        assert bad.value == 0, f"b = {b!r}: {bad.value} mismatches, first a = {first.value!r}"
