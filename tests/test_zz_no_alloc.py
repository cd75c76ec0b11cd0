"""ymkh_energy_noalloc (partial sums in a static device array, no library
allocation) against ymkh_energy_async (context-owned partials), through the
C ABI.  Collected last so that it also runs after every other GPU test has
used the library in the same process."""
import ctypes as C

import numpy as np
import pytest

from cases import CASES

pytestmark = pytest.mark.gpu


def _energies(lib, run, stream):
    import torch

    from kh_simulations_b200 import _lib

    out = torch.full((2,), float("nan"), dtype=torch.float64, device=run.device)
    _lib.check(lib.ymkh_energy_async(run.ctx, C.c_void_p(out.data_ptr()), C.c_void_p(stream.cuda_stream)),
               "ymkh_energy_async")
    ptrs = (C.c_void_p * 24)(*[run.state[i].data_ptr() for i in range(24)])
    rc = lib.ymkh_energy_noalloc(ptrs, run.d.nx, run.d.nz, C.c_void_p(out.data_ptr() + 8),
                                 C.c_void_p(stream.cuda_stream))
    _lib.check(rc, "ymkh_energy_noalloc")
    stream.synchronize()
    e = out.cpu().numpy()
    return e[0], e[1]


def test_noalloc_energy_equals_context_energy(cuda):
    import torch

    from kh_simulations_b200 import _lib
    from kh_simulations_b200.run import KHRun

    from kh_simulations_b200.config import loads

    lib = _lib.load()
    # 256 x 512 cells: 32 CTA partial sums in the static scratch
    text = CASES["no_filter"].replace("nz_override = 32", "nz_override = 256").replace("nx_override = 48",
                                                                                      "nx_override = 512")
    run = KHRun(loads(text, "noalloc"))
    run.init()
    stream = torch.cuda.Stream()
    # two calls in a row on the same state, then one after a step
    a1, b1 = _energies(lib, run, stream)
    a2, b2 = _energies(lib, run, stream)
    assert np.isfinite(a1) and a1 > 0
    assert b1 == a1 and b2 == a2 and a2 == a1
    run.step(1, stream)
    a3, b3 = _energies(lib, run, stream)
    assert b3 == a3 and a3 != a1
    run.close()


def test_noalloc_energy_rejects_oversize_grid(cuda):
    from kh_simulations_b200 import _lib

    lib = _lib.load()
    ptrs = (C.c_void_p * 24)(*([16] * 24))  # never dereferenced: the size check comes first
    nx, nz = 32768, _lib.NOALLOC_MAX_CELLS // 32768 + 1
    rc = lib.ymkh_energy_noalloc(ptrs, nx, nz, C.c_void_p(16), None)
    assert rc == -1  # YMKH_EINVAL
    buf = C.create_string_buffer(512)
    lib.ymkh_last_error(buf, 512)
    assert b"exceeds the static scratch limit" in buf.value
