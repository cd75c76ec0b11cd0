"""The debug build (libymkh_debug.so, -DYMKH_DEBUG=1): its fused kernels
check every global row copy and store against the array's extent and every
staged row against its shared-memory slot; a failed check is recorded in the
error word (YMKH_ERR_BOUNDS) and the access skipped.  On the parity cases
(every stage and run mode at 32 x 48, ragged 27 x 37), the tiny grids the
library accepts, and strips with TMA and per-element rows (walls, warm_T),
it must report a clean error word and give the release build's state bit
for bit.  Each build runs in its own process (one library per process)."""
from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]

CHILD = r'''
import ctypes as C, hashlib, json, sys
sys.path.insert(0, sys.argv[2]); sys.path.insert(0, sys.argv[2] + "/tests")
import numpy as np, torch
from kh_simulations_b200 import _lib
_lib.LIB_PATH = type(_lib.LIB_PATH)(sys.argv[1])
from kh_simulations_b200.config import loads
from kh_simulations_b200.run import KHRun
from cases import BASE, CASES
texts = dict(CASES)
for nz, nx in ((4, 8), (6, 6), (5, 13), (8, 10)):
    texts[f"tiny_{nz}x{nx}"] = BASE + f"nz_override = {nz}\nnx_override = {nx}\n"
texts["bulk_512"] = BASE + "nz_override = 48\nnx_override = 512\nkz_keep_max = 15\n"
texts["wall_300"] = BASE.replace("run_mode = 6", "run_mode = 0") + "nz_override = 32\nnx_override = 300\n"
texts["warm_250"] = BASE + "nz_override = 40\nnx_override = 250\nwarm_T = 0.01\n"
lib = _lib.load()
out = {"flags": int(lib.ymkh_build_flags()), "cases": {}}
for name, text in sorted(texts.items()):
    for mode in (_lib.FCT_FUSED, _lib.FCT_SPLIT):
        run = KHRun(loads(text, name))
        _lib.check(lib.ymkh_set_fct_mode(run.ctx, mode), "mode")
        if name.startswith("tiny"):
            d = run.d
            s0 = np.random.default_rng(d.nz * 100 + d.nx).normal(size=(24, d.nz, d.nx)) * 1e-3
            s0[12] += 1.0
            s0[18] += 1.0
            run.set_state(s0)
        else:
            run.init()
        run.step(3)
        torch.cuda.synchronize()
        rc = lib.ymkh_check(run.ctx, None)
        h = hashlib.sha1(run.state_numpy().tobytes()).hexdigest()
        out["cases"][f"{name}/{mode}"] = {"check": int(rc), "hash": h}
        run.close()
print("RESULT " + json.dumps(out))
'''


def _run(lib: Path) -> dict:
    p = subprocess.run([sys.executable, "-c", CHILD, str(lib), str(ROOT)], capture_output=True, text=True,
                       timeout=900)
    line = [ln for ln in p.stdout.splitlines() if ln.startswith("RESULT ")]
    assert p.returncode == 0 and line, p.stderr[-3000:]
    return json.loads(line[0][7:])


def test_debug_build_clean_and_identical(cuda):
    from kh_simulations_b200 import _lib
    from kh_simulations_b200 import build as b

    b.build(debug=True)  # normally built by build(); compiled here if absent or stale
    rel = _run(_lib.LIB_PATH)
    dbg = _run(_lib.DEBUG_LIB_PATH)
    assert rel["flags"] == 0 and dbg["flags"] == _lib.YMKH_BUILD_DEBUG
    assert rel["cases"].keys() == dbg["cases"].keys()
    for k, v in dbg["cases"].items():
        assert v["check"] == 0, (k, v)  # no out-of-range access, no timed-out wait
        assert v["hash"] == rel["cases"][k]["hash"], k
