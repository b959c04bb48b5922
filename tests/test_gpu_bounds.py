"""The index-checked debug build (libsns_b200_check.so, -DSNS_BOUNDS_CHECK) on the GPU.

Every shared-memory, tensor-memory and global index of the TMA-fed y/z passes, the two-stage
x pass and the fused forward-z + sweep is checked against its buffer in that build (an index
outside is recorded and replaced by 0).  A fresh process loads it (SNS_B200_LIB=check), runs
steps and right-hand sides of both forms at N = 32, 48, 128, 256 and 512 (every pass kernel
variant, sphere pruning, the radix-32 lane-pair x pass, the compensated sweep), checks one
RHS against the CPU oracle, and asserts that no index left its buffer.
"""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import ctypes as C, json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from spectral_solver_b200 import _lib, Solver
from oracle.ref_r2c import TaylorGreenR2C, half_to_full
lib = _lib.load()
assert lib._name.endswith("libsns_b200_check.so"), lib._name
out = {}
for n in (32, 48, 128, 256, 512):
    for prec in (0, 1):
        with Solver(n, 1600.0, seed=1, pert_amp=1e-3, pert_kmax=4, precision=prec) as s:
            s.step(1e-3, 2 if n < 512 else 1)
            if n <= 48 and prec == 0:
                o = TaylorGreenR2C(n, 1600.0)
                r = s.rhs([half_to_full(c) for c in o.u_hat])
                ref = [half_to_full(c) for c in o.compute_rhs()]
                num = sum(float(np.sum(np.abs(a - b) ** 2)) for a, b in zip(r, ref))
                den = sum(float(np.sum(np.abs(b) ** 2)) for b in ref)
                out[f"rhs_rel_l2_{n}"] = (num / den) ** 0.5
            out[f"E_{n}_{prec}"] = s.diagnostics(0.0)["kinetic_energy"]
cnt, line, idx = C.c_longlong(), C.c_int(), C.c_longlong()
assert lib.sns_debug_bounds(C.byref(cnt), C.byref(line), C.byref(idx)) == 0
out.update(count=cnt.value, line=line.value, index=idx.value)
print(json.dumps(out))
"""


def test_no_index_leaves_its_buffer():
    if not os.path.exists(os.path.join(ROOT, "spectral_solver_b200", "libsns_b200_check.so")):
        pytest.fail("libsns_b200_check.so is missing: run __graft_entry__.build()")
    env = dict(os.environ, SNS_B200_LIB="check")
    r = subprocess.run([sys.executable, "-c", SCRIPT, ROOT], capture_output=True, text=True, timeout=900, env=env,
                       cwd=ROOT)
    assert r.returncode == 0, r.stderr[-3000:]
    res = json.loads(r.stdout.strip().splitlines()[-1])
    assert res["count"] == 0, res
    for n in (32, 48):
        assert res[f"rhs_rel_l2_{n}"] < 1e-12
    assert all(0.1 < v < 0.13 for k, v in res.items() if k.startswith("E_"))


def test_normal_build_has_no_checks(lib):
    import ctypes as C
    cnt = C.c_longlong(0)
    assert lib.sns_debug_bounds(C.byref(cnt), None, None) == 0
    assert cnt.value == -1
