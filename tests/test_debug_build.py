"""The bounds-checked debug build (libgli_b200_debug.so, compiled with
-DGLI_B200_DEBUG): on valid inputs no device check fires and the values equal
the release build's within the parity bar.  Runs in a subprocess that loads
the debug library through GLI_B200_LIBRARY."""
import os
import subprocess
import sys

import pytest

from _common import GOLDEN

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DEBUG_LIB = os.path.join(REPO, "gausslectronitegrate_b200", "libgli_b200_debug.so")


def test_debug_library_exports_the_same_entry_points():
    import ctypes as C

    from gausslectronitegrate_b200 import _abi
    lib = C.CDLL(DEBUG_LIB)
    for name in _abi.EXPORTS:
        assert hasattr(lib, name), name


@pytest.mark.gpu
def test_debug_build_evaluations_pass_their_bounds_checks():
    code = f"""
import sys, numpy as np
sys.path.insert(0, {REPO!r}); sys.path.insert(0, {os.path.join(REPO, 'tests')!r})
import gausslectronitegrate_b200 as gli
from _common import assert_parity, core, g10
assert gli._abi.LIB_PATH.endswith('libgli_b200_debug.so')
c = core()
s = gli.compute_sparse_erida_gausslet_integrals(g10(), [(-16, 33)] * 3, 1e-16)
assert_parity(s.values, c['erida_val_33_1e-16'], what='debug ERIDA 33^3')
s = gli.compute_sparse_eri_gausslet_integrals(g10(), [(-2, 5)] * 3, 1e-5)
assert_parity(s.values, c['eri_val_5_1e-05'], what='debug ERI 5^3')
s = gli.compute_sparse_eri_gausslet_integrals(g10(), [(-3, 7)] * 3, 1e-10, form='mixed')
assert s.values.size == 3571977
print('debug ok')
"""
    env = dict(os.environ, GLI_B200_LIBRARY=DEBUG_LIB)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env, timeout=900)
    assert r.returncode == 0 and "debug ok" in r.stdout, r.stdout + r.stderr
