"""Drop-in check: the reference's own Python module (python/pymodule.c),
compiled unchanged against include/ and linked to libgli_b200.so by
``make -C oracle dropin`` (output oracle/_ref/dropin/, built where the
reference tree exists and carried with the repository), runs on top of this
library.  Each check runs in a subprocess so that the two modules' state stay
apart."""
import os
import subprocess
import sys

import pytest

from _common import GOLDEN

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DROPIN_DIR = os.path.join(REPO, "oracle", "_ref", "dropin")
HAVE = os.path.exists(os.path.join(DROPIN_DIR, "gausslectronitegrate_pymodule.so"))

needs_dropin = pytest.mark.skipif(not HAVE, reason="drop-in module not built (make -C oracle dropin)")


def _run(code):
    # the module directory goes in front of whatever the caller's PYTHONPATH holds
    # (a replaced path would hide the caller's own import hooks from the child)
    prev = os.environ.get("PYTHONPATH", "")
    env = dict(os.environ, PYTHONPATH=DROPIN_DIR + (os.pathsep + prev if prev else ""))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0, f"drop-in run failed:\n{r.stdout}\n{r.stderr}"
    return r.stdout


@needs_dropin
def test_dropin_imports_and_grid_helpers():
    out = _run("import gausslectronitegrate_pymodule as m;"
               "print(m.grid_num_points([(-1,3),(-2,5),(-2,4)]), m.grid_point_to_linear_index([(-1,3),(0,2),(-2,4)],[0,0,0]),"
               " m.linear_index_to_grid_point([(-1,3),(0,2),(-2,4)], 10))")
    assert out.split()[:2] == ["60", "10"]


@needs_dropin
@pytest.mark.gpu
def test_dropin_notebook_answers_on_gpu():
    code = f"""
import json, numpy as np, gausslectronitegrate_pymodule as gli
b = np.load({os.path.join(GOLDEN, 'reference_fixtures.npz')!r})['g10']
nb = json.load(open({os.path.join(GOLDEN, 'notebook_outputs.json')!r}))['notebook_outputs']
close = lambda x, y: abs(x - float(y)) <= 1e-12 * abs(float(y)) + 1e-14
eri = gli.compute_sparse_eri_gausslet_integrals(b, [(-1, 3)] * 3, 1e-16)
assert eri.num_entries == int(nb['eri_integrals'][4])
assert close(eri.integral_value(([1, 0, 0], [0, 0, -1], [0, 0, 1], [0, 0, 0])), nb['eri_integrals'][6])
assert close(gli.compute_eri_gausslet_integral(b, ([0, 0, 0],) * 4, 1e-16), nb['eri_integrals'][0])
erida = gli.compute_sparse_erida_gausslet_integrals(b, [(-3, 7)] * 3, 1e-16)
assert erida.num_entries == int(nb['erida_integrals'][4])
assert close(erida.integral_value(([-1, 0, 2], [0, 1, -1])), nb['erida_integrals'][6])
m = erida.fill_matrix([(-3, 7)] * 3)
assert np.linalg.norm(m - m.T) == 0.0
kgi = gli.compute_kinetic_gausslet_integrals(b, [(-1, 3), (-2, 5), (-2, 4)])
assert close(kgi[7, 7], nb['kinetic_integrals'][3])
pos, ch = [(-0.2, 1.3, 0.5), (0.7, 0, -2.1)], [2, 1]
ngi = gli.compute_nuclear_gausslet_integrals(b, [(-1, 3), (0, 2), (-2, 4)], pos, ch, 1e-16)
assert close(ngi[10, 10], nb['nuclear_integrals'][4])
basis = np.linalg.qr(np.random.default_rng(293).normal(size=(27, 27)))[0][:, :5]
p = eri.project(basis)
dense = eri.fill_tensor([(-1, 3)] * 3)
ref = np.einsum(basis, (4, 0), basis, (5, 1), basis, (6, 2), basis, (7, 3), dense, (4, 5, 6, 7), (0, 1, 2, 3), optimize=True)
assert np.linalg.norm(p - ref) < 1e-12
print('dropin ok')
"""
    assert "dropin ok" in _run(code)


@needs_dropin
@pytest.mark.gpu
def test_dropin_loads_the_cli_result_file():
    # load_sparse_eri_gausslet_integrals of the reference module (its HDF5
    # calls resolved by include/hdf5.h and include/hdf5_util.h of this
    # library; the loader also builds the O_h grid permutations, a GPU kernel)
    code = f"""
import numpy as np, gausslectronitegrate_pymodule as gli
eri = gli.load_sparse_eri_gausslet_integrals({os.path.join(GOLDEN, 'hdf5', 'eri_3x3x3.hdf5')!r})
c = np.load({os.path.join(GOLDEN, 'reference_core.npz')!r})
assert eri.num_entries == 1027 and eri.tol == 1e-16
assert eri.grid == ((-1, 3), (-1, 3), (-1, 3)) or list(map(tuple, eri.grid)) == [(-1, 3)] * 3
ref = c['eri_val_3_1e-16']
idx = c['eri_idx_3']
def lin(p):
    return ((p[0] + 1) * 3 + (p[1] + 1)) * 3 + (p[2] + 1)
v = eri.integral_value(([0, 0, 0], [0, 0, 0], [0, 0, 0], [0, 0, 0]))
k = int(np.searchsorted(idx, lin([0, 0, 0]) * (27 ** 3 + 27 ** 2 + 27 + 1)))
assert abs(v - ref[k]) <= 1e-15 * abs(ref[k])
print('load ok')
"""
    assert "load ok" in _run(code)
