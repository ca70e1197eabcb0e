"""Batched nuclear-attraction matrices (gli_b200_nuclear_batch / _dev).

A batch of linear H_n chains, each on its own grid, runs as one plan (one CUDA
graph per chunk of instances).  Checks: every instance of an FP64 batch equals
the single-matrix entry point (itself pinned to the reference) within the
parity tolerance; small instances against the oracle; the mixed form (tensor-
core contractions) within 5e-9 grid units of the FP64 form (1e-8 Ha at
spacing 0.5 bohr); the autotuner's recorded choice; argument errors.
"""
import json

import numpy as np
import pytest

from _common import assert_parity, g10
from gausslectronitegrate_b200.workloads import h_chain_batch
from oracle_binding import Oracle

pytestmark = pytest.mark.gpu

TOL = 1e-8


@pytest.fixture(scope="module")
def gli():
    import gausslectronitegrate_b200 as m
    if m.lib().gli_b200_device_count() == 0:
        pytest.fail("no CUDA device: the gpu tests need a B200")
    return m


def test_batch_matches_single_matrix_entry_point(gli):
    grids, pos, q = h_chain_batch(np.random.default_rng(7), 10, 2, 7, 0.5)
    grids[3] = [(-1, 3), (0, 2), (-2, 5)]  # a non-cubic, off-centre box
    outs = gli.compute_nuclear_gausslet_integrals_batch(g10(), grids, pos, q, TOL)
    for k in range(len(grids)):
        ref = gli.compute_nuclear_gausslet_integrals(g10(), grids[k], pos[k], q[k], TOL)
        assert_parity(outs[k], ref, what=f"batch instance {k} ({grids[k]})")
    st = (gli._abi.glong * 3)()
    gli.lib().gli_b200_last_nuclear_batch(st)
    assert st[0] == 0 or st[0] == 1  # the last call was the single-matrix entry point


def test_batch_small_instances_against_oracle(gli):
    grids = [[(-1, 2), (0, 2), (-1, 2)], [(-1, 3), (-1, 2), (0, 2)]]
    pos = [np.array([[0.3, -0.2, 0.1], [1.4, 0.1, -0.3]]), np.array([[-0.5, 0.25, 0.0]])]
    q = [[1, 2], [3]]
    outs = gli.compute_nuclear_gausslet_integrals_batch(g10(), grids, pos, q, 1e-5)
    ora = Oracle()
    for k in range(2):
        ref = ora.nuclear_matrix(g10(), grids[k], pos[k], q[k], 1e-5)
        assert_parity(outs[k], ref, what=f"batch instance {k} vs oracle")


@pytest.mark.parametrize("choice", ["17", "1", None])
def test_batch_mixed_against_fp64(gli, choice, monkeypatch):
    # the mixed form's contraction path is the autotuner's choice; "17" forces
    # the int8-sliced tensor-core contractions (one stream), "1" the FP64 ones,
    # None leaves the choice to the measurement
    if choice is not None:
        monkeypatch.setenv("GLI_B200_TUNE_NUCLEAR", choice)
    grids, pos, q = h_chain_batch(np.random.default_rng(11), 8, 4, 12, 0.5)
    fp = gli.compute_nuclear_gausslet_integrals_batch(g10(), grids, pos, q, TOL)
    mx = gli.compute_nuclear_gausslet_integrals_batch(g10(), grids, pos, q, TOL, form="mixed")
    worst = 0.0
    for k in range(len(grids)):
        err = np.max(np.abs(mx[k] - fp[k]))
        assert np.all(np.isfinite(mx[k]))
        assert err <= 5e-9, f"instance {k}: max abs err {err:.3e}"
        worst = max(worst, err)
    if choice == "17":
        assert worst > 0  # the sliced products did run
    if choice == "1":
        assert worst == 0  # the FP64 contractions, as in the FP64 form


def test_batch_autotuner_decision(gli):
    grids, pos, q = h_chain_batch(np.random.default_rng(3), 6, 3, 8, 0.5)
    gli.compute_nuclear_gausslet_integrals_batch(g10(), grids, pos, q, TOL)
    st = (gli._abi.glong * 3)()
    gli.lib().gli_b200_last_nuclear_batch(st)
    assert st[0] == 6 and st[1] >= 1 and st[2] in (1, 2, 4, 8)
    n = gli.lib().gli_b200_autotune_report(None, 0)
    import ctypes as C
    buf = C.create_string_buffer(int(n) + 1)
    gli.lib().gli_b200_autotune_report(buf, n + 1)
    rep = json.loads(buf.value.decode())
    keys = [k for k in rep if k.startswith("nuclear form=0") and "inst=6 " in k]
    assert keys, rep
    d = rep[keys[0]]
    assert d["best"] == st[2] and len(d["ms"]) == 4
    assert d["ms"][str(d["best"])] == min(d["ms"].values())


def test_batch_argument_errors(gli):
    with pytest.raises(ValueError):
        gli.compute_nuclear_gausslet_integrals_batch(g10(), [[(-1, 3)] * 3], [], [], TOL)
    with pytest.raises(ValueError):
        gli.compute_nuclear_gausslet_integrals_batch(g10(), [[(-1, 3)] * 3], [[[0, 0, 0]]], [[1]], TOL, form="f16")
