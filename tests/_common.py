"""Shared fixtures for the test suite: golden data loaders and the parity
tolerance.

Parity bar (FP64 form against the reference C core): every value x of the CUDA
path satisfies |x - ref| <= 1e-12 |ref| + 1e-14.  The reference's own tests
use 1e-13 absolute (test/test_eri_integrals.c:79) and 1e-12 for projections;
the relative term is the 1e-12 bound for the FP64 form, the absolute floor
covers near-zero entries whose summation order differs.
Integer outputs (class lists) are compared bit-exactly.
"""
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")

RTOL = 1e-12
ATOL = 1e-14


def fixtures():
    return np.load(os.path.join(GOLDEN, "reference_fixtures.npz"))


def core():
    return np.load(os.path.join(GOLDEN, "reference_core.npz"))


def notebook():
    with open(os.path.join(GOLDEN, "notebook_outputs.json")) as f:
        return json.load(f)["notebook_outputs"]


def g10():
    return fixtures()["g10"]


def sym_grid(L):
    return [(-(L // 2), L)] * 3


def assert_parity(x, ref, rtol=RTOL, atol=ATOL, what="values"):
    x = np.asarray(x, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    assert x.shape == ref.shape, f"{what}: shape {x.shape} vs {ref.shape}"
    err = np.abs(x - ref)
    bound = rtol * np.abs(ref) + atol
    bad = err > bound
    if np.any(bad):
        k = int(np.argmax(err - bound))
        raise AssertionError(f"{what}: {int(bad.sum())} of {x.size} entries out of tolerance; worst at {k}: "
                             f"{x.ravel()[k]!r} vs {ref.ravel()[k]!r} (|d| = {err.ravel()[k]:.3e})")
