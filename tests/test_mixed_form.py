"""The mixed form of the sparse ERI/ERIDA evaluation (form="mixed").

It screens the Gaussian-pair products within a first-order error bound
(gli_b200_last_screening), and the two bulk lattice stages run as int8-sliced
products on the tcgen05 tensor cores where they are large enough; tables and
the last stage stay FP64.  Its bar is an absolute error of at
most 1e-8 Ha on every class value.  Values are in grid units (spacing 1); an
integral on a grid of spacing h is the grid-unit value / h, so the strictest
workload in use (spacing 0.5 bohr) needs a grid-unit error below 5e-9, the
bound written here.  References: the compiled reference core's values
(golden fixtures) where they exist, else the FP64 form, which the parity tests
pin to the reference at 1e-12 relative.
"""
import ctypes as C

import numpy as np
import pytest

from _common import core, g10, sym_grid
from oracle_binding import Oracle

pytestmark = pytest.mark.gpu

MIXED_ABS_TOL = 5e-9  # grid units: 1e-8 Ha at spacing 0.5 bohr


@pytest.fixture(scope="module")
def gli():
    import gausslectronitegrate_b200 as m
    if m.lib().gli_b200_device_count() == 0:
        pytest.fail("no CUDA device: the gpu tests need a B200")
    return m


def _check(x, ref, what):
    x = np.asarray(x)
    ref = np.asarray(ref)
    assert x.shape == ref.shape
    assert np.all(np.isfinite(x)), what
    err = np.abs(x - ref)
    k = int(np.argmax(err))
    assert err[k] <= MIXED_ABS_TOL, f"{what}: max abs err {err[k]:.3e} at {k} ({x[k]!r} vs {ref[k]!r})"
    return float(err.max())


@pytest.mark.parametrize("tol", [1e-16, 1e-10, 1e-5])
def test_mixed_erida_33_against_reference(gli, tol):
    c = core()
    s = gli.compute_sparse_erida_gausslet_integrals(g10(), sym_grid(33), tol, form="mixed")
    assert np.array_equal(s.indices, c["erida_idx_33"])
    _check(s.values, c[f"erida_val_33_{tol:g}"], f"mixed ERIDA 33^3 tol {tol:g}")


@pytest.mark.parametrize("L,tol", [(3, 1e-16), (3, 1e-5), (5, 1e-5)])
def test_mixed_eri_against_reference(gli, L, tol):
    c = core()
    s = gli.compute_sparse_eri_gausslet_integrals(g10(), sym_grid(L), tol, form="mixed")
    _check(s.values, c[f"eri_val_{L}_{tol:g}"], f"mixed ERI {L}^3 tol {tol:g}")


def test_mixed_eri_5_tight_against_fp64_form(gli):
    # tol 1e-16 on 5^3: 138,187 classes, enough for the product form of the
    # last stage on the tensor cores, with key-count bounds above the counts
    fp = gli.compute_sparse_eri_gausslet_integrals(g10(), sym_grid(5), 1e-16)
    mx = gli.compute_sparse_eri_gausslet_integrals(g10(), sym_grid(5), 1e-16, form="mixed")
    _check(mx.values, fp.values, "mixed ERI 5^3 tol 1e-16")


def test_mixed_eri_7_against_fp64_form(gli):
    fp = gli.compute_sparse_eri_gausslet_integrals(g10(), sym_grid(7), 1e-10)
    mx = gli.compute_sparse_eri_gausslet_integrals(g10(), sym_grid(7), 1e-10, form="mixed")
    assert np.array_equal(fp.indices, mx.indices)
    _check(mx.values, fp.values, "mixed ERI 7^3 tol 1e-10")


def test_mixed_erida_129_against_fp64_form(gli):
    fp = gli.compute_sparse_erida_gausslet_integrals(g10(), sym_grid(129), 1e-10)
    mx = gli.compute_sparse_erida_gausslet_integrals(g10(), sym_grid(129), 1e-10, form="mixed")
    _check(mx.values, fp.values, "mixed ERIDA 129^3 tol 1e-10")


@pytest.mark.parametrize("kind,L", [("eri", 7), ("erida", 33)])
def test_mixed_screening_within_its_bound(gli, kind, L):
    # at tol 1e-16 the mixed form masks the products at a higher threshold;
    # without a tensor-core stage (neither of these sizes has one) the
    # screening is its only departure from the FP64 form, and every class
    # value stays within the stated bound
    fn = gli.compute_sparse_eri_gausslet_integrals if kind == "eri" else gli.compute_sparse_erida_gausslet_integrals
    fp = fn(g10(), sym_grid(L), 1e-16)
    mx = fn(g10(), sym_grid(L), 1e-16, form="mixed")
    scr = (C.c_double * 2)()
    gli.lib().gli_b200_last_screening(scr)
    paths = (C.c_int * 3)()
    gli.lib().gli_b200_last_paths(paths)
    tau, bound = scr[0], scr[1]
    assert 1e-16 < tau and 0 < bound <= 1e-9
    assert paths[0] == 0 and paths[1] == 0
    err = float(np.max(np.abs(mx.values - fp.values)))
    assert err <= bound, f"{kind} {L}^3: screening error {err:.3e} above its bound {bound:.3e} (tau {tau:.1e})"
    # the FP64 form masks at the caller's tol
    fn(g10(), sym_grid(L), 1e-16)
    gli.lib().gli_b200_last_screening(scr)
    assert scr[0] == 1e-16 and scr[1] == 0


def test_mixed_arbitrary_eri_list(gli):
    # non-canonical, unsorted, repeated indices on a non-cubic grid, against the oracle
    from gausslectronitegrate_b200 import _abi
    g = [(-1, 3), (0, 2), (-2, 4)]
    N = 24
    idx = np.random.default_rng(11).integers(0, N ** 4, size=400).astype(np.int64)
    idx[7] = idx[2]
    ref = Oracle().values("eri", g10(), g, idx, 1e-10)
    gd, keep = gli._parse_coeffs(g10(), "")
    vals = np.empty(idx.size)
    rc = gli.lib().gli_b200_sparse_values(_abi.GLI_KIND_ERI, C.byref(gd), C.byref(gli._grid_struct(g)),
                                          idx.ctypes.data_as(_abi.lptr), idx.size, 1e-10, _abi.GLI_FORM_MIXED,
                                          vals.ctypes.data_as(_abi.dptr))
    assert rc == 0
    _check(vals, ref, "mixed ERI arbitrary list")


def test_unknown_form_rejected(gli):
    with pytest.raises(ValueError):
        gli.compute_sparse_erida_gausslet_integrals(g10(), sym_grid(3), 1e-10, form="fp16")
