"""CPU tests of the oracle (oracle/gli_oracle.c): pinned against the reference's
golden fixtures, the notebook known answers and the compiled reference core.
These run without a GPU."""
import itertools
import os

import numpy as np
import pytest

from _common import core, fixtures, g10, notebook, sym_grid
from oracle_binding import Oracle, project_factored
import ref_binding

ORACLE = Oracle()


def _have_ref():
    return os.path.exists(ref_binding.REF_LIB_PATH)


# --- golden fixtures of the reference test suite (test/data/*.hdf5) -----------

def test_fixture_kinetic():
    # test/test_kinetic_integrals.c:32-53 (grid (0,2)(1,3)(-1,3), 1e-13)
    fx = fixtures()
    k = ORACLE.kinetic_matrix(g10(), [(0, 2), (1, 3), (-1, 3)])
    assert np.max(np.abs(k - fx["fixture_kinetic"])) <= 1e-13


def test_fixture_nuclear():
    # test/test_nuclear_integrals.c:32-76 (grid (0,2)(2,2)(-1,3), two nuclei, 1e-13)
    fx = fixtures()
    v = ORACLE.nuclear_matrix(g10(), [(0, 2), (2, 2), (-1, 3)], fx["fixture_nuclear_pos"],
                              fx["fixture_nuclear_charge"], float(fx["fixture_nuclear_tol"]))
    assert np.max(np.abs(v - fx["fixture_nuclear"])) <= 1e-13


def test_fixture_eri():
    # test/test_eri_integrals.c:45-85: sparse 3^3 then dense (-1,2)(0,2)(-1,3), 1e-13
    fx = fixtures()
    tol = float(fx["fixture_eri_tol"])
    g = sym_grid(3)
    idx = ORACLE.enumerate("eri", g)
    val = ORACLE.values("eri", g10(), g, idx, tol)
    dense = ORACLE.fill_dense("eri", g, idx, val, [(-1, 2), (0, 2), (-1, 3)])
    assert np.max(np.abs(dense - fx["fixture_eri"])) <= 1e-13


def test_fixture_erida():
    # test/test_erida_integrals.c:42-99: sparse 3^3 then dense (0,2)(-1,3)(-1,2), 1e-12
    fx = fixtures()
    tol = float(fx["fixture_erida_tol"])
    g = sym_grid(3)
    idx = ORACLE.enumerate("erida", g)
    val = ORACLE.values("erida", g10(), g, idx, tol)
    dense = ORACLE.fill_dense("erida", g, idx, val, [(0, 2), (-1, 3), (-1, 2)])
    assert np.max(np.abs(dense - fx["fixture_erida"])) <= 1e-12


def test_fixture_single_entries_match_dense():
    # test/test_erida_integrals.c:83-97 and test/test_eri_integrals.c:88-112 (1e-13)
    fx = fixtures()
    tol = float(fx["fixture_erida_tol"])
    dense = fx["fixture_erida"]
    pts = list(itertools.product(range(0, 2), range(-1, 2), range(-1, 1)))
    for a in range(len(pts)):
        for b in (0, 5, 11):
            v = ORACLE.single("erida", g10(), [pts[a], pts[b]], tol)
            assert abs(v - dense[a, b]) <= 1e-12


# --- notebook known answers (examples/*.ipynb outputs) -------------------------

def test_notebook_known_answers():
    nb = notebook()
    b = g10()
    eri_out, erida_out = nb["eri_integrals"], nb["erida_integrals"]
    kin_out, nuc_out = nb["kinetic_integrals"], nb["nuclear_integrals"]
    # examples/eri_integrals.ipynb cells 4-5
    assert ORACLE.single("eri", b, [[0, 0, 0]] * 4, 1e-16) == float(eri_out[0])
    assert ORACLE.single("eri", b, [[1, 0, 0], [0, 0, -1], [0, 0, 1], [0, 0, 0]], 1e-16) == float(eri_out[1])
    # cells 8-11: 1027 classes on 3^3, sparse value at the four points
    g = sym_grid(3)
    idx = ORACLE.enumerate("eri", g)
    assert idx.size == int(eri_out[4])
    val = ORACLE.values("eri", b, g, idx, 1e-16)
    key = ORACLE.canonical("eri", g, [[1, 0, 0], [0, 0, -1], [0, 0, 1], [0, 0, 0]])
    assert val[np.searchsorted(idx, key)] == float(eri_out[6])
    # examples/erida_integrals.ipynb cells 4, 5, 9, 11
    assert ORACLE.single("erida", b, [[0, 0, 0]] * 2, 1e-16) == float(erida_out[0])
    assert ORACLE.single("erida", b, [[-1, 0, 2], [0, 1, -1]], 1e-16) == float(erida_out[1])
    g7 = sym_grid(7)
    idx7 = ORACLE.enumerate("erida", g7)
    assert idx7.size == int(erida_out[4])
    v7 = ORACLE.values("erida", b, g7, idx7, 1e-16)
    key = ORACLE.canonical("erida", g7, [[-1, 0, 2], [0, 1, -1]])
    assert v7[np.searchsorted(idx7, key)] == float(erida_out[6])
    # examples/kinetic_integrals.ipynb cells 8-10
    assert ORACLE.kinetic_single(b, [[0, 0, 0], [0, 0, 0]]) == float(kin_out[3])
    assert ORACLE.kinetic_single(b, [[0, -2, -1], [0, -2, 1]]) == float(kin_out[5])
    # examples/nuclear_integrals.ipynb cells 12-13
    pos, ch = [(-0.2, 1.3, 0.5), (0.7, 0, -2.1)], [2, 1]
    assert ORACLE.nuclear_single(b, [[0, 0, 0], [0, 0, 0]], pos, ch, 1e-16) == float(nuc_out[4])
    assert ORACLE.nuclear_single(b, [[-1, 0, -2], [0, 1, 1]], pos, ch, 1e-16) == float(nuc_out[6])


def test_notebook_projection_residual():
    # examples/eri_integrals.ipynb cells 17-19: project vs dense einsum, ~1e-13
    b = g10()
    g = sym_grid(3)
    idx = ORACLE.enumerate("eri", g)
    val = ORACLE.values("eri", b, g, idx, 1e-16)
    dense = ORACLE.fill_dense("eri", g, idx, val, g)
    basis = np.linalg.qr(np.random.default_rng(293).normal(size=(27, 27)))[0][:, :5]
    ref = np.einsum(basis, (4, 0), basis, (5, 1), basis, (6, 2), basis, (7, 3), dense, (4, 5, 6, 7), (0, 1, 2, 3),
                    optimize=True)
    assert np.linalg.norm(project_factored(dense, basis) - ref) < 1e-12


# --- against the compiled reference core (bit-exact restatement) ---------------

def test_core_enumeration_bit_exact():
    c = core()
    for L in (3, 5, 33):
        assert np.array_equal(ORACLE.enumerate("erida", sym_grid(L)), c[f"erida_idx_{L}"])
    assert np.array_equal(ORACLE.enumerate("eri", sym_grid(3)), c["eri_idx_3"])


@pytest.mark.slow
def test_core_eri_enumeration_5_bit_exact():
    assert np.array_equal(ORACLE.enumerate("eri", sym_grid(5)), core()["eri_idx_5"])


def test_core_values_bit_exact():
    c = core()
    b = g10()
    for tol in (1e-16, 1e-10, 1e-5):
        assert np.array_equal(ORACLE.values("erida", b, sym_grid(5), c["erida_idx_5"], tol), c[f"erida_val_5_{tol:g}"])
    for tol in (1e-16, 1e-5, 1e-3):
        assert np.array_equal(ORACLE.values("eri", b, sym_grid(3), c["eri_idx_3"], tol), c[f"eri_val_3_{tol:g}"])
    assert np.array_equal(ORACLE.kinetic_matrix(b, [(-3, 6), (0, 5), (2, 4)]), c["kinetic_6x5x4"])
    assert np.array_equal(ORACLE.nuclear_matrix(b, sym_grid(3), [[0.0, 0.0, 0.0]], [1], 1e-5), c["nuclear_3_z1_1e-5"])


@pytest.mark.skipif(not _have_ref(), reason="reference core not built (make -C oracle ref)")
def test_against_reference_core_live():
    r = ref_binding.RefLib()
    b = g10()
    g = sym_grid(5)
    idx = r.enumerate("erida", g)
    assert np.array_equal(idx, ORACLE.enumerate("erida", g))
    assert np.array_equal(r.sparse_values("erida", b, g, idx, 1e-10), ORACLE.values("erida", b, g, idx, 1e-10))
    pts = [[1, -1, 0], [0, 2, -1], [1, 0, 0], [-1, 0, 1]]
    assert r.eri_single(b, pts, 1e-8) == ORACLE.single("eri", b, pts, 1e-8)


# --- O_h group (test/test_symmetry.c) --------------------------------------------

def _oh_matrices():
    mats = []
    for perm in itertools.permutations(range(3)):
        for signs in itertools.product((1, -1), repeat=3):
            m = np.zeros((3, 3), dtype=np.int64)
            for a in range(3):
                m[a, perm[a]] = signs[a]
            mats.append(m)
    return mats


def test_oh_closure():
    # test/test_symmetry.c:6-34: products of group elements stay in the group
    mats = _oh_matrices()
    keys = {m.tobytes() for m in mats}
    assert len(keys) == 48
    for a in mats:
        for b in mats:
            assert (a @ b).tobytes() in keys


def test_canonical_is_orbit_invariant():
    # every image of a tuple under O_h and the index swaps has the same class
    g = sym_grid(5)
    rng = np.random.default_rng(0)
    for _ in range(20):
        p = rng.integers(-2, 3, size=(4, 3))
        base = ORACLE.canonical("eri", g, p)
        for m in _oh_matrices()[::7]:
            q = p @ m.T
            assert ORACLE.canonical("eri", g, q) == base
            assert ORACLE.canonical("eri", g, q[[1, 0, 3, 2]]) == base
            assert ORACLE.canonical("eri", g, q[[2, 3, 0, 1]]) == base
