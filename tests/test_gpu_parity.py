"""GPU parity tests: the CUDA path, called through libgli_b200's C ABI (via the
Python mirror of the reference module), against the oracle, the reference's
golden fixtures and the compiled reference core's values.

Tolerance (FP64 form): |x - ref| <= 1e-12 |ref| + 1e-14 (tests/_common.py);
class lists bit-exact."""
import itertools

import numpy as np
import pytest

from _common import assert_parity, core, fixtures, g10, notebook, sym_grid
from oracle_binding import Oracle, project_factored

pytestmark = pytest.mark.gpu

ORACLE = Oracle()


@pytest.fixture(scope="module")
def gli():
    import gausslectronitegrate_b200 as m
    if m.lib().gli_b200_device_count() == 0:
        pytest.fail("no CUDA device: the gpu tests need a B200")
    return m


# --- enumeration: bit-exact ------------------------------------------------------

@pytest.mark.parametrize("L", [1, 3, 5, 7, 9, 17, 33])
def test_enumerate_erida_bit_exact(gli, L):
    s = gli.compute_sparse_erida_gausslet_integrals(g10(), sym_grid(L), 1e-5)
    ref = core()[f"erida_idx_{L}"] if L in (3, 5, 33) else ORACLE.enumerate("erida", sym_grid(L))
    assert np.array_equal(s.indices, ref)
    assert s.num_entries == L * (L + 1) * (L + 2) // 6


@pytest.mark.parametrize("mode", [None, "1", "live"])
@pytest.mark.parametrize("L", [1, 3, 5])
def test_enumerate_eri_bit_exact(gli, L, mode, monkeypatch):
    # the one-pass enumeration over the live slots, the thread-per-slot two
    # passes ("1") and the count and write passes over the live slots ("live")
    if mode:
        monkeypatch.setenv("GLI_B200_ENUM_TWO_PASS", mode)
    ref = core()[f"eri_idx_{L}"] if L in (3, 5) else ORACLE.enumerate("eri", sym_grid(L))
    s = gli.compute_sparse_eri_gausslet_integrals(g10(), sym_grid(L), 1e-3)
    assert np.array_equal(s.indices, ref)


@pytest.mark.parametrize("kind,L", [("eri", 7), ("erida", 129)])
def test_enumerate_one_pass_matches_two_pass(gli, kind, L, monkeypatch):
    import ctypes as C
    from gausslectronitegrate_b200 import _abi

    def run():
        gs = gli._grid_struct(sym_grid(L))
        out = _abi.SparseIndices()
        getattr(gli.lib(), f"enumerate_symmetry_reduced_{kind}_indices")(C.byref(gs), C.byref(out))
        idx = np.ctypeslib.as_array(out.indices, shape=(out.num,)).copy()
        getattr(gli.lib(), f"delete_sparse_{kind}_indices")(C.byref(out))
        return idx

    one = run()
    for mode in ("1", "live"):
        monkeypatch.setenv("GLI_B200_ENUM_TWO_PASS", mode)
        two = run()
        assert one.size == two.size and np.array_equal(one, two), mode


def test_enumerate_eri_7_properties(gli):
    # 3,571,977 classes on 7^3; sorted, unique, every entry canonical (sampled)
    import ctypes as C
    from gausslectronitegrate_b200 import _abi
    L = gli.lib()
    g = sym_grid(7)
    gs = _abi.Grid()
    for a in range(3):
        gs.coord_range[a].istart, gs.coord_range[a].num = g[a]
    out = _abi.SparseIndices()
    L.enumerate_symmetry_reduced_eri_indices(C.byref(gs), C.byref(out))
    idx = np.ctypeslib.as_array(out.indices, shape=(out.num,)).copy()
    L.delete_sparse_eri_indices(C.byref(out))
    assert idx.size == 3571977
    assert np.all(np.diff(idx) > 0)
    N = 343
    rng = np.random.default_rng(7)
    for k in rng.integers(0, idx.size, size=300):
        v = int(idx[k])
        pts = [(v // N ** 3) % N, (v // N ** 2) % N, (v // N) % N, v % N]
        p = [[q // 49 - 3, (q // 7) % 7 - 3, q % 7 - 3] for q in pts]
        assert ORACLE.canonical("eri", g, p) == v


# --- sparse values ---------------------------------------------------------------

@pytest.mark.parametrize("tol", [1e-16, 1e-10, 1e-5])
def test_erida_values_33(gli, tol):
    c = core()
    s = gli.compute_sparse_erida_gausslet_integrals(g10(), sym_grid(33), tol)
    assert np.array_equal(s.indices, c["erida_idx_33"])
    assert_parity(s.values, c[f"erida_val_33_{tol:g}"], what=f"ERIDA 33^3 tol {tol:g}")


@pytest.mark.parametrize("tol", [1e-16, 1e-10, 1e-5, 1e-3])
def test_eri_values_3(gli, tol):
    c = core()
    s = gli.compute_sparse_eri_gausslet_integrals(g10(), sym_grid(3), tol)
    assert_parity(s.values, c[f"eri_val_3_{tol:g}"], what=f"ERI 3^3 tol {tol:g}")


def test_eri_values_5(gli):
    c = core()
    s = gli.compute_sparse_eri_gausslet_integrals(g10(), sym_grid(5), 1e-5)
    assert_parity(s.values, c["eri_val_5_1e-05"], what="ERI 5^3 tol 1e-5")


def test_eri_values_arbitrary_list(gli):
    # non-canonical, unsorted, repeated indices on a non-cubic grid
    import ctypes as C
    from gausslectronitegrate_b200 import _abi
    g = [(-1, 3), (0, 2), (-2, 4)]
    N = 24
    idx = np.random.default_rng(3).integers(0, N ** 4, size=500).astype(np.int64)
    idx[10] = idx[3]
    ref = ORACLE.values("eri", g10(), g, idx, 1e-10)
    gd, keep = gli._parse_coeffs(g10(), "")
    vals = np.empty(idx.size)
    lib = gli.lib()
    rc = lib.gli_b200_sparse_values(_abi.GLI_KIND_ERI, C.byref(gd), C.byref(gli._grid_struct(g)),
                                    idx.ctypes.data_as(_abi.lptr), idx.size, 1e-10, 0, vals.ctypes.data_as(_abi.dptr))
    assert rc == 0
    assert_parity(vals, ref, what="ERI arbitrary list")


@pytest.mark.parametrize("form", [0, 1])
def test_eri_values_large_key_space(gli, form):
    # 9^3 grid: 765 axis keys, so the plan takes exact sizes (host-read counts)
    # and the class decode marks its key pairs in global memory; a seeded sample
    # of indices (any order) in both forms against the oracle
    import ctypes as C
    from gausslectronitegrate_b200 import _abi
    g = sym_grid(9)
    N = 9 ** 3
    rng = np.random.default_rng(11)
    # half random indices, half with the four points within two spacings of
    # one another (the large values)
    far = rng.integers(0, N ** 4, size=150)
    base = rng.integers(0, 9, size=(150, 1, 3))
    pts = np.clip(base + rng.integers(-2, 3, size=(150, 4, 3)), 0, 8)
    lin = (pts[..., 0] * 9 + pts[..., 1]) * 9 + pts[..., 2]
    lin[::2, 1] = lin[::2, 0]  # density-density classes (i i | k k)
    lin[::2, 3] = lin[::2, 2]
    near = ((lin[:, 0] * N + lin[:, 1]) * N + lin[:, 2]) * N + lin[:, 3]
    idx = np.concatenate([far, near]).astype(np.int64)
    ref = ORACLE.values("eri", g10(), g, idx, 1e-5)
    assert np.max(np.abs(ref)) > 0.1
    gd, keep = gli._parse_coeffs(g10(), "")
    vals = np.empty(idx.size)
    rc = gli.lib().gli_b200_sparse_values(_abi.GLI_KIND_ERI, C.byref(gd), C.byref(gli._grid_struct(g)),
                                          idx.ctypes.data_as(_abi.lptr), idx.size, 1e-5, form,
                                          vals.ctypes.data_as(_abi.dptr))
    assert rc == 0, gli.lib().gli_b200_last_error_message()
    if form == 0:
        assert_parity(vals, ref, what="ERI 9^3 sample")
    else:
        assert np.max(np.abs(vals - ref)) <= 1e-8


def test_eri_values_sample_7(gli):
    # ERI on 7^3: every one of the 3,571,977 classes evaluated (364 axis keys:
    # the plan reads its counts back), a seeded sample against the oracle
    s = gli.compute_sparse_eri_gausslet_integrals(g10(), sym_grid(7), 1e-10)
    idx, val = s.indices, s.values
    assert idx.size == 3571977
    pick = np.random.default_rng(5).choice(idx.size, size=300, replace=False)
    ref = ORACLE.values("eri", g10(), sym_grid(7), idx[pick], 1e-10)
    assert_parity(val[pick], ref, what="ERI 7^3 sample")


def test_erida_values_sample_129(gli):
    # ERIDA on 129^3: enumeration count, sortedness and a seeded sample of
    # classes against the oracle (the full CPU reference takes minutes)
    s = gli.compute_sparse_erida_gausslet_integrals(g10(), sym_grid(129), 1e-10)
    idx, val = s.indices, s.values
    assert idx.size == 129 * 130 * 131 // 6
    assert np.all(np.diff(idx) > 0)
    pick = np.random.default_rng(0).choice(idx.size, size=200, replace=False)
    ref = ORACLE.values("erida", g10(), sym_grid(129), idx[pick], 1e-10)
    assert_parity(val[pick], ref, what="ERIDA 129^3 sample")


@pytest.mark.parametrize("L", [65, 101, 131])
def test_erida_values_balanced_hosts(gli, L):
    # full pair triangles of more than 64 A keys: stage B hosts each pair on
    # either of its keys (65 and 101 keys: one regular tournament; 131 keys:
    # 127 in a tournament, 4 hosting the rest); a seeded sample of classes
    s = gli.compute_sparse_erida_gausslet_integrals(g10(), sym_grid(L), 1e-10)
    idx, val = s.indices, s.values
    assert idx.size == L * (L + 1) * (L + 2) // 6
    pick = np.random.default_rng(L).choice(idx.size, size=150, replace=False)
    ref = ORACLE.values("erida", g10(), sym_grid(L), idx[pick], 1e-10)
    assert_parity(val[pick], ref, what=f"ERIDA {L}^3 sample")


@pytest.mark.parametrize("form", [0, 1])
def test_erida_values_partial_triangle(gli, form):
    # a class list whose pairs do not fill the triangle (no class whose two
    # smallest displacement components are equal, so no pair (a, a)): stage B
    # keeps each pair on its A key
    import ctypes as C
    from gausslectronitegrate_b200 import _abi
    g = sym_grid(129)
    N = 129 ** 3
    full = gli.compute_sparse_erida_gausslet_integrals(g10(), g, 1e-10).indices
    a, b = full // N, full % N
    d = np.abs(np.stack([a // (129 * 129) - b // (129 * 129), (a // 129) % 129 - (b // 129) % 129,
                         a % 129 - b % 129], 1))
    ds = np.sort(d, axis=1)
    idx = np.ascontiguousarray(full[ds[:, 0] != ds[:, 1]])
    assert 0 < idx.size < full.size
    vals = np.empty(idx.size)
    gd, keep = gli._parse_coeffs(g10(), "")
    rc = gli.lib().gli_b200_sparse_values(_abi.GLI_KIND_ERIDA, C.byref(gd), C.byref(gli._grid_struct(g)),
                                          idx.ctypes.data_as(_abi.lptr), idx.size, 1e-10, form,
                                          vals.ctypes.data_as(_abi.dptr))
    assert rc == 0, gli.lib().gli_b200_last_error_message()
    pick = np.random.default_rng(3).choice(idx.size, size=150, replace=False)
    ref = ORACLE.values("erida", g10(), g, idx[pick], 1e-10)
    if form == 0:
        assert_parity(vals[pick], ref, what="ERIDA 129^3 partial triangle")
    else:
        assert np.max(np.abs(vals[pick] - ref)) <= 1e-8


# --- golden fixtures of the reference test suite --------------------------------

def test_fixture_eri_dense(gli):
    fx = fixtures()
    s = gli.compute_sparse_eri_gausslet_integrals(g10(), sym_grid(3), float(fx["fixture_eri_tol"]))
    dense = s.fill_tensor([(-1, 2), (0, 2), (-1, 3)])
    assert np.max(np.abs(dense - fx["fixture_eri"])) <= 1e-13


def test_fixture_erida_dense(gli):
    fx = fixtures()
    s = gli.compute_sparse_erida_gausslet_integrals(g10(), sym_grid(3), float(fx["fixture_erida_tol"]))
    dense = s.fill_matrix([(0, 2), (-1, 3), (-1, 2)])
    assert np.max(np.abs(dense - fx["fixture_erida"])) <= 1e-12


def test_fixture_kinetic(gli):
    fx = fixtures()
    k = gli.compute_kinetic_gausslet_integrals(g10(), [(0, 2), (1, 3), (-1, 3)])
    assert np.max(np.abs(k - fx["fixture_kinetic"])) <= 1e-13


def test_fixture_nuclear(gli):
    fx = fixtures()
    v = gli.compute_nuclear_gausslet_integrals(g10(), [(0, 2), (2, 2), (-1, 3)], fx["fixture_nuclear_pos"],
                                               list(fx["fixture_nuclear_charge"]), float(fx["fixture_nuclear_tol"]))
    assert np.max(np.abs(v - fx["fixture_nuclear"])) <= 1e-13


def test_fixture_single_entries(gli):
    # every dense fixture entry against the single-entry API (1e-13)
    fx = fixtures()
    tol = float(fx["fixture_eri_tol"])
    pts = list(itertools.product(range(-1, 1), range(0, 2), range(-1, 2)))
    dense = fx["fixture_eri"]
    rng = np.random.default_rng(1)
    for _ in range(25):
        a, b, c, d = rng.integers(0, len(pts), size=4)
        v = gli.compute_eri_gausslet_integral(g10(), [pts[a], pts[b], pts[c], pts[d]], tol)
        assert abs(v - dense[a, b, c, d]) <= 1e-13


# --- notebook known answers ------------------------------------------------------

def test_notebook_known_answers(gli):
    nb = notebook()
    b = g10()
    eri_out, erida_out = nb["eri_integrals"], nb["erida_integrals"]
    kin_out, nuc_out = nb["kinetic_integrals"], nb["nuclear_integrals"]
    close = lambda x, y: abs(x - float(y)) <= 1e-12 * abs(float(y)) + 1e-14
    assert close(gli.compute_eri_gausslet_integral(b, ([0, 0, 0],) * 4, 1e-16), eri_out[0])
    assert close(gli.compute_eri_gausslet_integral(b, ([1, 0, 0], [0, 0, -1], [0, 0, 1], [0, 0, 0]), 1e-16), eri_out[1])
    eri = gli.compute_sparse_eri_gausslet_integrals(b, sym_grid(3), 1e-16)
    assert eri.num_entries == int(eri_out[4])
    assert close(eri.integral_value(([0, 0, 0],) * 4), eri_out[5])
    assert close(eri.integral_value(([1, 0, 0], [0, 0, -1], [0, 0, 1], [0, 0, 0])), eri_out[6])
    assert close(gli.compute_erida_gausslet_integral(b, ([0, 0, 0], [0, 0, 0]), 1e-16), erida_out[0])
    assert close(gli.compute_erida_gausslet_integral(b, ([-1, 0, 2], [0, 1, -1]), 1e-16), erida_out[1])
    erida = gli.compute_sparse_erida_gausslet_integrals(b, sym_grid(7), 1e-16)
    assert erida.num_entries == int(erida_out[4])
    assert close(erida.integral_value(([-1, 0, 2], [0, 1, -1])), erida_out[6])
    m = erida.fill_matrix(sym_grid(7))
    assert np.linalg.norm(m - m.T) == 0.0
    grid = [(-1, 3), (-2, 5), (-2, 4)]
    kgi = gli.compute_kinetic_gausslet_integrals(b, grid)
    assert np.linalg.norm(kgi.T - kgi) == 0.0
    assert close(kgi[7, 7], kin_out[3])
    assert close(gli.compute_kinetic_gausslet_integral(b, ([0, -2, -1], [0, -2, 1])), kin_out[5])
    pos, ch = [(-0.2, 1.3, 0.5), (0.7, 0, -2.1)], [2, 1]
    ngrid = [(-1, 3), (0, 2), (-2, 4)]
    ngi = gli.compute_nuclear_gausslet_integrals(b, ngrid, pos, ch, 1e-16)
    assert np.linalg.norm(ngi.T - ngi) == 0.0
    io = gli.grid_point_to_linear_index(ngrid, [0, 0, 0])
    assert close(ngi[io, io], nuc_out[4])
    assert close(gli.compute_nuclear_gausslet_integral(b, ([-1, 0, -2], [0, 1, 1]), pos, ch, 1e-16), nuc_out[6])


# --- dense matrices against the reference core -------------------------------------

def test_kinetic_matrix(gli):
    c = core()
    assert_parity(gli.compute_kinetic_gausslet_integrals(g10(), [(-3, 6), (0, 5), (2, 4)]), c["kinetic_6x5x4"],
                  what="kinetic 6x5x4")


@pytest.mark.parametrize("case", ["z1", "h2"])
def test_nuclear_matrix(gli, case):
    c = core()
    if case == "z1":
        v = gli.compute_nuclear_gausslet_integrals(g10(), sym_grid(3), [[0.0, 0.0, 0.0]], [1], 1e-5)
        ref = c["nuclear_3_z1_1e-5"]
    else:
        v = gli.compute_nuclear_gausslet_integrals(g10(), [(-1, 2), (0, 3), (-1, 2)],
                                                   [[0.3, 0.1, -0.2], [-1.1, 0.6, 0.4]], [1, 2], 1e-3)
        ref = c["nuclear_2x3x2_h2_1e-3"]
    assert_parity(v, ref, what=f"nuclear {case}")


def test_nuclear_pairs_sampled(gli):
    # an 8^3 H4 chain at tol 1e-8 (the oracle on all pairs would take minutes):
    # a seeded sample of matrix entries against the oracle
    grid = [(-4, 8)] * 3
    pos = [[-2.1, 0.2, 0.1], [-0.6, -0.1, 0.0], [0.8, 0.1, -0.2], [2.3, 0.0, 0.1]]
    ch = [1, 1, 1, 1]
    v = gli.compute_nuclear_gausslet_integrals(g10(), grid, pos, ch, 1e-8)
    assert np.array_equal(v, v.T)
    pairs = np.random.default_rng(4).integers(0, 512, size=(60, 2))
    ref = ORACLE.nuclear_pairs(g10(), grid, pos, ch, 1e-8, pairs)
    assert_parity(v[pairs[:, 0], pairs[:, 1]], ref, what="nuclear 8^3 sample")


# --- projection / apply / completeness (test/test_eri_integrals.c:115-419) ---------

def test_project_eri(gli):
    s = gli.compute_sparse_eri_gausslet_integrals(g10(), sym_grid(3), 1e-5)
    i = np.arange(27 * 4)
    basis = (0.1 * np.sin(np.sqrt(3) * np.pi * ((557 * i) % 311) - 8) /
             (1.5 + np.cos(np.sqrt(5) * np.pi * ((541 * i) % 229)))).reshape(27, 4)
    dense = s.fill_tensor(sym_grid(3))
    assert np.max(np.abs(s.project(basis) - project_factored(dense, basis))) <= 1e-12


def test_project_eri_wide_basis_and_zero_rows(gli):
    # more than 32 columns (the slab filled, then contracted) and a basis with
    # zero rows (the contraction over the nonzero rows only); the first two
    # contractions run over the pairs j <= i of the (i j) symmetry
    s = gli.compute_sparse_eri_gausslet_integrals(g10(), sym_grid(3), 1e-10)
    dense = s.fill_tensor(sym_grid(3))
    rng = np.random.default_rng(21)
    basis = rng.normal(size=(27, 36))
    basis[[0, 5, 13, 26]] = 0.0
    got = s.project(basis)
    ref = project_factored(dense, basis)
    assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref)) * 27 ** 2
    assert np.max(np.abs(got - got.transpose(1, 0, 2, 3))) <= 1e-13 * np.max(np.abs(ref))


def test_eri_keyed_fill_equals_oracle_fill(gli):
    # a complete class list: dense entries come from the key-triple table; the
    # oracle canonicalises every entry and looks it up -- same class values in,
    # so the dense tensors must agree bit for bit
    s = gli.compute_sparse_eri_gausslet_integrals(g10(), sym_grid(5), 1e-5)
    dense_grid = [(-1, 3), (-2, 4), (0, 2)]
    got = s.fill_tensor(dense_grid)
    ref = ORACLE.fill_dense("eri", sym_grid(5), s.indices, s.values, dense_grid)
    assert np.array_equal(got, ref)


def test_eri_partial_list_fill_and_project(gli):
    # a partial list (every third class missing) keeps the canonical lookups:
    # missing classes read as zero, as in the reference
    full = gli.compute_sparse_eri_gausslet_integrals(g10(), sym_grid(3), 1e-5)
    keep = np.arange(full.indices.size) % 3 != 1
    part = gli.SparseERI._make(g10(), sym_grid(3), full.indices[keep], full.values[keep], 1e-5)
    got = part.fill_tensor(sym_grid(3))
    ref = ORACLE.fill_dense("eri", sym_grid(3), full.indices[keep], full.values[keep], sym_grid(3))
    assert np.array_equal(got, ref)
    basis = np.random.default_rng(9).normal(size=(27, 3))
    assert np.max(np.abs(part.project(basis) - project_factored(ref, basis))) <= 1e-12 * np.max(np.abs(ref)) * 27 ** 2


def test_project_erida(gli):
    s = gli.compute_sparse_erida_gausslet_integrals(g10(), sym_grid(5), 1e-5)
    basis = np.random.default_rng(5).normal(size=(125, 5))
    m = s.fill_matrix(sym_grid(5))
    ref = np.einsum(basis, (4, 0), basis, (4, 1), basis, (5, 2), basis, (5, 3), m, (4, 5), (0, 1, 2, 3), optimize=True)
    # the unnormalised basis makes entries O(1e4): the bound is relative to the largest entry
    assert np.max(np.abs(s.project(basis) - ref)) <= 1e-12 * np.max(np.abs(ref))


def test_apply_eri(gli):
    s = gli.compute_sparse_eri_gausslet_integrals(g10(), sym_grid(3), 1e-5)
    states = np.random.default_rng(401).normal(size=(27 * 27, 3))
    vint = s.fill_tensor(sym_grid(3)).transpose((0, 2, 1, 3)).reshape(27 * 27, 27 * 27)
    assert np.max(np.abs(s.apply(states) - vint @ states)) <= 1e-12


def test_completeness(gli):
    # no dense entry may be zero: ERI on 5^3, ERIDA on 7^3 (tol 1e-5)
    e = gli.compute_sparse_eri_gausslet_integrals(g10(), sym_grid(5), 1e-5)
    assert np.count_nonzero(e.fill_tensor(sym_grid(5)) == 0) == 0
    d = gli.compute_sparse_erida_gausslet_integrals(g10(), sym_grid(7), 1e-5)
    assert np.count_nonzero(d.fill_matrix(sym_grid(7)) == 0) == 0


# --- error paths -------------------------------------------------------------------

def test_errors(gli):
    b = g10()
    with pytest.raises(ValueError):
        gli.compute_sparse_eri_gausslet_integrals(b, [(-1, 3), (0, 2), (-1, 3)], 1e-5)
    with pytest.raises(ValueError):
        gli.compute_sparse_erida_gausslet_integrals(b, sym_grid(3), -1.0)
    with pytest.raises(ValueError):
        gli.compute_kinetic_gausslet_integrals(b[:-1], sym_grid(3))
    s = gli.compute_sparse_erida_gausslet_integrals(b, sym_grid(3), 1e-5)
    with pytest.raises(SyntaxError):
        s.fill_matrix(sym_grid(5))
    with pytest.raises(SyntaxError):
        s.integral_value(([-2, 0, 0], [2, 0, 0]))
    with pytest.raises(ValueError):
        s.project(np.zeros((26, 2)))
