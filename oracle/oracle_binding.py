"""ctypes binding of the CPU restatement ``oracle/gli_oracle.c``, built by
``make -C oracle restated`` into ``oracle/_build/libgli_oracle.so``.

TEST INFRASTRUCTURE ONLY: tests/, ``__graft_entry__.smoke()`` and bench.py's
CPU-baseline leg use it as the checker.  The product never imports it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB_PATH = os.path.join(HERE, "_build", "libgli_oracle.so")

_i64p = C.POINTER(C.c_int64)
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def build():
    """Compile the restatement (and, where GLI_REFERENCE_DIR names a checkout
    of the reference, the reference core) with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", HERE, "restated"], check=True)
    ref = os.environ.get("GLI_REFERENCE_DIR", "")
    if ref and os.path.isdir(os.path.join(ref, "src")):
        subprocess.run(["make", "-s", "-C", HERE, "ref"], check=True)
        # the reference's own Python module and CLI drivers linked against the
        # B200 library (the drop-in checks), once that library is built
        if os.path.exists(os.path.join(os.path.dirname(HERE), "gausslectronitegrate_b200", "libgli_b200.so")):
            subprocess.run(["make", "-s", "-C", HERE, "dropin", "cli"], check=True)


def _grid6(grid):
    return np.array([grid[0][0], grid[0][1], grid[1][0], grid[1][1], grid[2][0], grid[2][1]], dtype=np.int64)


def _p(a, t):
    return a.ctypes.data_as(t)


class Oracle:
    def __init__(self, path=ORACLE_LIB_PATH):
        if not os.path.exists(path):
            build()
        self.lib = L = C.CDLL(path)
        L.oracle_factors.argtypes = [_dp, C.c_int64, C.c_int64, C.c_double, _dp, _i64p]
        L.oracle_factors.restype = C.c_int64
        L.oracle_erida_products.argtypes = [_dp, C.c_int64, C.c_double, _dp, _i64p]
        L.oracle_erida_products.restype = C.c_int64
        L.oracle_eri_products.argtypes = [_dp, C.c_int64, C.c_int64, C.c_int64, C.c_double, _dp, _i64p]
        L.oracle_eri_products.restype = C.c_int64
        L.oracle_kinetic_single.argtypes = [_dp, C.c_int64, _i64p]
        L.oracle_kinetic_single.restype = C.c_double
        L.oracle_kinetic_matrix.argtypes = [_dp, C.c_int64, _i64p, _dp]
        L.oracle_nuclear_single.argtypes = [_dp, C.c_int64, _i64p, _dp, _ip, C.c_int, C.c_double]
        L.oracle_nuclear_single.restype = C.c_double
        L.oracle_nuclear_matrix.argtypes = [_dp, C.c_int64, _i64p, _dp, _ip, C.c_int, C.c_double, _dp]
        L.oracle_nuclear_pairs.argtypes = [_dp, C.c_int64, _i64p, _dp, _ip, C.c_int, C.c_double, _i64p, C.c_int64, _dp]
        L.oracle_erida_single.argtypes = [_dp, C.c_int64, _i64p, C.c_double]
        L.oracle_erida_single.restype = C.c_double
        L.oracle_eri_single.argtypes = [_dp, C.c_int64, _i64p, C.c_double]
        L.oracle_eri_single.restype = C.c_double
        for k in ("erida", "eri"):
            getattr(L, f"oracle_{k}_values").argtypes = [_dp, C.c_int64, _i64p, _i64p, C.c_int64, C.c_double, _dp]
            getattr(L, f"oracle_enumerate_{k}").argtypes = [_i64p, _i64p, C.c_int64]
            getattr(L, f"oracle_enumerate_{k}").restype = C.c_int64
            getattr(L, f"oracle_canonical_{k}").argtypes = [_i64p, _i64p]
            getattr(L, f"oracle_canonical_{k}").restype = C.c_int64
            getattr(L, f"oracle_fill_dense_{k}").argtypes = [_i64p, _i64p, _dp, C.c_int64, _i64p, _dp]
        L.oracle_apply_eri.argtypes = [_i64p, _i64p, _dp, C.c_int64, _dp, C.c_int64, _dp]
        L.oracle_coulomb_table.argtypes = [C.c_int, C.c_int64, _dp]

    @staticmethod
    def _c(coeffs):
        return np.ascontiguousarray(coeffs, dtype=np.float64)

    def factors(self, coeffs, shift, tol):
        c = self._c(coeffs)
        out = np.zeros(2 * c.size - 1)
        first = C.c_int64()
        n = self.lib.oracle_factors(_p(c, _dp), c.size, shift, tol, _p(out, _dp), C.byref(first))
        return out[:n].copy(), first.value

    def erida_products(self, coeffs, tol):
        c = self._c(coeffs)
        out = np.zeros(2 * c.size - 1)
        first = C.c_int64()
        n = self.lib.oracle_erida_products(_p(c, _dp), c.size, tol, _p(out, _dp), C.byref(first))
        return out[:n].copy(), first.value

    def eri_products(self, coeffs, s01, s23, tol):
        c = self._c(coeffs)
        out = np.zeros(4 * c.size - 3)
        first = C.c_int64()
        n = self.lib.oracle_eri_products(_p(c, _dp), c.size, s01, s23, tol, _p(out, _dp), C.byref(first))
        return out[:n].copy(), first.value

    def coulomb_table(self, eri, n):
        out = np.zeros(n)
        self.lib.oracle_coulomb_table(int(eri), n, _p(out, _dp))
        return out

    def kinetic_single(self, coeffs, pts):
        c = self._c(coeffs)
        p = np.asarray(pts, dtype=np.int64).ravel()
        return self.lib.oracle_kinetic_single(_p(c, _dp), c.size, _p(p, _i64p))

    def kinetic_matrix(self, coeffs, grid):
        c = self._c(coeffs)
        g = _grid6(grid)
        n = int(g[1] * g[3] * g[5])
        out = np.empty((n, n))
        self.lib.oracle_kinetic_matrix(_p(c, _dp), c.size, _p(g, _i64p), _p(out, _dp))
        return out

    @staticmethod
    def _nuc(positions, charges):
        pos = np.ascontiguousarray(np.asarray(positions, dtype=np.float64).reshape(-1, 3))
        ch = np.ascontiguousarray(np.asarray(charges, dtype=np.int32))
        return pos, ch

    def nuclear_single(self, coeffs, pts, positions, charges, tol):
        c = self._c(coeffs)
        p = np.asarray(pts, dtype=np.int64).ravel()
        pos, ch = self._nuc(positions, charges)
        return self.lib.oracle_nuclear_single(_p(c, _dp), c.size, _p(p, _i64p), _p(pos, _dp), _p(ch, _ip), ch.size, tol)

    def nuclear_matrix(self, coeffs, grid, positions, charges, tol):
        c = self._c(coeffs)
        g = _grid6(grid)
        pos, ch = self._nuc(positions, charges)
        n = int(g[1] * g[3] * g[5])
        out = np.empty((n, n))
        self.lib.oracle_nuclear_matrix(_p(c, _dp), c.size, _p(g, _i64p), _p(pos, _dp), _p(ch, _ip), ch.size, tol, _p(out, _dp))
        return out

    def nuclear_pairs(self, coeffs, grid, positions, charges, tol, pairs):
        c = self._c(coeffs)
        g = _grid6(grid)
        pos, ch = self._nuc(positions, charges)
        pr = np.ascontiguousarray(np.asarray(pairs, dtype=np.int64).reshape(-1, 2))
        out = np.empty(pr.shape[0])
        self.lib.oracle_nuclear_pairs(_p(c, _dp), c.size, _p(g, _i64p), _p(pos, _dp), _p(ch, _ip), ch.size, tol,
                                      _p(pr, _i64p), pr.shape[0], _p(out, _dp))
        return out

    def single(self, kind, coeffs, pts, tol):
        c = self._c(coeffs)
        p = np.ascontiguousarray(np.asarray(pts, dtype=np.int64).ravel())
        return getattr(self.lib, f"oracle_{kind}_single")(_p(c, _dp), c.size, _p(p, _i64p), tol)

    def values(self, kind, coeffs, grid, idx, tol):
        c = self._c(coeffs)
        g = _grid6(grid)
        ix = np.ascontiguousarray(idx, dtype=np.int64)
        out = np.empty(ix.size)
        getattr(self.lib, f"oracle_{kind}_values")(_p(c, _dp), c.size, _p(g, _i64p), _p(ix, _i64p), ix.size, tol, _p(out, _dp))
        return out

    def enumerate(self, kind, grid):
        g = _grid6(grid)
        fn = getattr(self.lib, f"oracle_enumerate_{kind}")
        n = fn(_p(g, _i64p), None, 0)
        if n < 0:
            raise ValueError("grid is not rotationally symmetric")
        out = np.empty(n, dtype=np.int64)
        fn(_p(g, _i64p), _p(out, _i64p), n)
        return out

    def canonical(self, kind, grid, pts):
        g = _grid6(grid)
        p = np.ascontiguousarray(np.asarray(pts, dtype=np.int64).ravel())
        return getattr(self.lib, f"oracle_canonical_{kind}")(_p(g, _i64p), _p(p, _i64p))

    def fill_dense(self, kind, grid, idx, val, dense_grid):
        gs, gd = _grid6(grid), _grid6(dense_grid)
        ix = np.ascontiguousarray(idx, dtype=np.int64)
        v = np.ascontiguousarray(val, dtype=np.float64)
        n = int(gd[1] * gd[3] * gd[5])
        out = np.empty((n,) * (4 if kind == "eri" else 2))
        getattr(self.lib, f"oracle_fill_dense_{kind}")(_p(gs, _i64p), _p(ix, _i64p), _p(v, _dp), ix.size, _p(gd, _i64p), _p(out, _dp))
        return out

    def apply(self, grid, idx, val, states):
        g = _grid6(grid)
        ix = np.ascontiguousarray(idx, dtype=np.int64)
        v = np.ascontiguousarray(val, dtype=np.float64)
        st = np.ascontiguousarray(states, dtype=np.float64)
        ns = 1 if st.ndim == 1 else st.shape[1]
        out = np.empty(st.shape)
        self.lib.oracle_apply_eri(_p(g, _i64p), _p(ix, _i64p), _p(v, _dp), ix.size, _p(st, _dp), ns, _p(out, _dp))
        return out


def project_factored(dense, basis):
    """Projection of a dense 4-index tensor onto a basis as four one-axis
    contractions -- the reference test's own check (test/test_eri_integrals.c:
    188-212, tensor_multiply_axis :426-455), done with numpy."""
    t = np.tensordot(dense, basis, axes=([3], [0]))          # (i,j,k,s)
    t = np.tensordot(t, basis, axes=([2], [0]))              # (i,j,s,r)
    t = np.tensordot(t, basis, axes=([1], [0]))              # (i,s,r,q)
    t = np.tensordot(t, basis, axes=([0], [0]))              # (s,r,q,p)
    return np.ascontiguousarray(t.transpose(3, 2, 1, 0))
