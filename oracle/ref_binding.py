"""ctypes binding of the reference C core built by ``oracle/Makefile`` into
``oracle/_ref/libgli_ref.so`` (test infrastructure: the checker, never the
product).

The struct layouts restate the reference headers:
  include/range.h:10-14            struct range
  include/grid.h:10-26             union cartesian_grid_point_3d, struct cartesian_grid_3d
  include/gausslet.h:10-14         struct gausslet_data
  include/nuclear_integrals.h:11-15, 31-37   struct atomic_nucleus / nuclear_gausslet_integrals
  include/kinetic_integrals.h:14-18          struct kinetic_gausslet_integrals
  include/eri_integrals.h:23-47              sparse_eri_indices / sparse_eri_gausslet_integrals
  include/erida_integrals.h:21-45            sparse_erida_indices / sparse_erida_gausslet_integrals
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB_PATH = os.path.join(HERE, "_ref", "libgli_ref.so")

glong = C.c_int64
dptr = C.POINTER(C.c_double)
lptr = C.POINTER(glong)


class Range(C.Structure):
    _fields_ = [("istart", glong), ("num", glong)]


class Grid(C.Structure):
    _fields_ = [("coord_range", Range * 3)]


class Point(C.Structure):
    _fields_ = [("c", glong * 3)]


class GaussletData(C.Structure):
    _fields_ = [("coefficients", dptr), ("indices", Range)]


class Nucleus(C.Structure):
    _fields_ = [("pos", C.c_double * 3), ("charge", C.c_int)]


class Kinetic(C.Structure):
    _fields_ = [("integral_values", dptr), ("grid", Grid)]


class Nuclear(C.Structure):
    _fields_ = [("integral_values", dptr), ("grid", Grid),
                ("nuclei", C.POINTER(Nucleus)), ("num_nuclei", C.c_int)]


class SparseIndices(C.Structure):
    _fields_ = [("indices", lptr), ("num", glong), ("grid", Grid)]


class SparseIntegrals(C.Structure):
    _fields_ = [("integral_values", dptr), ("indices", lptr),
                ("num_entries", glong), ("grid", Grid)]


def make_grid(spec):
    g = Grid()
    for a in range(3):
        g.coord_range[a].istart = int(spec[a][0])
        g.coord_range[a].num = int(spec[a][1])
    return g


def make_points(pts):
    arr = (Point * len(pts))()
    for k, p in enumerate(pts):
        for a in range(3):
            arr[k].c[a] = int(p[a])
    return arr


def grid_points(spec):
    return int(spec[0][1]) * int(spec[1][1]) * int(spec[2][1])


class RefLib:
    """The unmodified reference C core, called through its own C API."""

    def __init__(self, path=REF_LIB_PATH):
        if not os.path.exists(path):
            raise FileNotFoundError(f"reference core not built: {path} (run make -C oracle ref)")
        self.lib = L = C.CDLL(path)
        P, V = C.POINTER, None
        L.compute_kinetic_gausslet_integral.argtypes = [P(GaussletData), P(Point)]
        L.compute_kinetic_gausslet_integral.restype = C.c_double
        L.compute_kinetic_gausslet_integrals.argtypes = [P(GaussletData), P(Grid), P(Kinetic)]
        L.delete_kinetic_gausslet_integrals.argtypes = [P(Kinetic)]
        L.compute_nuclear_gausslet_integral.argtypes = [P(GaussletData), P(Point), P(Nucleus), C.c_int, C.c_double]
        L.compute_nuclear_gausslet_integral.restype = C.c_double
        L.compute_nuclear_gausslet_integrals.argtypes = [P(GaussletData), P(Grid), P(Nucleus), C.c_int, C.c_double, P(Nuclear)]
        L.delete_nuclear_gausslet_integrals.argtypes = [P(Nuclear)]
        L.compute_eri_gausslet_integral.argtypes = [P(GaussletData), P(Point), C.c_double]
        L.compute_eri_gausslet_integral.restype = C.c_double
        L.compute_erida_gausslet_integral.argtypes = [P(GaussletData), P(Point), C.c_double]
        L.compute_erida_gausslet_integral.restype = C.c_double
        for kind in ("eri", "erida"):
            getattr(L, f"enumerate_symmetry_reduced_{kind}_indices").argtypes = [P(Grid), P(SparseIndices)]
            getattr(L, f"delete_sparse_{kind}_indices").argtypes = [P(SparseIndices)]
            getattr(L, f"compute_sparse_{kind}_gausslet_integrals").argtypes = [
                P(GaussletData), P(Grid), lptr, glong, C.c_double, P(SparseIntegrals)]
            getattr(L, f"sparse_{kind}_gausslet_integrals_get_value").argtypes = [P(SparseIntegrals), glong]
            getattr(L, f"sparse_{kind}_gausslet_integrals_get_value").restype = C.c_double
            getattr(L, f"project_sparse_{kind}_gausslet_integrals").argtypes = [P(SparseIntegrals), dptr, glong, dptr]
            getattr(L, f"delete_sparse_{kind}_gausslet_integrals").argtypes = [P(SparseIntegrals)]
        L.fill_dense_eri_tensor.argtypes = [P(SparseIntegrals), P(Grid), dptr]
        L.fill_dense_erida_matrix.argtypes = [P(SparseIntegrals), P(Grid), dptr]
        L.apply_sparse_eri_tensor.argtypes = [P(SparseIntegrals), dptr, glong, dptr]

    # -- helpers -------------------------------------------------------------
    @staticmethod
    def _gdata(coeffs):
        c = np.ascontiguousarray(coeffs, dtype=np.float64)
        g = GaussletData()
        g.coefficients = c.ctypes.data_as(dptr)
        g.indices.num = c.size
        g.indices.istart = -(c.size - 1) // 2
        return g, c

    # -- single entries ------------------------------------------------------
    def kinetic_single(self, coeffs, pts):
        g, keep = self._gdata(coeffs)
        return self.lib.compute_kinetic_gausslet_integral(C.byref(g), make_points(pts))

    def nuclear_single(self, coeffs, pts, positions, charges, tol):
        g, keep = self._gdata(coeffs)
        nuc = (Nucleus * len(charges))()
        for k, (p, z) in enumerate(zip(positions, charges)):
            nuc[k].pos[:] = [float(v) for v in p]
            nuc[k].charge = int(z)
        return self.lib.compute_nuclear_gausslet_integral(C.byref(g), make_points(pts), nuc, len(charges), tol)

    def eri_single(self, coeffs, pts, tol):
        g, keep = self._gdata(coeffs)
        return self.lib.compute_eri_gausslet_integral(C.byref(g), make_points(pts), tol)

    def erida_single(self, coeffs, pts, tol):
        g, keep = self._gdata(coeffs)
        return self.lib.compute_erida_gausslet_integral(C.byref(g), make_points(pts), tol)

    # -- matrices ------------------------------------------------------------
    def kinetic_matrix(self, coeffs, grid):
        g, keep = self._gdata(coeffs)
        out = Kinetic()
        self.lib.compute_kinetic_gausslet_integrals(C.byref(g), C.byref(make_grid(grid)), C.byref(out))
        n = grid_points(grid)
        res = np.ctypeslib.as_array(out.integral_values, shape=(n, n)).copy()
        self.lib.delete_kinetic_gausslet_integrals(C.byref(out))
        return res

    def nuclear_matrix(self, coeffs, grid, positions, charges, tol):
        g, keep = self._gdata(coeffs)
        nuc = (Nucleus * len(charges))()
        for k, (p, z) in enumerate(zip(positions, charges)):
            nuc[k].pos[:] = [float(v) for v in p]
            nuc[k].charge = int(z)
        out = Nuclear()
        self.lib.compute_nuclear_gausslet_integrals(C.byref(g), C.byref(make_grid(grid)), nuc, len(charges), tol, C.byref(out))
        n = grid_points(grid)
        res = np.ctypeslib.as_array(out.integral_values, shape=(n, n)).copy()
        self.lib.delete_nuclear_gausslet_integrals(C.byref(out))
        return res

    # -- sparse ERI / ERIDA ---------------------------------------------------
    def enumerate(self, kind, grid):
        out = SparseIndices()
        getattr(self.lib, f"enumerate_symmetry_reduced_{kind}_indices")(C.byref(make_grid(grid)), C.byref(out))
        res = np.ctypeslib.as_array(out.indices, shape=(out.num,)).copy() if out.num else np.zeros(0, np.int64)
        getattr(self.lib, f"delete_sparse_{kind}_indices")(C.byref(out))
        return res

    def sparse_values(self, kind, coeffs, grid, indices, tol):
        g, keep = self._gdata(coeffs)
        idx = np.ascontiguousarray(indices, dtype=np.int64)
        out = SparseIntegrals()
        getattr(self.lib, f"compute_sparse_{kind}_gausslet_integrals")(
            C.byref(g), C.byref(make_grid(grid)), idx.ctypes.data_as(lptr), idx.size, tol, C.byref(out))
        res = np.ctypeslib.as_array(out.integral_values, shape=(idx.size,)).copy() if idx.size else np.zeros(0)
        getattr(self.lib, f"delete_sparse_{kind}_gausslet_integrals")(C.byref(out))
        return res

    def _sparse_struct(self, kind, grid, indices, values):
        s = SparseIntegrals()
        idx = np.ascontiguousarray(indices, dtype=np.int64)
        val = np.ascontiguousarray(values, dtype=np.float64)
        s.integral_values = val.ctypes.data_as(dptr)
        s.indices = idx.ctypes.data_as(lptr)
        s.num_entries = idx.size
        s.grid = make_grid(grid)
        return s, (idx, val)

    def fill_dense(self, kind, grid, indices, values, dense_grid):
        s, keep = self._sparse_struct(kind, grid, indices, values)
        n = grid_points(dense_grid)
        shape = (n, n, n, n) if kind == "eri" else (n, n)
        out = np.empty(shape)
        fn = self.lib.fill_dense_eri_tensor if kind == "eri" else self.lib.fill_dense_erida_matrix
        fn(C.byref(s), C.byref(make_grid(dense_grid)), out.ctypes.data_as(dptr))
        return out

    def project(self, kind, grid, indices, values, basis):
        s, keep = self._sparse_struct(kind, grid, indices, values)
        b = np.ascontiguousarray(basis, dtype=np.float64)
        m = b.shape[1]
        out = np.empty((m, m, m, m))
        getattr(self.lib, f"project_sparse_{kind}_gausslet_integrals")(
            C.byref(s), b.ctypes.data_as(dptr), m, out.ctypes.data_as(dptr))
        return out

    def apply(self, grid, indices, values, states):
        s, keep = self._sparse_struct("eri", grid, indices, values)
        st = np.ascontiguousarray(states, dtype=np.float64)
        m = 1 if st.ndim == 1 else st.shape[1]
        out = np.empty(st.shape)
        self.lib.apply_sparse_eri_tensor(C.byref(s), st.ctypes.data_as(dptr), m, out.ctypes.data_as(dptr))
        return out
