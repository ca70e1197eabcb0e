"""gausslectronitegrate_b200 -- B200 (sm_100a) implementation of the
gausslectronitegrate integral hot path.

The module mirrors the reference's Python interface (python/pymodule.c:
module functions at :1839-1921, types SparseERI :647-1108 and SparseERIDA
:1375-1752): same function names, argument meaning and exception types
(SyntaxError for unparsable arguments, ValueError for bad shapes and grids,
TypeError for a wrong dtype, RuntimeError for allocation and device
failures).  Every computation runs in libgli_b200's CUDA kernels through its
C ABI; there is no CPU fallback -- without a CUDA device the calls raise
RuntimeError.

Extension beyond the reference signature: compute_sparse_{eri,erida}_gausslet_integrals
accept an optional keyword ``form`` ("fp64", the default and drop-in form, or
"mixed").
"""
import ctypes as C

import numpy as np

from . import _abi

__all__ = [
    "grid_num_points", "grid_point_to_linear_index", "linear_index_to_grid_point",
    "compute_kinetic_gausslet_integral", "compute_kinetic_gausslet_integrals",
    "compute_nuclear_gausslet_integral", "compute_nuclear_gausslet_integrals",
    "compute_eri_gausslet_integral", "compute_sparse_eri_gausslet_integrals", "load_sparse_eri_gausslet_integrals",
    "compute_erida_gausslet_integral", "compute_sparse_erida_gausslet_integrals",
    "get_max_openmp_threads", "SparseERI", "SparseERIDA", "lib",
]

_lib = None


def lib():
    """The loaded libgli_b200 (ctypes.CDLL)."""
    global _lib
    if _lib is None:
        _lib = _abi.load()
    return _lib


def _raise_if_failed(syntax):
    L = lib()
    code = L.gli_b200_last_error()
    if code != 0:
        msg = L.gli_b200_last_error_message().decode(errors="replace")
        exc = ValueError if code == 2 else RuntimeError
        raise exc(f"{msg}; syntax: {syntax}")


# ---------------------------------------------------------------------------
# argument parsing, mirroring python/pymodule.c:17-297

def _parse_coeffs(obj, syntax):
    try:
        arr = np.asarray(obj)
    except Exception:
        raise ValueError(f"converting input argument 'gausslet_coeffs' to a NumPy array with degree 1 failed; syntax: {syntax}")
    if arr.ndim != 1:
        raise ValueError(f"'gausslet_coeffs' must have degree 1, received {arr.ndim}; syntax: {syntax}")
    if arr.shape[0] % 2 != 1:
        raise ValueError(f"'gausslet_coeffs' must have an odd number of entries; syntax: {syntax}")
    if not (np.issubdtype(arr.dtype, np.floating) or np.issubdtype(arr.dtype, np.integer)):
        raise TypeError(f"'gausslet_coeffs' must have 'double' format entries; syntax: {syntax}")
    arr = np.ascontiguousarray(arr, dtype=np.float64)
    g = _abi.GaussletData()
    g.coefficients = arr.ctypes.data_as(_abi.dptr)
    g.indices.num = arr.shape[0]
    g.indices.istart = -(arr.shape[0] - 1) // 2
    return g, arr


def _as_int(v, msg):
    try:
        if isinstance(v, (bool, np.bool_)):
            raise TypeError
        return int(v.__index__())
    except Exception:
        raise ValueError(msg)


def _parse_grid(obj, syntax):
    if not hasattr(obj, "__len__") or not hasattr(obj, "__getitem__"):
        raise ValueError(f"cannot interpret 'grid' as a sequence; syntax: {syntax}")
    if len(obj) != 3:
        raise ValueError(f"'grid' must be a sequence of length three (corresponding to the Cartesian axis directions); syntax: {syntax}")
    spec = []
    for i in range(3):
        r = obj[i]
        if not hasattr(r, "__len__") or not hasattr(r, "__getitem__"):
            raise ValueError(f"cannot interpret 'grid[{i}]' as a sequence; syntax: {syntax}")
        if len(r) != 2:
            raise ValueError(f"'grid[{i}]' must be a sequence of length two (start coordinate and number of grid points along direction {i}); syntax: {syntax}")
        start = _as_int(r[0], f"cannot interpret the first entry in 'grid[{i}]' as an integer; syntax: {syntax}")
        num = _as_int(r[1], f"cannot interpret the second entry in 'grid[{i}]' as an integer; syntax: {syntax}")
        if num <= 0:
            raise ValueError(f"number of grid points along direction {i} (second entry in 'grid[{i}]') must be a positive integer; syntax: {syntax}")
        spec.append((start, num))
    return spec


def _grid_struct(spec):
    g = _abi.Grid()
    for a in range(3):
        g.coord_range[a].istart = spec[a][0]
        g.coord_range[a].num = spec[a][1]
    return g


def _parse_point(obj, syntax):
    if not hasattr(obj, "__len__") or not hasattr(obj, "__getitem__"):
        raise ValueError(f"cannot interpret grid point as a sequence; syntax: {syntax}")
    if len(obj) != 3:
        raise ValueError(f"grid point must be a sequence of length three (corresponding to the Cartesian coordinates); syntax: {syntax}")
    return [_as_int(obj[i], f"cannot interpret the {i}-th entry in grid point as an integer; syntax: {syntax}")
            for i in range(3)]


def _parse_points(obj, syntax, num):
    if not hasattr(obj, "__len__") or not hasattr(obj, "__getitem__"):
        raise ValueError(f"cannot interpret 'grid_points' as a sequence; syntax: {syntax}")
    if len(obj) != num:
        raise ValueError(f"'grid_points' must be a sequence of length {num}; syntax: {syntax}")
    pts = []
    for k in range(num):
        p = obj[k]
        if not hasattr(p, "__len__") or not hasattr(p, "__getitem__"):
            raise ValueError(f"cannot interpret 'grid_points[{k}]' as a sequence; syntax: {syntax}")
        if len(p) != 3:
            raise ValueError(f"'grid_points[{k}]' must be a sequence of length three (corresponding to the Cartesian coordinates); syntax: {syntax}")
        pts.append([_as_int(p[i], f"cannot interpret the {i}-th entry in 'grid_points[{k}]' as an integer; syntax: {syntax}")
                    for i in range(3)])
    return pts


def _points_struct(pts):
    arr = (_abi.Point * len(pts))()
    for k, p in enumerate(pts):
        for a in range(3):
            arr[k].c[a] = p[a]
    return arr


def _parse_nuclei(positions, charges, syntax):
    if not hasattr(positions, "__len__"):
        raise ValueError(f"cannot interpret 'nuclear_positions' as a sequence; syntax: {syntax}")
    if not hasattr(charges, "__len__"):
        raise ValueError(f"cannot interpret 'nuclear_charges' as a sequence; syntax: {syntax}")
    if len(positions) != len(charges):
        raise ValueError(f"number of nuclear positions must be equal to the number of nuclear charges; syntax: {syntax}")
    n = len(positions)
    if n == 0:
        raise ValueError(f"'nuclear_positions' cannot be an empty sequence; syntax: {syntax}")
    nuc = (_abi.Nucleus * n)()
    for i in range(n):
        try:
            p = np.asarray(positions[i], dtype=np.float64)
        except Exception:
            raise ValueError(f"converting 'nuclear_positions[{i}]' to a NumPy array with degree 1 failed; syntax: {syntax}")
        if p.ndim != 1:
            raise ValueError(f"'nuclear_positions[{i}]' must have degree 1; syntax: {syntax}")
        if p.shape[0] != 3:
            raise ValueError(f"'nuclear_positions[{i}]' must be a vector with three entries; syntax: {syntax}")
        nuc[i].pos[:] = [float(v) for v in p]
        nuc[i].charge = _as_int(charges[i], f"cannot interpret 'nuclear_charges[{i}]' as an integer; syntax: {syntax}")
    return nuc, n


def _parse_tol(tol, syntax):
    try:
        return float(tol)
    except Exception:
        raise SyntaxError(f"error parsing input; syntax: {syntax}")


def _symmetric_extent(spec):
    return max(max(abs(s), abs(s + n - 1)) for s, n in spec)


# ---------------------------------------------------------------------------
# grid helpers (python/pymodule.c:300-419)

def grid_num_points(grid):
    """Overall number of points of a Cartesian grid."""
    spec = _parse_grid(grid, "grid_num_points(grid)")
    return spec[0][1] * spec[1][1] * spec[2][1]


def grid_point_to_linear_index(grid, point):
    """Convert a Cartesian grid point to a linear index."""
    syntax = "grid_point_to_linear_index(grid, point)"
    spec = _parse_grid(grid, syntax)
    p = _parse_point(point, syntax)
    for a, name in enumerate("xyz"):
        if p[a] < spec[a][0] or spec[a][0] + spec[a][1] - 1 < p[a]:
            raise ValueError(f"'point.{name}' out of grid coordinate range; syntax: {syntax}")
    return ((p[0] - spec[0][0]) * spec[1][1] + (p[1] - spec[1][0])) * spec[2][1] + (p[2] - spec[2][0])


def linear_index_to_grid_point(grid, idx):
    """Convert a linear index to a Cartesian grid point."""
    syntax = "linear_index_to_grid_point(grid, idx)"
    spec = _parse_grid(grid, syntax)
    try:
        idx = int(idx)
    except Exception:
        raise SyntaxError(f"error parsing input; syntax: {syntax}")
    n = spec[0][1] * spec[1][1] * spec[2][1]
    if idx < 0 or n <= idx:
        raise ValueError(f"'idx' out of range; syntax: {syntax}")
    iz = idx % spec[2][1]
    rm = idx // spec[2][1]
    iy = rm % spec[1][1]
    ix = rm // spec[1][1]
    return (spec[0][0] + ix, spec[1][0] + iy, spec[2][0] + iz)


def get_max_openmp_threads():
    """The reference reports its OpenMP thread count; this implementation runs
    on the GPU and uses no OpenMP, so the answer is 0 ("not available")."""
    return 0


# ---------------------------------------------------------------------------
# kinetic (python/pymodule.c:422-493)

def compute_kinetic_gausslet_integral(gausslet_coeffs, grid_points):
    """Evaluate a single kinetic overlap integral for Gausslet orbitals."""
    syntax = "compute_kinetic_gausslet_integral(gausslet_coeffs, grid_points)"
    g, keep = _parse_coeffs(gausslet_coeffs, syntax)
    pts = _points_struct(_parse_points(grid_points, syntax, 2))
    v = lib().compute_kinetic_gausslet_integral(C.byref(g), pts)
    _raise_if_failed(syntax)
    return v


def compute_kinetic_gausslet_integrals(gausslet_coeffs, grid):
    """Evaluate the kinetic overlap integrals for Gausslet orbitals (dense N x N)."""
    syntax = "compute_kinetic_gausslet_integrals(gausslet_coeffs, grid)"
    g, keep = _parse_coeffs(gausslet_coeffs, syntax)
    spec = _parse_grid(grid, syntax)
    out = _abi.Kinetic()
    L = lib()
    L.compute_kinetic_gausslet_integrals(C.byref(g), C.byref(_grid_struct(spec)), C.byref(out))
    _raise_if_failed(syntax)
    n = spec[0][1] * spec[1][1] * spec[2][1]
    return _adopt_matrix(out, n, L.delete_kinetic_gausslet_integrals)


class _OwnedMatrix:
    """A dense matrix that the library allocated in a result struct, handed
    to numpy without a copy: numpy keeps this object as the array's base, and
    the struct's delete_* runs when the array goes away."""

    def __init__(self, struct, n, deleter):
        self._struct, self._deleter = struct, deleter
        self.__array_interface__ = {"data": (C.cast(struct.integral_values, C.c_void_p).value, False),
                                    "shape": (n, n), "typestr": "<f8", "version": 3}

    def __del__(self):
        self._deleter(C.byref(self._struct))


def _adopt_matrix(struct, n, deleter):
    return np.asarray(_OwnedMatrix(struct, n, deleter))


# ---------------------------------------------------------------------------
# nuclear (python/pymodule.c:496-603)

def compute_nuclear_gausslet_integral(gausslet_coeffs, grid_points, nuclear_positions, nuclear_charges, tol):
    """Evaluate a single nuclear overlap integral for Gausslet orbitals."""
    syntax = ("compute_nuclear_gausslet_integral(gausslet_coeffs, grid_points, nuclear_positions, "
              "nuclear_charges, tol)")
    g, keep = _parse_coeffs(gausslet_coeffs, syntax)
    pts = _points_struct(_parse_points(grid_points, syntax, 2))
    nuc, n = _parse_nuclei(nuclear_positions, nuclear_charges, syntax)
    v = lib().compute_nuclear_gausslet_integral(C.byref(g), pts, nuc, n, _parse_tol(tol, syntax))
    _raise_if_failed(syntax)
    return v


def compute_nuclear_gausslet_integrals(gausslet_coeffs, grid, nuclear_positions, nuclear_charges, tol):
    """Evaluate the nuclear overlap integrals for Gausslet orbitals (dense N x N)."""
    syntax = "compute_nuclear_gausslet_integrals(gausslet_coeffs, grid, nuclear_positions, nuclear_charges, tol)"
    g, keep = _parse_coeffs(gausslet_coeffs, syntax)
    spec = _parse_grid(grid, syntax)
    nuc, n = _parse_nuclei(nuclear_positions, nuclear_charges, syntax)
    out = _abi.Nuclear()
    L = lib()
    L.compute_nuclear_gausslet_integrals(C.byref(g), C.byref(_grid_struct(spec)), nuc, n, _parse_tol(tol, syntax),
                                         C.byref(out))
    _raise_if_failed(syntax)
    npts = spec[0][1] * spec[1][1] * spec[2][1]
    return _adopt_matrix(out, npts, L.delete_nuclear_gausslet_integrals)


def compute_nuclear_gausslet_integrals_batch(gausslet_coeffs, grids, nuclear_positions, nuclear_charges, tol,
                                             form="fp64"):
    """Nuclear matrices of many instances in one call (extension: no
    counterpart in the reference module).  grids[k], nuclear_positions[k] and
    nuclear_charges[k] describe instance k exactly as for
    compute_nuclear_gausslet_integrals; all instances share the coefficients and
    tol.  form "fp64" (the reference's arithmetic) or "mixed" (tensor-core
    contractions, about 1e-9 relative).  Returns a list of N_k x N_k arrays."""
    syntax = ("compute_nuclear_gausslet_integrals_batch(gausslet_coeffs, grids, nuclear_positions, "
              "nuclear_charges, tol, form='fp64')")
    g, keep = _parse_coeffs(gausslet_coeffs, syntax)
    if form not in _FORMS:
        raise ValueError(f"'form' must be one of {sorted(_FORMS)}; syntax: {syntax}")
    if not (len(grids) == len(nuclear_positions) == len(nuclear_charges)):
        raise ValueError(f"grids, positions and charges must have one entry per instance; syntax: {syntax}")
    n = len(grids)
    if n == 0:
        return []
    specs = [_parse_grid(gr, syntax) for gr in grids]
    gstructs = (_abi.Grid * n)(*[_grid_struct(sp) for sp in specs])
    nucs, offsets = [], [0]
    for pos, q in zip(nuclear_positions, nuclear_charges):
        arr, cnt = _parse_nuclei(pos, q, syntax)
        nucs.extend(arr[k] for k in range(cnt))
        offsets.append(offsets[-1] + cnt)
    nuc_arr = (_abi.Nucleus * len(nucs))(*nucs)
    off = np.asarray(offsets, dtype=np.int64)
    outs = [np.empty((sp[0][1] * sp[1][1] * sp[2][1],) * 2) for sp in specs]
    ptrs = (C.c_void_p * n)(*[o.ctypes.data for o in outs])
    lib().gli_b200_nuclear_batch(C.byref(g), n, gstructs, off.ctypes.data_as(_abi.lptr), nuc_arr,
                                 _parse_tol(tol, syntax), _FORMS[form], ptrs)
    _raise_if_failed(syntax)
    return outs


# ---------------------------------------------------------------------------
# sparse ERI / ERIDA objects (python/pymodule.c:606-1108, 1334-1826)

_FORMS = {"fp64": _abi.GLI_FORM_FP64, "mixed": _abi.GLI_FORM_MIXED}


class _Sparse:
    _kind = None            # "eri" / "erida"
    _npts = None            # points per index tuple

    def __init__(self):
        raise TypeError(f"{type(self).__name__} objects are created by compute_sparse_{self._kind}_gausslet_integrals")

    @classmethod
    def _make(cls, coeffs, spec, indices, values, tol):
        self = object.__new__(cls)
        self._coeffs = np.ascontiguousarray(coeffs, dtype=np.float64)
        self._spec = [tuple(r) for r in spec]
        self._indices = np.ascontiguousarray(indices, dtype=np.int64)
        self._values = np.ascontiguousarray(values, dtype=np.float64)
        self._tol = float(tol)
        self._perm = None
        return self

    def _struct(self):
        s = _abi.SparseIntegrals()
        s.integral_values = self._values.ctypes.data_as(_abi.dptr)
        s.indices = self._indices.ctypes.data_as(_abi.lptr)
        s.num_entries = self._indices.size
        s.grid = _grid_struct(self._spec)
        return s

    def _perms(self):
        if self._perm is None:
            n = self._spec[0][1] * self._spec[1][1] * self._spec[2][1]
            tbl = (_abi.lptr * 48)()
            L = lib()
            L.evaluate_octahedral_grid_permutations(C.byref(_grid_struct(self._spec)), tbl)
            _raise_if_failed("evaluate_octahedral_grid_permutations(grid)")
            arrs = [np.ctypeslib.as_array(tbl[g], shape=(n,)).copy() for g in range(48)]
            libc = C.CDLL(None)
            for g in range(48):
                libc.free(C.cast(tbl[g], C.c_void_p))
            self._perm_arrays = arrs
            self._perm = (_abi.lptr * 48)(*[a.ctypes.data_as(_abi.lptr) for a in arrs])
        return self._perm

    def integral_value(self, grid_points):
        """Value of the tensor entry at the given points (after moving the box
        centre of the points to the origin, python/pymodule.c:711-779)."""
        syntax = "integral_value(grid_points)"
        pts = _parse_points(grid_points, syntax, self._npts)
        bias = [0, 0, 0]
        for a in range(3):
            c = min(p[a] for p in pts) + max(p[a] for p in pts)
            trans = int(c / 2)            # C division truncates toward zero
            bias[a] = c - 2 * trans
            for p in pts:
                p[a] -= trans
        for k, p in enumerate(pts):
            for a, name in enumerate("xyz"):
                if not (0 <= p[a] - self._spec[a][0] < self._spec[a][1]):
                    raise SyntaxError(f"{name}-coordinate of grid point {k} (after box center translation) out of range; syntax: {syntax}")
        n = self._spec[0][1] * self._spec[1][1] * self._spec[2][1]
        perm = self._perms()
        L = lib()
        best = None
        for bx in range(abs(bias[0]) + 1):
            for by in range(abs(bias[1]) + 1):
                for bz in range(abs(bias[2]) + 1):
                    lin = []
                    for p in pts:
                        q = (p[0] - bx * bias[0], p[1] - by * bias[1], p[2] - bz * bias[2])
                        lin.append(((q[0] - self._spec[0][0]) * self._spec[1][1] + (q[1] - self._spec[1][0])) * self._spec[2][1]
                                   + (q[2] - self._spec[2][0]))
                    if self._kind == "eri":
                        v = L.minimum_octahedral_orbit_eri_tensor_index(n, perm, *lin)
                    else:
                        v = L.minimum_octahedral_orbit_erida_tensor_index(n, perm, *lin)
                    best = v if best is None else min(best, v)
        fn = getattr(L, f"sparse_{self._kind}_gausslet_integrals_get_value")
        return fn(C.byref(self._struct()), best)

    def project(self, basis):
        syntax = "project(basis)"
        n = self._spec[0][1] * self._spec[1][1] * self._spec[2][1]
        try:
            b = np.ascontiguousarray(basis, dtype=np.float64)
        except Exception:
            raise ValueError(f"converting input argument to a NumPy array failed; syntax: {syntax}")
        if b.ndim != 2:
            raise ValueError(f"converting input argument to a NumPy array failed; syntax: {syntax}")
        if b.shape[0] != n:
            raise ValueError(f"leading dimension of basis matrix must be equal to the number of grid points ({n}); syntax: {syntax}")
        m = b.shape[1]
        if m == 0:
            raise ValueError(f"number of basis states cannot be zero; syntax: {syntax}")
        out = np.empty((m, m, m, m))
        getattr(lib(), f"project_sparse_{self._kind}_gausslet_integrals")(
            C.byref(self._struct()), b.ctypes.data_as(_abi.dptr), m, out.ctypes.data_as(_abi.dptr))
        _raise_if_failed(syntax)
        return out

    def _check_dense(self, dense_grid, syntax, label):
        spec = _parse_grid(dense_grid, syntax)
        ext = _symmetric_extent(spec)
        if any(self._spec[a][1] < 2 * ext + 1 for a in range(3)):
            raise SyntaxError(f"sparse {label} grid too small to fill all values for the provided grid (extent {ext}); syntax: {syntax}")
        return spec

    @property
    def grid(self):
        """underlying Cartesian grid"""
        return tuple(self._spec)

    @property
    def tol(self):
        """truncation tolerance used for calculating the integrals"""
        return self._tol

    @property
    def num_entries(self):
        """number of stored values after translational, octahedral and permutational symmetry reductions"""
        return int(self._indices.size)

    @property
    def gausslet_coeffs(self):
        """Gausslet coefficients used for calculating the integrals"""
        return self._coeffs.copy()

    # extensions: the raw sorted class list and values
    @property
    def indices(self):
        return self._indices.copy()

    @property
    def values(self):
        return self._values.copy()


class SparseERI(_Sparse):
    """Sparse (symmetry-reduced) ERI tensor of degree 4 (python/pymodule.c:606-1108)."""
    _kind = "eri"
    _npts = 4

    def fill_tensor(self, dense_grid):
        syntax = "fill_tensor(dense_grid)"
        spec = self._check_dense(dense_grid, syntax, "ERI")
        n = spec[0][1] * spec[1][1] * spec[2][1]
        out = np.empty((n, n, n, n))
        lib().fill_dense_eri_tensor(C.byref(self._struct()), C.byref(_grid_struct(spec)), out.ctypes.data_as(_abi.dptr))
        _raise_if_failed(syntax)
        return out

    def apply(self, states):
        syntax = "apply(states)"
        n = self._spec[0][1] * self._spec[1][1] * self._spec[2][1]
        try:
            st = np.ascontiguousarray(states, dtype=np.float64)
        except Exception:
            raise ValueError(f"converting input argument to a NumPy array failed; syntax: {syntax}")
        if st.ndim not in (1, 2):
            raise ValueError(f"converting input argument to a NumPy array failed; syntax: {syntax}")
        if st.shape[0] != n * n:
            raise ValueError(f"leading dimension of the input state matrix must be equal to the number of grid points squared ({n * n}); syntax: {syntax}")
        m = 1 if st.ndim == 1 else st.shape[1]
        if m == 0:
            raise ValueError(f"number of input states cannot be zero; syntax: {syntax}")
        out = np.empty(st.shape)
        lib().apply_sparse_eri_tensor(C.byref(self._struct()), st.ctypes.data_as(_abi.dptr), m,
                                      out.ctypes.data_as(_abi.dptr))
        _raise_if_failed(syntax)
        return out


class SparseERIDA(_Sparse):
    """Sparse (symmetry-reduced) ERIDA matrix (python/pymodule.c:1334-1752)."""
    _kind = "erida"
    _npts = 2

    def fill_matrix(self, dense_grid):
        syntax = "fill_matrix(dense_grid)"
        spec = self._check_dense(dense_grid, syntax, "ERIDA")
        n = spec[0][1] * spec[1][1] * spec[2][1]
        out = np.empty((n, n))
        lib().fill_dense_erida_matrix(C.byref(self._struct()), C.byref(_grid_struct(spec)), out.ctypes.data_as(_abi.dptr))
        _raise_if_failed(syntax)
        return out


def _compute_sparse(kind, gausslet_coeffs, grid, tol, form, syntax):
    g, coeffs = _parse_coeffs(gausslet_coeffs, syntax)
    tol = _parse_tol(tol, syntax)
    if tol < 0:
        raise ValueError(f"'tol' cannot be negative, received {tol:g}; syntax: {syntax}")
    spec = _parse_grid(grid, syntax)
    ext = _symmetric_extent(spec)
    for a in range(3):
        if spec[a][0] != -ext or spec[a][1] != 2 * ext + 1:
            raise ValueError(f"specified grid is not rotationally symmetric; syntax: {syntax}")
    if form not in _FORMS:
        raise ValueError(f"'form' must be one of {sorted(_FORMS)}; syntax: {syntax}")
    L = lib()
    gs = _grid_struct(spec)
    idx_s = _abi.SparseIndices()
    getattr(L, f"enumerate_symmetry_reduced_{kind}_indices")(C.byref(gs), C.byref(idx_s))
    _raise_if_failed(syntax)
    idx = np.ctypeslib.as_array(idx_s.indices, shape=(idx_s.num,)).copy() if idx_s.num else np.zeros(0, np.int64)
    getattr(L, f"delete_sparse_{kind}_indices")(C.byref(idx_s))
    vals = np.empty(idx.size)
    if idx.size:
        L.gli_b200_sparse_values(_abi.GLI_KIND_ERI if kind == "eri" else _abi.GLI_KIND_ERIDA, C.byref(g), C.byref(gs),
                                 idx.ctypes.data_as(_abi.lptr), idx.size, tol, _FORMS[form],
                                 vals.ctypes.data_as(_abi.dptr))
        _raise_if_failed(syntax)
    cls = SparseERI if kind == "eri" else SparseERIDA
    return cls._make(coeffs, spec, idx, vals, tol)


def compute_eri_gausslet_integral(gausslet_coeffs, grid_points, tol):
    """Evaluate a single electron repulsion integral (ERI) for Gausslet orbitals."""
    syntax = "compute_eri_gausslet_integral(gausslet_coeffs, grid_points, tol)"
    g, keep = _parse_coeffs(gausslet_coeffs, syntax)
    pts = _points_struct(_parse_points(grid_points, syntax, 4))
    v = lib().compute_eri_gausslet_integral(C.byref(g), pts, _parse_tol(tol, syntax))
    _raise_if_failed(syntax)
    return v


def compute_sparse_eri_gausslet_integrals(gausslet_coeffs, grid, tol, form="fp64"):
    """Symmetry-reduced ERI tensor of degree 4 for Gausslet orbitals on a
    rotationally symmetric grid; returns a SparseERI."""
    return _compute_sparse("eri", gausslet_coeffs, grid, tol, form,
                           "compute_sparse_eri_gausslet_integrals(gausslet_coeffs, grid, tol)")


def compute_erida_gausslet_integral(gausslet_coeffs, grid_points, tol):
    """Evaluate a single ERI in the integral diagonal approximation (ERIDA)."""
    syntax = "compute_erida_gausslet_integral(gausslet_coeffs, grid_points, tol)"
    g, keep = _parse_coeffs(gausslet_coeffs, syntax)
    pts = _points_struct(_parse_points(grid_points, syntax, 2))
    v = lib().compute_erida_gausslet_integral(C.byref(g), pts, _parse_tol(tol, syntax))
    _raise_if_failed(syntax)
    return v


def compute_sparse_erida_gausslet_integrals(gausslet_coeffs, grid, tol, form="fp64"):
    """Symmetry-reduced ERIDA matrix for Gausslet orbitals on a rotationally
    symmetric grid; returns a SparseERIDA."""
    return _compute_sparse("erida", gausslet_coeffs, grid, tol, form,
                           "compute_sparse_erida_gausslet_integrals(gausslet_coeffs, grid, tol)")


def load_sparse_eri_gausslet_integrals(filename):
    """Load a sparse ERI tensor from the HDF5 file that the reference CLI
    writes (cli/gli_eri_integrals.c:106-163): attributes grid_length and tol,
    datasets gausslet_coeffs, integral_values and four_indices.  Mirrors
    python/pymodule.c:1181-1331 (same checks, messages and exception types),
    reading the file with the library's own HDF5 reader (no libhdf5).
    Returns a SparseERI."""
    syntax = "load_sparse_eri_gausslet_integrals(filename)"
    if not isinstance(filename, str):
        raise SyntaxError(f"error parsing input; syntax: {syntax}")
    L = lib()
    f = L.gli_b200_h5_fopen(filename.encode(), 0, 0)
    if f < 0:
        raise RuntimeError(f"'H5Fopen' failed for file '{filename}'; syntax: {syntax}")
    try:
        gl = np.zeros(1, dtype=np.int64)
        if L.read_hdf5_attribute(f, b"grid_length", _abi.H5T_NATIVE_LLONG, gl.ctypes.data) < 0:
            raise RuntimeError(f"reading 'grid_length' attribute from HDF5 file '{filename}' failed")
        grid_length = int(gl[0])
        if grid_length <= 0:
            raise ValueError(f"read invalid negative 'grid_length' attribute from HDF5 file '{filename}'")
        tol = np.zeros(1)
        if L.read_hdf5_attribute(f, b"tol", _abi.H5T_NATIVE_DOUBLE, tol.ctypes.data) < 0:
            raise RuntimeError(f"reading 'tol' attribute from HDF5 file '{filename}' failed")
        dim = np.zeros(1, dtype=np.uint64)
        if L.get_hdf5_dataset_dims(f, b"gausslet_coeffs", dim.ctypes.data) < 0:
            raise RuntimeError(f"obtaining dimensions of Gausslet coefficients from HDF5 file '{filename}' failed")
        if int(dim[0]) % 2 != 1:
            raise RuntimeError(f"expecting an odd number of Gausslet coefficients in HDF5 file '{filename}'")
        coeffs = np.empty(int(dim[0]))
        if L.read_hdf5_dataset(f, b"gausslet_coeffs", _abi.H5T_NATIVE_DOUBLE, coeffs.ctypes.data) < 0:
            raise RuntimeError(f"reading Gausslet coefficients from HDF5 file '{filename}' failed")
        if L.get_hdf5_dataset_dims(f, b"integral_values", dim.ctypes.data) < 0:
            raise RuntimeError(f"obtaining dimensions of integral values from HDF5 file '{filename}' failed")
        values = np.empty(int(dim[0]))
        if L.read_hdf5_dataset(f, b"integral_values", _abi.H5T_NATIVE_DOUBLE, values.ctypes.data) < 0:
            raise RuntimeError(f"reading integral values from HDF5 file '{filename}' failed")
        indices = np.empty(int(dim[0]), dtype=np.int64)
        if L.read_hdf5_dataset(f, b"four_indices", _abi.H5T_NATIVE_LLONG, indices.ctypes.data) < 0:
            raise RuntimeError(f"reading four-indices from HDF5 file '{filename}' failed")
    finally:
        L.gli_b200_h5_fclose(f)
    e = -(grid_length - 1) // 2
    return SparseERI._make(coeffs, [(e, grid_length)] * 3, indices, values, float(tol[0]))


def save_sparse_eri_gausslet_integrals(eri, filename):
    """Write a SparseERI in the reference CLI's HDF5 layout
    (cli/gli_eri_integrals.c:106-163), so that the reference's loader, this
    module's loader and libhdf5 read it.  Extension: the reference module has
    no writer (its CLI writes the files).  The grid must be the rotationally
    symmetric cube that the file's single grid_length describes."""
    syntax = "save_sparse_eri_gausslet_integrals(eri, filename)"
    if not isinstance(eri, SparseERI) or not isinstance(filename, str):
        raise SyntaxError(f"error parsing input; syntax: {syntax}")
    spec = eri.grid
    n = spec[0][1]
    if any(tuple(a) != (-(n - 1) // 2, n) for a in spec):
        raise ValueError(f"the file format describes rotationally symmetric cubic grids only; syntax: {syntax}")
    L = lib()
    f = L.gli_b200_h5_fcreate(filename.encode(), 2, 0, 0)
    if f < 0:
        raise RuntimeError(f"'H5Fcreate' failed for '{filename}'")
    gl = np.array([n], dtype=np.int64)
    tol = np.array([eri.tol], dtype=np.float64)
    coeffs = np.ascontiguousarray(eri.gausslet_coeffs, dtype=np.float64)
    values = np.ascontiguousarray(eri.values, dtype=np.float64)
    indices = np.ascontiguousarray(eri.indices, dtype=np.int64)
    ok = (L.write_hdf5_scalar_attribute(f, b"grid_length", _abi.H5T_STD_I64LE, _abi.H5T_NATIVE_LLONG,
                                        gl.ctypes.data) >= 0 and
          L.write_hdf5_scalar_attribute(f, b"tol", _abi.H5T_IEEE_F64LE, _abi.H5T_NATIVE_DOUBLE, tol.ctypes.data) >= 0)
    for name, arr, store, mem in ((b"gausslet_coeffs", coeffs, _abi.H5T_IEEE_F64LE, _abi.H5T_NATIVE_DOUBLE),
                                  (b"integral_values", values, _abi.H5T_IEEE_F64LE, _abi.H5T_NATIVE_DOUBLE),
                                  (b"four_indices", indices, _abi.H5T_STD_I64LE, _abi.H5T_NATIVE_LLONG)):
        dims = np.array([arr.size], dtype=np.uint64)
        ok = ok and L.write_hdf5_dataset(f, name, 1, dims.ctypes.data, store, mem, arr.ctypes.data) >= 0
    closed = L.gli_b200_h5_fclose(f) >= 0
    if not (ok and closed):
        raise RuntimeError(f"writing sparse ERI file '{filename}' failed")
