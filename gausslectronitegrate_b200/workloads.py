"""Synthetic inputs of the hot-path configurations, shared by bench.py, the
golden-fixture script and the tests (one definition of each workload).

No dataset is involved anywhere: every input is the G10 gausslet coefficient
set, a grid and seeded random geometry or bases.
"""
import numpy as np


def sym_grid(L):
    """The rotationally symmetric odd grid (-(L // 2), L)^3 that the
    symmetry-reduced ERI / ERIDA paths accept (python/pymodule.c:1149-1166)."""
    return [(-(L // 2), L)] * 3


def h_chain_batch(rng, count, edge_lo, edge_hi, spacing):
    """Batch of linear H_n chains (the batched-nuclear configuration): n
    uniform in 2..8, bond lengths uniform in 1.0-3.0 bohr, every nucleus
    jittered by N(0, 0.1) bohr per coordinate, chain along x centred on the
    origin; grid edge uniform in edge_lo..edge_hi points, centred, at `spacing`
    bohr.  Returns (grids, positions in grid units = bohr / spacing, charges)."""
    grids, positions, charges = [], [], []
    for _ in range(count):
        n = int(rng.integers(2, 9))
        bonds = rng.uniform(1.0, 3.0, size=n - 1)
        x = np.concatenate([[0.0], np.cumsum(bonds)])
        x -= x.mean()
        pos = np.stack([x, np.zeros(n), np.zeros(n)], axis=1) + rng.normal(0.0, 0.1, size=(n, 3))
        edge = int(rng.integers(edge_lo, edge_hi + 1))
        grids.append([(-(edge // 2), edge)] * 3)
        positions.append(pos / spacing)
        charges.append([1] * n)
    return grids, positions, charges


def nuclear_batch_config(count=256):
    """The batched-nuclear configuration: `count` H_n chains on 8^3..24^3 grids
    at 0.5 bohr, seed 2024."""
    return h_chain_batch(np.random.default_rng(2024), count, 8, 24, 0.5)


# The 6x6x6 ERI configuration: its classes live on the odd stand-in 7^3 grid
# (-3, 7)^3; the projection runs over the 216 points of the dense 6^3 grid
# (-3, 6)^3 inside it onto 32 orthonormal columns.
ERI6_SPARSE = sym_grid(7)
ERI6_DENSE = [(-3, 6)] * 3
ERI6_STATES = 32


def eri6_dense_basis():
    """Orthonormal 216 x 32 basis: Q of the QR factorisation of a 216 x 32
    matrix of N(0, 1) entries drawn from numpy.random.default_rng(0), rows in
    the x-major order of the dense 6^3 grid."""
    rng = np.random.default_rng(0)
    a = rng.standard_normal((216, ERI6_STATES))
    q, _ = np.linalg.qr(a)
    return np.ascontiguousarray(q)


def dense_rows_in_sparse(sparse, dense):
    """Linear (x-major) index in the `sparse` grid of every point of `dense`
    (x-major order)."""
    xs = [np.arange(d[0], d[0] + d[1]) - s[0] for s, d in zip(sparse, dense)]
    X, Y, Z = np.meshgrid(*xs, indexing="ij")
    return ((X * sparse[1][1] + Y) * sparse[2][1] + Z).ravel()


def eri6_sparse_basis():
    """The dense basis zero-padded to the 343 points of the sparse 7^3 grid:
    projecting the 7^3 classes with it contracts exactly the 216^4 entries of
    the dense 6^3 grid (the other rows are zero)."""
    q = eri6_dense_basis()
    full = np.zeros((7 ** 3, ERI6_STATES))
    full[dense_rows_in_sparse(ERI6_SPARSE, ERI6_DENSE)] = q
    return full


def unique_projection_entries(m):
    """Index tuples (p, q, r, s) with p >= q, r >= s and (p, q) >= (r, s): one
    representative of each orbit of the 8-fold index symmetry of a projected
    ERI tensor with real orbitals (chemists' order)."""
    p, q = np.tril_indices(m)
    pq = p * m + q
    a, b = np.tril_indices(pq.size)
    return p[a], q[a], p[b], q[b]
