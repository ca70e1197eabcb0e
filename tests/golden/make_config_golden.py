"""Generate the full-size parity fixtures of the hot-path configurations
(tests/golden/config_golden.npz) from the reference C core compiled by
oracle/Makefile (oracle/_ref/libgli_ref.so).  Run once on a CPU box; the
fixture is committed and the GPU tests read it, so nothing at test time needs
the reference tree.

    GLI_REFERENCE_DIR=<reference checkout> make -C oracle ref
    OMP_NUM_THREADS=<cores> python tests/golden/make_config_golden.py [--cache DIR]

Contents (tol 1e-16 unless noted; values in grid units):

* ERI on the 6x6x6 configuration's odd stand-in 7^3 grid (-3, 7)^3, all
  3,571,977 classes evaluated by compute_sparse_eri_gausslet_integrals
  (src/eri_integrals.c:544-678):
  - eri7_idx / eri7_val: 2,000 classes drawn with default_rng(7) plus the 200
    of largest |value| (sorted, unique);
  - eri7_count, eri7_idx_sha256: size and SHA-256 of the whole class list;
  - eri7_checksums: sum, sum |v| and sum w v of all values with w drawn from
    default_rng(11) (uniform in [-1, 1)): a full-list check whose error
    budget is the sum of the per-class tolerances.
* ERIDA on the 128^3 configuration's odd stand-in 129^3 grid (-64, 129)^3:
  erida129_val, all 366,145 values in class order (src/erida_integrals.c:
  429-542), with erida129_idx_sha256 of the class list.
* The 6x6x6 projection: eri6_proj_unique, the projected tensor
  E[p,q,r,s] = sum_ijkl B[i,p] B[j,q] B[k,r] B[l,s] V[i,j,k,l] over the
  216^4 entries of the dense 6^3 grid (-3, 6)^3 that the reference's
  fill_dense_eri_tensor (src/eri_integrals.c:850-967) expands from the 7^3
  classes, B = workloads.eri6_dense_basis(); contracted axis by axis (the
  factored form of test/test_eri_integrals.c:426-455, whose direct form
  project_sparse_eri_gausslet_integrals is O(N^4 M^4)).  Stored at the
  representatives of workloads.unique_projection_entries(32).
* Batched nuclear, the largest instances: the first three 24^3 chains of
  workloads.nuclear_batch_config(), 48 seeded pairs each (16 coincident, 16
  within two points per axis, 16 uniform), compute_nuclear_gausslet_integral
  (src/nuclear_integrals.c:31-126) at tol 1e-8: nuc24_inst, nuc24_i, nuc24_j,
  nuc24_val.
"""
import argparse
import hashlib
import multiprocessing as mp
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "oracle"))

from gausslectronitegrate_b200 import workloads as W  # noqa: E402

OUT = os.path.join(HERE, "config_golden.npz")


def g10():
    return np.load(os.path.join(HERE, "reference_fixtures.npz"))["g10"]


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<i8").tobytes()).hexdigest()


def log(msg):
    print(f"[golden] {msg}", file=sys.stderr, flush=True)


def cached(cache, name, fn):
    path = os.path.join(cache, name + ".npy") if cache else None
    if path and os.path.exists(path):
        return np.load(path)
    t0 = time.time()
    a = fn()
    log(f"{name}: {time.time() - t0:.1f} s")
    if path:
        np.save(path, a)
    return a


def eri7_part(r, b, cache, out):
    g = W.ERI6_SPARSE
    idx = cached(cache, "eri7_idx", lambda: r.enumerate("eri", g))
    val = cached(cache, "eri7_val", lambda: r.sparse_values("eri", b, g, idx, 1e-16))
    pick = np.random.default_rng(7).choice(idx.size, size=2000, replace=False)
    big = np.argsort(-np.abs(val))[:200]
    sel = np.unique(np.concatenate([pick, big]))
    w = np.random.default_rng(11).uniform(-1.0, 1.0, size=idx.size)
    out.update(eri7_idx=idx[sel], eri7_val=val[sel], eri7_count=np.int64(idx.size), eri7_idx_sha256=sha(idx),
               eri7_checksums=np.array([val.sum(), np.abs(val).sum(), (w * val).sum()]))
    return idx, val


def erida129_part(r, b, cache, out):
    g = W.sym_grid(129)
    idx = cached(cache, "erida129_idx", lambda: r.enumerate("erida", g))
    val = cached(cache, "erida129_val", lambda: r.sparse_values("erida", b, g, idx, 1e-16))
    out.update(erida129_val=val, erida129_idx_sha256=sha(idx))


def projection_part(r, idx, val, cache, out):
    def run():
        t0 = time.time()
        V = r.fill_dense("eri", W.ERI6_SPARSE, idx, val, W.ERI6_DENSE)  # 216^4 doubles, 17.4 GB
        log(f"fill_dense_eri_tensor (216^4): {time.time() - t0:.1f} s")
        q = W.eri6_dense_basis()
        X = np.tensordot(V, q, axes=([3], [0]))  # (i, j, k, s)
        del V
        X = np.tensordot(X, q, axes=([2], [0]))  # (i, j, s, r)
        X = np.tensordot(X, q, axes=([1], [0]))  # (i, s, r, q)
        X = np.tensordot(X, q, axes=([0], [0]))  # (s, r, q, p)
        return np.ascontiguousarray(X.transpose(3, 2, 1, 0))
    E = cached(cache, "eri6_proj", run)
    p, q, r_, s = W.unique_projection_entries(W.ERI6_STATES)
    out.update(eri6_proj_unique=E[p, q, r_, s])
    # the 8-fold symmetry of the reference's own tensor, checked before it is relied on
    assert np.allclose(E, E.transpose(1, 0, 2, 3), rtol=0, atol=1e-12 * np.abs(E).max())
    assert np.allclose(E, E.transpose(2, 3, 0, 1), rtol=0, atol=1e-12 * np.abs(E).max())


def _nuc_one(job):
    from ref_binding import RefLib
    b, pi, pj, pos, q = job
    return RefLib().nuclear_single(b, [pi, pj], pos, q, 1e-8)


def nuclear_part(b, out):
    grids, pos, q = W.nuclear_batch_config()
    big = [k for k, g in enumerate(grids) if g[0][1] == 24][:3]
    rng = np.random.default_rng(5)
    jobs, inst, ii, jj = [], [], [], []
    for k in big:
        g = grids[k]
        lo = np.array([a[0] for a in g])
        n = np.array([a[1] for a in g])
        for kind in range(3):
            for _ in range(16):
                i = lo + rng.integers(0, n)
                if kind == 0:
                    j = i.copy()
                elif kind == 1:
                    j = np.clip(i + rng.integers(-2, 3, size=3), lo, lo + n - 1)
                else:
                    j = lo + rng.integers(0, n)
                lin_i = int(((i[0] - lo[0]) * n[1] + (i[1] - lo[1])) * n[2] + (i[2] - lo[2]))
                lin_j = int(((j[0] - lo[0]) * n[1] + (j[1] - lo[1])) * n[2] + (j[2] - lo[2]))
                jobs.append((b, [int(x) for x in i], [int(x) for x in j], pos[k], q[k]))
                inst.append(k)
                ii.append(lin_i)
                jj.append(lin_j)
    t0 = time.time()
    with mp.get_context("spawn").Pool(os.cpu_count()) as pool:
        vals = pool.map(_nuc_one, jobs)
    log(f"nuclear 24^3 pairs: {len(jobs)} in {time.time() - t0:.1f} s")
    out.update(nuc24_inst=np.array(inst, dtype=np.int64), nuc24_i=np.array(ii, dtype=np.int64),
               nuc24_j=np.array(jj, dtype=np.int64), nuc24_val=np.array(vals))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--cache", default=None, help="directory for intermediate arrays (reused when present)")
    args = ap.parse_args()
    if args.cache:
        os.makedirs(args.cache, exist_ok=True)
    from ref_binding import RefLib
    r = RefLib()
    b = g10()
    out = {}
    nuclear_part(b, out)
    idx, val = eri7_part(r, b, args.cache, out)
    erida129_part(r, b, args.cache, out)
    projection_part(r, idx, val, args.cache, out)
    np.savez_compressed(OUT, **out)
    log(f"written {OUT} ({os.path.getsize(OUT) / 1e6:.1f} MB)")


if __name__ == "__main__":
    main()
