"""Parity at the hot-path configurations' own sizes and tolerances, against
the reference C core's values committed in tests/golden/config_golden.npz (made
by tests/golden/make_config_golden.py; nothing here needs the reference tree).

* ERI on the 6x6x6 configuration's 7^3 stand-in, tol 1e-16, all 3,571,977
  classes evaluated on the GPU: the class list bit-exact (count and SHA-256),
  2,000 seeded classes plus the 200 largest against the reference at the
  parity bar, and three checksums over the whole list (src/eri_integrals.c:
  544-678).  The mixed form within 1e-8 Ha at 0.7 bohr (0.7e-8 grid units).
* ERIDA on the 128^3 configuration's 129^3 stand-in, tol 1e-16: every one of
  the 366,145 values (src/erida_integrals.c:429-542); the mixed form within
  1e-8 Ha at 0.3 bohr.
* The 6x6x6 projection onto 32 orthonormal columns (QR of default_rng(0)
  N(0, 1) entries) against the factored contraction of the reference's dense
  fill (src/eri_integrals.c:714-967, test/test_eri_integrals.c:426-455), at
  every representative of the tensor's 8-fold symmetry.
* Batched nuclear, the three largest (24^3) chains of the batch: 48 seeded
  pairs each against compute_nuclear_gausslet_integral
  (src/nuclear_integrals.c:31-126), tol 1e-8.
"""
import hashlib
import os

import numpy as np
import pytest

from _common import GOLDEN, assert_parity, g10

pytestmark = pytest.mark.gpu

ERI7_HA_PER_UNIT = 1.0 / 0.7    # 1/spacing: grid units -> Hartree
ERIDA129_HA_PER_UNIT = 1.0 / 0.3
MIXED_HA = 1e-8                 # the mixed form's bound against FP64


@pytest.fixture(scope="module")
def gli():
    import gausslectronitegrate_b200 as m
    if m.lib().gli_b200_device_count() == 0:
        pytest.fail("no CUDA device: the gpu tests need a B200")
    return m


@pytest.fixture(scope="module")
def golden():
    return np.load(os.path.join(GOLDEN, "config_golden.npz"))


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<i8").tobytes()).hexdigest()


@pytest.fixture(scope="module")
def eri7(gli):
    from gausslectronitegrate_b200 import workloads as W
    return {f: gli.compute_sparse_eri_gausslet_integrals(g10(), W.ERI6_SPARSE, 1e-16, form=f)
            for f in ("fp64", "mixed")}


def test_eri7_class_list(eri7, golden):
    s = eri7["fp64"]
    assert s.indices.size == int(golden["eri7_count"])
    assert _sha(s.indices) == str(golden["eri7_idx_sha256"])


def test_eri7_sample_tol16(eri7, golden):
    s = eri7["fp64"]
    pos = np.searchsorted(s.indices, golden["eri7_idx"])
    assert np.array_equal(s.indices[pos], golden["eri7_idx"])
    assert_parity(s.values[pos], golden["eri7_val"], what="ERI 7^3 tol 1e-16 (2,200 classes)")


def test_eri7_full_list_checksums(eri7, golden):
    # every class within |x - ref| <= 1e-12 |ref| + 1e-14 bounds each sum's
    # error by the same bar summed over the list
    v = eri7["fp64"].values
    w = np.random.default_rng(11).uniform(-1.0, 1.0, size=v.size)
    ref_sum, ref_abs, ref_w = golden["eri7_checksums"]
    budget = 1e-12 * ref_abs + 1e-14 * v.size
    for got, ref, what in ((v.sum(), ref_sum, "sum"), (np.abs(v).sum(), ref_abs, "sum |v|"),
                           ((w * v).sum(), ref_w, "weighted sum")):
        assert abs(got - ref) <= budget, f"ERI 7^3 {what}: {got!r} vs {ref!r}"


def test_eri7_mixed_form(eri7, golden):
    s = eri7["mixed"]
    pos = np.searchsorted(s.indices, golden["eri7_idx"])
    err_ha = np.max(np.abs(s.values[pos] - golden["eri7_val"])) * ERI7_HA_PER_UNIT
    assert err_ha <= MIXED_HA, f"mixed ERI 7^3 against the reference: {err_ha:.3e} Ha"
    full_ha = np.max(np.abs(s.values - eri7["fp64"].values)) * ERI7_HA_PER_UNIT
    assert full_ha <= MIXED_HA, f"mixed ERI 7^3 against the FP64 form (all classes): {full_ha:.3e} Ha"


@pytest.mark.parametrize("form", ["fp64", "mixed"])
def test_erida129_full_list_tol16(gli, golden, form):
    from gausslectronitegrate_b200 import workloads as W
    s = gli.compute_sparse_erida_gausslet_integrals(g10(), W.sym_grid(129), 1e-16, form=form)
    assert _sha(s.indices) == str(golden["erida129_idx_sha256"])
    ref = golden["erida129_val"]
    if form == "fp64":
        assert_parity(s.values, ref, what="ERIDA 129^3 tol 1e-16 (all 366,145 classes)")
    else:
        err_ha = np.max(np.abs(s.values - ref)) * ERIDA129_HA_PER_UNIT
        assert err_ha <= MIXED_HA, f"mixed ERIDA 129^3: {err_ha:.3e} Ha"


def test_eri6_projection(eri7, golden):
    from gausslectronitegrate_b200 import workloads as W
    E = eri7["fp64"].project(W.eri6_sparse_basis())
    p, q, r, s = W.unique_projection_entries(W.ERI6_STATES)
    ref = golden["eri6_proj_unique"]
    got = E[p, q, r, s]
    # the contraction sums 216^4 entries in a different order than the
    # factored reference: the bar is relative to the largest projected entry
    scale = np.max(np.abs(ref))
    err = np.max(np.abs(got - ref))
    assert err <= 1e-12 * scale, f"projection: max |d| {err:.3e} against max |E| {scale:.3e}"
    # and the projected tensor keeps the 8-fold symmetry of real orbitals
    assert np.max(np.abs(E - E.transpose(1, 0, 2, 3))) <= 1e-13 * scale
    assert np.max(np.abs(E - E.transpose(2, 3, 0, 1))) <= 1e-13 * scale


def test_nuclear_batch_24_pairs(gli, golden):
    from gausslectronitegrate_b200 import workloads as W
    grids, pos, q = W.nuclear_batch_config()
    inst = golden["nuc24_inst"]
    ids = sorted(set(int(k) for k in inst))
    outs = gli.compute_nuclear_gausslet_integrals_batch(g10(), [grids[k] for k in ids], [pos[k] for k in ids],
                                                        [q[k] for k in ids], 1e-8)
    by_id = dict(zip(ids, outs))
    got = np.array([by_id[int(k)][i, j] for k, i, j in zip(inst, golden["nuc24_i"], golden["nuc24_j"])])
    assert_parity(got, golden["nuc24_val"], what="nuclear 24^3 pair sample (3 chains x 48 pairs)")


def test_eri7_pinned_host_buffers(gli, eri7):
    # page-locked host arrays: the C call copies straight to and from them and
    # evaluates the 3.57 million classes in overlapped ranges, each its own plan
    import ctypes as C

    import torch

    from gausslectronitegrate_b200 import _abi
    from gausslectronitegrate_b200 import workloads as W
    s = eri7["fp64"]
    idx = torch.from_numpy(s.indices).pin_memory()
    out = torch.full((s.indices.size,), float("nan"), dtype=torch.float64).pin_memory()
    gd, keep = gli._parse_coeffs(np.ascontiguousarray(g10()), "")
    for _ in range(2):  # the second call replays the ranges' captured graphs
        rc = gli.lib().gli_b200_sparse_values(_abi.GLI_KIND_ERI, C.byref(gd), C.byref(gli._grid_struct(W.ERI6_SPARSE)),
                                              C.cast(idx.data_ptr(), _abi.lptr), s.indices.size, 1e-16,
                                              _abi.GLI_FORM_FP64, C.cast(out.data_ptr(), _abi.dptr))
        assert rc == 0, gli.lib().gli_b200_last_error_message().decode()
        assert_parity(out.numpy(), s.values, what="ERI 7^3 through pinned host buffers")
