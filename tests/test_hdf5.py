"""The sparse-ERI HDF5 format without libhdf5 (h5file.cu, include/hdf5.h,
include/hdf5_util.h; reference cli/gli_eri_integrals.c:106-163 writes it,
python/pymodule.c:1181-1331 loads it).

CPU tests: the library's reader against the reference's own files
(tests/golden/hdf5/: the CLI's 3^3 result examples/eri_3x3x3.hdf5, the CLI's
coefficient file, and the four test fixtures test/data/*.hdf5 that h5py wrote),
and the writer against the CLI's file: written from the same arrays, the file
comes out identical byte for byte.
"""
import ctypes as C
import os

import numpy as np
import pytest

from _common import GOLDEN, core, g10

H5 = os.path.join(GOLDEN, "hdf5")


@pytest.fixture(scope="module")
def gli():
    import gausslectronitegrate_b200 as m
    return m


def _dataset(L, f, name, mem, dtype):
    nd = C.c_int()
    assert L.get_hdf5_dataset_ndims(f, name.encode(), C.byref(nd)) == 0
    dims = np.zeros(max(nd.value, 1), dtype=np.uint64)
    assert L.get_hdf5_dataset_dims(f, name.encode(), dims.ctypes.data) == 0
    out = np.empty(tuple(int(x) for x in dims[:nd.value]), dtype=dtype)
    assert L.read_hdf5_dataset(f, name.encode(), mem, out.ctypes.data) == 0
    return out


def test_load_cli_result_file(gli):
    s = gli.load_sparse_eri_gausslet_integrals(os.path.join(H5, "eri_3x3x3.hdf5"))
    assert s.grid == ((-1, 3), (-1, 3), (-1, 3))
    assert s.tol == 1e-16
    assert np.array_equal(s.gausslet_coeffs, g10())
    assert np.array_equal(s.indices, core()["eri_idx_3"])
    # the CLI ran the reference core: its values, within the last bits of another build
    ref = core()["eri_val_3_1e-16"]
    assert np.max(np.abs(s.values - ref)) <= 1e-15 * np.max(np.abs(ref))
    # the value at byte 11336: ERI of the origin with itself (examples/eri_integrals.ipynb:59)
    raw = open(os.path.join(H5, "eri_3x3x3.hdf5"), "rb").read()
    assert np.frombuffer(raw, "<f8", count=1, offset=11336)[0] in s.values


def test_writer_reproduces_the_cli_file(gli, tmp_path):
    src = os.path.join(H5, "eri_3x3x3.hdf5")
    s = gli.load_sparse_eri_gausslet_integrals(src)
    out = str(tmp_path / "eri.hdf5")
    gli.save_sparse_eri_gausslet_integrals(s, out)
    assert open(out, "rb").read() == open(src, "rb").read()
    back = gli.load_sparse_eri_gausslet_integrals(out)
    assert np.array_equal(back.values, s.values) and np.array_equal(back.indices, s.indices)


def test_read_cli_coefficient_attribute(gli):
    L = gli.lib()
    f = L.gli_b200_h5_fopen(os.path.join(H5, "gli_eri_integrals_gausslet_data.hdf5").encode(), 0, 0)
    assert f >= 0
    dims = np.zeros(1, dtype=np.uint64)
    assert L.get_hdf5_attribute_dims(f, b"gausslet_coeffs", dims.ctypes.data) == 0
    c = np.empty(int(dims[0]))
    assert L.read_hdf5_attribute(f, b"gausslet_coeffs", gli._abi.H5T_NATIVE_DOUBLE, c.ctypes.data) == 0
    assert L.gli_b200_h5_fclose(f) == 0
    assert np.array_equal(c, g10())


@pytest.mark.parametrize("name,key", [("test_kinetic_integrals.hdf5", "kgi"), ("test_nuclear_integrals.hdf5", "ngi"),
                                      ("test_eri_integrals.hdf5", "eri"), ("test_erida_integrals.hdf5", "erida")])
def test_read_reference_fixtures(gli, name, key):
    # files that h5py wrote (another allocation layout, 2-D and 4-D datasets,
    # several attributes): the arrays equal those pinned in reference_fixtures.npz
    L = gli.lib()
    f = L.gli_b200_h5_fopen(os.path.join(H5, name).encode(), 0, 0)
    assert f >= 0
    arr = _dataset(L, f, key, gli._abi.H5T_NATIVE_DOUBLE, np.float64)
    short = {"kgi": "kinetic", "ngi": "nuclear", "eri": "eri", "erida": "erida"}[key]
    fx = np.load(os.path.join(GOLDEN, "reference_fixtures.npz"))
    assert np.array_equal(arr.ravel(), fx[f"fixture_{short}"].ravel())
    c = np.empty(135)
    assert L.read_hdf5_attribute(f, b"gausslet_coeffs", gli._abi.H5T_NATIVE_DOUBLE, c.ctypes.data) == 0
    assert np.array_equal(c, g10())
    assert L.gli_b200_h5_fclose(f) == 0


def test_errors(gli, tmp_path):
    L = gli.lib()
    missing = str(tmp_path / "none.hdf5")
    with pytest.raises(RuntimeError, match="H5Fopen"):
        gli.load_sparse_eri_gausslet_integrals(missing)
    bad = tmp_path / "bad.hdf5"
    bad.write_bytes(b"not an hdf5 file" * 16)
    assert L.gli_b200_h5_fopen(str(bad).encode(), 0, 0) < 0
    f = L.gli_b200_h5_fopen(os.path.join(H5, "eri_3x3x3.hdf5").encode(), 0, 0)
    x = np.zeros(4)
    assert L.read_hdf5_dataset(f, b"no_such_dataset", gli._abi.H5T_NATIVE_DOUBLE, x.ctypes.data) < 0
    assert L.read_hdf5_attribute(f, b"no_such_attribute", gli._abi.H5T_NATIVE_DOUBLE, x.ctypes.data) < 0
    assert L.gli_b200_h5_fclose(f) == 0
    assert L.gli_b200_h5_fclose(f) < 0  # closed already
