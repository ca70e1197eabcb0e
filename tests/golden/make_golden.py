"""Generate the golden fixtures under tests/golden/ (run here, where the
reference tree exists; the fixtures are committed and travel, the reference
does not).

Three sources, each pinned to the reference:

1. The reference's own fixture generators ``test/test_{kinetic,nuclear,eri,erida}_integrals.py``
   (independent NumPy/SciPy re-implementations, ``test/gaussian_integrals.py``)
   are run with a stand-in ``h5py`` module that captures what they would
   write.  Every captured dataset is then located byte-for-byte inside the
   shipped ``test/data/*.hdf5`` file, which pins the regenerated arrays to the
   reference's committed fixtures without an HDF5 library.
2. The reference C core compiled by ``oracle/Makefile`` (``oracle/_ref``)
   supplies class lists and values at sizes the CPU finishes in seconds.
3. The notebook known answers (examples/*.ipynb outputs) are read from the
   notebooks' JSON.

Usage:  GLI_REFERENCE_DIR=<reference checkout> python tests/golden/make_golden.py
"""
import json
import os
import sys
import types

import numpy as np

REF = os.environ.get("GLI_REFERENCE_DIR", "")
HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


class _CaptureFile:
    """Stand-in for h5py.File: records attrs and datasets instead of writing."""
    captured = {}

    def __init__(self, name, mode="r"):
        self.name = os.path.basename(name)
        self.attrs = {}
        self.data = {}

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        _CaptureFile.captured[self.name] = (self.attrs, self.data)
        return False

    def __setitem__(self, key, value):
        self.data[key] = np.asarray(value)


def _run_generators():
    fake = types.ModuleType("h5py")
    fake.File = _CaptureFile
    sys.modules["h5py"] = fake
    sys.path.insert(0, os.path.join(REF, "gausslets"))
    sys.path.insert(0, os.path.join(REF, "test"))
    cwd = os.getcwd()
    os.chdir(os.path.join(REF, "test"))
    try:
        import test_kinetic_integrals
        import test_nuclear_integrals
        import test_erida_integrals
        import test_eri_integrals
        test_kinetic_integrals.kinetic_integrals_data()
        test_nuclear_integrals.nuclear_integrals_data()
        test_erida_integrals.erida_integrals_data()
        test_eri_integrals.eri_integrals_data()
    finally:
        os.chdir(cwd)
    return _CaptureFile.captured


def _pin_to_hdf5(name, arr, rtol=1e-12):
    """Locate the dataset inside the shipped HDF5 file using the regenerated
    array as a guide and return (byte offset, the file's exact values).  The
    shipped bytes become the golden values; the regenerated array only has to
    agree within rtol (SciPy/NumPy versions differ in the last bits)."""
    raw = open(os.path.join(REF, "test", "data", name), "rb").read()
    arr = np.ascontiguousarray(arr, dtype="<f8").ravel()
    nbytes = arr.size * 8
    scale = np.max(np.abs(arr))
    for off in range(0, len(raw) - nbytes + 1):
        first = np.frombuffer(raw, dtype="<f8", count=1, offset=off)[0]
        if not abs(first - arr[0]) <= rtol * scale:
            continue
        cand = np.frombuffer(raw, dtype="<f8", count=arr.size, offset=off)
        if np.all(np.abs(cand - arr) <= rtol * scale):
            return off, cand.copy()
    raise SystemExit(f"{name}: regenerated array not found inside the shipped fixture")


def _notebook_outputs(path):
    nb = json.load(open(path))
    out = []
    for cell in nb["cells"]:
        for o in cell.get("outputs", []):
            t = o.get("data", {}).get("text/plain") or o.get("text")
            if t:
                out.append("".join(t).strip())
    return out


def main():
    if not os.path.isdir(os.path.join(REF, "test")):
        raise SystemExit("set GLI_REFERENCE_DIR to a checkout of the reference")
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    cap = _run_generators()
    from gausslets import get_gausslet_g10_coeffs  # the reference's coefficient source
    b, _ = get_gausslet_g10_coeffs()
    b = np.asarray(b, dtype=np.float64)

    fx = {"g10": b}
    pins = {}
    for fname, key, short in [("test_kinetic_integrals.hdf5", "kgi", "kinetic"),
                              ("test_nuclear_integrals.hdf5", "ngi", "nuclear"),
                              ("test_erida_integrals.hdf5", "erida", "erida"),
                              ("test_eri_integrals.hdf5", "eri", "eri")]:
        attrs, data = cap[fname]
        arr = data[key]
        pins[short], shipped = _pin_to_hdf5(fname, arr)
        fx[f"fixture_{short}"] = shipped.reshape(arr.shape)
        fx[f"fixture_{short}_regen_maxdiff"] = np.float64(np.max(np.abs(shipped - arr.ravel())))
        if "tol" in attrs:
            fx[f"fixture_{short}_tol"] = np.float64(attrs["tol"])
        if short == "nuclear":
            fx["fixture_nuclear_pos"] = np.array([attrs[f"nuclear_pos_{i}"] for i in range(attrs["num_nuclei"])])
            fx["fixture_nuclear_charge"] = np.array([attrs[f"nuclear_charge_{i}"] for i in range(attrs["num_nuclei"])])
        assert np.array_equal(np.asarray(attrs["gausslet_coeffs"]), b)
    np.savez_compressed(os.path.join(HERE, "reference_fixtures.npz"), **fx)

    # --- reference C core, small workloads -----------------------------------
    from ref_binding import RefLib
    r = RefLib()
    core = {}
    for L in (3, 5, 33):
        g = [(-(L // 2), L)] * 3
        idx = r.enumerate("erida", g)
        core[f"erida_idx_{L}"] = idx
        for tol in (1e-16, 1e-10, 1e-5):
            core[f"erida_val_{L}_{tol:g}"] = r.sparse_values("erida", b, g, idx, tol)
    for L in (3, 5):
        g = [(-(L // 2), L)] * 3
        idx = r.enumerate("eri", g)
        core[f"eri_idx_{L}"] = idx
    g3 = [(-1, 3)] * 3
    for tol in (1e-16, 1e-10, 1e-5, 1e-3):
        core[f"eri_val_3_{tol:g}"] = r.sparse_values("eri", b, g3, core["eri_idx_3"], tol)
    core["eri_val_5_1e-05"] = r.sparse_values("eri", b, [(-2, 5)] * 3, core["eri_idx_5"], 1e-5)
    core["kinetic_3"] = r.kinetic_matrix(b, g3)
    core["kinetic_6x5x4"] = r.kinetic_matrix(b, [(-3, 6), (0, 5), (2, 4)])
    core["nuclear_3_z1_1e-5"] = r.nuclear_matrix(b, g3, [[0.0, 0.0, 0.0]], [1], 1e-5)
    core["nuclear_2x3x2_h2_1e-3"] = r.nuclear_matrix(b, [(-1, 2), (0, 3), (-1, 2)],
                                                     [[0.3, 0.1, -0.2], [-1.1, 0.6, 0.4]], [1, 2], 1e-3)
    np.savez_compressed(os.path.join(HERE, "reference_core.npz"), **core)

    # --- notebook known answers ----------------------------------------------
    nb = {}
    eri_out = _notebook_outputs(os.path.join(REF, "examples", "eri_integrals.ipynb"))
    erida_out = _notebook_outputs(os.path.join(REF, "examples", "erida_integrals.ipynb"))
    kin_out = _notebook_outputs(os.path.join(REF, "examples", "kinetic_integrals.ipynb"))
    nuc_out = _notebook_outputs(os.path.join(REF, "examples", "nuclear_integrals.ipynb"))
    nb["notebook_outputs"] = {"eri_integrals": eri_out, "erida_integrals": erida_out,
                              "kinetic_integrals": kin_out, "nuclear_integrals": nuc_out}
    nb["hdf5_byte_offsets"] = pins
    with open(os.path.join(HERE, "notebook_outputs.json"), "w") as f:
        json.dump(nb, f, indent=1)
    print("fixtures written; HDF5 pins at byte offsets", pins)


if __name__ == "__main__":
    main()
