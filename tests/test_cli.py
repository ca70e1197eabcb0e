"""The reference's CLI drivers (cli/gli_eri_integrals.c,
cli/gli_eri_symmetry_reduction.c, cli/gli_erida_symmetry_reduction.c)
compiled unchanged against include/ and linked to libgli_b200.so by
``make -C oracle cli`` (output oracle/_ref/cli/, built where the reference tree
exists and carried with the repository).

CPU: the binaries link and run their argument checks and file errors.  GPU:
gli_eri_integrals on the reference's own coefficient file reproduces the
reference's 3^3 result file (examples/eri_3x3x3.hdf5) -- every metadata byte
identical, the values within the parity bar -- and the symmetry-reduction
tables print the reference's class counts.
"""
import os
import re
import subprocess

import numpy as np
import pytest

from _common import GOLDEN, assert_parity, core

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(REPO, "oracle", "_ref", "cli")
H5 = os.path.join(GOLDEN, "hdf5")
HAVE = all(os.path.exists(os.path.join(CLI, n)) for n in
           ("gli_eri_integrals", "gli_eri_symmetry_reduction", "gli_erida_symmetry_reduction"))
needs_cli = pytest.mark.skipif(not HAVE, reason="CLI drivers not built (make -C oracle cli)")


def _run(*args, timeout=600):
    return subprocess.run([os.path.join(CLI, args[0]), *args[1:]], capture_output=True, text=True, timeout=timeout)


@needs_cli
def test_cli_argument_and_file_errors(tmp_path):
    r = _run("gli_eri_symmetry_reduction")
    assert r.returncode == 255 and "expecting one input parameter" in r.stderr
    r = _run("gli_erida_symmetry_reduction", "4")
    assert r.returncode == 255 and "positive odd integer" in r.stderr
    r = _run("gli_eri_integrals", os.path.join(H5, "gli_eri_integrals_gausslet_data.hdf5"), "3", "-1", "x.hdf5")
    assert r.returncode == 255 and "'tol' cannot be negative" in r.stderr
    r = _run("gli_eri_integrals", str(tmp_path / "missing.hdf5"), "3", "1e-16", str(tmp_path / "out.hdf5"))
    assert r.returncode == 255 and "'H5Fopen' of Gausslet data file" in r.stderr


@needs_cli
@pytest.mark.gpu
def test_cli_eri_integrals_reproduces_reference_file(tmp_path):
    out = str(tmp_path / "eri_3x3x3.hdf5")
    r = _run("gli_eri_integrals", os.path.join(H5, "gli_eri_integrals_gausslet_data.hdf5"), "3", "1e-16", out)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "number of indices" in r.stdout and "1027" in r.stdout
    got = open(out, "rb").read()
    ref = open(os.path.join(H5, "eri_3x3x3.hdf5"), "rb").read()
    assert len(got) == len(ref)
    # the integral values occupy bytes 3128 .. 11344 (layout message of
    # integral_values in the reference file); everything else is identical
    lo, hi = 3128, 3128 + 8 * 1027
    assert got[:lo] == ref[:lo] and got[hi:] == ref[hi:]
    vals = np.frombuffer(got[lo:hi], "<f8")
    assert_parity(vals, core()["eri_val_3_1e-16"], what="CLI 3^3 values")
    import gausslectronitegrate_b200 as gli
    s = gli.load_sparse_eri_gausslet_integrals(out)
    assert np.array_equal(s.values, vals) and np.array_equal(s.indices, core()["eri_idx_3"])


def _counts(text):
    return [int(m.group(1)) for m in re.finditer(r"^\s*\d+ x \d+ x \d+\s+\d+\s+\d+\s+(\d+)", text, re.M)]


@needs_cli
@pytest.mark.gpu
def test_cli_symmetry_reduction_tables():
    r = _run("gli_eri_symmetry_reduction", "5")
    assert r.returncode == 0, r.stderr
    assert _counts(r.stdout) == [1, 1027, 138187]  # 1^3, 3^3 (examples/eri_integrals.ipynb:170), 5^3
    r = _run("gli_erida_symmetry_reduction", "9")
    assert r.returncode == 0, r.stderr
    assert _counts(r.stdout) == [L * (L + 1) * (L + 2) // 6 for L in (1, 3, 5, 7, 9)]
