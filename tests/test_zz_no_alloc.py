"""The allocation-free kinetic entry point, gli_b200_kinetic_matrix_noalloc.

Callers that must not allocate device memory when they need the kinetic matrix
-- a solver that reserved its device-memory budget before its first
iteration, code that runs while another framework captures a CUDA graph or
owns the allocator, a latency-critical loop -- use this entry point: it takes
the coefficients and the output matrix in device memory supplied by the caller
and keeps its only scratch (a per-axis table of at most 1024 entries) in a
static device array inside the library.

The test calls it through the C ABI twice in a row, on two different grids (so
the second call would expose anything the shared array kept from the first),
and compares each result with the allocating entry point
compute_kinetic_gausslet_integrals within the tolerance of the other parity
tests.  This file is collected last (its name sorts last), so a run that stops
at the first failure has already run every other test; it passes both alone in
a fresh process and after the rest of the suite.
"""
import ctypes as C

import numpy as np
import pytest

from _common import assert_parity, g10

pytestmark = pytest.mark.gpu


def test_kinetic_noalloc_matches_allocating_entry_point_twice():
    import torch

    import gausslectronitegrate_b200 as gli
    from gausslectronitegrate_b200 import _abi

    lib = gli.lib()
    if lib.gli_b200_device_count() == 0:
        pytest.fail("no CUDA device: the gpu tests need a B200")
    b = np.ascontiguousarray(g10())
    # the caller's own device buffers (the test is the caller; the entry point
    # under test allocates nothing)
    d_coeffs = torch.tensor(b, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    for grid in ([(-3, 7), (0, 4), (-2, 5)], [(-1, 3), (-2, 5), (-2, 4)]):
        n = grid[0][1] * grid[1][1] * grid[2][1]
        expected = gli.compute_kinetic_gausslet_integrals(b, grid)
        d_out = torch.full((n, n), float("nan"), dtype=torch.float64, device="cuda")
        rc = lib.gli_b200_kinetic_matrix_noalloc(C.c_void_p(d_coeffs.data_ptr()), b.size,
                                                 C.byref(gli._grid_struct(grid)), C.c_void_p(d_out.data_ptr()),
                                                 C.c_void_p(stream.cuda_stream))
        assert rc == 0, lib.gli_b200_last_error_message().decode()
        stream.synchronize()
        assert_parity(d_out.cpu().numpy(), expected, what=f"no-alloc kinetic matrix on {grid}")


def test_kinetic_noalloc_rejects_axes_beyond_its_table():
    import torch

    import gausslectronitegrate_b200 as gli

    lib = gli.lib()
    if lib.gli_b200_device_count() == 0:
        pytest.fail("no CUDA device: the gpu tests need a B200")
    b = np.ascontiguousarray(g10())
    d_coeffs = torch.tensor(b, dtype=torch.float64, device="cuda")
    d_out = torch.empty(1, dtype=torch.float64, device="cuda")
    grid = [(0, 1025), (0, 1), (0, 1)]  # largest axis one past the 1024-entry table
    rc = lib.gli_b200_kinetic_matrix_noalloc(C.c_void_p(d_coeffs.data_ptr()), b.size, C.byref(gli._grid_struct(grid)),
                                             C.c_void_p(d_out.data_ptr()), None)
    assert rc == 5  # GLI_ERR_LIMIT, before any kernel runs
    assert "1024" in lib.gli_b200_last_error_message().decode()


def test_kinetic_noalloc_rejects_host_pointers_before_launching():
    # a host array handed over as "device" memory would be written by the
    # kernels; the entry point checks both pointers and fails with
    # GLI_ERR_ARGUMENT before anything is queued
    import torch

    import gausslectronitegrate_b200 as gli

    lib = gli.lib()
    if lib.gli_b200_device_count() == 0:
        pytest.fail("no CUDA device: the gpu tests need a B200")
    b = np.ascontiguousarray(g10())
    d_coeffs = torch.tensor(b, dtype=torch.float64, device="cuda")
    grid = [(-1, 3), (-1, 3), (-1, 3)]
    pageable = np.zeros((27, 27))
    pinned = torch.zeros((27, 27), dtype=torch.float64).pin_memory()
    for what, coeffs, out in (("pageable matrix", d_coeffs.data_ptr(), pageable.ctypes.data),
                              ("pinned matrix", d_coeffs.data_ptr(), pinned.data_ptr()),
                              ("pageable coefficients", b.ctypes.data, None)):
        d_out = torch.empty((27, 27), dtype=torch.float64, device="cuda") if out is None else None
        launches = lib.gli_b200_launch_count()
        rc = lib.gli_b200_kinetic_matrix_noalloc(C.c_void_p(coeffs), b.size, C.byref(gli._grid_struct(grid)),
                                                 C.c_void_p(out if out is not None else d_out.data_ptr()), None)
        assert rc == 2, f"{what}: {lib.gli_b200_last_error_message().decode()}"  # GLI_ERR_ARGUMENT
        assert lib.gli_b200_launch_count() == launches, f"{what}: a kernel was launched"
    assert np.all(pageable == 0)
