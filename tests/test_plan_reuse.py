"""Repeated evaluations of one class list in device memory: the ERI 7^3
stand-in of the 6x6x6 configuration (364 axis keys: the exact plan, then CUDA
graph replays sized by it) and ERIDA lists (bounded plans, captured at once).
A replay reuses the plan of the one before it while the list is unchanged;
replays of the product form decode and check each class in the gather instead
of marking the list.  The caller may rewrite the list in place between
calls: a permutation of the same classes reuses the plan, classes outside it
make the library evaluate again with a new plan, and an index outside the
tensor is still reported.  Every result is checked against one evaluation of
the whole list (the parity bar of the reference's tests)."""
import ctypes as C

import numpy as np
import pytest

from _common import assert_parity, g10

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gli():
    import gausslectronitegrate_b200 as m
    if m.lib().gli_b200_device_count() == 0:
        pytest.fail("no CUDA device: the gpu tests need a B200")
    return m


CASES = {
    # (kind, grid): ERI 7^3 (sized plan, product form, pair-descriptor decode),
    # ERIDA 129^3 (bounded plan, product form), ERIDA 33^3 (bounded plan,
    # per-class stage C: the replays mark and compare with the saved plan)
    "eri7": (1, lambda W: W.ERI6_SPARSE),
    "erida129": (0, lambda W: W.sym_grid(129)),
    "erida33": (0, lambda W: W.sym_grid(33)),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_replays_follow_the_list_in_device_memory(gli, case):
    import torch

    from gausslectronitegrate_b200 import _abi
    from gausslectronitegrate_b200 import workloads as W
    kind, grid_of = CASES[case]
    grid = grid_of(W)
    compute = gli.compute_sparse_eri_gausslet_integrals if kind else gli.compute_sparse_erida_gausslet_integrals
    full = compute(g10(), grid, 1e-16)
    m = full.indices.size // 2
    first, second = full.indices[:m], full.indices[m:2 * m]
    ref_first, ref_second = full.values[:m], full.values[m:2 * m]
    b = np.ascontiguousarray(g10())
    gs = gli._grid_struct(grid)
    d_idx = torch.from_numpy(first.copy()).cuda()
    d_out = torch.empty(m, dtype=torch.float64, device="cuda")
    L = gli.lib()

    def run():
        d_out.fill_(float("nan"))
        torch.cuda.synchronize()
        rc = L.gli_b200_sparse_values_dev(kind, b.ctypes.data_as(_abi.dptr), b.size, C.byref(gs),
                                          C.c_void_p(d_idx.data_ptr()), m, 1e-16, _abi.GLI_FORM_FP64,
                                          C.c_void_p(d_out.data_ptr()), None)
        torch.cuda.synchronize()
        return rc

    # exact plan and capture; the first replay plans; later replays reuse it
    for k in range(4):
        assert run() == 0, L.gli_b200_last_error_message().decode()
        assert_parity(d_out.cpu().numpy(), ref_first, what=f"first half, call {k}")
    # the same classes in another order: every class lies in the reused plan
    perm = np.random.default_rng(5).permutation(m)
    d_idx.copy_(torch.from_numpy(first[perm]))
    for k in range(2):
        assert run() == 0, L.gli_b200_last_error_message().decode()
        assert_parity(d_out.cpu().numpy(), ref_first[perm], what=f"permuted first half, call {k}")
    # other classes: keys and pairs outside the plan
    d_idx.copy_(torch.from_numpy(second))
    for k in range(3):
        assert run() == 0, L.gli_b200_last_error_message().decode()
        assert_parity(d_out.cpu().numpy(), ref_second, what=f"second half, call {k}")
    # an index outside the tensor, then the list repaired
    bad = m // 3
    d_idx[bad] = -1
    assert run() != 0
    assert "outside" in L.gli_b200_last_error_message().decode()
    d_idx[bad] = int(second[bad])
    assert run() == 0, L.gli_b200_last_error_message().decode()
    assert_parity(d_out.cpu().numpy(), ref_second, what="second half after the bad index")


def test_stream_ordered_evaluations(gli):
    # gli_b200_sparse_values_dev_async: several evaluations queued on one
    # stream, their status read by one wait; a list rewritten in place between
    # them (so that a queued replay overflows its plan) is evaluated again in
    # the wait; an index outside the tensor is reported by the wait
    import torch

    from gausslectronitegrate_b200 import _abi
    from gausslectronitegrate_b200 import workloads as W
    full = gli.compute_sparse_eri_gausslet_integrals(g10(), W.ERI6_SPARSE, 1e-16)
    m = full.indices.size // 3
    parts = [full.indices[k * m:(k + 1) * m] for k in range(3)]
    refs = [full.values[k * m:(k + 1) * m] for k in range(3)]
    b = np.ascontiguousarray(g10())
    gs = gli._grid_struct(W.ERI6_SPARSE)
    L = gli.lib()
    stream = torch.cuda.Stream()
    d_idx = torch.from_numpy(parts[0].copy()).cuda()
    outs = [torch.full((m,), float("nan"), dtype=torch.float64, device="cuda") for _ in range(2)]

    def queue(out):
        t = _abi.glong()
        rc = L.gli_b200_sparse_values_dev_async(_abi.GLI_KIND_ERI, b.ctypes.data_as(_abi.dptr), b.size, C.byref(gs),
                                                C.c_void_p(d_idx.data_ptr()), m, 1e-16, _abi.GLI_FORM_FP64,
                                                C.c_void_p(out.data_ptr()), C.c_void_p(stream.cuda_stream),
                                                C.byref(t))
        assert rc == 0, L.gli_b200_last_error_message().decode()
        return t.value

    # per output buffer, the first call plans exactly (and waits once); the
    # next ones replay its sized graph, the first replay planning again and the
    # later ones reusing that plan
    tickets = [queue(outs[0]) for _ in range(3)] + [queue(outs[1]) for _ in range(3)]
    assert tickets == sorted(tickets)
    assert L.gli_b200_sparse_values_wait(tickets[-1]) == 0, L.gli_b200_last_error_message().decode()
    for o in outs[:2]:
        assert_parity(o.cpu().numpy(), refs[0], what="queued evaluations of the first third")
    # a replay queued after an in-place rewrite on the same stream
    with torch.cuda.stream(stream):
        d_idx.copy_(torch.from_numpy(parts[1]).to("cuda", non_blocking=False))
    t = queue(outs[0])
    assert L.gli_b200_sparse_values_wait(t) == 0, L.gli_b200_last_error_message().decode()
    assert_parity(outs[0].cpu().numpy(), refs[1], what="queued evaluation after the rewrite")
    # an unknown ticket, then an index outside the tensor
    assert L.gli_b200_sparse_values_wait(t) != 0
    with torch.cuda.stream(stream):
        d_idx.copy_(torch.from_numpy(parts[2]).cuda())
        d_idx[7] = -5
    t = queue(outs[1])
    assert L.gli_b200_sparse_values_wait(t) != 0
    assert "outside" in L.gli_b200_last_error_message().decode()
    with torch.cuda.stream(stream):
        d_idx[7] = int(parts[2][7])
    t = queue(outs[1])
    assert L.gli_b200_sparse_values_wait(t) == 0, L.gli_b200_last_error_message().decode()
    assert_parity(outs[1].cpu().numpy(), refs[2], what="queued evaluation after the repair")


def test_pinned_host_lists_pipeline(gli):
    # gli_b200_sparse_values with page-locked host arrays: after the exact call
    # and one replay, calls stream the list in ranges, gathering each as it
    # arrives behind the stages of the kept plan; a list rewritten in place
    # with classes outside that plan is evaluated again whole
    import torch

    from gausslectronitegrate_b200 import _abi
    from gausslectronitegrate_b200 import workloads as W
    full = gli.compute_sparse_eri_gausslet_integrals(g10(), W.ERI6_SPARSE, 1e-16)
    m = full.indices.size // 2
    halves = [full.indices[:m], full.indices[m:2 * m]]
    refs = [full.values[:m], full.values[m:2 * m]]
    idx = torch.from_numpy(halves[0].copy()).pin_memory()
    out = torch.empty(m, dtype=torch.float64).pin_memory()
    gd, keep = gli._parse_coeffs(np.ascontiguousarray(g10()), "")
    L = gli.lib()

    def run():
        out.fill_(float("nan"))
        return L.gli_b200_sparse_values(_abi.GLI_KIND_ERI, C.byref(gd), C.byref(gli._grid_struct(W.ERI6_SPARSE)),
                                        C.cast(idx.data_ptr(), _abi.lptr), m, 1e-16, _abi.GLI_FORM_FP64,
                                        C.cast(out.data_ptr(), _abi.dptr))

    for k in range(5):
        assert run() == 0, L.gli_b200_last_error_message().decode()
        assert_parity(out.numpy(), refs[0], what=f"pinned first half, call {k}")
    perm = np.random.default_rng(9).permutation(m)
    idx.copy_(torch.from_numpy(halves[0][perm]))
    assert run() == 0, L.gli_b200_last_error_message().decode()
    assert_parity(out.numpy(), refs[0][perm], what="pinned first half permuted")
    idx.copy_(torch.from_numpy(halves[1]))
    for k in range(4):
        assert run() == 0, L.gli_b200_last_error_message().decode()
        assert_parity(out.numpy(), refs[1], what=f"pinned second half, call {k}")


@pytest.mark.parametrize("case", ["eri7", "erida33"])
def test_stage_times_split_stage_c(gli, case):
    # with timing on, the stage times of graph replays are their own event
    # marks; stage C is the product GEMM (ERI 7^3; at ERIDA 33^3 the device
    # chooses the per-class dots) followed by the class-level kernel
    import torch

    from gausslectronitegrate_b200 import _abi
    from gausslectronitegrate_b200 import workloads as W
    kind, grid_of = CASES[case]
    grid = grid_of(W)
    L = gli.lib()
    gs = gli._grid_struct(grid)
    d_idx, m = C.c_void_p(), _abi.glong()
    assert L.gli_b200_enumerate_dev(kind, C.byref(gs), C.byref(d_idx), C.byref(m), None) == 0
    b = np.ascontiguousarray(g10())
    d_out = torch.empty(m.value, dtype=torch.float64, device="cuda")
    L.gli_b200_set_timing(1)
    try:
        for _ in range(3):
            rc = L.gli_b200_sparse_values_dev(kind, b.ctypes.data_as(_abi.dptr), b.size, C.byref(gs),
                                              d_idx, m.value, 1e-16, _abi.GLI_FORM_FP64,
                                              C.c_void_p(d_out.data_ptr()), None)
            assert rc == 0, L.gli_b200_last_error_message().decode()
        ms4, sz3, ms2 = (C.c_float * 4)(), (_abi.glong * 3)(), (C.c_float * 2)()
        L.gli_b200_last_stage_times(ms4, sz3)
        L.gli_b200_last_stage_c_times(ms2)
        plan = (_abi.glong * 4)()
        L.gli_b200_last_plan(plan)
    finally:
        L.gli_b200_set_timing(0)
        L.gli_b200_free_dev(d_idx, None)
    assert all(ms4[k] > 0 for k in range(1, 4)), list(ms4)
    assert ms2[1] > 0 and ms2[0] >= 0
    # (a bounded plan that the host bounds leave undecided queues both stage-C
    # paths: the product GEMM then launches and returns at once)
    assert ms2[0] > 0 or plan[3] == 0, (list(ms2), list(plan))
    assert abs(ms4[3] - (ms2[0] + ms2[1])) <= 1e-3 + 1e-3 * ms4[3], (list(ms4), list(ms2))
