"""Class-range partition of a sparse evaluation over ranks (one process per
GPU, torch.distributed).

Classes are independent (the reference's only split point is the OpenMP loop
over classes, src/eri_integrals.c:585 and src/erida_integrals.c:465), so the
sorted class list is cut into contiguous ranges, one per rank; every rank
builds its own copy of the lattice tables (a few MB, replicated rather than
sent), evaluates its range from device memory, and one all-gather assembles the
values in class order on every rank.  No other data crosses ranks.  On GPUs
the gather is NCCL's (plain peer transfers; nothing here multicasts).

Each rank's range is evaluated on its own, so its plan covers only the keys
its classes use: the values agree with a single-rank evaluation within the
FP64 parity bar, and bit for bit for a per-class evaluator.
"""
import ctypes as C

import numpy as np


def class_ranges(m, world_size):
    """Contiguous ranges [lo, hi) of a list of m classes, one per rank, sizes
    differing by at most one (the first m % world_size ranks one longer)."""
    if world_size < 1 or m < 0:
        raise ValueError("class_ranges needs m >= 0 and world_size >= 1")
    base, extra = divmod(m, world_size)
    out, lo = [], 0
    for r in range(world_size):
        hi = lo + base + (1 if r < extra else 0)
        out.append((lo, hi))
        lo = hi
    return out


def gather_values(local, ranges, rank, group=None):
    """All-gather of every rank's values (a 1-D float64 torch tensor of its
    range) into the whole list, in class order, on every rank.  Ranges of
    unequal length are padded to the longest for the collective and trimmed
    after it; every rank takes the same collective step."""
    import torch
    import torch.distributed as dist

    ws = len(ranges)
    width = max(hi - lo for lo, hi in ranges)
    lo, hi = ranges[rank]
    if local.numel() != hi - lo:
        raise ValueError(f"rank {rank} holds {local.numel()} values for a range of {hi - lo}")
    if ws == 1:
        return local
    send = torch.zeros(width, dtype=torch.float64, device=local.device)
    send[: hi - lo] = local
    recv = torch.empty(ws * width, dtype=torch.float64, device=local.device)
    dist.all_gather_into_tensor(recv, send, group=group)
    parts = [recv[r * width: r * width + (b - a)] for r, (a, b) in enumerate(ranges)]
    return torch.cat(parts)


def library_evaluator(kind, coeffs, grid, tol, form, stream=None):
    """The product evaluator: values of a device-resident class range through
    gli_b200_sparse_values_dev on the calling rank's GPU."""
    import torch

    from . import _abi, _grid_struct, lib

    L = lib()
    b = np.ascontiguousarray(coeffs, dtype=np.float64)
    gs = _grid_struct(grid)
    kind_id = _abi.GLI_KIND_ERI if kind == "eri" else _abi.GLI_KIND_ERIDA
    form_id = _abi.GLI_FORM_FP64 if form == "fp64" else _abi.GLI_FORM_MIXED

    def evaluate(d_idx):
        out = torch.empty(d_idx.numel(), dtype=torch.float64, device=d_idx.device)
        if d_idx.numel():
            s = stream if stream is not None else torch.cuda.current_stream(d_idx.device)
            rc = L.gli_b200_sparse_values_dev(kind_id, b.ctypes.data_as(_abi.dptr), b.size, C.byref(gs),
                                              C.c_void_p(d_idx.data_ptr()), d_idx.numel(), tol, form_id,
                                              C.c_void_p(out.data_ptr()), C.c_void_p(s.cuda_stream))
            if rc:
                raise RuntimeError(L.gli_b200_last_error_message().decode())
        return out

    return evaluate


def evaluate_sharded(indices, evaluate, rank, world_size, group=None):
    """Values of the whole sorted class list `indices` (a 1-D int64 torch
    tensor, the same on every rank) with each rank evaluating its contiguous
    range through `evaluate` (device tensor of indices -> tensor of values)
    and one all-gather.  Returns (all values, this rank's range)."""
    ranges = class_ranges(int(indices.numel()), world_size)
    lo, hi = ranges[rank]
    local = evaluate(indices[lo:hi].contiguous())
    return gather_values(local, ranges, rank, group), (lo, hi)
