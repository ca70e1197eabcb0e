"""Benchmark of the integral hot path on B200.

Workload (the metric's configuration, "ERI classes/sec ... mixed vs FP64
form"): ERI classes of the 6x6x6 configuration at spacing 0.7 bohr.  The
reference's symmetry-reduced path needs the odd rotationally symmetric grid, so
the 7^3 grid (-3, 7)^3 with its 3,571,977 symmetry-reduced classes stands in for
it; G10 gausslet coefficients, tol 1e-16, values scaled by 1/spacing to
Hartree.  Synthetic: the inputs are the coefficients and the grid.

One step = one evaluation of every class value from the class list already
resident in HBM (plan, staged contraction, write-back), i.e. one
gli_b200_sparse_values_dev_async call (the stream-ordered form of
gli_b200_sparse_values_dev) with the lattice tables cached; the statuses of the
timed steps are read after the last one, and the synchronous call's step time
is reported beside it (config.sync_call_ms_per_step).  The class
enumeration is measured apart, and so is a cold step (caches dropped: tables,
plan and graph built again inside the timed call).  The metric compares the
two forms: `value` is the chosen form (--form, default fp64: the drop-in, whose
values match the reference's own at its tol); the other form
is timed the same way beside it, and the mixed form's max abs error against
the FP64 form (and both against the reference C core on a seeded sample) is
reported in Hartree.  `dtype` names the arithmetic that ran, per stage, as the
library reports it (gli_b200_last_paths).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--form fp64|mixed] [--impl ours|reference]

Timing: W >= 3 untimed warm-up steps; each timed step is bracketed by CUDA
events on the stream the library launches on; L2 (126 MB) is flushed by
writing a 1 GB buffer between timed steps (outside the events).  The queued
steps run back to back on the device, each behind its flush; with the
synchronous call the end event waits for the host's return after the status
read-back (the flush, about 160 us on the device, is then the host's lead for
queueing the next step).  The K
steps are bracketed by a barrier and device synchronisation, and the slowest
rank's time counts.  N > 1 (torchrun, one process per GPU): every rank
evaluates its own copy of the workload (weak scaling, no data-path
collective); --shard splits one class list into contiguous ranges over the
ranks and gathers the values (strong scaling, NCCL all-gather).

Other hot-path configurations (--workload): erida33 (ERIDA 32^3, odd stand-in
33^3, spacing 0.5), erida129 (ERIDA 128^3, odd stand-in 129^3, spacing 0.3),
nuclear-batch (256 H_n chains), kinetic24 (24^3 kinetic matrix) and
erida129-surrogate (MLP far field); --profile-only K runs K untimed
evaluations for profilers.

--impl reference times the reference's own CPU implementation (the reference C
core compiled under oracle/_ref, OpenMP on all host cores; the repository's C
restatement of it when that build is absent) on a seeded sample of the same
class list and prints the same JSON line with "impl": "reference".
"""
import argparse
import ctypes as C
import faulthandler
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

faulthandler.enable()


def log(msg):
    print(f"[bench] {msg}", file=sys.stderr, flush=True)


METRIC = "ERI classes/sec on 1 B200, mixed vs FP64 form at <=1e-8 Ha max abs err"
TOL = 1e-16

# the hot-path configurations (--workload); the default line is the metric's (eri7)
WORKLOADS = {
    "eri7": (7, 0.7, "ERI 6x6x6 grid (odd stand-in 7^3, 3571977 classes), spacing 0.7 bohr, G10, tol 1e-16",
             "eri"),
    "erida33": (33, 0.5, "ERIDA 32^3 grid (odd stand-in 33^3, 6545 classes), spacing 0.5 bohr, G10, tol 1e-16",
                "erida"),
    "erida129": (129, 0.3, "ERIDA 128^3 grid (odd stand-in 129^3, 366145 classes), spacing 0.3 bohr, G10, "
                           "tol 1e-16", "erida"),
}
L_GRID, SPACING, WORKLOAD, KIND = WORKLOADS["eri7"]


def g10():
    return np.load(os.path.join(REPO, "tests", "golden", "reference_fixtures.npz"))["g10"]


def grid_spec():
    return [(-(L_GRID // 2), L_GRID)] * 3


def weak_scaling_value(my_ms, classes_per_rank, steps, world_size, device):
    """Whole-job throughput of a weak-scaling run: every rank evaluated its own
    copy of the workload (classes_per_rank classes per step) in my_ms device
    milliseconds; the job's time is the slowest rank's (all-reduce MAX), so the
    value is world_size * classes_per_rank * steps / max time.  Returns (value,
    max total ms); every rank takes the same collective steps."""
    import torch
    t = torch.tensor([float(my_ms)], dtype=torch.float64, device=device)
    if world_size > 1:
        import torch.distributed as dist
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.barrier()
    total_ms = float(t.item())
    return world_size * classes_per_rank * steps / (total_ms * 1e-3), total_ms


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def host_threads():
    """Host cores this process may run on (its CPU affinity)."""
    try:
        return len(os.sched_getaffinity(0))
    except (AttributeError, OSError):
        return os.cpu_count() or 1


def use_all_host_threads():
    """Makes the reference core's OpenMP runtime use every host core this
    process may run on, whatever OMP_NUM_THREADS the launcher set (torchrun
    sets 1 per rank; the reference arm runs on rank 0 alone).  Call before
    the reference library is loaded; returns the thread count."""
    n = host_threads()
    os.environ["OMP_NUM_THREADS"] = str(n)
    return n


class Clocks:
    """nvidia-smi clock/throttle sampling during the timed region."""

    def __init__(self, device):
        self.path = tempfile.mktemp(suffix=".csv")
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(device), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


CPU_SAMPLE = 8000  # classes per pass of the CPU reference when the list is larger


def cpu_reference_rate(b, spec, idx, tol, min_seconds=8.0):
    """Reference C core (oracle/_ref) on all host cores, repeated until about
    min_seconds of CPU work; lists longer than CPU_SAMPLE classes are timed on
    a seeded sample of that many classes.  Returns (classes/s, sample text,
    values of the whole list or None, indices of the sample)."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    from ref_binding import RefLib
    r = RefLib()
    sample = idx if idx.size <= CPU_SAMPLE else np.sort(
        np.random.default_rng(0).choice(idx, size=CPU_SAMPLE, replace=False))
    reps, t0 = 0, time.perf_counter()
    vals = None
    while True:
        vals = r.sparse_values(KIND, b, spec, sample, tol)
        reps += 1
        el = time.perf_counter() - t0
        if el >= min_seconds or reps >= 50:
            break
    what = (f"full {idx.size}-class list" if sample is idx else f"seeded sample of {sample.size} of {idx.size} classes")
    return reps * sample.size / el, f"{what} x {reps} passes ({el:.1f} s)", vals, sample


def cpu_baseline_subprocess(gpu_values_path, workload):
    """Times the reference core in a fresh process (no torch, so its OpenMP
    runtime is the only one loaded); compares its values with the GPU's."""
    env = dict(os.environ, OMP_NUM_THREADS=str(host_threads()))
    r = subprocess.run([sys.executable, os.path.abspath(__file__), "--cpu-baseline-json", gpu_values_path,
                        "--workload", workload], capture_output=True, text=True, timeout=600, env=env)
    if r.returncode != 0:
        raise RuntimeError(f"CPU baseline process failed: {r.stderr.strip()[-300:]}")
    return json.loads(r.stdout.strip().splitlines()[-1])


def cpu_baseline_main(gpu_values_path):
    b = g10()
    spec = grid_spec()
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    from ref_binding import RefLib
    gpu = np.load(gpu_values_path)
    idx = gpu["indices"]  # the class list the GPU evaluated (its enumeration is tested bit-exact)
    rate, sample, vals, sidx = cpu_reference_rate(b, spec, idx, TOL)
    pos = np.searchsorted(idx, sidx)
    errs = {f"max_abs_err_ha_gpu_{k}_vs_reference": float(np.max(np.abs(vals - gpu[k][pos])) / SPACING)
            for k in ("fp64", "mixed") if gpu[k].shape == idx.shape}
    print(json.dumps({"value": rate, "unit": "classes/s", "cores": int(os.environ.get("OMP_NUM_THREADS", "0")) or
                      host_threads(), "kind": "reference",
                      "sample": sample, **errs}))
    return 0


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    cores = use_all_host_threads()
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    from ref_binding import RefLib
    r = RefLib()
    b = g10()
    spec = grid_spec()
    full = r.enumerate(KIND, spec)
    idx = full if full.size <= CPU_SAMPLE else np.sort(
        np.random.default_rng(0).choice(full, size=CPU_SAMPLE, replace=False))
    for _ in range(min(args.warmup, 1)):
        r.sparse_values(KIND, b, spec, idx, TOL)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        r.sparse_values(KIND, b, spec, idx, TOL)
        times.append(time.perf_counter() - t0)
    tot = sum(times)
    value = args.steps * idx.size / tot
    line = {"metric": METRIC, "impl": "reference", "value": value, "unit": "classes/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "classes": int(idx.size), "form": "fp64 (reference C core)"},
            "cpu_baseline": {"value": value, "unit": "classes/s", "cores": cores, "kind": "reference",
                             "sample": (f"full {idx.size}-class list per step" if idx is full else
                                        f"seeded sample of {idx.size} of {full.size} classes per step") +
                                       f", {args.steps} steps"},
            "e2e": {"value": value, "unit": "classes/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch
    ws, rank, local = dist_env()
    if ws > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    log(f"rank {rank}/{ws} on cuda:{local}")
    import gausslectronitegrate_b200 as gli
    from gausslectronitegrate_b200 import _abi
    L = gli.lib()
    L.gli_b200_set_device(local)
    FORMS = {"fp64": _abi.GLI_FORM_FP64, "mixed": _abi.GLI_FORM_MIXED}
    KIND_ID = _abi.GLI_KIND_ERI if KIND == "eri" else _abi.GLI_KIND_ERIDA
    chosen = args.form
    other = "fp64" if chosen == "mixed" else "mixed"
    b = np.ascontiguousarray(g10())
    spec = grid_spec()
    gs = gli._grid_struct(spec)
    stream = torch.cuda.Stream()
    sptr = C.c_void_p(stream.cuda_stream)

    log("enumerating classes")
    # class list on the device (enumeration timed apart)
    d_idx = C.c_void_p()
    num = _abi.glong()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
        rc = L.gli_b200_enumerate_dev(KIND_ID, C.byref(gs), C.byref(d_idx), C.byref(num), sptr)
        e1.record(stream)
    if rc:
        raise RuntimeError(L.gli_b200_last_error_message().decode())
    stream.synchronize()
    enum_ms = e0.elapsed_time(e1)
    m = num.value
    out = torch.empty(m, dtype=torch.float64, device=f"cuda:{local}")
    flush = torch.empty(1024 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")
    coeff_p = b.ctypes.data_as(_abi.dptr)

    def step(f):
        rc = L.gli_b200_sparse_values_dev(KIND_ID, coeff_p, b.size, C.byref(gs), d_idx, m, TOL, f,
                                          C.c_void_p(out.data_ptr()), sptr)
        if rc:
            raise RuntimeError(L.gli_b200_last_error_message().decode())

    def queue(f):
        # the stream-ordered call: queued without a host wait; the status is
        # read by wait() after the timed steps
        t = _abi.glong()
        rc = L.gli_b200_sparse_values_dev_async(KIND_ID, coeff_p, b.size, C.byref(gs), d_idx, m, TOL, f,
                                                C.c_void_p(out.data_ptr()), sptr, C.byref(t))
        if rc:
            raise RuntimeError(L.gli_b200_last_error_message().decode())
        return t.value

    def wait(ticket):
        if L.gli_b200_sparse_values_wait(ticket):
            raise RuntimeError(L.gli_b200_last_error_message().decode())

    if args.profile_only:
        # untimed evaluations of the chosen form only (the command profilers run)
        for _ in range(args.profile_only):
            step(FORMS[chosen])
        stream.synchronize()
        L.gli_b200_free_dev(d_idx, sptr)
        log(f"{args.profile_only} evaluations of the {chosen} form")
        return 0

    log(f"{m} classes; accuracy check")
    vals, screening = {}, {}
    for name, f in FORMS.items():
        step(f)
        stream.synchronize()
        vals[name] = out.cpu().numpy().copy()
        scr = (C.c_double * 2)()
        L.gli_b200_last_screening(scr)
        screening[name] = {"product_threshold": scr[0], "bound_grid_units": scr[1]}
    scale = 1.0 / SPACING  # grid units -> Hartree at this spacing
    max_abs_err_ha = float(np.max(np.abs(vals["mixed"] - vals["fp64"])) * scale)

    def timed_forms(steps, queued=True):
        """Both forms timed under the same conditions: after warm-up, their
        timed steps alternate (chosen, other, chosen, ...), each behind its own
        L2 flush, while the clock sampler runs.  queued: each step is the
        stream-ordered call (the statuses read after the last step); else the
        synchronous call, whose return after its status read-back the end
        event waits for."""
        for name in (chosen, other):
            for _ in range(max(args.warmup, 3)):
                step(FORMS[name])
        stream.synchronize()
        # nvidia-smi samples every 200 ms, longer than the timed steps: the
        # sampler runs across one second of further (untimed) steps of both
        # forms that end where the timed steps begin, and across the timed steps
        clocks = Clocks(local)
        t_end = time.perf_counter() + 1.0
        while time.perf_counter() < t_end:
            for _ in range(10):
                step(FORMS[chosen])
                step(FORMS[other])
            stream.synchronize()
        if ws > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        ev = {n: ([torch.cuda.Event(enable_timing=True) for _ in range(steps)],
                  [torch.cuda.Event(enable_timing=True) for _ in range(steps)]) for n in (chosen, other)}
        launches = 0
        tickets = []
        t_wall = time.perf_counter()
        for k in range(steps):
            for name in (chosen, other):
                with torch.cuda.stream(stream):
                    flush.zero_()  # L2 flush between timed steps, outside the events
                    ev[name][0][k].record(stream)
                l0 = L.gli_b200_launch_count()
                if queued:
                    tickets.append(queue(FORMS[name]))
                else:
                    step(FORMS[name])
                if name == chosen:
                    launches += L.gli_b200_launch_count() - l0
                with torch.cuda.stream(stream):
                    ev[name][1][k].record(stream)
        if tickets:
            wait(tickets[-1])  # every step's status, in order
        stream.synchronize()
        torch.cuda.synchronize()
        wall = time.perf_counter() - t_wall
        clk = clocks.stop()
        clk["window"] = "1 s of untimed steps of both forms ending where the timed steps begin, and the timed steps"
        out = {}
        for name in (chosen, other):
            my_ms = sum(s_.elapsed_time(e_) for s_, e_ in zip(*ev[name]))
            value, total_ms = weak_scaling_value(my_ms, m, steps, ws, f"cuda:{local}")
            out[name] = {"value": value, "ms_per_step": total_ms / steps, "wall_s": wall, "launches": launches,
                         "clocks": clk}
        return out[chosen], out[other]

    log("timed steps")
    main, side = timed_forms(args.steps)
    log("timed steps through the synchronous call")
    main_sync, side_sync = timed_forms(args.steps, queued=False)

    # arithmetic that ran in each form (the library's report of its last evaluation)
    paths = {}
    for name, f in FORMS.items():
        step(f)
        stream.synchronize()
        p3 = (C.c_int * 3)()
        L.gli_b200_last_paths(p3)
        paths[name] = tuple(int(x) for x in p3)

    log("cold step (tables, plan and graph built inside the timed call)")
    cold = {}
    for name, f in FORMS.items():
        L.gli_b200_clear_caches()
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            flush.zero_()
        c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        with torch.cuda.stream(stream):
            c0.record(stream)
        step(f)
        with torch.cuda.stream(stream):
            c1.record(stream)
        stream.synchronize()
        cold[name] = {"device_ms": c0.elapsed_time(c1), "wall_ms": 1e3 * (time.perf_counter() - t0)}

    log("stage timing and FP64 peak probe")
    # per-stage device times of one step (library events on the same stream;
    # the first timed call warms the stream-ordered pool for the untimed path)
    stage = {}
    for name, f in FORMS.items():
        L.gli_b200_set_timing(1)
        for _ in range(3):  # (the third replay of the timed graph reuses its plan, as the timed steps do)
            step(f)
            stream.synchronize()
        ms4 = (C.c_float * 4)()
        sz3 = (_abi.glong * 3)()
        L.gli_b200_last_stage_times(ms4, sz3)
        ms2 = (C.c_float * 2)()
        L.gli_b200_last_stage_c_times(ms2)
        L.gli_b200_set_timing(0)
        plan4 = (_abi.glong * 4)()
        L.gli_b200_last_plan(plan4)
        stage[name] = {"tables": float(ms4[0]), "A": float(ms4[1]), "B": float(ms4[2]), "C": float(ms4[3]),
                       "C_product": float(ms2[0]), "C_class": float(ms2[1]),
                       "sizes": (int(sz3[0]), int(sz3[1]), int(sz3[2])), "plan": tuple(int(x) for x in plan4)}
    nA, nP, U = stage[chosen]["sizes"]
    peak = C.c_double()
    L.gli_b200_measure_fp64_peak(C.byref(peak))

    log("end-to-end through the C API (host buffers)")
    # e2e: the C call with host buffers (host->device copy of the class list and
    # device->host copy of the values inside the timed call); the host class
    # list comes from the reference-facing enumeration call
    idx_s = _abi.SparseIndices()
    getattr(L, f"enumerate_symmetry_reduced_{KIND}_indices")(C.byref(gs), C.byref(idx_s))
    idx_np = np.ctypeslib.as_array(idx_s.indices, shape=(idx_s.num,)).copy()
    getattr(L, f"delete_sparse_{KIND}_indices")(C.byref(idx_s))
    gd, keep = gli._parse_coeffs(b, "")
    # the step's inputs and result in page-locked host memory (the library
    # copies them straight to and from its device buffers)
    idx_pin = torch.from_numpy(idx_np).pin_memory()
    vals_pin = torch.empty(m, dtype=torch.float64).pin_memory()
    e2e_times = []
    for k in range(max(3, args.steps) + 1):
        t0 = time.perf_counter()
        rc = L.gli_b200_sparse_values(KIND_ID, C.byref(gd), C.byref(gs), C.cast(idx_pin.data_ptr(), _abi.lptr),
                                      m, TOL, FORMS[chosen], C.cast(vals_pin.data_ptr(), _abi.dptr))
        e2e_times.append(time.perf_counter() - t0)
        if rc:
            raise RuntimeError(L.gli_b200_last_error_message().decode())
    e2e_s = statistics.median(e2e_times[1:])

    if ws > 1:
        torch.distributed.destroy_process_group()
    if rank != 0:
        L.gli_b200_free_dev(d_idx, sptr)
        return 0

    cpu = None
    if not args.no_cpu_baseline:
        log("CPU baseline (reference core, separate process)")
        try:
            tmp = tempfile.mktemp(suffix=".npz")
            np.savez(tmp, fp64=vals["fp64"], mixed=vals["mixed"], indices=idx_np)
            cpu = cpu_baseline_subprocess(tmp, args.workload)
            os.unlink(tmp)
        except Exception as ex:  # the reference core must be prebuilt (make -C oracle ref)
            cpu = {"value": None, "unit": "classes/s", "cores": host_threads(), "kind": "reference",
                   "sample": f"unavailable: {ex}"}
    st = stage[chosen]
    # the dominant kernel: stage A, stage B, or one of stage C's two kernels
    # (its product GEMM, and the class gather or per-class dots after it)
    dom = max(("A", "B", "C_product", "C_class"), key=lambda k: st[k])
    roof = roofline(paths[chosen], dom, st, st["plan"], U, m, peak.value)
    # (measured DRAM bytes per launch are keyed by stage; "C" is the class gather)
    tkey = {"C_class": "C"}.get(dom, dom) + (":tc" if roof["bound"] == "hbm" and dom in ("A", "B") else "")
    roof["traffic"] = measured_traffic(f"{args.workload}:{tkey}")
    line = {
        "metric": METRIC, "value": main["value"], "unit": "classes/s", "n_gpus": ws, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": main["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": dtype_label(paths[chosen]),
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "classes": m, "form": chosen, "tol": TOL, "spacing_bohr": SPACING,
                   "l2": "flushed between timed steps (1 GB write)",
                   "max_abs_err_ha_mixed_vs_fp64": max_abs_err_ha,
                   "screening": screening,
                   "forms": {chosen: {"classes_per_s": main["value"], "ms_per_step": main["ms_per_step"]},
                             other: {"classes_per_s": side["value"], "ms_per_step": side["ms_per_step"]}},
                   "step_call": "gli_b200_sparse_values_dev_async (stream-ordered; statuses read after the timed "
                                "steps, every step's status checked)",
                   "sync_call_ms_per_step": {chosen: main_sync["ms_per_step"], other: side_sync["ms_per_step"]},
                   "mixed_over_fp64": (main["value"] / side["value"]) if chosen == "mixed" else
                   (side["value"] / main["value"]),
                   "enumeration_ms": enum_ms,
                   "cold_step_ms": cold,
                   "stage_paths": {k: {"A": "s8 tcgen05" if v[0] else "f64 dmma",
                                       "B": "s8 tcgen05" if v[1] else "f64 dmma",
                                       "C": ("f64 product gemm + " + GATHERS[v[2]]) if v[2] else "f64 per-class dots"}
                                   for k, v in paths.items()},
                   "stage_ms": {k: {s_: v[s_] for s_ in ("tables", "A", "B", "C", "C_product", "C_class")}
                                for k, v in stage.items()},
                   "stage_sizes": {k: {"keys_A": v["sizes"][0], "key_pairs": v["sizes"][1], "lattice_U": v["sizes"][2]}
                                   for k, v in stage.items()},
                   "wall_s_timed_region": main["wall_s"]},
        "roofline": roof,
        "e2e": {"value": m / e2e_s, "unit": "classes/s", "h2d_bytes_per_step": 8 * m + 8 * b.size,
                "d2h_bytes_per_step": 8 * m},
        "gpu_launches": main["launches"],
        "clocks": main["clocks"],
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)
    L.gli_b200_free_dev(d_idx, sptr)
    return 0


def run_sharded(args):
    """Strong scaling over one class list: every rank evaluates its contiguous
    range of the sorted list from device memory (gausslectronitegrate_b200.
    sharded) and one NCCL all-gather assembles the values on every rank; a step
    is both, timed on the device with CUDA events and taken as the slowest
    rank's.  value = classes of the whole list per second."""
    import torch
    import torch.distributed as dist

    from gausslectronitegrate_b200 import _abi
    from gausslectronitegrate_b200.sharded import class_ranges, evaluate_sharded, library_evaluator
    ws, rank, local = dist_env()
    if ws > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    import gausslectronitegrate_b200 as gli
    L = gli.lib()
    L.gli_b200_set_device(local)
    spec = grid_spec()
    gs = gli._grid_struct(spec)
    stream = torch.cuda.current_stream()
    # the class list (enumerated through the C API; setup, not timed) on this rank's GPU
    idx_s = _abi.SparseIndices()
    getattr(L, f"enumerate_symmetry_reduced_{KIND}_indices")(C.byref(gs), C.byref(idx_s))
    idx = torch.from_numpy(np.ctypeslib.as_array(idx_s.indices, shape=(idx_s.num,)).copy()).to(f"cuda:{local}")
    getattr(L, f"delete_sparse_{KIND}_indices")(C.byref(idx_s))
    m = int(idx.numel())
    evaluate = library_evaluator(KIND, g10(), spec, TOL, args.form, stream)
    flush = torch.empty(1024 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")
    for _ in range(max(args.warmup, 3)):
        evaluate_sharded(idx, evaluate, rank, ws)
    torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    ms = 0.0
    for _ in range(args.steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        vals, _ = evaluate_sharded(idx, evaluate, rank, ws)
        e1.record(stream)
        torch.cuda.synchronize()
        ms += e0.elapsed_time(e1)
    t = torch.tensor([ms], dtype=torch.float64, device=f"cuda:{local}")
    if ws > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.barrier()
        dist.destroy_process_group()
    total_ms = float(t.item())
    if rank == 0:
        lo, hi = class_ranges(m, ws)[0]
        print(json.dumps({"metric": METRIC, "value": m * args.steps / (total_ms * 1e-3), "unit": "classes/s",
                          "n_gpus": ws, "steps": args.steps, "warmup": max(args.warmup, 3),
                          "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "strong",
                          "vs_baseline": None, "dtype": "f64" if args.form == "fp64" else "see the unsharded line",
                          "data": "synthetic",
                          "config": {"workload": WORKLOAD, "classes": m, "form": args.form,
                                     "partition": f"contiguous class ranges, {hi - lo} classes on rank 0, "
                                                  "values all-gathered (NCCL)",
                                     "l2": "flushed between timed steps (1 GB write)"}}), flush=True)
    return 0


def run_kinetic(args):
    """Config: the kinetic matrix of a 24^3 grid (13,824 points: a 13,824^2
    FP64 matrix, 1.53 GB) at spacing 0.5 bohr.  A step is one matrix written
    into device memory (the 1-D table and the dense matrix kernel, through the
    allocation-free entry point, whose caller owns the output); the metric is
    matrix bytes written per second against the measured HBM bandwidth.  e2e:
    compute_kinetic_gausslet_integrals into host memory."""
    import torch
    import gausslectronitegrate_b200 as gli
    L = gli.lib()
    edge = 24
    grid = [(-(edge // 2), edge)] * 3
    N = edge ** 3
    b = np.ascontiguousarray(g10())
    d_b = torch.tensor(b, dtype=torch.float64, device="cuda")
    out = torch.empty((N, N), dtype=torch.float64, device="cuda")
    gs = gli._grid_struct(grid)
    stream = torch.cuda.current_stream()

    def step():
        rc = L.gli_b200_kinetic_matrix_noalloc(C.c_void_p(d_b.data_ptr()), b.size, C.byref(gs),
                                               C.c_void_p(out.data_ptr()), C.c_void_p(stream.cuda_stream))
        if rc:
            raise RuntimeError(L.gli_b200_last_error_message().decode())

    if args.profile_only:
        for _ in range(args.profile_only):
            step()
        torch.cuda.synchronize()
        return 0
    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    clocks = Clocks(0)
    t_end = time.perf_counter() + 1.0
    while time.perf_counter() < t_end:
        step()
        torch.cuda.synchronize()
    ms = []
    for _ in range(args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step()
        e1.record(stream)
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    clk = clocks.stop()
    # parity of a sample against the allocating entry point's host matrix (e2e)
    t0 = time.perf_counter()
    host = gli.compute_kinetic_gausslet_integrals(b, grid)
    e2e_s = time.perf_counter() - t0
    rows = np.random.default_rng(0).integers(0, N, size=64)
    assert np.array_equal(out[torch.from_numpy(rows).cuda()].cpu().numpy(), host[rows])
    bytes_ = 8.0 * N * N
    mean_ms = sum(ms) / len(ms)
    gbs = bytes_ / (mean_ms * 1e-3) / 1e9
    peak = measured_peaks()
    print(json.dumps({
        "metric": "kinetic matrix bytes written per second on 1 B200 (24^3 grid, 13,824^2 FP64)", "value": gbs,
        "unit": "GB/s", "n_gpus": 1, "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": mean_ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "kinetic matrix, 24^3 grid at 0.5 bohr, G10", "matrix_bytes": bytes_,
                   "l2": "inputs larger than L2 (1.53 GB written per step)"},
        "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak["hbm_gbs"], "unit": "GB/s",
                     "frac": gbs / peak["hbm_gbs"], "kernel": "k_kinetic_matrix",
                     "peak_source": peak_source(peak),
                     "traffic": measured_traffic("kinetic24")},
        "e2e": {"value": bytes_ / e2e_s / 1e9, "unit": "GB/s", "h2d_bytes_per_step": 8 * b.size,
                "d2h_bytes_per_step": bytes_},
        "clocks": clk}), flush=True)
    return 0


def run_projection(args):
    """Config: the 6x6x6 projection -- the ERI classes of the 7^3 stand-in at
    tol 1e-16 projected onto 32 orthonormal columns (Q of the QR factorisation
    of a default_rng(0) 216 x 32 N(0, 1) matrix) over the 216 points of the
    dense 6^3 grid (the basis zero-padded to the 343 points of the class grid).
    A step is one project() call through the C API (host basis in, host 32^4
    tensor out); the roofline counts the factored contraction's FLOPs over
    the 216 points against the measured FP64 peak."""
    import torch
    import gausslectronitegrate_b200 as gli
    from gausslectronitegrate_b200 import workloads as W
    eri = gli.compute_sparse_eri_gausslet_integrals(g10(), W.ERI6_SPARSE, TOL)
    basis = W.eri6_sparse_basis()
    for _ in range(max(args.warmup, 1)):
        eri.project(basis)
    ms = []
    clocks = Clocks(0)
    for _ in range(args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        E = eri.project(basis)
        ms.append(1e3 * (time.perf_counter() - t0))
    clk = clocks.stop()
    # the FLOPs the contraction executes: the first two contractions run over
    # the pairs j <= i of the tensor's (i j) symmetry, n (n + 1) / 2 of n^2,
    # and the first over the l >= k chunks of each slab's rows (64-row tiles
    # start their K loop at their smallest k: tiles at k0 = 0, 64, 128, 192)
    n, M = 216, W.ERI6_STATES
    pairs = n * (n + 1) / 2
    kept = sum(min(64, n - k0) * (n - k0 // 16 * 16) for k0 in range(0, n, 64)) / (n * n)
    flops = 2.0 * (pairs * n * n * M * kept + pairs * n * M * M + n ** 2 * M ** 3 + n * M ** 4)
    step = statistics.median(ms)
    peak = C.c_double()
    gli.lib().gli_b200_measure_fp64_peak(C.byref(peak))
    achieved = flops / (step * 1e-3) / 1e12
    print(json.dumps({
        "metric": "ERI projections/sec on 1 B200 (216 orbitals onto 32, from 3,571,977 classes)",
        "value": 1e3 / step, "unit": "projections/s", "n_gpus": 1, "steps": args.steps, "warmup": max(args.warmup, 1),
        "ms_per_step": step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "ERI 6x6x6 projection (7^3 classes, tol 1e-16, dense 6^3 points, 32 columns)",
                   "max_abs_E": float(np.abs(E).max())},
        "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak.value, "unit": "TFLOP/s",
                     "frac": achieved / peak.value if peak.value else None,
                     "algorithmic_flops_per_step": flops, "kernel": "k_dmma<KeyedSlabOp> + k_dmma<StridedOp>",
                     "flops_counted": "executed: first two contractions over the i >= j pairs, the first over the l >= k chunks",
                     "peak_source": "measured FP64 peak on this device (gli_b200_measure_fp64_peak)",
                     "note": "host-API step: includes the 8 MB output copy"},
        "clocks": clk}), flush=True)
    return 0


def run_nuclear_batch(args):
    """Config: 256 linear H_n chains (n uniform in 2..8, bonds 1.0-3.0 bohr,
    jitter N(0, 0.1) bohr), each on its own centred grid of 8^3..24^3 points at
    0.5 bohr; every matrix written to its own device buffer; one call per step
    (one CUDA graph per chunk of instances).  Metric: instances per second and
    matrix GB/s written; the mixed form's max abs error against FP64 in Ha on
    the first instances."""
    import torch
    import gausslectronitegrate_b200 as gli
    from gausslectronitegrate_b200 import _abi
    L = gli.lib()
    count = args.instances
    from gausslectronitegrate_b200 import workloads
    grids, pos, q = workloads.nuclear_batch_config(count)
    n = len(grids)
    specs = [gli._parse_grid(g, "") for g in grids]
    gstructs = (_abi.Grid * n)(*[gli._grid_struct(sp) for sp in specs])
    nucs, offs = [], [0]
    for p_, q_ in zip(pos, q):
        arr, cnt = gli._parse_nuclei(p_, q_, "")
        nucs.extend(arr[k] for k in range(cnt))
        offs.append(offs[-1] + cnt)
    nuc_arr = (_abi.Nucleus * len(nucs))(*nucs)
    off = np.asarray(offs, dtype=np.int64)
    Ns = [sp[0][1] * sp[1][1] * sp[2][1] for sp in specs]
    total_bytes = 8 * sum(N * N for N in Ns)
    outs = [torch.empty(N * N, dtype=torch.float64, device="cuda") for N in Ns]
    ptrs = (C.c_void_p * n)(*[o.data_ptr() for o in outs])
    gd, keep = gli._parse_coeffs(np.ascontiguousarray(g10()), "")
    stream = torch.cuda.Stream()
    forms = {"fp64": _abi.GLI_FORM_FP64, "mixed": _abi.GLI_FORM_MIXED}

    def call(f):
        rc = L.gli_b200_nuclear_batch_dev(C.byref(gd), n, gstructs, off.ctypes.data_as(_abi.lptr), nuc_arr, 1e-8,
                                          forms[f], ptrs, C.c_void_p(stream.cuda_stream))
        if rc:
            raise RuntimeError(L.gli_b200_last_error_message().decode())

    if args.profile_only:
        for _ in range(args.profile_only):
            call(args.form)
        stream.synchronize()
        return 0
    res = {}
    first = {}
    for f in ("fp64", "mixed"):
        for _ in range(max(args.warmup, 3)):
            call(f)
        stream.synchronize()
        first[f] = [o[:16384].cpu().numpy().copy() for o in outs[:4]]
        clocks = Clocks(0) if f == args.form else None
        ms = []
        for _ in range(args.steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            call(f)
            e1.record(stream)
            stream.synchronize()
            ms.append(e0.elapsed_time(e1))
        res[f] = {"ms_per_step": sum(ms) / len(ms), "instances_per_s": n / (sum(ms) / len(ms) * 1e-3),
                  "matrix_gb_per_s": total_bytes / (sum(ms) / len(ms) * 1e-3) / 1e9,
                  "clocks": clocks.stop() if clocks else None}
    err = max(float(np.max(np.abs(a - b))) for a, b in zip(first["mixed"], first["fp64"])) / 0.5
    stats = (_abi.glong * 3)()
    L.gli_b200_last_nuclear_batch(stats)
    buf = C.create_string_buffer(65536)
    L.gli_b200_autotune_report(buf, 65536)
    main_ = res[args.form]
    line = {"metric": "nuclear matrices/sec on 1 B200 (batched H_n chains)", "value": main_["instances_per_s"],
            "unit": "instances/s", "n_gpus": 1, "steps": args.steps, "warmup": max(args.warmup, 3),
            "ms_per_step": main_["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.form == "fp64" else "s8 tensor-core slices + f64", "data": "synthetic",
            "config": {"workload": f"{n} H_n chains (n 2..8), grids 8^3..24^3 at 0.5 bohr, G10, tol 1e-8",
                       "matrix_bytes_per_step": total_bytes, "forms": res,
                       "max_abs_err_ha_mixed_vs_fp64_first4": err, "graph_chunks": int(stats[1]),
                       "streams": int(stats[2]), "autotune": json.loads(buf.value.decode())},
            "clocks": main_["clocks"]}
    print(json.dumps(line), flush=True)
    return 0


def run_surrogate(args):
    """Config: ERIDA 128^3 (odd stand-in 129^3) at 0.3 bohr with the far-field
    surrogate: train on exact classes, evaluate with a 1% seeded audit against
    the 1e-6 Ha target (shells redone above half of it), compare with the exact
    evaluation."""
    import gausslectronitegrate_b200 as gli
    from gausslectronitegrate_b200 import _abi
    L = gli.lib()
    gd, keep = gli._parse_coeffs(np.ascontiguousarray(g10()), "")
    t0 = time.perf_counter()
    h = C.c_void_p()
    rc = L.gli_b200_surrogate_train(C.byref(gd), TOL, 12.0, args.train_steps, 2e-3, 0.0, 7, C.byref(h))
    if rc:
        raise RuntimeError(L.gli_b200_last_error_message().decode())
    train_s = time.perf_counter() - t0
    info = (C.c_double * 13)()
    L.gli_b200_surrogate_info(h, info)
    grid = [(-64, 129)] * 3
    gs = gli._grid_struct(grid)
    ex = gli.compute_sparse_erida_gausslet_integrals(g10(), grid, TOL)
    idx = ex.indices
    # audit threshold at half the 1e-6 Ha target: an audited shell whose sample
    # errs by more is evaluated exactly, so that its unaudited classes keep a margin
    shell_tol = 0.5e-6 * 0.3
    vals = np.empty(idx.size)
    rep = np.zeros((256, 4))
    exact_ms, sur_ms = [], []
    clocks = Clocks(0)
    for _ in range(max(args.steps, 2)):
        t0 = time.perf_counter()
        L.gli_b200_sparse_values(0, C.byref(gd), C.byref(gs), idx.ctypes.data_as(_abi.lptr), idx.size, TOL, 0,
                                 vals.ctypes.data_as(_abi.dptr))
        exact_ms.append(1e3 * (time.perf_counter() - t0))
        t0 = time.perf_counter()
        rc = L.gli_b200_erida_surrogate_values(h, C.byref(gd), C.byref(gs), idx.ctypes.data_as(_abi.lptr), idx.size,
                                               TOL, 0.01, 11, shell_tol, vals.ctypes.data_as(_abi.dptr),
                                               rep.ctypes.data_as(_abi.dptr), 256)
        sur_ms.append(1e3 * (time.perf_counter() - t0))
        if rc:
            raise RuntimeError(L.gli_b200_last_error_message().decode())
    clk = clocks.stop()
    L.gli_b200_surrogate_free(h)
    err = np.abs(vals - ex.values)
    # generalisation: the same network trained with a seeded 20% of the
    # displacements held out, its error on those it never saw (grid units),
    # beside the 1/r error that it corrects
    h2 = C.c_void_p()
    rc = L.gli_b200_surrogate_train(C.byref(gd), TOL, 12.0, args.train_steps, 2e-3, 0.2, 7, C.byref(h2))
    if rc:
        raise RuntimeError(L.gli_b200_last_error_message().decode())
    info2 = (C.c_double * 13)()
    L.gli_b200_surrogate_info(h2, info2)
    L.gli_b200_surrogate_free(h2)
    line = {"metric": "ERIDA classes/sec on 1 B200 with the far-field surrogate (1% audit, 1e-6 Ha)",
            "value": idx.size / (statistics.median(sur_ms[1:]) * 1e-3), "unit": "classes/s", "n_gpus": 1,
            "steps": len(sur_ms), "warmup": 1, "ms_per_step": statistics.median(sur_ms[1:]), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 network + f64 exact", "data": "synthetic",
            "config": {"workload": WORKLOADS["erida129"][2], "train_s": train_s, "train_steps": args.train_steps,
                       "surrogate_info": list(info), "exact_ms_host_buffers": statistics.median(exact_ms[1:]),
                       "max_abs_err_ha": float(err.max() / 0.3), "audited": int(rep[:, 1].sum()),
                       "shells_evaluated_in_full": [k for k in range(256) if rep[k, 0] > 0 and rep[k, 3] == 1],
                       "holdout_20pct": {"train_max_err_grid": info2[5], "holdout_max_err_grid": info2[6],
                                         "samples": info2[0], "held_out": info2[1]},
                       "exact_over_surrogate_speed": statistics.median(exact_ms[1:]) / statistics.median(sur_ms[1:])},
            "clocks": clk}
    print(json.dumps(line), flush=True)
    return 0


# the class gather of a product-form stage C (gli_b200_last_paths out[2])
GATHERS = {1: "k_gather_q", 2: "k_gather_q_plan"}


def dtype_label(paths):
    """The arithmetic of an evaluation from the library's per-stage report:
    f64 unless a stage ran as int8-sliced products on the tensor cores."""
    tc = [st for st, on in zip("AB", paths[:2]) if on]
    if not tc:
        return "f64"
    return f"s8 tensor-core slices (int32 exact) in stage{'s' if len(tc) > 1 else ''} {'+'.join(tc)}, f64 elsewhere"


def lattice_nS(U):
    """number of distinct u^2 + v^2 with 0 <= u, v < U (rows of stage A)"""
    u = np.arange(U, dtype=np.int64)
    return int(np.unique((u[:, None] ** 2 + u[None, :] ** 2).ravel()).size)


def roofline(paths, dom, st, plan, U, m, fp64_peak):
    """Roofline entry of the dominant kernel (from the library's stage events:
    stage A, stage B, or one of stage C's two kernels, C_product and C_class).
    FP64 kernels (the FP64 tensor-core GEMM k_dmma, or the per-class dots of
    stage C): the kernel's algorithmic FP64 FLOPs against the measured FP64
    peak (gli_b200_measure_fp64_peak: the faster of the FMA and m8n8k4 MMA
    probes).  Tensor-core stages of the mixed form: the sliced work is bound by
    the bytes it must move (int8 slices read, FP64 results written) against the
    measured HBM bandwidth.  paths = the library's per-stage report of the step
    (gli_b200_last_paths); plan = (nA, nP, used keys, stage C products): the
    (pair, key) products the product GEMM computed, 0 when stage C ran per
    class (one length-U dot product per class).  The class gather after the
    product GEMM moves 16 bytes per class (the class index in, its value out)
    against the measured HBM bandwidth."""
    nA, nP, nku, product = plan
    ms = st[dom]
    nS = lattice_nS(U)
    kp = (U + 63) // 64 * 64
    on_tensor_cores = bool((dom == "A" and paths[0]) or (dom == "B" and paths[1]))
    if dom == "C_class" and product:
        bytes_ = 16.0 * m
        achieved = bytes_ / (ms * 1e-3) / 1e9 if ms > 0 else None
        mp = measured_peaks()
        peak = mp["hbm_gbs"]
        return {"bound": "hbm", "stage": "C", "kernel": GATHERS[paths[2]],
                "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak if achieved and peak else None,
                "peak_source": peak_source(mp),
                "algorithmic_bytes_per_launch": bytes_, "products": product, "traffic": None}
    if not on_tensor_cores:
        flops = {"A": 2.0 * nA * nS * U, "B": 2.0 * nP * U * U,
                 "C_product": 2.0 * product * U, "C_class": 2.0 * m * U}[dom]
        kernel = {"A": "k_dmma<StageAOp>", "B": "k_dmma<StageBOp>", "C_product": "k_dmma<ProductOp>",
                  "C_class": "k_stage_c"}[dom]
        achieved = flops / (ms * 1e-3) / 1e12 if ms > 0 else None
        return {"bound": "fp64", "stage": dom[0], "kernel": kernel,
                "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                "frac": achieved / fp64_peak if achieved and fp64_peak else None,
                "peak_source": "measured FP64 peak on this device (gli_b200_measure_fp64_peak: "
                               "max of FMA and m8n8k4 MMA probes)",
                "algorithmic_flops_per_launch": flops, "traffic": None}
    S, BN = 5, 96
    nsp = (nS + 127) // 128 * 128
    bytes_ = {"A": S * nsp * kp + S * ((nA + BN - 1) // BN * BN) * kp + 8 * nA * nS,
              "B": 8.0 * nA * nS + 2 * S * nA * ((U + 127) // 128 * 128) * kp + 2 * S * nP * kp + 8 * nP * U}[dom]
    achieved = bytes_ / (ms * 1e-3) / 1e9 if ms > 0 else None
    mp = measured_peaks()
    peak = mp["hbm_gbs"]
    return {"bound": "hbm", "stage": dom,
            "kernel": {"A": "k_tc_gemm<5,5> (stage A)", "B": "k_slice_group + k_tc_gemm<5,5> (stage B)"}[dom],
            "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak if achieved and peak else None,
            "peak_source": peak_source(mp),
            "algorithmic_bytes_per_launch": bytes_, "traffic": None}


def measured_traffic(key):
    """DRAM bytes per launch of a workload's dominant kernel (key: the workload,
    or workload:stage) from the committed ncu summaries
    (profiles/dram_traffic.json), or None when no capture of it exists."""
    try:
        with open(os.path.join(REPO, "profiles", "dram_traffic.json")) as f:
            d = json.load(f).get(key)
        return d["bytes_per_launch"] if d else None
    except Exception:
        return None


def peak_source(mp):
    return ("MEASURED_PEAKS.json hbm_gbs (of measured)" if mp["source"] == "measured" else
            "6.65 TB/s, the profiling recipe's HBM figure for this pool (of fallback: MEASURED_PEAKS.json absent)")


def measured_peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return {"hbm_gbs": float(d["hbm_gbs"]), "bf16_tflops": float(d["bf16_tflops"]), "source": "measured"}
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--form", choices=["fp64", "mixed"], default="fp64",
                    help="the form of the line's value (the other is timed beside it)")
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--shard", action="store_true",
                    help="N > 1: split one class list over the ranks and all-gather the values (strong scaling)")
    ap.add_argument("--cpu-baseline-json", default=None, help=argparse.SUPPRESS)
    ap.add_argument("--workload", choices=["eri7", "erida33", "erida129", "nuclear-batch", "kinetic24",
                                           "eri6-proj", "erida129-surrogate"],
                    default="eri7", help="eri7 is the metric's configuration (the default line)")
    ap.add_argument("--profile-only", type=int, default=0, metavar="K",
                    help="run K untimed evaluations of --form and print nothing (for profilers)")
    ap.add_argument("--instances", type=int, default=256, help="nuclear-batch: number of H_n chains")
    ap.add_argument("--train-steps", type=int, default=40000, help="erida129-surrogate: training steps")
    args = ap.parse_args()
    global L_GRID, SPACING, WORKLOAD, KIND
    if args.workload in WORKLOADS:
        L_GRID, SPACING, WORKLOAD, KIND = WORKLOADS[args.workload]
    if args.cpu_baseline_json:
        return cpu_baseline_main(args.cpu_baseline_json)
    if args.workload == "nuclear-batch":
        return run_nuclear_batch(args)
    if args.workload == "kinetic24":
        return run_kinetic(args)
    if args.workload == "eri6-proj":
        return run_projection(args)
    if args.workload == "erida129-surrogate":
        return run_surrogate(args)
    if args.impl == "reference":
        return run_reference(args)
    if args.shard:
        return run_sharded(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
