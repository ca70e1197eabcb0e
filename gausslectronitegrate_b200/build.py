"""Build libgli_b200.so in-tree with nvcc for sm_100a.

    python -m gausslectronitegrate_b200.build [--debug]

Each translation unit under csrc/ is compiled to an object in _build/ (in
parallel), then linked with the static CUDA runtime into
gausslectronitegrate_b200/libgli_b200.so, which the Python layer loads.  The
build cross-compiles without a GPU.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(REPO, "_build", "gli_b200")
LIB = os.path.join(PKG, "libgli_b200.so")
# the debug build (device bounds checks, -DGLI_B200_DEBUG) goes to its own
# objects and library; GLI_B200_LIBRARY=<path> makes the package load it
BUILD_DEBUG = os.path.join(REPO, "_build", "gli_b200_debug")
LIB_DEBUG = os.path.join(PKG, "libgli_b200_debug.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["runtime.cu", "tables.cu", "enumerate.cu", "contract.cu", "kinetic.cu", "nuclear.cu", "dense.cu",
           "tc_gemm.cu", "autotune.cu", "surrogate.cu", "capi.cu", "h5file.cu"]


def _flags(debug):
    f = ARCH + ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC",
                "-I" + os.path.join(REPO, "include"), "-I" + CSRC, "-ccbin", "/usr/bin/g++",
                "-Xcudafe", "--diag_suppress=declared_but_not_referenced"]
    if debug:
        f += ["-DGLI_B200_DEBUG"]
    return f


def _stale(obj, src):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    deps = [src] + [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".cuh", ".h"))]
    deps += [os.path.join(REPO, "include", h) for h in ("gli_b200.h", "hdf5.h", "hdf5_util.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def build(debug=False, verbose=False):
    bdir, lib = (BUILD_DEBUG, LIB_DEBUG) if debug else (BUILD, LIB)
    os.makedirs(bdir, exist_ok=True)
    flags = _flags(debug)
    jobs = []
    objs = []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(bdir, src.replace(".cu", ".o"))
        objs.append(o)
        if _stale(o, s):
            jobs.append([NVCC] + flags + ["-c", s, "-o", o])

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        if verbose and (r.stdout or r.stderr):
            print(r.stdout, r.stderr, file=sys.stderr)

    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        list(ex.map(run, jobs))
    if jobs or not os.path.exists(lib):
        # the version script exports the C entry points and keeps every
        # internal (C++) symbol local to the library
        vs = os.path.join(bdir, "exports.map")
        with open(vs, "w") as f:
            f.write("{ global: compute_*; delete_*; enumerate_*; fill_dense_*; apply_sparse_*; project_sparse_*;"
                    " sparse_*; minimum_octahedral_*; evaluate_octahedral_*; gli_b200_*; get_hdf5_*; read_hdf5_*;"
                    " write_hdf5_*; get_time_ticks; get_tick_resolution; local: *; };\n")
        run([NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", lib] + objs +
            ["-Xlinker", "--version-script=" + vs, "-ccbin", "/usr/bin/g++"])
    return lib


if __name__ == "__main__":
    print(build(debug="--debug" in sys.argv, verbose=True))
