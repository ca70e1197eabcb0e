"""The C-ABI library without a device: it loads, exports every function that
include/gli_b200.h declares, and its host-only logic (the autotuner's choice
and cache) works.  No compute call is made."""
import ctypes as C
import os
import re
import subprocess

from _common import HERE

REPO = os.path.dirname(HERE)


def _declared_functions():
    """Names of the functions the header declares (prototypes at file scope;
    the static inline helpers, which the library need not export, excluded)."""
    text = open(os.path.join(REPO, "include", "gli_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    text = re.sub(r"//[^\n]*", " ", text)
    # drop preprocessor lines and the C++ linkage block they guard
    text = re.sub(r"#ifdef __cplusplus\s*extern \"C\" \{\s*#endif", " ", text)
    text = re.sub(r"#ifdef __cplusplus\s*\}\s*#endif", " ", text)
    text = "\n".join(ln for ln in text.splitlines() if not ln.lstrip().startswith("#"))
    flat, depth = [], 0
    for ch in text:  # every brace-enclosed body becomes one statement end
        if ch == "{":
            if depth == 0:
                flat.append(";")
            depth += 1
        elif ch == "}":
            depth -= 1
        elif depth == 0:
            flat.append(ch)
    names = set()
    for stmt in "".join(flat).split(";"):
        st = " ".join(stmt.split())
        m = re.match(r"^(?:extern \"C\" )?[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\((.*)\)$", st)
        if m and not st.startswith("typedef") and "static" not in st and "inline" not in st:
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_function():
    import gausslectronitegrate_b200 as gli
    path = gli._abi.LIB_PATH
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True, check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if ln.strip()}
    declared = _declared_functions()
    assert len(declared) > 40, declared
    missing = sorted(declared - exported)
    assert not missing, f"declared in include/gli_b200.h but not exported: {missing}"
    lib = C.CDLL(path)
    for name in gli._abi.EXPORTS:
        getattr(lib, name)


def test_autotuner_selftest_without_device():
    import gausslectronitegrate_b200 as gli
    assert gli.lib().gli_b200_autotune_selftest() == 0
