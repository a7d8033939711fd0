"""The C ABI library: it loads without a GPU, exports every function that
include/*.h declares, and answers argument errors before touching CUDA."""
import ctypes as C
import glob
import os
import re

import tb8gen_b200 as tbg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"^\s*(?:int|const char \*|uint64_t)\s+\**(tbg_\w+)\s*\(", text, re.M))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    assert "tbg_predecessors" in names and "tbg_check_successors" in names
    assert len(names) >= 20


def test_library_exports_every_declared_function():
    L = tbg.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing


def test_argument_errors_without_gpu():
    L = tbg.lib()
    assert L.tbg_material_select(99) == -1        # TBG_ERR_ARG
    assert L.tbg_material_from_name(None) == -1
    n = C.c_uint64()
    assert L.tbg_launches(C.byref(n)) == 0
    assert b"material" in L.tbg_last_error() or L.tbg_last_error() is not None


def _tbgen():
    path = os.path.join(ROOT, "tb8gen_b200", "tbgen")
    if not os.path.exists(path):
        import pytest
        pytest.skip("tbgen not built")
    return path


def test_tbgen_arguments_without_gpu():
    """The C host driver refuses bad arguments before it touches CUDA: no
    material, a segment size outside 0..64, a persistent-kernel mode other
    than 1 or 2."""
    import subprocess

    tbgen = _tbgen()
    r = subprocess.run([tbgen], capture_output=True, text=True, timeout=60)
    assert r.returncode != 0 and "usage: tbgen" in r.stderr
    for g in ("65", "-1"):
        r = subprocess.run([tbgen, "-S", "-g", g, "KRvK"], capture_output=True, text=True,
                           timeout=60)
        assert r.returncode != 0 and "-g takes" in r.stderr
    for k in ("0", "3"):
        r = subprocess.run([tbgen, "-k", k, "KRvK"], capture_output=True, text=True, timeout=60)
        assert r.returncode != 0 and "-k takes" in r.stderr


def test_tbgen_reports_library_errors_without_gpu():
    """Without a GPU, tbg_init fails and the driver exits with the library's
    message (no CPU fallback)."""
    import subprocess

    import torch

    if torch.cuda.is_available():
        import pytest
        pytest.skip("a GPU is present")
    r = subprocess.run([_tbgen(), "KRvK"], capture_output=True, text=True, timeout=120)
    assert r.returncode != 0 and "tbgen: init:" in r.stderr


def test_checkers_built_together():
    """Where the reference-worker harness has been built, the probe harness
    and the reference's programs have been built beside it (the probe parity
    tests skip, rather than fail, without them)."""
    ref = os.path.join(ROOT, "oracle", "_ref")
    if not os.path.exists(os.path.join(ref, "libtbref.so")):
        import pytest
        pytest.skip("reference checkers not built here")
    for name in ("libtbprobe.so", "tb8gen", "tb8gen_stub"):
        assert os.path.exists(os.path.join(ref, name)), name
