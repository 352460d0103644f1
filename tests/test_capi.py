"""CPU-side checks of the drop-in boundary: the library loads and exports every
entry point that include/*.h declares; the Python binding covers them all.
No compute call is made (no GPU here)."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")


def declared_symbols():
    names = set()
    for fn in os.listdir(INCLUDE):
        if not fn.endswith(".h"):
            continue
        txt = open(os.path.join(INCLUDE, fn)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"^\s*(?:[A-Za-z_][\w\s\*]*?)\b(rt_\w+)\s*\(", txt, flags=re.M):
            names.add(m.group(1))
    return names


@pytest.fixture(scope="module")
def libpath():
    from robtop_b200 import build

    return build.build()


def test_library_loads_and_exports_all_declared_symbols(libpath):
    lib = ctypes.CDLL(libpath)
    missing = [n for n in sorted(declared_symbols()) if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"
    out = subprocess.run(["nm", "-D", "--defined-only", libpath], capture_output=True, text=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if " T rt_" in l}
    assert declared_symbols() <= exported


def test_python_binding_covers_header():
    from robtop_b200 import _capi

    assert declared_symbols() <= set(_capi.SIGNATURES), declared_symbols() - set(_capi.SIGNATURES)


def test_params_default_without_gpu(libpath):
    from robtop_b200 import _capi

    p = _capi.Params()
    _capi.lib().rt_params_default(ctypes.byref(p))
    assert p.power_penalty == 3.0 and p.skip_layer1 == 1 and p.mode == _capi.MODE_WSFF


def test_ctx_create_fails_cleanly_without_gpu(libpath):
    import torch

    if torch.cuda.is_available():
        pytest.skip("GPU present")
    from robtop_b200 import _capi

    h = ctypes.c_void_p()
    st = _capi.lib().rt_ctx_create(0, None, ctypes.byref(h))
    assert st != _capi.RT_OK and not h.value
