"""The C ABI library loads and exports every function include/*.h declares;
no compute calls (no GPU needed)."""
import ctypes as C
import os
import re

import iceicle_b200 as ib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    inc = os.path.join(ROOT, "include")
    for fn in os.listdir(inc):
        if not fn.endswith(".h"):
            continue
        txt = open(os.path.join(inc, fn)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"^\s*(?:icx_status|void|const char\*)\s+(icx_\w+)\s*\(", txt, flags=re.M):
            names.add(m.group(1))
    return names


def test_library_exports_all_declared_symbols():
    lib = C.CDLL(ib.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_create_without_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        return
    h = C.c_void_p()
    st = ib.lib().icx_create(C.byref(h), 0)
    assert st == 8  # ICX_ERR_NO_DEVICE: there is no CPU fallback


def declared_arity():
    """number of parameters of every declared icx_* function"""
    out = {}
    inc = os.path.join(ROOT, "include")
    for fn in os.listdir(inc):
        if not fn.endswith(".h"):
            continue
        txt = open(os.path.join(inc, fn)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"^\s*(?:icx_status|void|const char\*)\s+(icx_\w+)\s*\(([^;]*?)\)\s*;", txt,
                             flags=re.M | re.S):
            params = m.group(2).strip()
            depth, n = 0, (0 if params in ("", "void") else 1)
            for ch in params:
                depth += ch == "("
                depth -= ch == ")"
                n += ch == "," and depth == 0
            out[m.group(1)] = n
    return out


def test_python_bindings_match_declared_parameters():
    """every ctypes signature the Python mirror sets has the header's
    parameter count (a mismatch would pass wrong arguments silently)"""
    lib = ib.lib()
    arity = declared_arity()
    checked = 0
    for name, n in arity.items():
        f = getattr(lib, name, None)
        if f is None or getattr(f, "argtypes", None) is None:
            continue
        assert len(f.argtypes) == n, (name, len(f.argtypes), n)
        checked += 1
    assert checked >= 40
