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


STRUCTS = {"icx_layout_info": "LayoutInfo", "icx_newton_options": "NewtonOptions",
           "icx_newton_report": "NewtonReport", "icx_explicit_options": "ExplicitOptions",
           "icx_explicit_report": "ExplicitReport", "icx_lpc_train_options": "LpcTrainOptions",
           "icx_lpc_train_report": "LpcTrainReport", "icx_tile_choice": "TileChoice",
           "icx_tune_report": "TuneReport", "icx_lm_options": "LMOptions", "icx_lm_report": "LMReport",
           "icx_pset_stats": "PsetStats"}


def test_python_structs_match_c_layout():
    """sizeof and every field's offset of the header's structs, compiled by
    gcc, against the ctypes mirrors (same field names)"""
    import subprocess
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "iceicle_b200.h"', "int main(void) {"]
    for cname, pname in STRUCTS.items():
        py = getattr(ib, pname)
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for f in py._fields_:
            lines.append(f'  printf("{cname} {f[0]} %zu\\n", offsetof({cname}, {f[0]}));')
    lines += ["  return 0;", "}"]
    out_dir = os.path.join(ROOT, "_build")
    os.makedirs(out_dir, exist_ok=True)
    src, exe = os.path.join(out_dir, "abi_layout.c"), os.path.join(out_dir, "abi_layout")
    open(src, "w").write("\n".join(lines) + "\n")
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), src, "-o", exe], check=True)
    got = {}
    for ln in subprocess.run([exe], check=True, capture_output=True, text=True).stdout.splitlines():
        s, key, v = ln.split()
        got[(s, key)] = int(v)
    for cname, pname in STRUCTS.items():
        py = getattr(ib, pname)
        assert got[(cname, "size")] == C.sizeof(py), (cname, got[(cname, "size")], C.sizeof(py))
        for f in py._fields_:
            assert got[(cname, f[0])] == getattr(py, f[0]).offset, (cname, f[0])
