"""Comparison of restart and VTU files written by two implementations. Test
infrastructure only."""
import numpy as np


def _blocks(lines):
    """(first, last, is_float, scale) of every DataArray: the line range of its
    values, whether it is Float64, and the largest magnitude it holds"""
    out, start, is_float = [], None, False
    for i, ln in enumerate(lines):
        if ln.startswith("<DataArray"):
            start, is_float = i, 'type="Float64"' in ln
        elif ln.startswith("</DataArray") and start is not None:
            vals = [abs(float(t)) for l2 in lines[start + 1:i] for t in l2.split()] if is_float else []
            out.append((start + 1, i - 1, is_float, max(vals) if vals else 0.0))
            start = None
    return out


def vtu_diff(a_text, b_text, rtol=1e-6):
    """None when the two ASCII VTU files agree, else the first difference.
    Agreement: the same lines with the same tokens; tags, attributes, names
    and every Int64 value (connectivity, offsets, cell types) identical; every
    Float64 value within rtol times the largest magnitude of its DataArray
    (both files print 8 significant digits of values that two implementations
    sum in different orders)."""
    a_lines, b_lines = a_text.splitlines(), b_text.splitlines()
    if len(a_lines) != len(b_lines):
        return f"{len(a_lines)} lines vs {len(b_lines)}"
    blocks = _blocks(b_lines)
    for i, (la, lb) in enumerate(zip(a_lines, b_lines)):
        ta, tb = la.split(), lb.split()
        if len(ta) != len(tb):
            return f"line {i + 1}: {len(ta)} tokens vs {len(tb)}"
        blk = next((b for b in blocks if b[0] <= i <= b[1]), None)
        if blk is None or not blk[2]:
            if ta != tb:
                return f"line {i + 1}: {la!r} vs {lb!r}"
            continue
        for x, y in zip(ta, tb):
            if abs(float(x) - float(y)) > rtol * blk[3]:
                return f"line {i + 1}: {x} vs {y} (array scale {blk[3]:g})"
    return None


def read_numbers(path):
    with open(path) as f:
        return np.array([float(t) for t in f.read().split()])
