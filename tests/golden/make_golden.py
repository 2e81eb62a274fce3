"""Generates the golden vectors under tests/golden/ from libsci's own CPU path.

Run from the repository root after `make -C oracle ref` (which compiles the reference sources into
oracle/_ref/libsci_ref.so):  python tests/golden/make_golden.py

codes.npz      for float32 and float64: inputs x, y (1031 values with specials) and, for every chunk
               code, the reference's output of code(x) / code(x, y) / fma(x, y, y).
workloads.npz  the plain fused workload at 4099 elements (a = linspace(0,1), b ~ U[-1,1) seed 0,
               c = 1): t = a*b + c*2, e = exp(t)*0.5, s = sum(sin(t)); and a seeded 64x64 float32
               matrix with its LU factors and row order from linear::factor.
elements.npz   for the eight integer element types: operands x, y, z (129 values inside the ranges
               where C++ defines every step) and the reference's host-loop results of the named
               integer expressions of oracle/ref_bridge.cpp (sci_ref_elements 0-6, 10-13).
               Written alone by: python tests/golden/make_golden.py elements
"""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from libsci_b200 import chunk as C  # noqa: E402
from tests import _oracle  # noqa: E402


def inputs(dtype, count, seed):
    rng = np.random.default_rng(seed)
    x = np.concatenate([rng.standard_normal(count // 2) * 3, rng.uniform(-100, 100, count - count // 2)]).astype(dtype)
    y = rng.uniform(0, 10, count).astype(dtype)
    specials = np.array([0.0, -0.0, np.inf, -np.inf, np.nan, 1e-45, -1e-45, 1e-38, 3e-39, 88.7, 89.5, -103.9,
                         -104.5, 1e6, 2e6, -3e7, 1e30, 710.0, -746.0, 0.5, 1.0, -1.0], dtype)
    x[: specials.size] = specials
    y[::97] = -0.0
    y[::101] = np.nan
    return x, y


def expression(code, a, b):
    if code < C.CODE["add"]:
        return C.Node(C.CODES[code], [a])
    if code == C.CODE["fuse"]:
        return a * b + b
    return C.Node(C.CODES[code], [a, b])


def main():
    ref = _oracle.reference()
    if ref is None:
        raise SystemExit("build oracle/_ref first: make -C oracle ref")
    out = {}
    for dtype, suffix in ((np.float32, "f32"), (np.float64, "f64")):
        n = 1031
        x, y = inputs(dtype, n, seed=11)
        out[f"x_{suffix}"], out[f"y_{suffix}"] = x, y
        a, b = C.Reference(x.ctypes.data, n, dtype), C.Reference(y.ctypes.data, n, dtype)
        for code in range(C.CODE["fuse"] + 1):
            out[f"{C.CODES[code]}_{suffix}"] = _oracle.execute(ref, C.record_output(expression(code, a, b)), n, dtype)
    np.savez_compressed(ROOT / "tests" / "golden" / "codes.npz", **out)

    n = 4099
    step = 1.0 / (n - 1.0)
    a = (np.arange(n, dtype=np.float64) * step).astype(np.float32)
    b = np.random.default_rng(0).uniform(-1, 1, n).astype(np.float32)
    c = np.ones(n, np.float32)
    ra, rb, rc = (C.Reference(v.ctypes.data, n, np.float32) for v in (a, b, c))
    t = _oracle.execute(ref, C.record_output(ra * rb + rc * 2.0), n, np.float32)
    rt = C.Reference(t.ctypes.data, n, np.float32)
    e = _oracle.execute(ref, C.record_output(C.unary("exponential", rt) * 0.5), n, np.float32)
    s = _oracle.reduce(ref, C.record_reduce(C.unary("sin", rt)), C.SUM, n)
    g = np.random.default_rng(21).standard_normal((64, 64)).astype(np.float32)
    factors = g.copy()
    rows = np.zeros(64, np.uint64)
    ref.sci_ref_factor_f32(factors.ctypes.data, rows.ctypes.data, 64)
    np.savez_compressed(ROOT / "tests" / "golden" / "workloads.npz", a=a, b=b, c=c, t=t, e=e, s=np.float64(s),
                        lu_input=g, lu_rows=rows, lu_factors=factors)
    print("wrote tests/golden/codes.npz and tests/golden/workloads.npz")


def elements():
    from tests.test_elements import INTEGERS, operands, reference_elements

    ref = _oracle.reference()
    if ref is None:
        raise SystemExit("build oracle/_ref first: make -C oracle ref")
    out = {}
    for dtype in INTEGERS:
        name = np.dtype(dtype).name
        x, y, z = operands(dtype, 129, seed=29)
        out[f"x_{name}"], out[f"y_{name}"], out[f"z_{name}"] = x, y, z
        for which in list(range(7)) + [10, 11, 12, 13]:
            out[f"{which}_{name}"] = reference_elements(ref, which, (x, y, z), dtype)
    np.savez_compressed(ROOT / "tests" / "golden" / "elements.npz", **out)
    print("wrote tests/golden/elements.npz")


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "elements":
        elements()
    else:
        main()
