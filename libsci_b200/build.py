"""Builds libsci_b200/libsci_cuda.so for sm_100a with nvcc (in-tree, so the library travels).

Usage: python -m libsci_b200.build [--jobs N]. Each .cu compiles to an object in parallel, then
one nvcc call links the shared library. Rebuilds only what changed (by modification time).
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
SOURCES = HERE / "csrc"
OBJECTS = HERE / "_build"
LIBRARY = HERE / "libsci_cuda.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]


def _headers() -> list[Path]:
    return sorted(SOURCES.glob("*.cuh")) + sorted(SOURCES.glob("*.hpp")) + [HERE.parent / "include" / "sci_cuda.h"]


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    stamp = target.stat().st_mtime
    return any(d.stat().st_mtime > stamp for d in deps if d.exists())


def build(jobs: int | None = None, verbose: bool = False) -> Path:
    OBJECTS.mkdir(exist_ok=True)
    headers = _headers()
    units = sorted(SOURCES.glob("*.cu"))
    todo = []
    for unit in units:
        obj = OBJECTS / (unit.stem + ".o")
        if _stale(obj, [unit] + headers):
            todo.append((unit, obj))

    def compile_one(item):
        unit, obj = item
        cmd = [NVCC, *ARCH, *FLAGS, "-c", str(unit), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        result = subprocess.run(cmd, capture_output=True, text=True)
        if result.returncode != 0:
            raise RuntimeError(f"nvcc failed on {unit.name}:\n{result.stderr}")
        return unit.name

    # The kernel source NVRTC specialises at run time, embedded in the library (specialize.cu).
    embedded = OBJECTS / "embedded_sources.cu"
    embedded_sources = [SOURCES / "sci_math.cuh", SOURCES / "chunk_kernel.cuh", SOURCES / "gradient_kernel.cuh",
                        SOURCES / "batch_kernel.cuh"]
    if _stale(embedded, embedded_sources):
        text = "// Generated by libsci_b200/build.py: the chunk kernel source NVRTC specialises.\n"
        symbols = ("sci_embedded_math", "sci_embedded_kernel", "sci_embedded_gradient", "sci_embedded_batch")
        for symbol, path in zip(symbols, embedded_sources):
            body = path.read_text()
            assert ")SCIEMBED\"" not in body
            text += f'extern const char *const {symbol} = R"SCIEMBED({body})SCIEMBED";\n'
        embedded.write_text(text)
    if _stale(OBJECTS / "embedded_sources.o", [embedded]):
        todo.append((embedded, OBJECTS / "embedded_sources.o"))

    with ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as pool:
        for name in pool.map(compile_one, todo):
            if verbose:
                print("compiled", name, flush=True)
    objects = [OBJECTS / (u.stem + ".o") for u in units] + [OBJECTS / "embedded_sources.o"]
    if _stale(LIBRARY, objects):
        cmd = [NVCC, *ARCH, "-shared", "-o", str(LIBRARY), *map(str, objects), "-cudart", "shared", "-lnvrtc",
               "-L/usr/local/cuda/lib64", "-L/usr/local/cuda/lib64/stubs"]
        if verbose:
            print(" ".join(cmd), flush=True)
        result = subprocess.run(cmd, capture_output=True, text=True)
        if result.returncode != 0:
            raise RuntimeError(f"linking libsci_cuda.so failed:\n{result.stderr}")
    return LIBRARY


if __name__ == "__main__":
    parser = argparse.ArgumentParser()
    parser.add_argument("--jobs", type=int, default=None)
    parser.add_argument("-v", "--verbose", action="store_true")
    args = parser.parse_args()
    print(build(args.jobs, args.verbose))
    sys.exit(0)
