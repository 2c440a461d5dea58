"""Builds the device FIM library (libressim_fim.so) in-tree for sm_100a with nvcc.

Each source compiles to an object in ressim_b200/_build/ in parallel (only the ones whose source
or headers changed), then one nvcc call links the shared object."""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "libressim_fim.so")
SOURCES = ["rf_assembly.cu", "rf_linear.cu", "rf_direct.cu", "rf_state.cu", "rf_api.cu", "rf_noalloc.cu",
           "rf_blackoil.cu", "rf_adjoint.cu", "rf_level.cu", "rf_fiber.cu"]
COMPILE_FLAGS = [
    "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
    "-Xcompiler", "-fPIC", "--fmad=false", "-Xptxas", "-O3",
]
LINK_FLAGS = ["-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-cudart", "static"]


def _headers() -> list[str]:
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if not f.endswith(".cu")]
    hs.append(os.path.join(HERE, "..", "include", "ressim_fim.h"))
    return hs


def _obj(src: str) -> str:
    return os.path.join(OBJ, src.replace(".cu", ".o"))


def _stale(src: str, newest_header: float) -> bool:
    o = _obj(src)
    if not os.path.exists(o):
        return True
    t = os.path.getmtime(o)
    return os.path.getmtime(os.path.join(CSRC, src)) > t or newest_header > t


def needs_build() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "ressim_fim.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    if not force and not needs_build():
        return OUT
    nvcc = os.environ.get("NVCC", "nvcc")
    os.makedirs(OBJ, exist_ok=True)
    newest = max(os.path.getmtime(h) for h in _headers())
    todo = [s for s in SOURCES if force or _stale(s, newest)]

    def compile_one(src: str) -> None:
        cmd = [nvcc, *COMPILE_FLAGS, "-c", os.path.join(CSRC, src), "-o", _obj(src)]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)

    if todo:
        with ThreadPoolExecutor(max_workers=max(1, min(len(todo), os.cpu_count() or 1))) as ex:
            for f in [ex.submit(compile_one, s) for s in todo]:
                f.result()
    cmd = [nvcc, *LINK_FLAGS, "-o", OUT, *[_obj(s) for s in SOURCES]]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv))
