"""Build the product library libp3miden_b200.so in-tree with nvcc (sm_100a).

Usage: python build.py  (or import and call build()).
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
OUT = HERE / "libp3miden_b200.so"

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC,-fvisibility=hidden,-O2",
    "--expt-relaxed-constexpr",
    "-shared",
]


def sources():
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.cpp")) + sorted(CSRC.glob("*.h"))


GEN_GL = CSRC / "gen_gl_src.inc"


def write_generated() -> None:
    """Embed gl.cuh's text as a C++ raw string (gen_gl_src.inc): the prelude of
    the constraint kernels the library generates and compiles at run time
    with NVRTC (csrc/symair.cuh)."""
    src = (CSRC / "gl.cuh").read_text()
    assert ")P3GGL\"" not in src
    text = 'R"P3GGL(' + src + ')P3GGL"\n'
    if not GEN_GL.exists() or GEN_GL.read_text() != text:
        GEN_GL.write_text(text)


def needs_build() -> bool:
    if not OUT.exists() or not GEN_GL.exists():
        return True
    t = OUT.stat().st_mtime
    return any(s.stat().st_mtime > t for s in sources())


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not needs_build():
        return OUT
    write_generated()
    nvcc = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
    cmd = [nvcc, *NVCC_FLAGS, "-o", str(OUT), str(CSRC / "p3g_all.cu"), str(CSRC / "lde_noalloc.cu"), "-lcudart",
           "-lnvrtc", "-Xlinker", "-rpath,/usr/local/cuda/lib64"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(OUT)
