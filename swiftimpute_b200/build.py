"""Build the in-tree native library ``swiftimpute_b200/lib/libswiftimpute_b200.so``.

nvcc compiles every ``csrc/*.cu`` / ``csrc/*.cpp`` for sm_100a only and links
one shared library next to the package, so it travels with the source tree.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB_DIR = PKG / "lib"
OBJ_DIR = PKG / "_build"
LIB = LIB_DIR / "libswiftimpute_b200.so"

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3",
                  "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]
CXXFLAGS = ["-O3", "-std=c++17", "-fPIC"]


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} {cmd[-1]}")
    if r.stderr.strip():
        sys.stderr.write(r.stderr)


def sources() -> list[Path]:
    return sorted([*CSRC.glob("*.cu"), *CSRC.glob("*.cpp")])


def build(verbose: bool = False, force: bool = False) -> Path:
    OBJ_DIR.mkdir(exist_ok=True)
    LIB_DIR.mkdir(exist_ok=True)
    headers = [*CSRC.glob("*.hpp"), *CSRC.glob("*.cuh"), *(PKG.parent / "include").glob("*.h"),
               *(PKG.parent / "include").glob("**/*.hpp")]
    newest_header = max((h.stat().st_mtime for h in headers), default=0.0)
    objs = []
    for src in sources():
        obj = OBJ_DIR / (src.name + ".o")
        objs.append(obj)
        if (not force and obj.exists() and obj.stat().st_mtime > src.stat().st_mtime
                and obj.stat().st_mtime > newest_header):
            continue
        if src.suffix == ".cu":
            cmd = [NVCC, *CUFLAGS, "-I", str(PKG.parent / "include"), "-c", str(src), "-o", str(obj)]
        else:
            cmd = [os.environ.get("CXX", "g++"), *CXXFLAGS, "-I", str(PKG.parent / "include"),
                   "-I", str(Path(os.environ.get("CUDA_HOME", "/usr/local/cuda")) / "include"),
                   "-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd))
        _run(cmd)
    if force or not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart"]
        if verbose:
            print(" ".join(cmd))
        _run(cmd)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
