"""Build recipe for the phiray-b200 native library.

Compiles every CUDA source under ``csrc/`` for sm_100a and links them into
``libphiray_b200.so`` beside this file (in-tree, so the built library travels
with the repository snapshot). No floating-point contraction anywhere
(``--fmad=false``): the kernels compute each expression the way phiray's
shaders write it, which is what lets a CPU twin reproduce them bit for bit.

Usage: ``python -m phiray_b200.build [--verbose]``.
"""

from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
OUT = HERE / "libphiray_b200.so"
OBJ = HERE / "_build"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
HOST_CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build phiray-b200")


def flags(extra: list[str] | None = None) -> list[str]:
    f = [
        *ARCH,
        "-O3",
        "-lineinfo",
        "--fmad=false",
        "-std=c++17",
        "-ccbin",
        HOST_CXX,
        "-Xcompiler",
        "-fPIC,-ffp-contract=off",
        "-I",
        str(HERE.parent / "include"),
    ]
    if extra:
        f += extra
    return f


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(verbose: bool = False, force: bool = False, ptxas_info: bool = False) -> Path:
    OBJ.mkdir(exist_ok=True)
    headers = sorted(CSRC.glob("*.cuh")) + sorted((HERE.parent / "include").glob("*.h"))
    objs = []
    jobs = []
    for src in sources():
        obj = OBJ / (src.stem + ".o")
        objs.append(obj)
        if force or _stale(obj, [src, *headers]):
            extra = ["-Xptxas", "-v"] if ptxas_info else []
            jobs.append([nvcc(), *flags(extra), "-c", str(src), "-o", str(obj)])
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            results = list(ex.map(lambda c: subprocess.run(c, capture_output=True, text=True), jobs))
        for cmd, r in zip(jobs, results):
            if verbose or r.returncode != 0 or ptxas_info:
                sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
            if r.returncode != 0:
                raise RuntimeError(f"nvcc failed on {cmd[-3]}")
    if force or jobs or _stale(OUT, objs):
        link = [nvcc(), *ARCH, "-ccbin", HOST_CXX, "-shared", "-o", str(OUT), *map(str, objs), "-lcudart"]
        r = subprocess.run(link, capture_output=True, text=True)
        if verbose or r.returncode != 0:
            sys.stderr.write(" ".join(link) + "\n" + r.stdout + r.stderr)
        if r.returncode != 0:
            raise RuntimeError("link of libphiray_b200.so failed")
    return OUT


def build_test_probe(verbose: bool = False) -> Path:
    """The tests' device probe of the shared math (tests/mathprobe.cu) as
    tests/libmathprobe.so, with the library's flags. Test infrastructure:
    nothing in the package loads it."""
    src = HERE.parent / "tests" / "mathprobe.cu"
    out = src.with_name("libmathprobe.so")
    deps = [src, HERE.parent / "include" / "phiray_math.h"]
    if _stale(out, deps):
        cmd = [nvcc(), *flags(), "-shared", "-o", str(out), str(src), "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if verbose or r.returncode != 0:
            sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed on tests/mathprobe.cu")
    return out


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, force="--force" in sys.argv, ptxas_info="--ptxas" in sys.argv)
    print(OUT)
