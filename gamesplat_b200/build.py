"""Build libgs_cuda.so (in-tree) with nvcc for sm_100a.

Every source under gamesplat_b200/csrc is compiled with
  -gencode arch=compute_100a,code=sm_100a -lineinfo -O3
and linked with the static CUDA runtime (and the system zlib, for the gsanim
archive reader) into gamesplat_b200/libgs_cuda.so.
Host C++ is compiled with -ffp-contract=off so host-side float results
(camera uniforms, PLY transforms) match the reference's host code.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG.parent / "_build"
LIB = PKG / "libgs_cuda.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def sources() -> list[Path]:
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _needs_build() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = sources() + list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + [PKG.parent / "include" / "gs_api.h"]
    return any(p.stat().st_mtime > t for p in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not _needs_build():
        return LIB
    BUILD.mkdir(exist_ok=True)
    cc = nvcc()
    common = ["-std=c++17", "-O3", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
              "-I", str(PKG.parent / "include")]

    def compile_one(src: Path) -> Path:
        obj = BUILD / (src.name + ".o")
        cmd = [cc, *ARCH, "-lineinfo", *common, "-c", str(src), "-o", str(obj)]
        if src.suffix == ".cu":
            cmd += ["-Xptxas", "-v"] if verbose else []
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stdout}\n{r.stderr}")
        if verbose and r.stderr:
            sys.stderr.write(r.stderr)
        return obj

    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(compile_one, sources()))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [cc, *ARCH, "-shared", "-cudart", "static", *[str(o) for o in objs], "-lz", "-o", str(tmp)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    tmp.replace(LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
