"""In-tree build of the sm_100a library and the mriSolver executable.

    python impatient-mri_b200/build.py          # incremental
    python impatient-mri_b200/build.py --clean

Produces
    impatient-mri_b200/libimpatient_b200.so   (C-ABI: include/impatient_b200.h)
    impatient-mri_b200/bin/mriSolver          (the reference's command line)
Objects go to impatient-mri_b200/_build/.  Only nvcc and the system g++ are used.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INC = PKG.parent / "include"
BUILD = PKG / "_build"
LIB = PKG / "libimpatient_b200.so"
EXE = PKG / "bin" / "mriSolver"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                     "-Xcompiler", "-Wall", "-ccbin", "g++"]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-Wall"]


def _cuda_home() -> Path:
    env = os.environ.get("CUDA_HOME") or os.environ.get("CUDA_PATH")
    if env:
        return Path(env)
    nvcc = shutil.which("nvcc")
    return Path(nvcc).resolve().parent.parent if nvcc else Path("/usr/local/cuda")


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + sorted(INC.glob("*.h"))


def _stale(obj: Path, src: Path) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(p.stat().st_mtime > t for p in [src, *_headers(), Path(__file__)])


def _compile(src: Path, verbose: bool) -> Path:
    obj = BUILD / (src.name + ".o")
    if not _stale(obj, src):
        return obj
    cuda = _cuda_home()
    if src.suffix == ".cu":
        cmd = [str(cuda / "bin" / "nvcc"), *NVCC_FLAGS, "-c", str(src), "-o", str(obj)]
    else:
        cmd = ["g++", *CXX_FLAGS, f"-I{cuda / 'include'}", "-c", str(src), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {src.name}\n{r.stdout}\n{r.stderr}")
    return obj


def build(verbose: bool = False, jobs: int | None = None) -> Path:
    BUILD.mkdir(exist_ok=True)
    (PKG / "bin").mkdir(exist_ok=True)
    srcs = sorted(CSRC.glob("*.cu")) + [p for p in sorted(CSRC.glob("*.cpp"))
                                         if p.name != "mriSolver_main.cpp"]
    with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    cuda = _cuda_home()
    newest = max(o.stat().st_mtime for o in objs)
    if not LIB.exists() or LIB.stat().st_mtime < newest:
        cmd = [str(cuda / "bin" / "nvcc"), *ARCH, "-shared", "-o", str(LIB), *map(str, objs),
               f"-L{cuda / 'lib64'}", f"-Xlinker=-rpath,{cuda / 'lib64'}",
               "-lcudart_static", "-lrt", "-ldl", "-lpthread", "-ccbin", "g++"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed\n{r.stdout}\n{r.stderr}")
    main_src = CSRC / "mriSolver_main.cpp"
    if not EXE.exists() or EXE.stat().st_mtime < LIB.stat().st_mtime or _stale(EXE, main_src):
        cmd = ["g++", "-O2", "-std=c++17", str(main_src), "-o", str(EXE), f"-L{PKG}",
               "-limpatient_b200", "-Wl,-rpath,$ORIGIN/.."]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"mriSolver link failed\n{r.stdout}\n{r.stderr}")
    return LIB


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--clean", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    if a.clean and BUILD.exists():
        shutil.rmtree(BUILD)
    print(build(verbose=a.verbose))
    return 0


if __name__ == "__main__":
    sys.exit(main())
