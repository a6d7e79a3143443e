"""Build recipe for the in-tree shared libraries.

* ``lib/libg4b200.so``  -- the sm_100a CUDA kernels behind the C ABI of
  ``include/g4b.h`` (nvcc, ``-gencode arch=compute_100a,code=sm_100a``).
* ``lib/libg4host.so``  -- the C++ host layer (reference-shaped classes,
  deck/lattice parsing, beam loading, the step driver) linked against
  ``libg4b200.so``.

nvcc cross-compiles for sm_100a without a GPU.  Object files are rebuilt only
when a source or header is newer than the object.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
HOST = CSRC / "host"
LIB = PKG / "lib"
OBJ = PKG / "_build"
INCLUDE = ROOT / "include"

NVCC = os.environ.get("G4B_NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
CXX = "/usr/bin/g++"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
    "-ccbin", CXX, "--expt-relaxed-constexpr", "-I", str(INCLUDE),
]
CXX_FLAGS = ["-O2", "-fPIC", "-std=c++17", "-Wall", "-I", str(INCLUDE),
             "-I", "/usr/local/cuda/include"]

DEVICE_LIB = LIB / "libg4b200.so"
HOST_LIB = LIB / "libg4host.so"


def _newer(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build step failed:\n" + " ".join(map(str, cmd)) +
                           "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def build_device(verbose_ptxas: bool = False) -> Path:
    """Compile every csrc/*.cu for sm_100a and link libg4b200.so."""
    OBJ.mkdir(exist_ok=True)
    LIB.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    sources = sorted(CSRC.glob("*.cu"))
    jobs = []
    for src in sources:
        obj = OBJ / (src.stem + ".o")
        if _newer(obj, [src] + headers):
            flags = list(NVCC_FLAGS)
            if verbose_ptxas:
                flags += ["-Xptxas", "-v"]
            jobs.append([NVCC, *flags, "-c", str(src), "-o", str(obj)])
    logs = []
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            logs = list(ex.map(_run, jobs))
    objs = [OBJ / (s.stem + ".o") for s in sources]
    if jobs or _newer(DEVICE_LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-o", str(DEVICE_LIB), *map(str, objs),
              "-ccbin", CXX])
    if verbose_ptxas:
        for log in logs:
            print(log)
    return DEVICE_LIB


def build_host() -> Path:
    """Compile csrc/host/*.cpp into libg4host.so linked to libg4b200.so."""
    if not HOST.exists():
        return HOST_LIB
    OBJ.mkdir(exist_ok=True)
    sources = sorted(HOST.glob("*.cpp"))
    headers = list(HOST.glob("*.h")) + list(INCLUDE.glob("*.h"))
    objs = []
    jobs = []
    for src in sources:
        obj = OBJ / ("host_" + src.stem + ".o")
        objs.append(obj)
        if _newer(obj, [src] + headers):
            jobs.append([CXX, *CXX_FLAGS, "-c", str(src), "-o", str(obj)])
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            list(ex.map(_run, jobs))
    if objs and (jobs or _newer(HOST_LIB, objs + [DEVICE_LIB])):
        _run([CXX, "-shared", "-o", str(HOST_LIB), *map(str, objs),
              "-L", str(LIB), "-lg4b200", "-Wl,-rpath,$ORIGIN"])
    return HOST_LIB


def build_all(verbose_ptxas: bool = False) -> None:
    build_device(verbose_ptxas)
    build_host()


if __name__ == "__main__":
    import sys
    build_all(verbose_ptxas="-v" in sys.argv)
    print("built", DEVICE_LIB, HOST_LIB)
