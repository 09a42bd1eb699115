"""In-tree build of the engine (libpspin.so), its drivers and the oracle.

    python -m cuda_pspin_b200.build          # everything
    python -m cuda_pspin_b200.build --lib    # libpspin.so only

Outputs stay inside the repository (cuda_pspin_b200/lib, cuda_pspin_b200/bin,
oracle/liboracle.so) so that they travel with the source tree.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "lib")
BIN_DIR = os.path.join(HERE, "bin")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")
HOST_CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

LIB_SOURCES = ["abi.cu", "sweep.cu", "pt.cu", "setup.cu", "noalloc.cu", "sweep_cluster.cu", "sweep_multi.cu", "sweep_resident.cu", "analysis.cu", "tcfield.cu", "learned.cu", "cube.cu", "layout.cpp"]


def cutlass_dir() -> str:
    """The CUTLASS 4 header tree (sm100 collectives) for tcfield.cu: the
    CUTLASS_DIR environment variable, else the copy the flashinfer package
    ships under its data directory (located without importing it)."""
    d = os.environ.get("CUTLASS_DIR")
    where = "CUTLASS_DIR"
    if not d:
        import importlib.util
        spec = importlib.util.find_spec("flashinfer")
        if spec is not None and spec.origin:
            d = os.path.join(os.path.dirname(spec.origin), "data", "cutlass")
            where = "the flashinfer package's data/cutlass"
    if not d or not os.path.isfile(os.path.join(d, "include", "cutlass", "cutlass.h")):
        raise RuntimeError(f"CUTLASS headers not found (looked at {where}: {d!r}); set CUTLASS_DIR to a "
                           "CUTLASS 4.x checkout containing include/cutlass/cutlass.h")
    return d


def reference_dir() -> str:
    """The reference checkout (giacomotrinca/cuda_pspin) that the oracle's
    reference rebuild compiles from: PSPIN_REF, else /root/reference."""
    return os.environ.get("PSPIN_REF", "/root/reference")


DRIVERS = {
    "pspin_pt": ["drivers/pt_main.cpp"],
    "pspin_pt_sparse": ["drivers/pt_sparse_main.cpp"],
    "pspin_mc": ["drivers/mc_main.cpp"],
    "pspin_sa": ["drivers/sa_main.cpp"],
    "pspin_smoothed_cube": ["drivers/cube_main.cpp"],
}


def _run(cmd: list[str]) -> None:
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build_lib(force: bool = False) -> str:
    """Compiles every source to an object under _build/ (skipped when newer
    than the source and the shared headers) and links libpspin.so."""
    os.makedirs(LIB_DIR, exist_ok=True)
    obj_dir = os.path.join(ROOT, "_build", "obj")
    os.makedirs(obj_dir, exist_ok=True)
    out = os.path.join(LIB_DIR, "libpspin.so")
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(ROOT, "include", "pspin.h"))
    cutlass = cutlass_dir()
    flags = [NVCC, "-O3", "-std=c++17", *ARCH, "-lineinfo", "-ccbin", HOST_CXX,
             f"-I{cutlass}/include", f"-I{cutlass}/tools/util/include", "--expt-relaxed-constexpr",
             "-diag-suppress", "20012", "-Xcompiler", "-fPIC,-fopenmp,-O3"]
    if os.environ.get("PSPIN_PTXAS_V"):
        flags += ["-Xptxas", "-v"]
    objs = []
    for f in LIB_SOURCES:
        src = os.path.join(CSRC, f)
        obj = os.path.join(obj_dir, f + ".o")
        objs.append(obj)
        if force or _newer(obj, [src, *headers]):
            _run([*flags, "-c", src, "-o", obj])
    if force or _newer(out, objs):
        _run([NVCC, *ARCH, "-ccbin", HOST_CXX, "-shared", "-o", out, *objs, "-lcurand", "-lgomp",
              "-Xlinker", f"-rpath,{CUDA}/lib64"])
    return out


def build_drivers(force: bool = False) -> None:
    os.makedirs(BIN_DIR, exist_ok=True)
    lib = os.path.join(LIB_DIR, "libpspin.so")
    common = [os.path.join(CSRC, "drivers", "common.cpp")]
    for name, srcs in DRIVERS.items():
        paths = [os.path.join(CSRC, s) for s in srcs]
        if not all(os.path.exists(p) for p in paths):
            continue
        out = os.path.join(BIN_DIR, name)
        deps = paths + common + [lib, os.path.join(CSRC, "drivers", "common.h")]
        if not force and not _newer(out, deps):
            continue
        _run([HOST_CXX, "-O2", "-std=c++17", "-Wall", f"-I{ROOT}/include", f"-I{CSRC}/drivers",
              *paths, *common, "-o", out, f"-L{LIB_DIR}", "-lpspin",
              f"-Wl,-rpath,$ORIGIN/../lib", f"-Wl,-rpath,{CUDA}/lib64"])


def build_oracle(force: bool = False) -> None:
    odir = os.path.join(ROOT, "oracle")
    out = os.path.join(odir, "liboracle.so")
    deps = [os.path.join(odir, "oracle.c"), os.path.join(odir, "oracle.h")]
    if not force and not _newer(out, deps):
        return
    _run(["make", "-C", odir, "liboracle.so"])


def build_ref() -> None:
    """Reference rebuild for sm_100a under oracle/_ref (only where the
    reference sources are present)."""
    ref = reference_dir()
    if not os.path.isdir(os.path.join(ref, "src")):
        return
    if shutil.which("make") is None:
        return
    _run(["make", "-C", os.path.join(ROOT, "oracle"), "ref", "compat", f"PSPIN_REF={ref}"])


def main(argv: list[str] | None = None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--lib", action="store_true")
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--no-ref", action="store_true")
    a = ap.parse_args(argv)
    build_lib(a.force)
    if a.lib:
        return 0
    build_drivers(a.force)
    build_oracle(a.force)
    if not a.no_ref:
        build_ref()
    return 0


if __name__ == "__main__":
    sys.exit(main())
