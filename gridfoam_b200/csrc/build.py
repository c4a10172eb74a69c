"""Build the gridfoam_b200 CUDA library in-tree for sm_100a.

``python -m gridfoam_b200.csrc.build`` compiles every ``*.cu`` file of this
directory with nvcc into ``gridfoam_b200/_lib/libgridfoam_b200.so``.  The
CUDA runtime is linked statically so the library only needs the driver.
"""

from __future__ import annotations

import os
import pathlib
import shutil
import subprocess
import sys

HERE = pathlib.Path(__file__).resolve().parent
PKG = HERE.parent
REPO = PKG.parent
LIB_DIR = PKG / "_lib"
LIB_PATH = LIB_DIR / "libgridfoam_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and pathlib.Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found; set NVCC or put the CUDA toolkit on PATH")


def sources() -> list[pathlib.Path]:
    return sorted(HERE.glob("*.cu"))


def needs_build() -> bool:
    if not LIB_PATH.exists():
        return True
    mtime = LIB_PATH.stat().st_mtime
    deps = sources() + sorted(HERE.glob("*.cuh")) + [REPO / "include" / "gridfoam_b200.h"]
    return any(p.stat().st_mtime > mtime for p in deps)


def build(verbose: bool = False, force: bool = False) -> pathlib.Path:
    """Compile the shared library (no-op when it is up to date)."""
    if not force and not needs_build():
        return LIB_PATH
    LIB_DIR.mkdir(exist_ok=True)
    obj_dir = LIB_DIR / "obj"
    obj_dir.mkdir(exist_ok=True)
    nvcc = nvcc_path()
    common = [
        "-O3",
        "-lineinfo",
        "-std=c++17",
        "-Xcompiler",
        "-fPIC",
        "-I",
        str(REPO / "include"),
        *ARCH,
    ]
    if verbose:
        common += ["-Xptxas", "-v"]
    from concurrent.futures import ThreadPoolExecutor

    objs = [obj_dir / (src.stem + ".o") for src in sources()]

    def compile_one(pair):
        src, obj = pair
        subprocess.run([nvcc, *common, "-dc", str(src), "-o", str(obj)], check=True)

    # The translation units are independent (relocatable device code,
    # linked below), so they compile in parallel.
    with ThreadPoolExecutor(max_workers=max(1, min(len(objs), os.cpu_count() or 1))) as pool:
        list(pool.map(compile_one, zip(sources(), objs)))
    tmp = LIB_PATH.with_suffix(".so.tmp")
    cmd = [nvcc, *ARCH, "-shared", "-cudart", "static", "-o", str(tmp), *map(str, objs)]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    path = build(verbose="-v" in sys.argv, force=True)
    print(path)
