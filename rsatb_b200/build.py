"""Builds the sm_100a shared library ``rsatb_b200/_lib/librsatb_b200.so``.

Every ``csrc/*.cu`` file is compiled by nvcc for ``sm_100a`` only, in
parallel, into ``_build/``; the objects are linked into one shared library
with the C ABI of ``include/rsatb_b200.h``.  A translation unit is rebuilt
when it or any header under ``csrc/`` or ``include/`` is newer than its
object.  ``python -m rsatb_b200.build`` runs it from the command line.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OBJ_DIR = ROOT / "_build" / "obj"
LIB_DIR = PKG / "_lib"
LIB_PATH = LIB_DIR / "librsatb_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "-Xptxas", "-warn-spills",
]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found; the rsatb_b200 library needs the CUDA 12.9 toolkit")


def cuda_lib_dir() -> Path:
    return Path(nvcc_path()).resolve().parent.parent / "lib64"


def _headers_mtime() -> float:
    paths = list(CSRC.glob("*.cuh")) + list((ROOT / "include").glob("*.h"))
    return max((p.stat().st_mtime for p in paths), default=0.0)


def _compile(src: Path, obj: Path, extra: list[str]) -> tuple[Path, str]:
    cmd = [nvcc_path(), *ARCH, *NVCC_FLAGS, *extra, "-I", str(ROOT / "include"),
           "-c", str(src), "-o", str(obj)]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n{proc.stdout}\n{proc.stderr}")
    return obj, proc.stderr


def build(verbose: bool = False, force: bool = False, jobs: int | None = None) -> Path:
    """Compiles the changed translation units and relinks the library."""
    OBJ_DIR.mkdir(parents=True, exist_ok=True)
    LIB_DIR.mkdir(parents=True, exist_ok=True)
    hdr = _headers_mtime()
    sources = sorted(CSRC.glob("*.cu"))
    todo = []
    for src in sources:
        obj = OBJ_DIR / (src.stem + ".o")
        if force or not obj.exists() or obj.stat().st_mtime < max(src.stat().st_mtime, hdr):
            todo.append((src, obj))
    extra = ["-Xptxas", "-v"] if verbose else []
    if todo:
        n = jobs or min(len(todo), os.cpu_count() or 4)
        with cf.ThreadPoolExecutor(max_workers=n) as pool:
            futs = [pool.submit(_compile, s, o, extra) for s, o in todo]
            for f in futs:
                _, log = f.result()
                if verbose and log:
                    sys.stderr.write(log)
    objs = [OBJ_DIR / (s.stem + ".o") for s in sources]
    newest = max(o.stat().st_mtime for o in objs)
    if force or todo or not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < newest:
        libdir = cuda_lib_dir()
        cmd = [nvcc_path(), *ARCH, "-shared", "-o", str(LIB_PATH), *map(str, objs),
               "-L", str(libdir), "-lcufft",
               "-Xlinker", f"-rpath,{libdir}"]
        proc = subprocess.run(cmd, capture_output=True, text=True)
        if proc.returncode != 0:
            raise RuntimeError(f"link failed:\n{proc.stdout}\n{proc.stderr}")
    return LIB_PATH


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(LIB_PATH)
