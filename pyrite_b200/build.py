"""Build ``libpyrite_b200.so`` in-tree with nvcc for sm_100a.

Usage: ``python -m pyrite_b200.build`` (or ``__graft_entry__.build()``).
Each translation unit compiles separately (parallel), then links into one
shared library with the CUDA runtime linked statically, so the library loads
through ctypes with no other CUDA library on the path.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
SRC = PKG / "csrc"
OUT_DIR = PKG / "_lib"
LIB = OUT_DIR / "libpyrite_b200.so"
INCLUDE = PKG.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
          f"-I{INCLUDE}"]
# Transport keeps IEEE separate multiply and add so its FP64 path replays the
# reference's event decisions; the scorers may contract.
PER_FILE = {
    "pb_transport.cu": ["-fmad=false"],
}
SOURCES = ["pb_capi.cu", "pb_transport.cu", "pb_cxr.cu", "pb_brem.cu", "pb_brem_node.cu", "pb_char.cu", "pb_mlp.cu", "pb_coherent.cu"]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build pyrite_b200")
    return cand


def _stale(obj: Path, src: Path) -> bool:
    if not obj.exists():
        return True
    deps = [src, *SRC.glob("*.cuh"), *SRC.glob("*.h"), *INCLUDE.glob("*.h")]
    return any(d.stat().st_mtime > obj.stat().st_mtime for d in deps)


def build(verbose: bool = False, force: bool = False) -> Path:
    OUT_DIR.mkdir(exist_ok=True)
    objdir = OUT_DIR / "obj"
    objdir.mkdir(exist_ok=True)
    cc = nvcc()
    jobs = []
    for name in SOURCES:
        src = SRC / name
        obj = objdir / (name + ".o")
        if force or _stale(obj, src):
            cmd = [cc, *ARCH, *COMMON, *PER_FILE.get(name, []), "-c", str(src), "-o", str(obj)]
            jobs.append((name, cmd))
    if jobs:
        with ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4)) as ex:
            results = list(ex.map(lambda j: (j[0], subprocess.run(j[1], capture_output=True, text=True)), jobs))
        for name, r in results:
            if verbose or r.returncode != 0:
                sys.stderr.write(r.stdout + r.stderr)
            if r.returncode != 0:
                raise RuntimeError(f"nvcc failed on {name}")
    objs = [str(objdir / (n + ".o")) for n in SOURCES]
    if force or jobs or not LIB.exists():
        cmd = [cc, *ARCH, "-shared", "-o", str(LIB), *objs, "-cudart", "static"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("nvcc link failed")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="--force" in sys.argv))
