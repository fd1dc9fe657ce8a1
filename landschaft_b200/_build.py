"""Build of the native library (``liblsb_omni.so``) for sm_100a, in-tree.

``nvcc`` cross-compiles without a GPU.  The library is written next to this
file so that it travels with the source tree.
"""

from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB = PKG / "liblsb_omni.so"
SOURCES = ([CSRC / "omni_capi.cu", CSRC / "omni_adv.cu", CSRC / "omni_win_128_hot.cu", CSRC / "graph_pairs.cu",
            CSRC / "graph_solve.cu"] +
           [CSRC / f"omni_win_{nt}_{kind}.cu" for nt in (256, 512) for kind in ("hot", "gen")])
DEPS = SOURCES + sorted(CSRC.glob("*.cuh")) + [PKG.parent / "include" / "lsb_omniscape.h"]

NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build landschaft_b200")


def up_to_date() -> bool:
    if not LIB.exists():
        return False
    t = LIB.stat().st_mtime
    return all(p.stat().st_mtime <= t for p in DEPS if p.exists())


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile ``liblsb_omni.so`` unless it is newer than its sources (translation units in parallel)."""
    if not force and up_to_date():
        return LIB
    from concurrent.futures import ThreadPoolExecutor

    objdir = PKG / "_build"
    objdir.mkdir(exist_ok=True)
    nv = nvcc()

    def compile_one(src: Path):
        obj = objdir / (src.stem + ".o")
        cmd = [nv, *NVCC_FLAGS, "-c", "-o", str(obj), str(src)]
        if verbose:
            cmd += ["-Xptxas", "-v"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        return src, obj, r

    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        results = list(ex.map(compile_one, SOURCES))
    for src, _, r in results:
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src.name} ({r.returncode}):\n{r.stderr[-4000:]}")
        if verbose and r.stderr:
            print(r.stderr)
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nv, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", str(tmp), *(str(o) for _, o, _ in results)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed ({r.returncode}):\n{r.stderr[-4000:]}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force=True, verbose=True))
