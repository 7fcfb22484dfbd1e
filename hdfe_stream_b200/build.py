"""Build libhdfe_b200.so, in-tree, for sm_100a (nvcc; no GPU needed).

    python -m hdfe_stream_b200.build          # or __graft_entry__.build()

Each csrc/*.cu compiles to an object under _build/ (in parallel), linked into
hdfe_stream_b200/libhdfe_b200.so; a file is recompiled only when it or a
header is newer than its object.
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
INCLUDE = PKG.parent / "include"
OUT = PKG / "libhdfe_b200.so"
BUILD = PKG / "_build"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         f"-I{INCLUDE}", f"-I{CSRC}"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise FileNotFoundError("nvcc not found (CUDA toolkit needed to build libhdfe_b200)")


def _headers_mtime() -> float:
    hs = list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    return max((h.stat().st_mtime for h in hs), default=0.0)


def build(verbose: bool = False, force: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    cc = nvcc()
    hdr = _headers_mtime()
    sources = sorted(CSRC.glob("*.cu"))
    jobs = []
    for src in sources:
        obj = BUILD / (src.stem + ".o")
        if force or not obj.exists() or obj.stat().st_mtime < max(src.stat().st_mtime, hdr):
            jobs.append((src, obj))

    def compile_one(job):
        src, obj = job
        cmd = [cc, *ARCH, *FLAGS, "-c", str(src), "-o", str(obj)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stderr}")
        if verbose and r.stderr.strip():
            print(r.stderr, file=sys.stderr)
        return src.name

    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        for name in ex.map(compile_one, jobs):
            if verbose:
                print(f"compiled {name}")
    objs = [str(BUILD / (s.stem + ".o")) for s in sources]
    newest = max((Path(o).stat().st_mtime for o in objs), default=0.0)
    if force or jobs or not OUT.exists() or OUT.stat().st_mtime < newest:
        tmp = OUT.with_suffix(".so.tmp")
        # the shared CUDA runtime (the one torch loads, when it is loaded first),
        # with the toolkit's copy as the fallback
        cmd = [cc, *ARCH, "-shared", "-o", str(tmp), *objs, "-cudart", "shared",
               "-Xlinker", "-rpath,/usr/local/cuda/lib64"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}")
        os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv))
