"""Build libkrakenb200.so (sm_100a) in tree with nvcc.

The library is plain CUDA C++ behind the C ABI of include/krakenb200.h; it
links the CUDA runtime statically and has no torch dependency.  Translation
units that restate the reference arithmetic are compiled with --fmad=false
(no multiply-add contraction, so FP64 results match the reference's CPU path
bit for bit); the precision-tier units keep FMA.

    python krakenn.jl_b200/build.py          # incremental
    python krakenn.jl_b200/build.py --force  # rebuild everything
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
INCLUDE = PKG.parent / "include"
BUILD = PKG / "_build"
LIB = PKG / "libkrakenb200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
          "--expt-relaxed-constexpr", f"-I{INCLUDE}"]

# unit -> extra flags
UNITS = {
    "kb_error.cu": [],
    "kb_d2q9.cu": ["--fmad=false"],
    "kb_d3q19.cu": ["--fmad=false"],
    "kb_d3q19_dev.cu": [],
    "kb_reduce.cu": [],
    "kb_batch.cu": [],
    "kb_graph.cu": [],
    "kb_umma.cu": [],
    "kb_surrogate.cu": [],
}


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libkrakenb200.so")
    return cand


def _deps(unit: Path) -> list[Path]:
    return [unit] + sorted(CSRC.glob("*.cuh")) + [INCLUDE / "krakenb200.h"]


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _compile(unit: str, flags: list[str], verbose: bool) -> Path:
    src = CSRC / unit
    obj = BUILD / (src.stem + ".o")
    cmd = [nvcc(), *ARCH, *COMMON, *flags, "-c", str(src), "-o", str(obj)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {unit}:\n{res.stdout}\n{res.stderr}")
    if verbose and res.stderr:
        sys.stderr.write(res.stderr)
    return obj


def build(force: bool = False, verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    jobs = {}
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        for unit, flags in UNITS.items():
            obj = BUILD / (Path(unit).stem + ".o")
            if force or verbose or _stale(obj, _deps(CSRC / unit)):
                jobs[unit] = ex.submit(_compile, unit, flags, verbose)
        for unit, fut in jobs.items():
            fut.result()
    objs = [BUILD / (Path(u).stem + ".o") for u in UNITS]
    if force or jobs or _stale(LIB, objs):
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", str(tmp), *map(str, objs)]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true", help="print ptxas register/spill report")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))
