"""Build the parity oracle (test infrastructure) into oracle/_build/.

    gcc -O2 -ffp-contract=off -fopenmp -fPIC -shared kb_oracle.c -lm

-ffp-contract=off keeps every multiply and add separately rounded, as the
reference's Julia CPU path does.  The shared object is used only by tests/,
the smoke check and the CPU-baseline leg of bench.py.

The reference (Kraken.jl) is Julia; there is no C/C++ source in it to
compile into oracle/_ref, so this restatement is the only CPU oracle.
"""
from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "kb_oracle.c"
OUT = HERE / "_build" / "libkboracle.so"


def build(force: bool = False) -> Path:
    OUT.parent.mkdir(exist_ok=True)
    if not force and OUT.exists() and OUT.stat().st_mtime >= SRC.stat().st_mtime:
        return OUT
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        raise RuntimeError("no C compiler found to build the oracle")
    tmp = OUT.with_suffix(".so.tmp")
    cmd = [cc, "-O2", "-std=c11", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC",
           "-shared", str(SRC), "-o", str(tmp), "-lm"]
    subprocess.run(cmd, check=True)
    tmp.replace(OUT)
    return OUT


if __name__ == "__main__":
    print(build(force=True))
