"""Extract the reference's own known-answer data into tests/golden/reference_pins.json.

Reads Kraken.jl's test and benchmark sources as text (it does not run them)
and copies the literal arrays the hot-path tests check against:
  - Ghia et al. centreline u at Re=100 (test/test_cavity.jl, "Cavity 2D Re=100")
  - the reduced Ghia set of the MRT test (test/test_mrt.jl)
  - De Vahl Davis Nusselt numbers (hpc/natconv_gpu.jl, DE_VAHL_DAVIS)
  - the measured natural-convection Nu quoted in test/test_thermal.jl

Run in a checkout that has the reference tree:
    python tests/golden/make_golden.py /path/to/Kraken.jl
"""
from __future__ import annotations

import json
import re
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent


def _array(src: str, name: str, start: int = 0) -> tuple[list[float], int]:
    m = re.compile(rf"{name}\s*=\s*\[([^\]]*)\]", re.S).search(src, start)
    if not m:
        raise ValueError(f"{name} not found")
    vals = [float(t) for t in re.split(r"[,\s]+", m.group(1).strip()) if t]
    return vals, m.end()


def main(ref: Path) -> None:
    cav = (ref / "test" / "test_cavity.jl").read_text()
    gy, end = _array(cav, "ghia_y")
    gu, _ = _array(cav, "ghia_u", end)
    mrt = (ref / "test" / "test_mrt.jl").read_text()
    my, end = _array(mrt, "ghia_y")
    mu, _ = _array(mrt, "ghia_u", end)
    hpc = (ref / "hpc" / "natconv_gpu.jl").read_text()
    m = re.search(r"DE_VAHL_DAVIS\s*=\s*Dict\(([^)]*)\)", hpc)
    dvd = {k: float(v) for k, v in re.findall(r"([\d.e+-]+)\s*=>\s*([\d.]+)", m.group(1))}
    th = (ref / "test" / "test_thermal.jl").read_text()
    nu_ref = float(re.search(r"Nu_ref\s*=\s*([\d.]+)", th).group(1))
    out = {
        "source": "Kraken.jl test/test_cavity.jl, test/test_mrt.jl, test/test_thermal.jl, "
                  "hpc/natconv_gpu.jl (literal arrays copied by tests/golden/make_golden.py)",
        "ghia_re100": {"y": gy, "u": gu},
        "ghia_re100_mrt": {"y": my, "u": mu},
        "de_vahl_davis_nu": {str(int(float(k))): v for k, v in dvd.items()},
        "natconv_ra1e3_nu_ref": nu_ref,
    }
    (HERE / "reference_pins.json").write_text(json.dumps(out, indent=1) + "\n")
    print("wrote", HERE / "reference_pins.json")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path to the Kraken.jl source tree>")
    main(Path(sys.argv[1]))
