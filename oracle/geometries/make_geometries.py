"""Regenerate the committed benchmark geometries (build-time step, not part
of the product).

Compiles export_geometry.cpp against the detray headers of a reference
checkout (path given by --ref or $DETRAY_REF) and the vecmem stand-in
oracle/shim, and packs the tables of the benchmark detectors into the
compressed .npz files the product loads (detray_b200/geometries/):

  toy_4brl_7edc.npz          toy barrel + endcap detector, 4 barrel layers,
                             7 endcap discs per side, 0.15 mm Si modules
  toy_4brl_7edc_maps.npz     the same with the builder's material maps on
                             the portals (20 x 20 bins on cylinders, 5 x 20
                             on discs)
  telescope_10x1m_300um.npz  10 1 m x 1 m Si planes normal to x at
                             x = 0, 50, ..., 450 mm, 0.3 mm thick
  wire_chamber_10l_cells.npz wire chamber: 10 layers of 10 mm square drift
                             cells from r = 500 mm, 1 m half length, 50 mrad
                             stereo angle, 15 um tungsten wires
  wire_chamber_10l_straws.npz the same with circular straw tubes
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
OUT = REPO / "detray_b200" / "geometries"
sys.path.insert(0, str(REPO))

from detray_b200 import geometry  # noqa: E402

GEOMETRIES = {
    "toy_4brl_7edc": ["toy", "4", "7", "0.15"],
    "toy_4brl_7edc_maps": ["toy", "4", "7", "0.15", "maps"],
    "telescope_10x1m_300um": ["telescope", "500", "500", "0.3"],
    "wire_chamber_10l_cells": ["wire", "10", "1", "0.015"],
    "wire_chamber_10l_straws": ["wire", "10", "0", "0.015"],
}
TELESCOPE_POSITIONS = [str(50.0 * i) for i in range(10)]


def build_exporter(ref: Path, out: Path) -> None:
    cmd = ["g++", "-std=c++20", "-O3", "-march=x86-64-v3", "-w", "-DDETRAY_ALGEBRA_ARRAY=1",
           "-DDETRAY_CUSTOM_SCALARTYPE=double", f"-I{HERE.parent / 'shim'}",
           f"-I{ref / 'core/include'}",
           f"-I{ref / 'plugins/algebra/array/include'}",
           f"-I{ref / 'detectors/include'}", f"-I{ref / 'tests/include'}",
           f"-I{ref / 'io/include'}", f"-I{REPO / 'include'}",
           str(HERE / "export_geometry.cpp"), "-o", str(out)]
    subprocess.run(cmd, check=True)


def main() -> None:
    args = sys.argv[1:]
    ref = (Path(args[args.index("--ref") + 1]) if "--ref" in args
           else Path(os.environ.get("DETRAY_REF", "")))
    if not (ref / "core" / "include" / "detray").exists():
        raise SystemExit("give the reference checkout: --ref PATH or "
                         "DETRAY_REF=PATH")
    with tempfile.TemporaryDirectory() as tmp:
        exe = Path(tmp) / "export_geometry"
        build_exporter(ref, exe)
        for name, args in GEOMETRIES.items():
            raw = Path(tmp) / f"{name}.bin"
            extra = TELESCOPE_POSITIONS if args[0] == "telescope" else args[4:]
            subprocess.run([str(exe), *args[:4], str(raw), *extra], check=True)
            tables = geometry.read_raw_tables(raw)
            geometry.save_npz(tables, OUT / f"{name}.npz")
            print(f"wrote {name}.npz: "
                  + ", ".join(f"{k}={len(v)}" for k, v in tables.items()))


if __name__ == "__main__":
    main()
