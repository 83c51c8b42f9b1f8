"""Extract the reference's known-answer vectors for the propagation path
into JSON fixtures (run where the reference checkout exists; the fixtures
are committed so the tests do not need it):

  bethe_pdg.json  muon mean dE/dx against the PDG tables, the cases of
                  tests/unit_tests/cpu/material/bethe_equation.cpp (the
                  instantiations that are commented out there are skipped:
                  the reference does not meet its 5 % bound on them).
  telescope_smoke.npz  the surface sequence of the smoke test's telescope
                  sample from the reference propagator.
  json_telescope/ the reference's JSON writer output for the 10-plane
                  telescope (geometry + homogeneous material) and
                  tables.npz, dprop::flatten of what the reference's JSON
                  reader builds from those files (needs oracle/_ref/ref_json).

Usage: python tests/golden/make_golden.py [reference checkout]
"""
from __future__ import annotations

import json
import os
import re
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent


def strip_comments_keep_lines(text: str) -> str:
    """Blank out /* */ and // comments, keeping line numbers."""
    def blank(m):
        return re.sub(r"[^\n]", " ", m.group(0))
    text = re.sub(r"/\*.*?\*/", blank, text, flags=re.S)
    return re.sub(r"//[^\n]*", blank, text)


def bethe_cases(ref: Path) -> list[dict]:
    rel = "tests/unit_tests/cpu/material/bethe_equation.cpp"
    text = strip_comments_keep_lines((ref / rel).read_text())
    pat = re.compile(
        r"make_tuple\(\s*(\w+)<scalar>\(\)\s*,\s*(\w+)<scalar>\(\)\s*,\s*"
        r"([0-9.eE+-]+)f\s*\*\s*unit<scalar>::GeV\s*,\s*([0-9.eE+-]+)f\s*\)",
        re.S)
    out = []
    for m in pat.finditer(text):
        line = text.count("\n", 0, m.start()) + 1
        out.append({"material": m.group(1), "particle": m.group(2),
                    "p_gev": float(m.group(3)),
                    "dedx_mev_cm2_per_g": float(m.group(4)),
                    "source": f"{rel}:{line}"})
    return out


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    ref = Path(argv[0]) if argv else Path(os.environ.get("DETRAY_REF", ""))
    if not (ref / "tests").exists():
        raise SystemExit("give the reference checkout: make_golden.py PATH "
                         "or DETRAY_REF=PATH")
    cases = bethe_cases(ref)
    (HERE / "bethe_pdg.json").write_text(json.dumps(cases, indent=1) + "\n")
    print(f"bethe_pdg.json: {len(cases)} cases")
    json_fixture(HERE / "json_telescope")
    smoke_fixture(HERE / "telescope_smoke.npz")


def smoke_fixture(out: Path) -> None:
    """Surface sequence of the smoke test's telescope sample (256 muons,
    seed 7, 2 T) from the reference propagator: __graft_entry__.smoke()
    checks against it where the oracle library is not built."""
    import numpy as np
    sys.path.insert(0, str(HERE.parent.parent))
    from oracle import ref_oracle
    from detray_b200 import abi, tracks
    from detray_b200.units import T
    if not ref_oracle.available("f64"):
        print("oracle not built: smoke fixture not written")
        return
    cfg = abi.make_config(max_records=16)
    trk = tracks.telescope_tracks(256, seed=7)
    ref = ref_oracle.propagate(ref_oracle.build_telescope(),
                               {"kind": "const", "b": (0.0, 0.0, 2.0 * T)},
                               cfg, trk)
    np.savez_compressed(out, rec_barcode=ref["rec_barcode"][:10])
    print(f"{out.name}: {ref['rec_barcode'][:10].shape}")


def json_fixture(out: Path) -> None:
    import tempfile
    sys.path.insert(0, str(HERE.parent.parent))
    from oracle import ref_oracle
    from detray_b200 import geometry
    if not ref_oracle.json_available():
        print("oracle/_ref/ref_json missing: JSON fixture not written")
        return
    files = ref_oracle.write_json("telescope", out)
    # the writer stamps today's date into the headers: keep the fixture
    # stable by blanking it
    for f in files:
        doc = json.loads(Path(f).read_text())
        doc["header"]["common"]["date"] = ""
        Path(f).write_text(json.dumps(doc, indent=1) + "\n")
    with tempfile.TemporaryDirectory() as tmp:
        tables = ref_oracle.read_json_tables("telescope", files,
                                             Path(tmp) / "t.bin")
    geometry.save_npz(tables, out / "tables.npz")
    print(f"{out.name}: {[Path(f).name for f in files]} + tables.npz")


if __name__ == "__main__":
    main()
