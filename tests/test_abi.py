"""The C ABI without a GPU: the library loads, exports every function
include/detray_b200/dprop.h declares, its structs have the layouts the
ctypes mirrors (detray_b200/abi.py) assume, and argument validation answers
before any device work."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

from detray_b200 import abi

REPO = Path(__file__).resolve().parent.parent
HEADER = REPO / "include" / "detray_b200" / "dprop.h"


@pytest.fixture(scope="module")
def lib():
    from detray_b200 import build, propagator
    build.build_library()
    return propagator.load_library()


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(dprop_\w+)\s*\(", text)))


def test_exports_every_declared_function(lib):
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    from detray_b200 import propagator
    assert sorted(propagator.ABI_SYMBOLS) == names


def test_version_and_defaults(lib):
    assert lib.dprop_abi_version() == abi.DPROP_ABI_VERSION
    c = abi.Config()
    lib.dprop_config_default(C.byref(c))
    ref = abi.make_config()
    for name, _ in abi.Config._fields_:
        a, b = getattr(c, name), getattr(ref, name)
        if hasattr(a, "__len__"):
            assert list(a) == list(b), name
        else:
            assert a == pytest.approx(b), name


STRUCTS = {
    "dprop_config": abi.Config,
    "dprop_tracks": abi.Tracks,
    "dprop_results": abi.Results,
    "dprop_launch": abi.Launch,
    "dprop_detector_desc": abi.DetectorDesc,
    "dprop_surface_desc": abi.SurfaceDesc,
    "dprop_mask_desc": abi.MaskDesc,
    "dprop_transform_desc": abi.TransformDesc,
    "dprop_slab_desc": abi.SlabDesc,
    "dprop_grid_desc": abi.GridDesc,
    "dprop_volume_desc": abi.VolumeDesc,
    "dprop_tape": abi.Tape,
    "dprop_gradients": abi.Gradients,
    "dprop_sequence": abi.Sequence,
    "dprop_scan_results": abi.ScanResults,
    "dprop_validation": abi.Validation,
}


def test_struct_layouts_match_ctypes(tmp_path):
    lines = ["#include <stdio.h>", "#include <stddef.h>",
             '#include "detray_b200/dprop.h"', "int main(void) {"]
    for cname, ct in STRUCTS.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in ct._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", '
                         f"offsetof({cname}, {fname}));")
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", f"-I{REPO / 'include'}", str(src),
                    "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True,
                         text=True).stdout.split("\n")
    got = {}
    for line in out:
        if line:
            s, f, v = line.split()
            got[(s, f)] = int(v)
    for cname, ct in STRUCTS.items():
        assert got[(cname, "size")] == C.sizeof(ct), cname
        for fname, _ in ct._fields_:
            assert got[(cname, fname)] == getattr(ct, fname).offset, \
                (cname, fname)


def test_argument_validation_without_device(lib):
    assert lib.dprop_propagate(None, None, None, None, None, None, 0,
                               None) == abi.DPROP_E_INVALID
    assert b"NULL" in lib.dprop_last_error()
    assert lib.dprop_propagate_adjoint(None, None, None, None, None, None,
                                       None, 0, None) == abi.DPROP_E_INVALID
    assert lib.dprop_backward(None, None, None, None, None, None, 0,
                              None) == abi.DPROP_E_INVALID
    # the energy-loss gradient is a valid configuration; the missing
    # detector is what fails
    cfg = abi.make_config(use_eloss_gradient=1)
    assert lib.dprop_propagate(C.byref(cfg), None, None, None, None, None, 1,
                               None) == abi.DPROP_E_INVALID
    assert lib.dprop_propagate_direct(None, None, None, None, None, None, 0,
                                      None) == abi.DPROP_E_INVALID
    assert lib.dprop_helix_scan(None, None, None, 0, 0.0, None,
                                None) == abi.DPROP_E_INVALID
    assert lib.dprop_validate_navigation(None, None, 4, 0, 0, 0.1, None,
                                         None) == abi.DPROP_E_INVALID
