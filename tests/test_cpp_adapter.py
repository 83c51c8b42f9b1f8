"""The C++ source-level drop-in (include/detray_b200/propagator.hpp):
dprop::propagator_adapter<metadata> with state(track, field_view, det) and
propagate(state, actor_states), as the reference's device test calls
propagator::propagate (tests/integration_tests/device/cuda/
propagator_cuda_kernel.cu:42-70).  A compiled C++ program
(tests/native/adapter_test.cpp) propagates a batch through it; its actor
states and propagator states must hold exactly what the ctypes path returns
for the same tracks."""
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parent.parent
LIB_DIR = REPO / "detray_b200" / "_lib"
SRC = REPO / "tests" / "native" / "adapter_test.cpp"
LIMIT2 = 600.0


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _compile(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    if not (LIB_DIR / "libdetray_b200.so").exists():
        pytest.skip("CUDA library not built")
    exe = tmp_path / "adapter_test"
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror",
           f"-I{REPO / 'include'}", str(SRC), f"-L{LIB_DIR}", "-ldetray_b200",
           f"-Wl,-rpath,{LIB_DIR}", "-o", str(exe)]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    assert proc.returncode == 0, proc.stderr
    return exe


def test_adapter_compiles_and_links(tmp_path):
    """The drop-in header compiles warning-free as C++17 against the C ABI
    header alone and links with the library."""
    _compile(tmp_path)


def test_raw_tables_round_trip(tmp_path):
    """geometry.write_raw_tables -> read_raw_tables is the identity (the C++
    reader reads the same layout)."""
    from detray_b200 import geometry
    t = geometry.load_geometry("toy_4brl_7edc")
    path = tmp_path / "toy.raw"
    geometry.write_raw_tables(t, path)
    u = geometry.read_raw_tables(path)
    for name, _ in geometry.TABLES:
        assert np.array_equal(t[name], u[name]), name


def _parse(data, n):
    off = 8
    n_exited = int(np.frombuffer(data[:8], np.uint64)[0])
    out = []
    for _ in range(n):
        u = np.frombuffer(data[off:off + 32], np.uint32)
        off += 32
        d = np.frombuffer(data[off:off + 8 * 9], np.float64)
        off += 72
        bsf = int(np.frombuffer(data[off:off + 8], np.uint64)[0])
        off += 8
        bvec = np.frombuffer(data[off:off + 48], np.float64)
        off += 48
        recs = []
        for _k in range(int(u[4])):
            bc = int(np.frombuffer(data[off:off + 8], np.uint64)[0])
            off += 8
            vals = np.frombuffer(data[off:off + 8 * 28], np.float64)
            off += 8 * 28
            fl = int(np.frombuffer(data[off:off + 4], np.uint32)[0])
            off += 4
            recs.append((bc, vals[:6], vals[6:27], vals[27], fl))
        out.append({"status": int(u[0]), "n_steps": int(u[1]),
                    "n_trials": int(u[2]), "n_records": int(u[3]),
                    "n_transports": int(u[5]), "n_material": int(u[6]),
                    "has_bound": bool(u[7]), "path_length": d[0],
                    "final": d[1:9], "bound_surface": bsf, "bound": bvec,
                    "records": recs})
    assert off == len(data)
    return n_exited, out


@pytest.mark.gpu
def test_adapter_matches_ctypes_path(tmp_path, torch_cuda):
    """Batch of 2000 toy tracks through the C++ adapter - half with the
    configuration's path limit, half with an aborter state of 600 mm - and
    the same tracks through dprop_propagate_host from Python with the same
    launch: status, counters, final parameters, every record and the
    updater's last bound parameters agree bit for bit; the first tracks run
    one propagate call each give the batch's results (checked inside the
    program)."""
    from detray_b200 import abi, geometry, propagator, tracks
    from detray_b200.units import T
    exe = _compile(tmp_path)
    n = 2000
    tables = geometry.load_geometry("toy_4brl_7edc")
    geometry.write_raw_tables(tables, tmp_path / "toy.raw")
    cfg = abi.make_config(max_records=32, search_window=(3, 3))
    (tmp_path / "cfg.bin").write_bytes(bytes(cfg))
    trk = np.ascontiguousarray(tracks.toy_tracks(n, seed=31), np.float64)
    (tmp_path / "trk.bin").write_bytes(trk.tobytes())
    proc = subprocess.run(
        [str(exe), str(tmp_path / "toy.raw"), str(tmp_path / "cfg.bin"),
         str(tmp_path / "trk.bin"), str(n), str(LIMIT2),
         str(tmp_path / "out.bin")], capture_output=True, text=True,
        timeout=600)
    assert proc.returncode == 0, proc.stderr
    n_exited, got = _parse((tmp_path / "out.bin").read_bytes(), n)

    det = propagator.Detector(tables)
    field = propagator.Field.constant((0.0, 0.0, 2.0 * T))
    lc = propagator.make_launch(method=abi.METHOD_PERSISTENT, sort_tracks=1)
    cfg2 = abi.make_config(max_records=32, search_window=(3, 3),
                           path_limit=LIMIT2)
    halves = [(0, n // 2, cfg), (n // 2, n, cfg2)]
    exited = 0
    for lo, hi, c in halves:
        ref = propagator.propagate_host(c, det, field, trk[:, lo:hi],
                                        launch=lc, jagged=True)
        offs = ref["rec_offsets"]
        for j in range(hi - lo):
            g = got[lo + j]
            assert g["status"] == ref["status"][j]
            exited += int(ref["status"][j] == abi.TRK_EXITED)
            assert g["n_steps"] == ref["n_steps"][j]
            assert g["n_trials"] == ref["n_trials"][j]
            assert g["n_records"] == ref["n_records"][j]
            assert g["n_transports"] == ref["n_transports"][j]
            assert g["n_material"] == ref["n_material"][j]
            assert g["path_length"] == np.float64(ref["path_length"][j])
            assert np.array_equal(g["final"],
                                  ref["final_free"][:, j].astype(np.float64))
            b, e = int(offs[j]), int(offs[j + 1])
            assert len(g["records"]) == e - b
            last = None
            for k, (bc, bnd, cov, path, fl) in enumerate(g["records"]):
                o = b + k
                assert bc == int(ref["rec_barcode"].reshape(-1)[o])
                assert np.array_equal(
                    bnd, ref["rec_bound"].reshape(6, -1)[:, o].astype(np.float64))
                assert np.array_equal(
                    cov, ref["rec_cov"].reshape(21, -1)[:, o].astype(np.float64))
                assert path == np.float64(ref["rec_path"].reshape(-1)[o])
                assert fl == int(ref["rec_flags"].reshape(-1)[o])
                if fl & 1:
                    last = (bc, bnd)
            assert g["has_bound"] == (last is not None)
            if last is not None:
                assert g["bound_surface"] == last[0]
                assert np.array_equal(g["bound"], last[1])
    assert n_exited == exited
    # the 600 mm aborter stops tracks the default limit lets through
    short = [g["status"] for g in got[n // 2:]]
    assert short.count(abi.TRK_PATH_LIMIT) > 0
