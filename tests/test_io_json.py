"""Detector JSON reader (detray_b200.io_json) against the reference's own
JSON IO: files written by detray::io::write_detector must give the tables
dprop::flatten produces from what detray::io::read_detector builds out of
the same files.  Every table is byte-identical except the inverse
placements, which the reference inverts numerically (4x4) and the reader as
R^T, -R^T t: those agree to 1e-14 relative."""
import json
from pathlib import Path

import numpy as np
import pytest

from tests.parity import compare

GOLDEN = Path(__file__).resolve().parent / "golden" / "json_telescope"


def assert_tables_match(ref: dict, got: dict):
    from detray_b200 import geometry
    for name, _ in geometry.TABLES:
        a, b = ref[name], got[name]
        assert a.shape == b.shape, name
        if name != "transforms":
            assert a.tobytes() == b.tobytes(), name
            continue
        assert a["rot"].tobytes() == b["rot"].tobytes()
        assert a["translation"].tobytes() == b["translation"].tobytes()
        np.testing.assert_allclose(b["inv_rot"], a["inv_rot"], rtol=0,
                                   atol=1e-14)
        # the error of -R^T t scales with |t| in every component
        scale = 1.0 + np.linalg.norm(a["translation"], axis=1)[:, None]
        assert np.all(np.abs(b["inv_translation"] - a["inv_translation"])
                      <= 1e-14 * scale)


def test_golden_telescope_files():
    """Committed fixture: the reference writer's telescope files and the
    tables its reader builds from them."""
    from detray_b200 import geometry, io_json
    ref = geometry.load_npz(GOLDEN / "tables.npz")
    got = io_json.read_detector(sorted(GOLDEN.glob("*.json")))
    assert_tables_match(ref, got)
    assert len(got["surfaces"]) == 16 and len(got["slabs"]) == 10


@pytest.fixture(scope="module")
def json_oracle(oracle):
    if not oracle.json_available():
        pytest.skip("reference JSON IO tool not built")
    return oracle


@pytest.mark.parametrize("kind", ["telescope", "wire_cells", "wire_straws",
                                  "toy", "toy_maps"])
def test_reader_matches_reference_reader(json_oracle, tmp_path, kind):
    from detray_b200 import io_json
    files = json_oracle.write_json(kind, tmp_path / kind)
    ref = json_oracle.read_json_tables(kind, files, tmp_path / "ref.bin")
    got = io_json.read_detector(files)
    assert_tables_match(ref, got)


def test_json_detector_propagates_like_reference_tables(core_host, json_oracle,
                                                       tmp_path):
    """The few-ulp difference of the inverse placements does not change the
    propagation: fp64 host core on the reader's tables against the same core
    on the reference reader's tables, toy detector with material maps."""
    from detray_b200 import abi, geometry, io_json, tracks
    from tests.test_core_host_parity import run_core, TIGHT
    files = json_oracle.write_json("toy_maps", tmp_path / "toy")
    ref_t = json_oracle.read_json_tables("toy_maps", files, tmp_path / "r.bin")
    got_t = io_json.read_detector(files)
    cfg = abi.make_config(max_records=32, search_window=(3, 3))
    trk = tracks.toy_tracks(1500, seed=21)
    ref = run_core(core_host, json_oracle, geometry.Descriptor(ref_t).desc,
                   cfg, trk, 8)
    got = run_core(core_host, json_oracle, geometry.Descriptor(got_t).desc,
                   cfg, trk, 8)
    assert ref["n_records"].mean() > 5
    s = compare(ref, got, max_seq_mismatch_frac=0.0, tol_abs=TIGHT,
                tol_rel=1e-9, cov_rel=1e-7)
    assert s["seq_mismatch"] == 0 and s["status_mismatch"] == 0


@pytest.mark.gpu
def test_json_detector_on_device(json_oracle, core_host, tmp_path):
    """A detector loaded from JSON runs on the GPU: fp32 device propagation
    on the reader's tables (toy detector with material maps) against the
    fp64 host core on the reference reader's tables."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from detray_b200 import abi, geometry, io_json, propagator, tracks
    from detray_b200.units import T
    from tests.test_core_host_parity import run_core
    from tests.test_gpu_parity import COV_REL, TOL_ABS, TOL_REL
    files = json_oracle.write_json("toy_maps", tmp_path / "toy")
    ref_t = json_oracle.read_json_tables("toy_maps", files, tmp_path / "r.bin")
    det = propagator.Detector(io_json.read_detector(files))
    field = propagator.Field.constant((0.0, 0.0, 2.0 * T))
    cfg = abi.make_config(max_records=32, search_window=(3, 3))
    trk = tracks.toy_tracks(5000, seed=22)
    ref = run_core(core_host, json_oracle, geometry.Descriptor(ref_t).desc,
                   cfg, trk, 8)
    dev = torch.tensor(trk, dtype=torch.float32, device="cuda")
    res = propagator.propagate(cfg, det, field, dev)
    torch.cuda.synchronize()
    got = {k: v.cpu().numpy() for k, v in res.tensors.items()}
    got["rec_barcode"] = got["rec_barcode"].view(np.uint64)
    compare(ref, got, max_seq_mismatch_frac=1e-3, tol_abs=TOL_ABS,
            tol_rel=TOL_REL, cov_rel=COV_REL)


# ------------------------------------------------------------ error handling
def _write(path: Path, doc: dict) -> str:
    path.write_text(json.dumps(doc))
    return str(path)


def _geometry_doc(shape=5, index_in_coll=(0, 1)):
    ident = {"translation": [0.0, 0.0, 0.0],
             "rotation": [1.0, 0, 0, 0, 1.0, 0, 0, 0, 1.0]}
    surfaces = []
    for k, idx in enumerate(index_in_coll):
        surfaces.append({
            "type": 1, "source": 0, "transform": ident,
            "masks": [{"shape": shape, "volume_link": 0,
                       "boundaries": [10.0, 10.0]}],
            "index_in_coll": idx})
    return {"header": {"common": {"version": "", "detector": "d", "date": "",
                                  "tag": "geometry"}},
            "data": {"volumes": [{"name": "v", "index": 0, "type": 0,
                                  "transform": ident,
                                  "surfaces": surfaces}]}}


def test_reader_rejects_bad_input(tmp_path):
    from detray_b200 import io_json
    ok = _write(tmp_path / "ok.json", _geometry_doc())
    t = io_json.read_detector([ok])
    assert len(t["surfaces"]) == 2 and len(t["transforms"]) == 3
    # annulus (shape id 0) is not on the propagation path
    bad = _write(tmp_path / "annulus.json", _geometry_doc(shape=0))
    with pytest.raises(ValueError, match="shape"):
        io_json.read_detector([bad])
    # surface indices that leave a hole
    bad = _write(tmp_path / "hole.json", _geometry_doc(index_in_coll=(0, 2)))
    with pytest.raises(ValueError, match="holes"):
        io_json.read_detector([bad])
    # no geometry file, unknown tag, two geometry files
    mat = {"header": {"common": {"version": "", "detector": "d", "date": "",
                                 "tag": "homogeneous_material"}},
           "data": None}
    mat_f = _write(tmp_path / "mat.json", mat)
    with pytest.raises(ValueError, match="geometry"):
        io_json.read_detector([mat_f])
    other = dict(mat, header={"common": dict(mat["header"]["common"],
                                             tag="volume_grids")})
    with pytest.raises(ValueError, match="tag"):
        io_json.read_detector([ok, _write(tmp_path / "o.json", other)])
    with pytest.raises(ValueError, match="two files"):
        io_json.read_detector([ok, ok])
    # material for a surface that does not exist
    mat["data"] = {"volumes": [{"volume_link": 0, "surface_material": [{
        "type": 6, "surface_idx": 5, "thickness": 1.0,
        "material": {"params": [93.7, 465.2, 28.03, 14.0, 0.002329, 0.0,
                                1.0]}}]}]}
    mat_f = _write(tmp_path / "mat2.json", mat)
    with pytest.raises(ValueError, match="missing surface"):
        io_json.read_detector([ok, mat_f])
