"""Direct navigation on the GPU (dprop_propagate_direct): fp32 device runs
against the reference's direct-navigator propagation (fp64 oracle), chained
as a Kalman-filter step would chain them - the records of a device
propagation are the sequence of the direct run, and the last record of the
forward direct run starts the backward one.  Tolerances as in
test_gpu_parity."""
import numpy as np
import pytest

from tests.parity import compare
from tests.test_gpu_parity import COV_REL, TOL_ABS, TOL_REL

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _host(res):
    out = {k: v.cpu().numpy() for k, v in res.tensors.items()}
    out["rec_barcode"] = out["rec_barcode"].view(np.uint64)
    return out


@pytest.mark.parametrize("kind", ["toy", "wire_chamber_10l_cells"])
def test_direct_device_vs_oracle(torch_cuda, oracle, kind):
    from detray_b200 import abi, geometry, propagator, tracks
    from detray_b200.units import T
    torch = torch_cuda
    if kind == "toy":
        tables = geometry.load_geometry("toy_4brl_7edc")
        ref_det = oracle.build_toy()
        trk = tracks.toy_tracks(8000, seed=41, pt_range=(1.0, 50.0))
    else:
        tables = geometry.load_geometry(kind)
        ref_det = oracle.build_wire_chamber(square_cells=True)
        trk = tracks.toy_tracks(4000, seed=42, pt_range=(1.0, 50.0),
                                eta_range=(-1.0, 1.0), vertex_sigma=(0, 0, 0))
    det = propagator.Detector(tables)
    field = propagator.Field.constant((0.0, 0.0, 2.0 * T))
    cfg = abi.make_config(max_records=64, search_window=(3, 3),
                          estimate_scattering_noise=0)
    dev_trk = torch.tensor(trk, dtype=torch.float32, device="cuda")

    # sequence: the transported records of a device propagation
    seq_run = propagator.propagate(cfg, det, field, dev_trk)
    seq = seq_run.tensors["rec_barcode"]
    lens = torch.clamp(seq_run.tensors["n_records"], max=cfg.max_records)
    fw = propagator.propagate_direct(cfg, det, field, seq, lens, 1,
                                     tracks=dev_trk)
    torch.cuda.synchronize()
    seq_h = _host(seq_run)
    fw_h = _host(fw)
    lens_h = lens.cpu().numpy().astype(np.uint32)
    assert np.all(fw_h["status"] == abi.TRK_EXITED)
    same = [np.array_equal(fw_h["rec_barcode"][:lens_h[t], t],
                           seq_h["rec_barcode"][:lens_h[t], t])
            for t in range(len(lens_h))]
    assert np.mean(same) == 1.0

    fw_ref = oracle.propagate_direct(ref_det, field.spec, cfg,
                                     seq_h["rec_barcode"], lens_h, 1,
                                     tracks=trk)
    s = compare(fw_ref, fw_h, max_seq_mismatch_frac=0.0, tol_abs=TOL_ABS,
                tol_rel=TOL_REL, cov_rel=COV_REL)
    print(kind, "forward", s)

    # backward from the last record of the forward run
    idx = torch.arange(lens.shape[0], device="cuda")
    last = torch.clamp(lens.long() - 1, min=0)
    sbc = fw.tensors["rec_barcode"][last, idx].contiguous()
    sb = fw.tensors["rec_bound"][:, last, idx].contiguous()
    bw = propagator.propagate_direct(cfg, det, field, seq, lens, -1,
                                     start_barcode=sbc, start_bound=sb)
    torch.cuda.synchronize()
    bw_h = _host(bw)
    bw_ref = oracle.propagate_direct(
        ref_det, field.spec, cfg, seq_h["rec_barcode"], lens_h, -1,
        start_barcode=sbc.cpu().numpy().view(np.uint64),
        start_bound=sb.cpu().numpy().astype(np.float64))
    s = compare(bw_ref, bw_h, max_seq_mismatch_frac=0.0, tol_abs=TOL_ABS,
                tol_rel=TOL_REL, cov_rel=COV_REL)
    print(kind, "backward", s)
    p0 = 1 / np.abs(trk[7])
    np.testing.assert_allclose(1 / np.abs(bw_h["final_free"][7]), p0,
                               rtol=2e-3)


def test_direct_device_argument_checks(torch_cuda):
    from detray_b200 import abi, geometry, propagator, tracks
    from detray_b200.units import T
    torch = torch_cuda
    det = propagator.Detector(geometry.load_geometry("telescope_10x1m_300um"))
    field = propagator.Field.constant((0.0, 0.0, 2.0 * T))
    cfg = abi.make_config(max_records=16)
    seq = torch.zeros((16, 4), dtype=torch.int64, device="cuda")
    lens = torch.zeros(4, dtype=torch.int32, device="cuda")
    trk = torch.tensor(tracks.telescope_tracks(4, seed=1), dtype=torch.float32,
                       device="cuda")
    # empty sequences: every track ends at once without records
    res = propagator.propagate_direct(cfg, det, field, seq, lens, 1,
                                      tracks=trk)
    torch.cuda.synchronize()
    assert torch.all(res.tensors["status"] == abi.TRK_EXITED)
    assert torch.all(res.tensors["n_records"] == 0)
    with pytest.raises(propagator.PropagationError):
        propagator.propagate_direct(cfg, det, field, seq, lens, 2, tracks=trk)
    with pytest.raises(propagator.PropagationError):
        propagator.propagate_direct(cfg, det, field, seq, lens, 1)
