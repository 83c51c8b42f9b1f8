"""Helix truth scan on the GPU (dprop_helix_scan) against the reference's
detector scan, and GPU-side navigation validation with it: the caching
navigator's surface sequence (all surfaces it reached, no material, so the
track stays on its helix) against the helix truth of the same tracks.

Tolerances: the fp64 scan runs the reference's iteration with the device's
math library, so it lands on the same surfaces and on paths equal to 1e-6
mm; the fp32 scan evaluates the helix in single precision, its roots are
good to a few um and a track grazing a mask edge (<= 0.5 %) may see a
different surface."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _host(scan):
    out = {k: v.cpu().numpy() for k, v in scan.items()
           if not k.startswith("_")}
    out["barcode"] = out["barcode"].view(np.uint64)
    out["volume_link"] = out["volume_link"].view(np.uint16)
    return out


def _compare(ref, got, path_tol):
    from detray_b200 import abi
    n = len(ref["status"])
    assert np.array_equal(ref["status"] == abi.SCAN_OK,
                          got["status"] == abi.SCAN_OK)
    same = np.zeros(n, dtype=bool)
    worst = 0.0
    for t in range(n):
        if ref["status"][t] != abi.SCAN_OK:
            same[t] = True
            continue
        k = ref["n_hits"][t]
        if got["n_hits"][t] != k or not np.array_equal(
                ref["barcode"][:k, t], got["barcode"][:k, t]):
            continue
        same[t] = True
        worst = max(worst, float(np.max(np.abs(
            ref["path"][:k, t] - got["path"][:k, t]))))
    assert worst <= path_tol, worst
    return same.mean(), worst


@pytest.mark.parametrize("kind", ["toy", "wire_chamber_10l_cells"])
def test_scan_device_vs_oracle(torch_cuda, oracle, kind):
    from detray_b200 import geometry, propagator, tracks
    from detray_b200.units import T
    torch = torch_cuda
    b = (0.0, 0.0, 2.0 * T)
    if kind == "toy":
        det = propagator.Detector(geometry.load_geometry("toy_4brl_7edc"))
        ref_det = oracle.build_toy()
        trk = tracks.toy_tracks(1000, seed=61, pt_range=(0.5, 50.0))
    else:
        det = propagator.Detector(geometry.load_geometry(kind))
        ref_det = oracle.build_wire_chamber(square_cells=True)
        trk = tracks.toy_tracks(1000, seed=62, pt_range=(0.5, 50.0),
                                eta_range=(-1.0, 1.0))
    ref = oracle.helix_scan(ref_det, b, trk, 1e-3)
    d64 = _host(propagator.helix_scan(
        det, b, torch.tensor(trk, dtype=torch.float64, device="cuda"), 1e-3))
    frac64, worst64 = _compare(ref, d64, 1e-6)
    d32 = _host(propagator.helix_scan(
        det, b, torch.tensor(trk, dtype=torch.float32, device="cuda"), 1e-3))
    frac32, worst32 = _compare(ref, d32, 5e-2)
    print(kind, "fp64 same", frac64, worst64, "fp32 same", frac32, worst32)
    assert frac64 >= 0.999
    assert frac32 >= 0.995


def test_navigation_validation(torch_cuda):
    """The caching navigator reaches the surfaces the helix crosses, in the
    same order: GPU propagation (RKN4, no material, every reached surface
    recorded) against the GPU fp64 helix scan of the same tracks."""
    from detray_b200 import abi, geometry, propagator, tracks
    from detray_b200.units import T
    torch = torch_cuda
    det = propagator.Detector(geometry.load_geometry("toy_4brl_7edc"))
    b = (0.0, 0.0, 2.0 * T)
    field = propagator.Field.constant(b)
    trk = tracks.toy_tracks(20000, seed=63, pt_range=(1.0, 100.0))
    cfg = abi.make_config(max_records=64, search_window=(3, 3),
                          use_material_interactor=0,
                          estimate_scattering_noise=0, record_all_surfaces=1)
    res = propagator.propagate(cfg, det, field,
                               torch.tensor(trk, dtype=torch.float32,
                                            device="cuda"))
    scan = propagator.helix_scan(
        det, b, torch.tensor(trk, dtype=torch.float64, device="cuda"), 1e-3)
    missed, extra = propagator.validate_navigation(scan, res,
                                                   cfg.max_records, 0.1)
    torch.cuda.synchronize()
    missed = missed.cpu().numpy()
    extra = extra.cpu().numpy()
    status = res.tensors["status"].cpu().numpy()
    good = (missed == 0) & (extra == 0)
    print("navigation validation: tracks without holes or extra surfaces",
          good.mean(), "missed", missed.sum(), "extra", extra.sum(),
          "exited", np.mean(status == abi.TRK_EXITED))
    assert good.mean() >= 0.98
