"""GPU: adjoint-mode propagation and the reverse sweep through the C ABI
(dprop_propagate_adjoint, dprop_backward) and the PyTorch autograd binding.

The derivative math is checked on CPU against finite differences and the
reference's Jacobians (test_adjoint_host.py, double precision).  Here the
device implementation (float32) is checked against that double-precision
host core on the same tracks and loss:
  * records: same surfaces for all but <= 0.2 % of the tracks;
  * dL/d(initial parameters): |d| <= 2e-3 |g| + 1e-3 * rms(g) per component
    (float32 Jacobian chains of up to ~20 surfaces);
  * dL/d(alignment): per surface |d| <= 2e-3 |g| + 1e-3 * rms(g).
"""
import numpy as np
import pytest

from tests import adjoint_host as ah

pytestmark = pytest.mark.gpu

# device float32 gradient against fp64 finite differences: relative, with a
# floor of 1e-3 of the component's rms
TOL_FD = 5e-3


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _setup(kind, n):
    from detray_b200 import abi, geometry, propagator, tracks
    from detray_b200.units import T
    if kind == "telescope":
        tables = geometry.load_geometry("telescope_10x1m_300um")
        cfg = abi.make_config(max_records=16)
        trk = tracks.telescope_tracks(n, seed=31)
        trk[0] += 5.0
    else:
        tables = geometry.load_geometry("toy_4brl_7edc")
        cfg = abi.make_config(max_records=32, search_window=(3, 3))
        trk = tracks.toy_tracks(n, seed=32, pt_range=(1.0, 20.0),
                                eta_range=(-3.0, 3.0))
    det = propagator.Detector(tables)
    field = propagator.Field.constant((0.0, 0.0, 2.0 * T))
    return tables, det, field, cfg, trk


def _device_adjoint(torch, cfg, det, field, trk, W, sort=1):
    from detray_b200 import adjoint, propagator
    dev = torch.tensor(trk, dtype=torch.float32, device="cuda")
    rec = adjoint.propagate_adjoint(cfg, det, field, dev,
                                    launch=propagator.make_launch(sort_tracks=sort))
    gb = torch.tensor(W, dtype=torch.float32, device="cuda")
    gfree, galign = adjoint.backward(cfg, det, rec, gb)
    torch.cuda.synchronize()
    res = {k: v.cpu().numpy() for k, v in rec.results.tensors.items()}
    res["rec_barcode"] = res["rec_barcode"].view(np.uint64)
    return rec, res, gfree.cpu().numpy(), galign.cpu().numpy()


def _close(got, want, rel=2e-3, rms_frac=1e-3):
    scale = np.sqrt(np.mean(want ** 2)) + 1e-30
    return np.abs(got - want) <= rel * np.abs(want) + rms_frac * scale


@pytest.mark.parametrize("kind,n", [("telescope", 2000), ("toy", 4000)])
def test_device_gradients_match_host_core(torch_cuda, core_host, kind, n):
    tables, det, field, cfg, trk = _setup(kind, n)
    href, htape = ah.forward(core_host, tables, cfg, trk)
    W = ah.random_weights(href, cfg.max_records, seed=7)
    hfree, halign = ah.backward(core_host, tables, cfg, trk, href, htape, W)
    _, dres, dfree, dalign = _device_adjoint(torch_cuda, cfg, det, field, trk, W)
    same = ah.same_records(href, {"n_records": dres["n_records"].astype(np.uint32),
                                  "rec_barcode": dres["rec_barcode"]})
    assert same.mean() >= 0.998, same.mean()
    # every gradient component of every track whose records agree, within
    # the tolerance (measured on B200: worst 6.7e-4 relative)
    for i in (0, 1, 2, 3, 4, 5, 6, 7):
        ok = _close(dfree[i][same], hfree[i][same])
        assert ok.all(), (i, int((~ok).sum()))
    # alignment: only tracks whose records agree contribute on the host side;
    # redo the host sweep without the others
    Wm = W * same[None, None, :]
    _, halign_m = ah.backward(core_host, tables, cfg, trk, href, htape, Wm)
    _, _, _, dalign_m = _device_adjoint(torch_cuda, cfg, det, field, trk, Wm)
    hit = np.abs(halign_m).sum(axis=1) > 0
    assert hit.sum() >= 5
    ok = _close(dalign_m[hit], halign_m[hit])
    assert ok.all(), int((~ok).sum())


def test_adjoint_mode_keeps_the_propagation(torch_cuda):
    """Adjoint mode records the same surfaces and parameters as the normal
    propagation (it only adds the tape).  Scattering-noise estimation is off:
    it reads the covariance, which adjoint mode transports without the
    reference's first-surface quirk, and may then move a mask edge."""
    from detray_b200 import propagator
    tables, det, field, cfg, trk = _setup("toy", 4000)
    cfg.estimate_scattering_noise = 0
    W = np.zeros((6, cfg.max_records, trk.shape[1]), dtype=np.float32)
    _, ares, _, _ = _device_adjoint(torch_cuda, cfg, det, field, trk, W)
    dev = torch_cuda.tensor(trk, dtype=torch_cuda.float32, device="cuda")
    nres = propagator.propagate(cfg, det, field, dev,
                                launch=propagator.make_launch(sort_tracks=1))
    torch_cuda.cuda.synchronize()
    n = {k: v.cpu().numpy() for k, v in nres.tensors.items()}
    n["rec_barcode"] = n["rec_barcode"].view(np.uint64)
    same = ah.same_records(ares, n) & (ares["status"] == n["status"])
    assert same.mean() >= 0.999, same.mean()
    m = ah.transported_mask({"n_records": n["n_records"],
                             "rec_flags": n["rec_flags"]}, cfg.max_records)
    m &= same[None, :]
    np.testing.assert_allclose(ares["rec_bound"][:, m], n["rec_bound"][:, m],
                               rtol=1e-5, atol=1e-5)


def test_autograd_matches_backward(torch_cuda):
    """torch.autograd through propagate_differentiable equals the direct
    reverse sweep, for a residual loss on loc0/loc1 with alignment."""
    from detray_b200 import adjoint, propagator
    torch = torch_cuda
    tables, det, field, cfg, trk = _setup("telescope", 1000)
    tracks = torch.tensor(trk, dtype=torch.float32, device="cuda",
                          requires_grad=True)
    align = torch.zeros((det.n_surfaces, 6), dtype=torch.float64,
                        device="cuda", requires_grad=True)
    lc = propagator.make_launch(sort_tracks=1)
    rec, mask = adjoint.propagate_differentiable(cfg, det, field, tracks,
                                                 align, lc)
    gen = torch.Generator(device="cuda").manual_seed(3)
    targets = rec[:2].detach() + 0.01 * torch.randn(
        rec[:2].shape, device="cuda", generator=gen)
    loss = (((rec[:2] - targets) ** 2) * mask[None]).sum()
    loss.backward()
    grad_bound = torch.zeros_like(rec)
    grad_bound[:2] = 2.0 * (rec[:2] - targets).detach() * mask[None]
    arec = adjoint.propagate_adjoint(cfg, det, field, tracks.detach(), lc)
    gfree, galign = adjoint.backward(cfg, det, arec, grad_bound)
    torch.cuda.synchronize()
    torch.testing.assert_close(tracks.grad, gfree, rtol=1e-5, atol=1e-6)
    torch.testing.assert_close(align.grad, galign, rtol=1e-4, atol=1e-7)
    assert float(align.grad.abs().sum()) > 0.0
    with pytest.raises(propagator.PropagationError):
        adjoint.propagate_differentiable(cfg, det, field, tracks,
                                         align.detach() + 1.0, lc)


def test_adjoint_edge_cases(torch_cuda):
    """Empty batch, a track that records nothing, missing arrays."""
    import ctypes as C
    from detray_b200 import abi, adjoint, propagator
    torch = torch_cuda
    tables, det, field, cfg, trk = _setup("telescope", 4)
    lib = propagator.load_library()
    tape = abi.Tape()
    res = propagator.alloc_device_results(0, cfg.max_records)
    ts = abi.Tracks()
    assert lib.dprop_propagate_adjoint(C.byref(cfg), None, det.handle,
                                       field.handle, C.byref(ts),
                                       C.byref(res.struct), C.byref(tape), 0,
                                       None) == abi.DPROP_OK
    dev = torch.tensor(trk, dtype=torch.float32, device="cuda")
    dev[4:7, 0] = torch.tensor([-1.0, 0.0, 0.0])   # leaves the telescope
    rec = adjoint.propagate_adjoint(cfg, det, field, dev)
    gb = torch.ones((6, cfg.max_records, 4), device="cuda")
    gfree, galign = adjoint.backward(cfg, det, rec, gb)
    torch.cuda.synchronize()
    g = gfree.cpu().numpy()
    if int(rec.results.tensors["n_records"][0]) == 0:
        assert np.all(g[:, 0] == 0.0)
    assert np.all(np.isfinite(g))
    bad = abi.Tape()
    r = propagator.alloc_device_results(4, cfg.max_records)
    rc = lib.dprop_propagate_adjoint(C.byref(cfg), None, det.handle,
                                     field.handle,
                                     C.byref(propagator.tracks_struct(dev)),
                                     C.byref(r.struct), C.byref(bad), 4, None)
    assert rc == abi.DPROP_E_INVALID


def test_device_gradients_in_field_map_match_finite_differences(torch_cuda,
                                                                core_host):
    """Benchmark configuration 4 in small: the toy detector in the solenoid
    field map with use_field_gradient (the transport Jacobian carries the
    field's gradient).  The device's float32 gradients with respect to the
    initial position, direction and q/p, for a random linear loss on the
    recorded bound parameters, against fp64 central finite differences of
    the host core's forward propagation, every component of every track
    whose records agree (steps capped at 2 mm so that the landing error of
    the forward stays below the tolerance)."""
    from detray_b200 import abi, fields, geometry, propagator, tracks
    from tests.test_adjoint_host import STEPS, _analytic, _perturbed
    fmap = fields.solenoid_map()
    tables = geometry.load_geometry("toy_4brl_7edc")
    det = propagator.Detector(tables)
    field = propagator.Field.grid(fmap)
    cfg = abi.make_config(max_records=32, search_window=(3, 3),
                          step_constraint=2.0, use_field_gradient=1)
    trk = tracks.toy_tracks(48, seed=12, pt_range=(0.5, 50.0),
                            eta_range=(-2.5, 2.5), pt_log_uniform=False)
    href, _ = ah.forward(core_host, tables, cfg, trk, field=fmap)
    W = ah.random_weights(href, cfg.max_records, seed=3)
    _, dres, dfree, _ = _device_adjoint(torch_cuda, cfg, det, field, trk, W)
    same_dev = ah.same_records(
        href, {"n_records": dres["n_records"].astype(np.uint32),
               "rec_barcode": dres["rec_barcode"]})
    checked = 0
    worst = 0.0
    for which in (0, 1, 2, "phi", "theta", 7):
        h = STEPS[which]
        rp, _ = ah.forward(core_host, tables, cfg, _perturbed(trk, which, h),
                           field=fmap, adjoint=False)
        rm, _ = ah.forward(core_host, tables, cfg, _perturbed(trk, which, -h),
                           field=fmap, adjoint=False)
        ok = ah.same_records(rp, rm) & same_dev
        fd = ah.loss_difference(rp, rm, W) / (2 * h)
        an = _analytic(dfree.astype(np.float64), trk, which)
        scale = np.sqrt(np.mean(fd[ok] ** 2)) + 1e-30
        err = np.abs(an - fd)[ok] / (np.abs(fd[ok]) + 1e-3 * scale)
        print(which, float(err.max()))
        worst = max(worst, float(err.max()))
        checked += int(ok.sum())
        assert (err < TOL_FD).all(), (which, float(err.max()))
    assert checked >= 6 * 40
    print("worst", worst)
