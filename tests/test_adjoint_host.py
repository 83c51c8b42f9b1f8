"""Reverse-mode derivatives through the propagation, on CPU (test-only host
build of the core, double precision).

* The surface-to-surface Jacobians on the adjoint tape equal the reference's
  own (the per-step factors of the full Jacobian its parameter transporter
  accumulates, propagator/actors/parameter_updater.hpp:369-381).
* dL/d(initial parameters) and dL/d(alignment) of a random linear loss on the
  recorded bound parameters agree with central finite differences of the
  propagation.  The forward ends its last step before a surface at the
  straight-line distance to it and accepts the point within the navigation
  tolerance, while the Jacobians (the reference's) describe the exact helix
  intersection.  The landing point misses the surface by about the step's
  sagitta projected on the normal, L^2 / (2 R) for a step L on a helix of
  radius R, so the finite difference of the forward carries a term of that
  size (0.075 mm for a 50 mm step at R = 16.7 m, i.e. 8 % of the rotation
  derivative of a plane hit 1 mm from its centre).  The finite-difference
  tests therefore cap the step length (stepping.step_constraint), which makes
  the landing error negligible; the adjoint itself does not depend on it.
"""
import ctypes as C

import numpy as np
import pytest

from detray_b200 import abi, alignment, geometry, tracks
from tests import adjoint_host as ah

T = 0.000299792458


def _angles(trk):
    d = trk[4:7]
    phi = np.arctan2(d[1], d[0])
    th = np.arctan2(np.hypot(d[0], d[1]), d[2])
    return phi, th


def _perturbed(trk, which, h):
    t = trk.copy()
    if which in (0, 1, 2, 7):
        t[which] += h
        return t
    phi, th = _angles(t)
    if which == "phi":
        phi = phi + h
    else:
        th = th + h
    t[4:7] = np.stack([np.cos(phi) * np.sin(th), np.sin(phi) * np.sin(th),
                       np.cos(th)])
    return t


def _analytic(gfree, trk, which):
    if which in (0, 1, 2, 7):
        return gfree[which]
    phi, th = _angles(trk)
    if which == "phi":
        dd = np.stack([-np.sin(phi) * np.sin(th), np.cos(phi) * np.sin(th),
                       0.0 * th])
    else:
        dd = np.stack([np.cos(phi) * np.cos(th), np.sin(phi) * np.cos(th),
                       -np.sin(th)])
    return (gfree[4:7] * dd).sum(axis=0)


STEPS = {0: 1e-4, 1: 1e-4, 2: 1e-4, "phi": 1e-7, "theta": 1e-7, 7: 1e-9}


def _fd_initial(core_host, tables, cfg, trk, W, which):
    h = STEPS[which]
    rp, _ = ah.forward(core_host, tables, cfg, _perturbed(trk, which, h),
                       adjoint=False)
    rm, _ = ah.forward(core_host, tables, cfg, _perturbed(trk, which, -h),
                       adjoint=False)
    return ah.loss_difference(rp, rm, W) / (2 * h), ah.same_records(rp, rm)


def _fd_alignment(core_host, tables, cfg, trk, W, sf, j):
    h = 1e-4 if j < 3 else 1e-7
    dl = np.zeros(6)
    dl[j] = h
    rp, _ = ah.forward(core_host, alignment.apply_alignment(tables, {sf: dl}),
                       cfg, trk, adjoint=False)
    rm, _ = ah.forward(core_host, alignment.apply_alignment(tables, {sf: -dl}),
                       cfg, trk, adjoint=False)
    same = ah.same_records(rp, rm).all()
    return ah.loss_difference(rp, rm, W).sum() / (2 * h), same


def _rel(a, b, floor):
    return np.abs(a - b) / (np.abs(a) + np.abs(b) + floor)


def _hit_surfaces(res, cfg, tables, shapes=(0, 1, 2)):
    m = ah.transported_mask(res, cfg.max_records)
    bc = res["rec_barcode"][m]
    idx = ((bc >> np.uint64(27)) & np.uint64(0x1FFFFF)).astype(np.int64)
    sfs, counts = np.unique(idx, return_counts=True)
    keep = np.isin(tables["surfaces"]["shape"][sfs], shapes)
    order = np.argsort(-counts[keep], kind="stable")
    return sfs[keep][order]


@pytest.mark.parametrize("material", [1, 0])
def test_telescope_gradients_match_finite_differences(core_host, material):
    tables = geometry.load_geometry("telescope_10x1m_300um")
    cfg = abi.make_config(max_records=16, use_material_interactor=material,
                          step_constraint=1.0)
    trk = tracks.telescope_tracks(8, seed=11)
    trk[0] += 5.0  # start between the first two planes
    res, tape = ah.forward(core_host, tables, cfg, trk)
    assert (res["n_records"] > 5).all()
    W = ah.random_weights(res, cfg.max_records, seed=1)
    gfree, galign = ah.backward(core_host, tables, cfg, trk, res, tape, W)
    for which in (0, 1, 2, "phi", "theta", 7):
        fd, same = _fd_initial(core_host, tables, cfg, trk, W, which)
        assert same.all()
        an = _analytic(gfree, trk, which)
        rel = _rel(fd, an, 1e-6 * np.abs(an).max() + 1e-12)
        assert rel.max() < 1e-4 and np.median(rel) < 1e-5, (which, rel)
    arel = []
    for sf in _hit_surfaces(res, cfg, tables)[:3]:
        for j in range(6):
            fd, same = _fd_alignment(core_host, tables, cfg, trk, W, sf, j)
            assert same
            arel.append(_rel(fd, galign[sf, j],
                             1e-6 * np.abs(galign[sf]).max() + 1e-12))
    assert max(arel) < 2e-4 and np.median(arel) < 1e-5, arel


def test_toy_gradients_match_finite_differences(core_host):
    tables = geometry.load_geometry("toy_4brl_7edc")
    cfg = abi.make_config(max_records=32, search_window=(3, 3),
                          step_constraint=2.0)
    trk = tracks.toy_tracks(24, seed=12, pt_range=(1.0, 10.0),
                            eta_range=(-2.5, 2.5))
    res, tape = ah.forward(core_host, tables, cfg, trk)
    W = ah.random_weights(res, cfg.max_records, seed=2)
    gfree, galign = ah.backward(core_host, tables, cfg, trk, res, tape, W)
    rels = []
    for which in (0, 1, 2, "phi", "theta", 7):
        fd, same = _fd_initial(core_host, tables, cfg, trk, W, which)
        an = _analytic(gfree, trk, which)
        rel = _rel(fd, an, 1e-6 * np.abs(an).max() + 1e-12)[same]
        rels.append(rel)
        assert same.sum() >= 20 and rel.max() < 1e-2, (which, rel)
    rels = np.concatenate(rels)
    assert np.median(rels) < 2e-5, np.median(rels)
    arel = []
    for sf in _hit_surfaces(res, cfg, tables)[:3]:
        for j in range(6):
            fd, same = _fd_alignment(core_host, tables, cfg, trk, W, sf, j)
            if same:
                arel.append(_rel(fd, galign[sf, j],
                                 1e-6 * np.abs(galign[sf]).max() + 1e-12))
    assert len(arel) >= 12 and max(arel) < 1e-3 and np.median(arel) < 1e-4


@pytest.fixture(scope="module")
def solenoid():
    from detray_b200 import fields
    return fields.solenoid_map()


@pytest.mark.parametrize("grad", [0, 1])
def test_field_map_gradients_match_finite_differences(core_host, solenoid,
                                                       grad):
    """Toy detector in the solenoid field map.  With use_field_gradient the
    transport Jacobian carries the field's gradient (the reference's
    with-gradient Jacobian): the gradients agree with the finite differences
    to < 1e-3 (measured ~1e-4 worst, ~1e-6 median).  Without it (the
    reference default) the field map is not differentiated, which inside the
    toy detector still gives < 5e-3."""
    tables = geometry.load_geometry("toy_4brl_7edc")
    cfg = abi.make_config(max_records=32, search_window=(3, 3),
                          step_constraint=2.0, use_field_gradient=grad)
    trk = tracks.toy_tracks(24, seed=12, pt_range=(0.5, 50.0),
                            eta_range=(-2.5, 2.5), pt_log_uniform=False)
    res, tape = ah.forward(core_host, tables, cfg, trk, field=solenoid)
    W = ah.random_weights(res, cfg.max_records, seed=3)
    gfree, _ = ah.backward(core_host, tables, cfg, trk, res, tape, W)
    rels = []
    for which in (0, 1, 2, "phi", "theta", 7):
        h = STEPS[which]
        rp, _ = ah.forward(core_host, tables, cfg, _perturbed(trk, which, h),
                           field=solenoid, adjoint=False)
        rm, _ = ah.forward(core_host, tables, cfg, _perturbed(trk, which, -h),
                           field=solenoid, adjoint=False)
        same = ah.same_records(rp, rm)
        fd = ah.loss_difference(rp, rm, W) / (2 * h)
        an = _analytic(gfree, trk, which)
        rel = _rel(fd, an, 1e-6 * np.abs(an).max() + 1e-12)[same]
        assert same.sum() >= 20 and rel.max() < (1e-3 if grad else 5e-3), (
            which, rel)
        rels.append(rel)
    assert np.median(np.concatenate(rels)) < 2e-5


def test_field_map_alignment_gradients_with_field_gradient(core_host,
                                                           solenoid):
    """Alignment gradients in the solenoid map with use_field_gradient: a
    shifted surface moves the track, whose later transport then depends on
    the position columns of the Jacobian."""
    tables = geometry.load_geometry("toy_4brl_7edc")
    cfg = abi.make_config(max_records=32, search_window=(3, 3),
                          step_constraint=2.0, use_field_gradient=1)
    trk = tracks.toy_tracks(24, seed=14, pt_range=(0.5, 5.0),
                            eta_range=(-1.0, 1.0), pt_log_uniform=False)
    res, tape = ah.forward(core_host, tables, cfg, trk, field=solenoid)
    W = ah.random_weights(res, cfg.max_records, seed=5)
    _, galign = ah.backward(core_host, tables, cfg, trk, res, tape, W)
    checked = 0
    for sf in _hit_surfaces(res, cfg, tables)[:3]:
        for j in range(6):
            h = 1e-4 if j < 3 else 1e-7
            dl = np.zeros(6)
            dl[j] = h
            rp, _ = ah.forward(core_host,
                               alignment.apply_alignment(tables, {sf: dl}),
                               cfg, trk, field=solenoid, adjoint=False)
            rm, _ = ah.forward(core_host,
                               alignment.apply_alignment(tables, {sf: -dl}),
                               cfg, trk, field=solenoid, adjoint=False)
            if not ah.same_records(rp, rm).all():
                continue
            fd = ah.loss_difference(rp, rm, W).sum() / (2 * h)
            rel = _rel(fd, galign[sf, j],
                       1e-6 * np.abs(galign[sf]).max() + 1e-12)
            assert rel < 1e-3, (sf, j, fd, galign[sf, j])
            checked += 1
    assert checked >= 12


def test_loss_on_one_record_component(core_host):
    """d(b_k)/d(x0) for single records equals the finite difference of the
    recorded parameter (telescope, q/p row and time: identity through the
    chain, as the reference Jacobian defines them)."""
    tables = geometry.load_geometry("telescope_10x1m_300um")
    cfg = abi.make_config(max_records=16, step_constraint=1.0)
    trk = tracks.telescope_tracks(3, seed=21)
    trk[0] += 5.0
    res, tape = ah.forward(core_host, tables, cfg, trk)
    cap = cfg.max_records
    h = 1e-4
    tp = trk.copy()
    tp[1] += h
    tm = trk.copy()
    tm[1] -= h
    rp, _ = ah.forward(core_host, tables, cfg, tp, adjoint=False)
    rm, _ = ah.forward(core_host, tables, cfg, tm, adjoint=False)
    for k in (0, 4, 8):
        for comp in range(5):
            W = np.zeros((6, cap, trk.shape[1]))
            W[comp, k, :] = 1.0
            g, _ = ah.backward(core_host, tables, cfg, trk, res, tape, W)
            fd = (rp["rec_bound"][comp, k] - rm["rec_bound"][comp, k]) / (2 * h)
            np.testing.assert_allclose(g[1], fd, rtol=1e-5, atol=1e-9)
    # time: identity row and column
    W = np.zeros((6, cap, trk.shape[1]))
    W[5, 3, :] = 1.0
    g, _ = ah.backward(core_host, tables, cfg, trk, res, tape, W)
    np.testing.assert_array_equal(g[3], np.ones(trk.shape[1]))


@pytest.mark.parametrize("kind", ["toy", "telescope", "toy_map"])
def test_tape_jacobians_match_reference(core_host, oracle, solenoid, kind):
    """Every surface-to-surface Jacobian on the tape equals the reference's:
    its accumulated full Jacobian P_k after record k gives the step factor
    P_k P_{k-1}^-1 (from the third transported surface on: the reference
    does not restart the transport Jacobian at the first surface, so its
    second factor integrates from the track start)."""
    field = {"kind": "const", "b": (0, 0, 2 * T)}
    if kind.startswith("toy"):
        det = oracle.build_toy()
        cfg = abi.make_config(max_records=32, search_window=(3, 3))
        trk = tracks.toy_tracks(300, seed=4)
        if kind == "toy_map":
            field = solenoid
    else:
        det = oracle.build_telescope()
        cfg = abi.make_config(max_records=16)
        trk = tracks.telescope_tracks(200, seed=3)
    tables = det.tables()
    ref = oracle.propagate(det, field, cfg, trk, full_jacobian=True)
    res, tape = ah.forward(core_host, tables, cfg, trk,
                           field=None if field.get("kind") == "const" else field)
    np.testing.assert_array_equal(ref["rec_barcode"], res["rec_barcode"])
    mask = ah.transported_mask(res, cfg.max_records)
    compared = 0
    worst = 0.0
    for t in range(trk.shape[1]):
        ks = np.nonzero(mask[:, t])[0]
        P = [ref["rec_jac"][:, k, t].reshape(6, 6) for k in ks]
        for j in range(2, len(ks)):
            Jref = P[j] @ np.linalg.inv(P[j - 1])
            G = tape["rec"][:20, ks[j], t].reshape(4, 5)
            err = np.abs(Jref[:4, :5] - G).max() / max(1.0, np.abs(G).max())
            worst = max(worst, err)
            # q/p row and time column of the reference factor: identity
            np.testing.assert_allclose(Jref[4], np.eye(6)[4], atol=1e-9)
            np.testing.assert_allclose(Jref[:, 5], np.eye(6)[:, 5], atol=1e-9)
            compared += 1
    assert compared > 500
    assert worst < 1e-8, worst


def test_kick_derivatives_match_finite_differences(core_host):
    """dq+/dq- and dq+/d(d.n) of the material kick, through single-surface
    records of the telescope (one plane hit at different incidences)."""
    tables = geometry.load_geometry("telescope_10x1m_300um")
    cfg = abi.make_config(max_records=16, step_constraint=1.0)
    trk = tracks.telescope_tracks(4, seed=5, pt=0.5)  # low momentum
    trk[0] += 5.0
    res, tape = ah.forward(core_host, tables, cfg, trk)
    mq = tape["rec"][ah.K_TAPE_REC - 7]
    assert np.all(mq[ah.transported_mask(res, cfg.max_records)] > 0.99)
    cap = cfg.max_records
    W = np.zeros((6, cap, trk.shape[1]))
    W[4, 2, :] = 1.0  # q/p at the third plane
    g, _ = ah.backward(core_host, tables, cfg, trk, res, tape, W)
    h = 1e-9
    tp = trk.copy()
    tp[7] += h
    tm = trk.copy()
    tm[7] -= h
    rp, _ = ah.forward(core_host, tables, cfg, tp, adjoint=False)
    rm, _ = ah.forward(core_host, tables, cfg, tm, adjoint=False)
    fd = (rp["rec_bound"][4, 2] - rm["rec_bound"][4, 2]) / (2 * h)
    np.testing.assert_allclose(g[7], fd, rtol=1e-6)
    assert np.all(np.abs(g[7] - 1.0) > 1e-6)  # the kicks do contribute
