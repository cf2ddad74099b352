"""The host planner (boxes, counted costs, partition, leaf choice) against the reference's own
planner tests (test/test_cost.jl, test/test_geometry_windows.jl:1-52) and against the oracle's
pure-Python restatement of src/Box.jl and src/Cost.jl. No device is used."""
import math

import numpy as np
import pytest

from oracle import planner as P


def _same_box(a, b):
    for k in ("theta_lo", "theta_hi", "phi_start", "phi_extent"):
        assert a[k] == b[k], (k, a[k], b[k])
    assert a["touches_north"] == b["touches_north"] and a["touches_south"] == b["touches_south"]


def _caps(rng, n1, r=0.2):
    th = np.concatenate([r * np.sqrt(rng.random(n1)), np.pi - r * np.sqrt(rng.random(n1))])
    return th, 2 * np.pi * rng.random(2 * n1)


def test_bounding_box_is_exactly_minimal(pf):
    # test/test_geometry_windows.jl:1-28
    rng = np.random.default_rng(21)
    th = 0.3 + 0.4 * rng.random(500)
    ph = 1.0 + 0.5 * rng.random(500)
    b = pf.bounding_box(th, ph)
    assert b["theta_lo"] == th.min() and b["theta_hi"] == th.max()
    assert math.isclose(b["phi_extent"], ph.max() - ph.min(), rel_tol=1e-12)
    assert not b["touches_north"] and not b["touches_south"]
    _same_box(b, P.bounding_box(th, ph))
    # points straddling phi = 0: the minimal arc wraps
    phw = np.concatenate([0.05 * rng.random(200), 2 * np.pi - 0.05 * rng.random(200)])
    bw = pf.bounding_box(np.full(400, 1.0), phw)
    assert bw["phi_extent"] < 0.15
    _same_box(bw, P.bounding_box(np.full(400, 1.0), phw))
    # a full circle is a full circle; negative and > 2 pi longitudes are reduced mod 2 pi
    phf = 2 * np.pi * rng.random(500) - 3.0
    assert pf.bounding_box(np.full(500, 1.0), phf)["phi_extent"] > 2 * np.pi - 0.2
    _same_box(pf.bounding_box(np.full(500, 1.0), phf), P.bounding_box(np.full(500, 1.0), phf))
    # a pole in range forces the full longitude range
    bp = pf.bounding_box(np.concatenate([[0.0], 0.2 * rng.random(100)]), 0.1 * rng.random(101))
    assert bp["touches_north"] and bp["phi_extent"] == 2 * np.pi
    # one point
    b1 = pf.bounding_box([0.7], [7.0])
    assert b1["phi_extent"] == 0.0 and b1["phi_start"] == pytest.approx(7.0 - 2 * np.pi)


def test_partition_bands_stay_whole_components_separate(pf):
    # test/test_geometry_windows.jl:30-52, and the oracle's partition group by group
    rng = np.random.default_rng(22)
    kw = dict(lmax=256, ntrans=1, tol=1e-8)
    half = np.deg2rad(8)
    tb = np.pi / 2 + half * (2 * rng.random(3000) - 1)
    pb = 2 * np.pi * rng.random(3000)
    ta, pa = _caps(rng, 1500)
    tc = 0.2 * np.sqrt(rng.random(2000))
    pc = 2 * np.pi * rng.random(2000)
    for (th, ph), want in (((tb, pb), 1), ((ta, pa), 2), ((tc, pc), 1)):
        groups, boxes, costs = pf.partition_boxes(th, ph, **kw)
        assert len(groups) == want
        og, ob, oc = P.partition_boxes_costed(th, ph, 256, 1, 1e-8)
        assert len(og) == len(groups)
        for g, b, c, g2, b2, c2 in zip(groups, boxes, costs, og, ob, oc):
            assert np.array_equal(g, g2)
            _same_box(b, b2)
            assert c == pytest.approx(c2, rel=1e-12)
    bb = pf.bounding_box(tb, pb)
    assert bb["theta_hi"] - bb["theta_lo"] < 2.1 * half


def test_partition_many_fragments_and_maxboxes(pf):
    # several disjoint patches in longitude and latitude: splits stop at maxboxes
    rng = np.random.default_rng(23)
    th, ph = [], []
    for k in range(5):
        th.append(0.6 + 0.3 * k + 0.05 * rng.random(400))
        ph.append(1.2 * k + 0.1 * rng.random(400))
    th, ph = np.concatenate(th), np.concatenate(ph)
    for mb in (1, 3, 8):
        groups, _, _ = pf.partition_boxes(th, ph, lmax=512, tol=1e-8, maxboxes=mb)
        og, _, _ = P.partition_boxes_costed(th, ph, 512, 1, 1e-8, mb)
        assert 1 <= len(groups) <= mb
        assert [list(g) for g in groups] == [list(g) for g in og]
        assert sorted(np.concatenate(groups)) == list(range(len(th)))


@pytest.mark.parametrize("L,lo,hi,tol,B", [(256, 0.0, 0.35, 1e-8, 1), (512, 0.4, 0.9, 1e-8, 2),
                                           (1024, 2.6, np.pi, 1e-6, 1), (2048, 0.0, 0.35, 1e-10, 1),
                                           (300, 1.2, 1.9, 1e-8, 4)])
def test_cost_stretch_counts_like_the_reference(pf, L, lo, hi, tol, B):
    # the library's counted cost (its leaf sizing) against the oracle's own counting
    box = dict(theta_lo=lo, theta_hi=hi, phi_start=0.0, phi_extent=2 * np.pi,
               touches_north=lo == 0.0, touches_south=hi == np.pi)
    assert pf.cost_stretch(box, 12345, L, B, tol) == pytest.approx(
        P.cost_stretch(box, 12345, L, B, tol), rel=1e-12)
    assert pf.cost_direct(12345, L, B) == P.cost_direct(12345, L, B)


def test_degenerate_geometry_costs_inf(pf):
    # test/test_cost.jl:28-31
    rng = np.random.default_rng(70)
    b = pf.bounding_box(0.01 * rng.random(20), 2 * np.pi * rng.random(20))
    assert pf.cost_stretch(b, 20, 8, 1, 1e-12) == math.inf


def test_select_method(pf):
    # test/test_cost.jl:46-72
    rng = np.random.default_rng(72)
    th = np.deg2rad(20) * np.sqrt(rng.random(4000))
    ph = 2 * np.pi * rng.random(4000)
    for L in (256, 512, 1024, 2048):
        assert pf.select_method(th, ph, lmax=L, tol=1e-8) == "stretch"
        assert P.select_method(th, ph, L, 1e-8) == "stretch"
    t, p = 0.3 * rng.random(12), 2 * np.pi * rng.random(12)
    assert pf.select_method(t, p, lmax=4, tol=1e-8) == "direct" == P.select_method(t, p, 4, 1e-8)
    ta, pa = _caps(rng, 2000)
    assert pf.select_method(ta, pa, lmax=512, tol=1e-8) == "multibox"
    assert P.select_method(ta, pa, 512, 1e-8) == "multibox"
    # host-only plan geometry reports the choice
    g = pf.plan_geometry(ta, pa, lmax=512, tol=1e-8)
    assert g["kind"] == "multibox"
    groups, boxes, _ = pf.partition_boxes(ta, pa, lmax=512, tol=1e-8)
    assert g["ring_work"] == sum(
        pf.plan_geometry(ta[gr], pa[gr], lmax=512, tol=1e-8, method="stretch")["ring_work"]
        for gr in groups)


def test_cost_constants_installable(pf):
    # test/test_cost.jl:74-86
    old = pf.cost_constants()
    assert old["ring"] == 1.0 and old["fft"] == 0.394 and old["spread"] == 0.334
    try:
        c = pf.set_cost_constants(ring=2.0)
        assert c["ring"] == 2.0 and c["fft"] == old["fft"] and pf.cost_calibrated()
        # the model's costs scale with the installed constants
        assert pf.cost_direct(100, 10, 1) == P.cost_direct(100, 10, 1, dict(P.DEFAULT_COST, ring=2.0))
        with pytest.raises(ValueError):
            pf.set_cost_constants(fft=-1.0)
    finally:
        pf.set_cost_constants(ring=old["ring"], fft=old["fft"], spread=old["spread"],
                              ft_conn=old["ft_conn"])
