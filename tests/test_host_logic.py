"""Host-side logic of the Python mirror (argument checks, layouts, method choice) that
needs no device."""
import numpy as np
import pytest

from helpers import cap_points


def test_layout_helpers_follow_sph_mode(pf, O):
    # src/Layout.jl:13-20: (lmax+1, 2lmax+1), column 2m for m >= 0 and 2|m|-1 for m < 0
    assert pf.coeff_size(5) == (6, 11)
    for (l, m) in ((0, 0), (3, 2), (3, -2), (7, -7), (7, 7)):
        assert pf.sph_mode(l, m) == O.sph_mode(l, m)
    assert pf.sph_mode(4, 0) == (4, 0)
    assert pf.sph_mode(4, 3) == (1, 6)
    assert pf.sph_mode(4, -3) == (1, 5)


def test_host_arrays_are_column_major(pf):
    a = pf.zeros_alm(6, device="cpu")
    assert a.shape == (7, 13) and a.flags.f_contiguous
    a3 = pf.zeros_alm(6, ntrans=3, device="cpu")
    assert a3.shape == (7, 13, 3) and a3.flags.f_contiguous
    f = pf.zeros_field(10, ntrans=2, device="cpu")
    assert f.shape == (10, 2) and f.flags.f_contiguous


def test_plan_argument_errors_before_any_device_use(pf):
    # src/Plan.jl:98-102 and src/Layout.jl:35-56
    th, ph = np.full(10, 0.1), np.zeros(10)
    with pytest.raises(pf.DimensionMismatch):
        pf.Plan(th, ph[:9], lmax=8)
    with pytest.raises(ValueError):
        pf.Plan(th, ph, lmax=-1)
    with pytest.raises(ValueError):
        pf.Plan(th, ph, lmax=8, ntrans=0)
    with pytest.raises(ValueError):
        pf.Plan(th, ph, lmax=8, method="nufsht")
    with pytest.raises(ValueError):
        pf.Plan(th, ph, lmax=8, precision="fp16")
    with pytest.raises(ValueError):
        pf.Plan(th, ph, lmax=8, tol=0.0)


def test_refused_geometry_and_auto_fallback(pf):
    # src/Windows.jl:66-75: a patch this small at this bandlimit has no admissible
    # periodisation; method "stretch" refuses, "auto" answers with the direct leaf
    # (src/Cost.jl:121-122,184-186)
    th = 0.02 + 0.03 * np.random.default_rng(0).random(50)
    ph = np.random.default_rng(1).random(50)
    with pytest.raises(pf.RefusedGeometry):
        pf.plan_geometry(th, ph, lmax=32, tol=1e-10, method="stretch")
    g = pf.plan_geometry(th, ph, lmax=32, tol=1e-10, method="auto")
    assert g["kind"] == "direct"
    g = pf.plan_geometry(th, ph, lmax=32, tol=1e-10, method="direct")
    assert g["kind"] == "direct"


def test_southern_cap_is_reflected_north(pf):
    # src/Stretch.jl:151-158
    th, ph = cap_points(2000, rng=np.random.default_rng(3))
    g = pf.plan_geometry(np.pi - th, ph, lmax=512, tol=1e-8)
    assert g["kind"] == "pole" and g["flip"] == 1
    gn = pf.plan_geometry(th, ph, lmax=512, tol=1e-8)
    assert gn["flip"] == 0
    for k in ("nth", "nph", "mmax", "ring_work"):
        assert g[k] == gn[k]


def test_interior_and_full_geometries(pf):
    rng = np.random.default_rng(4)
    # at lmax 256 this band is cheapest as a pole periodisation; at 1024 as an interior one
    th = 0.9 + 0.12 * (2 * rng.random(500) - 1)
    assert pf.plan_geometry(th, rng.random(500), lmax=256, tol=1e-8)["kind"] == "pole"
    g = pf.plan_geometry(th, rng.random(500), lmax=1024, tol=1e-8)
    assert g["kind"] == "interior" and g["nth"] == g["nth_half"]
    th = np.concatenate([[0.0, np.pi], np.pi * rng.random(100)])
    g = pf.plan_geometry(th, rng.random(102), lmax=64, tol=1e-8, method="stretch")
    assert g["kind"] == "full"
    # the cost model prefers the direct leaf for so few points (src/Cost.jl:171-201)
    assert pf.plan_geometry(th, rng.random(102), lmax=64, tol=1e-8)["kind"] == "direct"
