"""Stretch geometry, window and grid sizes (test/test_geometry_windows.jl) on the oracle, and
the product library's host geometry against it (no device is touched)."""
import numpy as np
import pytest

from helpers import cap_points


def test_derived_relations(O):
    # test/test_geometry_windows.jl:55-66
    for (thhi, L, eps) in ((0.35, 512, 1e-8), (0.6, 1024, 1e-10), (1.0, 2048, 1e-6)):
        g = O.stretch_geometry(0.0, thhi, L, eps)
        beta = O.es_beta(eps)
        assert g.beta == pytest.approx(beta)
        assert g.eps_apo == pytest.approx(np.sqrt(2 * beta / (L * g.h)))
        assert g.K == max(1, int(np.ceil(L * g.h * (1 + g.eps_apo) ** 2 / np.pi)))
        assert g.Theta1 == pytest.approx(np.pi / (1 + g.eps_apo))
        assert g.sigma == pytest.approx((np.pi - g.Theta1) / 2)
        assert g.ThetaT == pytest.approx(g.Theta1 + g.sigma)


def test_window_contract(O):
    # test/test_geometry_windows.jl:68-77
    g = O.stretch_geometry(0.0, 0.35, 512, 1e-8)
    for Th in np.linspace(0, g.Theta1, 50):
        assert g.window(Th) == 1.0
    assert g.window(np.pi) == 0.0
    ws = [g.window(Th) for Th in np.linspace(g.Theta1, np.pi, 200)]
    assert np.all(np.diff(ws) <= 1e-12)


def test_es_cdf_converged_and_monotone(O):
    # test/test_geometry_windows.jl:79-92
    beta = O.es_beta(1e-8)
    for u in (-1.0, -0.3, 0.0, 0.7, np.pi / 2):
        assert np.isfinite(O.es_cdf(beta, u))
    assert O.es_cdf(beta, -np.pi / 2) == 0.0
    assert O.es_cdf(beta, np.pi / 2) > 0
    vals = [O.es_cdf(beta, u) for u in np.linspace(-np.pi / 2, np.pi / 2, 60)]
    assert vals == sorted(vals)
    # the composite Gauss-Legendre rule is converged: it equals a fine trapezoid reference
    t = np.linspace(-np.pi / 2, 0.7, 400001)
    ref = np.trapezoid(np.exp(beta * (np.cos(t) - 1)) * np.cos(t), t)
    assert O.es_cdf(beta, 0.7) == pytest.approx(ref, rel=1e-9)


def test_coordinate_maps_invert(O):
    # test/test_geometry_windows.jl:94-102
    for (lo, hi, L) in ((0.0, 0.4, 512), (0.8, 1.2, 1024), (0.0, np.pi, 256)):
        g = O.stretch_geometry(lo, hi, L, 1e-8)
        for th in np.linspace(max(lo, 1e-6), hi, 20):
            assert g.to_theta(g.to_stretch(th)) == pytest.approx(th, abs=1e-10)


def test_interior_never_pads_across_a_pole(O):
    # test/test_geometry_windows.jl:104-115
    for (lo, hi, L) in ((0.02, 0.35, 256), (0.01, 0.5, 512), (2.7, 3.13, 512)):
        g = O.stretch_geometry(lo, hi, L, 1e-8)
        if g.kind == "interior":
            pad = g.h * g.eps_apo
            assert g.theta_lo - pad >= -1e-12
            assert g.theta_hi + pad <= np.pi + 1e-12


def test_degenerate_geometry_refused(O):
    # test/test_geometry_windows.jl:117-121
    with pytest.raises(ValueError):
        O.stretch_geometry(0.0, 0.05, 32, 1e-10)
    with pytest.raises(ValueError):
        O.stretch_geometry(0.4, 0.45, 16, 1e-12)


def test_full_sphere(O):
    # test/test_geometry_windows.jl:123-128
    g = O.stretch_geometry(0.0, np.pi, 256, 1e-8)
    assert g.kind == "full"
    assert g.K == 256
    assert g.window(1.0) == 1.0


def _smooth(n):
    for p in (2, 3, 5):
        while n % p == 0:
            n //= p
    return n == 1


def test_grid_sizes_smooth_and_even(O):
    # test/test_geometry_windows.jl:131-154
    for n in (1, 2, 7, 100, 122, 227, 1000, 4097):
        assert O.next_smooth(n) >= n and _smooth(O.next_smooth(n))
        e = O.next_smooth_even(n)
        assert e >= n and e % 2 == 0 and _smooth(e)
    assert O.next_smooth_even(135) == 144
    assert O.next_smooth_even(225) == 240


@pytest.mark.parametrize("L,tol", [(256, 1e-8), (1024, 1e-8), (2048, 1e-8), (2048, 1e-6), (512, 1e-4)])
def test_library_host_geometry_matches_oracle(pf, O, L, tol):
    # the product's plan-time geometry (pfsht_plan_geometry, host only) equals the oracle's
    M = int(round(4 * (L * np.deg2rad(20)) ** 2))
    th, ph = cap_points(min(M, 50000), rng=np.random.default_rng(L))
    g = pf.plan_geometry(th, ph, lmax=L, tol=tol)
    # the leaf's sizes depend on the points only through their colatitude extent
    lo, hi = th.min(), th.max()
    ext = np.array([lo, hi, 0.5 * (lo + hi)])
    ref = O.Stretch(ext, np.zeros(3), L, tol, nufft="direct")
    for k in ("nth_half", "nth", "nph", "mmax", "K", "ring_work", "flip"):
        assert g[k] == ref.info[k], k
    assert g["kind"] == ref.info["kind"]
    assert g["eps_apo"] == pytest.approx(ref.info["eps_apo"], rel=1e-15)
    assert g["nufft_w"] == int(np.ceil(-np.log10(tol / 10)))


def test_baseline_config_sizes(pf):
    # the sizes the lmax 256/1024/2048 cap configurations run at (src/Stretch.jl:164-194)
    expect = {256: (80, 160, 360, 178), 1024: (216, 432, 1080, 513), 2048: (360, 720, 1920, 921)}
    for L, (nh, nth, nph, mmax) in expect.items():
        th = np.array([1e-3, np.deg2rad(20.0)])
        g = pf.plan_geometry(th, np.zeros(2), lmax=L, tol=1e-8, method="stretch")
        assert (g["nth_half"], g["nth"], g["nph"], g["mmax"]) == (nh, nth, nph, mmax)
