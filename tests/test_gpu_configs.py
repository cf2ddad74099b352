"""The benchmark's lmax = 1024 workload as a parity case: M = 4 (L theta*)^2 = 511,063 points on
the 20 degree cap (cos theta uniform), tol 1e-8, ntrans in {1, 4} with independent complex N(0,1)
coefficients per transform; forward and adjoint checked separately against the oracle's
stretched leaf at full size, per column against the single-transform plan, by the dot test, and
with coefficients in the m >= 0 slots only (the other reading of the workload's wording)."""
import numpy as np
import pytest

from helpers import cap_points, cn, dot_rel, plan_grid, rel, to_dev, to_host

pytestmark = pytest.mark.gpu


def _fwd(plan, alm):
    return to_host(plan * to_dev(np.asfortranarray(alm)))


def _adj(plan, g):
    return to_host(plan.H * to_dev(np.asfortranarray(g)))


def test_lmax1024_cap_ntrans_1_and_4(pf, O, cuda):
    L, tol, B = 1024, 1e-8, 4
    M = int(round(4 * (L * np.deg2rad(20.0)) ** 2))
    assert M == 511063
    rng = np.random.default_rng(1)
    th, ph = cap_points(M, rng=rng)
    p1 = pf.Plan(th, ph, lmax=L, tol=tol)
    p4 = pf.Plan(th, ph, lmax=L, tol=tol, ntrans=B)
    assert p1.info["kind"] == "pole" and p4.info["nf1"] == p1.info["nf1"]
    ref = O.Stretch(th, ph, L, tol, nufft="es", nufft_grid=plan_grid(p1))
    alm = O.rand_alm(L, ntrans=B, rng=rng)
    g = np.asfortranarray(cn(rng, M, B))
    # forward and adjoint of one transform against the oracle at full size
    f1 = _fwd(p1, alm[:, :, 0])
    assert rel(f1, ref.forward(alm[:, :, :1], nthreads=16)[:, 0]) < 1e-11
    a1 = _adj(p1, np.ascontiguousarray(g[:, 0]))
    assert O.alm_reldiff(a1, ref.adjoint(np.asfortranarray(g[:, :1]), nthreads=16)[:, :, 0], L) < 1e-10
    assert dot_rel(f1, g[:, 0], alm[:, :, 0], a1) < 1e-12
    # four transforms in one plan: each column as the single plan, each pair by the dot test
    f4 = _fwd(p4, alm)
    a4 = _adj(p4, g)
    for b in range(B):
        assert rel(f4[:, b], _fwd(p1, alm[:, :, b])) < 1e-12
        assert O.alm_reldiff(a4[:, :, b], _adj(p1, np.ascontiguousarray(g[:, b])), L) < 1e-12
        assert dot_rel(f4[:, b], g[:, b], alm[:, :, b], a4[:, :, b]) < 1e-12
    # coefficients in the m >= 0 slots only
    a0 = np.array(alm[:, :, 0], order="F")
    a0[:, 1::2] = 0  # columns 2|m| - 1 hold m < 0
    assert rel(_fwd(p1, a0), ref.forward(a0[:, :, None], nthreads=16)[:, 0]) < 1e-11
