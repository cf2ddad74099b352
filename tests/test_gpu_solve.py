"""solve! (src/Analysis.jl:375-436) on the device: the reference's inversion testset
(test/test_analysis.jl:121-180) and agreement with the oracle's restatement of the solver."""
import numpy as np
import pytest

from helpers import cap_points, cn, plan_grid, rel

pytestmark = pytest.mark.gpu


def _np(t):
    return np.asfortranarray(t.permute(*reversed(range(t.dim()))).contiguous().cpu().numpy().T)


def test_inversion_modes_and_null_space(pf, O, cuda):
    rng = np.random.default_rng(52)
    L, n = 8, 400
    th = 0.6 * np.sqrt(rng.random(n))
    ph = 2 * np.pi * rng.random(n)
    plan = pf.Plan(th, ph, lmax=L, method="direct")
    alm_true = O.rand_alm(L, rng=rng)[:, :, 0]
    f = np.asfortranarray(O.Direct(th, ph, L).forward(alm_true)[:, 0])
    rec, info = pf.solve(pf.zeros_alm(L, device="cpu"), plan, f, mode="cg", rtol=1e-10, maxiter=2000)
    assert info["mode"] == "cg" and info["iters"] >= 1
    assert {"shannon", "Δℓ", "relres"} <= set(info)
    assert info["shannon"] < 0.2 * (L + 1) ** 2
    r_short, i_short = pf.solve(pf.zeros_alm(L, device="cpu"), plan, f, mode="cg", rtol=1e-10,
                                maxiter=50)
    D = O.Direct(th, ph, L)
    res_short = np.linalg.norm(D.forward(r_short)[:, 0] - f) / np.linalg.norm(f)
    res_long = np.linalg.norm(D.forward(rec)[:, 0] - f) / np.linalg.norm(f)
    assert i_short["iters"] == 50 and i_short["relres"] > info["relres"]
    assert res_long < res_short and res_long < 1e-4
    # a well-covered geometry converges
    rng = np.random.default_rng(56)
    tg = np.arccos(2 * rng.random(3000) - 1)
    pg = 2 * np.pi * rng.random(3000)
    plg = pf.Plan(tg, pg, lmax=6, method="direct")
    at = O.rand_alm(6, rng=rng)[:, :, 0]
    fg = np.asfortranarray(O.Direct(tg, pg, 6).forward(at)[:, 0])
    rg, ig = pf.solve(pf.zeros_alm(6, device="cpu"), plg, fg, mode="cg", rtol=1e-12, maxiter=500)
    assert ig["shannon"] > 0.8 * 49
    assert np.linalg.norm(O.Direct(tg, pg, 6).forward(rg)[:, 0] - fg) / np.linalg.norm(fg) < 1e-9
    assert O.alm_reldiff(rg, at, 6) < 1e-8
    # wiener requires its prior; unknown modes are refused
    with pytest.raises(ValueError):
        pf.solve(pf.zeros_alm(L, device="cpu"), plan, f, mode="wiener")
    prior = [1.0 / (1 + l) ** 2 for l in range(L + 1)]
    r2, i2 = pf.solve(pf.zeros_alm(L, device="cpu"), plan, f, mode="wiener", prior=prior, rtol=1e-8)
    assert i2["mode"] == "wiener" and i2["iters"] >= 1
    with pytest.raises(ValueError):
        pf.solve(pf.zeros_alm(L, device="cpu"), plan, f, mode="nonsense")


@pytest.mark.parametrize("mode,weighted", [("cg", False), ("wiener", True), ("minnorm", False)])
def test_device_solver_matches_oracle_solver(pf, O, cuda, mode, weighted):
    from oracle import analysis as A
    import torch
    rng = np.random.default_rng(90)
    L, tol = 128, 1e-8
    th, ph = cap_points(3000, theta_star=np.deg2rad(30), rng=rng)
    plan = pf.Plan(th, ph, lmax=L, tol=tol, method="stretch")
    so = O.Stretch(th, ph, L, tol, nufft="es", nufft_grid=plan_grid(plan))
    f = cn(rng, len(th))
    w = 0.5 + rng.random(len(th)) if weighted else None
    prior = [1.0 / (1 + l) ** 2 for l in range(L + 1)] if mode == "wiener" else None
    kw = dict(mode=mode, rtol=1e-14, maxiter=6, prior=prior)
    ref, it_ref, rel_ref = A.solve(lambda a: so.forward(a)[:, 0], lambda g: so.adjoint(g)[:, :, 0],
                                   f, L, w=w, **kw)
    a_dev = pf.zeros_alm(L, device=cuda)
    out, info = pf.solve(a_dev, plan, torch.from_numpy(f).to(cuda), w=w, **kw)
    assert info["iters"] == it_ref == 6
    assert info["relres"] == pytest.approx(rel_ref, rel=1e-8)
    assert O.alm_reldiff(_np(out), ref, L) < 1e-9


def test_solver_stops_where_the_reference_breaks(pf, O, cuda):
    # converged runs: the same iteration count as the oracle's loop, for several tolerances
    from oracle import analysis as A
    import torch
    rng = np.random.default_rng(91)
    L, tol = 96, 1e-8
    th, ph = cap_points(4000, theta_star=np.deg2rad(40), rng=rng)
    plan = pf.Plan(th, ph, lmax=L, tol=tol, method="stretch", ntrans=1)
    so = O.Stretch(th, ph, L, tol, nufft="es", nufft_grid=plan_grid(plan))
    at = O.rand_alm(L, rng=rng)[:, :, 0]
    f = so.forward(at)[:, 0]
    for rtol in (1e-2, 1e-3):
        _, it_ref, rel_ref = A.solve(lambda a: so.forward(a)[:, 0], lambda g: so.adjoint(g)[:, :, 0],
                                     f, L, rtol=rtol, maxiter=300)
        _, info = pf.solve(pf.zeros_alm(L, device=cuda), plan, torch.from_numpy(f).to(cuda),
                           rtol=rtol, maxiter=300)
        assert info["iters"] == it_ref < 300 and info["relres"] <= rtol
        assert info["relres"] == pytest.approx(rel_ref, rel=1e-6)


def test_solve_on_a_spin_plan(pf, O, cuda):
    # solve! over a spin-2 stretched plan: six CG iterations agree with the oracle's loop over the
    # oracle's spin stretched leaf, and a well-covered spin Direct problem recovers its modes
    from oracle import analysis as A
    import torch
    rng = np.random.default_rng(92)
    L, tol, s = 96, 1e-8, 2
    th, ph = cap_points(3000, theta_star=np.deg2rad(30), rng=rng)
    plan = pf.Plan(th, ph, lmax=L, tol=tol, method="stretch", spin=s)
    so = O.Stretch(th, ph, L, tol, nufft="es", nufft_grid=plan_grid(plan), spin=s)
    f = cn(rng, len(th))
    ref, it_ref, rel_ref = A.solve(lambda a: so.forward(a)[:, 0], lambda g: so.adjoint(g)[:, :, 0],
                                   f, L, mode="cg", rtol=1e-14, maxiter=6)
    out, info = pf.solve(pf.zeros_alm(L, device=cuda), plan, torch.from_numpy(f).to(cuda),
                         mode="cg", rtol=1e-14, maxiter=6)
    assert info["iters"] == it_ref == 6
    assert info["relres"] == pytest.approx(rel_ref, rel=1e-8)
    mask = O.spin_valid_mask(L, s)
    got = _np(out)
    assert np.abs(got - ref)[mask].max() < 1e-9 * np.abs(ref)[mask].max()
    # the whole sphere, many points, low degree: the modes come back
    L2, n = 10, 2000
    th2 = np.arccos(2 * rng.random(n) - 1)
    ph2 = 2 * np.pi * rng.random(n)
    pd = pf.Plan(th2, ph2, lmax=L2, method="direct", spin=s)
    at = O.rand_spin_alm(L2, s, rng=rng)[:, :, 0]
    fd = O.SpinDirect(th2, ph2, L2, s).forward(at)[:, 0]
    rec, inf2 = pf.solve(pf.zeros_alm(L2, device="cpu"), pd, np.asfortranarray(fd), mode="cg",
                         rtol=1e-12, maxiter=500)
    m2 = O.spin_valid_mask(L2, s)
    assert np.abs(np.asarray(rec) - at)[m2].max() < 1e-8 and inf2["relres"] <= 1e-12
