"""The serving loop: each request's result is the same alone and in a mix of concurrent
requests over several resident plans, and plans past the HBM budget are refused."""
import numpy as np
import pytest

from helpers import cap_points, rel

pytestmark = pytest.mark.gpu


def _server_plans(pf, rng):
    specs = [(96, 10, 1, 1e-8, "fp64"), (256, 20, 1, 1e-6, "mixed"), (384, 15, 2, 1e-8, "fp64"),
             (512, 25, 1, 1e-6, "mixed"), (200, 8, 3, 1e-8, "fp64")]
    plans = []
    for L, cap, B, tol, prec in specs:
        th, ph = cap_points(max(500, int(4 * (L * np.deg2rad(cap)) ** 2)),
                            theta_star=np.deg2rad(cap), rng=rng)
        plans.append(pf.Plan(th, ph, lmax=L, tol=tol, ntrans=B, precision=prec))
    return plans


def _request(pf, O, p, fwd, rng):
    if fwd:
        a = pf.zeros_alm(p.lmax, p.ntrans, device="pinned")
        a[...] = O.rand_alm(p.lmax, ntrans=p.ntrans, rng=rng).reshape(a.shape, order="F")
        return a, pf.zeros_field(p.npts, p.ntrans, device="pinned")
    f = pf.zeros_field(p.npts, p.ntrans, device="pinned")
    f[...] = (rng.standard_normal(f.shape) + 1j * rng.standard_normal(f.shape))
    return f, pf.zeros_alm(p.lmax, p.ntrans, device="pinned")


def test_results_alone_equal_results_in_the_mix(pf, O, cuda):
    rng = np.random.default_rng(70)
    plans = _server_plans(pf, rng)
    srv = pf.Server(hbm_budget_gb=120, nslots=6)
    ids = [srv.add(p) for p in plans]
    jobs = []
    for k in range(30):
        i = int(rng.integers(len(plans)))
        fwd = bool(rng.integers(2))
        inp, out = _request(pf, O, plans[i], fwd, rng)
        jobs.append((i, fwd, inp, out))
    # alone: one request at a time
    alone = []
    for i, fwd, inp, out in jobs:
        rid = srv.submit(ids[i], fwd, inp, out)
        srv.wait(rid)
        srv.release(rid)
        alone.append(out.copy())
        out[...] = np.nan
    # in the mix: all submitted at once, running concurrently across plans
    rids = [srv.submit(ids[i], fwd, inp, out) for i, fwd, inp, out in jobs]
    lat = [srv.wait(r) for r in rids]
    assert all(x > 0 for x in lat)
    for (i, fwd, inp, out), ref in zip(jobs, alone):
        p = plans[i]
        if fwd:
            assert np.array_equal(out, ref)
        else:
            # the adjoint adds some partial sums atomically: equal up to their order
            tol = 2e-6 if p.info["precision"] == 1 else 1e-13
            assert O.alm_reldiff(out, ref, p.lmax) < tol
    # and equal to the plan's own host-buffer apply
    i, fwd, inp, out = jobs[0]
    ref = np.zeros_like(out)
    if fwd:
        plans[i].mul(ref, inp)
        assert np.array_equal(out, ref)
    st = srv.stats()
    assert st["completed"] == 60 and st["queued"] == 0 and st["running"] == 0
    srv.close()


def test_requests_on_one_plan_run_as_a_group(pf, O, cuda):
    # requests queued for one plan are admitted together and pipelined through the plan's copy
    # streams (copies of one overlapping the kernels of its neighbours); each result equals the
    # plan's own host-buffer apply of its input
    rng = np.random.default_rng(72)
    th, ph = cap_points(40000, rng=rng)
    p = pf.Plan(th, ph, lmax=384, tol=1e-8)
    srv = pf.Server(hbm_budget_gb=120, nslots=2)
    pid = srv.add(p)
    jobs = [(bool(k % 3), *_request(pf, O, p, bool(k % 3), rng)) for k in range(12)]
    rids = [srv.submit(pid, fwd, inp, out) for fwd, inp, out in jobs]
    for r in rids:
        srv.wait(r)
    for fwd, inp, out in jobs:
        ref = np.zeros_like(out)
        if fwd:
            p.mul(ref, inp)
            assert np.array_equal(out, ref)
        else:
            p.mul_adjoint(ref, inp)
            assert O.alm_reldiff(out, ref, p.lmax) < 1e-13
    assert srv.stats()["completed"] == 12
    srv.close()


def test_budget_refuses_plans(pf, O, cuda):
    rng = np.random.default_rng(71)
    th, ph = cap_points(20000, rng=rng)
    p = pf.Plan(th, ph, lmax=256, tol=1e-8)
    srv = pf.Server(hbm_budget_gb=1e-3, nslots=2)
    with pytest.raises(MemoryError):
        srv.add(p)
    srv.close()
