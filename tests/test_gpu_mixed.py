"""The mixed form (FP64 recurrence and exponents, FP32 compensated ring accumulation, FP32
NUFFT) against the FP64 direct sum, as the reference's Float32 end-to-end test does
(test/test_transforms.jl:158-208), with the error stated per case."""
import numpy as np
import pytest

from helpers import cap_points, cn, dot_rel, rel, to_dev, to_host

pytestmark = pytest.mark.gpu

THETA_STAR = np.deg2rad(20.0)


def _fwd(plan, alm):
    return to_host(plan * to_dev(alm if alm.shape[2] > 1 else alm[:, :, 0]))


def _adj(plan, g):
    return to_host(plan.H * to_dev(g))


@pytest.mark.parametrize("L", [128, 256, 512])
def test_mixed_vs_direct(pf, O, cuda, L):
    # delivered accuracy of the mixed form at tol 1e-6 against FP64 direct evaluation: the
    # reference gates its own FP32 apply at 1e-3; the mixed form keeps the FP64 recurrence and
    # compensates its sums, so it is held to 10 tol like the FP64 form
    rng = np.random.default_rng(50 + L)
    n = 150
    th = THETA_STAR * np.sqrt(rng.random(n))
    ph = 2 * np.pi * rng.random(n)
    pm = pf.Plan(th, ph, lmax=L, tol=1e-6, method="stretch", precision="mixed")
    assert pm.info["precision"] == 1
    assert pm.info["nufft_w"] == 7
    alm = O.rand_alm(L, rng=rng)
    ref = O.Direct(th, ph, L)
    f = _fwd(pm, alm)
    err = rel(f, ref.forward(alm, nthreads=8)[:, 0])
    print(f"mixed forward L={L}: max rel error vs FP64 direct {err:.2e}")
    assert err < 1e-5
    g = cn(rng, n)
    a = _adj(pm, g)
    aerr = O.alm_reldiff(a, ref.adjoint(g, nthreads=8)[:, :, 0], L)
    print(f"mixed adjoint L={L}: max rel error vs FP64 direct {aerr:.2e}")
    assert aerr < 1e-5
    # forward and adjoint are transposes to FP32 round-off
    assert dot_rel(f, g, alm[:, :, 0], a) < 1e-5


def test_mixed_request_below_1e6_runs_fp64(pf, O, cuda):
    rng = np.random.default_rng(51)
    th, ph = cap_points(2000, rng=rng)
    p = pf.Plan(th, ph, lmax=128, tol=1e-8, precision="mixed")
    assert p.info["precision"] == 0
    q = pf.Plan(th, ph, lmax=128, tol=1e-8)
    alm = O.rand_alm(128, rng=rng)
    assert np.array_equal(_fwd(p, alm), _fwd(q, alm))


@pytest.mark.parametrize("B", [1, 3])
def test_mixed_matches_fp64_plan(pf, O, cuda, B):
    # the mixed and FP64 forms of one geometry agree to the mixed form's accuracy, for single
    # and batched transforms (the 2-transform kernels run for B = 3)
    rng = np.random.default_rng(52)
    L = 512
    th, ph = cap_points(40000, rng=rng)
    pm = pf.Plan(th, ph, lmax=L, tol=1e-6, precision="mixed", ntrans=B)
    pd = pf.Plan(th, ph, lmax=L, tol=1e-10, ntrans=B)
    alm = O.rand_alm(L, ntrans=B, rng=rng, weight=lambda l: 1.0 / (l + 1))
    e = rel(_fwd(pm, alm), _fwd(pd, alm))
    print(f"mixed vs FP64 plan forward, B={B}: {e:.2e}")
    assert e < 1e-5
    g = np.asfortranarray(cn(rng, len(th), B)) if B > 1 else cn(rng, len(th))
    ea = O.alm_reldiff(_adj(pm, g), _adj(pd, g), L)
    print(f"mixed vs FP64 plan adjoint, B={B}: {ea:.2e}")
    assert ea < 1e-5


def test_mixed_full_size_against_fp64(pf, O, cuda):
    # lmax 2048 on the 20-degree cap at tol 1e-6: the mixed form against the FP64 form of the
    # same points at tol 1e-10, forward and adjoint, and the dot test
    rng = np.random.default_rng(53)
    L = 2048
    M = int(round(4 * (L * THETA_STAR) ** 2))
    th, ph = cap_points(M, rng=rng)
    pm = pf.Plan(th, ph, lmax=L, tol=1e-6, precision="mixed")
    pd = pf.Plan(th, ph, lmax=L, tol=1e-10)
    alm = O.rand_alm(L, rng=rng, weight=lambda l: 1.0 / (l + 1))
    fm = _fwd(pm, alm)
    e = rel(fm, _fwd(pd, alm))
    print(f"mixed vs FP64 forward at lmax 2048: {e:.2e}")
    assert e < 1e-5
    g = cn(rng, M)
    am = _adj(pm, g)
    ea = O.alm_reldiff(am, _adj(pd, g), L)
    print(f"mixed vs FP64 adjoint at lmax 2048: {ea:.2e}")
    assert ea < 1e-5
    assert dot_rel(fm, g, alm[:, :, 0], am) < 1e-5
