"""The benchmark's headline workload as a parity case at full size: lmax 2048, the 20-degree cap
with M = round(4 (lmax theta*)^2) = 2,044,253 points of which 1% sit within 1e-9 theta* of the
cap boundary, coefficients complex N(0,1)/(l+1) in every valid sph_mode slot, tol 1e-8 (FP64)
and 1e-6 (mixed form). These are the inputs bench.py times, made by its own generators.

Gates follow the reference's device-vs-host and accuracy checks (gpu/runtests.jl:86-120,
test/test_transforms.jl:59-82,111-123): the forward against the oracle's stretched leaf on the
plan's NUFFT grid <= 1e-11, the adjoint <= 1e-10, the dot test <= 1e-12, and on a seeded
subsample of 1024 points the forward against the oracle's Direct sum within 10 tol, for the
FP64 plan and for the mixed plan."""
import numpy as np
import pytest

from bench import rand_alm_host, workload
from helpers import cn, dot_rel, plan_grid, rel, to_dev, to_host

pytestmark = pytest.mark.gpu

L = 2048


@pytest.fixture(scope="module")
def headline(O):
    M, th, ph, rng = workload(L)
    assert M == 2044253
    on_edge = np.abs(th - np.deg2rad(20.0)) <= 1e-9 * np.deg2rad(20.0)
    assert on_edge.sum() >= M // 100
    alm = np.asfortranarray(rand_alm_host(L, rng).transpose(2, 1, 0))  # (L+1, 2L+1, 1)
    g = cn(rng, M)
    sub = np.sort(np.random.default_rng(7).choice(M, 1024, replace=False))
    # the subsample holds boundary points as well
    sub = np.union1d(sub, np.flatnonzero(on_edge)[:16])
    fd = O.Direct(th[sub], ph[sub], L).forward(alm, nthreads=16)[:, 0]
    return dict(M=M, th=th, ph=ph, alm=alm, g=g, sub=sub, fd=fd)


def test_headline_fp64_against_the_oracle(pf, O, cuda, headline):
    h = headline
    tol = 1e-8
    plan = pf.Plan(h["th"], h["ph"], lmax=L, tol=tol)
    assert plan.info["kind"] == "pole"
    ref = O.Stretch(h["th"], h["ph"], L, tol, nufft="es", nufft_grid=plan_grid(plan))
    assert ref.ring_work() == plan.info["ring_work"]
    f = to_host(plan * to_dev(h["alm"][:, :, 0]))
    assert rel(f, ref.forward(h["alm"], nthreads=16)[:, 0]) < 1e-11
    a = to_host(plan.H * to_dev(h["g"]))
    a_ref = ref.adjoint(h["g"], nthreads=16)[:, :, 0]
    assert O.alm_reldiff(a, a_ref, L) < 1e-10
    assert dot_rel(f, h["g"], h["alm"][:, :, 0], a) < 1e-12
    # delivered accuracy against the exact sum on the subsample (l2 and max)
    fs = f[h["sub"]]
    assert np.linalg.norm(fs - h["fd"]) / np.linalg.norm(h["fd"]) < 10 * tol
    assert rel(fs, h["fd"]) < 10 * tol


def test_headline_mixed_against_the_oracle_direct(pf, O, cuda, headline):
    h = headline
    tol = 1e-6
    plan = pf.Plan(h["th"], h["ph"], lmax=L, tol=tol, precision="mixed")
    assert plan.info["precision"] == 1  # the mixed form is in use at this tol
    f = to_host(plan * to_dev(h["alm"][:, :, 0]))
    fs = f[h["sub"]]
    assert np.linalg.norm(fs - h["fd"]) / np.linalg.norm(h["fd"]) < 10 * tol
    a = to_host(plan.H * to_dev(h["g"]))
    # the mixed form rounds its sums to FP32: the dot test holds to its tolerance
    assert dot_rel(f, h["g"], h["alm"][:, :, 0], a) < 10 * tol
