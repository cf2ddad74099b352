"""Batched applies (one captured graph per direction) against the same plans applied one by one:
plans of uneven lmax, cap, ntrans and tolerance, FP64 and mixed forms, and a refused geometry
answered by the Direct leaf."""
import numpy as np
import pytest

from helpers import cap_points, rel

pytestmark = pytest.mark.gpu


def _plans(pf, rng):
    specs = [  # (lmax, cap degrees, ntrans, tol, precision)
        (128, 10, 1, 1e-8, "fp64"), (300, 25, 3, 1e-8, "fp64"), (200, 15, 2, 1e-6, "mixed"),
        (512, 20, 1, 1e-6, "mixed"), (96, 30, 5, 1e-8, "fp64"), (400, 6, 1, 1e-8, "fp64"),
        (256, 12, 4, 1e-6, "mixed"), (700, 18, 1, 1e-8, "fp64")]
    plans = []
    for L, cap, B, tol, prec in specs:
        th, ph = cap_points(max(500, int(4 * (L * np.deg2rad(cap)) ** 2)),
                            theta_star=np.deg2rad(cap), rng=rng)
        plans.append(pf.Plan(th, ph, lmax=L, tol=tol, ntrans=B, precision=prec))
    # a patch too small for the stretched construction: the Direct leaf answers it
    th = 0.02 + 0.03 * rng.random(60)
    plans.append(pf.Plan(th, rng.random(60), lmax=32, tol=1e-10))
    assert plans[-1].info["kind"] == "direct"
    return plans


def _inputs(pf, plans, rng, cuda):
    import torch
    alms, fs = [], []
    for p in plans:
        a = pf.zeros_alm(p.lmax, p.ntrans, device=cuda)
        a.real.normal_()
        a.imag.normal_()
        f = pf.zeros_field(p.npts, p.ntrans, device=cuda)
        f.real.normal_()
        f.imag.normal_()
        alms.append(a)
        fs.append(f)
    torch.cuda.synchronize()
    return alms, fs


def test_batch_matches_single_plans(pf, O, cuda):
    import torch
    torch.manual_seed(0)
    rng = np.random.default_rng(60)
    plans = _plans(pf, rng)
    batch = pf.Batch(plans, nstreams=4)
    for call in range(2):  # new arrays on the second call: the pointer table changes
        alms, fins = _inputs(pf, plans, rng, cuda)
        fb = [pf.zeros_field(p.npts, p.ntrans, device=cuda) for p in plans]
        ab = [pf.zeros_alm(p.lmax, p.ntrans, device=cuda) for p in plans]
        batch.forward(fb, alms)
        batch.adjoint(ab, fins)
        torch.cuda.synchronize()
        for p, a, f, fbi, abi in zip(plans, alms, fins, fb, ab):
            f1 = p * a
            a1 = p.H * f
            torch.cuda.synchronize()
            assert rel(fbi.cpu().numpy(), f1.cpu().numpy()) < 1e-14, (call, p)
            # adjoint: some partial sums are added atomically, so equal up to their order, which
            # shows at FP64 round-off, or FP32 round-off for the mixed form's spreading
            tol = 2e-6 if p.info["precision"] == 1 else 1e-13
            assert O.alm_reldiff(abi.cpu().numpy(), a1.cpu().numpy(), p.lmax) < tol, (call, p)
    info = batch.info()
    # the ring passes of all nine plans, every tile shape, run in one persistent launch per
    # direction (these plans use no eight-rings-per-lane adjoint tiles)
    assert info["ring_launches_fwd"] == 1 and info["ring_launches_adj"] == 1
    assert info["graph_nodes_fwd"] > 0 and info["graph_nodes_adj"] > 0


def test_batch_rejects_bad_input(pf, O, cuda):
    rng = np.random.default_rng(61)
    th, ph = cap_points(2000, rng=rng)
    p = pf.Plan(th, ph, lmax=64, tol=1e-8)
    with pytest.raises(ValueError):
        pf.Batch([p, p])
    b = pf.Batch([p])
    with pytest.raises(pf.DimensionMismatch):
        b.forward([pf.zeros_field(10, device=cuda)], [pf.zeros_alm(64, device=cuda)])
