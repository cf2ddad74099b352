"""MultiBox plans (src/MultiBox.jl): one stretched leaf per box of the partition, synthesis as
the disjoint union of the boxes' fields and the adjoint as the sum of their coefficients."""
import numpy as np
import pytest

from helpers import cn, dot_rel, rel, to_dev, to_host

pytestmark = pytest.mark.gpu


def _caps(rng, n1, r):
    th = np.concatenate([r * np.sqrt(rng.random(n1)), np.pi - r * np.sqrt(rng.random(n1))])
    return th, 2 * np.pi * rng.random(2 * n1)


def _fwd(plan, alm):
    return to_host(plan * to_dev(np.asfortranarray(alm)))


def _adj(plan, g):
    return to_host(plan.H * to_dev(np.asfortranarray(g)))


def test_two_caps_against_direct(pf, O, cuda):
    # test/test_transforms.jl:210-224
    rng = np.random.default_rng(37)
    L, tol = 256, 1e-8
    th, ph = _caps(rng, 80, 0.25)
    pc = pf.Plan(th, ph, lmax=L, tol=tol, method="multibox")
    assert pc.info["kind"] == "multibox" and pc.algorithm == "MultiBoxAlgorithm"
    assert len(pc.boxes()) == 2
    alm = O.rand_alm(L, rng=rng)[:, :, 0]
    fd = O.Direct(th, ph, L).forward(alm)[:, 0]
    fc = _fwd(pc, alm)
    assert rel(fc, fd) < 10 * tol
    g = cn(rng, len(th))
    assert dot_rel(fc, g, alm, _adj(pc, g)) < 1e-12


def test_auto_picks_multibox_and_equals_its_boxes(pf, O, cuda):
    rng = np.random.default_rng(74)
    L, tol = 512, 1e-8
    th, ph = _caps(rng, 2000, 0.2)
    p = pf.Plan(th, ph, lmax=L, tol=tol)
    assert p.info["kind"] == "multibox"
    boxes = p.boxes()
    groups, _, _ = pf.partition_boxes(th, ph, lmax=L, tol=tol)
    assert len(boxes) == len(groups) == 2
    for b, g in zip(boxes, groups):
        assert np.array_equal(b["indices"], g)
        assert b["kind"] == "pole" and b["npts"] == len(g)
    assert p.ring_work() == sum(b["ring_work"] for b in boxes)
    alm = O.rand_alm(L, rng=rng)[:, :, 0]
    g = cn(rng, len(th))
    f = _fwd(p, alm)
    a = _adj(p, g)
    fsum = np.zeros_like(f)
    asum = np.zeros_like(a)
    for b in boxes:
        idx = b["indices"]
        pb = pf.Plan(th[idx], ph[idx], lmax=L, tol=tol, method="stretch",
                     fft_lengths=(b["nf1"], b["nf2"]))
        fsum[idx] = _fwd(pb, alm)
        asum += _adj(pb, np.ascontiguousarray(g[idx]))
    # the same leaves on the same points: the forward is the same arithmetic, the adjoint's
    # atomically added partial sums agree to their order
    assert np.array_equal(f, fsum)
    assert O.alm_reldiff(a, asum, L) < 1e-13
    assert dot_rel(f, g, alm, a) < 1e-12


@pytest.mark.parametrize("B", [1, 3])
def test_ntrans_mixed_and_host_buffers(pf, O, cuda, B):
    rng = np.random.default_rng(75 + B)
    L = 300
    th, ph = _caps(rng, 1500, 0.22)
    M = len(th)
    p64 = pf.Plan(th, ph, lmax=L, tol=1e-8, ntrans=B, method="multibox")
    pmx = pf.Plan(th, ph, lmax=L, tol=1e-6, ntrans=B, method="multibox", precision="mixed")
    assert pmx.info["precision"] == 1 and all(b["precision"] == 1 for b in pmx.boxes())
    alm = O.rand_alm(L, ntrans=B, rng=rng)
    alm = alm[:, :, 0] if B == 1 else alm
    f64 = _fwd(p64, alm)
    assert rel(_fwd(pmx, alm), f64) < 2e-5
    # host-buffer applies through the C ABI equal the device applies
    ah = pf.zeros_alm(L, B, device="pinned")
    ah[...] = alm
    fh = pf.zeros_field(M, B, device="pinned")
    p64.mul(fh, ah)
    assert np.array_equal(fh, f64)
    g = cn(rng, M) if B == 1 else np.asfortranarray(cn(rng, M, B))
    gh = pf.zeros_field(M, B, device="pinned")
    gh[...] = g
    a_host = pf.zeros_alm(L, B, device="pinned")
    p64.mul_adjoint(a_host, gh)
    a_dev = _adj(p64, g)
    assert O.alm_reldiff(a_host, a_dev, L) < 1e-13
    for b in range(B):
        sel = (lambda x: x) if B == 1 else (lambda x: x[..., b])
        assert dot_rel(sel(f64), sel(g), sel(alm), sel(a_dev)) < 1e-12


def test_multibox_in_the_serving_loop_not_in_batches(pf, O, cuda):
    rng = np.random.default_rng(79)
    L = 200
    th, ph = _caps(rng, 800, 0.25)
    p = pf.Plan(th, ph, lmax=L, tol=1e-8, method="multibox")
    with pytest.raises(Exception):
        pf.Batch([p])
    with pytest.raises(Exception):
        pf.ring_forward(p, pf.zeros_alm(L, device=cuda),
                        to_dev(np.zeros((10, 2 * L + 1, 1), np.complex128, order="F")))
    srv = pf.Server(hbm_budget_gb=10, nslots=2)
    pid = srv.add(p)
    a = pf.zeros_alm(L, device="pinned")
    a[...] = O.rand_alm(L, rng=rng)[:, :, 0]
    out = pf.zeros_field(len(th), device="pinned")
    rid = srv.submit(pid, True, a, out)
    srv.wait(rid)
    ref = pf.zeros_field(len(th), device="pinned")
    p.mul(ref, a)
    assert np.array_equal(out, ref)
    srv.close()
    # stage profile of a multi-box plan sums its boxes' stages
    p.profile_start()
    _ = p * to_dev(np.asfortranarray(a))
    st = p.profile_stop()
    assert st["ring_fwd"][1] == 2 and st["interp"][1] == 2


def test_device_planner_equals_host_planner(pf, O, cuda):
    # the planner's scans on the device give the host planner's boxes, groups and costs
    import torch
    rng = np.random.default_rng(80)
    sets = []
    th, ph = _caps(rng, 40000, 0.2)
    sets.append((th, ph, 512))
    t, p = [], []
    for k in range(5):
        t.append(0.6 + 0.3 * k + 0.05 * rng.random(9000))
        p.append(1.2 * k + 0.1 * rng.random(9000) - 2.0)  # negative longitudes: reduced mod 2 pi
    sets.append((np.concatenate(t), np.concatenate(p), 1024))
    half = np.deg2rad(8)
    sets.append((np.pi / 2 + half * (2 * rng.random(60000) - 1), 2 * np.pi * rng.random(60000), 256))
    sets.append((np.full(5000, 1.0), np.concatenate([0.05 * rng.random(2500),
                                                     2 * np.pi - 0.05 * rng.random(2500)]), 128))
    for th, ph, L in sets:
        dth = torch.from_numpy(th).to(cuda)
        dph = torch.from_numpy(ph).to(cuda)
        assert pf.bounding_box(dth, dph) == pf.bounding_box(th, ph)
        for mb in (3, 8):
            gh, bh, ch = pf.partition_boxes(th, ph, lmax=L, tol=1e-8, maxboxes=mb)
            gd, bd, cd = pf.partition_boxes(dth, dph, lmax=L, tol=1e-8, maxboxes=mb)
            assert len(gh) == len(gd)
            for a, b in zip(gh, gd):
                assert np.array_equal(a, b)
            assert bh == bd and ch == cd
        assert pf.select_method(dth, dph, lmax=L, tol=1e-8) == pf.select_method(th, ph, lmax=L, tol=1e-8)
    # a plan of >= 2^15 points is planned on the device: the same boxes as the host partition
    th, ph, L = sets[0]
    plan = pf.Plan(torch.from_numpy(th).to(cuda), torch.from_numpy(ph).to(cuda), lmax=L, tol=1e-8)
    assert plan.info["kind"] == "multibox"
    gh, _, _ = pf.partition_boxes(th, ph, lmax=L, tol=1e-8)
    assert [list(b["indices"]) for b in plan.boxes()] == [list(g) for g in gh]
    alm = O.rand_alm(L, rng=rng)[:, :, 0]
    g = cn(rng, len(th))
    f = _fwd(plan, alm)
    assert dot_rel(f, g, alm, _adj(plan, g)) < 1e-12
