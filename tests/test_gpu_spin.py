"""Spin-weighted plans on the device (src/Spin.jl) against the oracle's SpinRings, SpinDirect and
spin stretched leaf, and the reference's spin testset (test/test_spin.jl)."""
import numpy as np
import pytest

from helpers import cap_points, cn, dot_rel, plan_grid, rel, to_dev, to_host

pytestmark = pytest.mark.gpu


def _fwd(plan, alm):
    return to_host(plan * to_dev(np.asfortranarray(alm)))


def _adj(plan, g):
    return to_host(plan.H * to_dev(np.asfortranarray(g)))


def _spin_rel(O, a, b, L, s):
    """Largest difference over the valid spin coefficients relative to the largest reference."""
    mask = O.spin_valid_mask(L, s)
    a = np.asarray(a).reshape(L + 1, 2 * L + 1, -1)
    b = np.asarray(b).reshape(L + 1, 2 * L + 1, -1)
    return float(np.abs(a - b)[mask].max() / np.abs(b[mask]).max())


@pytest.mark.parametrize("s", [1, 2, -2, 3])
def test_spin_direct_matches_oracle(pf, O, cuda, s):
    # SpinDirectLeaf (src/Spin.jl:557-630) on the whole sphere, poles included
    rng = np.random.default_rng(90 + s)
    L, M = 64, 400
    th = np.arccos(2 * rng.random(M) - 1)
    th[:3] = [0.0, np.pi, np.pi / 2]
    ph = 2 * np.pi * rng.random(M)
    plan = pf.Plan(th, ph, lmax=L, tol=1e-10, method="direct", spin=s)
    assert plan.info["kind"] == "direct" and plan.info["spin"] == s
    ref = O.SpinDirect(th, ph, L, s)
    alm = O.rand_spin_alm(L, s, rng=rng)
    f = _fwd(plan, alm[:, :, 0])
    assert rel(f, ref.forward(alm)[:, 0]) < 1e-12
    g = cn(rng, M)
    a = _adj(plan, g)
    assert _spin_rel(O, a, ref.adjoint(g)[:, :, 0], L, s) < 1e-12
    # entries below l = max(|m|, |s|) are zero after the adjoint
    assert np.all(a[~O.spin_valid_mask(L, s)] == 0)
    assert dot_rel(f, g, alm[:, :, 0], a) < 1e-12


@pytest.mark.parametrize("s,caps", [(2, "north"), (-1, "south"), (3, "band")])
def test_spin_ring_pass_matches_oracle(pf, O, cuda, s, caps):
    rng = np.random.default_rng(100 + s)
    L, tol = 256, 1e-8
    th, ph = cap_points(3000, rng=rng)
    if caps == "south":
        th = np.pi - th
    elif caps == "band":
        th = np.pi / 2 + 0.3 * (2 * rng.random(3000) - 1)
    plan = pf.Plan(th, ph, lmax=L, tol=tol, method="stretch", spin=s)
    ref = O.Stretch(th, ph, L, tol, nufft="es", nufft_grid=plan_grid(plan), spin=s)
    rings = O.SpinRings(ref.tables()["theta_rings"], L, s, tol, reflect=bool(plan.info["flip"]))
    assert plan.ring_work() == rings.ring_work() == ref.ring_work()
    assert plan.info["mmax"] == rings.mmax
    alm = O.rand_spin_alm(L, s, rng=rng)
    n = plan.info["nrings"]
    G = to_dev(np.zeros((n, 2 * L + 1, 1), np.complex128, order="F"))
    pf.ring_forward(plan, to_dev(alm), G)
    assert rel(to_host(G), rings.rings_from_alm(alm)) < 1e-11
    Gr = np.asfortranarray(cn(rng, n, 2 * L + 1, 1))
    a = to_dev(np.zeros_like(alm, order="F"))
    pf.ring_adjoint(plan, to_dev(Gr), a)
    assert _spin_rel(O, to_host(a), rings.alm_from_rings(Gr), L, s) < 1e-11


@pytest.mark.parametrize("s,where", [(2, "north"), (1, "south"), (-2, "band")])
def test_spin_stretch_apply_matches_oracle(pf, O, cuda, s, where):
    rng = np.random.default_rng(110 + s)
    L, tol, M = 256, 1e-8, 5000
    th, ph = cap_points(M, rng=rng)
    if where == "south":
        th = np.pi - th
    elif where == "band":
        th = np.pi / 2 + 0.25 * (2 * rng.random(M) - 1)
    plan = pf.Plan(th, ph, lmax=L, tol=tol, method="stretch", spin=s)
    ref = O.Stretch(th, ph, L, tol, nufft="es", nufft_grid=plan_grid(plan), spin=s)
    info = plan.info
    assert (info["nth"], info["nph"], info["mmax"]) == (ref.info["nth"], ref.info["nph"],
                                                          ref.info["mmax"])
    alm = O.rand_spin_alm(L, s, rng=rng)
    f = _fwd(plan, alm[:, :, 0])
    assert rel(f, ref.forward(alm, nthreads=8)[:, 0]) < 1e-11
    g = cn(rng, M)
    a = _adj(plan, g)
    assert _spin_rel(O, a, ref.adjoint(g, nthreads=8)[:, :, 0], L, s) < 1e-10
    assert dot_rel(f, g, alm[:, :, 0], a) < 1e-12


def test_spin_stretch_against_spin_direct(pf, O, cuda):
    # test/test_spin.jl:160-175: the stretched spin leaf against SpinDirect at 10 tol
    L, tol = 256, 1e-8
    for s in (1, 2, -1):
        rng = np.random.default_rng(42 + s)
        th = np.deg2rad(20) * np.sqrt(rng.random(120))
        ph = 2 * np.pi * rng.random(120)
        a = np.asfortranarray(cn(rng, L + 1, 2 * L + 1))
        fd = O.SpinDirect(th, ph, L, s).forward(a)[:, 0]
        plan = pf.Plan(th, ph, lmax=L, tol=tol, method="stretch", spin=s)
        fs = _fwd(plan, a)
        assert rel(fs, fd) < 10 * tol
        g = cn(rng, 120)
        assert dot_rel(fs, g, a, _adj(plan, g)) < 1e-12


def test_spin_multibox_host_buffers_and_mixed(pf, O, cuda):
    # two caps as a multi-box plan of spin 2 (src/MultiBox.jl:50 passes spin to every box)
    rng = np.random.default_rng(120)
    L, tol, s = 200, 1e-8, 2
    n1 = 600
    th = np.concatenate([0.25 * np.sqrt(rng.random(n1)), np.pi - 0.25 * np.sqrt(rng.random(n1))])
    ph = 2 * np.pi * rng.random(2 * n1)
    plan = pf.Plan(th, ph, lmax=L, tol=tol, method="multibox", spin=s)
    assert plan.info["kind"] == "multibox" and all(b["spin"] == s for b in plan.boxes())
    alm = O.rand_spin_alm(L, s, rng=rng)[:, :, 0]
    fd = O.SpinDirect(th, ph, L, s).forward(alm)[:, 0]
    f = _fwd(plan, alm)
    assert rel(f, fd) < 10 * tol
    g = cn(rng, len(th))
    a = _adj(plan, g)
    assert dot_rel(f, g, alm, a) < 1e-12
    # host-buffer applies move the columns of the retained orders and equal the device applies
    hb = plan.host_bytes()
    mu = max(b["mmax"] for b in plan.boxes())
    assert mu < L and hb["h2d_forward"] == 16 * (L + 1) * (2 * mu + 1)
    ah = pf.zeros_alm(L, device="pinned")
    ah[...] = alm
    fh = pf.zeros_field(len(th), device="pinned")
    plan.mul(fh, ah)
    assert np.array_equal(fh, f)
    gh = pf.zeros_field(len(th), device="pinned")
    gh[...] = g
    a_host = pf.zeros_alm(L, device="pinned")
    a_host[...] = 1.0  # overwritten, padding included
    plan.mul_adjoint(a_host, gh)
    assert _spin_rel(O, a_host, a, L, s) < 1e-13
    assert np.all(np.asarray(a_host)[~O.spin_valid_mask(L, s)] == 0)
    # mixed precision: FP32 NUFFT, FP64 ring pass
    pmx = pf.Plan(th, ph, lmax=L, tol=1e-6, method="multibox", spin=s, precision="mixed")
    assert rel(_fwd(pmx, alm), fd) < 2e-5


def test_spin_rejections(pf, O, cuda):
    rng = np.random.default_rng(121)
    th, ph = cap_points(200, rng=rng)
    with pytest.raises(ValueError):
        pf.Plan(th, ph, lmax=4, tol=1e-8, spin=5)
    p = pf.Plan(th, ph, lmax=128, tol=1e-8, method="stretch", spin=1)
    p0 = pf.Plan(th, ph, lmax=128, tol=1e-8, method="stretch", spin=0)
    assert p0.info["spin"] == 0 and p.info["spin"] == 1
    assert "spin=1" in repr(p)


@pytest.mark.parametrize("method", ["stretch", "direct"])
def test_spin_ntrans_columns_and_serving(pf, O, cuda, method):
    # ntrans = 3: each column is the single-transform plan's result (src/Plan.jl:137-148 on
    # (lmax+1, 2lmax+1, ntrans) arrays); a spin plan also runs in the serving loop
    rng = np.random.default_rng(130)
    L, s, B = 160, -2, 3
    th, ph = cap_points(1500 if method == "stretch" else 300, rng=rng)
    M = len(th)
    p3 = pf.Plan(th, ph, lmax=L, tol=1e-8, method=method, spin=s, ntrans=B)
    p1 = pf.Plan(th, ph, lmax=L, tol=1e-8, method=method, spin=s)
    alm = O.rand_spin_alm(L, s, ntrans=B, rng=rng)
    g = np.asfortranarray(cn(rng, M, B))
    f3 = _fwd(p3, alm)
    a3 = _adj(p3, g)
    for b in range(B):
        assert rel(f3[:, b], _fwd(p1, alm[:, :, b])) < 1e-13
        assert _spin_rel(O, a3[:, :, b], _adj(p1, np.ascontiguousarray(g[:, b])), L, s) < 1e-13
        assert dot_rel(f3[:, b], g[:, b], alm[:, :, b], a3[:, :, b]) < 1e-12
    srv = pf.Server(hbm_budget_gb=4, nslots=2)
    pid = srv.add(p1)
    ah = pf.zeros_alm(L, device="pinned")
    ah[...] = alm[:, :, 0]
    out = pf.zeros_field(M, device="pinned")
    srv.wait(srv.submit(pid, True, ah, out))
    ref = pf.zeros_field(M, device="pinned")
    p1.mul(ref, ah)
    assert np.array_equal(out, ref)
    srv.close()


def test_spin_plans_in_a_batch(pf, O, cuda):
    # spin plans join batches with scalar plans: their ring passes run on the batch's streams,
    # the scalar plans' in the merged launches; every result equals the plan's own apply
    import torch
    rng = np.random.default_rng(140)
    plans = []
    th, ph = cap_points(2000, rng=rng)
    plans.append(pf.Plan(th, ph, lmax=192, tol=1e-8, method="stretch", spin=2))
    plans.append(pf.Plan(th, ph, lmax=192, tol=1e-8, method="stretch"))
    th2, ph2 = cap_points(300, theta_star=np.deg2rad(40.0), rng=rng)
    plans.append(pf.Plan(np.pi - th2, ph2, lmax=96, tol=1e-8, method="direct", spin=-1, ntrans=2))
    plans.append(pf.Plan(np.pi - th, ph, lmax=150, tol=1e-8, method="stretch", spin=3, ntrans=3))
    batch = pf.Batch(plans, nstreams=2)
    for call in range(2):  # new arrays on the second call: the pointer table changes
        alms, fins = [], []
        for p in plans:
            if p.spin:
                a = O.rand_spin_alm(p.lmax, p.spin, ntrans=p.ntrans, rng=rng)
            else:
                a = O.rand_alm(p.lmax, ntrans=p.ntrans, rng=rng)
            alms.append(to_dev(a if p.ntrans > 1 else a[:, :, 0]))
            g = cn(rng, p.npts, p.ntrans)
            fins.append(to_dev(g if p.ntrans > 1 else g[:, 0]))
        fb = [pf.zeros_field(p.npts, p.ntrans, device=cuda) for p in plans]
        ab = [pf.zeros_alm(p.lmax, p.ntrans, device=cuda) for p in plans]
        for x in ab:
            x.fill_(1.0)  # the batch adjoint overwrites every slot
        batch.forward(fb, alms)
        batch.adjoint(ab, fins)
        torch.cuda.synchronize()
        for p, a, f, fbi, abi in zip(plans, alms, fins, fb, ab):
            f1 = to_host(p * a)
            a1 = to_host(p.H * f)
            assert rel(to_host(fbi), f1) < 1e-14, (call, p)
            got = to_host(abi)
            assert np.abs(got - a1).max() <= 1e-13 * np.abs(a1).max(), (call, p)
            if p.spin:
                assert np.all(got.reshape(p.lmax + 1, 2 * p.lmax + 1, -1)[~O.spin_valid_mask(p.lmax, p.spin)] == 0)
