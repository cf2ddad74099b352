"""Device applies against the direct sum, on the reference's own transform test cases
(test/test_transforms.jl), plus the lower seams (NUFFT, DFS), the host-buffer entry points,
batching, determinism and the degree-split adjoint ring pass."""
import numpy as np
import pytest

from helpers import cap_points, cn, dot_rel, plan_grid, rel, to_dev, to_host

pytestmark = pytest.mark.gpu

THETA_STAR = np.deg2rad(20.0)


def _sqrt_cap(rng, n):
    # test/test_transforms.jl:67-68: theta* sqrt(u), phi uniform
    return THETA_STAR * np.sqrt(rng.random(n)), 2 * np.pi * rng.random(n)


def _randn_alm(O, L, rng, B=1):
    # randn(ComplexF64, coeff_size(L)...) with the padding slots cleared
    return O.rand_alm(L, ntrans=B, rng=rng)


def _fwd(plan, alm):
    return to_host(plan * to_dev(alm if alm.shape[2] > 1 else alm[:, :, 0]))


def _adj(plan, g):
    return to_host(plan.H * to_dev(g))


@pytest.mark.parametrize("L", [128, 256, 512])
@pytest.mark.parametrize("tol", [1e-4, 1e-8])
def test_stretch_vs_direct_across_degree_and_tolerance(pf, O, cuda, L, tol):
    # test/test_transforms.jl:59-83: delivered accuracy at or better than the tolerance
    rng = np.random.default_rng(32 + L)
    th, ph = _sqrt_cap(rng, 150)
    ps = pf.Plan(th, ph, lmax=L, tol=tol, method="stretch")
    pd = pf.Plan(th, ph, lmax=L, method="direct")
    alm = _randn_alm(O, L, rng)
    fd_ref = O.Direct(th, ph, L).forward(alm, nthreads=8)[:, 0]
    fd = _fwd(pd, alm)
    fs = _fwd(ps, alm)
    assert rel(fd, fd_ref) < 1e-12
    assert rel(fs, fd_ref) < 10 * tol
    assert ps.info["nph"] % 2 == 0


def test_worst_case_spectra(pf, O, cuda):
    # test/test_transforms.jl:85-110: a single l = lmax row, and a red spectrum
    rng = np.random.default_rng(33)
    L, tol = 256, 1e-8
    th, ph = _sqrt_cap(rng, 200)
    ps = pf.Plan(th, ph, lmax=L, tol=tol, method="stretch")
    ref = O.Direct(th, ph, L)
    alm = O.zeros_alm(L)
    for m in range(-L, L + 1):
        alm[O.sph_mode(L, m) + (0,)] = rng.standard_normal() + 1j * rng.standard_normal()
    assert rel(_fwd(ps, alm), ref.forward(alm)[:, 0]) < 10 * tol
    almr = O.rand_alm(L, rng=rng, weight=lambda l: 1.0 / (1 + l) ** 2)
    assert rel(_fwd(ps, almr), ref.forward(almr)[:, 0]) < 10 * tol


@pytest.mark.parametrize("L", [256, 512])
def test_adjoint_is_exact_transpose(pf, O, cuda, L):
    # test/test_transforms.jl:112-123
    rng = np.random.default_rng(34)
    th, ph = _sqrt_cap(rng, 120)
    ps = pf.Plan(th, ph, lmax=L, tol=1e-8, method="stretch")
    alm = _randn_alm(O, L, rng)
    g = cn(rng, 120)
    assert dot_rel(_fwd(ps, alm), g, alm[:, :, 0], _adj(ps, g)) < 1e-12


@pytest.mark.parametrize("centre", [0.9, np.pi - 0.3])
def test_off_pole_and_southern_patches(pf, O, cuda, centre):
    # test/test_transforms.jl:125-140
    rng = np.random.default_rng(35)
    L, tol = 256, 1e-8
    th = centre + 0.12 * (2 * rng.random(150) - 1)
    ph = 1.0 + 0.4 * rng.random(150)
    ps = pf.Plan(th, ph, lmax=L, tol=tol, method="stretch")
    if centre > np.pi / 2:
        assert ps.info["flip"] == 1
    alm = _randn_alm(O, L, rng)
    f = _fwd(ps, alm)
    assert rel(f, O.Direct(th, ph, L).forward(alm)[:, 0]) < 10 * tol
    g = cn(rng, 150)
    assert dot_rel(f, g, alm[:, :, 0], _adj(ps, g)) < 1e-12
    # and the device apply agrees with the oracle's own stretched leaf at round-off
    so = O.Stretch(th, ph, L, tol, nufft="es", nufft_grid=plan_grid(ps))
    assert rel(f, so.forward(alm)[:, 0]) < 1e-11
    assert O.alm_reldiff(_adj(ps, g), so.adjoint(g)[:, :, 0], L) < 1e-10


def test_interior_patch_matches_oracle(pf, O, cuda):
    # a band that is cheapest as an interior periodisation (no DFS reflection)
    rng = np.random.default_rng(4)
    L = 1024
    th = 0.9 + 0.12 * (2 * rng.random(3000) - 1)
    ph = 2 * np.pi * rng.random(3000)
    ps = pf.Plan(th, ph, lmax=L, tol=1e-8, method="stretch")
    assert ps.info["kind"] == "interior"
    so = O.Stretch(th, ph, L, 1e-8, nufft="es", nufft_grid=plan_grid(ps))
    alm = O.rand_alm(L, rng=rng)
    f = _fwd(ps, alm)
    assert rel(f, so.forward(alm, nthreads=8)[:, 0]) < 1e-11
    g = cn(rng, 3000)
    a = _adj(ps, g)
    assert O.alm_reldiff(a, so.adjoint(g, nthreads=8)[:, :, 0], L) < 1e-10
    assert dot_rel(f, g, alm[:, :, 0], a) < 1e-12


@pytest.mark.parametrize("B", [3, 5])
def test_ntrans_batching(pf, O, cuda, B):
    # test/test_transforms.jl:142-156; B = 3 runs the 2-transform kernels then a single one,
    # B = 5 the 4-transform kernels then a single one
    rng = np.random.default_rng(36)
    L = 256
    th, ph = _sqrt_cap(rng, 100)
    p1 = pf.Plan(th, ph, lmax=L, tol=1e-8, method="stretch")
    pB = pf.Plan(th, ph, lmax=L, tol=1e-8, method="stretch", ntrans=B)
    almB = _randn_alm(O, L, rng, B)
    fB = _fwd(pB, almB)
    g = np.asfortranarray(cn(rng, 100, B))
    aB = _adj(pB, g)
    for b in range(B):
        assert rel(fB[:, b], _fwd(p1, almB[:, :, b:b + 1])) < 1e-9
        assert O.alm_reldiff(aB[:, :, b], _adj(p1, np.ascontiguousarray(g[:, b])), L) < 1e-9


def test_direct_leaf_matches_ylm(pf, O, cuda):
    # test/test_transforms.jl:20-57: the Direct leaf against the closed form and its adjoint
    rng = np.random.default_rng(31)
    L = 64
    th = np.pi * rng.random(300)
    ph = 2 * np.pi * rng.random(300)
    pd = pf.Plan(th, ph, lmax=L, method="direct")
    assert pd.algorithm == "DirectAlgorithm"
    alm = _randn_alm(O, L, rng)
    ref = O.Direct(th, ph, L)
    f = _fwd(pd, alm)
    assert rel(f, ref.forward(alm)[:, 0]) < 1e-13
    g = cn(rng, 300)
    a = _adj(pd, g)
    assert O.alm_reldiff(a, ref.adjoint(g)[:, :, 0], L) < 1e-13
    assert dot_rel(f, g, alm[:, :, 0], a) < 1e-13
    # single harmonics against the closed form (test/test_transforms.jl:33-43)
    for (l, m) in [(0, 0), (5, -3), (17, 17), (64, -1)]:
        e = O.zeros_alm(L)
        e[O.sph_mode(l, m) + (0,)] = 1.0
        y = np.array([O.ylm(l, m, t, p) for t, p in zip(th[:20], ph[:20])])
        assert np.abs(_fwd(pd, e)[:20] - y).max() < 1e-13


@pytest.mark.parametrize("L,B", [(256, 1), (700, 1), (300, 3)])
def test_host_buffers_equal_device_applies(pf, O, cuda, L, B):
    # pfsht_forward_host / pfsht_adjoint_host move the sph_mode staircase in blocks of orders:
    # what the padding slots hold on input is ignored, and the adjoint leaves them zero
    rng = np.random.default_rng(40)
    th, ph = cap_points(20000, rng=rng)
    ps = pf.Plan(th, ph, lmax=L, tol=1e-8, ntrans=B)
    alm = O.rand_alm(L, ntrans=B, rng=rng)
    pad = ~O.valid_mask(L)
    dirty = alm.copy(order="F")
    dirty[pad] = np.nan
    # orders above the plan's retained maximum are not read either (the polar truncation)
    mu = ps.info["mmax"]
    assert mu < L
    dirty[:, 2 * mu + 1:] = np.nan
    a_in = np.asfortranarray(dirty if B > 1 else dirty[:, :, 0])
    f_host = pf.zeros_field(len(th), ntrans=B, device="cpu")
    ps.mul(f_host, a_in)
    f_dev = _fwd(ps, alm)
    assert np.array_equal(f_host, f_dev)
    g = np.asfortranarray(cn(rng, len(th), B)) if B > 1 else cn(rng, len(th))
    a_host = pf.zeros_alm(L, ntrans=B, device="cpu")
    a_host[...] = np.nan
    ps.mul_adjoint(a_host, g)
    a_dev = _adj(ps, g)
    a3 = a_host if B > 1 else a_host[:, :, None]
    assert np.all(a3[pad] == 0)
    # the adjoint adds some partial sums atomically: equal up to the order of those additions
    assert O.alm_reldiff(a_host, a_dev, L) < 1e-14
    assert np.all(a3[:, 2 * mu + 1:] == 0)
    # the coefficient staircase of the orders up to mmax crosses PCIe, in blocks of orders
    hb = ps.host_bytes()
    valid = ((L + 1) + 2 * sum(L + 1 - m for m in range(1, mu + 1))) * 16 * B
    assert valid <= hb["h2d_forward"] < 1.15 * valid
    assert hb["d2h_adjoint"] == hb["h2d_forward"]
    assert hb["d2h_forward"] == hb["h2d_adjoint"] == len(th) * 16 * B


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-8), ("mixed", 1e-6)])
def test_adjoint_is_deterministic(pf, O, cuda, precision, tol):
    # with the deterministic option, spreading runs its bins in colours whose tiles are disjoint
    # (plain adds, fixed order) and the ring pass holds each order's rings in one warp: two
    # adjoints agree bit for bit, as the reference's threaded and serial adjoints do
    # (test/test_backends.jl:202-259); they equal the default plan's to round-off
    rng = np.random.default_rng(43)
    L = 512
    th, ph = cap_points(50000, rng=rng)
    ps = pf.Plan(th, ph, lmax=L, tol=tol, precision=precision, deterministic=True)
    g = to_dev(cn(rng, len(th)))
    a1 = to_host(ps.H * g)
    a2 = to_host(ps.H * g)
    assert np.array_equal(a1, a2)
    pd = pf.Plan(th, ph, lmax=L, tol=tol, precision=precision)
    assert O.alm_reldiff(a1, to_host(pd.H * g), L) < (2e-6 if precision == "mixed" else 1e-13)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-8), ("mixed", 1e-6)])
def test_tma_transposes_equal_plain_ones(pf, O, cuda, precision, tol):
    # the NUFFT's fine-row transposes with TMA-staged tiles move the same values as the plain-load
    # kernels: forwards agree bit for bit, adjoints to the order of their atomic additions; every
    # bounded tile wait ended
    import ctypes as C
    rng = np.random.default_rng(45)
    L = 700
    th, ph = cap_points(60000, rng=rng)
    pt = pf.Plan(th, ph, lmax=L, tol=tol, precision=precision)
    pp = pf.Plan(th, ph, lmax=L, tol=tol, precision=precision, transpose="plain")
    assert pt.info["nf1"] == pp.info["nf1"] and pt.info["nf2"] == pp.info["nf2"]
    alm = O.rand_alm(L, rng=rng)
    g = cn(rng, len(th))
    assert np.array_equal(_fwd(pt, alm), _fwd(pp, alm))
    assert O.alm_reldiff(_adj(pt, g), _adj(pp, g), L) < (2e-6 if precision == "mixed" else 1e-14)
    n = C.c_int32(-1)
    assert pf._lib.load().pfsht_wait_timeouts(C.byref(n)) == 0
    assert n.value == 0


@pytest.mark.parametrize("precision,tol,B", [("fp64", 1e-8, 1), ("mixed", 1e-6, 1), ("fp64", 1e-8, 2)])
def test_register_spreading_equals_window_spreading(pf, O, cuda, precision, tol, B):
    # spreading with each bin's tile held in registers adds the same products in the same order
    # per cell as the sliding-window kernel: with the deterministic option (plain adds, colour
    # order) the adjoints agree bit for bit, by default to the order of the atomic additions
    rng = np.random.default_rng(46)
    L = 600
    th, ph = cap_points(70000, rng=rng)
    kw = dict(lmax=L, tol=tol, precision=precision, ntrans=B, fft_lengths="minimal")
    g = to_dev(np.asfortranarray(cn(rng, len(th), B)) if B > 1 else cn(rng, len(th)))
    pr = pf.Plan(th, ph, deterministic=True, **kw)
    pw = pf.Plan(th, ph, deterministic=True, spread="window", **kw)
    assert np.array_equal(to_host(pr.H * g), to_host(pw.H * g))
    ar = to_host(pf.Plan(th, ph, **kw).H * g)
    aw = to_host(pf.Plan(th, ph, spread="window", **kw).H * g)
    assert O.alm_reldiff(ar, aw, L) < (2e-6 if precision == "mixed" else 1e-13)


@pytest.mark.parametrize("bin_rows,bin_cols", [(32, 0), (9, 4), (1, 1)])
def test_spreading_bin_shapes(pf, O, cuda, bin_rows, bin_cols):
    # bins taller than the register tile holds (32 rows at w = 9) fall back to the sliding
    # window; short and narrow bins use the register tile with few row pairs: every shape gives
    # the default plan's adjoint to the order of the atomic additions, and its forward
    rng = np.random.default_rng(47)
    L = 400
    th, ph = cap_points(40000, rng=rng)
    kw = dict(lmax=L, tol=1e-8, fft_lengths="minimal")
    g = to_dev(cn(rng, len(th)))
    alm = O.rand_alm(L, rng=rng)
    pd = pf.Plan(th, ph, **kw)
    ps = pf.Plan(th, ph, bin_rows=bin_rows, bin_cols=bin_cols, **kw)
    assert O.alm_reldiff(to_host(ps.H * g), to_host(pd.H * g), L) < 1e-13
    fd, fs = _fwd(pd, alm), _fwd(ps, alm)
    assert np.max(np.abs(fs - fd)) <= 1e-13 * np.max(np.abs(fd))


@pytest.mark.parametrize("L,B", [(512, 1), (300, 2)])
def test_async_host_applies_in_flight_together(pf, O, cuda, L, B):
    # pfsht_forward_host_async / pfsht_adjoint_host_async: two rounds of a forward and an adjoint
    # issued back to back on one plan before one wait; each result equals its device apply
    import torch
    rng = np.random.default_rng(44)
    th, ph = cap_points(30000, rng=rng)
    ps = pf.Plan(th, ph, lmax=L, tol=1e-8, ntrans=B)

    def pinned(a):
        t = torch.from_numpy(np.ascontiguousarray(np.asarray(a).T)).pin_memory()
        return t.numpy().T

    rounds = []
    for _ in range(2):
        alm = O.rand_alm(L, ntrans=B, rng=rng)
        g = np.asfortranarray(cn(rng, len(th), B)) if B > 1 else cn(rng, len(th))
        a_in = pinned(alm if B > 1 else alm[:, :, 0])
        g_in = pinned(g)
        f_out = pinned(np.zeros((len(th), B) if B > 1 else len(th), np.complex128))
        a_out = pinned(np.full(alm.shape if B > 1 else alm.shape[:2], np.nan, np.complex128))
        ps.mul_async(f_out, a_in)
        ps.mul_adjoint_async(a_out, g_in)
        rounds.append((alm, g, f_out, a_out))
    ps.host_sync()
    for alm, g, f_out, a_out in rounds:
        assert np.array_equal(f_out, _fwd(ps, alm))
        assert O.alm_reldiff(a_out, _adj(ps, g), L) < 1e-14
        a3 = a_out if B > 1 else a_out[:, :, None]
        assert np.all(a3[~O.valid_mask(L)] == 0)


def test_forward_is_deterministic(pf, O, cuda):
    # the forward path has no atomics: two applies agree bit for bit
    rng = np.random.default_rng(41)
    L = 512
    th, ph = cap_points(50000, rng=rng)
    ps = pf.Plan(th, ph, lmax=L, tol=1e-8)
    alm = to_dev(O.rand_alm(L, rng=rng)[:, :, 0])
    f1 = to_host(ps * alm)
    f2 = to_host(ps * alm)
    assert np.array_equal(f1, f2)


@pytest.mark.parametrize("seg", [-1, 64, 192, 256, 1024])
def test_adjoint_degree_segments_match_oracle(pf, O, cuda, seg):
    # the adjoint ring pass split along the degree axis, each piece started from the
    # recurrence state saved at plan time, against the oracle's unsplit walk
    rng = np.random.default_rng(42)
    L = 512
    th, ph = cap_points(6000, rng=rng)
    plan = pf.Plan(th, ph, lmax=L, tol=1e-8, segment_degrees=seg)
    ref = O.Stretch(th, ph, L, 1e-8, nufft="es", nufft_grid=plan_grid(plan))
    n = plan.info["nrings"]
    Gr = np.asfortranarray(cn(rng, n, 2 * L + 1, 1))
    a = to_dev(np.zeros((L + 1, 2 * L + 1, 1), np.complex128, order="F"))
    pf.ring_adjoint(plan, to_dev(Gr), a)
    assert O.alm_reldiff(to_host(a), ref.rings.alm_from_rings(Gr), L) < 1e-12
    g = cn(rng, len(th))
    assert O.alm_reldiff(_adj(plan, g), ref.adjoint(g, nthreads=8)[:, :, 0], L) < 1e-10


def test_direct_plan_adjoint_segments(pf, O, cuda):
    # a direct plan over few points splits every order along the degree axis
    rng = np.random.default_rng(43)
    L = 700
    th = np.pi * rng.random(100)
    ph = 2 * np.pi * rng.random(100)
    ref = O.Direct(th, ph, L)
    g = cn(rng, 100)
    a_ref = ref.adjoint(g, nthreads=8)[:, :, 0]
    for seg in (-1, 128, 0):
        pd = pf.Plan(th, ph, lmax=L, method="direct", segment_degrees=seg)
        assert O.alm_reldiff(_adj(pd, g), a_ref, L) < 1e-12


@pytest.mark.parametrize("typ", [1, 2])
def test_nufft_seam_matches_direct_sum(pf, O, cuda, typ):
    # src/NUFFT.jl:17-25 seam against the DirectSum backend (src/NUFFT.jl:85-129)
    rng = np.random.default_rng(44)
    n1, n2, M, tol = 40, 30, 500, 1e-9
    x = 2 * np.pi * rng.random(M) - np.pi
    y = 4 * np.pi * rng.random(M) - 2 * np.pi   # any real values, taken modulo 2 pi
    p = pf.NUFFT(typ, n1, n2, +1 if typ == 2 else -1, x, y, tol)
    if typ == 2:
        c = np.asfortranarray(cn(rng, n1, n2))
        out = to_dev(np.zeros(M, np.complex128))
        p.exec(to_dev(c), out)
        ref = O.nufft_direct(2, n1, n2, +1, x, y, c)[:, 0]
    else:
        c = cn(rng, M)
        out = to_dev(np.zeros((n1, n2), np.complex128, order="F"))
        p.exec(to_dev(c), out)
        ref = O.nufft_direct(1, n1, n2, -1, x, y, c)[:, :, 0]
    assert rel(to_host(out), ref) < 200 * tol


def test_timed_fine_grid_lengths(pf, O, cuda):
    # NUFFT fine-grid lengths picked by timing the library FFT: within 10% above the minimum,
    # the same for the same shape within a process, and the transform agrees with the
    # minimal-length plan to the tolerance
    rng = np.random.default_rng(90)
    th, ph = cap_points(20000, rng=rng)
    L, tol = 700, 1e-8
    pt = pf.Plan(th, ph, lmax=L, tol=tol)
    pm = pf.Plan(th, ph, lmax=L, tol=tol, fft_lengths="minimal")
    geo = pf.plan_geometry(th, ph, lmax=L, tol=tol)
    assert plan_grid(pm) == (geo["nf1"], geo["nf2"])
    for a, b in zip(plan_grid(pt), plan_grid(pm)):
        assert b <= a <= b + b // 10
    assert plan_grid(pf.Plan(th, ph, lmax=L, tol=tol)) == plan_grid(pt)
    alm = O.rand_alm(L, rng=rng)
    assert rel(_fwd(pt, alm), _fwd(pm, alm)) < 10 * tol
    g = cn(rng, len(th))
    assert O.alm_reldiff(_adj(pt, g), _adj(pm, g), L) < 10 * tol
    with pytest.raises(ValueError):
        pf.Plan(th, ph, lmax=L, tol=tol, fft_lengths="fast")
    # lengths given explicitly: the same transform as the timed plan that chose them
    pg = pf.Plan(th, ph, lmax=L, tol=tol, fft_lengths=plan_grid(pt))
    assert plan_grid(pg) == plan_grid(pt)
    assert np.array_equal(_fwd(pg, alm), _fwd(pt, alm))
    with pytest.raises(ValueError):
        pf.Plan(th, ph, lmax=L, tol=tol, fft_lengths=(pm.info["nf1"] - 1, pm.info["nf2"]))


@pytest.mark.parametrize("typ,iflag", [(1, 1), (1, -1), (2, 1), (2, -1)])
def test_nufft_seam_both_signs_odd_sizes(pf, O, cuda, typ, iflag):
    # either exponent sign in both types, odd mode counts
    rng = np.random.default_rng(82 + typ + iflag)
    n1, n2, M, tol = 45, 27, 700, 1e-9
    x = 2 * np.pi * rng.random(M) - np.pi
    y = 2 * np.pi * rng.random(M)
    p = pf.NUFFT(typ, n1, n2, iflag, x, y, tol)
    if typ == 2:
        c = np.asfortranarray(cn(rng, n1, n2))
        out = to_dev(np.zeros(M, np.complex128))
        p.exec(to_dev(c), out)
        ref = O.nufft_direct(2, n1, n2, iflag, x, y, c)[:, 0]
    else:
        c = cn(rng, M)
        out = to_dev(np.zeros((n1, n2), np.complex128, order="F"))
        p.exec(to_dev(c), out)
        ref = O.nufft_direct(1, n1, n2, iflag, x, y, c)[:, :, 0]
    assert rel(to_host(out), ref) < 200 * tol


@pytest.mark.parametrize("spin", [0, 1])
def test_dfs_kernels_match_oracle(pf, O, cuda, spin):
    # src/DFS.jl:13-56: device dfs_double! / dfs_fold! against the oracle, bit for bit
    rng = np.random.default_rng(45)
    F = np.asfortranarray(cn(rng, 9, 12, 2))
    Ft = to_dev(np.zeros((18, 12, 2), np.complex128, order="F"))
    pf.dfs_double(to_dev(F), Ft, spin=spin)
    assert np.array_equal(to_host(Ft), O.dfs_double(F, spin=spin))
    T = np.asfortranarray(cn(rng, 18, 12, 2))
    Fd = to_dev(np.zeros((9, 12, 2), np.complex128, order="F"))
    pf.dfs_fold(to_dev(T), Fd, spin=spin)
    assert np.array_equal(to_host(Fd), O.dfs_fold(T, spin=spin))


def test_refused_geometry_runs_the_direct_leaf(pf, O, cuda):
    # src/Windows.jl:66-75 with src/Cost.jl:121-122: AUTO answers a refused geometry with the
    # direct leaf on the device
    rng = np.random.default_rng(0)
    th = 0.02 + 0.03 * rng.random(50)
    ph = rng.random(50)
    with pytest.raises(pf.RefusedGeometry):
        pf.Plan(th, ph, lmax=32, tol=1e-10, method="stretch")
    p = pf.Plan(th, ph, lmax=32, tol=1e-10)
    assert p.info["kind"] == "direct"
    alm = _randn_alm(O, 32, rng)
    assert rel(_fwd(p, alm), O.Direct(th, ph, 32).forward(alm)[:, 0]) < 1e-13


def test_bench_workload_dot_and_direct_subsample(pf, O, cuda):
    # lmax 2048 on the 20-degree cap: size-independent checks at full size. The adjoint is
    # the transpose at round-off; on a subsample of points the forward matches the direct sum
    # within 10 tol (the reference's accuracy gate)
    rng = np.random.default_rng(46)
    L, tol = 2048, 1e-8
    M = int(round((L * THETA_STAR) ** 2 * 4))
    th, ph = cap_points(M, rng=rng)
    ps = pf.Plan(th, ph, lmax=L, tol=tol)
    alm = O.rand_alm(L, rng=rng)
    f = _fwd(ps, alm)
    g = cn(rng, M)
    a = _adj(ps, g)
    assert dot_rel(f, g, alm[:, :, 0], a) < 1e-12
    idx = rng.choice(M, 24, replace=False)
    fd = O.Direct(th[idx], ph[idx], L).forward(alm, nthreads=8)[:, 0]
    assert rel(f[idx], fd) < 10 * tol
