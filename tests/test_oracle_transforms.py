"""The oracle's Direct and stretched leaves against the reference's transform tests
(test/test_transforms.jl, test/test_backends.jl) and the mpmath fixtures."""
import json
import os

import numpy as np
import pytest

from helpers import cap_points, cn, dot_rel, rel

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_direct_matches_high_precision_sum(O):
    # test/test_transforms.jl:9-31: Direct against the explicit sum of a Y, gate 1e-13
    d = json.load(open(os.path.join(GOLDEN, "direct_small.json")))
    L = d["lmax"]
    alm = O.zeros_alm(L)
    for k, (l, m) in enumerate(d["modes"]):
        r, c = O.sph_mode(l, m)
        alm[r, c, 0] = d["alm_re"][k] + 1j * d["alm_im"][k]
    D = O.Direct(d["theta"], d["phi"], L)
    f = D.forward(alm)[:, 0]
    ref = np.array([a + 1j * b for a, b in d["f"]])
    assert np.abs(f - ref).max() / np.abs(ref).max() < 1e-13
    g = np.array(d["g_re"]) + 1j * np.array(d["g_im"])
    a = D.adjoint(g)
    adj_ref = np.array([x + 1j * y for x, y in d["adjoint"]])
    got = np.array([a[O.sph_mode(l, m)[0], O.sph_mode(l, m)[1], 0] for (l, m) in d["modes"]])
    assert np.abs(got - adj_ref).max() / np.abs(adj_ref).max() < 1e-13


def test_direct_single_harmonic_and_dot(O):
    # test/test_transforms.jl:33-43 and the Direct dot test
    rng = np.random.default_rng(32)
    L, n = 8, 25
    th = 0.5 * rng.random(n) + 0.1
    ph = 2 * np.pi * rng.random(n)
    D = O.Direct(th, ph, L)
    for (l, m) in ((0, 0), (1, -1), (5, 3), (8, -8)):
        alm = O.zeros_alm(L)
        r, c = O.sph_mode(l, m)
        alm[r, c, 0] = 1.0
        f = D.forward(alm)[:, 0]
        ref = np.array([O.ylm(l, m, th[i], ph[i]) for i in range(n)])
        assert np.abs(f - ref).max() < 1e-13
    alm = O.rand_alm(L, rng=rng)
    g = cn(rng, n)
    assert dot_rel(D.forward(alm), g, alm, D.adjoint(g)) < 1e-13


def test_direct_ntrans_per_column(O):
    # test/test_transforms.jl:45-56
    rng = np.random.default_rng(33)
    L, n, B = 12, 30, 3
    th, ph = 0.4 * rng.random(n), 2 * np.pi * rng.random(n)
    p1, pB = O.Direct(th, ph, L), O.Direct(th, ph, L, ntrans=B)
    almB = O.rand_alm(L, ntrans=B, rng=rng)
    fB = pB.forward(almB)
    for b in range(B):
        assert np.abs(fB[:, b] - p1.forward(almB[:, :, b:b + 1])[:, 0]).max() < 1e-13


@pytest.mark.parametrize("L", [128, 256, 512])
@pytest.mark.parametrize("tol", [1e-4, 1e-8])
def test_stretch_vs_direct(O, L, tol):
    # test/test_transforms.jl:59-82: delivered accuracy < 10 tol, and n_phi even
    rng = np.random.default_rng(34 + L)
    n = 150
    th, ph = cap_points(n, rng=rng, area_uniform=False)
    alm = O.rand_alm(L, rng=rng)
    fd = O.Direct(th, ph, L).forward(alm)
    S = O.Stretch(th, ph, L, tol, nufft="direct")
    assert rel(S.forward(alm), fd) < 10 * tol
    assert S.info["nph"] % 2 == 0
    # the fast NUFFT delivers the same accuracy
    assert rel(O.Stretch(th, ph, L, tol, nufft="es").forward(alm), fd) < 10 * tol


def test_stretch_worst_case_spectra(O):
    # test/test_transforms.jl:84-109: a single l = lmax mode and a red spectrum
    rng = np.random.default_rng(35)
    L, tol, n = 256, 1e-8, 200
    th, ph = cap_points(n, rng=rng, area_uniform=False)
    D = O.Direct(th, ph, L)
    S = O.Stretch(th, ph, L, tol, nufft="direct")
    alm = O.zeros_alm(L)
    for m in range(-L, L + 1):
        r, c = O.sph_mode(L, m)
        alm[r, c, 0] = rng.standard_normal() + 1j * rng.standard_normal()
    assert rel(S.forward(alm), D.forward(alm)) < 10 * tol
    almr = O.rand_alm(L, rng=rng, weight=lambda l: 1.0 / (1.0 + l) ** 2)
    assert rel(S.forward(almr), D.forward(almr)) < 10 * tol


@pytest.mark.parametrize("L", [256, 512])
def test_stretch_adjoint_exact_transpose(O, L):
    # test/test_transforms.jl:111-123: dot test < 1e-12
    rng = np.random.default_rng(36)
    n = 120
    th, ph = cap_points(n, rng=rng, area_uniform=False)
    for kind in ("direct", "es"):
        S = O.Stretch(th, ph, L, 1e-8, nufft=kind)
        alm = O.rand_alm(L, rng=rng)
        g = cn(rng, n)
        assert dot_rel(S.forward(alm), g, alm, S.adjoint(g)) < 1e-12


@pytest.mark.parametrize("center,tag", [(0.9, "mid-latitude"), (np.pi - 0.3, "southern")])
def test_stretch_off_pole_and_southern(O, center, tag):
    # test/test_transforms.jl:125-140
    rng = np.random.default_rng(37)
    L, tol, n = 256, 1e-8, 150
    th = center + 0.12 * (2 * rng.random(n) - 1)
    ph = 1.0 + 0.4 * rng.random(n)
    alm = O.rand_alm(L, rng=rng)
    S = O.Stretch(th, ph, L, tol, nufft="direct")
    if tag == "southern":
        assert S.info["flip"] == 1
    assert rel(S.forward(alm), O.Direct(th, ph, L).forward(alm)) < 10 * tol
    g = cn(rng, n)
    assert dot_rel(S.forward(alm), g, alm, S.adjoint(g)) < 1e-12


def test_stretch_interior_band(O):
    # a mid-latitude band at lmax 1024 takes the interior (two-sided window) periodisation
    rng = np.random.default_rng(39)
    L, tol, n = 1024, 1e-8, 60
    th = 0.9 + 0.12 * (2 * rng.random(n) - 1)
    ph = 2 * np.pi * rng.random(n)
    S = O.Stretch(th, ph, L, tol, nufft="es")
    assert S.info["kind"] == "interior"
    alm = O.rand_alm(L, rng=rng)
    assert rel(S.forward(alm, 8), O.Direct(th, ph, L).forward(alm, 8)) < 10 * tol
    g = cn(rng, n)
    assert dot_rel(S.forward(alm, 8), g, alm, S.adjoint(g, 8)) < 1e-12


def test_stretch_ntrans_per_column(O):
    # test/test_transforms.jl:142-156
    rng = np.random.default_rng(38)
    L, B, n = 256, 3, 100
    th, ph = cap_points(n, rng=rng, area_uniform=False)
    p1 = O.Stretch(th, ph, L, 1e-8, nufft="direct")
    pB = O.Stretch(th, ph, L, 1e-8, ntrans=B, nufft="direct")
    almB = O.rand_alm(L, ntrans=B, rng=rng)
    fB = pB.forward(almB)
    for b in range(B):
        assert np.abs(fB[:, b] - p1.forward(almB[:, :, b:b + 1])[:, 0]).max() < 1e-9


@pytest.mark.parametrize("tol", [1e-6, 1e-10])
def test_es_nufft_vs_direct_sum(O, tol):
    # test/test_backends.jl:1-19: fast NUFFT against DirectSum, < 200 tol, both types
    rng = np.random.default_rng(81)
    n1, n2, M = 40, 64, 300
    x = 2 * np.pi * rng.random(M) - 0.5
    y = 2 * np.pi * rng.random(M)
    c = cn(rng, n1, n2)
    for iflag in (1, -1):
        ref = O.nufft_direct(2, n1, n2, iflag, x, y, c)
        es = O.ESNufft(n1, n2, x, y, tol)
        assert rel(es.exec(2, iflag, c), ref) < 200 * tol
        f = cn(rng, M)
        ref1 = O.nufft_direct(1, n1, n2, iflag, x, y, f)
        assert rel(es.exec(1, iflag, f), ref1) < 200 * tol


@pytest.mark.parametrize("grid", [(84, 128), (96, 147), (105, 135)])
def test_es_nufft_longer_fine_grids(O, grid):
    # fine grids above the minimum (2 n) keep the accuracy: the deconvolution follows the length
    rng = np.random.default_rng(83)
    n1, n2, M, tol = 40, 64, 300, 1e-9
    x = 2 * np.pi * rng.random(M)
    y = 2 * np.pi * rng.random(M)
    c = cn(rng, n1, n2)
    es = O.ESNufft(n1, n2, x, y, tol, grid=grid)
    assert (es.params()["nf1"], es.params()["nf2"]) == grid
    assert rel(es.exec(2, 1, c), O.nufft_direct(2, n1, n2, 1, x, y, c)) < 200 * tol
    f = cn(rng, M)
    assert rel(es.exec(1, -1, f), O.nufft_direct(1, n1, n2, -1, x, y, f)) < 200 * tol
    with pytest.raises(ValueError):
        O.ESNufft(n1, n2, x, y, tol, grid=(79, 128))


def test_es_nufft_type1_is_adjoint_of_type2(O):
    rng = np.random.default_rng(82)
    n1, n2, M = 32, 48, 500
    x, y = 2 * np.pi * rng.random(M), 2 * np.pi * rng.random(M)
    es = O.ESNufft(n1, n2, x, y, 1e-9)
    c, f = cn(rng, n1, n2), cn(rng, M)
    lhs = np.vdot(es.exec(2, 1, c)[:, 0], f)
    rhs = np.vdot(c.ravel(order="F"), es.exec(1, -1, f)[:, :, 0].ravel(order="F"))
    assert abs(lhs - rhs) / abs(lhs) < 1e-13


def test_polynomial_kernel_matches_exact_kernel(O):
    # FINUFFT's piecewise-polynomial kernel evaluation changes the result only at the
    # kernel's own truncation level
    rng = np.random.default_rng(83)
    n1, n2, M = 40, 64, 400
    x, y = 2 * np.pi * rng.random(M), 2 * np.pi * rng.random(M)
    c = cn(rng, n1, n2)
    a = O.ESNufft(n1, n2, x, y, 1e-8, kernel="poly").exec(2, 1, c)
    b = O.ESNufft(n1, n2, x, y, 1e-8, kernel="exact").exec(2, 1, c)
    assert rel(a, b) < 1e-8


def test_dfs_double_fold_transpose(O):
    # test/test_backends.jl:187-200
    rng = np.random.default_rng(84)
    F = cn(rng, 10, 12, 2)
    G = cn(rng, 20, 12, 2)
    for s in (0, 1):
        lhs = O.cdot(O.dfs_double(F, s), G)
        rhs = O.cdot(F, O.dfs_fold(G, s))
        assert abs(lhs - rhs) / abs(lhs) < 1e-14


def test_fft_against_numpy(O):
    rng = np.random.default_rng(85)
    for n in (6, 45, 135, 720, 1440, 77):
        a = cn(rng, n, 3)
        assert rel(O.fft_cols(a, -1), np.fft.fft(a, axis=0)) < 1e-13
        assert rel(O.fft_cols(a, +1), np.fft.ifft(a, axis=0) * n) < 1e-13
    a = cn(rng, 5, 96)
    assert rel(O.fft_rows(a, -1), np.fft.fft(a, axis=1)) < 1e-13


def test_threaded_apply_matches_serial(O):
    # test/test_backends.jl:45-62: threaded equals serial (same arithmetic)
    rng = np.random.default_rng(86)
    L, n = 256, 300
    th, ph = cap_points(n, rng=rng)
    S = O.Stretch(th, ph, L, 1e-8, nufft="es")
    alm = O.rand_alm(L, rng=rng)
    assert np.abs(S.forward(alm, 1) - S.forward(alm, 4)).max() <= 1e-12 * np.abs(S.forward(alm, 1)).max()
