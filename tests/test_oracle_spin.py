"""The oracle's spin-weighted transforms (src/Spin.jl) pinned to the reference's spin testset
(test/test_spin.jl) and to 80-digit Wigner-d values (tests/golden/wigner_d_kat.json)."""
import json
import os

import numpy as np
import pytest

from helpers import cn, dot_rel, rel

HERE = os.path.dirname(os.path.abspath(__file__))


def test_wigner_d_closed_forms_endpoints_symmetry(O):
    b = 0.37
    cases = [((1, 0, 0), np.cos(b)), ((1, 1, 0), -np.sin(b) / np.sqrt(2)),
             ((1, 0, 1), np.sin(b) / np.sqrt(2)), ((1, 1, 1), (1 + np.cos(b)) / 2),
             ((1, 1, -1), (1 - np.cos(b)) / 2), ((1, -1, 0), np.sin(b) / np.sqrt(2)),
             ((1, 0, -1), -np.sin(b) / np.sqrt(2)), ((2, 0, 0), (3 * np.cos(b) ** 2 - 1) / 2),
             ((3, 0, 0), (5 * np.cos(b) ** 3 - 3 * np.cos(b)) / 2)]
    for (l, m, n), ref in cases:
        assert O.wigner_d(l, m, n, b) == pytest.approx(ref, rel=1e-13, abs=1e-15)
    assert O.wigner_d(5, 2, 2, 0.0) == 1.0
    assert O.wigner_d(5, 2, 3, 0.0) == 0.0
    assert abs(O.wigner_d(4, 2, -2, np.pi)) == 1.0
    for l, m, n in ((7, 3, -2), (40, 11, 5), (200, 60, -7)):
        assert O.wigner_d(l, m, n, 0.9) == pytest.approx((-1) ** (m - n) * O.wigner_d(l, n, m, 0.9),
                                                         abs=1e-12)


def test_wigner_d_high_degree_against_80_digits(O):
    for case in json.load(open(os.path.join(HERE, "golden", "wigner_d_kat.json"))):
        g = O.wigner_d(case["l"], case["m"], case["n"], case["beta"])
        r = float(case["d"])
        assert abs(g) <= 1 + 1e-10
        if abs(r) > 1e-300:
            assert abs(g - r) / abs(r) < 1e-10, case


@pytest.mark.parametrize("L", [128, 256, 512])
def test_spin_engine_against_wigner_d(O, L):
    # test/test_spin.jl:53-82: errors against the ring maximum; dropped entries negligible
    th = np.linspace(0.01, 0.6, 200)
    eng = O.SpinRings(th, L, 2, 0.0)
    for m in (L // 4, L // 2, 3 * L // 4, L - 1):
        alm = np.zeros((L + 1, 2 * L + 1), np.complex128, order="F")
        alm[O.spin_coeff_index(L, m, L)] = 1
        G = eng.rings_from_alm(alm)[:, m + L, 0].real
        refs = np.array([np.sqrt((2 * L + 1) / (4 * np.pi)) * O.wigner_d(L, m, -2, t) for t in th])
        peak = np.abs(refs).max()
        assert peak > 0
        dropped = (G == 0) & (refs != 0)
        assert np.max(np.abs(G - refs)[~dropped] / peak) < 1e-12
        assert (np.abs(refs[dropped]) / peak).max(initial=0.0) < 1e-30


def test_spin_chunks_poles_and_reflection(O):
    thw = np.linspace(0.01, 1.4, 300)
    for L in (256, 1024):
        assert O.SpinRings(thw, L, 2, 0.0).nchunks > 1
    L, s = 6, 2
    th = np.array([0.0, 0.3, np.pi / 2, np.pi - 0.3, np.pi])
    eng = O.SpinRings(th, L, s, 0.0)
    for m in (-3, 0, 2, 5):
        alm = np.zeros((L + 1, 2 * L + 1), np.complex128, order="F")
        alm[O.spin_coeff_index(5, m, L)] = 1
        G = eng.rings_from_alm(alm)[:, m + L, 0].real
        for j, t in enumerate(th):
            ref = np.sqrt(11 / (4 * np.pi)) * O.wigner_d(5, m, -s, t)
            assert G[j] == pytest.approx(ref, abs=1e-13)
    L, s = 8, 1
    tha = np.linspace(0.2, 1.1, 9)
    eng = O.SpinRings(tha, L, s, 0.0, reflect=True)
    for l, m in ((3, 2), (7, -5), (8, 0)):
        alm = np.zeros((L + 1, 2 * L + 1), np.complex128, order="F")
        alm[O.spin_coeff_index(l, m, L)] = 1
        G = eng.rings_from_alm(alm)[:, m + L, 0].real
        for j, t in enumerate(tha):
            ref = np.sqrt((2 * l + 1) / (4 * np.pi)) * O.wigner_d(l, m, -s, np.pi - t)
            assert G[j] == pytest.approx(ref, abs=1e-12)


def test_spin_engine_adjoint_is_transpose(O):
    rng = np.random.default_rng(40)
    L, s = 40, -2
    th = np.sort(0.05 + 0.5 * rng.random(30))
    eng = O.SpinRings(th, L, s, 1e-10)
    alm = O.rand_spin_alm(L, s, rng=rng)
    G = eng.rings_from_alm(alm)
    Gr = np.asfortranarray(cn(rng, len(th), 2 * L + 1, 1))
    lhs = np.vdot(G.ravel(order="F"), Gr.ravel(order="F"))
    rhs = np.vdot(alm.ravel(order="F"), eng.alm_from_rings(Gr).ravel(order="F"))
    assert abs(lhs - rhs) / abs(lhs) < 1e-13


def test_spin_harmonics_direct_and_stretch(O):
    # test/test_spin.jl:134-175
    for l, m in ((0, 0), (3, 2), (12, -5)):
        assert O.sylm(0, l, m, 0.8, 2.1) == pytest.approx(O.ylm(l, m, 0.8, 2.1), abs=1e-13)
    rng = np.random.default_rng(41)
    L, s, n = 8, 1, 25
    th = 0.4 * rng.random(n) + 0.2
    ph = 2 * np.pi * rng.random(n)
    D = O.SpinDirect(th, ph, L, s)
    alm = np.zeros((L + 1, 2 * L + 1), np.complex128, order="F")
    alm[O.spin_coeff_index(4, 2, L)] = 1
    ref = np.array([O.sylm(s, 4, 2, t, p) for t, p in zip(th, ph)])
    assert np.abs(D.forward(alm)[:, 0] - ref).max() < 1e-12
    a = np.asfortranarray(cn(rng, L + 1, 2 * L + 1))
    g = cn(rng, n)
    assert dot_rel(D.forward(a)[:, 0], g, a, D.adjoint(g)[:, :, 0]) < 1e-12
    L, tol = 256, 1e-8
    for s in (1, 2, -1):
        rng = np.random.default_rng(42 + s)
        th = np.deg2rad(20) * np.sqrt(rng.random(120))
        ph = 2 * np.pi * rng.random(120)
        a = np.asfortranarray(cn(rng, L + 1, 2 * L + 1))
        fd = O.SpinDirect(th, ph, L, s).forward(a)[:, 0]
        S = O.Stretch(th, ph, L, tol, nufft="direct", spin=s)
        fs = S.forward(a)[:, 0]
        assert np.abs(fs - fd).max() / np.abs(fd).max() < 10 * tol
        g = cn(rng, 120)
        assert dot_rel(fs, g, a, S.adjoint(g)[:, :, 0]) < 1e-12
