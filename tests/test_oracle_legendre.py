"""The oracle's associated-Legendre engine against the reference's known answers and
properties (test/test_legendre.jl), pinned to mpmath fixtures in tests/golden/."""
import json
import os

import numpy as np
import pytest

from helpers import cn

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_alf_against_high_precision_known_answers(O):
    # test/test_legendre.jl:66-91: Float64 alf vs BigFloat, gate 1e-11
    d = json.load(open(os.path.join(GOLDEN, "alf_kat.json")))
    worst = 0.0
    for c in d["cases"]:
        ref = float(c["value"])
        if abs(ref) < 2.2250738585072014e-308:
            continue
        got = O.alf(c["l"], c["m"], c["theta"])
        assert got != 0.0, c  # the block scaling must not flush a representable value
        worst = max(worst, abs(got - ref) / abs(ref))
    assert worst < 1e-11, worst


def test_outer_ring_case_is_not_negligible(O):
    # the outer-ring turning-point cases are the ones an unscaled recurrence returns 0 for
    d = json.load(open(os.path.join(GOLDEN, "alf_kat.json")))
    cap = [c for c in d["cases"] if c["source"].startswith("outer ring")]
    assert len(cap) == 5
    for c in cap:
        assert O.alf(c["l"], c["m"], c["theta"]) != 0.0
        assert c["log10_abs"] > -300


def test_closed_form_ylm(O):
    # test/test_legendre.jl:93-106
    th, ph = 0.7, 1.1
    i4pi = 1 / np.sqrt(4 * np.pi)
    assert O.ylm(0, 0, 0.3, 1.2) == pytest.approx(i4pi, rel=1e-14)
    assert O.ylm(1, 0, th, ph) == pytest.approx(np.sqrt(3 / (4 * np.pi)) * np.cos(th), rel=1e-14)
    assert O.ylm(1, 1, th, ph) == pytest.approx(
        -np.sqrt(3 / (8 * np.pi)) * np.sin(th) * np.exp(1j * ph), rel=1e-14)
    assert O.ylm(1, -1, th, ph) == pytest.approx(
        np.sqrt(3 / (8 * np.pi)) * np.sin(th) * np.exp(-1j * ph), rel=1e-14)
    assert O.ylm(2, 2, th, ph) == pytest.approx(
        np.sqrt(15 / (32 * np.pi)) * np.sin(th) ** 2 * np.exp(2j * ph), rel=1e-14)
    for (l, m) in ((3, 2), (7, 5), (40, 13)):
        assert O.alf(l, -m, th) == pytest.approx((-1) ** m * O.alf(l, m, th), rel=1e-14)


def test_polar_truncation_bounds_dropped_content(O):
    # test/test_legendre.jl:52-67
    for (L, th, eps) in ((512, 0.4, 1e-8), (1024, 0.6, 1e-8), (2048, 0.35, 1e-6)):
        mm = O.polar_mmax(th, L, eps)
        if mm >= L:
            continue
        peak = max(abs(O.alf(L, m, th)) for m in range(mm + 1))
        dropped = max(abs(O.alf(L, m, th)) for m in range(mm + 1, min(L, mm + 40) + 1))
        assert dropped <= eps * peak
    ms = [O.polar_mmax(t, 512, 1e-8) for t in np.linspace(1e-4, np.pi / 2, 40)]
    assert ms == sorted(ms)


def test_ring_engine_dot_test(O):
    # test/test_legendre.jl:69-85: <R a, g> = <a, R^T g> to round-off
    rng = np.random.default_rng(11)
    for L in (16, 64):
        th = np.sort(0.05 + 0.9 * rng.random(37))
        eng = O.Rings(th, L, 1e-12)
        alm = np.asfortranarray(cn(rng, L + 1, 2 * L + 1, 1))
        G = eng.rings_from_alm(alm)
        Gr = np.asfortranarray(cn(rng, len(th), 2 * L + 1, 1))
        ar = eng.alm_from_rings(Gr)
        lhs = O.cdot(G, Gr)
        rhs = O.cdot(alm, ar)
        assert abs(lhs - rhs) <= 1e-11 * abs(lhs)


def test_ring_engine_matches_per_point_alf(O):
    # test/test_legendre.jl:87-98
    L = 48
    th = np.sort([0.02, 0.11, 0.37, 0.8, 1.4, 2.7])
    eng = O.Rings(th, L, 1e-13)
    alm = O.zeros_alm(L)
    r, c = O.sph_mode(30, 7)
    alm[r, c, 0] = 1.0
    G = eng.rings_from_alm(alm)
    for j, t in enumerate(th):
        assert abs(G[j, 7 + L, 0] - O.alf(30, 7, t)) <= 1e-13


def test_ring_work_counted_and_reduced(O):
    # test/test_legendre.jl:100-107
    L = 512
    th = np.linspace(1e-3, 0.5, 120)
    w_opt, _ = O.counted_ring_work(th, L, 1e-8)
    w_all = len(th) * sum(L - m + 1 for m in range(L + 1))
    assert 0 < w_opt < w_all
    assert O.Rings(th, L, 1e-8).work() == w_opt


def test_nested_ranges_equal_brute_force(O):
    # test/test_legendre.jl:109-128, including ring sets that straddle the equator
    for (lo, hi, L) in ((1e-3, 0.4, 256), (1.2, 2.0, 256), (0.5, 2.6, 512)):
        th = np.linspace(lo, hi, 77)
        mlim = [O.polar_mmax(t, L, 1e-8) for t in th]
        jlo, jhi = O.nested_ranges(mlim, L)
        for m in range(L + 1):
            keep = [j for j, v in enumerate(mlim) if v >= m]
            if not keep:
                assert jhi[m] < jlo[m]
            else:
                assert (jlo[m], jhi[m]) == (keep[0], keep[-1])
                assert keep == list(range(keep[0], keep[-1] + 1))


def test_nested_ranges_reject_non_unimodal(O):
    with pytest.raises(ValueError):
        O.nested_ranges([3, 5, 2, 6], 8)


def test_threaded_ring_walk_equals_serial(O):
    # ext/PartialFSHTOhMyThreadsExt.jl:31-42 threads over interleaved orders; the result is
    # the serial one bit for bit (test/test_backends.jl:45-62)
    rng = np.random.default_rng(5)
    L = 128
    th = np.sort(0.02 + 0.4 * rng.random(50))
    eng = O.Rings(th, L, 1e-8)
    alm = np.asfortranarray(cn(rng, L + 1, 2 * L + 1, 1))
    assert np.array_equal(eng.rings_from_alm(alm, 1), eng.rings_from_alm(alm, 4))
    G = np.asfortranarray(cn(rng, len(th), 2 * L + 1, 1))
    assert np.array_equal(eng.alm_from_rings(G, 1), eng.alm_from_rings(G, 4))
