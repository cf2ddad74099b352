"""Generate the golden fixtures of tests/golden/ with mpmath (high precision).

PartialFSHT.jl keeps no golden vectors: its tests pin the associated-Legendre evaluation
against BigFloat at fixed known-answer cases and pin the Direct leaf against an explicit
sum of a_lm Y_lm. This script evaluates the same cases with mpmath at 80 significant
digits (the role of Julia's BigFloat) and writes them as JSON:

  alf_kat.json     normalised P_l^m(cos theta) (Condon-Shortley) at the cases of
                   test/test_legendre.jl:71-90 and examples/02_accuracy_and_tolerance.jl:62,
                   plus the outer-ring turning-point cases of test/test_legendre.jl:71-81
  direct_small.json  f_i = sum a_lm Y_lm(theta_i, phi_i) and the adjoint sum
                   conj(Y_lm) f_i for a small seeded case (test/test_transforms.jl:9-31)
  wigner_d_kat.json  d^l_{mn}(beta) at the high-degree cases of test/test_spin.jl:23-33
                   (python tests/golden/make_golden.py wigner)

Run from the repository root:  python tests/golden/make_golden.py
"""
import json
import os
import sys

import mpmath as mp
import numpy as np

mp.mp.dps = 80
HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def alf_mp(l, m, theta):
    """Normalised associated Legendre function with the Condon-Shortley phase,
    P_l^m = (-1)^m c_m sin^m, P_{m+1}^m = sqrt(2m+3) cos P_m^m, then the three-term
    recurrence, all at mpmath precision (no exponent range limit)."""
    am = abs(m)
    if am > l:
        return mp.mpf(0)
    t = mp.mpf(theta)
    s, x = mp.sin(t), mp.cos(t)
    c = 1 / mp.sqrt(4 * mp.pi)
    for k in range(1, am + 1):
        c *= mp.sqrt(mp.mpf(2 * k + 1) / (2 * k))
    p2 = (-1) ** am * c * s ** am
    flip = -1 if (m < 0 and am % 2 == 1) else 1
    if l == am:
        return flip * p2
    p1 = mp.sqrt(2 * am + 3) * x * p2
    for el in range(am + 2, l + 1):
        a = mp.sqrt(mp.mpf((2 * el - 1) * (2 * el + 1)) / ((el - am) * (el + am)))
        b = mp.sqrt(mp.mpf(2 * el + 1) / (2 * el - 3) * mp.mpf((el - am - 1) * (el + am - 1))
                    / ((el - am) * (el + am)))
        p1, p2 = a * x * p1 - b * p2, p1
    return flip * p1


def check_against_legenp():
    """Independent cross-check of alf_mp with mpmath's hypergeometric legenp."""
    worst = 0
    for (l, m, th) in ((5, 2, 0.7), (12, 7, 1.1), (30, 0, 0.3), (40, 13, 2.2)):
        x = mp.cos(mp.mpf(th))
        norm = mp.sqrt((2 * l + 1) / (4 * mp.pi) * mp.factorial(l - m) / mp.factorial(l + m))
        ref = norm * mp.legenp(l, m, x, type=2)
        got = alf_mp(l, m, th)
        worst = max(worst, abs(got - ref) / abs(ref))
    assert worst < mp.mpf(10) ** -60, worst
    return float(worst)


def main():
    sys.path.insert(0, ROOT)
    from oracle import oracle as O  # only to obtain the geometry-driven (theta, m) cases

    cases = []
    # test/test_legendre.jl:83-90 (L, m, theta) and the turning-point cases of
    # examples/02_accuracy_and_tolerance.jl:62
    for (l, m, th) in ((4096, 1000, 0.4), (4096, 3000, 1.2), (8192, 4000, 0.9), (2048, 0, 1.5),
                       (513, 513, 1.0), (100, 7, 3.0), (2048, 700, 0.35), (4096, 1400, 0.35),
                       (8192, 1600, 0.20)):
        cases.append({"l": l, "m": m, "theta": th, "source": "known answer"})
    # test/test_legendre.jl:71-81: the outer ring of a 20-degree cap at the polar-limit order
    for L in (256, 1024, 2048, 4096, 8192):
        g = O.stretch_geometry(0.0, 20 * np.pi / 180, L, 1e-8)
        thmax = g.h * (1 + g.eps_apo)
        m = O.polar_mmax(thmax, L, 1e-8)
        cases.append({"l": L, "m": m, "theta": thmax, "source": "outer ring of a 20deg cap"})
    for c in cases:
        v = alf_mp(c["l"], c["m"], c["theta"])
        c["value"] = mp.nstr(v, 30)
        c["log10_abs"] = float(mp.log10(abs(v))) if v != 0 else None
    out = {"generator": "tests/golden/make_golden.py (mpmath, 80 digits)",
           "legenp_crosscheck_rel": check_against_legenp(), "cases": cases}
    json.dump(out, open(os.path.join(HERE, "alf_kat.json"), "w"), indent=1)

    # small Direct case: explicit sums at high precision
    rng = np.random.default_rng(31)
    L, n = 12, 25
    theta = (0.4 * rng.random(n)).tolist()
    phi = (2 * np.pi * rng.random(n)).tolist()
    modes = [(l, m) for l in range(L + 1) for m in range(-l, l + 1)]
    are = rng.standard_normal(len(modes)).tolist()
    aim = rng.standard_normal(len(modes)).tolist()
    fre = rng.standard_normal(n).tolist()
    fim = rng.standard_normal(n).tolist()
    Y = {}
    for i in range(n):
        for (l, m) in modes:
            Y[(i, l, m)] = alf_mp(l, m, theta[i]) * mp.expj(m * mp.mpf(phi[i]))
    f = []
    for i in range(n):
        acc = mp.mpc(0)
        for k, (l, m) in enumerate(modes):
            acc += mp.mpc(are[k], aim[k]) * Y[(i, l, m)]
        f.append([float(acc.real), float(acc.imag)])
    adj = []
    for (l, m) in modes:
        acc = mp.mpc(0)
        for i in range(n):
            acc += mp.conj(Y[(i, l, m)]) * mp.mpc(fre[i], fim[i])
        adj.append([float(acc.real), float(acc.imag)])
    out = {"generator": "tests/golden/make_golden.py (mpmath, 80 digits)",
           "source": "test/test_transforms.jl:9-31 (Direct against the explicit sum)",
           "lmax": L, "theta": theta, "phi": phi, "modes": modes, "alm_re": are,
           "alm_im": aim, "f": f, "g_re": fre, "g_im": fim, "adjoint": adj}
    json.dump(out, open(os.path.join(HERE, "direct_small.json"), "w"))
    print("wrote", os.path.join(HERE, "alf_kat.json"), os.path.join(HERE, "direct_small.json"))


def wigner_d_mp(l, m, n, beta):
    """d^l_{mn}(beta) at mpmath precision: the extremal closed form at l0 = max(|m|, |n|)
    (src/Spin.jl:10-16, with d^j_{a,b} = (-1)^{a-b} d^j_{b,a} to move the extremal index
    second) and the degree recurrence of src/Spin.jl:6-8, no scaling needed."""
    if abs(m) > l or abs(n) > l:
        return mp.mpf(0)
    b = mp.mpf(beta)
    c, s = mp.cos(b / 2), mp.sin(b / 2)
    l0 = max(abs(m), abs(n))

    def extremal(j, a, bb):
        lb = mp.sqrt(mp.binomial(2 * j, j - a))
        if bb == j:
            return lb * c ** (j + a) * s ** (j - a)
        return (-1) ** (j - a) * lb * c ** (j - a) * s ** (j + a)

    if abs(n) == l0:
        d1 = extremal(l0, m, l0 if n == l0 else -l0)
    else:
        d1 = extremal(l0, n, l0 if m == l0 else -l0) * (-1) ** ((n - m) % 2)
    d0 = mp.mpf(0)
    Lc = l0
    cb = mp.cos(b)
    if l0 == 0:
        d0, d1, Lc = d1, d1 * cb, 1
    while Lc < l:
        L1 = Lc + 1
        den = Lc * mp.sqrt(L1 * L1 - m * m) * mp.sqrt(L1 * L1 - n * n)
        c1 = (2 * Lc + 1) * (Lc * L1 * cb - m * n) / den
        c0 = L1 * mp.sqrt(max(0, Lc * Lc - m * m)) * mp.sqrt(max(0, Lc * Lc - n * n)) / den
        d0, d1 = d1, c1 * d1 - c0 * d0
        Lc = L1
    return d1 if l > l0 or l0 == 0 else d1


def wigner_kat():
    """The high-degree Wigner-d cases of test/test_spin.jl:23-33."""
    cases = [(512, 100, -2, 0.8), (2048, 700, -1, 0.5), (4096, 30, -2, 1.1), (1024, 0, 0, 2.0),
             (300, 250, 3, 0.05), (64, -20, 5, 2.9)]
    out = []
    for l, m, n, b in cases:
        out.append({"l": l, "m": m, "n": n, "beta": b, "d": mp.nstr(wigner_d_mp(l, m, n, b), 40)})
    json.dump(out, open(os.path.join(HERE, "wigner_d_kat.json"), "w"), indent=1)


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "wigner":
        wigner_kat()
        sys.exit(0)
    main()
