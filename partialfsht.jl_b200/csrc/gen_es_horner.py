"""Generate es_horner_table.h: per-tap polynomial approximations of the ES NUFFT kernel.

The kernel is phi(z) = exp(beta (sqrt(1 - z^2) - 1)), |z| < 1, with width w cells and
beta = 2.30 w (the published FINUFFT choice at upsampling 2). A point at grid coordinate g
touches cells i0 + a, a = 0..w-1, i0 = ceil(g - w/2); with s = i0 - g + w/2 in [0, 1) tap a
is phi((s + a - w/2) / (w/2)). Each tap is replaced by its Chebyshev interpolant of degree
w + 2 on s in [0, 1), written as a polynomial in v = s - 1/2 and evaluated by Horner's rule
(the approach FINUFFT takes for its default kernel evaluation). The interpolant is computed
at 60 significant digits with mpmath and rounded to double.

Run: python gen_es_horner.py > es_horner_table.h
"""
import mpmath as mp

mp.mp.dps = 60
WMIN, WMAX = 2, 16


def degree(w):
    return w + 2


def es(z, beta):
    if abs(z) >= 1:
        return mp.mpf(0)
    return mp.e ** (beta * (mp.sqrt(1 - z * z) - 1))


def tap_coeffs(w, a, beta, d):
    n = d + 1
    # Chebyshev nodes in t = 2 s - 1 (first kind)
    ts = [mp.cos(mp.pi * (i + mp.mpf(1) / 2) / n) for i in range(n)]
    ys = [es(((t + 1) / 2 + a - mp.mpf(w) / 2) / (mp.mpf(w) / 2), beta) for t in ts]
    cheb = []
    for k in range(n):
        s = mp.fsum(ys[i] * mp.cos(k * mp.pi * (i + mp.mpf(1) / 2) / n) for i in range(n))
        cheb.append(s * 2 / n if k else s / n)
    # Chebyshev series in t -> power series in t (T_{k+1} = 2 t T_k - T_{k-1})
    T = [[mp.mpf(1)], [mp.mpf(0), mp.mpf(1)]]
    for k in range(2, n):
        nxt = [mp.mpf(0)] * (k + 1)
        for i, c in enumerate(T[k - 1]):
            nxt[i + 1] += 2 * c
        for i, c in enumerate(T[k - 2]):
            nxt[i] -= c
        T.append(nxt)
    poly = [mp.mpf(0)] * n
    for k in range(n):
        for i, c in enumerate(T[k]):
            poly[i] += cheb[k] * c
    # t = 2 v
    return [poly[i] * mp.mpf(2) ** i for i in range(n)]


def main():
    out = []
    out.append("// Generated by gen_es_horner.py; do not edit. Per-tap Horner coefficients of the")
    out.append("// ES NUFFT kernel exp(beta (sqrt(1 - z^2) - 1)), beta = 2.30 w, degree w + 2, in")
    out.append("// v = s - 1/2 where s = i0 - g + w/2 in [0, 1) is the point's offset to its first cell.")
    out.append("// The float copies (rounded to 9 digits) serve the single-precision NUFFT.")
    out.append("#pragma once")
    out.append("")
    out.append("namespace pf {")
    out.append("")
    out.append("template <int W> struct EsHorner;")
    for w in range(WMIN, WMAX + 1):
        d = degree(w)
        beta = mp.mpf("2.30") * w
        rows = [tap_coeffs(w, a, beta, d) for a in range(w)]
        vals = ", ".join(mp.nstr(c, 17, min_fixed=-1, max_fixed=-1) if abs(c) > mp.mpf(10) ** -40
                         else "0.0" for r in rows for c in r)
        fvals = ", ".join((mp.nstr(c, 9, min_fixed=-1, max_fixed=-1) + "f") if abs(c) > mp.mpf(10) ** -30
                          else "0.0f" for r in rows for c in r)
        out.append(f"__constant__ double kEsHorner{w}[{w * (d + 1)}] = {{{vals}}};")
        out.append(f"__constant__ float kEsHornerF{w}[{w * (d + 1)}] = {{{fvals}}};")
        out.append(f"template <> struct EsHorner<{w}> {{")
        out.append(f"    static constexpr int NC = {d + 1};")
        out.append(f"    __device__ static const double* coef() {{ return kEsHorner{w}; }}")
        out.append(f"    __device__ static const float* coef_f() {{ return kEsHornerF{w}; }}")
        out.append("};")
    out.append("")
    out.append("}  // namespace pf")
    print("\n".join(out))


if __name__ == "__main__":
    main()
