"""Pure-Python restatement of PartialFSHT.jl's planner: minimal boxes, the counted cost model,
the partition into boxes and the leaf choice (src/Box.jl, src/Cost.jl).

TEST INFRASTRUCTURE ONLY: the checker of the library's host planner. The ring counts and grid
sizes come from the oracle's own restatement of the geometry (oracle.py), not from the library.
"""
from __future__ import annotations

import math

import numpy as np

from . import oracle as O

TWO_PI = 2 * math.pi
POLAR_TOL = math.sqrt(np.finfo(np.float64).eps)  # sqrt(eps(Float64)), src/Box.jl:62
K_MARGIN = 2                                      # _K_MARGIN, src/Stretch.jl:86
DEFAULT_COST = {"ring": 1.0, "fft": 0.394, "spread": 0.334, "ft_conn": 5.18}  # src/Cost.jl:58


def jl_mod(x, y):
    """Julia's floating mod (result has the sign of y)."""
    x = np.asarray(x, dtype=np.float64)
    r = np.fmod(x, y)
    return np.where((r != 0) & ((r < 0) != (y < 0)), r + y, r)


def max_gap(v):
    """_max_gap (src/Box.jl:223-258): (lo, hi, gap, at) by n - 1 equal buckets."""
    v = np.asarray(v, dtype=np.float64)
    n = len(v)
    lo = float(v.min())
    hi = float(v.max())
    if n < 2 or hi <= lo:
        return lo, hi, 0.0, lo
    nb = n - 1
    w = (hi - lo) / nb
    k = np.clip(np.floor((v - lo) / w).astype(np.int64), 0, nb - 1)
    bmin = np.full(nb, np.inf)
    bmax = np.full(nb, -np.inf)
    np.minimum.at(bmin, k, v)
    np.maximum.at(bmax, k, v)
    gap, at, prev = 0.0, hi, lo
    for j in np.flatnonzero(np.isfinite(bmin)):
        d = bmin[j] - prev
        if d > gap:
            gap, at = float(d), float(bmin[j])
        prev = bmax[j]
    return lo, hi, gap, at


def _arc(lo, hi, gap, at):
    """Longitude arc from a gap scan, the wrap-around gap included (src/Box.jl:82-96)."""
    wrap = TWO_PI - hi + lo
    start = at
    if wrap >= gap:
        gap, start = wrap, lo
    ext = TWO_PI - gap
    if ext <= 0:
        return lo, 0.0
    if ext >= TWO_PI:
        return 0.0, TWO_PI
    return start, ext


def bounding_box(theta, phi):
    """bounding_box (src/Box.jl:42-73)."""
    theta = np.asarray(theta, dtype=np.float64)
    lo = max(float(theta.min()), 0.0)
    hi = min(float(theta.max()), math.pi)
    tn, ts = lo <= POLAR_TOL, hi >= math.pi - POLAR_TOL
    if tn or ts:
        return dict(theta_lo=lo, theta_hi=hi, phi_start=0.0, phi_extent=TWO_PI,
                    touches_north=tn, touches_south=ts)
    ps = jl_mod(phi, TWO_PI)
    if len(ps) == 1:
        return dict(theta_lo=lo, theta_hi=hi, phi_start=float(ps[0]), phi_extent=0.0,
                    touches_north=False, touches_south=False)
    st, ext = _arc(*max_gap(ps))
    return dict(theta_lo=lo, theta_hi=hi, phi_start=st, phi_extent=ext,
                touches_north=False, touches_south=False)


def group_box(tv, pv, g):
    """_group_box (src/Box.jl:261-287)."""
    lo, hi, _, _ = max_gap(tv[g])
    tn, ts = lo <= POLAR_TOL, hi >= math.pi - POLAR_TOL
    if tn or ts:
        return dict(theta_lo=lo, theta_hi=hi, phi_start=0.0, phi_extent=TWO_PI,
                    touches_north=tn, touches_south=ts)
    st, ext = _arc(*max_gap(pv[g]))
    return dict(theta_lo=lo, theta_hi=hi, phi_start=st, phi_extent=ext,
                touches_north=False, touches_south=False)


def _fftunits(n):
    return 0.0 if n <= 1 else float(n) * math.log2(float(n))


def cost_direct(npts, lmax, ntrans, c=DEFAULT_COST):
    """cost_direct (src/Cost.jl:107-108)."""
    return c["ring"] * float(npts) * (lmax + 1) ** 2 * ntrans / 2


def cost_stretch(box, npts, lmax, ntrans, tol, c=DEFAULT_COST):
    """cost_stretch (src/Cost.jl:117-142): the leaf's own sizing, counted."""
    geom = O.try_stretch_geometry(box["theta_lo"], box["theta_hi"], lmax, tol)
    if geom is None:
        return math.inf
    K = int(geom.K) + K_MARGIN
    if geom.kind == "interior":
        nth = O.next_smooth(2 * K + 1)
        nth_half = nth
    else:
        nth_half = O.next_smooth(K + 1)
        nth = 2 * nth_half
    tr, _ = geom.rings(nth_half)
    if not np.all(np.diff(tr) >= 0):
        tr = tr[::-1]
    rings, mmax = O.counted_ring_work(tr, lmax, tol)
    nph = O.next_smooth_even(2 * mmax + 1)
    fft = _fftunits(nph) * len(tr) + _fftunits(nth * nph)
    taps = 2 * math.ceil(abs(math.log10(max(float(tol), 1e-16)))) + 2
    spread = float(npts) * taps * taps
    return ntrans * (c["ring"] * rings + c["fft"] * fft + c["spread"] * spread)


def _split_below(v, g, thresh):
    a = g[v[g] < thresh]
    if len(a) == 0 or len(a) == len(g):
        return None
    return a, g[v[g] >= thresh]


def best_gap_split(tv, pv, g):
    """_best_gap_split (src/Box.jl:289-307)."""
    tlo, thi, gt, at_t = max_gap(tv[g])
    _, _, gp, at_p = max_gap(pv[g])
    mid = (tlo + thi) / 2
    wphi = gp * math.sin(min(max(mid, POLAR_TOL), math.pi - POLAR_TOL))
    if gt >= wphi:
        return _split_below(tv, g, at_t) if gt > 0 else None
    return _split_below(pv, g, at_p) if gp > 0 else None


def partition_boxes_costed(theta, phi, lmax, ntrans, tol, maxboxes=8, c=DEFAULT_COST):
    """partition_boxes_costed with cost_stretch (src/Box.jl:156-200)."""
    tv = np.asarray(theta, dtype=np.float64)
    pv = jl_mod(phi, TWO_PI)
    cost = lambda b, n: cost_stretch(b, n, lmax, ntrans, tol, c)  # noqa: E731
    groups = [np.arange(len(tv))]
    boxes = [group_box(tv, pv, groups[0])]
    costs = [cost(boxes[0], len(tv))]
    while len(groups) < maxboxes:
        best_gain, best = 0.0, None
        for gi, g in enumerate(groups):
            if len(g) < 2:
                continue
            sp = best_gap_split(tv, pv, g)
            if sp is None:
                continue
            ga, gb = sp
            ba, bb = group_box(tv, pv, ga), group_box(tv, pv, gb)
            gain = costs[gi] - (cost(ba, len(ga)) + cost(bb, len(gb)))
            if gain > best_gain:
                best_gain, best = gain, (gi, ga, gb, ba, bb)
        if best is None:
            break
        gi, ga, gb, ba, bb = best
        del groups[gi], boxes[gi], costs[gi]
        for g, b in ((ga, ba), (gb, bb)):
            groups.append(g)
            boxes.append(b)
            costs.append(cost(b, len(g)))
    return groups, boxes, costs


def select_method(theta, phi, lmax, tol, ntrans=1, c=DEFAULT_COST):
    """select_method for AutoAlgorithm (src/Cost.jl:171-201), no NUFSHT extension."""
    n = len(theta)
    box = bounding_box(theta, phi)
    best, bestc = "direct", cost_direct(n, lmax, ntrans, c)
    cs = cost_stretch(box, n, lmax, ntrans, tol, c)
    if cs < bestc:
        best, bestc = "stretch", cs
    groups, _, gcosts = partition_boxes_costed(theta, phi, lmax, ntrans, tol, 8, c)
    if len(groups) > 1 and sum(gcosts) < bestc:
        best = "multibox"
    return best
