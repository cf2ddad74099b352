"""Restatement of PartialFSHT.jl's solve! (src/Analysis.jl:375-436) in numpy over the oracle's
own transforms.

TEST INFRASTRUCTURE ONLY: the checker of the library's device solver.
"""
from __future__ import annotations

import numpy as np


def solve(fwd, adj, f, lmax, *, mode="cg", rtol=1e-6, maxiter=500, prior=None, w=None):
    """CG on the normal equations with the reference's update order and stopping rule.
    fwd(alm) -> field and adj(field) -> coefficients are the plan's transforms (complex128
    arrays in the reference layouts). Returns (alm, iters, relres)."""
    fw = np.array(f, dtype=np.complex128, copy=True)
    if w is not None:
        fw = fw * (w if fw.ndim == 1 else w[:, None])
    rhs = adj(fw)
    reg = None
    if mode == "wiener":
        reg = np.array([1.0 / c if c > 0 else 0.0 for c in prior[: lmax + 1]])
    tol = min(rtol, 1e-12) if mode == "minnorm" else rtol
    alm = np.zeros_like(rhs)
    r = rhs.copy()
    p = r.copy()
    rsold = np.vdot(r, r)
    rhsn = np.sqrt(abs(np.vdot(rhs, rhs)))
    if rhsn == 0:
        return alm, 0, 0.0
    # l of every sph_mode slot (row + |m| of the column), for the prior
    nr, nc = lmax + 1, 2 * lmax + 1
    ell = np.arange(nr)[:, None] + (np.arange(nc)[None, :] + 1) // 2
    iters, rel = 0, 1.0
    for i in range(1, maxiter + 1):
        iters = i
        fb = fwd(p)
        if w is not None:
            fb = fb * (w if fb.ndim == 1 else w[:, None])
        Ap = adj(fb)
        if reg is not None:
            s = np.where(ell <= lmax, reg[np.minimum(ell, lmax)], 0.0)
            Ap = Ap + (s if Ap.ndim == 2 else s[:, :, None]) * p
        pAp = np.vdot(p, Ap)
        alpha = 0.0 if pAp == 0 else rsold / pAp
        alm = alm + alpha * p
        r = r - alpha * Ap
        rsnew = np.vdot(r, r)
        rel = np.sqrt(abs(rsnew)) / rhsn
        if rel <= tol:
            break
        p = r + (rsnew / rsold) * p
        rsold = rsnew
    return alm, iters, rel
