"""Shared helpers for the tests: seeded cap point sets and host/device array moves."""
import numpy as np

THETA_STAR = np.deg2rad(20.0)


def cap_points(M, theta_star=THETA_STAR, rng=None, area_uniform=True):
    """cos(theta) uniform in [cos theta*, 1] (area-uniform) or theta* sqrt(u)
    (benchmark/calibrate.jl:56); phi uniform in [0, 2 pi)."""
    rng = np.random.default_rng(0) if rng is None else rng
    if area_uniform:
        th = np.arccos(1 - (1 - np.cos(theta_star)) * rng.random(M))
    else:
        th = theta_star * np.sqrt(rng.random(M))
    ph = 2 * np.pi * rng.random(M)
    return th, ph


def cn(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def to_dev(a, device="cuda:0"):
    """numpy array (any order) -> CUDA tensor with the same Fortran layout."""
    import torch
    a = np.asarray(a)
    t = torch.from_numpy(np.ascontiguousarray(a.T)).to(device)
    return t.permute(*reversed(range(a.ndim)))


def to_host(t):
    """CUDA tensor -> numpy array of the same shape (Fortran order)."""
    return np.asfortranarray(t.permute(*reversed(range(t.dim()))).contiguous().cpu().numpy().T)


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def dot_rel(f, g, alm, a):
    lhs = np.vdot(np.ravel(f, order="F"), np.ravel(g, order="F"))
    rhs = np.vdot(np.ravel(alm, order="F"), np.ravel(a, order="F"))
    return abs(lhs - rhs) / abs(lhs)


def plan_grid(plan):
    """The NUFFT fine-grid lengths a device plan uses (for the oracle's ES NUFFT)."""
    return plan.info["nf1"], plan.info["nf2"]
