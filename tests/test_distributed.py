"""Point decomposition across ranks (the reference's MPIBackend, ext/PartialFSHTMPIExt.jl and
test/mpi_ranks.jl) with world_size-2 gloo ranks on the CPU. The per-rank operator is the
oracle's stretched leaf standing in for a device plan; what is tested is the decomposition
(local synthesis, all-reduced adjoint) of pfsht_b200.distributed."""
import os
import socket

import numpy as np
import pytest


class _OraclePlan:
    """CPU stand-in with the Plan apply interface, over one rank's points."""

    def __init__(self, O, theta, phi, lmax, tol):
        self.S = O.Stretch(theta, phi, lmax, tol, nufft="es")
        self.lmax = lmax

    def mul(self, f, alm):
        f[:] = self.S.forward(alm[:, :, None])[:, 0]
        return f

    def mul_adjoint(self, alm, f):
        alm[:] = self.S.adjoint(f)[:, :, 0]
        return alm


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import sys

    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "tests"))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from __graft_entry__ import load_package
        from helpers import cap_points
        from oracle import oracle as O
        pf = load_package()
        dmod = sys.modules["pfsht_b200.distributed"] if "pfsht_b200.distributed" in sys.modules \
            else __import__("pfsht_b200.distributed", fromlist=["x"])
        L, tol = 128, 1e-8
        th, ph = cap_points(3000, rng=np.random.default_rng(9))
        alm = O.rand_alm(L, rng=np.random.default_rng(10))[:, :, 0]
        g = (np.random.default_rng(11).standard_normal(3000)
             + 1j * np.random.default_rng(12).standard_normal(3000))
        t_loc, p_loc, (lo, hi) = dmod.shard_points(th, ph, rank, world)
        plan = dmod.PointShardedPlan(_OraclePlan(O, t_loc, p_loc, L, tol))
        f = np.zeros(hi - lo, np.complex128)
        plan.mul(f, np.asfortranarray(alm))
        a = np.zeros_like(alm, order="F")
        plan.mul_adjoint(a, g[lo:hi].copy())
        np.save(os.path.join(out, f"f{rank}.npy"), f)
        np.save(os.path.join(out, f"a{rank}.npy"), a)
        np.save(os.path.join(out, f"range{rank}.npy"), np.array([lo, hi]))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_point_sharded_adjoint_allreduce(O, tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       start_method="spawn", join=True)
    from helpers import cap_points
    L, tol = 128, 1e-8
    th, ph = cap_points(3000, rng=np.random.default_rng(9))
    alm = O.rand_alm(L, rng=np.random.default_rng(10))
    g = (np.random.default_rng(11).standard_normal(3000)
         + 1j * np.random.default_rng(12).standard_normal(3000))
    D = O.Direct(th, ph, L)
    f_ref = D.forward(alm, 8)[:, 0]
    a_ref = D.adjoint(g, 8)[:, :, 0]
    f = np.zeros(3000, np.complex128)
    for r in range(world):
        lo, hi = np.load(tmp_path / f"range{r}.npy")
        f[lo:hi] = np.load(tmp_path / f"f{r}.npy")
        a = np.load(tmp_path / f"a{r}.npy")
        # every rank holds the same, globally summed adjoint
        assert O.alm_reldiff(a, a_ref, L) < 10 * tol
    assert np.abs(f - f_ref).max() / np.abs(f_ref).max() < 10 * tol
    # "partial really is partial" (test/mpi_ranks.jl): one rank's adjoint alone is not it
    Dh = O.Direct(th[:1500], ph[:1500], L)
    assert O.alm_reldiff(Dh.adjoint(g[:1500], 8)[:, :, 0], a_ref, L) > 1e-3
