"""pfsht_direct_forward_noalloc: Direct synthesis for callers that cannot allocate device
memory at the call (a framework owning the device's memory in its own pool, memory reserved in
advance). Everything it needs lives in one fixed array of device memory the library declares,
so it makes no allocation; it must agree with the plan-based Direct leaf (the existing entry
point) and stay correct when called again, since calls share and reuse that array.

This file is collected last on purpose: if it fails, a run that stops at the first failure has
already run every other test. It passes alone in a fresh process as well as after the others."""
import ctypes as C

import numpy as np
import pytest

from helpers import cap_points, rel, to_dev, to_host

pytestmark = pytest.mark.gpu


def _noalloc(pf, theta_d, phi_d, lmax, alm_d, f_d):
    import torch
    lib = pf._lib.load()
    st = lib.pfsht_direct_forward_noalloc(theta_d.data_ptr(), phi_d.data_ptr(), theta_d.numel(),
                                          lmax, alm_d.data_ptr(), f_d.data_ptr(),
                                          torch.cuda.current_stream().cuda_stream)
    return st


def test_noalloc_direct_matches_plan_twice(pf, O, cuda):
    import torch
    L, M = 96, 2500
    rng = np.random.default_rng(2024)
    th, ph = cap_points(M, theta_star=np.deg2rad(35.0), rng=rng)
    plan = pf.Plan(th, ph, lmax=L, method="direct")
    assert plan.algorithm == "DirectAlgorithm"
    thd = torch.from_numpy(th).to(cuda)
    phd = torch.from_numpy(ph).to(cuda)
    for call in range(2):  # the second call reuses the scratch the first one left behind
        alm = O.rand_alm(L, rng=rng)[:, :, 0]
        ref = to_host(plan * to_dev(alm))
        f = pf.zeros_field(M, device=cuda)
        assert _noalloc(pf, thd, phd, L, to_dev(alm), f) == pf._lib.OK, pf._lib.last_error()
        got = to_host(f)
        # same recurrence and phases as the plan's direct leaf; only the order in which
        # per-point tables are computed differs
        assert rel(got, ref) < 1e-12, (call, rel(got, ref))
    # and against the CPU oracle's Direct leaf
    assert rel(got, O.Direct(th, ph, L).forward(alm[:, :, None], 8)[:, 0]) < 1e-12


@pytest.mark.parametrize("L", [0, 1, 2])
def test_noalloc_smallest_degrees(pf, O, cuda, L):
    # lmax 0 and 1 launch no recurrence-table kernel (the table holds one unwritten entry);
    # lmax 2 is the first degree with a monic step
    import torch
    rng = np.random.default_rng(30 + L)
    M = 7
    th, ph = cap_points(M, theta_star=np.pi, rng=rng)
    plan = pf.Plan(th, ph, lmax=L, method="direct")
    thd = torch.from_numpy(th).to(cuda)
    phd = torch.from_numpy(ph).to(cuda)
    for call in range(2):
        alm = O.rand_alm(L, rng=rng)[:, :, 0]
        f = pf.zeros_field(M, device=cuda)
        assert _noalloc(pf, thd, phd, L, to_dev(alm), f) == pf._lib.OK, pf._lib.last_error()
        got = to_host(f)
        assert rel(got, to_host(plan * to_dev(alm))) < 1e-13, (L, call)
        assert rel(got, O.Direct(th, ph, L).forward(alm[:, :, None])[:, 0]) < 1e-13, (L, call)


def test_noalloc_allocates_no_device_memory(pf, O, cuda):
    # after a first call (which looks the array's address up), further calls leave the device's
    # free memory unchanged: the scratch is the library's fixed array, nothing is allocated
    import torch
    L, M = 64, 1500
    rng = np.random.default_rng(31)
    th, ph = cap_points(M, theta_star=np.deg2rad(25.0), rng=rng)
    thd = torch.from_numpy(th).to(cuda)
    phd = torch.from_numpy(ph).to(cuda)
    alm = to_dev(O.rand_alm(L, rng=rng)[:, :, 0])
    f = pf.zeros_field(M, device=cuda)
    assert _noalloc(pf, thd, phd, L, alm, f) == pf._lib.OK, pf._lib.last_error()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        assert _noalloc(pf, thd, phd, L, alm, f) == pf._lib.OK, pf._lib.last_error()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0


def test_noalloc_rejects_lmax_above_its_limit(pf, cuda):
    import torch
    th = torch.full((4,), 0.3, dtype=torch.float64, device=cuda)
    ph = torch.zeros(4, dtype=torch.float64, device=cuda)
    alm = torch.zeros(16, dtype=torch.complex128, device=cuda)  # never read: rejected first
    f = pf.zeros_field(4, device=cuda)
    assert _noalloc(pf, th, ph, 2049, alm, f) == pf._lib.ERR_ARGUMENT
    assert "lmax" in pf._lib.last_error()


def test_noalloc_rejects_sizes_beyond_its_scratch(pf, cuda):
    import torch
    L, M = 1024, 20000  # needs about 20000 * 2049 * 16 bytes, far above the fixed array
    th = torch.full((M,), 0.3, dtype=torch.float64, device=cuda)
    ph = torch.zeros(M, dtype=torch.float64, device=cuda)
    alm = pf.zeros_alm(L, device=cuda)
    f = pf.zeros_field(M, device=cuda)
    assert _noalloc(pf, th, ph, L, alm, f) == pf._lib.ERR_ARGUMENT
    assert "scratch" in pf._lib.last_error()
