"""bench.py's host-side arithmetic (no GPU): the workload's sizes and draws, the coefficient
generators' valid slots, and the per-stage roofline figures from stage times."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def test_workload_sizes_and_boundary_points():
    for L, M in ((256, 31941), (1024, 511063)):
        m, th, ph, _ = bench.workload(L)
        assert m == M == len(th) == len(ph)
        assert th.max() <= bench.THETA_STAR and th.min() >= 0 and 0 <= ph.min() and ph.max() < 2 * np.pi
        near = np.sum(th > bench.THETA_STAR * (1 - 1e-9))
        assert near >= M // 100


def test_coefficient_generators_fill_valid_slots_only(O):
    rng = np.random.default_rng(3)
    L = 40
    a = bench.rand_alm_host(L, rng, ntrans=2).transpose(2, 1, 0)  # (L+1, 2L+1, B)
    valid = O.valid_mask(L)
    assert np.all(a[~valid] == 0) and np.all(a[valid] != 0)
    s = 2
    sa = bench.rand_spin_alm_host(L, s, rng)
    sv = O.spin_valid_mask(L, s)
    assert np.all(sa[~sv] == 0) and np.all(sa[sv] != 0)
    assert sa.flags["F_CONTIGUOUS"]


def test_stage_rooflines_arithmetic():
    info = dict(lmax=2048, npts=2044253, nufft_w=9, ring_work=304773641, nth=720, ncols=1843,
                nf1=1458, nf2=4096, nrows=742, mmax=921)
    st = {"ring_adj": (0.556, 2), "interp": (0.278, 2), "fft_fine1_fwd": (0.04, 2),
          "nufft_pad": (0.0288, 2)}
    r = bench.stage_rooflines(info, st, 34.0, 6453.7)
    assert "fft_fine1_fwd" not in r  # library FFTs are not ours
    # 10 flops per retained triple per direction
    assert abs(r["ring_adj"]["fp64_tflops"] - 10 * 304773641 / 0.278e-3 / 1e12) < 0.01
    assert abs(r["ring_adj"]["frac_fp64"] - r["ring_adj"]["fp64_tflops"] / 34.0) < 1e-3
    assert "fp64_tflops" not in r["nufft_pad"] and r["nufft_pad"]["alg_gbs"] > 0
    # ntrans scales the work
    r4 = bench.stage_rooflines(info, st, 34.0, 6453.7, B=4)
    assert abs(r4["ring_adj"]["fp64_tflops"] - 4 * r["ring_adj"]["fp64_tflops"]) < 0.05


def test_forward_stage_set_covers_the_forward_chain():
    assert set(bench.FWD_STAGES) == {"ring_fwd", "fft_theta_fwd", "nufft_pad", "fft_fine1_fwd",
                                     "rows_fwd", "fft_fine2_fwd", "interp"}
