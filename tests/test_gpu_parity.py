"""Device parity against the CPU oracle: ring pass, full stretched apply, dot test.
Mirrors the reference's gpu/runtests.jl and test/test_transforms.jl gates."""
import numpy as np
import pytest

from helpers import cap_points, cn, dot_rel, plan_grid, rel, to_dev, to_host

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("L", [128, 512])
def test_ring_pass_matches_oracle(pf, O, cuda, L):
    # gpu/runtests.jl:42-66 compares the device ring pass with the host one
    rng = np.random.default_rng(11)
    th, ph = cap_points(4000, rng=rng)
    plan = pf.Plan(th, ph, lmax=L, tol=1e-8)
    ref = O.Stretch(th, ph, L, 1e-8, nufft="es", nufft_grid=plan_grid(plan))
    alm = O.rand_alm(L, rng=rng)
    G_ref = ref.rings.rings_from_alm(alm)
    n = plan.info["nrings"]
    G = to_dev(np.zeros((n, 2 * L + 1, 1), np.complex128, order="F"))
    pf.ring_forward(plan, to_dev(alm), G)
    # the device fuses each product into an FMA where Julia rounds it separately, so the
    # two recurrences differ at round-off that grows with the degree (~1e-13 at L = 512)
    assert rel(to_host(G), G_ref) < 1e-11
    Gr = np.asfortranarray(cn(rng, n, 2 * L + 1, 1))
    a_ref = ref.rings.alm_from_rings(Gr)
    a = to_dev(np.zeros_like(alm, order="F"))
    pf.ring_adjoint(plan, to_dev(Gr), a)
    assert O.alm_reldiff(to_host(a), a_ref, L) < 1e-12


@pytest.mark.parametrize("L", [128, 256, 512])
def test_stretch_apply_matches_oracle(pf, O, cuda, L):
    rng = np.random.default_rng(12)
    M = int(round(4 * (L * np.deg2rad(20)) ** 2))  # 31,941 at lmax 256: the workload's M
    th, ph = cap_points(M, rng=rng)
    plan = pf.Plan(th, ph, lmax=L, tol=1e-8)
    ref = O.Stretch(th, ph, L, 1e-8, nufft="es", nufft_grid=plan_grid(plan))
    alm = O.rand_alm(L, rng=rng)
    f = to_host(plan * to_dev(alm[:, :, 0]))
    f_ref = ref.forward(alm, nthreads=8)[:, 0]
    assert rel(f, f_ref) < 1e-11
    g = cn(rng, M)
    a = to_host(plan.H * to_dev(g))
    a_ref = ref.adjoint(g, nthreads=8)[:, :, 0]
    assert O.alm_reldiff(a, a_ref, L) < 1e-10
    assert dot_rel(f, g, alm[:, :, 0], a) < 1e-12


def test_ring_adjoint_is_deterministic(pf, O, cuda):
    # the reference's threaded adjoint ring pass equals its serial one bit for bit
    # (test/test_backends.jl:202-259): with the deterministic option every order's retained rings
    # sit in one item whose warp adds its ring tiles' sums in a fixed order, so two passes agree
    # bit for bit
    rng = np.random.default_rng(13)
    L = 1024
    th, ph = cap_points(100000, rng=rng)
    plan = pf.Plan(th, ph, lmax=L, tol=1e-8, deterministic=True)
    n = plan.info["nrings"]
    Gr = to_dev(np.asfortranarray(cn(rng, n, 2 * L + 1, 1)))
    out = []
    for _ in range(2):
        a = to_dev(np.zeros((L + 1, 2 * L + 1, 1), np.complex128, order="F"))
        pf.ring_adjoint(plan, Gr, a)
        out.append(to_host(a))
    assert np.array_equal(out[0], out[1])
