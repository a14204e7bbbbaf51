"""The CPU oracle against analytic known answers (the reference ships no fixtures).

Each test pins one restated routine: the FFTPACK5 halfcomplex convention, the
single-mode Poisson solve, CIC mass conservation and weights, the f(R)
background fixed point, MG convergence by the reference's own criterion, the
MOVE kick of a linear potential and the P(k) of a single mode.
"""
import numpy as np
import pytest

from conftest import random_particles


def test_rfft1f_halfcomplex_convention(orc):
    n = 16
    x = np.random.default_rng(0).standard_normal(n)
    r = orc.rfft1f(x)
    F = np.fft.fft(x)
    assert np.isclose(r[0], F[0].real / n)
    for m in range(1, n // 2):
        assert np.isclose(r[2 * m - 1], 2 * F[m].real / n)     # r(2m)
        assert np.isclose(r[2 * m], -2 * F[m].imag / n)        # r(2m+1)
    assert np.isclose(r[n - 1], F[n // 2].real / n)
    np.testing.assert_allclose(orc.rfft1b(r), x, atol=1e-13)


def test_potential_single_mode(orc):
    N = 16
    i = np.arange(N)
    x, y, z = np.meshgrid(i, i, i, indexing="ij")
    kx, ky, kz = 2, 3, 5
    f = np.sin(2 * np.pi * (kx * x + ky * y + kz * z) / N)
    delta = np.ascontiguousarray(f.transpose(2, 1, 0)).reshape(-1)
    a = 0.5
    phi = orc.potential(delta.astype(np.float64), N, a, 0.3, 0.05)
    P16 = 6.28318530718
    lam = sum(2 * np.cos(P16 * k / N) for k in (kx, ky, kz)) - 6.0
    trfi = float(np.float32(np.float32(1.5) * np.float32(0.3) / np.float32(a)))
    np.testing.assert_allclose(phi, delta * trfi / lam, atol=1e-12)


def test_density_mass_and_single_particle(orc):
    N = 16
    parts = random_particles(8, N, seed=1)
    fi = orc.density(parts[0], parts[1], parts[2], N, fp64=True)
    assert abs(np.sum(fi + 1.0) - N ** 3) < 1e-9 * N ** 3
    # one particle at (2.25, 3.5, 16.75): weights split over the periodic wrap in z
    one = [np.array([v], np.float32) for v in (2.25, 3.5, 16.75)]
    fi = orc.density(*one, N, fp64=True).reshape(N, N, N)   # [k][j][i]
    W = N ** 3
    w = lambda d: np.array([1 - d, d])
    cube = np.einsum("k,j,i->kji", w(0.75), w(0.5), w(0.25)) * W
    got = np.zeros((2, 2, 2))
    for dk, kk in enumerate((15, 0)):
        for dj, jj in enumerate((2, 3)):
            for di, ii in enumerate((1, 2)):
                got[dk, dj, di] = fi[kk, jj, ii] + 1.0
    np.testing.assert_allclose(got, cube, rtol=1e-12)


def _fr_cfg(m, N, n=1, **kw):
    return m.make_config(N, N // 2, float(N), mg_model=1, fr_n=n, fr0=-1e-5, **kw)


@pytest.mark.parametrize("n", [0, 1, 2])
def test_fr_background_is_a_fixed_point(orc, n):
    """delta = 0 and u = u_bg solve the f(R) equation: the residual is ~0."""
    import mgglam_b200 as m
    N = 16
    cfg = _fr_cfg(m, N, n)
    a = 0.7
    delta = np.zeros(N ** 3, np.float64)
    u, rep = orc.scalar_field(delta, np.zeros_like(delta), cfg, a, 1)
    Om, OmL = np.float32(0.3089), np.float32(0.6911)
    a32 = np.float32(a)
    R = 3.0 * (float(Om / (a32 * a32 * a32)) + 4.0 * float(OmL))
    R0 = 3.0 * (float(Om) + 4.0 * float(OmL))
    fR = -1e-5 * (R0 / R) ** (n + 1)
    # stored normalised at exit (PMP2extradof.f90:131-146): u / u_bg == 1
    np.testing.assert_allclose(u, 1.0, rtol=1e-10)
    assert rep.residual[0] < 1e-12


def test_fr_converges_by_reference_criterion(orc):
    import mgglam_b200 as m
    N = 32
    cfg = _fr_cfg(m, N, 1, iter_count_max=10)
    parts = random_particles(16, N, seed=2, clustered=True)
    delta = orc.density(parts[0], parts[1], parts[2], N, fp64=True)
    u, rep = orc.scalar_field(delta, np.zeros_like(delta), cfg, 0.8, 1)
    res = [rep.residual[i] for i in range(rep.cycles)]
    assert rep.exit_reason in (1, 2)
    assert res[-1] < 0.05 * res[0]
    assert np.all(u > 0)


def test_move_linear_potential_kick(orc):
    """Phi = g*x: the 2x-gradient stencil gives GX = PCONST * 2g everywhere off the wrap."""
    import mgglam_b200 as m
    N = 16
    cfg = m.make_config(N, 2, float(N), mg_flag=0)
    i = np.arange(N, dtype=np.float64)
    g = 0.01
    phi = np.broadcast_to(g * i, (N, N, N)).reshape(-1)
    parts = [np.array([6.3, 7.7, 8.1, 9.9, 5.5, 4.4, 7.2, 8.8], np.float32) for _ in range(3)]
    parts += [np.zeros(8, np.float32) for _ in range(3)]
    a, da, fv = 0.5, 0.02, 1.0
    out, _ = orc.move(phi, None, parts, cfg, a, da, fv)
    a32, da32 = np.float32(a), np.float32(da)
    Om, OmL = np.float32(0.3089), np.float32(0.6911)
    pconst = float(-np.sqrt(a32 / (Om + OmL * a32 * a32 * a32)) * da32 * np.float32(0.5) / np.float32(fv))
    np.testing.assert_allclose(out[3], pconst * 2 * g, rtol=1e-6)
    np.testing.assert_allclose(out[4], 0.0, atol=1e-12)


def test_power_single_mode(orc):
    """delta = A cos(2 pi k.x/N): all power in bin |k| with P = Box^3 A^2/4 per mode pair."""
    N = 16
    box = 100.0
    i = np.arange(N)
    x, y, z = np.meshgrid(i, i, i, indexing="ij")
    A = 0.3
    k = (3, 0, 0)
    f = A * np.cos(2 * np.pi * (k[0] * x + k[1] * y + k[2] * z) / N)
    delta = np.ascontiguousarray(f.transpose(2, 1, 0)).reshape(-1).astype(np.float32)
    pk = orc.power(delta, N, box)
    b = 3  # bin index |k| = 3 -> entry 2
    total = pk["pk"][b - 1] * pk["nmodes"][b - 1] / box ** 3
    assert abs(total - 2 * (A / 2) ** 2) < 1e-6
    others = np.delete(pk["pk"], b - 1)
    assert np.max(np.abs(others)) < 1e-8 * pk["pk"][b - 1]
