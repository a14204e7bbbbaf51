"""Analytic known-answer tests of the scalar-field solvers (manufactured solutions).

The reference keeps sine-field tests for each model as commented density fields
(PMP2mod_density.f90:98-182) with the expected profile written next to the
solution (WriteScalarFieldToFile, PMP2extradof.f90:1581-1656).  Here the same
idea is restated from each model's field equation: pick the scalar field
u(z) = profile of a sine along one axis, and set the density contrast to the
value for which the discrete operator vanishes at every cell, i.e. with the
7-point Laplacian of the sine, (2 cos(2 pi k / N) - 2) sin, in place of its
continuum -(2 pi k / N)^2 sin.  The multigrid solve from the background must
then return u itself, up to FP32 rounding:

- f(R): u^(n+1) = |fR| = |fR_bg| (1 + A sin); after the exit rescaling the
  returned field is (1 + A sin)^(1/(n+1)), and
  delta = -(a / Om) c~^2 lap(fR) + (R_bg a^3 / (3 Om)) ((fR_bg / fR)^(1/(n+1)) - 1)
  (n = 1 on the GPU, n = 0, 1, 2 and V, F, W cycles on the oracle).
- symmetron: u = 1 + A sin and
  delta = (a / a*)^3 (1 - u^2 + 2 (c~ xi / a)^2 lap(u) / u) - 1.
- coupled scalar field: u = A sin, phi = phibar + u / c~^2 and
  delta = (lap(u) / f1 - (V'(phi) - V'(phibar)) / f1 + A'(phibar)) / A'(phi) - 1
  with f1 = 3 Om / a, A'(phi) = beta exp(beta phi), V'(phi) = -alpha lambda^2 a^2 / phi^(1+alpha).

The k-mouflage operator is affine in the density contrast too, but its
gradient terms make a closed form long; there the density is taken from the
oracle's own operator, delta = -OP(u, 0) / (OP(u, 1) - OP(u, 0)) at every cell,
for a 3-D profile u = A (sin 2x + sin y cos 2z) in the weak-field regime
(A = 1e-3) and a screened one (A = 1, where the nonlinear term varies the
operator's density coefficient across the box).  That checks that the solve
converges to the operator's root, on the oracle and on the GPU.

The nDGP operator holds the density inside a square root; its root density
follows in closed form from the operator's own terms (oracle.dgp_root_density:
Sigma = ((alpha + 4/3 lap)^2 - alpha^2) 3/8 = fct1 delta + G(u)).  Only
derivatives of the field enter that equation, so the solve returns the profile
up to a constant, and the check is on the field minus its mean (oracle only).

The oracle (C++ restatement) is checked on the CPU; the GPU path through the
C ABI in both precision forms at 32^3 (per-colour sweeps) and 128^3 (fused and
marching sweeps).
"""
import numpy as np
import pytest

import mgglam_b200 as m

AMP, KWAVE, AEXPN = 0.1, 2, 1.0


def bg_at(tab, a, col):
    """Linear interpolation in the background table at the first row with a_row >= a."""
    ist = 0
    while ist < tab.shape[0] - 1 and tab[ist, 0] < a:
        ist += 1
    ist = max(ist, 1)
    r0, r1 = tab[ist - 1], tab[ist]
    return r0[col] + (r1[col] - r0[col]) / (r1[0] - r0[0]) * (a - r0[0])


def manufactured(model, n, precision=0, cycle="V", frn=1):
    """(cfg, background table or None, density grid, expected returned field along z)."""
    z = np.arange(1, n + 1, dtype=np.float64)
    s = np.sin(2.0 * np.pi * KWAVE * (z - 0.5) / n)
    lap_of_sine = (2.0 * np.cos(2.0 * np.pi * KWAVE / n) - 2.0) * s
    a = AEXPN
    tab = None
    if model == "fr":
        box = 4.0 * n
        cfg = m.make_config(n, n // 2, box, mg_model=m.MODEL_FR, fr_n=frn, fr0=-1e-5, iter_count_max=40,
                            res_conv=1e-12, precision=precision, cycle=cycle)
        ct = 2997.92458 * n / box
        r_bg = 3.0 * (cfg.om / a ** 3 + 4.0 * cfg.oml)
        r0_bg = 3.0 * (cfg.om + 4.0 * cfg.oml)
        fr_bg = cfg.fr0 * (r0_bg / r_bg) ** (frn + 1)
        delta = (-(a / cfg.om) * ct ** 2 * fr_bg * AMP * lap_of_sine
                 + r_bg / 3.0 * a ** 3 / cfg.om * ((1.0 + AMP * s) ** (-1.0 / (frn + 1)) - 1.0))
        expect = (1.0 + AMP * s) ** (1.0 / (frn + 1))
    elif model == "sym":
        box = float(n)
        cfg = m.make_config(n, n // 2, box, mg_model=m.MODEL_SYMMETRON, iter_count_max=40, res_conv=1e-12,
                            precision=precision)
        ct = 2997.92458 * n / box
        u = 1.0 + AMP * s
        delta = (a / cfg.sym_astar) ** 3 * (1.0 - u ** 2 + 2.0 * (ct * cfg.sym_xi / a) ** 2 * AMP * lap_of_sine / u) - 1.0
        expect = u
    else:
        box = float(n)
        cfg = m.make_config(n, n // 2, box, mg_model=m.MODEL_CSF, iter_count_max=40, res_conv=1e-12,
                            precision=precision)
        tab, _ = m.background_table(cfg)   # also fixes cfg.csf_lambda
        phibar = bg_at(tab, a, 1)
        ct2 = (2997.92458 * n / box) ** 2
        beta, alpha, lam = cfg.csf_beta, cfg.csf_alpha, cfg.csf_lambda
        f1 = 3.0 * cfg.om / a

        def a_prime(ph):
            return beta * np.exp(beta * ph)

        def v_prime(ph):
            return -alpha * lam ** 2 * a ** 2 / ph ** (1.0 + alpha)

        u = AMP * s
        phi = phibar + u / ct2
        delta = (AMP * lap_of_sine / f1 - (v_prime(phi) - v_prime(phibar)) / f1 + a_prime(phibar)) / a_prime(phi) - 1.0
        expect = u
    grid = np.broadcast_to(delta[:, None, None], (n, n, n)).astype(np.float32)
    return cfg, tab, grid, expect


def kmf_manufactured(orc, n, amp, precision=0):
    """(cfg, background table, density, expected field) of the k-mouflage case on an n^3 mesh
    (cell size 2 Mpc/h, mode numbers fixed in units of the box)."""
    cfg = m.make_config(n, n // 2, 2.0 * n, mg_model=m.MODEL_KMOUFLAGE, iter_count_max=40, res_conv=1e-14,
                        precision=precision)
    tab, _ = m.background_table(cfg)
    c = (np.arange(n) + 0.5) * 2.0 * np.pi / n
    zz, yy, xx = np.meshgrid(c, c, c, indexing="ij")
    u = (amp * (np.sin(2 * xx) + np.sin(yy) * np.cos(2 * zz))).astype(np.float32).ravel()
    op0 = orc.kmf_operator(np.zeros(n ** 3, np.float32), u, cfg, AEXPN, tab)
    op1 = orc.kmf_operator(np.ones(n ** 3, np.float32), u, cfg, AEXPN, tab)
    delta = (-op0 / (op1 - op0)).astype(np.float32)
    return cfg, tab, delta, u


@pytest.mark.parametrize("amp", [1e-3, 1.0])
def test_oracle_kmf_returns_manufactured_solution(orc, amp):
    cfg, tab, delta, u = kmf_manufactured(orc, 32, amp)
    out, rep = orc.scalar_field(delta, np.zeros_like(delta), cfg, AEXPN, 1, bg=tab)
    err = float(np.max(np.abs(out.astype(np.float64) - u))) / amp
    assert err < 1e-5, (amp, err, rep.cycles)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("n", [32, 128])
@pytest.mark.parametrize("amp", [1e-3, 1.0])
def test_gpu_kmf_returns_manufactured_solution(orc, amp, n, precision):
    cfg, tab, delta, u = kmf_manufactured(orc, n, amp, precision)
    box = m.Box(cfg)
    try:
        box.set_background(tab)
        box.upload_grid(m.GRID_FI, delta)
        box.set_time(AEXPN, 0.01)
        rep = box.scalar_field(1)
        out = box.download_grid(m.GRID_FI2).astype(np.float64)
    finally:
        box.close()
    err = float(np.max(np.abs(out - u))) / amp
    assert err < (1e-5 if precision == 0 else 1e-4), (amp, n, precision, err, rep.cycles)


@pytest.mark.parametrize("amp", [1e-2, 1.0, 10.0])
def test_oracle_dgp_returns_manufactured_solution(orc, amp):
    n = 32
    cfg = m.make_config(n, n // 2, 2.0 * n, mg_model=m.MODEL_DGP, iter_count_max=60, res_conv=1e-14)
    c = (np.arange(n) + 0.5) * 2.0 * np.pi / n
    zz, yy, xx = np.meshgrid(c, c, c, indexing="ij")
    u = (amp * (np.sin(2 * xx) + np.sin(yy) * np.cos(2 * zz))).astype(np.float32).ravel()
    delta, bad = orc.dgp_root_density(u, cfg, AEXPN)
    assert bad == 0
    out, rep = orc.scalar_field(delta.astype(np.float32), np.zeros(u.size, np.float32), cfg, AEXPN, 1)
    dev = (out.astype(np.float64) - out.mean()) - (u.astype(np.float64) - u.mean())
    assert float(np.max(np.abs(dev))) / amp < 1e-5, (amp, float(np.max(np.abs(dev))) / amp, rep.cycles)


@pytest.mark.parametrize("model,cycle,frn", [("fr", "V", 1), ("fr", "F", 1), ("fr", "W", 1), ("fr", "V", 0),
                                              ("fr", "V", 2), ("sym", "V", 1), ("csf", "V", 1)])
def test_oracle_returns_manufactured_solution(orc, model, cycle, frn):
    cfg, tab, grid, expect = manufactured(model, 32, cycle=cycle, frn=frn)
    u, rep = orc.scalar_field(grid.ravel(), np.zeros(grid.size, np.float32), cfg, AEXPN, 1, bg=tab)
    u = u.reshape(grid.shape).astype(np.float64)
    err = float(np.max(np.abs(u - expect[:, None, None])))
    assert err < 1e-6, (model, err, rep.cycles)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("n", [32, 128])
@pytest.mark.parametrize("model", ["fr", "sym", "csf"])
def test_gpu_returns_manufactured_solution(model, n, precision):
    cfg, tab, grid, expect = manufactured(model, n, precision)
    box = m.Box(cfg)
    try:
        if tab is not None:
            box.set_background(tab)
        box.upload_grid(m.GRID_FI, grid)
        box.set_time(AEXPN, 0.01)
        rep = box.scalar_field(1)
        u = box.download_grid(m.GRID_FI2).reshape(grid.shape).astype(np.float64)
    finally:
        box.close()
    err = float(np.max(np.abs(u - expect[:, None, None])))
    # FP32 storage of the field and the density: a few units of the last place of
    # the profile in the plain path; the precision form's FP32 updates add a few more
    assert err < (2e-6 if precision == 0 else 1e-5), (model, n, precision, err, rep.cycles)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("n", [32, 128])
@pytest.mark.parametrize("amp", [1e-2, 1.0, 10.0])
def test_gpu_dgp_returns_manufactured_solution(orc, amp, n, precision):
    """The nDGP root density on the GPU (per-colour sweeps at 32^3, the marching
    colour sweeps at 128^3): the solve returns the profile up to its constant mode."""
    cfg = m.make_config(n, n // 2, 2.0 * n, mg_model=m.MODEL_DGP, iter_count_max=60, res_conv=1e-14,
                        precision=precision)
    c = (np.arange(n) + 0.5) * 2.0 * np.pi / n
    zz, yy, xx = np.meshgrid(c, c, c, indexing="ij")
    u = (amp * (np.sin(2 * xx) + np.sin(yy) * np.cos(2 * zz))).astype(np.float32).ravel()
    delta, bad = orc.dgp_root_density(u, cfg, AEXPN)
    assert bad == 0
    box = m.Box(cfg)
    try:
        box.upload_grid(m.GRID_FI, delta.astype(np.float32))
        box.set_time(AEXPN, 0.01)
        rep = box.scalar_field(1)
        out = box.download_grid(m.GRID_FI2).astype(np.float64)
    finally:
        box.close()
    dev = (out - out.mean()) - (u.astype(np.float64) - u.mean())
    err = float(np.max(np.abs(dev))) / amp
    print(f"nDGP manufactured n={n} amp={amp} precision={precision}: {err:.2e} of the amplitude, {rep.cycles} cycles")
    assert err < (1e-5 if precision == 0 else 1e-4), (amp, n, precision, err, rep.cycles)
