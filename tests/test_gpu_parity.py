"""GPU parity: every kernel of the PM step against the CPU oracle on the same inputs.

Tolerances (FP32 storage on both sides, FP64 arithmetic where the reference
uses Real*8): grids within 1e-5 relative to the field's scale, particle
positions within 2 ulp of the grid coordinate, sort keys and per-cell counts
exact.
"""
import numpy as np
import pytest

from conftest import random_particles

pytestmark = pytest.mark.gpu

N, NROW, BOX = 32, 16, 32.0


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.fixture(scope="module")
def m():
    import mgglam_b200
    return mgglam_b200


def make_box(m, mg_model=1, **kw):
    cfg = m.make_config(N, NROW, BOX, mg_model=mg_model, **kw)
    return m.Box(cfg), cfg


@pytest.mark.parametrize("clustered", [False, True])
def test_density_matches_oracle_and_is_deterministic(m, orc, clustered):
    parts = random_particles(NROW, N, seed=3, clustered=clustered)
    box, _ = make_box(m)
    box.upload_particles(*parts)
    box.set_time(0.5, 0.01)
    box.density()
    g1 = box.download_grid(m.GRID_FI)
    box.density()
    g2 = box.download_grid(m.GRID_FI)
    assert np.array_equal(g1.view(np.uint32), g2.view(np.uint32)), "CIC is not bit-reproducible"
    ref = orc.density(parts[0], parts[1], parts[2], N)
    ref64 = orc.density(parts[0], parts[1], parts[2], N, fp64=True)
    # against the FP64 oracle the GPU's single rounding is tighter than the Real*4 path
    assert np.max(np.abs(g1 - ref64) / (1.0 + np.abs(ref64))) < 1e-6
    assert np.max(np.abs(g1 - ref) / (1.0 + np.abs(ref))) < 1e-5
    # total mass: sum(delta + 1) = N^3
    assert abs(float(np.sum(g1.astype(np.float64) + 1.0)) - N ** 3) < 1e-3 * N ** 3 * 1e-3
    box.close()


def test_density_permutation_invariant(m):
    """Same particles in another order give the bit-identical grid."""
    parts = random_particles(NROW, N, seed=5, clustered=True)
    perm = np.random.default_rng(1).permutation(NROW ** 3)
    box, _ = make_box(m)
    box.upload_particles(*parts)
    box.density()
    a = box.download_grid(m.GRID_FI)
    box.upload_particles(*[p[perm] for p in parts])
    box.density()
    b = box.download_grid(m.GRID_FI)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    box.close()


@pytest.mark.parametrize("n,nrow,case", [(32, 16, "uniform"), (32, 16, "clustered"), (32, 16, "edges"),
                                         (256, 128, "clustered")])
def test_cic_keys_exact(m, n, nrow, case):
    """Row counts, row offsets and per-cell counts of the GPU's counting sort equal
    np.bincount of the reference's keys I = INT(X), J = INT(Y), K = INT(Z)
    (PMP2mod_density.f90:235-248), exactly; with particles on the faces of the
    box (x = 1 and x = NGRID + 1 - ulp) in the edge case."""
    parts = random_particles(nrow, n, seed=47, clustered=(case == "clustered"))
    if case == "edges":
        rng = np.random.default_rng(3)
        top = np.nextafter(np.float32(n + 1), np.float32(0))
        for c in range(3):
            pick = rng.choice(nrow ** 3, size=nrow ** 3 // 8, replace=False)
            parts[c][pick[: pick.size // 2]] = np.float32(1.0)
            parts[c][pick[pick.size // 2:]] = top
    cfg = m.make_config(n, nrow, float(n), mg_flag=0)
    box = m.Box(cfg)
    try:
        box.upload_particles(*parts)
        box.density()
        rc, rs, cc = box.cic_keys()
    finally:
        box.close()
    I, J, K = (np.asarray(p, np.float32).astype(np.int64) for p in parts[:3])
    assert I.min() >= 1 and I.max() <= n
    row = (J - 1) + n * (K - 1)
    want = np.bincount(row, minlength=n * n)
    np.testing.assert_array_equal(rc, want)
    np.testing.assert_array_equal(rs, np.concatenate([[0], np.cumsum(want)]))
    np.testing.assert_array_equal(cc, np.bincount((I - 1) + n * row, minlength=n ** 3))


def test_potential_matches_oracle(m, orc):
    rng = np.random.default_rng(7)
    delta = rng.standard_normal(N ** 3).astype(np.float32)
    delta -= np.float32(delta.mean())
    box, _ = make_box(m)
    box.set_time(0.37, 0.01)
    box.upload_grid(m.GRID_FI, delta)
    box.potential()
    phi = box.download_grid(m.GRID_FI)
    ref = orc.potential(delta, N, 0.37, 0.3089, 0.0486)
    ref64 = orc.potential(delta.astype(np.float64), N, 0.37, 0.3089, 0.0486)
    assert rel_err(phi, ref64) < 1e-5
    assert rel_err(phi, ref) < 1e-5
    box.close()


def test_potential_single_mode_eigenvalue(m):
    """A single Fourier mode is divided by its 7-point eigenvalue (PMP2main.f90:805-816)."""
    i = np.arange(N)
    kx, ky, kz = 3, 5, 1
    x, y, z = np.meshgrid(i, i, i, indexing="ij")
    f = np.cos(2 * np.pi * (kx * x + ky * y + kz * z) / N)
    delta = np.ascontiguousarray(f.transpose(2, 1, 0)).reshape(-1).astype(np.float32)
    box, _ = make_box(m)
    a = 0.5
    box.set_time(a, 0.01)
    box.upload_grid(m.GRID_FI, delta)
    box.potential()
    phi = box.download_grid(m.GRID_FI).astype(np.float64)
    P16 = 6.28318530718
    G = lambda k: 2 * np.cos(P16 * k / N)
    lam = G(kx) + G(ky) + G(kz) - 6.0
    trfi = np.float32(np.float32(1.5) * np.float32(0.3089) / np.float32(a))
    expect = delta.astype(np.float64) * float(trfi) / lam
    assert rel_err(phi, expect) < 2e-6
    box.close()


def test_power_matches_oracle(m, orc):
    parts = random_particles(NROW, N, seed=11, clustered=True)
    box, _ = make_box(m)
    box.upload_particles(*parts)
    pk = box.power(recompute_density=True)
    fi = orc.density(parts[0], parts[1], parts[2], N)
    ref = orc.power(fi, N, BOX)
    np.testing.assert_array_equal(pk["nmodes"], ref["nmodes"])
    np.testing.assert_allclose(pk["k"], ref["k"], rtol=1e-6)
    np.testing.assert_allclose(pk["pk"], ref["pk"], rtol=2e-5)
    np.testing.assert_array_equal(pk["nmodeslog"], ref["nmodeslog"])
    sel = ref["nmodeslog"] > 0
    np.testing.assert_allclose(pk["pklog"][sel], ref["pklog"][sel], rtol=2e-5)
    box.close()


def test_move_matches_oracle(m, orc):
    rng = np.random.default_rng(13)
    phi = rng.standard_normal(N ** 3).astype(np.float32)
    parts = random_particles(NROW, N, seed=17, vscale=0.5)
    box, cfg = make_box(m, mg_flag=0)
    box.upload_particles(*parts)
    box.upload_grid(m.GRID_FI, phi)
    a, da, fv = 0.25, 0.01, 1.2
    box.set_time(a, da)
    e = box.move(fv)
    got = box.download_particles()
    ref, e_ref = orc.move(phi, None, parts, cfg, a, da, fv)
    for g, r in zip(got[:3], ref[:3]):
        assert np.max(np.abs(g - r)) <= 2 * np.spacing(np.float32(N + 1))
    for g, r in zip(got[3:], ref[3:]):
        assert rel_err(g, r) < 1e-6
    assert abs(e - e_ref) <= 1e-6 * abs(e_ref)
    box.close()


def test_potential_mg_matches_oracle(m, orc):
    rng = np.random.default_rng(19)
    fi = rng.standard_normal(N ** 3).astype(np.float32)
    fi2 = (1.0 + 0.1 * rng.standard_normal(N ** 3)).astype(np.float32)
    for model in (1, 2, 3, 4, 5):
        box, cfg = make_box(m, mg_model=model)
        box.set_time(0.8, 0.01)
        box.upload_grid(m.GRID_FI, fi)
        box.upload_grid(m.GRID_FI2, fi2)
        box.potential_mg()
        got = box.download_grid(m.GRID_FI)
        ref = orc.potential_mg(fi, fi2, cfg, 0.8)
        assert rel_err(got, ref) < 1e-6, model
        box.close()


def fr_density(orc):
    parts = random_particles(NROW, N, seed=23, clustered=True)
    return orc.density(parts[0], parts[1], parts[2], N)


@pytest.mark.parametrize("frn", [0, 1, 2])
@pytest.mark.parametrize("cycle", ["V", "F", "W"])
def test_scalar_field_fr_matches_oracle(m, orc, frn, cycle):
    delta = fr_density(orc)
    box, cfg = make_box(m, mg_model=1, fr_n=frn, cycle=cycle, iter_count_max=3)
    a = 0.6
    box.set_time(a, 0.01)
    box.upload_grid(m.GRID_FI, delta)
    rep = box.scalar_field(1)
    u = box.download_grid(m.GRID_FI2)
    u_ref, rep_ref = orc.scalar_field(delta, np.zeros_like(delta), cfg, a, 1)
    assert rep.cycles == rep_ref.cycles
    assert rel_err(u, u_ref) < 1e-5
    for i in range(rep.cycles):
        assert abs(rep.residual[i] - rep_ref.residual[i]) <= 1e-3 * rep_ref.residual[i]
    box.close()


@pytest.mark.parametrize("model", [2, 3])
def test_scalar_field_dgp_sym_match_oracle(m, orc, model):
    """nDGP reads same-colour diagonal neighbours: the GPU's colour sweeps read the
    field as it was before the sweep, so the oracle runs the same snapshot order
    and the two agree to FP32 rounding.  Symmetron's 7-point sweep is order-free."""
    delta = fr_density(orc)
    box, cfg = make_box(m, mg_model=model, iter_count_max=4)
    a = 0.8
    box.set_time(a, 0.01)
    box.upload_grid(m.GRID_FI, delta)
    rep = box.scalar_field(1)
    u = box.download_grid(m.GRID_FI2)
    u_ref, rep_ref = orc.scalar_field(delta, np.zeros_like(delta), cfg, a, 1, order="snapshot")
    assert rep.cycles == rep_ref.cycles
    assert rel_err(u, u_ref) < 1e-5, rel_err(u, u_ref)
    for i in range(rep.cycles):
        assert abs(rep.residual[i] - rep_ref.residual[i]) <= 1e-3 * rep_ref.residual[i]
    box.close()


@pytest.mark.parametrize("model", [2, 4])
def test_scalar_field_converges_to_the_serial_order_solution(m, orc, bg, model):
    """The reference's serial in-place order (one OpenMP thread) and the GPU's
    snapshot order are two schedules of the same nonlinear Gauss-Seidel iteration:
    run to the residual floor (up to 40 cycles), they reach the same discrete
    solution.  nDGP stagnates on the clustered density of the other tests (both
    orders stop at the same residual, a quarter of the first), so it is run on the
    density of a known root (the manufactured field of the known-answer tests,
    amplitude 1), where it converges; its solution is defined up to a constant."""
    kw = dict(iter_count_max=40, res_conv=1e-12)
    if model == 4:
        delta = fr_density(orc)
        box, cfg = model_box(m, model, bg, **kw)
        tab = bg[model][0]
        a = 0.5
    else:
        box, cfg = make_box(m, mg_model=model, **kw)
        tab = None
        a = 1.0
        c = (np.arange(N) + 0.5) * 2.0 * np.pi / N
        zz, yy, xx = np.meshgrid(c, c, c, indexing="ij")
        prof = (np.sin(2 * xx) + np.sin(yy) * np.cos(2 * zz)).astype(np.float32).ravel()
        d64, bad = orc.dgp_root_density(prof, cfg, a)
        assert bad == 0
        delta = d64.astype(np.float32)
    box.set_time(a, 0.01)
    box.upload_grid(m.GRID_FI, delta)
    rep = box.scalar_field(1)
    u = box.download_grid(m.GRID_FI2).astype(np.float64)
    box.close()
    u_ref, rep_ref = orc.scalar_field(delta, np.zeros_like(delta), cfg, a, 1, bg=tab, order="serial")
    u_ref = u_ref.astype(np.float64)
    if model == 2:
        u, u_ref = u - u.mean(), u_ref - u_ref.mean()
    print(f"model {model}: cycles GPU {rep.cycles} serial oracle {rep_ref.cycles}; final residuals "
          f"{rep.residual[rep.cycles - 1]:.3e} / {rep_ref.residual[rep_ref.cycles - 1]:.3e}; "
          f"field difference {rel_err(u, u_ref):.3e}")
    # both at the residual floor of FP32 storage
    assert rep.residual[rep.cycles - 1] < 1e-3 * rep.residual[0]
    assert rep_ref.residual[rep_ref.cycles - 1] < 1e-3 * rep_ref.residual[0]
    assert rel_err(u, u_ref) < 1e-4, rel_err(u, u_ref)


@pytest.mark.parametrize("model,frn", [(1, 1), (1, 0), (1, 2), (3, 0)])
def test_scalar_field_fused_sweep_n128(m, orc, model, frn):
    """N = 128 takes the fused red-black sweep on levels 0 and 1; same result as the oracle."""
    n, nrow = 128, 64
    parts = random_particles(nrow, n, seed=29, clustered=True)
    delta = orc.density(parts[0], parts[1], parts[2], n)
    cfg = m.make_config(n, nrow, float(n), mg_model=model, fr_n=frn, iter_count_max=3)
    box = m.Box(cfg)
    a = 0.7
    box.set_time(a, 0.01)
    box.upload_grid(m.GRID_FI, delta)
    rep = box.scalar_field(1)
    u = box.download_grid(m.GRID_FI2)
    u_ref, rep_ref = orc.scalar_field(delta, np.zeros_like(delta), cfg, a, 1)
    assert rep.cycles == rep_ref.cycles
    assert rel_err(u, u_ref) < 1e-5, rel_err(u, u_ref)
    for i in range(rep.cycles):
        assert abs(rep.residual[i] - rep_ref.residual[i]) <= 1e-3 * rep_ref.residual[i]
    box.close()


# ---------------------------------------------------- k-mouflage and csf ----
@pytest.fixture(scope="module")
def bg(m):
    """Background tables of k-mouflage (4) and the coupled scalar field (5)."""
    out = {}
    for model in (4, 5):
        cfg = m.make_config(N, NROW, BOX, mg_model=model)
        out[model] = m.background_table(cfg)
    return out


def model_box(m, model, bg, **kw):
    tab, lam = bg[model]
    cfg = m.make_config(N, NROW, BOX, mg_model=model, **kw)
    if model == 4:
        cfg.kmf_lambda = lam
    else:
        cfg.csf_lambda = lam
    box = m.Box(cfg)
    box.set_background(tab)
    return box, cfg


@pytest.mark.parametrize("model", [4, 5])
@pytest.mark.parametrize("cycle", ["V", "W"])
def test_scalar_field_kmf_csf_match_oracle(m, orc, bg, model, cycle):
    delta = fr_density(orc)
    box, cfg = model_box(m, model, bg, cycle=cycle, iter_count_max=4)
    a = 0.5
    box.set_time(a, 0.01)
    box.upload_grid(m.GRID_FI, delta)
    rep = box.scalar_field(1)
    u = box.download_grid(m.GRID_FI2)
    # k-mouflage: 19-point stencil whose same-colour diagonal neighbours the GPU
    # reads from a snapshot taken before each colour sweep; the oracle runs the
    # same snapshot order.  csf: 7-point, where the order does not matter.
    u_ref, rep_ref = orc.scalar_field(delta, np.zeros_like(delta), cfg, a, 1, bg=bg[model][0], order="snapshot")
    assert rep.cycles == rep_ref.cycles
    assert rel_err(u, u_ref) < 1e-5, rel_err(u, u_ref)
    for i in range(rep.cycles):
        assert abs(rep.residual[i] - rep_ref.residual[i]) <= 1e-3 * rep_ref.residual[i]
    box.close()


@pytest.mark.parametrize("model", [2, 4, 5])
def test_scalar_field_march_sweep_n128(m, orc, bg, model):
    """N = 128: the nDGP, k-mouflage and csf colour sweeps, residuals and FAS
    right-hand sides of levels 0 and 1 take the marching shared-memory kernels;
    same result as the snapshot-order oracle (tolerances as at N = 32)."""
    n, nrow = 128, 64
    parts = random_particles(nrow, n, seed=31, clustered=True)
    delta = orc.density(parts[0], parts[1], parts[2], n)
    cfg = m.make_config(n, nrow, float(n), mg_model=model, iter_count_max=3)
    tab = None
    if model in (4, 5):
        tab, lam = bg[model]
        if model == 4:
            cfg.kmf_lambda = lam
        else:
            cfg.csf_lambda = lam
    box = m.Box(cfg)
    if tab is not None:
        box.set_background(tab)
    a = 0.6
    box.set_time(a, 0.01)
    box.upload_grid(m.GRID_FI, delta)
    rep = box.scalar_field(1)
    u = box.download_grid(m.GRID_FI2)
    u_ref, rep_ref = orc.scalar_field(delta, np.zeros_like(delta), cfg, a, 1, bg=tab, order="snapshot")
    assert rep.cycles == rep_ref.cycles
    assert rel_err(u, u_ref) < 1e-5, rel_err(u, u_ref)
    for i in range(rep.cycles):
        assert abs(rep.residual[i] - rep_ref.residual[i]) <= 1e-3 * rep_ref.residual[i]
    box.close()


@pytest.mark.parametrize("model", [4, 5])
def test_move_with_background_matches_oracle(m, orc, bg, model):
    rng = np.random.default_rng(31)
    phi = rng.standard_normal(N ** 3).astype(np.float32)
    fi2 = (0.01 * rng.standard_normal(N ** 3)).astype(np.float32)
    parts = random_particles(NROW, N, seed=37, vscale=0.5)
    box, cfg = model_box(m, model, bg)
    box.upload_particles(*parts)
    box.upload_grid(m.GRID_FI, phi)
    box.upload_grid(m.GRID_FI2, fi2)
    a, da, fv = 0.5, 0.01, 1.2
    box.set_time(a, da)
    e = box.move(fv)
    got = box.download_particles()
    ref, e_ref = orc.move(phi, fi2, parts, cfg, a, da, fv, bg=bg[model][0])
    for g, r in zip(got[:3], ref[:3]):
        assert np.max(np.abs(g - r)) <= 2 * np.spacing(np.float32(N + 1))
    for g, r in zip(got[3:], ref[3:]):
        assert rel_err(g, r) < 1e-6
    assert abs(e - e_ref) <= 1e-6 * abs(e_ref)
    box.close()
