"""Background table of the k-mouflage and coupled-scalar-field models (host code).

mgg_background_table restates Fix_Parameter_lambda and extradof_ini_background
(PMP2mod_MGbackground.f90:37-185, 469-731): a shooting solve for lambda such
that H(a=1) = H0, then the table BackgroundEvolution(1:100020, 1:6).  No GPU
is needed; the checks are properties of the solution:
  * the shooting condition aH/H0 = 1 at a = 1 to the reference's 1e-6;
  * column 3 is d(column 2)/dN and column 4 is d(column 3)/dN (N = ln a);
  * the oracle's multigrid solve with the table converges.
"""
import numpy as np
import pytest

from conftest import random_particles


@pytest.fixture(scope="module")
def m():
    import mgglam_b200
    return mgglam_b200


@pytest.fixture(scope="module")
def tables(m):
    out = {}
    for model in (4, 5):
        cfg = m.make_config(32, 16, 32.0, mg_model=model)
        tab, lam = m.background_table(cfg)
        out[model] = (cfg, tab, lam)
    return out


@pytest.mark.parametrize("model", [4, 5])
def test_background_shooting_condition(tables, model):
    cfg, tab, lam = tables[model]
    assert tab.shape == (100020, 6)
    assert np.isfinite(tab).all()
    assert np.isfinite(lam) and lam > 0
    assert (cfg.kmf_lambda if model == 4 else cfg.csf_lambda) == lam
    a = tab[:, 0]
    assert np.all(np.diff(a) > 0)
    assert abs(a[0] - 1.0 / (1.0 + 1.0e6)) < 1e-12
    # a = 1 is row 100001 (N = 0); aH/H0 = 1 there
    i1 = 100000
    assert abs(a[i1] - 1.0) < 1e-12
    assert abs(tab[i1, 4] - 1.0) < 1e-6


@pytest.mark.parametrize("model", [4, 5])
def test_background_columns_are_derivatives(tables, model):
    _, tab, _ = tables[model]
    N = np.log(tab[:, 0])
    sl = slice(50000, 100000, 10)   # a in [1e-3, 1]
    d2 = np.gradient(tab[:, 1], N)[sl]
    d3 = np.gradient(tab[:, 2], N)[sl]
    assert np.max(np.abs(d2 - tab[sl, 2])) <= 1e-5 * max(1.0, np.max(np.abs(tab[sl, 2])))
    assert np.max(np.abs(d3 - tab[sl, 3])) <= 1e-4 * max(1.0, np.max(np.abs(tab[sl, 3])))


def test_background_rejects_other_models(m):
    cfg = m.make_config(32, 16, 32.0, mg_model=1)
    with pytest.raises(m.MGGError):
        m.background_table(cfg)


@pytest.mark.parametrize("model", [4, 5])
def test_oracle_kmf_csf_multigrid_converges(orc, tables, model):
    cfg, tab, _ = tables[model]
    parts = random_particles(16, 32, seed=23, clustered=True)
    delta = orc.density(parts[0], parts[1], parts[2], 32)
    u, rep = orc.scalar_field(delta, np.zeros_like(delta), cfg, 0.5, 1, bg=tab)
    r = [rep.residual[i] for i in range(rep.cycles)]
    assert rep.cycles == 4
    assert all(np.isfinite(r))
    assert all(r[i + 1] < 0.2 * r[i] for i in range(len(r) - 1)), r
    assert np.isfinite(u).all() and np.abs(u).max() > 0
