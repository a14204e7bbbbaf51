"""Precision form (MGG_PREC_MIXED) against the oracle's FP64 mode and the plain path.

In the precision form the f(R) n = 1 smoother forms P and the cubic root in
FP32 (Newton from the cell's current value, with the FP64 closed form where
that start is unusable), and the per-cell residual, FAS right-hand side and
level-1 restriction are FP32 with FP64 norm accumulation; CIC, FFT,
POTENT_FOR_MG and MOVE are the plain path's.  The nDGP, symmetron,
k-mouflage and csf sweeps of the fused / marching kernels are FP32 as well,
and so are their residuals and FAS right-hand sides.  The errors of both
GPU paths are stated against the oracle run in FP64 (FP64 grids and
arithmetic) on the same particles, for the fields the step produces: density,
potential, scalar field, positions after one step and P(k).  The smoother is
the fused sweep of levels of 128^3 and up, so the mesh is 128^3.
"""
import numpy as np
import pytest

from conftest import random_particles

pytestmark = pytest.mark.gpu

N, NROW = 128, 64


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.fixture(scope="module")
def m():
    import mgglam_b200
    return mgglam_b200


def gpu_step(m, cfg, parts, a, astep):
    """One main-loop body, routine by routine, keeping every intermediate field."""
    box = m.Box(cfg)
    box.upload_particles(*parts)
    box.set_time(a, astep)
    box.density()
    out = {"density": box.download_grid(m.GRID_FI)}
    rep = box.scalar_field(1)
    out["cycles"] = rep.cycles
    out["residual"] = [rep.residual[i] for i in range(rep.cycles)]
    box.potential()
    box.potential_mg()
    out["potential"] = box.download_grid(m.GRID_FI)
    out["scalar"] = box.download_grid(m.GRID_FI2)
    box.move(1.0)
    out["parts"] = box.download_particles()
    p = box.power(True)
    out["pk"], out["k"] = p["pk"], p["k"]
    box.close()
    return out


def oracle_step_fp64(orc, cfg, parts, a, astep):
    delta = orc.density(parts[0], parts[1], parts[2], N, fp64=True)
    u, rep = orc.scalar_field(delta, np.zeros_like(delta), cfg, a, 1)
    phi = orc.potential(delta, N, a, cfg.om, cfg.omb)
    phi = orc.potential_mg(phi, u, cfg, a)
    newp, _ = orc.move(phi, u, parts, cfg, a, astep, 1.0)
    d1 = orc.density(newp[0], newp[1], newp[2], N, fp64=True)
    pk = orc.power(d1.astype(np.float32), N, cfg.box)
    return {"density": delta, "scalar": u, "potential": phi, "parts": newp, "pk": pk["pk"], "cycles": rep.cycles}


def test_precision_form_errors_against_fp64_oracle(m, orc):
    parts = random_particles(NROW, N, seed=53, clustered=True, vscale=0.3)
    a, astep = 0.6, 0.01
    kw = dict(mg_model=1, fr_n=1, fr0=-1e-5, iter_count_max=4)
    plain = gpu_step(m, m.make_config(N, NROW, float(N), **kw), parts, a, astep)
    mixed = gpu_step(m, m.make_config(N, NROW, float(N), precision=m.PREC_MIXED, **kw), parts, a, astep)
    ref = oracle_step_fp64(orc, m.make_config(N, NROW, float(N), **kw), parts, a, astep)

    # CIC and FFT are the plain kernels in both forms
    assert np.array_equal(mixed["density"], plain["density"])
    assert rel_err(mixed["density"], ref["density"]) < 1e-6
    assert mixed["cycles"] == plain["cycles"] == ref["cycles"]
    # the first cycle's residual is far above the FP32 storage floor and agrees
    # closely; later cycles sit near that floor (c~^2/dx^2 times the rounding of
    # u^2), where rounding differences of the smoother move it by a few per cent
    rm, rp = mixed["residual"], plain["residual"]
    assert abs(rm[0] - rp[0]) <= 1e-2 * rp[0], (rm, rp)
    assert all(x <= 1.25 * y for x, y in zip(rm, rp)), (rm, rp)
    errs = {}
    for path, out in (("plain", plain), ("mixed", mixed)):
        e = {"scalar": rel_err(out["scalar"], ref["scalar"]),
             "potential": rel_err(out["potential"], ref["potential"]),
             "positions": max(float(np.max(np.abs(np.asarray(g, np.float64) - np.asarray(r, np.float64))))
                              for g, r in zip(out["parts"][:3], ref["parts"][:3])),
             "pk": float(np.max(np.abs(out["pk"][:N // 4] / ref["pk"][:N // 4] - 1.0)))}
        errs[path] = e
    # the bars of the plain path's single-step parity, for both forms
    for path in ("plain", "mixed"):
        assert errs[path]["scalar"] < 1e-5, errs
        assert errs[path]["potential"] < 1e-5, errs
        assert errs[path]["positions"] < 1e-3, errs       # grid units
        assert errs[path]["pk"] < 1e-4, errs              # k < k_Nyq / 2
    assert rel_err(mixed["scalar"], plain["scalar"]) < 1e-5


@pytest.mark.parametrize("frn,fr0", [(0, -1e-5), (2, -1e-6)])
def test_precision_form_fr_n0_n2_close_to_plain(m, frn, fr0):
    """f(R) n = 0 (FP32 quadratic root, cancellation-free form) and n = 2 (FP32
    Newton on the quartic): within 1e-4 of the plain path, same cycle counts."""
    parts = random_particles(NROW, N, seed=59, clustered=True)
    outs, cycles = [], []
    for prec in (m.PREC_PLAIN, m.PREC_MIXED):
        box = m.Box(m.make_config(N, NROW, float(N), fr_n=frn, fr0=fr0, precision=prec, iter_count_max=3))
        box.upload_particles(*parts)
        box.set_time(0.7, 0.01)
        box.density()
        cycles.append(box.scalar_field(1).cycles)
        outs.append(box.download_grid(m.GRID_FI2))
        box.close()
    assert cycles[0] == cycles[1]
    assert np.isfinite(outs[1]).all()
    assert rel_err(outs[1], outs[0]) < 1e-4, rel_err(outs[1], outs[0])
    assert not np.array_equal(outs[0], outs[1])   # the precision form did run


@pytest.mark.parametrize("model", [2, 3, 4, 5])
def test_precision_form_other_models_close_to_plain(m, model):
    """nDGP, symmetron, k-mouflage and csf sweeps, residuals and right-hand sides in
    FP32 (fused / marching kernels at 128^3): the solve stays within 1e-4 of the plain
    path's and takes the same cycles."""
    parts = random_particles(NROW, N, seed=71, clustered=True)
    tab = None
    if model in (4, 5):
        tab, _ = m.background_table(m.make_config(N, NROW, float(N), mg_model=model))
    outs, cycles = [], []
    for prec in (m.PREC_PLAIN, m.PREC_MIXED):
        cfg = m.make_config(N, NROW, float(N), mg_model=model, precision=prec, iter_count_max=3)
        box = m.Box(cfg)
        if tab is not None:
            box.set_background(tab)
        box.upload_particles(*parts)
        box.set_time(0.7, 0.01)
        box.density()
        rep = box.scalar_field(1)
        cycles.append(rep.cycles)
        outs.append(box.download_grid(m.GRID_FI2))
        box.close()
    assert cycles[0] == cycles[1]
    assert np.isfinite(outs[1]).all()
    assert rel_err(outs[1], outs[0]) < 1e-4, rel_err(outs[1], outs[0])
    assert not np.array_equal(outs[0], outs[1])   # the precision form did run
