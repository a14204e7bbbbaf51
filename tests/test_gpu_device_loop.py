"""The multigrid exit test on the device against the host loop.

A context's first solve, and every solve while per-kernel profiling is on, runs
the cycles eagerly and tests for the exit (PMP2extradof.f90:107-121) on the
host after each cycle.  Later solves run as one CUDA graph: a while node whose
body is a cycle, the level-0 residual norm and the exit test on the device.
Both must give the same residuals, cycle counts and exit reasons bit for bit,
and the same particles, for each exit reason: the residual target (1),
stagnation (2) and the cycle limit (3); on the 64^3 mesh (level-0 norm by the
plain residual kernel) and the 128^3 mesh (by the marching operator).  With
iter_count_max above 1024 the cycle graph is replayed under the host loop
instead, with the same results.

mgg_step waits for the device once, at its end, and mgg_run_steps once per run
(its steps queued as CUDA graphs, each solve a while node): both equal
mgg_step called step by step, bit for bit.  A step that fails (here a
particle outside [1, NGRID+1), which the density flags) leaves the particles
and the step state as they were.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

A0 = 0.05


@pytest.fixture(scope="module")
def m():
    import mgglam_b200
    return mgglam_b200


def run_steps(m, cfg, steps, profile):
    astep0 = m.astep_for_nsteps(A0, 40)
    b = m.Box(cfg)
    try:
        b.make_ics(seed=3, aexpn=A0, astep=astep0)
        if profile:
            b.profile(True)
        st = b.new_state(A0, astep0)
        reps = []
        for _ in range(steps):
            b.step(st)
            r = st.report
            reps.append((r.cycles, r.exit_reason, np.array(r.residual[:64], np.float64), st.ekin))
        return reps, b.download_particles(), (st.aexpn, st.astep, st.istep)
    finally:
        b.close()


CASES = {   # name: (ngrid, nrow, config)
    "limit": (64, 32, dict(iter_count_max=3, res_conv=1e-12)),
    "stagnation": (64, 32, dict(iter_count_max=40, res_conv=1e-12)),
    "target": (64, 32, dict(iter_count_max=8, res_conv=1.0)),
    "W_128": (128, 64, dict(iter_count_max=6, res_conv=1e-12, cycle="W")),
    "F_128_mixed": (128, 64, dict(iter_count_max=40, res_conv=1e-12, cycle="F", precision=1)),
    "dgp_128": (128, 64, dict(mg_model=2, iter_count_max=40, res_conv=1e-12)),
    # above the device loop's limit: the cycle graph replayed under the host loop
    "host_loop_graph": (64, 32, dict(iter_count_max=1500, res_conv=1e-12)),
}


@pytest.mark.parametrize("case", list(CASES))
def test_device_exit_test_equals_host_loop(m, case):
    ngrid, nrow, extra = CASES[case]
    kw = dict(mg_model=1, fr_n=1)
    kw.update(extra)
    cfg = m.make_config(ngrid, nrow, float(ngrid), **kw)
    host, ph, sh = run_steps(m, cfg, 4, profile=True)
    dev, pd, sd = run_steps(m, cfg, 4, profile=False)
    print(f"{case}: cycles {[r[0] for r in dev]}, exit reasons {[r[1] for r in dev]}")
    for (hc, hr, hres, he), (dc, dr, dres, de) in zip(host, dev):
        assert (dc, dr) == (hc, hr)
        assert np.array_equal(dres.view(np.uint64), hres.view(np.uint64))
        assert de == he
    assert sd == sh
    assert all(np.array_equal(a.view(np.uint32), b.view(np.uint32)) for a, b in zip(pd, ph))
    reasons = {r[1] for r in dev}
    expect = {"limit": 3, "stagnation": 2, "target": 1}.get(case)
    if expect is not None:
        assert expect in reasons, reasons


def test_failed_step_leaves_particles_and_state(m):
    cfg = m.make_config(64, 32, 64.0, mg_model=1, fr_n=1, iter_count_max=3)
    astep0 = m.astep_for_nsteps(A0, 40)
    b = m.Box(cfg)
    try:
        b.make_ics(seed=4, aexpn=A0, astep=astep0)
        st = b.new_state(A0, astep0)
        b.step(st)                      # the first, eager solve
        b.step(st)                      # a graphed solve: the device loop is live
        parts = [a.copy() for a in b.download_particles()]
        bad = [a.copy() for a in parts]
        bad[0][17] = np.float32(64 + 5.0)   # outside [1, NGRID+1): clamped and flagged
        b.upload_particles(*bad)
        before = (st.aexpn, st.astep, st.istep, st.ekin)
        with pytest.raises(m.MGGError) as e:
            b.step(st)
        assert e.value.code == 6   # MGG_ERR_NUMERIC
        assert (st.aexpn, st.astep, st.istep, st.ekin) == before
        after = b.download_particles()
        assert all(np.array_equal(a.view(np.uint32), c.view(np.uint32)) for a, c in zip(after, bad))
        # the flags are cleared: with the particle back inside, the box steps on
        b.upload_particles(*parts)
        b.step(st)
        assert st.istep == before[2] + 1
    finally:
        b.close()


RUNS = {   # name: (config, a0, astep0)
    "fr_V": (dict(mg_model=1, fr_n=1, iter_count_max=4), A0, None),
    "fr2_F_mixed": (dict(mg_model=1, fr_n=2, iter_count_max=6, cycle="F", precision=1), A0, None),
    "dgp_W": (dict(mg_model=2, iter_count_max=5, cycle="W"), A0, None),
    "sym_crossing_astar": (dict(mg_model=3, iter_count_max=4), 0.47, 0.01),   # a* = 0.5 inside the run
    "mg_off": (dict(mg_flag=0), A0, None),
}


@pytest.mark.parametrize("case", list(RUNS))
def test_run_steps_equals_step_by_step(m, case):
    """mgg_run_steps (all steps queued as graphs, one wait) against mgg_step called per step."""
    extra, a0, da0 = RUNS[case]
    cfg = m.make_config(64, 32, 64.0, **extra)
    da0 = da0 or m.astep_for_nsteps(a0, 40)
    nsteps = 7

    def fresh():
        b = m.Box(cfg)
        b.make_ics(seed=9, aexpn=a0, astep=da0)
        return b, b.new_state(a0, da0)

    a, sa = fresh()
    b, sb = fresh()
    try:
        ref = []
        for _ in range(nsteps + 1):
            a.step(sa)
            r = sa.report
            ref.append((r.cycles, r.exit_reason, np.array(r.residual[:64]), sa.ekin))
        b.step(sb)                                   # the first, tuning step on its own
        reps, ek = b.run_steps(sb, nsteps)
        got = [(sb.report.cycles, 0, None, None)] + [
            (r.cycles, r.exit_reason, np.array(r.residual[:64]), e) for r, e in zip(reps, ek)]
        for k in range(1, nsteps + 1):
            assert got[k][:2] == ref[k][:2], (k, got[k][:2], ref[k][:2])
            assert np.array_equal(got[k][2].view(np.uint64), ref[k][2].view(np.uint64)), k
            assert got[k][3] == ref[k][3], k
        assert (sb.aexpn, sb.astep, sb.istep, sb.ekin) == (sa.aexpn, sa.astep, sa.istep, sa.ekin)
        assert sb.report.cycles == sa.report.cycles and sb.report.exit_reason == sa.report.exit_reason
        pa, pb = a.download_particles(), b.download_particles()
        assert all(np.array_equal(x.view(np.uint32), y.view(np.uint32)) for x, y in zip(pa, pb))
        print(f"{case}: cycles {[g[0] for g in got[1:]]}")
        if case == "sym_crossing_astar":
            assert got[1][0] == 0 and got[-1][0] > 0   # no solve before a*, solves after it
    finally:
        a.close()
        b.close()


def test_failed_run_leaves_particles_and_state(m):
    cfg = m.make_config(64, 32, 64.0, mg_model=1, fr_n=1, iter_count_max=3)
    astep0 = m.astep_for_nsteps(A0, 40)
    b = m.Box(cfg)
    try:
        b.make_ics(seed=4, aexpn=A0, astep=astep0)
        st = b.new_state(A0, astep0)
        b.run_steps(st, 2)                 # the first step alone, the second graphed
        parts = [a.copy() for a in b.download_particles()]
        bad = [a.copy() for a in parts]
        bad[1][5] = np.float32(0.25)       # outside [1, NGRID+1): the first recorded step fails
        b.upload_particles(*bad)
        before = (st.aexpn, st.astep, st.istep, st.ekin)
        with pytest.raises(m.MGGError) as e:
            b.run_steps(st, 5)
        assert e.value.code == 6   # MGG_ERR_NUMERIC
        assert (st.aexpn, st.astep, st.istep, st.ekin) == before
        after = b.download_particles()
        assert all(np.array_equal(x.view(np.uint32), y.view(np.uint32)) for x, y in zip(after, bad))
        b.upload_particles(*parts)
        reps, _ = b.run_steps(st, 3)
        assert st.istep == before[2] + 3 and all(r.cycles > 0 for r in reps)
    finally:
        b.close()


_COARSE_SCRIPT = r'''
import sys
import numpy as np
sys.path.insert(0, sys.argv[2])
import mgglam_b200 as m
out = {}
cases = [("fr1_V", dict(mg_model=1, fr_n=1), 0.05), ("fr0_W", dict(mg_model=1, fr_n=0, cycle="W"), 0.05),
         ("fr2_F", dict(mg_model=1, fr_n=2, cycle="F"), 0.05), ("dgp_V", dict(mg_model=2), 0.05),
         ("sym_W", dict(mg_model=3, cycle="W"), 0.6), ("kmf_F", dict(mg_model=4, cycle="F"), 0.05),
         ("csf_V", dict(mg_model=5), 0.05)]
for name, kw, a0 in cases:
    cfg = m.make_config(128, 32, 128.0, iter_count_max=4, **kw)
    tab = None
    if cfg.mg_model in (4, 5):
        tab, _ = m.background_table(cfg)
    b = m.Box(cfg)
    if tab is not None:
        b.set_background(tab)
    b.make_ics(seed=13, aexpn=a0, astep=0.002)
    st = b.new_state(a0, 0.002)
    res = []
    for _ in range(3):
        b.step(st)
        res.append(np.array(st.report.residual[:64]))
        res.append(np.array([st.report.cycles, st.report.exit_reason], np.float64))
    out[name + "_res"] = np.concatenate(res)
    out[name + "_x"] = np.concatenate(b.download_particles())
    out[name + "_u"] = b.download_grid(m.GRID_FI2)
    b.close()
np.savez(sys.argv[1], **out)
'''


def test_small_level_cycle_equals_separate_launches(tmp_path):
    """The cycle below 16^3 cells runs as one single-block launch (MGG_COARSE_N=0:
    as separate launches per level operation; 32: from 32^3 down).  Same per-cell
    code in the same order of passes: particles, scalar field, residuals and cycle
    counts after three steps are bit-identical for every model and cycle type."""
    import os
    import subprocess
    import sys
    from conftest import PKG
    script = tmp_path / "coarse.py"
    script.write_text(_COARSE_SCRIPT)
    out = {}
    for tag, env in (("off", {"MGG_COARSE_N": "0"}), ("16", {}), ("32", {"MGG_COARSE_N": "32"})):
        f = tmp_path / f"{tag}.npz"
        r = subprocess.run([sys.executable, str(script), str(f), PKG], env=dict(os.environ, **env),
                           capture_output=True, text=True, timeout=900)
        assert r.returncode == 0, r.stderr[-2000:]
        out[tag] = np.load(f)
    for tag in ("16", "32"):
        for key in out["off"].files:
            a, b = out[tag][key], out["off"][key]
            assert np.array_equal(a.view(np.uint8), b.view(np.uint8)), (tag, key)
