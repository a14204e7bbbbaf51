"""The multigrid exit test on the device against the host loop.

A context's first solve, and every solve while per-kernel profiling is on, runs
the cycles eagerly and tests for the exit (PMP2extradof.f90:107-121) on the
host after each cycle.  Later solves run as one CUDA graph: a while node whose
body is a cycle, the level-0 residual norm and the exit test on the device.
Both must give the same residuals, cycle counts and exit reasons bit for bit,
and the same particles, for each exit reason: the residual target (1),
stagnation (2) and the cycle limit (3); on the 64^3 mesh (level-0 norm by the
plain residual kernel) and the 128^3 mesh (by the marching operator).

mgg_step waits for the device once, at its end.  A step that fails (here a
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
