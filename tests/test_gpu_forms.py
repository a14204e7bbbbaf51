"""The forms beside the drop-in path: mgg_step, the batched form and the server.

Every kernel is deterministic and boxes share no device state, so the checks
are bit-identity: one mgg_step equals the routine-by-routine main-loop body;
a box advanced in a batch equals the same box advanced alone; a request served
in a mix with others (on a reused context) equals the same request run alone
on a fresh context.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

A0 = 0.05


@pytest.fixture(scope="module")
def m():
    import mgglam_b200
    return mgglam_b200


def box_with_ics(m, cfg, seed, astep0):
    """A box with its initial conditions (and, for k-mouflage / csf, its background table)."""
    tab = None
    if cfg.mg_flag == 1 and cfg.mg_model in (m.MODEL_KMOUFLAGE, m.MODEL_CSF):
        tab, _ = m.background_table(cfg)   # also sets the model's lambda in cfg
    b = m.Box(cfg)
    if tab is not None:
        b.set_background(tab)
    b.make_ics(seed=seed, aexpn=A0, astep=astep0)
    return b


def same_particles(a, b):
    return all(np.array_equal(x.view(np.uint32), y.view(np.uint32)) for x, y in zip(a, b))


def test_step_equals_routine_sequence(m):
    cfg = m.make_config(32, 16, 32.0, mg_model=1, fr_n=1, iter_count_max=3)
    astep0 = m.astep_for_nsteps(A0, 40)
    a = box_with_ics(m, cfg, 5, astep0)
    b = box_with_ics(m, cfg, 5, astep0)
    sa = a.start(A0, astep0)
    sb = b.new_state(A0, astep0)
    for i in range(1, 4):
        a.pm_step(sa, i)
        b.step(sb)
        assert sb.istep == i
        assert np.float32(sb.aexpn) == np.float32(sa.aexpn)
        assert sb.ekin == sa.ekin
        assert sb.report.cycles == sa.reports[-1].cycles
    assert same_particles(a.download_particles(), b.download_particles())
    a.close()
    b.close()


def test_batch_equals_single(m):
    astep0 = m.astep_for_nsteps(A0, 40)
    # f(R) with V, F and W cycles, the coupled scalar field and k-mouflage, both precision forms
    cfgs = [m.make_config(32, 16, 32.0, mg_model=1, fr_n=1, fr0=-1e-5, iter_count_max=3),
            m.make_config(32, 16, 32.0, mg_model=1, fr_n=2, fr0=-1e-6, iter_count_max=3),
            m.make_config(64, 32, 64.0, mg_model=1, fr_n=1, fr0=-1e-4, iter_count_max=3),
            m.make_config(32, 16, 32.0, mg_model=1, fr_n=1, fr0=-1e-5, iter_count_max=3, cycle="F"),
            m.make_config(64, 32, 64.0, mg_model=1, fr_n=1, fr0=-1e-5, iter_count_max=3, cycle="W",
                          precision=m.PREC_MIXED),
            m.make_config(32, 16, 32.0, mg_model=5, iter_count_max=3, cycle="W"),
            m.make_config(32, 16, 32.0, mg_model=4, iter_count_max=3, precision=m.PREC_MIXED)]
    seeds = [1, 2, 3, 4, 5, 6, 7]
    batch = [box_with_ics(m, c, s, astep0) for c, s in zip(cfgs, seeds)]
    states = [b.new_state(A0, astep0) for b in batch]
    for _ in range(3):
        m.step_batch(batch, states)
    for b, c, s, st in zip(batch, cfgs, seeds, states):
        alone = box_with_ics(m, c, s, astep0)
        sa = alone.new_state(A0, astep0)
        for _ in range(3):
            alone.step(sa)
        assert st.ekin == sa.ekin and st.istep == sa.istep == 3
        assert same_particles(b.download_particles(), alone.download_particles())
        alone.close()
        b.close()


def test_server_results_equal_alone(m):
    astep0 = m.astep_for_nsteps(A0, 40)
    reqs = [(m.make_config(32, 16, 32.0, mg_model=1, fr_n=1, iter_count_max=3), 11, 3),
            (m.make_config(64, 32, 64.0, mg_model=2, iter_count_max=3), 12, 2),
            (m.make_config(32, 16, 32.0, mg_model=3, iter_count_max=3), 13, 3),
            (m.make_config(32, 16, 32.0, mg_model=1, fr_n=2, iter_count_max=3), 14, 2),
            (m.make_config(32, 16, 32.0, mg_model=5, iter_count_max=3), 15, 2),
            (m.make_config(32, 16, 32.0, mg_model=1, fr_n=1, iter_count_max=3, cycle="F"), 16, 2),
            (m.make_config(32, 16, 32.0, mg_model=5, iter_count_max=3, cycle="W"), 17, 2),
            (m.make_config(32, 16, 32.0, mg_model=4, iter_count_max=3, cycle="W"), 18, 2)]
    srv = m.Server(hbm_budget_gb=8.0, max_active=3)
    ids = [srv.submit(c, s, A0, astep0, n) for c, s, n in reqs]
    got = [srv.wait(i, c.ngrid // 2) for i, (c, _, _) in zip(ids, reqs)]
    srv.close()
    for (c, s, n), (info, k, nm, pk) in zip(reqs, got):
        assert info.status == 0 and info.steps == n
        assert info.t_submit_ms <= info.t_admit_ms <= info.t_done_ms
        box = box_with_ics(m, c, s, astep0)
        st = box.new_state(A0, astep0)
        for _ in range(n):
            box.step(st)
        box.set_time(st.aexpn, st.astep)
        p = box.power(True)
        assert np.array_equal(p["k"], k) and np.array_equal(p["nmodes"], nm)
        assert np.array_equal(p["pk"], pk), (c.mg_model, np.max(np.abs(p["pk"] - pk)))
        assert info.ekin == st.ekin
        box.close()


def test_step_host_equals_upload_step_download(m):
    from conftest import random_particles
    cfg = m.make_config(32, 16, 32.0, mg_model=1, fr_n=1, iter_count_max=3)
    astep0 = m.astep_for_nsteps(A0, 40)
    parts = random_particles(16, 32, seed=8, vscale=0.3)
    a = m.Box(cfg)
    b = m.Box(cfg)
    sa, sb = a.new_state(A0, astep0), b.new_state(A0, astep0)
    host = [p.copy() for p in parts]
    for _ in range(2):
        b.step_host(sb, host)
    a.upload_particles(*parts)
    for _ in range(2):
        a.step(sa)
    assert sa.ekin == sb.ekin and np.float32(sa.aexpn) == np.float32(sb.aexpn)
    assert same_particles(a.download_particles(), host)
    a.close()
    b.close()


def test_step_host_pipelined_equals_step_host(m):
    """The pipelined host-array step (velocities downloaded behind the next step)
    gives the particles of the synchronous one, step after step, once synchronised."""
    import torch
    from conftest import random_particles
    cfg = m.make_config(64, 32, 64.0, mg_model=1, fr_n=1, iter_count_max=3)
    astep0 = m.astep_for_nsteps(A0, 40)
    parts = random_particles(32, 64, seed=9, vscale=0.3)
    a = m.Box(cfg)
    b = m.Box(cfg)
    sa, sb = a.new_state(A0, astep0), b.new_state(A0, astep0)
    ha = [p.copy() for p in parts]
    hb = [torch.from_numpy(p.copy()).pin_memory().numpy() for p in parts]   # page-locked, as a driver would
    for _ in range(3):
        a.step_host(sa, ha)
        b.step_host_pipelined(sb, hb)
    b.synchronize()
    assert sa.ekin == sb.ekin and np.float32(sa.aexpn) == np.float32(sb.aexpn)
    assert same_particles(ha, hb)
    assert same_particles(a.download_particles(), b.download_particles())
    a.close()
    b.close()


def test_server_small_request_passes_a_waiting_large_one(m):
    """Bounded bypass: with room for one 128^3 box and a little more, a second 128^3
    request waits for the first, and a 32^3 request that arrives after it starts
    while the first runs; every request completes."""
    import ctypes
    astep0 = m.astep_for_nsteps(A0, 40)
    big = m.make_config(128, 64, 128.0, mg_model=1, fr_n=1, iter_count_max=3)
    small = m.make_config(32, 16, 32.0, mg_model=1, fr_n=1, iter_count_max=3)
    lib = m.load_library()
    bb = lib.mgg_box_bytes(ctypes.byref(big))
    bs = lib.mgg_box_bytes(ctypes.byref(small))
    srv = m.Server(hbm_budget_gb=(bb + 2 * bs) / 1e9, max_active=3)
    ia = srv.submit(big, 21, A0, astep0, 6)
    ib = srv.submit(big, 22, A0, astep0, 2)
    ic = srv.submit(small, 23, A0, astep0, 2)
    a = srv.wait(ia, 64)[0]
    b = srv.wait(ib, 64)[0]
    c = srv.wait(ic, 16)[0]
    srv.close()
    assert a.status == b.status == c.status == 0
    assert b.t_admit_ms >= a.t_done_ms          # the second large request waited for memory
    assert c.t_admit_ms < a.t_done_ms           # the small one passed it
