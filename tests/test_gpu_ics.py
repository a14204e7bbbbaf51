"""The device initial-condition generator (mgg_make_ics) against the linear theory it
restates (PMP2start.f90:265-460, 797-873).

- P(k): the CIC density of the Zel'dovich particles, binned as GetPower(0) bins
  it, equals D(a0)^2 P_BBKS(k), times the squared CIC window of the mesh, bin by
  bin within cosmic variance (sigma_P / P = sqrt(2 / Nmodes), Nmodes counting +k
  and -k) for k below a quarter of the particle lattice's Nyquist frequency.
  P_BBKS is the BBKS transfer function with the Sugiyama shape parameter,
  A k^ns T(k)^2 normalised to sigma8 with a top-hat of 8 Mpc/h, restated here in
  numpy.  The same expectation is first checked on the CPU against the numpy
  Zel'dovich generator of the benchmark's CPU arm, so the expectation itself is
  pinned independently of the device code.
- Velocities: BLOCKS sets x = Q - XCONS GR + 0.5 and v = VCONS GR
  (PMP2start.f90:397-460), so v = -(VCONS/XCONS) d for the displacement d, with
  VCONS/XCONS = -(AEXPV/AEXPN) sqrt(AEXPV) sqrt(Om + OmL AEXPV^3) and
  AEXPV = AEXPN - ASTEP/2 (PMP2start.f90:826-837).
- Determinism: a seed gives bit-identical particles in two contexts, and the
  same white noise on a mesh twice as fine (the displacement in grid units
  doubles with NGRID at a fixed box).
"""
import numpy as np
import pytest

COSMO = dict(om=0.3089, oml=0.6911, omb=0.0486, hubble=0.6774, ns=0.9667, sigma8=0.8159)


def bbks_power():
    """P(k) = A k^ns T_BBKS(k)^2 [(Mpc/h)^3, k in h/Mpc], sigma8-normalised."""
    om, omb, h, ns, s8 = COSMO["om"], COSMO["omb"], COSMO["hubble"], COSMO["ns"], COSMO["sigma8"]
    gamma = om * h * np.exp(-omb * (1.0 + np.sqrt(2 * h) / om))

    def T(k):
        q = k / gamma
        return np.log(1 + 2.34 * q) / (2.34 * q) * (1 + 3.89 * q + (16.1 * q) ** 2 + (5.46 * q) ** 3
                                                    + (6.71 * q) ** 4) ** -0.25

    lk = np.linspace(np.log(1e-5), np.log(1e3), 20001)
    k = np.exp(lk)
    x = k * 8.0
    wt = 3 * (np.sin(x) - x * np.cos(x)) / x ** 3
    s2 = np.trapezoid(k ** 3 * k ** ns * T(k) ** 2 * wt ** 2, lk) / (2 * np.pi ** 2)
    amp = s8 ** 2 / s2
    return lambda kk: amp * kk ** ns * T(kk) ** 2


def growth(a):
    """Linear growth D(a) = 5 Om / 2 E(a) int_0^a da' / (a' E(a'))^3 (unnormalised)."""
    om, oml = COSMO["om"], COSMO["oml"]
    E = lambda x: np.sqrt(om / x ** 3 + oml + (1 - om - oml) / x ** 2)
    n = 200000
    xs = a * (np.arange(n) + 0.5) / n
    return 2.5 * om * E(a) * np.sum(1.0 / (xs * E(xs)) ** 3) * a / n


def expected_bins(ngrid, nrow, box, a):
    """Mode-averaged D^2 P(k) W_CIC(k)^2 per GetPower(0) bin I = 1..ngrid/2
    (MP = max(INT(RK + 0.5), 1), half-spectrum modes counted twice unless kx = 0 or ngrid/2)."""
    P = bbks_power()
    D = growth(a) / growth(1.0)
    f = np.fft.fftfreq(ngrid, 1.0 / ngrid)
    fr = np.arange(ngrid // 2 + 1)
    mz, my, mx = np.meshgrid(f, f, fr, indexing="ij")
    wk = np.sqrt(mx ** 2 + my ** 2 + mz ** 2)
    W = np.ones_like(wk)
    for mc in (mx, my, mz):
        W *= np.sinc(mc / ngrid) ** 2
    kk = 2 * np.pi * wk / box
    with np.errstate(divide="ignore", invalid="ignore"):
        pm = np.where((wk > 0) & (wk < nrow // 2), D ** 2 * P(kk), 0.0) * W ** 2
    mult = np.where((mx == 0) | (mx == ngrid // 2), 1.0, 2.0)
    I = np.maximum((wk.astype(np.float32) + np.float32(0.5)).astype(np.int64), 1)
    nb = ngrid // 2
    sel = (wk > 0) & (I <= nb)
    num = np.bincount(I[sel], weights=(pm * mult)[sel], minlength=nb + 1)
    cnt = np.bincount(I[sel], weights=mult[sel], minlength=nb + 1)
    return num[1:] / np.maximum(cnt[1:], 1), cnt[1:]


def check_spectrum(pk, nmodes, ngrid, nrow, box, a):
    """Bins I < nrow/4: every bin within 5 sigma of the expectation, reduced chi^2 < 3,
    and the mode-weighted mean ratio within 3 %.  Returns (ratios, pulls)."""
    exp, cnt = expected_bins(ngrid, nrow, box, a)
    nb = nrow // 4
    np.testing.assert_array_equal(nmodes[:nb], cnt[:nb])
    r = pk[:nb] / exp[:nb]
    sig = np.sqrt(2.0 / nmodes[:nb])
    pull = (r - 1.0) / sig
    assert np.all(np.abs(pull) < 5.0), (r, pull)
    assert float(np.mean(pull ** 2)) < 3.0, (r, pull)
    mean = float(np.sum(r * nmodes[:nb]) / np.sum(nmodes[:nb]))
    assert abs(mean - 1.0) < 0.03, (mean, r)
    return r, pull


def test_expected_spectrum_matches_the_cpu_generator(orc):
    """The expectation against the numpy Zel'dovich generator of the CPU arm (CPU only)."""
    import bench

    ngrid, nrow, box, a = 128, 64, 256.0, 0.05
    parts = bench.numpy_ics(nrow, ngrid, box, 3, a, 0.001)
    fi = orc.density(parts[0], parts[1], parts[2], ngrid)
    pk = orc.power(fi, ngrid, box)
    check_spectrum(pk["pk"], pk["nmodes"], ngrid, nrow, box, a)


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [42, 7])
def test_ics_spectrum_is_linear_theory(seed):
    import mgglam_b200 as m

    ngrid, nrow, box, a = 128, 64, 256.0, 0.05
    b = m.Box(m.make_config(ngrid, nrow, box, mg_flag=0))
    try:
        b.make_ics(seed=seed, aexpn=a, astep=0.001)
        pk = b.power(recompute_density=True)
    finally:
        b.close()
    r, pull = check_spectrum(pk["pk"], pk["nmodes"], ngrid, nrow, box, a)
    print(f"seed {seed}: P/P_lin per bin {np.round(r, 3).tolist()}")


@pytest.mark.gpu
def test_ics_velocity_is_the_zeldovich_factor_of_the_displacement():
    import mgglam_b200 as m

    ngrid, nrow, box, a, da = 64, 32, 128.0, 0.05, 0.004
    b = m.Box(m.make_config(ngrid, nrow, box, mg_flag=0))
    try:
        b.make_ics(seed=11, aexpn=a, astep=da)
        parts = b.download_particles()
    finally:
        b.close()
    f32 = np.float32
    aexpv = f32(f32(a) - f32(da) / f32(2.0))
    vfac = float(aexpv / f32(a)) * np.sqrt(float(aexpv)) * np.sqrt(float(f32(COSMO["om"]) + f32(COSMO["oml"]) * aexpv ** 3))
    lat = np.arange(nrow, dtype=np.float64)
    qk, qj, qi = np.meshgrid(lat, lat, lat, indexing="ij")
    qfact = ngrid / nrow
    for comp, q in enumerate((qi, qj, qk)):
        Q = (qfact * q + 1.0 + 0.5).ravel()
        d = parts[comp].astype(np.float64) - Q
        d = (d + ngrid / 2) % ngrid - ngrid / 2          # undo the periodic wrap
        v = parts[3 + comp].astype(np.float64)
        assert np.max(np.abs(d)) > 1e-3                   # the field is not empty
        # positions are stored in FP32: d carries the rounding of x ~ NGRID
        tol = 4 * np.spacing(np.float32(ngrid + 1)) * vfac + 1e-6 * np.max(np.abs(v))
        assert np.max(np.abs(v - vfac * d)) < tol, (comp, np.max(np.abs(v - vfac * d)), tol)


@pytest.mark.gpu
def test_ics_are_deterministic_per_seed():
    import mgglam_b200 as m

    def ics(ngrid, nrow, box, seed):
        b = m.Box(m.make_config(ngrid, nrow, box, mg_flag=0))
        try:
            b.make_ics(seed=seed, aexpn=0.05, astep=0.001)
            return b.download_particles()
        finally:
            b.close()

    p1 = ics(64, 32, 128.0, 5)
    p2 = ics(64, 32, 128.0, 5)
    for a, b in zip(p1, p2):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    p3 = ics(64, 32, 128.0, 6)
    assert not np.array_equal(p1[0], p3[0])
    # the same noise on a twice finer mesh of the same box: displacements double in grid units
    fine = ics(128, 32, 128.0, 5)
    lat = np.arange(32, dtype=np.float64)
    qk, qj, qi = np.meshgrid(lat, lat, lat, indexing="ij")
    for comp, q in enumerate((qi, qj, qk)):
        dc = p1[comp].astype(np.float64) - (2.0 * q + 1.5).ravel()
        dc = (dc + 32) % 64 - 32
        df = fine[comp].astype(np.float64) - (4.0 * q + 1.5).ravel()
        df = (df + 64) % 128 - 64
        assert np.max(np.abs(df - 2.0 * dc)) < 1e-4 * max(1.0, np.max(np.abs(df))) + 8 * np.spacing(np.float32(129))
