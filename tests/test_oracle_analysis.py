"""The oracle's restatement of the analysis routines after the step (CPU only).

GetPower(1) (PMP2mod_power.f90:20-108) with DENSITrsd (PMP2mod_density.f90:
407-557) and DensDistr (PMP2mod_density.f90:1041-1126) have no golden vectors
in the reference; these known answers pin the restatement:
  * the quadrupole weight of a single Fourier mode along z is P2(1) = 1, along
    x P2(0) = -1/2, so P2/P0 = 2.5 and -1.25 after the (2L+1)/2 factor;
  * DENSITrsd(0) with Xscale = 1 is DENSIT;
  * with zero velocities the redshift-space monopole is the real-space P(k)
    and the quadrupole averaged over the three axes vanishes (sum of P2 over
    three orthogonal lines of sight is zero for every mode);
  * the PDF of a uniform grid is one bin, RMS 0, mean 1; bin edges follow
    floor(log10(1 + delta) / 0.001).
"""
import numpy as np
import pytest

from conftest import random_particles


def mode_grid(n, axis, m=3, amp=0.1):
    i, j, k = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    c = (i, j, k)[axis]
    f = (amp * np.cos(2 * np.pi * m * c / n)).astype(np.float32)
    return np.ascontiguousarray(np.transpose(f, (2, 1, 0))).reshape(-1)   # index i + n (j + n k)


@pytest.mark.parametrize("axis,ratio", [(2, 2.5), (0, -1.25), (1, -1.25)])
def test_quadrupole_of_single_modes(orc, axis, ratio):
    n = 32
    fi = mode_grid(n, axis)
    m = orc.power_pol(fi, n, 32.0, 0)
    q = orc.power_pol(fi, n, 32.0, 1)
    assert m["pk"][2] > 0
    assert q["pk"][2] / m["pk"][2] == pytest.approx(ratio, rel=1e-6)
    others = np.delete(np.arange(n // 2), 2)
    assert np.max(np.abs(m["pk"][others])) < 1e-12 * m["pk"][2]


def test_density_rsd_real_space_at_full_mesh_is_densit(orc):
    parts = random_particles(16, 32, seed=3, clustered=True)
    a = orc.density(parts[0], parts[1], parts[2], 32)
    b = orc.density_rsd(parts, 32, 32, 0, 0.5, 0.3089, 0.6911)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_power_rsd_without_velocities(orc):
    parts = random_particles(16, 64, seed=5, clustered=True, vscale=0.0)
    r = orc.power_rsd(parts, 64, 64.0, 0.5, 0.3089, 0.6911)
    assert r["preal"].shape == (16,)
    assert np.all(r["preal"] > 0)
    assert np.max(np.abs(r["p0"] / r["preal"] - 1.0)) < 1e-5
    assert np.max(np.abs(r["p2"])) < 1e-5 * np.max(r["preal"])


def test_power_rsd_velocities_change_the_quadrupole(orc):
    parts = random_particles(16, 64, seed=5, clustered=True, vscale=2.0)
    r = orc.power_rsd(parts, 64, 64.0, 0.5, 0.3089, 0.6911)
    assert np.max(np.abs(r["p2"])) > 1e-3 * np.max(r["preal"])


def test_pdf_uniform_grid(orc):
    nc, den, rms, mean = orc.density_pdf(np.zeros(16 ** 3, np.float32), 16)
    assert nc[2001] == 16 ** 3 and nc.sum() == 16 ** 3
    assert den[2001] == 16 ** 3
    assert rms == 0.0 and mean == 1.0


def test_pdf_bins_and_moments(orc):
    rng = np.random.default_rng(7)
    n = 16
    v = np.exp(rng.normal(0.0, 1.5, n ** 3)).astype(np.float32)          # 1 + delta, lognormal
    v[:5] = [0.0, 1e-4, 1e3, 1.0, 10.0]                                  # empty, both clamps, two edges
    fi = (v - np.float32(1.0)).astype(np.float32)
    nc, den, rms, mean = orc.density_pdf(fi, n)
    w = (fi + np.float32(1.0)).astype(np.float32)
    with np.errstate(divide="ignore"):
        l = np.log10(w.astype(np.float64)).astype(np.float32).astype(np.float64)
    idx = np.where(w > 0, np.clip(np.floor(l / 0.001), -2001, 2001), -2001).astype(int) + 2001
    assert np.array_equal(nc, np.bincount(idx, minlength=4003))
    assert np.allclose(den, np.bincount(idx, weights=w.astype(np.float64), minlength=4003), rtol=1e-13, atol=0)
    assert nc[0] >= 2 and nc[-1] >= 1 and nc[2001] >= 1 and nc[3001] >= 1
    assert mean == pytest.approx(w.astype(np.float64).mean(), rel=1e-12)
    assert rms == pytest.approx(np.sqrt((w * w).astype(np.float64).mean() - mean ** 2), rel=1e-9)
