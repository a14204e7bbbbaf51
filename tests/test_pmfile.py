"""PM snapshot files in the reference's format (WriteDataPM / ReadDataPM,
PMP2mod_tools.f90:237-487): byte layout checked against an independent
big-endian encoding with Python's struct, then a write/read round trip.
No GPU needed."""
import struct

import numpy as np
import pytest

from conftest import random_particles

HDR_FMT = ">45s4fi7f4i3fq100f"   # HEADER, AEXPN..ASTEP, ISTEP, PARTW..AEU0, NROW..Nseed, Om..hubble, Nparticles, extras


@pytest.fixture(scope="module")
def m():
    import mgglam_b200
    return mgglam_b200


def test_header_record_layout(m, tmp_path):
    cfg = m.make_config(64, 32, 100.0)
    h = m.pm_header(cfg, 0.5, 0.01, 17, 0.02, ekin=1.25, title="test snapshot", nrealization=3, nseed=9)
    parts = random_particles(32, 64, seed=1)
    m.pm_write(str(tmp_path), 17, h, parts)
    raw = (tmp_path / "PMcrd.0017.DAT").read_bytes()
    assert struct.calcsize(HDR_FMT) == 529
    assert len(raw) == 529 + 8
    assert struct.unpack(">i", raw[:4])[0] == 529 and struct.unpack(">i", raw[-4:])[0] == 529
    f = struct.unpack(HDR_FMT, raw[4:-4])
    assert f[0].rstrip() == b"test snapshot"
    assert f[1:5] == (np.float32(0.5), np.float32(0.02), 0.0, np.float32(0.01))
    assert f[5] == 17
    assert f[6] == np.float32(64.0 ** 3 / 32 ** 3) and f[8] == np.float32(1.25)
    assert f[13:17] == (32, 64, 3, 9)
    assert f[17:20] == (np.float32(cfg.om), np.float32(cfg.oml), np.float32(0.6774))
    assert f[20] == 32 ** 3
    assert f[21 + 99] == np.float32(100.0)


def test_particle_records_and_round_trip(m, tmp_path):
    # two records: 1024^2 particles and a partial one
    n = 1024 ** 2 + 4096
    rng = np.random.default_rng(3)
    parts = [(1.0 + rng.random(n) * 128).astype(np.float32) for _ in range(3)] + \
            [rng.standard_normal(n).astype(np.float32) for _ in range(3)]
    cfg = m.make_config(128, 64, 128.0)
    h = m.pm_header(cfg, 0.3, 0.01, 5, 0.02)
    h.nparticles = n
    m.pm_write(str(tmp_path), -1, h, parts)
    raw = (tmp_path / "PMcrs0.DAT").read_bytes()
    rec = 6 * 1024 ** 2 * 4
    assert len(raw) == 2 * rec                      # the partial record is written at full length
    x0 = np.frombuffer(raw[:4 * 1024 ** 2], dtype=">f4")
    assert np.array_equal(x0, parts[0][:1024 ** 2])
    vz1 = np.frombuffer(raw[rec + 5 * 4 * 1024 ** 2: rec + 5 * 4 * 1024 ** 2 + 4 * 4096], dtype=">f4")
    assert np.array_equal(vz1, parts[5][1024 ** 2:])
    h2, back = m.pm_read(str(tmp_path), -1)
    assert h2.nparticles == n and h2.ngrid == 128 and h2.istep == 5
    for a, b in zip(parts, back):
        assert np.array_equal(a, b)


def test_read_moves_coordinates_off_the_upper_edge(m, tmp_path):
    cfg = m.make_config(16, 8, 16.0)
    parts = random_particles(8, 16, seed=2)
    parts[0][0] = np.float32(17.0)       # INT(x) = NGRID + 1
    h = m.pm_header(cfg, 0.5, 0.01, 1, 0.02)
    m.pm_write(str(tmp_path), 1, h, parts)
    _, back = m.pm_read(str(tmp_path), 1)
    assert back[0][0] == np.float32(np.float32(17.0) - np.float32(1e-3))
    assert np.array_equal(back[0][1:], parts[0][1:])
