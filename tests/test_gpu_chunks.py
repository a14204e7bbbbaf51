"""The plane chunk of the marching kernels does not change any result.

The autotuner picks, per device and level size, how many planes one block of
the fused smoother, the marching sweeps, the coarse residual, the FAS
right-hand side and the level-1 restriction marches over.  Every cell gets the
same arithmetic whatever the chunk, so the fields must be bit-identical.  Each
case runs in a fresh process with MGG_CHUNK forcing one chunk for all tuned
kernels, and once with the tuner's own choice.
"""
import hashlib
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r'''
import sys, hashlib
sys.path.insert(0, "mg-glam-durham_b200"); sys.path.insert(0, "tests")
import numpy as np
import mgglam_b200 as m
from conftest import random_particles
parts = random_particles(128, 256, seed=13, clustered=True)
out = []
for model, prec in ((1, 0), (1, 1), (3, 1), (2, 1)):
    cfg = m.make_config(256, 128, 256.0, mg_model=model, precision=prec, iter_count_max=2)
    b = m.Box(cfg)
    b.upload_particles(*parts)
    b.set_time(0.7, 0.01)
    b.density()
    b.scalar_field(1)
    b.scalar_field(2)
    out.append(hashlib.md5(b.download_grid(m.GRID_FI2).tobytes()).hexdigest())
    b.close()
print(" ".join(out))
'''


def run(chunk):
    env = dict(os.environ)
    env.pop("MGG_CHUNK", None)
    if chunk:
        env["MGG_CHUNK"] = str(chunk)
    r = subprocess.run([sys.executable, "-c", SCRIPT], cwd=ROOT, env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return r.stdout.strip().split()[-4:]


def test_fields_identical_for_any_chunk():
    tuned = run(None)
    assert run(16) == tuned
    assert run(32) == tuned
