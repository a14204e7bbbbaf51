"""mgg_density_noalloc: the CIC density for callers that cannot allocate.

Some hosts cannot call cudaMalloc: their device memory all comes from their
own pool or arena, or they must not allocate (and possibly synchronise the
device) in the middle of their work.  mgg_density_noalloc takes the caller's
device arrays and keeps its scratch in one fixed device array inside the
library.  This file checks, through the C ABI, that it gives the same grid as
mgg_density -- the tolerance of the density tests, and in fact bit-identical,
since both accumulate the CIC weights as integers -- on two calls in a row with
different particle sets and grid sizes, so the second call cannot lean on what
the first left in the shared scratch.  It is named to run after every other
test file and needs no state from them.
"""
import numpy as np
import pytest

from conftest import random_particles

pytestmark = pytest.mark.gpu


def test_density_noalloc_matches_density_on_two_calls():
    import torch

    import mgglam_b200 as m

    cases = [(64, 32, 41, True), (32, 24, 43, False)]   # (NGRID, NROW, seed, clustered)
    for ngrid, nrow, seed, clustered in cases:
        parts = random_particles(nrow, ngrid, seed=seed, clustered=clustered)
        cfg = m.make_config(ngrid, nrow, float(ngrid), mg_flag=0)
        box = m.Box(cfg)
        box.upload_particles(*parts)
        box.set_time(0.5, 0.01)
        box.density()
        ref = box.download_grid(m.GRID_FI)
        box.close()

        dev = torch.device("cuda", cfg.device)
        with torch.cuda.device(dev):
            x, y, z = (torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(dev) for a in parts[:3])
            fi = torch.full((ngrid ** 3,), float("nan"), dtype=torch.float32, device=dev)
            torch.cuda.synchronize(dev)
            m.density_noalloc(x.data_ptr(), y.data_ptr(), z.data_ptr(), x.numel(), ngrid, fi.data_ptr())
            got = fi.cpu().numpy()

        assert np.isfinite(got).all()
        assert np.max(np.abs(got - ref) / (1.0 + np.abs(ref))) < 1e-5
        assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


def test_density_noalloc_rejects_sizes_beyond_its_scratch():
    import mgglam_b200 as m

    with pytest.raises(m.MGGError) as e:
        m.density_noalloc(1, 1, 1, 1000, 512, 1)
    assert m.ERR_NAMES[e.value.code] == "ARG"
    with pytest.raises(m.MGGError) as e:
        m.density_noalloc(1, 1, 1, (1 << 21) + 1, 64, 1)
    assert m.ERR_NAMES[e.value.code] == "ARG"


def test_density_noalloc_refuses_a_capturing_stream():
    """The call waits for its own result on the host, which a stream under graph
    capture cannot do: it is refused with MGG_ERR_STATE before any work is queued,
    and the capture ends cleanly."""
    import torch

    import mgglam_b200 as m

    dev = torch.device("cuda", 0)
    x = torch.full((64,), 2.5, dtype=torch.float32, device=dev)
    fi = torch.zeros(16 ** 3, dtype=torch.float32, device=dev)
    s = torch.cuda.Stream(device=dev)
    g = torch.cuda.CUDAGraph()
    torch.cuda.synchronize(dev)
    err = None
    with torch.cuda.graph(g, stream=s):
        try:
            m.density_noalloc(x.data_ptr(), x.data_ptr(), x.data_ptr(), x.numel(), 16, fi.data_ptr(), s.cuda_stream)
        except m.MGGError as e:
            err = e
        fi.add_(1.0)   # the capture holds one node of its own
    assert err is not None and m.ERR_NAMES[err.code] == "STATE", err
    torch.cuda.synchronize(dev)
