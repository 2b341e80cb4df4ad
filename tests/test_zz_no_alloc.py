"""irbc_bin_particles_noalloc: the binning for callers that cannot allocate
device memory while they run (allocator callbacks, memory-pool hooks,
fixed device-memory budgets).  Its scratch is a static device array shared
by all calls, so this test runs two calls in a row with different inputs
and checks each against irbc_bin_particles, which takes its scratch from
cudaMalloc.  The outputs are integer cell indices, offsets and particle
orders, compared exactly.  Collected last so that a stop-at-first-failure
run has already run every other test."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _params(G, Lx, Ly, Lz):
    return G.default_params(Lx=Lx, Ly=Ly, Lz=Lz, Ns=0)


def _run(G, fn, p, pos, r, ncell):
    import torch
    n = pos.shape[1]
    dev = [torch.tensor(pos[k], dtype=torch.float64, device="cuda") for k in range(3)]
    cell = torch.full((n,), -7, dtype=torch.int32, device="cuda")
    start = torch.full((ncell + 1,), -7, dtype=torch.int32, device="cuda")
    order = torch.full((n,), -7, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    rc = fn(C.byref(p), dev[0].data_ptr(), dev[1].data_ptr(), dev[2].data_ptr(), n, r[0], r[1], r[2],
            cell.data_ptr(), start.data_ptr(), order.data_ptr())
    return rc, cell.cpu().numpy(), start.cpu().numpy(), order.cpu().numpy()


def test_noalloc_binning_matches_allocating_binning_twice():
    import irbc_b200 as G
    L = G.lib()
    cases = [((60.0, 40.0, 40.0), 300000, (0.31, 0.77, 0.05), 1),
             ((32.0, 24.0, 20.0), 120000, (0.9, 0.1, 0.5), 2)]
    for (Lx, Ly, Lz), n, r, seed in cases:
        rng = np.random.default_rng(seed)
        pos = np.stack([rng.uniform(0, Lx, n), rng.uniform(0, Ly, n), rng.uniform(0, Lz, n)])
        p = _params(G, Lx, Ly, Lz)
        ncell = int(Lx) * int(Ly) * (int(Lz) + 1)
        ra = _run(G, L.irbc_bin_particles, p, pos, r, ncell)
        rb = _run(G, L.irbc_bin_particles_noalloc, p, pos, r, ncell)
        assert ra[0] == 0 and rb[0] == 0
        for a, b in zip(ra[1:], rb[1:]):
            np.testing.assert_array_equal(a, b)
        assert rb[2][-1] == n and (np.diff(rb[2]) >= 0).all()


def test_noalloc_binning_rejects_boxes_beyond_its_scratch():
    import irbc_b200 as G
    L = G.lib()
    p = _params(G, 128.0, 128.0, 64.0)  # 1,064,960 cells > 1,048,576
    pos = np.zeros((3, 16))
    rc = _run(G, L.irbc_bin_particles_noalloc, p, pos, (0.5, 0.5, 0.5), 128 * 128 * 65)[0]
    assert rc == -4
