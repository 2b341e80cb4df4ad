"""irbc_bin_particles_noalloc: the binning for callers that cannot allocate
device memory while they run (allocator callbacks, memory-pool hooks,
fixed device-memory budgets).  Its scratch is a static device array shared
by all calls, so this test runs two calls in a row with different inputs
and checks each against irbc_bin_particles, which takes its scratch from
cudaMalloc, and the cells against a numpy restatement of the reference's
binning (Src/solfuncs.cpp:139-147), edge positions included.  The outputs
are integer cell indices, offsets and particle orders, compared exactly.
It also checks the entry point's defining property: after a first call
(which loads the kernels), further calls leave the device's free memory
unchanged.  Collected last so that a stop-at-first-failure run has already
run every other test."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _params(G, Lx, Ly, Lz):
    return G.default_params(Lx=Lx, Ly=Ly, Lz=Lz, Ns=0)


def _np_cells(L, x, y, z, r):
    """cindex cell of each particle in the shifted grid: bbound's wrap by
    repeated subtraction, floor, and cell 0 for indices outside the grid
    (x == Lx after the shift lands there)"""
    def bb(v, period):
        v = v.copy()
        while (v > period).any():
            v[v > period] -= period
        while (v < 0).any():
            v[v < 0] += period
        return v
    nx, ny, nz = int(L[0]), int(L[1]), int(L[2]) + 1
    fx = np.floor(bb(x - r[0], L[0])).astype(np.int64)
    fy = np.floor(bb(y - r[1], L[1])).astype(np.int64)
    fz = np.floor(z - r[2] + 1.0).astype(np.int64)
    ok = (fx >= 0) & (fx < nx) & (fy >= 0) & (fy < ny) & (fz >= 0) & (fz < nz)
    return np.where(ok, (fx * ny + fy) * nz + fz, 0)


class _Buffers:
    """device arrays for one binning call, allocated before any call runs"""

    def __init__(self, pos, ncell):
        import torch
        n = pos.shape[1]
        self.n = n
        self.dev = [torch.tensor(pos[k], dtype=torch.float64, device="cuda") for k in range(3)]
        self.cell = torch.full((max(n, 1),), -7, dtype=torch.int32, device="cuda")
        self.start = torch.full((ncell + 1,), -7, dtype=torch.int32, device="cuda")
        self.order = torch.full((max(n, 1),), -7, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()

    def call(self, fn, p, r):
        return fn(C.byref(p), self.dev[0].data_ptr(), self.dev[1].data_ptr(), self.dev[2].data_ptr(), self.n,
                  r[0], r[1], r[2], self.cell.data_ptr(), self.start.data_ptr(), self.order.data_ptr())

    def out(self):
        return self.cell.cpu().numpy()[:self.n], self.start.cpu().numpy(), self.order.cpu().numpy()[:self.n]


def _positions(L, n, seed):
    rng = np.random.default_rng(seed)
    pos = np.stack([rng.uniform(0, L[0], n), rng.uniform(0, L[1], n), rng.uniform(0, L[2], n)])
    # edge positions: x == Lx (cell 0 after the shift), x just below Lx, a
    # denormal, the top wall z == Lz and the layer just below it, y == 0
    pos[0, :6] = [0.0, L[0], L[0] - 1e-8, 1e-300, 0.5 * L[0], 1.0]
    pos[2, :6] = [L[2], L[2] - 1e-9, 0.0, L[2], 1e-12, L[2] - 0.999]
    pos[1, :6] = [0.0, L[1], 1e-300, L[1] - 1e-9, 0.0, 0.5 * L[1]]
    return pos


def test_noalloc_binning_matches_allocating_binning_twice():
    import torch
    import irbc_b200 as G
    lib = G.lib()
    cases = [((60.0, 40.0, 40.0), 300000, (0.31, 0.77, 0.05), 1),
             ((32.0, 24.0, 20.0), 120000, (0.9, 0.1, 0.999), 2)]
    for L, n, r, seed in cases:
        pos = _positions(L, n, seed)
        p = _params(G, *L)
        ncell = int(L[0]) * int(L[1]) * (int(L[2]) + 1)
        a, b = _Buffers(pos, ncell), _Buffers(pos, ncell)
        assert a.call(lib.irbc_bin_particles, p, r) == 0
        assert b.call(lib.irbc_bin_particles_noalloc, p, r) == 0
        ra, rb = a.out(), b.out()
        for x, y in zip(ra, rb):
            np.testing.assert_array_equal(x, y)
        want = _np_cells(L, pos[0], pos[1], pos[2], r)
        np.testing.assert_array_equal(rb[0], want)
        counts = np.bincount(want, minlength=ncell)
        np.testing.assert_array_equal(rb[1], np.concatenate([[0], np.cumsum(counts)]))
        np.testing.assert_array_equal(rb[2], np.argsort(want, kind="stable"))
        del a, b
        torch.cuda.synchronize()


def test_noalloc_binning_allocates_nothing_and_handles_no_particles():
    import torch
    import irbc_b200 as G
    lib = G.lib()
    L, r = (48.0, 32.0, 24.0), (0.4, 0.6, 0.2)
    p = _params(G, *L)
    ncell = int(L[0]) * int(L[1]) * (int(L[2]) + 1)
    full = _Buffers(_positions(L, 50000, 3), ncell)
    empty = _Buffers(np.zeros((3, 0)), ncell)
    # a first call loads the kernels (which may take device memory for
    # their code); from then on the free memory must not move
    assert full.call(lib.irbc_bin_particles_noalloc, p, r) == 0
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        assert full.call(lib.irbc_bin_particles_noalloc, p, r) == 0
        assert empty.call(lib.irbc_bin_particles_noalloc, p, r) == 0
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    # no particles: every start is 0, whatever the previous call left in
    # the shared counters
    np.testing.assert_array_equal(empty.out()[1], np.zeros(ncell + 1, np.int32))


def test_noalloc_binning_rejects_boxes_beyond_its_scratch():
    import irbc_b200 as G
    lib = G.lib()
    p = _params(G, 128.0, 128.0, 64.0)  # 1,064,960 cells > 1,048,576
    buf = _Buffers(np.zeros((3, 16)), 128 * 128 * 65)
    assert buf.call(lib.irbc_bin_particles_noalloc, p, (0.5, 0.5, 0.5)) == -4
