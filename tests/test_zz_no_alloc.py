"""The neighbour-list entry point that allocates nothing.

cr_neighbor_list_noalloc is for callers that cannot allocate device memory
themselves (a host framework that hands out only fixed, pre-sized buffers, or
code that must not call cudaMalloc/cudaFree because those synchronise the
device and are refused during stream capture).  It must build the same list as
the context's own cr_calc_neighbor_list, from device buffers the caller owns.
This file is collected last so that a run stopping at the first failure has
already run every other test; it also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from cudaring_b200 import DPM2D, _lib, synth

pytestmark = pytest.mark.gpu

MAX_VERTICES = 65536  # CR_NOALLOC_MAX_VERTICES in include/cudaring.h


def _rows(nbr_slot_major, cnt, nv, width):
    """Reference layout: ascending neighbour ids per vertex, -1 padded to width."""
    out = np.full((nv, width), -1, dtype=np.int64)
    for v in range(nv):
        row = np.sort(nbr_slot_major[np.arange(cnt[v]) * nv + v])
        out[v, : len(row)] = row
    return out.reshape(-1)


CR_OK, CR_EINVAL, CR_ENBR_OVERFLOW = 0, 1, 6


def _context_build(rings, phi, seed=31):
    """The packing and the context's own list of it (the expected result)."""
    c = synth.workload_config("smooth_lj", rings)
    pk = synth.make_packing(c["nv"], c["a0"], c["calA0"], phi, seed=seed, placement="rsa")
    d = DPM2D.from_packing(pk, **{k: c[k] for k in ("potential", "interaction", "ea", "el", "eb", "ec", "LJcutoff")})
    cut = d.setDisplacementCutoff(0.5, 2 * pk.rad.mean())
    d.calcNeighborList(cut)
    ref = {"cnt": d.getMaxNeighborList(), "width": d.getNeighborListSize(), "rows": d.getNeighbors(), "cut": cut}
    d.close()
    return pk, ref


class _Inputs:
    """Caller-owned device buffers for one packing."""

    def __init__(self, pk, cap, dev):
        import torch

        self.nv = pk.num_vertices
        self.cap = cap
        self.pos = torch.tensor(pk.pos, dtype=torch.float64, device=dev)
        self.rad = torch.tensor(pk.rad, dtype=torch.float64, device=dev)
        self.ring_of = torch.tensor(np.repeat(np.arange(pk.num_particles), pk.nv_list), dtype=torch.int32, device=dev)
        self.nbr = torch.empty(cap * self.nv, dtype=torch.int32, device=dev)
        self.cnt = torch.empty(self.nv, dtype=torch.int32, device=dev)
        self.box = np.ascontiguousarray(pk.box, dtype=np.float64)
        self.max_rad = float(pk.rad.max())

    def call(self, cut, stream=None):
        import torch

        self.nbr.fill_(-7)
        self.cnt.fill_(-7)
        torch.cuda.synchronize()
        mc = C.c_long(-1)
        rc = _lib.lib().cr_neighbor_list_noalloc(self.pos.data_ptr(), self.rad.data_ptr(), self.ring_of.data_ptr(),
                                                 self.nv, self.box.ctypes.data, self.max_rad, cut, self.cap,
                                                 self.nbr.data_ptr(), self.cnt.data_ptr(), C.byref(mc), stream)
        return rc, mc.value, self.cnt.cpu().numpy().astype(np.int64)


@pytest.mark.parametrize("rings,phi", [(64, 0.40), (4, 0.30)])
def test_noalloc_matches_context_build_twice(cuda_device, rings, phi):
    pk, ref = _context_build(rings, phi)
    x = _Inputs(pk, 64, cuda_device)
    for _ in range(2):
        rc, mc, got_cnt = x.call(ref["cut"])
        assert rc == CR_OK
        assert mc == ref["cnt"].max()
        assert np.array_equal(got_cnt, ref["cnt"])
        assert np.array_equal(_rows(x.nbr.cpu().numpy().astype(np.int64), got_cnt, x.nv, ref["width"]), ref["rows"])


def test_noalloc_on_a_caller_stream(cuda_device):
    import torch

    pk, ref = _context_build(64, 0.40, seed=5)
    x = _Inputs(pk, 64, cuda_device)
    s = torch.cuda.Stream(device=cuda_device)
    for _ in range(2):
        rc, mc, got_cnt = x.call(ref["cut"], C.c_void_p(s.cuda_stream))
        assert rc == CR_OK and mc == ref["cnt"].max()
        assert np.array_equal(got_cnt, ref["cnt"])
        assert np.array_equal(_rows(x.nbr.cpu().numpy().astype(np.int64), got_cnt, x.nv, ref["width"]), ref["rows"])


def test_noalloc_overflow_keeps_complete_counts(cuda_device):
    pk, ref = _context_build(64, 0.40, seed=9)
    top = int(ref["cnt"].max())
    assert top >= 2
    x = _Inputs(pk, top - 1, cuda_device)
    rc, mc, got_cnt = x.call(ref["cut"])
    assert rc == CR_ENBR_OVERFLOW
    assert mc == top
    assert np.array_equal(got_cnt, ref["cnt"])
    # a capacity that fits again gives the full list on the next call
    x2 = _Inputs(pk, top, cuda_device)
    rc, mc, got_cnt = x2.call(ref["cut"])
    assert rc == CR_OK and mc == top
    assert np.array_equal(_rows(x2.nbr.cpu().numpy().astype(np.int64), got_cnt, x2.nv, ref["width"]), ref["rows"])


def test_noalloc_coarsens_a_dilute_grid(cuda_device):
    """A dilute box needs more cells than the scratch array holds; the grid is
    coarsened and the list stays the context's."""
    pk, ref = _context_build(16, 0.0005, seed=13)
    cmin = (1.0 + ref["cut"]) * 2.0 * float(pk.rad.max())
    assert (pk.box[0] // cmin) * (pk.box[1] // cmin) > 65536  # CR_NOALLOC_MAX_CELLS
    x = _Inputs(pk, 64, cuda_device)
    rc, mc, got_cnt = x.call(ref["cut"])
    assert rc == CR_OK
    assert mc == ref["cnt"].max()
    assert np.array_equal(got_cnt, ref["cnt"])
    assert np.array_equal(_rows(x.nbr.cpu().numpy().astype(np.int64), got_cnt, x.nv, ref["width"]), ref["rows"])


def test_noalloc_rejects_sizes_beyond_its_scratch(cuda_device):
    import torch

    small = torch.zeros(16, dtype=torch.float64, device=cuda_device)
    ints = torch.zeros(16, dtype=torch.int32, device=cuda_device)
    box = np.array([10.0, 10.0])
    mc = C.c_long(0)
    rc = _lib.lib().cr_neighbor_list_noalloc(small.data_ptr(), small.data_ptr(), ints.data_ptr(), MAX_VERTICES + 1,
                                             box.ctypes.data, 0.1, 1.5, 8, ints.data_ptr(), ints.data_ptr(),
                                             C.byref(mc), None)
    assert rc == CR_EINVAL  # before any buffer is touched
