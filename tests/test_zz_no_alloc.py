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


@pytest.mark.parametrize("rings,phi", [(64, 0.40), (4, 0.30)])
def test_noalloc_matches_context_build_twice(cuda_device, rings, phi):
    import torch

    c = synth.workload_config("smooth_lj", rings)
    pk = synth.make_packing(c["nv"], c["a0"], c["calA0"], phi, seed=31, placement="rsa")
    d = DPM2D.from_packing(pk, **{k: c[k] for k in ("potential", "interaction", "ea", "el", "eb", "ec", "LJcutoff")})
    cut = d.setDisplacementCutoff(0.5, 2 * pk.rad.mean())
    d.calcNeighborList(cut)
    ref_cnt = d.getMaxNeighborList()
    width = d.getNeighborListSize()
    ref_rows = d.getNeighbors()
    d.close()

    nv = pk.num_vertices
    cap = 64
    dev = cuda_device
    pos = torch.tensor(pk.pos, dtype=torch.float64, device=dev)
    rad = torch.tensor(pk.rad, dtype=torch.float64, device=dev)
    ring_of = torch.tensor(np.repeat(np.arange(pk.num_particles), pk.nv_list), dtype=torch.int32, device=dev)
    nbr = torch.empty(cap * nv, dtype=torch.int32, device=dev)
    cnt = torch.empty(nv, dtype=torch.int32, device=dev)
    box = np.ascontiguousarray(pk.box, dtype=np.float64)
    L = _lib.lib()
    for _ in range(2):
        nbr.fill_(-7)
        cnt.fill_(-7)
        torch.cuda.synchronize()
        mc = C.c_long(-1)
        rc = L.cr_neighbor_list_noalloc(pos.data_ptr(), rad.data_ptr(), ring_of.data_ptr(), nv, box.ctypes.data,
                                        float(pk.rad.max()), cut, cap, nbr.data_ptr(), cnt.data_ptr(), C.byref(mc),
                                        None)
        assert rc == 0
        got_cnt = cnt.cpu().numpy().astype(np.int64)
        assert mc.value == ref_cnt.max()
        assert np.array_equal(got_cnt, ref_cnt)
        assert np.array_equal(_rows(nbr.cpu().numpy().astype(np.int64), got_cnt, nv, width), ref_rows)


def test_noalloc_rejects_sizes_beyond_its_scratch(cuda_device):
    import torch

    small = torch.zeros(16, dtype=torch.float64, device=cuda_device)
    ints = torch.zeros(16, dtype=torch.int32, device=cuda_device)
    box = np.array([10.0, 10.0])
    mc = C.c_long(0)
    rc = _lib.lib().cr_neighbor_list_noalloc(small.data_ptr(), small.data_ptr(), ints.data_ptr(), MAX_VERTICES + 1,
                                             box.ctypes.data, 0.1, 1.5, 8, ints.data_ptr(), ints.data_ptr(),
                                             C.byref(mc), None)
    assert rc == 1  # CR_EINVAL, before any buffer is touched
