"""The one-launch neighbour-list build in both of its forms.

Cell buckets: every vertex takes a slot of its cell's 16-entry bucket by an
atomic, then after one grid barrier the stencil search sorts each stencil
cell's ids and gathers their data by id.  Cell sort: when a cell holds more
than 16 vertices, the same launch falls back to the counting sort by cell
(scan, scatter, rank) before the search.  Both give the list of the
multi-kernel build, entry for entry (stencil order, ascending id inside a
cell), and the reference's sets (the oracle's O(Nv^2) scan).  The two count
arrays of the bucket form alternate between builds, so builds are run in
sequences that mix the two forms, with positions moved between them.
"""
import numpy as np
import pytest

import oracle
from cudaring_b200 import DPM2D, synth

pytestmark = pytest.mark.gpu

# cut distances (Lennard-Jones cutoff 2.5 + 0.5 or + 3.5): on the packing below
# every cell within its bucket at the first, up to 20 vertices in a cell at the second
SPARSE, DENSE = 3.0, 6.0


def _context(pk, c, spin_limit=None):
    d = DPM2D.from_packing(pk, **{k: c[k] for k in ("potential", "interaction", "ea", "el", "eb", "ec", "LJcutoff",
                                                      "dt")})
    if spin_limit is not None:
        # no polls: the first one-launch build gives up at its barrier and the
        # context builds with the multi-kernel path from then on
        d.setSpinLimit(spin_limit)
    return d


def _max_cell_occupancy(pk, cut):
    """Largest cell count of the grid the context picks for `cut` (cells no
    smaller than (1 + cut) * 2 * max radius; no coarsening below one full
    GPU of build CTAs)."""
    cmin = (1.0 + cut) * 2.0 * pk.rad.max() * (1.0 + 1e-9)
    ncx, ncy = int(np.floor(pk.box[0] / cmin)), int(np.floor(pk.box[1] / cmin))
    x = pk.pos.reshape(-1, 2)
    w = x - pk.box * np.floor(x / pk.box)
    cx = np.clip((w[:, 0] * (ncx / pk.box[0])).astype(int), 0, ncx - 1)
    cy = np.clip((w[:, 1] * (ncy / pk.box[1])).astype(int), 0, ncy - 1)
    return np.bincount(cy * ncx + cx).max(), ncx, ncy


@pytest.fixture(scope="module")
def packing(cuda_device):
    # 192 smooth-LJ rings (7,392 vertices) at phi 0.40
    c = synth.workload_config("smooth_lj", 192)
    pk = synth.make_packing(c["nv"], c["a0"], c["calA0"], 0.40, seed=23, placement="rsa")
    pk.vel = np.repeat(np.random.default_rng(8).normal(0.0, 0.05, size=(192, 2)), pk.nv_list, axis=0).reshape(-1)
    return pk, c


def _lists(d):
    n = d.getNeighborListSize()
    return d.getNeighbors().reshape(d.numVertices, n), d.getMaxNeighborList()


def test_cut_distances_reach_both_forms(packing):
    pk, _ = packing
    occ_sparse, nx, ny = _max_cell_occupancy(pk, SPARSE)
    assert nx >= 3 and ny >= 3 and occ_sparse <= 16
    occ_dense, nx, ny = _max_cell_occupancy(pk, DENSE)
    assert nx >= 3 and ny >= 3 and occ_dense > 16


def test_builds_match_multi_kernel_build_and_oracle(packing):
    pk, c = packing
    d = _context(pk, c)
    ref = _context(pk, c, spin_limit=-1)
    S = oracle.System(pk.nv_list, pk.box, c["potential"], c["interaction"], c["ea"], c["el"], c["eb"], c["ec"],
                      lj_cutoff=c["LJcutoff"])
    for x in (d, ref):
        # rebuilds inside NVELoop at cut distance 3.0, once a vertex moved a mean radius
        x.setDisplacementCutoff(0.5, 2.0 * x.getMeanVertexRadius())
        x.calcNeighborList(SPARSE)
        x.resetLastPositions()
        x.initNVE(0.0, readState=True)
    assert ref.getDegraded() and not d.getDegraded()
    for cut in [SPARSE, SPARSE, DENSE, SPARSE, DENSE, DENSE, SPARSE, SPARSE, SPARSE]:
        d.calcNeighborList(cut)
        ref.calcNeighborList(cut)
        assert not d.getDegraded()
        nb, cnt = _lists(d)
        nb_r, cnt_r = _lists(ref)
        assert d.getNeighborListSize() == ref.getNeighborListSize()
        assert np.array_equal(cnt, cnt_r)
        assert np.array_equal(nb, nb_r)  # same entries in the same order
        x = d.getVertexPositions()
        onb, ocnt, _ = S.neighbor_list(x, pk.rad, cut)
        assert np.array_equal(cnt, ocnt)
        olist = onb.reshape(d.numVertices, -1)
        for v in range(0, d.numVertices, 97):
            assert set(nb[v, :cnt[v]]) == set(olist[v, :ocnt[v]])
        # move the rings a little between builds (same trajectory on both:
        # the lists are equal, so are the forces)
        d.NVELoop(25)
        ref.NVELoop(25)
        assert np.max(np.abs(d.getVertexPositions() - ref.getVertexPositions())) < 1e-9
    d.close()
    ref.close()


def test_step_sequences_rebuild_through_both_forms(packing):
    # rebuilds inside NVELoop use the early-exit one-launch build; with the
    # dense cut every rebuild takes the cell-sort form, with the sparse one
    # the bucket form; a context that never used the one-launch build agrees
    pk, c = packing
    for cutoff in (SPARSE - 2.5, DENSE - 2.5):
        d = _context(pk, c)
        ref = _context(pk, c, spin_limit=-1)
        for x in (d, ref):
            # rebuild once a vertex has moved 0.02 mean radii
            cut = x.setDisplacementCutoff(cutoff, 0.02 * x.getMeanVertexRadius())
            assert cut == pytest.approx(cutoff + 2.5)
            x.calcNeighborList(cut)
            x.resetLastPositions()
            x.initNVE(0.0, readState=True)
        assert ref.getDegraded() and not d.getDegraded()
        d.NVELoop(300)
        ref.NVELoop(300)
        assert d.getUpdateCount() == ref.getUpdateCount() and d.getUpdateCount() >= 3
        assert np.max(np.abs(d.getVertexPositions() - ref.getVertexPositions())) < 1e-9
        nb, cnt = _lists(d)
        nb_r, cnt_r = _lists(ref)
        assert np.array_equal(cnt, cnt_r) and np.array_equal(nb, nb_r)
        d.close()
        ref.close()
