"""Edge cases of the step path: a neighbour list that outgrows its capacity
inside a captured step sequence, rings with empty lists, the smallest rings
(three vertices), the largest ring a tile holds, and the inputs the context
rejects."""
import numpy as np
import pytest

import oracle
from cudaring_b200 import DPM2D, synth
from cudaring_b200._lib import CudaRingError

from conftest import rel_inf

pytestmark = pytest.mark.gpu
TOL = 1e-12
KW = dict(potential="harmonic", interaction="vertexVertex", ea=1.0, el=1.0, eb=0.01, ec=1.0)


def _oracle_forces(pk, kw, cut_off=0.5):
    S = oracle.System(pk.nv_list, pk.box, kw["potential"], kw["interaction"], kw["ea"], kw["el"], kw["eb"], kw["ec"],
                      lj_cutoff=kw.get("LJcutoff", 2.5))
    S.neighbor_list(pk.pos, pk.rad, S.cut_distance(cut_off))
    return S.force_energy(pk.pos, pk.rad, pk.a0, pk.l0, pk.theta0)


def _dilated_list(d, pk, cutoff):
    """Build the list at positions and box scaled by 3 (few neighbours, the
    smallest capacity), then restore the dense state without a rebuild."""
    d.setBoxSize(pk.box * 3)
    d.setVertexPositions(pk.pos * 3)
    d.calcNeighborList(d.setDisplacementCutoff(cutoff, 2 * pk.rad.mean()))
    d.setBoxSize(pk.box)
    d.setVertexPositions(pk.pos)


def test_list_overflow_inside_a_step_sequence_resumes_exactly(cuda_device):
    # 64 harmonic rings at phi 0.85 with a wide list (cutDistance 3): dense
    # lists.  Context A builds its first list on the dilated state, so the
    # rebuild inside the first captured chunk finds more neighbours than the
    # capacity: the chunk aborts, the host grows the list and resumes from the
    # failed build.  Context B starts with a large capacity.  The two runs must
    # be identical.
    c = synth.workload_config("bidisperse_harmonic", 64)
    pk = synth.make_packing(c["nv"], c["a0"], c["calA0"], 0.85, seed=17, placement="uniform")
    out = []
    for grow_first in (False, True):
        d = DPM2D.from_packing(pk, **KW, dt=0.005)
        d.setPrecision("fp64")
        d.setLanes(2)
        if grow_first:
            d.calcNeighborList(d.setDisplacementCutoff(2.0, 2 * pk.rad.mean()))
        _dilated_list(d, pk, 2.0)
        small_cap = d.getNeighborListSize()
        d.initNVE(0.0, readState=True)
        d.NVELoop(300)
        out.append((d.getVertexPositions(), d.getVertexVelocities(), d.getUpdateCount(), small_cap,
                    d.getNeighborListSize()))
        d.close()
    (xa, va, ua, capa, lsa), (xb, vb, ub, capb, lsb) = out
    assert capa < lsa  # context A's list grew during the run
    assert ua == ub and ua >= 1
    assert np.array_equal(xa, xb)
    assert np.array_equal(va, vb)


def test_single_ring_has_an_empty_list_and_shape_forces_only(cuda_device):
    # a box several ring diameters wide (the shape kernels unwrap a ring by
    # the minimum image, which needs rings smaller than half the box)
    pk = synth.make_packing([16], [1.0], 1.0, 0.05, seed=3, placement="uniform")
    with DPM2D.from_packing(pk, **KW) as d:
        d.calcNeighborList(d.setDisplacementCutoff(0.5, 2 * pk.rad.mean()))
        assert not np.any(d.getMaxNeighborList())
        d.calcForceEnergy()
        out = _oracle_forces(pk, KW)
        assert rel_inf(d.getVertexForces(), out["force"]) < TOL
        # NVE on a lone ring conserves energy and momentum
        d.initNVE(0.01, readState=False)
        e0 = d.getEnergy()
        p0 = d.getVertexVelocities().reshape(-1, 2).sum(0)
        d.NVELoop(2000)
        assert abs(d.getEnergy() - e0) / abs(e0) < 1e-3
        assert np.abs(d.getVertexVelocities().reshape(-1, 2).sum(0) - p0).max() < 1e-9


@pytest.mark.parametrize("interaction", ["vertexVertex", "vertexSmooth"])
def test_three_vertex_rings_match_oracle(cuda_device, interaction):
    pk = synth.make_packing([3] * 24, [1.0] * 12 + [1.96] * 12, 1.0, 0.6, seed=8, placement="uniform")
    kw = dict(KW, interaction=interaction)
    with DPM2D.from_packing(pk, **kw) as d:
        d.calcNeighborList(d.setDisplacementCutoff(0.5, 2 * pk.rad.mean()))
        d.calcForceEnergy()
        out = _oracle_forces(pk, kw)
        assert rel_inf(d.getVertexForces(), out["force"]) < TOL
        assert d.getPotentialEnergy() == pytest.approx(out["potential_energy"], rel=1e-12)


def test_largest_ring_of_a_tile_matches_oracle(cuda_device):
    # 128 vertices: one ring per one-lane tile; two lanes per vertex cannot hold it
    pk = synth.make_packing([128] * 4 + [20] * 8, [4.0] * 4 + [1.0] * 8, 1.0, 0.6, seed=9, placement="uniform")
    with DPM2D.from_packing(pk, **KW) as d:
        assert d.getLanes() == 1
        with pytest.raises(CudaRingError):
            d.setLanes(2)
        d.calcNeighborList(d.setDisplacementCutoff(0.5, 2 * pk.rad.mean()))
        d.calcForceEnergy()
        out = _oracle_forces(pk, KW)
        assert rel_inf(d.getVertexForces(), out["force"]) < TOL


def test_invalid_contexts_are_rejected(cuda_device):
    with pytest.raises(CudaRingError):
        DPM2D([16, 2])  # a ring needs three vertices
    with pytest.raises(CudaRingError):
        DPM2D([129])  # larger than a tile
    with DPM2D([16, 16]) as d:
        with pytest.raises(CudaRingError):
            d.setBoxSize(np.array([0.0, 1.0]))
        with pytest.raises(CudaRingError):
            d.setTimeStep(-1.0)
