"""Recovery when a grid-barrier wait gives up.

The multi-step kernel and the one-launch neighbour-list build wait on grid
barriers that need every CTA of their grid resident at once; a GPU shared
with other work may not hold them all.  Every such wait is bounded
(cr_set_spin_limit).  Here the bound is negative, so every wait that does
not find its barrier complete gives up at once: the kernels return an
error status (nothing hangs), and the context
must go back to the state the call started from, switch to one launch per op
with the multi-kernel list build, and finish the call on the same trajectory
as a context that never used the barrier kernels.
"""
import numpy as np
import pytest

from cudaring_b200 import DPM2D, synth

from conftest import rel_inf

pytestmark = pytest.mark.gpu


def _context(pk, c):
    d = DPM2D.from_packing(pk, **{k: c[k] for k in ("potential", "interaction", "ea", "el", "eb", "ec", "LJcutoff",
                                                      "dt")})
    cut = d.setDisplacementCutoff(0.5, 2.0 * d.getMeanVertexRadius())
    d.calcNeighborList(cut)
    d.resetLastPositions()
    d.calcForceEnergy()
    d.initNVE(0.0, readState=True)
    return d, cut


@pytest.fixture(scope="module")
def packing(cuda_device):
    # 256 smooth-LJ rings (about 10k vertices, about a hundred tiles) at phi
    # 0.40 with thermal ring velocities
    c = synth.workload_config("smooth_lj", 256)
    pk = synth.make_packing(c["nv"], c["a0"], c["calA0"], 0.40, seed=41, placement="rsa")
    pk.vel = np.repeat(np.random.default_rng(4).normal(0.0, 0.1, size=(256, 2)), pk.nv_list, axis=0).reshape(-1)
    return pk, c


def test_stalled_multistep_sequence_reruns_one_launch_per_op(packing):
    pk, c = packing
    ref, _ = _context(pk, c)
    ref.setMultistep(0)
    ref.NVELoop(400)
    d, _ = _context(pk, c)
    d.setSpinLimit(-1)
    d.NVELoop(400)
    assert d.getDegraded()
    assert not ref.getDegraded()
    assert d.getUpdateCount() >= 1
    # the fallback rebuilt the list at the sequence's start: neighbour order
    # and rebuild times differ, so trajectories agree to rounding, not bit for bit
    assert rel_inf(d.getVertexPositions(), ref.getVertexPositions()) < 1e-9
    assert d.getEnergy() == pytest.approx(ref.getEnergy(), rel=1e-9)
    # later calls stay on the fallback and keep matching
    d.NVELoop(100)
    ref.NVELoop(100)
    assert rel_inf(d.getVertexPositions(), ref.getVertexPositions()) < 1e-9
    d.close()
    ref.close()


def test_stalled_list_build_retries_with_the_multi_kernel_build(packing):
    pk, c = packing
    ref, cut = _context(pk, c)
    d, _ = _context(pk, c)
    d.setSpinLimit(-1)
    d.calcNeighborList(cut)
    assert d.getDegraded()
    assert np.array_equal(d.getMaxNeighborList(), ref.getMaxNeighborList())
    assert np.array_equal(d.getNeighbors(), ref.getNeighbors())
    d.calcForceEnergy()
    assert rel_inf(d.getVertexForces(), ref.getVertexForces()) < 1e-12
    d.close()
    ref.close()
