"""The library against the reference's own CUDA build on the same B200.

oracle/_ref/ref_gpu_nve is farceri/cudaRing's DPM2D compiled from its
sources (oracle/build_ref_gpu.sh) behind a small driver that reads a packing
in the reference's directory format with the reference's own reader, runs
NVELoop() steps and writes the final state.  The library reads the same
files (cudaring_b200.packing_io) and runs the same steps; the two
trajectories must agree to FP64 rounding amplified by the dynamics, with the
same number of neighbour-list rebuilds.  Skipped where the binary was not
built (it needs the reference checkout at build time).
"""
import os
import subprocess

import numpy as np
import pytest

from cudaring_b200 import DPM2D, packing_io, synth

from conftest import rel_inf

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "oracle", "_ref", "ref_gpu_nve")


def _run_reference(dirname, npart, steps, dt, ea, el, eb, pot, inter, out):
    r = subprocess.run(["timeout", "300", BIN, dirname, str(npart), "0", str(steps), repr(dt), repr(ea), repr(el),
                        repr(eb), pot, inter, "2.5", out], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    import json

    info = json.loads(r.stdout.strip().splitlines()[-1])
    raw = np.fromfile(out, dtype=np.float64)
    return info, raw[: raw.size // 2], raw[raw.size // 2:]


@pytest.mark.skipif(not os.path.exists(BIN), reason="reference CUDA build not present")
@pytest.mark.parametrize("pot,inter", [("lj", "smooth"), ("harmonic", "vertex")])
def test_nve_matches_reference_cuda_build(cuda_device, tmp_path, pot, inter):
    c = synth.workload_config("smooth_lj", 64)
    pk = synth.make_packing(c["nv"], c["a0"], c["calA0"], 0.40, seed=31, placement="rsa")
    rng = np.random.default_rng(2)
    pk.vel = np.repeat(rng.normal(0.0, 0.3, size=(pk.num_particles, 2)), pk.nv_list, axis=0).reshape(-1)
    if pot == "harmonic":
        pk.rad = pk.rad * 1.5  # overlapping vertices, so the harmonic pairs act
    ea, el, eb, dt, steps = 1.0, 1.0, 0.01, 0.002, 300
    d = str(tmp_path / "packing")
    packing_io.save_packing_arrays(d, pk, digits=17)
    info, pos_ref, vel_ref = _run_reference(d, pk.num_particles, steps, dt, ea, el, eb, pot, inter,
                                            str(tmp_path / "final.bin"))
    assert info["cuda_error"] == "no error"

    pk2 = packing_io.load_packing(d)
    assert np.array_equal(pk2.pos, pk.pos) and np.array_equal(pk2.vel, pk.vel)
    potential = {"lj": "lennardJones", "harmonic": "harmonic"}[pot]
    interaction = {"smooth": "vertexSmooth", "vertex": "vertexVertex"}[inter]
    m = DPM2D.from_packing(pk2, potential=potential, interaction=interaction, ea=ea, el=el, eb=eb, ec=1.0,
                           LJcutoff=2.5, dt=dt)
    cut = m.setDisplacementCutoff(0.5, 2.0 * m.getMeanVertexRadius())
    m.calcNeighborList(cut)
    m.calcForceEnergy()
    m.initNVE(0.0, readState=True)
    e0 = m.getEnergy()
    assert e0 == pytest.approx(info["energy_start"], rel=1e-12)
    m.NVELoop(steps)
    assert m.getUpdateCount() == info["updates"]
    assert rel_inf(m.getVertexPositions(), pos_ref) < 1e-10
    assert rel_inf(m.getVertexVelocities(), vel_ref) < 1e-7
    assert m.getEnergy() == pytest.approx(info["energy_end"], rel=1e-10)


def test_save_packing_from_context_round_trip(cuda_device, tmp_path):
    c = synth.workload_config("smooth_lj", 8)
    pk = synth.make_packing(c["nv"], c["a0"], c["calA0"], 0.40, seed=5, placement="rsa")
    m = DPM2D.from_packing(pk, potential="lennardJones", interaction="vertexSmooth", ea=1.0, el=1.0, eb=0.01)
    m.calcNeighborList(m.setDisplacementCutoff(0.5, 2.0 * m.getMeanVertexRadius()))
    m.calcForceEnergy()
    packing_io.save_packing(str(tmp_path), m, digits=17, params={"ea": 1.0})
    q = packing_io.load_packing(str(tmp_path))
    for name, got in (("pos", q.pos), ("vel", q.vel), ("rad", q.rad), ("l0", q.l0), ("theta0", q.theta0),
                      ("a0", q.a0), ("box", q.box)):
        assert np.array_equal(got, getattr(pk, name)), name
    shapes = np.loadtxt(os.path.join(tmp_path, "shapes.dat"))
    assert np.allclose(shapes[:, 0], m.getAreas(), rtol=1e-15, atol=0)
