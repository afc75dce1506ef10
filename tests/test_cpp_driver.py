"""The C++ drop-in boundary: a driver shaped like the reference's runNVE.cpp
(tests/cpp/run_nve.cpp), written against include/cudaring/DPM2D.hpp and
FileIO.hpp, compiled, linked against libcudaring.so and run.

On CPU the driver is compiled and linked (no device calls).  On the GPU it
reads a packing written in the reference's directory format, runs NVE one
step per NVELoop() call, and its final state must equal the same sequence of
calls made through the Python binding.
"""
import json
import os
import subprocess

import numpy as np
import pytest

from cudaring_b200 import DPM2D, packing_io, simControl, synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "cudaring_b200", "lib")


def _build_driver(tmp_path):
    exe = str(tmp_path / "run_nve")
    cmd = ["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "run_nve.cpp"), "-L", LIBDIR, "-lcudaring",
           f"-Wl,-rpath,{LIBDIR}", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_cpp_driver_compiles_and_links(tmp_path):
    from cudaring_b200 import build

    build.build()
    exe = _build_driver(tmp_path)
    r = subprocess.run(["ldd", exe], capture_output=True, text=True)
    assert "libcudaring.so" in r.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("pot,inter", [("lj", "smooth"), ("harmonic", "vv")])
def test_cpp_driver_matches_python_path(cuda_device, tmp_path, pot, inter):
    rings, steps, dt_unit, T = 32, 300, 2e-3, 1e-3
    c = synth.workload_config("smooth_lj", rings)
    pk = synth.make_packing(c["nv"], c["a0"], c["calA0"], 0.45, seed=77, placement="rsa")
    pk.vel = np.repeat(np.random.default_rng(5).normal(0.0, 0.02, size=(rings, 2)), pk.nv_list, axis=0).reshape(-1)
    in_dir, out_dir = str(tmp_path / "in") + "/", str(tmp_path / "out") + "/"
    os.makedirs(out_dir)
    packing_io.save_packing_arrays(in_dir, pk, digits=17)

    exe = _build_driver(tmp_path)
    r = subprocess.run([exe, in_dir, out_dir, repr(dt_unit), repr(T), str(steps), str(rings), pot, inter],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    cpp = json.loads(r.stdout.strip().splitlines()[-1])
    got = packing_io.load_packing(out_dir, rings)

    # the same calls through the Python binding (runNVE.cpp:62-135 order)
    back = packing_io.load_packing(in_dir, rings)
    d = DPM2D(back.nv_list)
    if pot == "lj":
        d.setPotentialType(simControl.potentialEnum.lennardJones)
        d.setLJcutoff(1.5)
    if inter == "smooth":
        d.setInteractionType(simControl.interactionEnum.vertexSmooth)
    d.setVertexPositions(back.pos)
    d.setVertexRadii(back.rad)
    d.setRestAreas(back.a0)
    d.setRestLengths(back.l0)
    d.setRestAngles(back.theta0)
    d.setBoxSize(back.box)
    d.setEnergyCosts(1e5, 20, 10, 1)
    d.setVertexVelocities(back.vel)
    d.setTimeStep(dt_unit * d.getMeanParticleSize())
    d.initNVE(T, readState=True)
    cut = d.setDisplacementCutoff(0.5, 2 * d.getMeanVertexRadius())
    d.calcNeighborList(cut)
    d.calcForceEnergy()
    d.resetUpdateCount()
    e0 = d.getEnergy()
    for _ in range(steps):
        d.NVELoop(1)
    assert cpp["steps"] == steps
    assert cpp["updates"] == d.getUpdateCount()
    assert cpp["updates"] > 0  # the run crossed neighbour rebuilds
    assert cpp["energy0"] == pytest.approx(e0, rel=1e-15)
    assert cpp["energy"] == pytest.approx(d.getEnergy(), rel=1e-13)
    # positions: written with 17 digits, so they round-trip exactly
    assert np.array_equal(got.pos, d.getVertexPositions())
    assert np.array_equal(got.vel, d.getVertexVelocities())
    d.close()
