"""Packing files in the reference's directory format (cudaring_b200.packing_io)."""
import os

import numpy as np

from cudaring_b200 import packing_io, synth


def _packing():
    c = synth.workload_config("bidisperse_harmonic", 8)
    pk = synth.make_packing(c["nv"], c["a0"], c["calA0"], 0.5, seed=3, placement="rsa")
    pk.vel = np.random.default_rng(0).normal(size=pk.pos.shape)
    return pk


def test_round_trip_exact_at_17_digits(tmp_path):
    pk = _packing()
    packing_io.save_packing_arrays(str(tmp_path), pk, digits=17)
    q = packing_io.load_packing(str(tmp_path))
    for name in ("nv_list", "pos", "vel", "rad", "l0", "theta0", "a0", "box"):
        assert np.array_equal(getattr(q, name), getattr(pk, name)), name


def test_reference_text_layout(tmp_path):
    # setprecision(14) decimals; 2-D rows tab separated with a trailing tab
    # (FileIO.h save1DFile / save2DFile / save1DIndexFile)
    pk = _packing()
    packing_io.save_packing_arrays(str(tmp_path), pk)
    with open(os.path.join(tmp_path, "positions.dat")) as f:
        first = f.readline()
    assert first.endswith("\t\n") and first.count("\t") == 2
    x, y = (float(t) for t in first.split())
    assert x == float(f"{pk.pos[0]:.14g}") and y == float(f"{pk.pos[1]:.14g}")
    with open(os.path.join(tmp_path, "numVertexInParticleList.dat")) as f:
        assert [int(v) for v in f.read().split()] == list(pk.nv_list)
    q = packing_io.load_packing(str(tmp_path))
    assert np.allclose(q.pos, pk.pos, rtol=1e-13, atol=0)
    assert q.box.shape == (2,)
