"""CPU checks of the boundary and host logic: the C ABI library loads and
exports every symbol include/cudaring.h declares (no compute calls), the C++
facade compiles against it, and the synthetic generator follows the
reference's conventions."""
import math
import os
import subprocess

import numpy as np
import pytest

from cudaring_b200 import _lib, build, synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def libcr():
    build.build()
    return _lib.lib()


def test_library_exports_every_declared_symbol(libcr):
    syms = _lib.declared_symbols()
    assert len(syms) > 60
    missing = [s for s in syms if not hasattr(libcr, s)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIBPATH], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    assert set(syms) <= exported


def test_header_prototypes_parse_to_ctypes():
    protos = _lib.parse_header()
    ret, args = protos["cr_create"]
    assert ret == "int" and len(args) == 3
    assert protos["cr_last_error"][0].startswith("const char")


def test_cpp_facade_compiles(tmp_path):
    src = tmp_path / "drv.cpp"
    src.write_text('#include "cudaring/DPM2D.hpp"\n'
                   "int main(){ std::vector<long> nv(4, 16); cudaring::DPM2D d(nv);"
                   " double c = d.setDisplacementCutoff(0.5, 0.2); d.calcNeighbors(c); d.calcForceEnergy();"
                   " d.initNVE(1e-3, false); d.NVELoop(); return 0; }\n")
    r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-I", os.path.join(ROOT, "include"), str(src)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_null_context_is_rejected_without_gpu(libcr):
    # argument checks happen before any device call
    assert libcr.cr_set_time_step(None, 0.1) == 1
    assert libcr.cr_calc_force_energy(None) == 1
    assert libcr.cr_destroy(None) == 1


def test_ring_rest_shape_matches_reference_formula():
    # src/DPM2D.cu:1577-1581
    nv, a0, calA0 = 16, 1.0, 1.0
    l0, th0, rad = synth.ring_rest_shape(nv, a0, calA0)
    calA = calA0 * nv * math.tan(math.pi / nv) / math.pi
    assert l0 == pytest.approx(2 * math.sqrt(math.pi * calA * a0) / nv, rel=1e-15)
    assert th0 == pytest.approx(2 * math.pi / nv)
    assert rad == pytest.approx(l0 / 2)


def test_packing_phi_and_orientation():
    c = synth.workload_config("smooth_lj")
    pk = synth.make_packing(c["nv"], c["a0"], c["calA0"], c["phi"], seed=1)
    assert pk.num_vertices == 512 * 32 + 512 * 45 == 39424
    assert synth.preferred_phi(pk.nv_list, pk.a0, pk.rad, pk.box) == pytest.approx(0.85, rel=1e-12)
    # counter-clockwise rings: positive signed shoelace area
    first = pk.first_vertex()
    for q in (0, 600):
        n = pk.nv_list[q]
        x = pk.pos.reshape(-1, 2)[first[q]:first[q] + n]
        x = x - x[0]
        area = 0.5 * np.sum(x[:, 0] * np.roll(x[:, 1], -1) - np.roll(x[:, 0], -1) * x[:, 1])
        assert area > 0


def test_rsa_centres_do_not_overlap():
    rng = np.random.default_rng(3)
    r = rng.uniform(0.5, 0.7, 200)
    L = 40.0
    c = synth.rsa_centres(r, L, rng)
    d = c[:, None, :] - c[None, :, :]
    d -= L * np.round(d / L)
    dist = np.sqrt((d ** 2).sum(-1)) + np.eye(200) * 1e9
    assert (dist >= r[:, None] + r[None, :] - 1e-12).all()


def test_tuning_entry_points_reject_a_null_context(libcr):
    # the step-structure switches validate their context before any device call
    assert libcr.cr_set_multistep(None, 1) == 1
    assert libcr.cr_set_use_graphs(None, 1) == 1
    assert libcr.cr_set_lanes(None, 2) == 1
    assert libcr.cr_hessian_solve(None, None, None, 1e-10, 10, None, None) == 1


def test_benchmark_workloads_are_named():
    for name, rings in (("bidisperse_harmonic", 32), ("smooth_lj", 1024), ("rigid_ellipses", 4096),
                        ("dense_harmonic", 256)):
        c = synth.workload_config(name)
        n = c["n"] if c.get("rigid") else len(c["nv"])
        assert n == rings
    assert len(synth.workload_config("smooth_lj", 64)["nv"]) == 64
    with pytest.raises(ValueError):
        synth.workload_config("cfg2")
