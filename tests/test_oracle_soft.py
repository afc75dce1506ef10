"""The soft-disk pre-packing restatement (oracle/particles.py) against the
fixtures produced by the reference's own kernels (tests/golden/soft_*.npz):
setRandomParticles on the drand48 stream, the particle neighbour list, the
particle forces, particle FIRE, the driver's minimisation loop and
initVerticesOnParticles.
"""
import numpy as np
import pytest

from oracle import particles as P

from conftest import golden_files, load_golden, rel_inf

POTS = {0: "harmonic", 1: "lennardJones", 2: "adhesive", 3: "wca"}


def _random(g):
    return P.set_random_particles(g["in_nv_list"], g["in_a0"], g["in_l0"], g["in_rad"], [1.0, 1.0],
                                  float(g["param_phi0"]), float(g["param_extra_rad"]), int(g["param_seed"]))


def test_drand48_matches_the_c_library():
    # the restated generator against libc's erand48 on the state srand48(seed) sets
    import ctypes
    libc = ctypes.CDLL(None)
    libc.erand48.restype = ctypes.c_double
    libc.erand48.argtypes = [ctypes.POINTER(ctypes.c_ushort * 3)]
    for seed in (0, 1, 4242, 20261203):
        xs = (ctypes.c_ushort * 3)(0x330E, seed & 0xFFFF, (seed >> 16) & 0xFFFF)
        want = [libc.erand48(ctypes.byref(xs)) for _ in range(50)]
        assert list(P.Drand48(seed).take(50)) == want


@pytest.mark.parametrize("path", golden_files("soft_"), ids=lambda p: p.split("/")[-1][:-4])
def test_random_particles_list_and_forces(path):
    g = load_golden(path)
    a0, l0, rad, box, ppos, prad = _random(g)
    assert np.array_equal(a0, g["out_a0"])
    assert np.array_equal(l0, g["out_l0"])
    assert np.array_equal(rad, g["out_rad"])
    assert np.array_equal(box, g["out_box"])
    assert np.array_equal(ppos, g["out_ppos"])
    assert np.array_equal(prad, g["out_prad"])
    rows, cnt, ls = P.particle_neighbor_list(ppos, prad, box, float(g["param_cut"]))
    assert ls == int(g["out_plist_size"])
    assert np.array_equal(cnt, g["out_pmax"])
    assert np.array_equal(rows, g["out_pneighbors"])
    f, e = P.particle_force_energy(ppos, prad, box, rows, cnt, ls, POTS[int(g["param_potential"])],
                                   lj_cutoff=float(g["param_lj_cutoff"]))
    assert rel_inf(f, g["out_pforce"]) < 1e-12
    assert rel_inf(e, g["out_penergy"]) < 1e-12


# FIRE on harmonic disks, the potential of the reference driver; random
# disks under WCA / LJ start from overlaps with forces of order 1e10, which
# no finite trajectory comparison survives.
@pytest.mark.parametrize("path", golden_files("soft_harmonic"), ids=lambda p: p.split("/")[-1][:-4])
def test_particle_fire_ten_iterations(path):
    g = load_golden(path)
    _, _, _, box, ppos, prad = _random(g)
    F = P.ParticleFire(ppos, prad, box, g["param_fire"], int(g["param_min_step"]), 0,
                       POTS[int(g["param_potential"])], lj_cutoff=float(g["param_lj_cutoff"]))
    F.build(float(g["param_cut"]))
    F.forces()
    F.loop(10)
    # the FIRE sums run in another order than the reference's: rounding-level
    # differences, relative to the largest coordinate / velocity
    assert rel_inf(F.x, g["out_fire10_ppos"]) < 1e-12
    assert rel_inf(F.v, g["out_fire10_pvel"]) < 1e-9
    assert F.dt == pytest.approx(float(g["out_fire10_state"][0]), rel=1e-15)
    assert F.a == pytest.approx(float(g["out_fire10_state"][1]), rel=1e-15)
    assert F.num_step == int(g["out_fire10_state"][2])


def test_minimization_and_vertices_on_particles():
    g = load_golden(golden_files("soft_harmonic")[0])
    a0, l0, _, box, ppos, prad = _random(g)
    F = P.ParticleFire(ppos, prad, box, g["param_fire"], int(g["param_min_step"]))
    cut = float(g["param_cut"])
    F.build(cut)
    F.forces()
    tol = float(g["param_tol"])
    it = F.minimize(cut, tol, 1000000)
    assert F.max_force() <= tol
    # the same basin: iterations within a few percent, positions to 1e-8
    assert abs(it - int(g["out_min_iters"])) <= max(5, int(0.05 * int(g["out_min_iters"])))
    assert np.abs(F.x - g["out_min_ppos"]).max() < 1e-8
    draws = P.Drand48(7).take(2 * len(l0))
    assert np.array_equal(draws, g["in_draws"])
    pos = P.vertices_on_particles(g["in_nv_list"], a0, l0, g["out_min_ppos"], draws)
    assert np.abs(pos - g["out_vpos"]).max() < 1e-14
