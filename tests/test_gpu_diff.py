"""Derivatives (cr_hvp, cr_calc_pressure, cr_param_derivatives,
cr_hessian_solve) and the gradients built on them (cudaring_b200.diff),
checked against central finite differences (h = 1e-6 relative) of the
library's own FP64 forces and energies, against the same differences of the
CPU oracle's forces (an FP64 reference that uses no derivative code), and
through test-side torch.autograd.Functions.
"""
import numpy as np
import pytest
import torch

import oracle
from cudaring_b200 import DPM2D, diff, synth, workloads
from oracle.integrators import nve_adjoint_reference

from conftest import rel_inf

pytestmark = pytest.mark.gpu
KW = dict(potential="harmonic", interaction="vertexVertex", ea=1.0, el=1.0, eb=0.01, ec=1.0)


def _system(n=16, phi=0.70, seed=4, rad_scale=1.3, placement="uniform", **kw):
    c = synth.workload_config("bidisperse_harmonic", n)
    pk = synth.make_packing(c["nv"], c["a0"], c["calA0"], phi, seed=seed, placement=placement)
    pk.rad = pk.rad * rad_scale  # overlapping rings: every term of U acts
    args = dict(KW, **kw)
    d = DPM2D.from_packing(pk, **args)
    d.calcNeighborList(d.setDisplacementCutoff(0.5, 2.0 * d.getMeanVertexRadius()))
    d.calcForceEnergy()
    return d, pk, args


def _forces_at(d, x):
    d.setVertexPositions(x)
    d.calcNeighborList(d.setDisplacementCutoff(0.5, 2.0 * d.getMeanVertexRadius()))
    d.calcForceEnergy()
    return d.getVertexForces(), d.getPotentialEnergy()


@pytest.mark.parametrize("potential", ["harmonic", "lennardJones", "wca"])
def test_hvp_matches_force_differences(cuda_device, potential):
    d, pk, args = _system(potential=potential, rad_scale=1.3 if potential == "harmonic" else 1.0)
    x = d.getVertexPositions()
    v = np.random.default_rng(1).normal(size=x.shape)
    hv = d.hvp(v)
    eps = 1e-6
    fp, _ = _forces_at(d, x + eps * v)
    fm, _ = _forces_at(d, x - eps * v)
    fd = -(fp - fm) / (2 * eps)
    assert rel_inf(hv, fd) < 2e-6
    # the oracle's forces, differenced the same way
    S = oracle.System(pk.nv_list, pk.box, potential, "vertexVertex", args["ea"], args["el"], args["eb"], args["ec"],
                      lj_cutoff=2.5)
    ofd = []
    for sgn in (+1, -1):
        xs = x + sgn * eps * v
        S.neighbor_list(xs, pk.rad, S.cut_distance(0.5))
        ofd.append(S.force_energy(xs, pk.rad, pk.a0, pk.l0, pk.theta0)["force"])
    assert rel_inf(hv, -(ofd[0] - ofd[1]) / (2 * eps)) < 2e-6


def _variant(case):
    # smooth vertex-segment LJ / harmonic, or FENE monomers on vertex-vertex harmonic
    if case == "lj_smooth":
        # rings placed without overlap: LJ across the gaps, no r^-12 blow-up
        d, pk, args = _system(potential="lennardJones", interaction="vertexSmooth", rad_scale=1.0, phi=0.5,
                              placement="rsa")
    elif case == "harmonic_smooth":
        d, pk, args = _system(interaction="vertexSmooth")
    else:
        d, pk, args = _system()
        from cudaring_b200.dpm2d import simControl
        d.setMonomerType(simControl.monomerEnum.FENE)
        d.setFENEconstants(1.0, 1.5)
        d.calcForceEnergy()
    return d, pk, args


@pytest.mark.parametrize("case", ["lj_smooth", "harmonic_smooth", "fene"])
def test_hvp_smooth_interaction_and_fene(cuda_device, case):
    d, pk, args = _variant(case)
    x = d.getVertexPositions()
    v = np.random.default_rng(3).normal(size=x.shape)
    hv = d.hvp(v)
    eps = 1e-6
    fp, _ = _forces_at(d, x + eps * v)
    fm, _ = _forces_at(d, x - eps * v)
    assert rel_inf(hv, -(fp - fm) / (2 * eps)) < 2e-6
    # the same differences of the oracle's FP64 forces
    S = oracle.System(pk.nv_list, pk.box, args["potential"], args["interaction"], args["ea"], args["el"], args["eb"],
                      args["ec"], lj_cutoff=2.5, monomer=1 if case == "fene" else 0,
                      stiff=1.0 if case == "fene" else 0.0, ext=1.5 if case == "fene" else 0.0)
    ofd = []
    for sgn in (+1, -1):
        xs = x + sgn * eps * v
        S.neighbor_list(xs, pk.rad, S.cut_distance(0.5))
        ofd.append(S.force_energy(xs, pk.rad, pk.a0, pk.l0, pk.theta0)["force"])
    assert rel_inf(hv, -(ofd[0] - ofd[1]) / (2 * eps)) < 2e-6


@pytest.mark.parametrize("case", ["lj_smooth", "fene"])
def test_pressure_smooth_interaction_and_fene(cuda_device, case):
    d, pk, _ = _variant(case)
    x, box = d.getVertexPositions(), d.getBoxSize()
    P = d.calcPressure()
    h = 1e-6
    U = []
    for lam in (1 + h, 1 - h):
        d.setBoxSize(box * lam)
        _, u = _forces_at(d, x * lam)
        U.append(u)
    d.setBoxSize(box)
    fd = -(U[0] - U[1]) / (box[0] * box[1] * ((1 + h) ** 2 - (1 - h) ** 2))
    assert P == pytest.approx(fd, rel=1e-6, abs=1e-9)


def test_pressure_is_affine_energy_derivative(cuda_device):
    d, pk, _ = _system()
    x, box = d.getVertexPositions(), d.getBoxSize()
    P = d.calcPressure()
    h = 1e-6
    U = []
    for lam in (1 + h, 1 - h):
        d.setBoxSize(box * lam)
        _, u = _forces_at(d, x * lam)
        U.append(u)
    d.setBoxSize(box)
    A0 = box[0] * box[1]
    fd = -(U[0] - U[1]) / (A0 * ((1 + h) ** 2 - (1 - h) ** 2))
    assert P == pytest.approx(fd, rel=1e-6, abs=1e-9)


@pytest.mark.parametrize("param", ["ea", "el", "eb", "lnCalA0"])
def test_parameter_derivatives(cuda_device, param):
    d, pk, args = _system()
    x = d.getVertexPositions()
    dU, dP, dF, dPdx = d.paramDerivatives(param)
    # U, F and P are linear in ea, el, eb at fixed positions, so a wide step
    # costs nothing in truncation and avoids cancellation against the rest of U
    h = 1e-6 if param == "lnCalA0" else 1e-3
    res = []
    for sgn in (+1, -1):
        if param == "lnCalA0":
            f = np.exp(0.5 * sgn * h)
            d.setRestLengths(pk.l0 * f)
            d.setVertexRadii(pk.rad * f)
        else:
            a = dict(args)
            a[param] = args[param] * (1 + sgn * h)
            d.setEnergyCosts(a["ea"], a["el"], a["eb"], a["ec"])
        F, U = _forces_at(d, x)
        res.append((F, U, d.calcPressure()))
    scale = 1.0 if param == "lnCalA0" else args[param]
    fdU = (res[0][1] - res[1][1]) / (2 * h * scale)
    fdF = (res[0][0] - res[1][0]) / (2 * h * scale)
    fdP = (res[0][2] - res[1][2]) / (2 * h * scale)
    assert dU == pytest.approx(fdU, rel=1e-6, abs=1e-9)
    assert rel_inf(dF, fdF) < 1e-5
    assert dP == pytest.approx(fdP, rel=1e-5, abs=1e-8)
    # dP/dx against differences of the pressure along a random direction
    d.setEnergyCosts(args["ea"], args["el"], args["eb"], args["ec"])
    d.setRestLengths(pk.l0)
    d.setVertexRadii(pk.rad)
    w = np.random.default_rng(2).normal(size=x.shape)
    P2 = []
    h = 1e-6
    for sgn in (+1, -1):
        _forces_at(d, x + sgn * h * w)
        P2.append(d.calcPressure())
    assert float(dPdx @ w) == pytest.approx((P2[0] - P2[1]) / (2 * h), rel=1e-5, abs=1e-8)


@pytest.mark.parametrize("precond", ["block_jacobi", "none"])
def test_hessian_solve(cuda_device, precond):
    d, pk, args = _system(n=16, phi=0.80, seed=6)
    # minimise so that H is positive on the complement of the translations
    d.initFIRE([0.2, 0.5, 1.1, 0.99, 1e-2, 1e-1, 0.2], 20, 0, d.numVertices)
    _, fmax = d.minimizeFIRE(1e-12, 200000)
    assert fmax < 1e-10
    d.calcNeighborList(d.setDisplacementCutoff(0.5, 2.0 * d.getMeanVertexRadius()))
    # a right-hand side in the range of H (rings without contacts add zero
    # modes beyond the uniform translations)
    b = d.hvp(np.random.default_rng(3).normal(size=2 * d.numVertices))
    d.setCGPreconditioner(precond)
    x, it, rr = d.hessianSolve(b, 1e-10, 200000)
    assert rr <= 1e-10
    hx = d.hvp(x)
    assert np.linalg.norm(hx - b) / np.linalg.norm(b) < 1e-8


@pytest.mark.parametrize("interaction,potential", [("vertexVertex", "harmonic"), ("vertexSmooth", "lennardJones"),
                                                   ("vertexSmooth", "harmonic")])
def test_hessian_diag_blocks_match_hvp(cuda_device, interaction, potential):
    # the block-Jacobi preconditioner's 2 x 2 blocks (one hyper-dual launch,
    # each thread seeding its own vertex) against H e for unit vectors e
    d, pk, args = _system(n=16, phi=0.80, seed=9, interaction=interaction, potential=potential)
    blocks = d.hessianDiagBlocks()
    nv = d.numVertices
    for v in (0, 7, nv // 2, nv - 1):
        for c in (0, 1):
            e = np.zeros(2 * nv)
            e[2 * v + c] = 1.0
            col = d.hvp(e)[2 * v:2 * v + 2]
            want = blocks[v, [0, 1]] if c == 0 else blocks[v, [1, 2]]
            assert np.allclose(col, want, rtol=1e-10, atol=1e-10 * np.abs(blocks).max())


class MinimizedEnergyPressure(torch.autograd.Function):
    """(U*, P*) of the FIRE minimum as a function of theta = (ea, el, eb,
    calA0); the backward pass returns the adjoint gradients."""

    @staticmethod
    def forward(ctx, theta, packing):
        d, U, P, g = _minimised(packing, theta.tolist(), want_grad=True)
        d.close()
        ctx.save_for_backward(torch.tensor([[g["dU"][k] for k in diff.PARAMS], [g["dP"][k] for k in diff.PARAMS]],
                                           dtype=torch.float64))
        return torch.tensor([U, P], dtype=torch.float64)

    @staticmethod
    def backward(ctx, grad):
        (J,) = ctx.saved_tensors
        return grad @ J, None


def _minimised(pk, theta, want_grad=False):
    ea, el, eb, calA0 = theta
    f = np.sqrt(calA0 / 1.0)
    q = synth.Packing(nv_list=pk.nv_list, pos=pk.pos.copy(), vel=np.zeros_like(pk.pos), rad=pk.rad * f,
                      l0=pk.l0 * f, theta0=pk.theta0, a0=pk.a0, box=pk.box, centres=pk.centres)
    d = DPM2D.from_packing(q, potential="harmonic", interaction="vertexVertex", ea=ea, el=el, eb=eb, ec=1.0)
    d.calcNeighborList(d.setDisplacementCutoff(0.5, 2.0 * d.getMeanVertexRadius()))
    d.calcForceEnergy()
    sig = d.getMeanParticleSize()
    # dt = 1e-3 sigma: the vertex radius here is 0.05 sigma and the contact
    # stiffness ec / (2 r)^2 makes 1e-2 sigma unstable
    d.initFIRE([0.2, 0.5, 1.1, 0.99, 1e-3 * sig, 1e-2 * sig, 0.2], 20, 0, d.numVertices)
    _, fmax = d.minimizeFIRE(1e-13, 400000)
    assert fmax <= 1e-12
    d.calcNeighborList(d.setDisplacementCutoff(0.5, 2.0 * d.getMeanVertexRadius()))
    d.calcForceEnergy()
    U, P = d.getPotentialEnergy(), d.calcPressure()
    g = diff.minimized_gradients(d, calA0, tol=1e-10) if want_grad else None
    return d, U, P, g


@pytest.fixture(scope="module")
def jammed_packing(cuda_device):
    # rings nv 32, harmonic, above jamming (phi 0.88), relaxed; calA0 = 1 at the reference point
    d, info = workloads.prepared_deformable("dense_harmonic", 16, seed=21)
    pk = synth.Packing(nv_list=d.numVertexInParticleList, pos=d.getVertexPositions(),
                       vel=np.zeros(2 * d.numVertices), rad=d.getVertexRadii(), l0=d.getRestLengths(),
                       theta0=d.getRestAngles(), a0=d.getRestAreas(), box=d.getBoxSize(),
                       centres=np.zeros((d.numParticles, 2)))
    d.close()
    return pk


def test_minimized_gradients_match_central_differences(jammed_packing):
    theta = torch.tensor([1.0, 1.0, 0.01, 1.0], dtype=torch.float64, requires_grad=True)
    out = MinimizedEnergyPressure.apply(theta, jammed_packing)
    U, P = float(out[0].detach()), float(out[1].detach())
    assert U > 0 and P > 0  # above jamming
    gU = torch.autograd.grad(out[0], theta, retain_graph=True)[0].numpy()
    gP = torch.autograd.grad(out[1], theta)[0].numpy()
    base = theta.detach().numpy()
    for i in range(4):
        h = 1e-6 * base[i]
        vals = []
        for sgn in (+1, -1):
            t = base.copy()
            t[i] += sgn * h
            d, u, p, _ = _minimised(jammed_packing, t)
            d.close()
            vals.append((u, p))
        fdU = (vals[0][0] - vals[1][0]) / (2 * h)
        fdP = (vals[0][1] - vals[1][1]) / (2 * h)
        assert gU[i] == pytest.approx(fdU, rel=1e-4, abs=1e-9 * max(1.0, abs(U))), diff.PARAMS[i]
        assert gP[i] == pytest.approx(fdP, rel=1e-3, abs=1e-6 * max(1.0, abs(P))), diff.PARAMS[i]


class NVEEnergy(torch.autograd.Function):
    """J = U + K after nsteps velocity-Verlet steps, as a function of x0."""

    @staticmethod
    def forward(ctx, x0, d, v0, nsteps, dt, checkpoint):
        J, gx, _ = diff.nve_gradient(d, x0.numpy(), v0, nsteps, dt, checkpoint)
        ctx.save_for_backward(torch.from_numpy(gx))
        return torch.tensor(J, dtype=torch.float64)

    @staticmethod
    def backward(ctx, g):
        (gx,) = ctx.saved_tensors
        return g * gx, None, None, None, None, None


def test_nve_gradient_through_checkpoints(cuda_device):
    d, pk, args = _system(n=8, phi=0.60, seed=12, rad_scale=1.2)
    x0 = d.getVertexPositions()
    v0 = np.repeat(np.random.default_rng(5).normal(0, 0.05, size=(8, 2)), pk.nv_list, axis=0).reshape(-1)
    nsteps, dt = 200, 0.002
    x = torch.tensor(x0, dtype=torch.float64, requires_grad=True)
    J = NVEEnergy.apply(x, d, v0, nsteps, dt, 20)
    J.backward()
    g = x.grad.numpy()
    # the same gradient without checkpoints (one segment) agrees to rounding
    _, g1, _ = diff.nve_gradient(d, x0, v0, nsteps, dt, checkpoint=nsteps)
    assert rel_inf(g, g1) < 1e-10
    # the FP64 reference gradient: the same recursion with Hessian-vector
    # products from central differences of the CPU oracle's forces
    S = oracle.System(pk.nv_list, pk.box, "harmonic", "vertexVertex", 1.0, 1.0, 0.01, 1.0)
    q = synth.Packing(nv_list=pk.nv_list, pos=x0.copy(), vel=v0.copy(), rad=pk.rad, l0=pk.l0, theta0=pk.theta0,
                      a0=pk.a0, box=pk.box, centres=pk.centres)
    J_ref, g_ref, _ = nve_adjoint_reference(S, q, nsteps, dt)
    assert float(J.detach()) == pytest.approx(J_ref, rel=1e-10)
    assert rel_inf(g, g_ref) < 1e-6
    rng = np.random.default_rng(7)
    h = 1e-6
    for i in rng.choice(len(x0), 6, replace=False):
        e = np.zeros_like(x0)
        e[i] = h
        fd = (diff.nve_run(d, x0 + e, v0, nsteps, dt) - diff.nve_run(d, x0 - e, v0, nsteps, dt)) / (2 * h)
        assert g[i] == pytest.approx(fd, rel=1e-4, abs=1e-6 * np.abs(g).max())
