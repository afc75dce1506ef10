"""Gradients built on the library's derivative entry points.

* ``minimized_gradients``: derivatives of the minimised potential energy U*
  and of the pressure P* at a FIRE minimum x*(theta) with respect to the
  shape constants (ea, el, eb) and calA0.  At a minimum F(x*, theta) = 0, so

      dU*/dtheta = dU/dtheta + lam_U . dF/dtheta,   H lam_U = dU/dx = -F,
      dP*/dtheta = dP/dtheta + lam_P . dF/dtheta,   H lam_P = dP/dx,

  with H the Hessian at x* (cr_hessian_solve, conjugate gradients on H-vector
  products), and dU/dtheta, dP/dtheta, dF/dtheta, dP/dx the fixed-position
  derivatives of cr_param_derivatives (lam_U vanishes with F; it is solved
  for anyway so both gradients take the same path).

* ``nve_gradient``: d J / d(x0, v0) of J = U(x_N) + |v_N|^2 / 2 after N
  velocity-Verlet steps, by the adjoint of the Verlet map with checkpoints:
  the forward run keeps (x, v) every ``checkpoint`` steps, the backward pass
  re-runs each segment from its checkpoint and applies, per step,

      v_{n+1} = v_h + h/2 F(x_{n+1}):  xb -= h/2 H(x_{n+1}) vb
      x_{n+1} = x_n + h v_h:           vb += h xb
      v_h = v_n + h/2 F(x_n):          xb -= h/2 H(x_n) vb

  (xb, vb the adjoints; H symmetric), starting from xb = -F(x_N), vb = v_N.
"""
from __future__ import annotations

import numpy as np

from .dpm2d import DPM2D

PARAMS = ("ea", "el", "eb", "calA0")


def minimized_gradients(d: DPM2D, calA0: float, tol: float = 1e-10, max_iter: int = 200000) -> dict:
    """Gradients of U* and P* at the current (minimised) state of ``d``."""
    d.calcNeighborList(d.setDisplacementCutoff(0.5, 2.0 * d.getMeanVertexRadius()))
    d.calcForceEnergy()
    U = d.getPotentialEnergy()
    P = d.calcPressure()
    F = d.getVertexForces()
    out = {"U": U, "P": P, "dU": {}, "dP": {}, "cg": {}}
    rhs_U = -F
    lam_U, itU, rrU = d.hessianSolve(rhs_U, tol, max_iter)
    _, _, _, dPdx = d.paramDerivatives("ea")
    lam_P, itP, rrP = d.hessianSolve(dPdx, tol, max_iter)
    out["cg"] = {"U": (itU, rrU), "P": (itP, rrP)}
    for name in PARAMS:
        key = "lnCalA0" if name == "calA0" else name
        dU, dP, dF, _ = d.paramDerivatives(key)
        gU = dU + float(lam_U @ dF)
        gP = dP + float(lam_P @ dF)
        if name == "calA0":  # chain rule from ln(calA0)
            gU, gP = gU / calA0, gP / calA0
        out["dU"][name] = gU
        out["dP"][name] = gP
    return out


def _energy(d: DPM2D) -> float:
    return d.getPotentialEnergy() + d.getKineticEnergy()


def _refresh(d: DPM2D, x: np.ndarray, v: np.ndarray | None = None) -> None:
    d.setVertexPositions(x)
    if v is not None:
        d.setVertexVelocities(v)
    d.calcNeighborList(d.setDisplacementCutoff(0.5, 2.0 * d.getMeanVertexRadius()))
    d.calcForceEnergy()


def nve_run(d: DPM2D, x0: np.ndarray, v0: np.ndarray, nsteps: int, dt: float) -> float:
    """J after nsteps velocity-Verlet steps from (x0, v0)."""
    d.setTimeStep(dt)
    _refresh(d, x0, v0)
    d.initNVE(0.0, readState=True)
    d.NVELoop(nsteps)
    return _energy(d)


def nve_gradient(d: DPM2D, x0: np.ndarray, v0: np.ndarray, nsteps: int, dt: float, checkpoint: int = 20):
    """(J, dJ/dx0, dJ/dv0) with checkpoints every ``checkpoint`` steps."""
    d.setTimeStep(dt)
    h = dt
    _refresh(d, x0, v0)
    d.initNVE(0.0, readState=True)
    cps = [(x0.copy(), v0.copy())]
    done = 0
    while done < nsteps:
        n = min(checkpoint, nsteps - done)
        d.NVELoop(n)
        done += n
        cps.append((d.getVertexPositions(), d.getVertexVelocities()))
    J = _energy(d)
    xN, vN = cps[-1]
    _refresh(d, xN)
    xb = -d.getVertexForces()
    vb = vN.copy()
    seg_starts = list(range(0, nsteps, checkpoint))
    for k in reversed(range(len(seg_starts))):
        n0 = seg_starts[k]
        n1 = min(n0 + checkpoint, nsteps)
        # recompute the segment's positions x_n0 .. x_n1
        xs = [cps[k][0]]
        _refresh(d, cps[k][0], cps[k][1])
        d.initNVE(0.0, readState=True)
        for _ in range(n1 - n0):
            d.NVELoop(1)
            xs.append(d.getVertexPositions())
        for m in reversed(range(n1 - n0)):
            _refresh(d, xs[m + 1])
            xb = xb - 0.5 * h * d.hvp(vb)
            vb = vb + h * xb
            _refresh(d, xs[m])
            xb = xb - 0.5 * h * d.hvp(vb)
    return J, xb, vb
