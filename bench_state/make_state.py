"""Writes the benchmark's prepared input state, bench_state/smooth_lj_1024.npz.

The smooth-LJ workload (1024 deformable rings, nv 32/45 bidisperse 1:1.4,
smooth vertex-segment LJ rc 2.5, calA0 1.05, shape constants ea 1e5, el 20,
eb 10) placed without overlap at phi 0.40 (seed 20261203), compressed to
phi 0.85 with FIRE and relaxed (cudaring_b200.workloads.prepared_deformable).
Both arms of bench.py start from this file, so the reference arm needs
neither the GPU library nor the 52k FIRE iterations of the preparation.
Velocities are not stored: each run draws them from its own seed.

    python bench_state/make_state.py        (needs a CUDA device)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))


def main(out: str = os.path.join(HERE, "smooth_lj_1024.npz")) -> None:
    from cudaring_b200 import workloads

    d, info = workloads.prepared_deformable("smooth_lj", 1024, seed=20261203)
    np.savez_compressed(out, nv_list=d.numVertexInParticleList, pos=d.getVertexPositions(), rad=d.getVertexRadii(),
                        l0=d.getRestLengths(), theta0=d.getRestAngles(), a0=d.getRestAreas(), box=d.getBoxSize(),
                        fire_iterations=info["fire_iterations"], max_force=info["max_force"], phi=info["phi"],
                        seed=info["seed"])
    d.close()
    print(f"wrote {out}: {int(d.numVertices)} vertices, phi {info['phi']:.4f}, "
          f"{info['fire_iterations']} FIRE iterations, max |F| {info['max_force']:.2e}")


if __name__ == "__main__":
    main(*sys.argv[1:])
