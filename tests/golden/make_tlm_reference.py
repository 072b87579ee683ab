"""Tangent-linear FP64 derivatives of the time-averaged drag for the adjoint
configuration, computed by the reference's own TimeLoop on forward-mode dual
numbers (oracle/_ref/liboctlb_ref_tlm.so, `make -C oracle tlm REF=<reference tree>`), and saved as
golden values beside the finite-difference ones of make_adjoint_reference.py:

  adjoint_c5_tlm.npz        1,000 advance_one calls, objective over the last 250
  adjoint_c5_short_tlm.npz  24 calls, objective over the last 12

One run carries every direction at once: derivative 0 = d/d u_max (every
tree-boundary wall velocity seeded with d u_w / u_w = 1 / u_max), 1 = d/d tau
(d omega / d tau = -omega^2: TimeLoop's omega and LevelCoupler's scales
follow), 2..9 = the 8 seeded body-force directions of
make_adjoint_reference.directions().  Exact derivatives of the discrete
FP64 map, so they pin both the GPU adjoint and the finite differences.

  python tests/golden/make_tlm_reference.py [--steps 1000 --window 250 --out adjoint_c5_tlm.npz]
  python tests/golden/make_tlm_reference.py --steps 24 --window 12 --out adjoint_c5_short_tlm.npz
"""
import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
from make_adjoint_reference import case, directions, SEED  # noqa: E402


def tlm_objective(steps, window, u_max=0.05, progress=False):
    """(J, dJ/du_max, dJ/dtau, dJ . d_k for the 8 body-force directions)."""
    sys.path.insert(0, ROOT)
    from oracle import oracle
    L = oracle.load("tlm")
    if L is None:
        raise RuntimeError("oracle/_ref/liboctlb_ref_tlm.so is missing: make -C oracle tlm REF=<reference tree>")
    mesh, init, info = case(u_max)
    nd = L.tlm_dirs()
    omega = info["omega"]
    om_seed = np.zeros(nd)
    om_seed[1] = -omega * omega
    wall_seed = np.zeros(nd)
    wall_seed[0] = 1.0 / u_max
    d = directions(mesh)
    dirs = np.zeros((nd,) + d.shape[1:])
    dirs[2:2 + len(d)] = d
    sim = oracle.Sim(L, mesh, omega, init, link_mode=True, omega_seed=om_seed, wall_seed=wall_seed)
    sim.set_body_force_tlm(None, dirs)
    J, dJ = 0.0, np.zeros(nd)
    t0 = time.time()
    for s in range(steps):
        sim.advance(1)
        if s >= steps - window:
            f, df = sim.drag_tlm(mesh.obstacle)
            J += f[0]
            dJ += df[0]
        if progress and (s + 1) % 50 == 0:
            print(f"{s + 1}/{steps} {time.time() - t0:.0f}s", flush=True)
    return J / window, dJ[0] / window, dJ[1] / window, dJ[2:2 + len(d)] / window


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--window", type=int, default=250)
    ap.add_argument("--out", default="adjoint_c5_tlm.npz")
    args = ap.parse_args()
    J, du, dtau, ddir = tlm_objective(args.steps, args.window, progress=True)
    np.savez(os.path.join(HERE, args.out), steps=args.steps, window=args.window, seed=SEED, u_max=0.05,
             tau=case()[2]["tau"], J=J, dJ_du=du, dJ_dtau=dtau, dJ_dir=ddir)
    print("J", J, "dJ/du_max", du, "dJ/dtau", dtau, "dJ.dir", ddir)


if __name__ == "__main__":
    main()
