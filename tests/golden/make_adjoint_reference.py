"""FP64 finite-difference derivatives of the time-averaged drag for the
adjoint configuration, computed with the reference's own TimeLoop
(oracle/_ref, FP64), and saved as golden values:

  adjoint_c5.npz   channel 128x32x32 finest cells, two levels, D = 8, Re = 40,
                   1,000 TimeLoop::advance_one calls (the forest's levels are 1
                   and 2 and the recursion starts at level 0, so each call
                   takes 4 finest steps: 4,000 finest steps); objective J = the
                   x component of MomentumExchangeDrag::force_on_fluid_if over
                   the cylinder, averaged over the last 250 calls (the last
                   1,000 finest steps).
                   Central differences, h = 1e-4 relative, for the inlet u_max
                   and tau; for the body force, J(+d) - J(-d) over 2 along each
                   of 8 directions d ~ N(0, 1e-6) per cell and component
                   (numpy default_rng(seed), seed stored).

The body force enters at the reference's DomainBoundaryHandler::apply() hook
(restated in oracle/ref_capi.cpp; the reference has none).  Runs the 21
forward runs in parallel worker processes (spawn).

  python tests/golden/make_adjoint_reference.py [--steps 1000] [--window 250] [--workers 7]
  python tests/golden/make_adjoint_reference.py --steps 24 --window 12 --out adjoint_c5_short.npz
(the second: a 24-coarse-step horizon for a quick test).
"""
import argparse
import multiprocessing as mp
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
from octlb_b200.cases import ADJOINT_SEED as SEED, ADJOINT_DIRS as N_DIRS  # noqa: E402


def case(u_max=0.05, tau=None):
    """The adjoint channel (octlb_b200.cases.adjoint_channel)."""
    from octlb_b200 import cases
    return cases.adjoint_channel(u_max, tau)


def directions(mesh):
    from octlb_b200 import cases
    return cases.adjoint_directions(mesh)


def objective(job):
    """J = mean drag x over the last `window` of `steps` coarse steps."""
    u_max, tau, dir_index, sign, steps, window = job
    sys.path.insert(0, ROOT)
    from oracle import oracle
    ref = oracle.load("ref")
    mesh, init, info = case(u_max, tau)
    sim = oracle.Sim(ref, mesh, info["omega"], init, link_mode=True)
    if dir_index >= 0:
        sim.set_body_force(sign * directions(mesh)[dir_index])
    acc = 0.0
    for s in range(steps):
        sim.advance(1)
        if s >= steps - window:
            acc += sim.drag(mesh.obstacle)[0]
    return job, acc / window


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--window", type=int, default=250)
    ap.add_argument("--workers", type=int, default=7)
    ap.add_argument("--rel", type=float, default=1e-4)
    ap.add_argument("--out", default="adjoint_c5.npz")
    args = ap.parse_args()
    u0, tau0 = 0.05, case()[2]["tau"]
    hu, ht = args.rel * u0, args.rel * tau0
    jobs = [(u0, tau0, -1, 0, args.steps, args.window),
            (u0 + hu, tau0, -1, 0, args.steps, args.window), (u0 - hu, tau0, -1, 0, args.steps, args.window),
            (u0, tau0 + ht, -1, 0, args.steps, args.window), (u0, tau0 - ht, -1, 0, args.steps, args.window)]
    for k in range(N_DIRS):
        jobs += [(u0, tau0, k, 1.0, args.steps, args.window), (u0, tau0, k, -1.0, args.steps, args.window)]
    t0 = time.time()
    res = {}
    with mp.get_context("spawn").Pool(args.workers) as pool:
        for job, J in pool.imap_unordered(objective, jobs):
            res[job] = J
            print(f"{len(res)}/{len(jobs)} {job[:4]} J={J:.15e} {time.time() - t0:.0f}s", flush=True)
    J0 = res[jobs[0]]
    dJ_du = (res[jobs[1]] - res[jobs[2]]) / (2 * hu)
    dJ_dtau = (res[jobs[3]] - res[jobs[4]]) / (2 * ht)
    dJ_dir = np.array([(res[jobs[5 + 2 * k]] - res[jobs[6 + 2 * k]]) / 2.0 for k in range(N_DIRS)])
    np.savez(os.path.join(HERE, args.out), steps=args.steps, window=args.window, seed=SEED,
             u_max=u0, tau=tau0, rel_h=args.rel, J=J0, dJ_du=dJ_du, dJ_dtau=dJ_dtau, dJ_dir=dJ_dir)
    print("J", J0, "dJ/du_max", dJ_du, "dJ/dtau", dJ_dtau, "dJ.dir", dJ_dir)


if __name__ == "__main__":
    main()
