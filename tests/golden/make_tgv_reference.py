"""FP64 reference run of the throughput configuration's physics at 64^3:
the Taylor-Green vortex (u0 = 0.05, tau = 0.55, k = 2 pi / 64) on a periodic
box, stepped by the reference's own BlockLattice<double> collide ->
fill_periodic_halo -> stream (oracle/_ref; block_lattice.cpp:376-417,
918-964, 502-721), 1,000 steps.  Saved as tgv64_reference.npz:

  ke[k], mass[k]    kinetic energy sum(rho |u|^2 / 2) and mass sum(rho) after
                    10 k steps, k = 0..100 (FP64)
  sample_rho/u      rho and u after 1,000 steps on the cells [2::4]^3 (16^3)
  sum_u2, sum_rho   sum |u|^2 and sum rho over every cell after 1,000 steps

  python tests/golden/make_tgv_reference.py     (about a minute, one core)
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N, U0, TAU, STEPS, EVERY = 64, 0.05, 0.55, 1000, 10
SAMPLE = (slice(2, None, 4),) * 3


def energy(rho, u):
    return 0.5 * float(np.sum(rho * np.sum(u * u, axis=-1))), float(np.sum(rho))


def main():
    from oracle import oracle
    from octlb_b200 import cases
    ref = oracle.load("ref")
    assert ref is not None, "build oracle/_ref first (make -C oracle ref REF=<reference tree>)"
    mesh, init, info = cases.tgv_periodic(N, u0=U0, tau=TAU)
    blk = oracle.Block(ref, N)
    blk.set_core(init[0])
    ke, mass = [], []
    rho, u = oracle.rho_u(blk.core())
    e, m = energy(rho, u)
    ke.append(e)
    mass.append(m)
    for _ in range(STEPS // EVERY):
        blk.run_periodic(info["omega"], EVERY)
        rho, u = oracle.rho_u(blk.core())
        e, m = energy(rho, u)
        ke.append(e)
        mass.append(m)
    np.savez_compressed(os.path.join(HERE, "tgv64_reference.npz"), n=N, u0=U0, tau=TAU, steps=STEPS,
                        every=EVERY, ke=np.array(ke), mass=np.array(mass), sample_rho=rho[SAMPLE],
                        sample_u=u[SAMPLE], sum_u2=float(np.sum(u * u)), sum_rho=float(np.sum(rho)))
    print("ke decay", ke[-1] / ke[0])


if __name__ == "__main__":
    main()
