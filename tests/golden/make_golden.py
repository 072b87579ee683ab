"""Generates the golden vectors in this folder from the reference's own code
(oracle/_ref/liboctlb_ref.so, built by `make -C oracle ref REF=<reference tree>` from the reference
sources).  Run from the repository root:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from oracle import oracle  # noqa: E402
from test_oracle_pins import link_case  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    ref = oracle.load("ref")
    assert ref is not None, "build oracle/_ref first (make -C oracle ref REF=<reference tree>)"
    n, steps, omega = 6, 7, 1.7
    rng = np.random.default_rng(11)
    pin = rng.standard_normal((n + 2, n + 2, n + 2, 19)) * 1e-3
    b = oracle.Block(ref, n)
    b.set_padded(pin)
    b.run_periodic(omega, steps)
    pout = b.padded()
    lb = link_case(ref)
    np.savez_compressed(os.path.join(HERE, "block_paths.npz"), periodic_n=n, periodic_steps=steps,
                        periodic_omega=omega, periodic_in=pin, periodic_out=pout,
                        links_out=lb.padded(), links_drag=lb.drag())

    from octlb_b200 import cases
    mesh, init, info = cases.cavity_forest(cells=16, n=8, lid=0.1, tau=0.6, band_cells=8)
    sim = oracle.Sim(ref, mesh, info["omega"], init)
    sim.advance(3)
    rho, u = oracle.rho_u(sim.core())
    np.savez_compressed(os.path.join(HERE, "amr_cavity.npz"), levels=mesh.levels, steps=3, rho=rho, u=u)
    print("golden vectors written")


if __name__ == "__main__":
    main()
