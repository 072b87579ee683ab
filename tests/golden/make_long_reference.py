"""Long FP64 runs of the reference's own TimeLoop (oracle/_ref) for the
benchmark configurations, saved as small golden vectors:

  long_c1_cavity.npz    32^3 lid-driven cavity (4^3 leaves of 8^3 cells),
                        tau 0.6, lid 0.1, 250 coarse steps (1,000 cell steps):
                        final rho, u (float32)
  long_c2_amr.npz       two-level cavity, 64^3 base + refined band under the
                        lid, tau 0.56 (one global omega), lid 0.05, 625 coarse
                        steps (5,000 base-level steps): total mass per coarse
                        step, centreline velocity profiles at the end, the
                        final rho and u (float32) on every cell of even local
                        indices (1 in 8, all blocks), and sum |u|^2, sum rho
                        over all cells
  long_c2_amr_physical.npz  the same cavity with tau rescaled per level
                        (tau_coarse 0.56, tau_fine 0.62: the physical coupler
                        mode, restated around the reference's components), the
                        same records
  long_c3_cylinder.npz  three-level channel 256x64x64 finest cells, D = 16
                        exact-circle Bouzidi cylinder, u_max 0.05, Re 100,
                        2,500 coarse steps (20,000 finest steps): the
                        momentum-exchange force after every coarse step

Run from the repository root:
  python tests/golden/make_long_reference.py c1|c2|c3|c2p [--out DIR]
Full final fields are also written (float32) to DIR when given.
"""
import argparse
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle  # noqa: E402
from octlb_b200 import cases  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def config(name):
    if name == "c1":
        mesh, init, info = cases.cavity_forest(cells=32, n=8, lid=0.1, tau=0.6)
        return mesh, init, info, 250, False
    if name == "c2":
        mesh, init, info = cases.cavity_forest(cells=64, n=8, lid=0.05, tau=0.56, band_cells=8)
        return mesh, init, info, 625, False
    if name == "c3":
        mesh, init, info = cases.cylinder_forest()
        return mesh, init, info, 2500, True
    if name == "c2p":  # C2 with tau rescaled per level (physical coupler mode)
        mesh, init, info = cases.cavity_forest(cells=64, n=8, lid=0.05, tau=0.56, band_cells=8)
        return mesh, init, info, 625, False
    raise ValueError(name)


def physical_omegas(mesh, tau):
    """Per-level rates of the physical coupler mode: tau_{l+1} - 1/2 =
    2 (tau_l - 1/2) from the coarsest level with blocks."""
    lmin, lmax = int(mesh.levels.min()), int(mesh.levels.max())
    return np.array([1.0 / (2.0 ** (l - lmin) * (tau - 0.5) + 0.5) for l in range(lmax + 1)])


def centerlines(mesh, rho, u):
    """u_x along y and u_y along x through the box centre (z = 0.5), taken from
    the cells whose boxes contain the lines (any level)."""
    n = mesh.n
    out = {}
    for name, axis, comp in (("ux_of_y", 1, 0), ("uy_of_x", 0, 1)):
        pos, val = [], []
        for b in range(mesh.n_blocks):
            bd = mesh.bounds[b]
            dx = (bd[3] - bd[0]) / n
            other = [a for a in (0, 1) if a != axis][0]
            ok = True
            idx = []
            for a, c in ((other, 0.5), (2, 0.5)):
                if not (bd[a] <= c < bd[3 + a]):
                    ok = False
                idx.append(int((c - bd[a]) / dx) if ok else 0)
            if not ok:
                continue
            for k in range(n):
                ijk = [0, 0, 0]
                ijk[axis] = k
                ijk[other] = idx[0]
                ijk[2] = idx[1]
                pos.append(bd[axis] + (k + 0.5) * dx)
                val.append(u[b, ijk[0], ijk[1], ijk[2], comp])
        order = np.argsort(pos)
        out[name + "_pos"] = np.asarray(pos)[order]
        out[name] = np.asarray(val)[order]
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("name", choices=["c1", "c2", "c3", "c2p"])
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    ref = oracle.load("ref")
    assert ref is not None, "build oracle/_ref first (make -C oracle ref REF=<reference tree>)"
    mesh, init, info, steps, links = config(args.name)
    sim = oracle.Sim(ref, mesh, info["omega"], init, link_mode=links)
    if args.name == "c2p":
        sim.set_physical(physical_omegas(mesh, info["tau"]))
    forces, masses = [], []
    t0 = time.time()
    for s in range(steps):
        sim.advance(1)
        if args.name == "c3":
            forces.append(sim.drag(mesh.obstacle))
        if args.name in ("c2", "c2p"):
            rho, _ = oracle.rho_u(sim.core())
            masses.append(rho[mesh.kinds == 0].sum())
        if s % 50 == 0:
            print(args.name, s, time.time() - t0, flush=True)
    rho, u = oracle.rho_u(sim.core())
    if args.out:
        os.makedirs(args.out, exist_ok=True)
        np.savez_compressed(os.path.join(args.out, f"full_{args.name}.npz"), rho=rho.astype(np.float32),
                            u=u.astype(np.float32))
    if args.name == "c1":
        np.savez_compressed(os.path.join(HERE, "long_c1_cavity.npz"), steps=steps,
                            rho=rho.astype(np.float32), u=u.astype(np.float32))
    elif args.name in ("c2", "c2p"):
        # the final fields on the cells of even local indices (1 cell in 8,
        # every block of both levels) for the field-wide L2 of u, and the sums
        # of |u|^2 and rho over every cell
        lat = (slice(None), slice(0, None, 2), slice(0, None, 2), slice(0, None, 2))
        np.savez_compressed(os.path.join(HERE, "long_c2_amr.npz" if args.name == "c2" else "long_c2_amr_physical.npz"),
                            steps=steps, mass=np.asarray(masses),
                            lattice_rho=rho[lat].astype(np.float32), lattice_u=u[lat].astype(np.float32),
                            sum_u2=float(np.sum(u * u)), sum_rho=float(np.sum(rho)),
                            **centerlines(mesh, rho, u))
    else:
        np.savez_compressed(os.path.join(HERE, "long_c3_cylinder.npz"), steps=steps, force=np.asarray(forces))
    print(args.name, "done", time.time() - t0)


if __name__ == "__main__":
    main()
