"""Case builders: the callers of the per-level step (the reference's
examples/cavity3d and examples/cylinder3d drivers play this role).

Each builder returns (mesh, init_pops, info) with synthetic, seeded inputs of
the shapes the benchmark configurations name:

* ``tgv_periodic``   periodic box, Taylor-Green vortex initial condition
* ``cavity_shell``   lid-driven cavity as one block with a solid shell and a
                     moving top layer (half-way bounce-back + moving-wall term)
* ``cavity_forest``  lid-driven cavity on an octree forest with tree-boundary
                     walls (optionally a refined band under the lid)
* ``cylinder_forest`` channel flow past a cylinder: exact-circle Bouzidi q,
                     parabolic inlet, zero-gradient outlet, refinement near the
                     cylinder
* ``cavity3d``       the reference's cavity3d example itself: one block of
                     resolution + 1 lattice nodes per axis, InterpolatedVelocity
                     on every face with the lid on y+, ConstRhoBGK, parameters
                     from the reference's UnitConverter
"""
import math

import numpy as np

from . import (Forest, Mesh, Q, C, feq, BULK, SOLID, BOUZIDI, TB_WALL, TB_OUTFLOW, FD_VELOCITY)


def tgv_fields(nx, ny, nz, u0):
    """Taylor-Green vortex on an nx*ny*nz periodic box, k = 2 pi / n per axis."""
    x = (np.arange(nx) + 0.5) * 2 * math.pi / nx
    y = (np.arange(ny) + 0.5) * 2 * math.pi / ny
    z = (np.arange(nz) + 0.5) * 2 * math.pi / nz
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    u = np.stack([u0 * np.sin(X) * np.cos(Y) * np.cos(Z),
                  -u0 * np.cos(X) * np.sin(Y) * np.cos(Z),
                  np.zeros_like(X)], axis=-1)
    p = u0 * u0 / 16.0 * (np.cos(2 * X) + np.cos(2 * Y)) * (np.cos(2 * Z) + 2.0)
    rho = 1.0 + 3.0 * p
    return rho, u


def tgv_periodic(n, u0=0.05, tau=0.55):
    rho, u = tgv_fields(n, n, n, u0)
    mesh = Mesh(n, [0], [0, 0, 0, 1, 1, 1], periodic=1)
    init = feq(rho, u).reshape(1, n, n, n, Q)
    return mesh, init, {"omega": 1.0 / tau, "tau": tau}


def cavity_shell(n=32, lid=0.1, tau=0.6):
    """(n+2)^3 block: solid shell, fluid n^3, top (+y) shell layer moves with
    (lid, 0, 0).  Links stream rule with q = 1 everywhere (half-way
    bounce-back), the moving-wall term on links pulled from the lid."""
    m = n + 2
    kinds = np.full((m, m, m), SOLID, np.uint8)
    kinds[1:-1, 1:-1, 1:-1] = BULK
    moving = np.zeros((m, m, m), np.uint8)
    moving[:, -1, :] = 1
    wall_u = np.zeros((m, m, m, 3))
    wall_u[:, -1, :, 0] = lid
    mesh = Mesh(m, [0], [0, 0, 0, 1, 1, 1], kinds=kinds[None], moving=moving[None], wall_u=wall_u[None])
    init = np.zeros((1, m, m, m, Q))
    return mesh, init, {"omega": 1.0 / tau, "tau": tau}


def _tb_spec(forest, fn):
    spec = np.zeros((len(forest.tree_boundary), 8))
    for k, (b, d) in enumerate(forest.tree_boundary):
        spec[k] = fn(int(b), int(d))
    return spec


def cavity_forest(cells=32, n=8, lid=0.1, tau=0.6, band_cells=0):
    """Cavity of cells^3 base cells in blocks of n^3, walls on every tree
    boundary, +y wall moving with (lid,0,0).  band_cells > 0 refines the top
    band of that many base cells one level (2:1)."""
    assert cells % n == 0
    base = int(round(math.log2(cells // n)))
    f = Forest((1, 1, 1), (0, 0, 0), (0, 0, 0, 1, 1, 1)).refine_uniform(base)
    if band_cells:
        h = band_cells / cells
        f.refine_box((0, 1 - h, 0, 1, 1, 1), base + 1)
    f.balance().build()

    def spec(b, d):
        if d == 3:
            return [TB_WALL, lid, 0, 0, -1, 0, 0, 0]
        return [TB_WALL, 0, 0, 0, -1, 0, 0, 0]

    mesh = Mesh.from_forest(f, n, tree_boundary_spec=_tb_spec(f, spec))
    init = np.zeros((mesh.n_blocks, n, n, n, Q))
    return mesh, init, {"omega": 1.0 / tau, "tau": tau, "forest": f}


def cavity3d(resolution=30, tau=0.509, phys_length=1.0, phys_velocity=1.0, phys_viscosity=0.001):
    """The reference's cavity3d case (examples/cavity3d/cavity3d_case.h:
    41-106, 148-197): one block of resolution + 1 nodes per axis at rest,
    every face InterpolatedVelocity, the y+ face moving with the lid's
    lattice velocity along x; ConstRhoBGK with the boundary cells in the
    statistics.  The lattice velocity and omega follow the reference's
    UnitConverter (unit_converter.cpp:8-26): dx = L / resolution,
    dt = (tau - 1/2) / 3 dx^2 / nu, u_lid = U dt / dx, omega = 1 / tau.
    Returns (mesh, init_pops, info); info holds the face types and wall
    velocities for GpuLattice.set_fd_boundary (the mesh still needs
    stamp_fd_kinds)."""
    n = resolution + 1
    dx = phys_length / resolution
    dt = (tau - 0.5) / 3.0 * dx * dx / phys_viscosity
    u_lid = phys_velocity * dt / dx
    mesh, init, _ = cavity_forest(cells=n, n=n, lid=0.0, tau=tau)
    u_wall = np.zeros((6, 3))
    u_wall[3, 0] = u_lid
    return mesh, init, {"omega": 1.0 / tau, "tau": tau, "u_lid": u_lid, "dx": dx, "resolution": resolution,
                        "phys_length": phys_length, "types": [FD_VELOCITY] * 6, "u_wall": u_wall}


def cavity3d_centerline(ux, info, y_over_h):
    """u / u_lid on the cavity's vertical centerline x = z = L / 2 at the
    heights y_over_h, sampled as the reference samples it
    (cavity3d_case.h:232-300, 323-337): trilinear interpolation between
    lattice nodes i dx, base node floor(coord / dx) clamped to [0, n - 2];
    the Dirichlet cells carry their prescribed velocity (the lid's on the
    interior top-face cells, 0 elsewhere on the faces).  ux: [n, n, n] x
    velocity of the block's cells."""
    n = ux.shape[0]
    dx, lid, L = info["dx"], info["u_lid"], info["phys_length"]
    u = np.array(ux, dtype=np.float64)
    face = np.zeros((n, n, n), bool)
    face[[0, -1], :, :] = face[:, [0, -1], :] = face[:, :, [0, -1]] = True
    u[face] = 0.0
    u[1:-1, -1, 1:-1] = lid

    def base(c):
        return min(max(int(math.floor(c / dx)), 0), n - 2)

    def sample(x, y, z):
        i, j, k = base(x), base(y), base(z)
        wx, wy, wz = (x - i * dx) / dx, (y - j * dx) / dx, (z - k * dx) / dx
        c = u[i:i + 2, j:j + 2, k:k + 2]
        cx_ = c[0] * (1 - wx) + c[1] * wx
        cy_ = cx_[0] * (1 - wy) + cx_[1] * wy
        return cy_[0] * (1 - wz) + cy_[1] * wz

    return np.array([sample(0.5 * L, yh * L, 0.5 * L) / lid for yh in y_over_h])


def relative_l2(sim, ref):
    """sqrt(sum (sim - ref)^2 / sum ref^2) (cavity3d_case.h:128-139)."""
    sim, ref = np.asarray(sim, np.float64), np.asarray(ref, np.float64)
    return float(np.sqrt(np.sum((sim - ref) ** 2) / np.sum(ref * ref)))


def circle_links(mesh, center, radius, axis_free=2):
    """Exact-circle Bouzidi q for every non-solid cell x and D3Q19 direction i
    whose source x - c_i is an in-block cell inside the circle (cylinder along
    `axis_free`): q is the first root t in (0, 1] of |x - t c_i dx - center| = R
    (host FP64), the fraction of the link from x to the wall.  Marks the cells
    inside as SOLID in mesh.kinds."""
    n = mesh.n
    ax = [a for a in range(3) if a != axis_free]
    cells, qs = [], []
    idx = np.arange(n)
    for b in range(mesh.n_blocks):
        bd = mesh.bounds[b]
        dx = (bd[3] - bd[0]) / n
        ctr = [bd[a] + (idx + 0.5) * dx for a in range(3)]
        X = np.meshgrid(*ctr, indexing="ij")
        px, py = X[ax[0]] - center[0], X[ax[1]] - center[1]
        inside = px * px + py * py < radius * radius
        if not inside.any():
            continue
        kinds = mesh.kinds[b]
        kinds[inside] = SOLID
        solid = kinds == SOLID
        for i in range(1, Q):
            c = C[i]
            # x - c_i in block and solid, x itself not solid
            src = np.zeros((n, n, n), bool)
            sl_dst = tuple(slice(max(0, c[a]), n + min(0, c[a])) for a in range(3))
            sl_src = tuple(slice(max(0, -c[a]), n - max(0, c[a])) for a in range(3))
            src[sl_dst] = solid[sl_src]
            cand = src & ~solid
            if not cand.any():
                continue
            d = -c.astype(float) * dx
            dx_, dy_ = d[ax[0]], d[ax[1]]
            a2 = dx_ * dx_ + dy_ * dy_
            if a2 == 0.0:
                continue
            qx, qy = px[cand], py[cand]
            b2 = 2 * (qx * dx_ + qy * dy_)
            c2 = qx * qx + qy * qy - radius * radius
            disc = b2 * b2 - 4 * a2 * c2
            ok = disc >= 0
            t = np.full(qx.shape, -1.0)
            t[ok] = (-b2[ok] - np.sqrt(disc[ok])) / (2 * a2)
            good = (t > 0.0) & (t <= 1.0)
            xyz = np.argwhere(cand)[good]
            for (x, y, z), tt in zip(xyz, t[good]):
                cells.append((b, x, y, z, i))
                qs.append(tt)
    mesh.link_cells = np.asarray(cells, np.int32).reshape(-1, 5)
    mesh.link_q = np.asarray(qs, np.float64)
    return mesh


def cylinder_forest(length=256, height=64, n=8, diameter=16.0, center=(64.0, 32.0), levels=3,
                    refine_dist=None, u_max=0.05, re=100.0, periodic_z=True):
    """Channel length x height x height finest cells, cylinder along z.

    Level L-1 (finest) covers the box within refine_dist (default 2D) of the
    cylinder surface; coarser levels elsewhere, 2:1 balanced.  Inlet -x:
    moving wall with a parabolic profile in y (u_max at mid-height);
    outlet +x: zero-gradient ghost copy; y walls: half-way bounce-back;
    z periodic.  Returns mesh, initial state (rest), info with omega of the
    finest level for Re = u_max D / nu."""
    fine = 2 ** (levels - 1)
    base_cells = height // fine            # coarsest cells across the height
    assert base_cells % n == 0 and length % height == 0
    bx = length // height
    tree_cells = height                    # finest cells per tree edge
    base_level = int(round(math.log2(base_cells // n)))
    f = Forest((bx, 1, 1), (0, 0, 1 if periodic_z else 0), (0, 0, 0, float(length), float(height), float(height)))
    f.refine_uniform(base_level)
    rd = 2.0 * diameter if refine_dist is None else refine_dist
    for k in range(1, levels):
        # finest level within rd of the surface, each coarser level twice as far
        r = diameter / 2 + rd * 2 ** (levels - 1 - k)
        f.refine_box((center[0] - r, center[1] - r, -1, center[0] + r, center[1] + r, height + 1), base_level + k)
    f.balance().build()

    def spec(b, d):
        if d == 0:
            return [TB_WALL, u_max, 0, 0, 1, 0.0, float(height), 0]
        if d == 1:
            return [TB_OUTFLOW, 0, 0, 0, -1, 0, 0, 0]
        return [TB_WALL, 0, 0, 0, -1, 0, 0, 0]

    mesh = Mesh.from_forest(f, n, tree_boundary_spec=_tb_spec(f, spec))
    circle_links(mesh, center, diameter / 2.0)
    # obstacle mask for the momentum exchange: the cylinder's solid cells
    mesh.obstacle = (mesh.kinds == SOLID).astype(np.uint8)
    nu = u_max * diameter / re                  # finest-level lattice units
    tau = 3.0 * nu + 0.5
    init = np.zeros((mesh.n_blocks, n, n, n, Q))
    return mesh, init, {"omega": 1.0 / tau, "tau": tau, "forest": f, "tree_cells": tree_cells}


# The adjoint configuration: channel 128x32x32 finest cells, two levels, D = 8,
# Re = 40; body-force perturbation directions drawn from a recorded seed.
ADJOINT_SEED = 20261203
ADJOINT_DIRS = 8


def adjoint_channel(u_max=0.05, tau=None):
    """The adjoint channel; tau defaults to the Re = 40 value."""
    mesh, init, info = cylinder_forest(length=128, height=32, n=8, diameter=8.0, center=(32.0, 16.0),
                                       levels=2, u_max=u_max, re=40.0)
    if tau is not None:
        info["tau"], info["omega"] = tau, 1.0 / tau
    return mesh, init, info


def adjoint_directions(mesh, seed=ADJOINT_SEED, count=ADJOINT_DIRS):
    """Per-cell body-force directions d ~ N(0, 1e-6), [count][blocks][n^3][3]."""
    rng = np.random.default_rng(seed)
    return rng.normal(0.0, 1e-6, size=(count, mesh.n_blocks, mesh.n ** 3, 3))
