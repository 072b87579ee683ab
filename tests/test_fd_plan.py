"""Host-side resolution of the finite-difference domain boundary pass
(octlb_fd_plan, the table octlb_gpu_set_fd_boundary uploads): the stencil of
every velocity / pressure Dirichlet cell -- its role from the block's
extents, its prescribed velocity, each velocity read (fluid cell, prescribed
velocity, overlap padding, mirror image with flipped components) and each
density read (rewritten earlier in the reference's walk or not) -- is
evaluated here in FP64 exactly as the device kernels evaluate it
(octlb_b200/csrc/lbm_fd.cu), and must reproduce the oracle's restatement of
the reference's pass (oracle/fd_boundary.py, pinned to the reference) to
1e-8 on random post-stream states (the records hold prescribed velocities
and target densities in FP32, 6e-8 relative; a wrong read is off by 1e-3): one 16^3 block (cavity3d's walls and
lid), a velocity inlet with its ramp against a pressure outlet, and eight
8^3 blocks (roles from each block's own extents)."""
import ctypes
import os
import sys

import numpy as np
import pytest

from oracle import fd_boundary as fb

HERE = os.path.dirname(os.path.abspath(__file__))

UREAD = np.dtype({"names": ["idx", "code", "flip"], "formats": ["<i8", "<i4", "<i4"], "offsets": [0, 8, 12],
                  "itemsize": 16})
RREAD = np.dtype({"names": ["idx", "val", "code", "urow", "d", "o"],
                  "formats": ["<i8", "<f4", "<i4", "<i4", "<i4", "<i4"], "offsets": [0, 8, 12, 16, 20, 24],
                  "itemsize": 32})
CELL = np.dtype({"names": ["slot", "kind", "role", "d", "o", "ax", "nrm", "u_base", "ramp_end", "rho_target", "u", "r"],
                 "formats": ["<i8", "<i4", "<i4", "<i4", "<i4", ("<i4", 3), ("<i4", 3), ("<f4", 3), "<f4", "<f4",
                             (UREAD, 7), (RREAD, 6)],
                 "offsets": [0, 8, 12, 16, 20, 24, 36, 48, 60, 64, 72, 184], "itemsize": 376})


def plan(ob, mesh, types, u_wall, rho_target, inlet=None, ramp=0.0, inlets=None):
    L = ob.capi.lib()
    assert L.octlb_fd_record_bytes() == CELL.itemsize
    t = np.ascontiguousarray(types, np.int32)
    u = np.ascontiguousarray(u_wall, np.float64)
    r = np.ascontiguousarray(rho_target, np.float64)
    iu = None if inlet is None else np.ascontiguousarray(inlet, np.float64)
    P = ctypes.POINTER
    if inlets is not None:
        arr = ob.fd_inlets(inlets)
        args = (ctypes.byref(mesh.c_tables()), t.ctypes.data_as(P(ctypes.c_int)), u.ctypes.data_as(P(ctypes.c_double)),
                r.ctypes.data_as(P(ctypes.c_double)), arr)
        n = L.octlb_fd_plan_inlets(*args, None, 0)
        assert n > 0, n
        rec = np.zeros(n, CELL)
        L.octlb_fd_plan_inlets(*args, rec.ctypes.data_as(ctypes.c_void_p), n)
        return rec
    n = L.octlb_fd_plan(ctypes.byref(mesh.c_tables()), t.ctypes.data_as(P(ctypes.c_int)),
                        u.ctypes.data_as(P(ctypes.c_double)), r.ctypes.data_as(P(ctypes.c_double)),
                        None if iu is None else iu.ctypes.data_as(P(ctypes.c_double)), float(ramp), None, 0)
    assert n > 0, n
    rec = np.zeros(n, CELL)
    L.octlb_fd_plan(ctypes.byref(mesh.c_tables()), t.ctypes.data_as(P(ctypes.c_int)),
                    u.ctypes.data_as(P(ctypes.c_double)), r.ctypes.data_as(P(ctypes.c_double)),
                    None if iu is None else iu.ctypes.data_as(P(ctypes.c_double)), float(ramp),
                    rec.ctypes.data_as(ctypes.c_void_p), n)
    return rec


def emulate(rec, state, omega, t):
    """The device pass in FP64: state [cells][19] (block-major core slots),
    returns the rewritten rows [rows][19]."""
    C, W = fb.C.astype(np.float64), fb.W

    def ramp(tt, te):
        if te <= 0:
            return 1.0
        x = min(max(tt / te, 0.0), 1.0)
        return x ** 3 * (10 + x * (-15 + 6 * x))

    def presc(row):
        c = rec[row]
        return ramp(t, float(c["ramp_end"])) * c["u_base"].astype(np.float64)

    def vel(f):
        return (C.T @ f) / (1.0 + f.sum())

    def read_u(r):
        if r["code"] == 0:
            u = np.zeros(3)
        elif r["code"] == 1:
            u = vel(state[r["idx"]])
        else:
            u = presc(r["idx"])
        for a in range(3):
            if r["flip"] >> a & 1:
                u[a] = -u[a]
        return u

    def bm(f, d, o, u):
        return (2.0 * f[C[:, d] == o].sum() + f[C[:, d] == 0].sum() + 1.0) / (1.0 + o * u[d])

    new = np.zeros((len(rec), 19))

    def read_rho(r):
        code = r["code"]
        if code == 0:
            return float(r["val"])
        f = state[r["idx"]] if code in (1, 3) else new[r["idx"]]
        if code in (1, 2):
            return 1.0 + f.sum()
        return bm(f, r["d"], r["o"], presc(r["urow"]))

    def normal(u0, u1, u2, nn):
        return -nn * (-3 * u0 + 4 * u1 - u2) / 2

    for role in (1, 2, 3):
        for row in np.nonzero(rec["role"] == role)[0]:
            c = rec[row]
            uu = [read_u(c["u"][j]) for j in range(7)]
            du = [None] * 3
            if role == 1:
                d, o = int(c["d"]), int(c["o"])
                rho = float(c["rho_target"]) if c["kind"] == 6 else bm(state[c["slot"]], d, o, uu[0])
                du[d] = normal(uu[0], uu[1], uu[2], o)
                t0 = min((d + 1) % 3, (d + 2) % 3)
                t1 = 3 - d - t0
                du[t0] = (uu[3] - uu[4]) / 2
                du[t1] = (uu[5] - uu[6]) / 2
            elif role == 2:
                p, d1, d2 = c["ax"]
                du[p] = (uu[1] - uu[2]) / 2
                du[d1] = normal(uu[0], uu[3], uu[4], c["nrm"][0])
                du[d2] = normal(uu[0], uu[5], uu[6], c["nrm"][1])
                r = [read_rho(c["r"][j]) for j in range(4)]
                rho = 2 / 3 * (r[0] + r[1]) - 1 / 6 * (r[2] + r[3])
            else:
                for a in range(3):
                    du[a] = normal(uu[0], uu[1 + 2 * a], uu[2 + 2 * a], c["nrm"][a])
                r = [read_rho(c["r"][j]) for j in range(6)]
                rho = 4 / 9 * (r[0] + r[1] + r[2]) - 1 / 9 * (r[3] + r[4] + r[5])
            s = -rho / 3.0 / omega
            pi = np.array([2 * du[0][0], du[0][1] + du[1][0], du[0][2] + du[2][0], 2 * du[1][1],
                           du[1][2] + du[2][1], 2 * du[2][2]]) * s
            new[row] = fb._eq(rho, uu[0]) + fb._fneq_from_pi(pi)
    return new


def check(ob, mesh, types, u_wall, rho_target, inlet=None, ramp=0.0, t=0.0, seed=3, inlets=None):
    stamped = ob.stamp_fd_kinds(mesh, types)
    rec = plan(ob, stamped, types, u_wall, rho_target, inlet, ramp, inlets)
    n = mesh.n
    rng = np.random.default_rng(seed)
    fpre = 0.01 * rng.standard_normal((mesh.n_blocks, n, n, n, 19))
    omega = 1.0 / 0.6
    new = emulate(rec, fpre.reshape(-1, 19), omega, t)
    specs = None
    if inlets is not None:
        specs = {f: d for f, d in enumerate(inlets) if d is not None}
    elif inlet is not None:
        specs = {f: (inlet[f], ramp) for f in range(6) if np.any(inlet[f] != 0)}
    worst = 0.0
    for b in range(mesh.n_blocks):
        bd = np.asarray(mesh.bounds[b], np.float64)
        want = fb.reconstruct(fpre[b], stamped.kinds[b], omega, u_lid=u_wall[3], rho_target=rho_target,
                              inlets=specs, t=t, origin=bd[:3], cell_width=(bd[3] - bd[0]) / n)
        got = fpre[b].copy().reshape(-1, 19)
        sl = rec["slot"]
        mine = ((sl // n ** 3) == b) & (rec["role"] >= 1)  # role 0: bounce-back, not rewritten
        got[sl[mine] % n ** 3] = new[mine]
        worst = max(worst, float(np.abs(got.reshape(want.shape) - want).max()))
    assert worst <= 1e-8, worst
    return rec


def test_cavity_walls_and_lid(ob):
    from octlb_b200 import cases
    mesh, init, info = cases.cavity_forest(cells=16, n=16, lid=0.0, tau=0.6)
    u = np.zeros((6, 3))
    u[3, 0] = 0.05
    rec = check(ob, mesh, [ob.FD_VELOCITY] * 6, u, np.ones(6))
    assert set(np.unique(rec["role"])) == {1, 2, 3}


def test_inlet_ramp_and_pressure_outlet(ob):
    from octlb_b200 import cases
    mesh, init, info = cases.cavity_forest(cells=16, n=16, lid=0.0, tau=0.6)
    types = [ob.FD_VELOCITY, ob.FD_PRESSURE] + [ob.FD_VELOCITY] * 4
    u = np.zeros((6, 3))
    inlet = np.zeros((6, 3))
    inlet[0, 0] = 0.02
    rho = np.ones(6)
    rho[1] = 1.002
    for t in (0.0, 7.0, 40.0):
        check(ob, mesh, types, u, rho, inlet, ramp=20.0, t=t)


def test_eight_blocks_roles_from_block_extents(ob):
    sys.path.insert(0, HERE)
    from test_const_rho import brick_cavity
    mesh, info = brick_cavity(lid=0.0, n=8)
    u = np.zeros((6, 3))
    u[3, 0] = 0.05
    check(ob, mesh, [ob.FD_VELOCITY] * 6, u, np.ones(6))


def test_pressure_outlet_across_blocks(ob):
    """A pressure outlet on x+ spanning four 8^3 blocks: its cells on a
    block's rim are edges and corners of that block, whose velocity reads
    give 0 and density reads 1 (the reference's ExtrapolatedU and
    PrescribedRho off a flat face), beside an inlet on x-."""
    sys.path.insert(0, HERE)
    from test_const_rho import brick_cavity
    mesh, info = brick_cavity(lid=0.0, n=8)
    types = [ob.FD_VELOCITY, ob.FD_PRESSURE] + [ob.FD_VELOCITY] * 4
    inlet = np.zeros((6, 3))
    inlet[0, 0] = 0.02
    rho = np.ones(6)
    rho[1] = 1.002
    rec = check(ob, mesh, types, np.zeros((6, 3)), rho, inlet, ramp=20.0, t=9.0)
    p = rec[rec["kind"] == 6]
    assert set(np.unique(p["role"])) == {1, 2, 3}
    assert np.any(p["u"]["code"][p["role"] >= 2][:, 0] == 0)


@pytest.mark.parametrize("kind", [2, 3])
def test_poiseuille_inlets(ob, kind):
    """The duct inlet fields (octlb_fd_plan_inlets): per-block parabolas
    (Poiseuille) and a physical channel patch (channel Poiseuille) on x- of
    eight 8^3 blocks, with their ramp, at three times."""
    sys.path.insert(0, HERE)
    from test_const_rho import brick_cavity
    mesh, info = brick_cavity(lid=0.0, n=8)
    types = [ob.FD_VELOCITY, ob.FD_PRESSURE] + [ob.FD_VELOCITY] * 4
    inlet = ob.fd_inlet(kind, (1.0, 0.0, 0.0), 0.03, (8, 8), (0.1, 0.9, 0.2, 0.8), 20.0)
    for t in (0.0, 7.0, 40.0):
        rec = check(ob, mesh, types, np.zeros((6, 3)), np.ones(6), t=t, inlets=[inlet] + [None] * 5)
    assert np.count_nonzero(rec["u_base"][:, 0] > 0) > 0 and np.all(rec["ramp_end"][rec["u_base"][:, 0] > 0] == 20.0)


def test_inlet_validation(ob):
    """Out-of-range inlet kinds and degenerate profiles are refused."""
    from octlb_b200 import cases
    mesh, init, info = cases.cavity_forest(cells=16, n=16, lid=0.0, tau=0.6)
    types = [ob.FD_VELOCITY] * 6
    for bad in (ob.fd_inlet(4), ob.fd_inlet(ob.INLET_POISEUILLE, n_inplane=(0, 8)),
                ob.fd_inlet(ob.INLET_CHANNEL_POISEUILLE, patch=(0.5, 0.5, 0.0, 1.0))):
        with pytest.raises(AssertionError):
            plan(ob, ob.stamp_fd_kinds(mesh, types), types, np.zeros((6, 3)), np.ones(6), inlets=[bad] + [None] * 5)


def test_no_slip_walls_and_lid(ob):
    """No-slip faces (kBounceBack: the collide's full-way swap, no
    reconstruction) around an InterpolatedVelocity lid: the lid's edge and
    corner cells read bounce-back neighbours as plain cells."""
    from octlb_b200 import cases
    mesh, init, info = cases.cavity_forest(cells=16, n=16, lid=0.0, tau=0.6)
    u = np.zeros((6, 3))
    u[3, 0] = 0.05
    types = [ob.FD_NO_SLIP] * 3 + [ob.FD_VELOCITY] + [ob.FD_NO_SLIP] * 2
    rec = check(ob, mesh, types, u, np.ones(6))
    assert np.any(rec["role"] == 0) and np.any(rec["role"] >= 1)
