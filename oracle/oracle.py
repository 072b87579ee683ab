"""Python handles on the two CPU oracles.  TEST INFRASTRUCTURE ONLY: used by
tests/, __graft_entry__.smoke() and bench.py's CPU legs as the checker, never
by the product.

* ``liboctlb_oracle.so``  -- plain-C restatement (octlb_oracle.c), always built.
* ``_ref/liboctlb_ref.so`` -- the reference's own BlockLattice / LevelCoupler /
  GhostSchedule / TimeLoop / MomentumExchangeDrag, compiled from its sources by
  `make -C oracle ref REF=<reference tree>` where the reference tree is available; prebuilt files
  travel with the repository.
* ``_ref/liboctlb_ref_tlm.so`` -- the same sources compiled on a forward-mode
  dual number (`make -C oracle tlm REF=<reference tree>`): the tangent-linear FP64 reference, whose
  force carries its derivatives along seeded parameter directions.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORC_PATH = os.path.join(HERE, "liboctlb_oracle.so")
REF_PATH = os.path.join(HERE, "_ref", "liboctlb_ref.so")
TLM_PATH = os.path.join(HERE, "_ref", "liboctlb_ref_tlm.so")
Q = 19
P = ctypes.c_void_p


def _p(a, t=ctypes.c_double):
    return None if a is None else a.ctypes.data_as(ctypes.POINTER(t))


def build(ref=True, reference_tree=None):
    """make -C oracle, and with ref the reference build from its source tree
    (`reference_tree`, else the OCTLB_REFERENCE environment variable).  A tree
    that is named but holds no reference sources is an error; with none named
    the reference build is skipped (its prebuilt files, if any, stay)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    src = reference_tree or os.environ.get("OCTLB_REFERENCE")
    if not ref or not src:
        return
    if not os.path.isdir(os.path.join(src, "src", "solver", "lbm")):
        raise FileNotFoundError(f"{src} holds no reference sources (src/solver/lbm)")
    subprocess.run(["make", "-s", "-C", HERE, "ref", "tlm", f"REF={src}"], check=True)


def load(which):
    """'orc' (C restatement), 'ref' (the reference) or 'tlm' (the reference
    on dual numbers; same ref_* entry points plus tlm_*)."""
    path = {"orc": ORC_PATH, "ref": REF_PATH, "tlm": TLM_PATH}[which]
    if not os.path.exists(path):
        return None
    L = ctypes.CDLL(path)
    pre = "orc_" if which == "orc" else "ref_"
    for fn in ("block_new", "sim_new"):
        if hasattr(L, pre + fn):
            getattr(L, pre + fn).restype = P
    for fn in ("feq", "bouzidi_pull"):
        getattr(L, pre + fn).restype = ctypes.c_double
        getattr(L, pre + fn).argtypes = ([ctypes.c_int] + [ctypes.c_double] * 4 if fn == "feq"
                                         else [ctypes.c_double] * 4)
    if hasattr(L, "ref_sim_average_rho"):
        L.ref_sim_average_rho.restype = ctypes.c_double
        L.ref_sim_average_rho.argtypes = [P]
    if which == "tlm":
        L.tlm_dirs.restype = ctypes.c_int
    if which == "orc":
        L.orc_periodic_slabs_mlups.restype = ctypes.c_double
        L.orc_periodic_slabs_mlups.argtypes = [ctypes.c_int] * 5 + [ctypes.c_double, ctypes.c_int]
    L._pre = pre
    return L


class Block:
    """One BlockLattice<double> (reference layout, halo 1) in either oracle."""

    def __init__(self, L, nx, ny=None, nz=None):
        ny = nx if ny is None else ny
        nz = nx if nz is None else nz
        self.L, self.pre, self.shape = L, L._pre, (nx, ny, nz)
        self.h = P(getattr(L, self.pre + "block_new")(nx, ny, nz))

    def __del__(self):
        if getattr(self, "h", None):
            getattr(self.L, self.pre + "block_free")(self.h)
            self.h = None

    def _f(self, name):
        return getattr(self.L, self.pre + name)

    def initialize(self, rho, u):
        self._f("block_initialize")(self.h, ctypes.c_double(rho), *[ctypes.c_double(v) for v in u])

    def set_kinds(self, kinds):
        k = np.ascontiguousarray(kinds, np.uint8)
        self._f("block_set_kinds")(self.h, _p(k, ctypes.c_uint8))

    def padded(self):
        nx, ny, nz = self.shape
        out = np.zeros((nx + 2, ny + 2, nz + 2, Q))
        self._f("block_get_padded")(self.h, _p(out))
        return out

    def set_padded(self, pad):
        a = np.ascontiguousarray(pad, np.float64)
        self._f("block_set_padded")(self.h, _p(a))

    def core(self):
        return self.padded()[1:-1, 1:-1, 1:-1]

    def set_core(self, core):
        pad = self.padded()
        pad[1:-1, 1:-1, 1:-1] = core
        self.set_padded(pad)

    def collide(self, omega):
        self._f("block_collide")(self.h, ctypes.c_double(omega))

    def fill_periodic(self):
        self._f("block_fill_periodic")(self.h)

    def stream(self):
        self._f("block_stream")(self.h)

    def snapshot(self):
        self._f("block_snapshot")(self.h)

    def set_links(self, cell_pop, q):
        cp = np.ascontiguousarray(cell_pop, np.int32).reshape(-1, 4)
        qq = np.ascontiguousarray(q, np.float64).reshape(-1)
        self._f("block_set_links")(self.h, ctypes.c_int(len(qq)), _p(cp, ctypes.c_int), _p(qq))

    def add_moving_wall(self, moving, wall_u):
        m = np.ascontiguousarray(moving, np.uint8)
        w = np.ascontiguousarray(wall_u, np.float64)
        self._f("block_add_moving_wall")(self.h, _p(m, ctypes.c_uint8), _p(w))

    def run_periodic(self, omega, steps):
        self._f("block_run_periodic")(self.h, ctypes.c_double(omega), ctypes.c_int(steps))

    def run_periodic_mt(self, omega, steps, threads=None):
        """run_periodic on several host threads (C restatement only), bitwise
        equal to it."""
        threads = threads or os.cpu_count() or 1
        rc = self._f("block_run_periodic_mt")(self.h, ctypes.c_double(omega), ctypes.c_int(steps),
                                              ctypes.c_int(threads))
        assert rc == 0, "run_periodic_mt needs a block without a link table"

    def fields(self):
        """rho [nx][ny][nz] and u [nx][ny][nz][3] of the core (C restatement)."""
        rho = np.zeros(self.shape)
        u = np.zeros(self.shape + (3,))
        self._f("block_fields")(self.h, _p(rho), _p(u))
        return rho, u

    def run_walls(self, omega, steps, moving=None, wall_u=None):
        m = None if moving is None else np.ascontiguousarray(moving, np.uint8)
        w = None if wall_u is None else np.ascontiguousarray(wall_u, np.float64)
        self._f("block_run_walls")(self.h, ctypes.c_double(omega), ctypes.c_int(steps),
                                   _p(m, ctypes.c_uint8), _p(w))

    def drag(self, mask=None):
        out = np.zeros(3)
        m = None if mask is None else np.ascontiguousarray(mask, np.uint8)
        self._f("block_drag")(self.h, _p(m, ctypes.c_uint8), _p(out))
        return out


def rho_u(pops):
    """rho = 1 + sum f, u = sum f c / rho (block_lattice.h:113-125)."""
    from octlb_b200 import C
    rho = 1.0 + pops.sum(-1)
    u = np.einsum("...q,qd->...d", pops, C.astype(np.float64)) / rho[..., None]
    return rho, u


class Sim:
    """TimeLoop over a forest (reference oracle only: ref_sim_*).  On the
    tangent-linear library, omega_seed[k] / wall_seed[k] seed direction k:
    d omega, and d u_w / u_w for every tree-boundary wall velocity."""

    def __init__(self, L, mesh, omega, init_pops=None, link_mode=False, omega_seed=None, wall_seed=None):
        self.L, self.mesh = L, mesh
        if hasattr(L, "tlm_set_seeds"):
            nd = L.tlm_dirs()
            om = np.zeros(nd) if omega_seed is None else np.ascontiguousarray(omega_seed, np.float64)
            ws = np.zeros(nd) if wall_seed is None else np.ascontiguousarray(wall_seed, np.float64)
            assert om.shape == (nd,) and ws.shape == (nd,)
            L.tlm_set_seeds(_p(om), _p(ws))
        n = mesh.n
        self._keep = [mesh]
        init = None if init_pops is None else np.ascontiguousarray(init_pops, np.float64)
        self._keep.append(init)
        lc = mesh.link_cells if len(mesh.link_q) else np.zeros((0, 5), np.int32)
        self.h = P(L.ref_sim_new(
            ctypes.c_int(mesh.n_blocks), _p(mesh.levels, ctypes.c_int), _p(mesh.bounds),
            ctypes.c_int(len(mesh.same_level)), _p(mesh.same_level, ctypes.c_int),
            ctypes.c_int(len(mesh.coarse_fine)), _p(mesh.coarse_fine, ctypes.c_int), _p(mesh.coarse_fine_bounds),
            ctypes.c_int(len(mesh.tree_boundary)), _p(mesh.tree_boundary, ctypes.c_int), _p(mesh.tree_boundary_spec),
            ctypes.c_int(n), ctypes.c_double(omega), _p(mesh.kinds, ctypes.c_uint8), _p(init),
            ctypes.c_int(len(mesh.link_q)), _p(np.ascontiguousarray(lc, np.int32), ctypes.c_int), _p(mesh.link_q),
            ctypes.c_int(1 if link_mode else 0)))

    def __del__(self):
        if getattr(self, "h", None):
            self.L.ref_sim_free(self.h)
            self.h = None

    def advance(self, steps=1):
        self.L.ref_sim_advance(self.h, ctypes.c_int(steps))

    def set_physical(self, omega_level):
        """The physical coupler mode (not the reference's loop): level l
        collides with omega_level[l] and the pair (l, l + 1) is coupled by a
        LevelCoupler built with omega_level[l]; TimeLoop::advance's phase
        order restated around the reference's own components.  Before the
        first advance."""
        w = np.ascontiguousarray(omega_level, np.float64)
        self._keep.append(w)
        self.L.ref_sim_set_physical(self.h, _p(w), ctypes.c_int(len(w)))

    def set_const_rho(self, on=True):
        """The reference TimeLoop rebuilt with use_const_rho_bgk (before the
        first advance)."""
        self.L.ref_sim_set_const_rho(self.h, ctypes.c_int(1 if on else 0))

    def average_rho(self):
        """TimeLoop::average_rho()."""
        return float(self.L.ref_sim_average_rho(self.h))

    def advance_phases(self):
        """One advance_one of a single-level mesh; the core populations after
        the stream and after the post-stream boundary pass (the two sides of
        the FD reconstruction), [n_blocks][n][n][n][19] each."""
        n = self.mesh.n
        a = np.zeros((self.mesh.n_blocks, n, n, n, Q))
        b = np.zeros_like(a)
        self.L.ref_sim_advance_phases(self.h, _p(a), _p(b))
        return a, b

    def advance_phases_padded(self):
        """One advance_one of a single-level mesh; the padded populations
        (halo 1) at the start and after collide, ghost exchange, stream and
        the post-stream pass: [5][n_blocks][n+2][n+2][n+2][19]."""
        m = self.mesh.n + 2
        out = np.zeros((5, self.mesh.n_blocks, m, m, m, Q))
        self.L.ref_sim_advance_phases_padded(self.h, _p(out))
        return out

    def kinds(self):
        """BcKind of every core cell, [n_blocks][n][n][n]."""
        n = self.mesh.n
        out = np.zeros((self.mesh.n_blocks, n, n, n), np.uint8)
        self.L.ref_sim_get_kinds(self.h, _p(out, ctypes.c_uint8))
        return out

    # DomainBcType and OverlapPaddingMode (domain_boundary_handler.h:14-36)
    NO_SLIP, MOVING_LID, INTERPOLATED_VELOCITY, OUTFLOW, INTERPOLATED_PRESSURE = range(5)
    PADDING_POST_STREAM, PADDING_MIRROR, PADDING_HYBRID = range(3)

    def set_fd_boundary(self, types, u_wall=None, rho_target=None, padding_mode=2, const_rho=False, inlet_u=None,
                        ramp_end_t=0.0, inlets=None):
        """The reference's ConcreteDomainBoundaryHandler on every tree-boundary
        face (faces in FaceDir order x-, x+, y-, y+, z-, z+): spec types,
        wall velocities [6][3], target densities [6]; the face cells stamped
        with the spec's BcKind and the TimeLoop rebuilt around the handler
        (optionally with ConstRhoBGK); faces with a nonzero inlet_u row [6][3]
        take a uniform inlet of that velocity ramped over ramp_end_t steps --
        or, with inlets (six dicts of kind, u, u_peak, n_inplane, patch,
        ramp_end_t, or None), the reference's inlet field of that kind
        (1 uniform, 2 Poiseuille, 3 channel Poiseuille).  Before the first
        advance."""
        t = np.ascontiguousarray(types, np.int32).reshape(6)
        u = np.zeros((6, 3)) if u_wall is None else np.ascontiguousarray(u_wall, np.float64).reshape(6, 3)
        r = np.ones(6) if rho_target is None else np.ascontiguousarray(rho_target, np.float64).reshape(6)
        if inlets is not None:
            kind = np.zeros(6, np.int32)
            par = np.zeros((6, 11))
            for f, d in enumerate(inlets):
                if d is None:
                    continue
                kind[f] = int(d["kind"])
                par[f, 0:3] = d["u"]
                par[f, 3] = d["u_peak"]
                par[f, 4:6] = d["n_inplane"]
                par[f, 6:10] = d["patch"]
                par[f, 10] = d["ramp_end_t"]
            self._keep += [t, u, r, kind, par]
            self.L.ref_sim_set_fd_boundary_inlets(self.h, _p(t, ctypes.c_int), _p(u), _p(r),
                                                  ctypes.c_int(padding_mode), ctypes.c_int(1 if const_rho else 0),
                                                  _p(kind, ctypes.c_int), _p(par))
            return
        iu = None if inlet_u is None else np.ascontiguousarray(inlet_u, np.float64).reshape(6, 3)
        self._keep += [t, u, r, iu]
        self.L.ref_sim_set_fd_boundary(self.h, _p(t, ctypes.c_int), _p(u), _p(r), ctypes.c_int(padding_mode),
                                       ctypes.c_int(1 if const_rho else 0), _p(iu), ctypes.c_double(ramp_end_t))

    def set_body_force(self, force):
        """Body force [n_blocks][n^3][3] (or None): 3 w_i (c_i . F) added to the
        post-collision populations of kBulk cells of each level step, at the
        DomainBoundaryHandler::apply() hook (restated; not reference code)."""
        f = None if force is None else np.ascontiguousarray(force, np.float64)
        self._keep.append(f)
        self.L.ref_sim_set_body_force(self.h, _p(f))

    def set_body_force_tlm(self, force, dirs):
        """Tangent-linear library: body force (or None = 0) with its
        derivative dirs[k] ([k][n_blocks][n^3][3]) along direction k."""
        m = self.mesh.n_blocks * self.mesh.n ** 3 * 3
        f = None if force is None else np.ascontiguousarray(force, np.float64).reshape(m)
        d = np.ascontiguousarray(dirs, np.float64).reshape(-1, m)
        self._keep += [f, d]
        self.L.tlm_sim_set_body_force(self.h, _p(f), _p(d), ctypes.c_int(d.shape[0]))

    def drag_tlm(self, mask=None):
        """Tangent-linear library: the force (3,) and its derivatives (3, k)."""
        nd = self.L.tlm_dirs()
        out, dout = np.zeros(3), np.zeros((3, nd))
        m = None if mask is None else np.ascontiguousarray(mask, np.uint8)
        self.L.tlm_sim_drag(self.h, _p(m, ctypes.c_uint8), _p(out), _p(dout))
        return out, dout

    def core(self):
        n = self.mesh.n
        out = np.zeros((self.mesh.n_blocks, n, n, n, Q))
        self.L.ref_sim_get_core(self.h, _p(out))
        return out

    def drag(self, mask=None):
        out = np.zeros(3)
        m = None if mask is None else np.ascontiguousarray(mask, np.uint8)
        self.L.ref_sim_drag(self.h, _p(m, ctypes.c_uint8), _p(out))
        return out

    def counters(self):
        c = np.zeros(32, np.int32)
        s = np.zeros(32, np.int32)
        calls = np.zeros(2 * 4096, np.int32)
        ncalls = self.L.ref_sim_counters(self.h, _p(c, ctypes.c_int), _p(s, ctypes.c_int),
                                         _p(calls, ctypes.c_int), ctypes.c_int(4096))
        ml = self.L.ref_sim_max_level(self.h)
        return c[:ml + 1].tolist(), s[:ml + 1].tolist(), calls[:2 * min(ncalls, 4096)].reshape(-1, 2).tolist()

    def plan(self):
        out = np.zeros((65536, 10), np.int32)
        n = self.L.ref_sim_plan(self.h, _p(out, ctypes.c_int), ctypes.c_int(65536))
        return out[:n]

    def coupler_full(self, level):
        self.L.ref_sim_coupler_full(self.h, ctypes.c_int(level))

    def coupler_half(self, level):
        self.L.ref_sim_coupler_half(self.h, ctypes.c_int(level))

    def coupler_restrict(self, level):
        self.L.ref_sim_coupler_restrict(self.h, ctypes.c_int(level))
