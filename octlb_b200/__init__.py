"""octlb_b200 -- B200 (sm_100a) per-level time step of OctLB.

Host mirror of the reference's solver entry points for this path:

* ``Forest``        -- OctreeForest + FacePairList (p4est in the reference):
                       brick of trees, refine, 2:1 balance, flattened faces.
* ``Mesh``          -- the flattened tables octlb_gpu_create consumes
                       (leaves, BcKind per cell, faces, Bouzidi links, ...).
* ``GpuLattice``    -- one GPU context: every level's SoA populations plus the
                       flattened GhostSchedule / LevelCoupler tables.
* ``GpuTimeLoop``   -- the reference TimeLoop's method names
                       (src/solver/lbm/time_loop/time_loop.h:47-121) over a
                       GpuLattice.

All compute runs in the in-tree CUDA library liboctlb_b200.so; importing this
package without it raises ImportError.
"""
import ctypes

import numpy as np

from . import capi
from .capi import (BULK, SOLID, BOUNCE_BACK, MOVING_BOUNCE_BACK, BOUZIDI, VELOCITY_DIRICHLET,
                   PRESSURE_DIRICHLET, OUTFLOW, FP32, FP16_SHIFTED, STREAM_ROTATE, STREAM_LINKS,
                   TB_NONE, TB_WALL, TB_OUTFLOW, COUPLER_REFERENCE, COUPLER_PHYSICAL, ORDER_AB, ORDER_AA,
                   INLET_NONE, INLET_UNIFORM, INLET_POISEUILLE, INLET_CHANNEL_POISEUILLE, OctlbError)

capi.lib()  # fail loudly at import when the library is missing

Q = 19
# D3Q19 in the reference's population order (descriptor/definition/common.h:165-197)
C = np.array([[0, 0, 0], [-1, 0, 0], [0, -1, 0], [0, 0, -1], [-1, -1, 0], [-1, 1, 0], [-1, 0, -1],
              [-1, 0, 1], [0, -1, -1], [0, -1, 1], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 1, 0],
              [1, -1, 0], [1, 0, 1], [1, 0, -1], [0, 1, 1], [0, 1, -1]], dtype=np.int64)
OPP = np.array([0, 10, 11, 12, 13, 14, 15, 16, 17, 18, 1, 2, 3, 4, 5, 6, 7, 8, 9])
W = np.array([1 / 3] + [1 / 18] * 3 + [1 / 36] * 6 + [1 / 18] * 3 + [1 / 36] * 6)


def feq(rho, u):
    """Shifted second-order equilibrium f_eq - w (dynamics/lbm.h:50-64).

    rho: (...), u: (..., 3) -> (..., 19)."""
    rho = np.asarray(rho, dtype=np.float64)
    u = np.asarray(u, dtype=np.float64)
    cu = np.einsum("...d,qd->...q", u, C.astype(np.float64))
    usq = np.sum(u * u, axis=-1)[..., None]
    return rho[..., None] * W * (1.0 + 3.0 * cu + 4.5 * cu * cu - 1.5 * usq) - W


class Forest:
    """Brick of octrees with refinement and 2:1 balance (include/octlb_forest.h)."""

    def __init__(self, bricks=(1, 1, 1), periodic=(0, 0, 0), domain=(0, 0, 0, 1, 1, 1)):
        self._L = capi.lib()
        dom = np.asarray(domain, dtype=np.float64)
        self._h = self._L.octlb_forest_new(*[int(b) for b in bricks], *[int(p) for p in periodic],
                                           capi.ptr(dom, ctypes.c_double))
        if not self._h:
            raise ValueError("invalid brick")
        self.bricks, self.periodic, self.domain = tuple(bricks), tuple(periodic), tuple(domain)

    def __del__(self):
        if getattr(self, "_h", None):
            self._L.octlb_forest_free(self._h)
            self._h = None

    def refine_uniform(self, level):
        self._L.octlb_forest_refine_uniform(self._h, int(level))
        return self

    def refine_box(self, box, level):
        b = np.asarray(box, dtype=np.float64)
        self._L.octlb_forest_refine_box(self._h, capi.ptr(b, ctypes.c_double), int(level))
        return self

    def balance(self):
        self._L.octlb_forest_balance(self._h)
        return self

    def build(self):
        L, h = self._L, self._h
        n = L.octlb_forest_build(h)
        self.levels = np.zeros(n, np.int32)
        self.bounds = np.zeros((n, 6), np.float64)
        L.octlb_forest_leaves(h, capi.ptr(self.levels, ctypes.c_int), capi.ptr(self.bounds, ctypes.c_double))
        ns = L.octlb_forest_num_same_level(h)
        self.same_level = np.zeros((ns, 3), np.int32)
        L.octlb_forest_same_level(h, capi.ptr(self.same_level, ctypes.c_int))
        nc = L.octlb_forest_num_coarse_fine(h)
        self.coarse_fine = np.zeros((nc, 8), np.int32)
        self.coarse_fine_bounds = np.zeros((nc, 30), np.float64)
        L.octlb_forest_coarse_fine(h, capi.ptr(self.coarse_fine, ctypes.c_int),
                                   capi.ptr(self.coarse_fine_bounds, ctypes.c_double))
        nt = L.octlb_forest_num_tree_boundary(h)
        self.tree_boundary = np.zeros((nt, 2), np.int32)
        L.octlb_forest_tree_boundary(h, capi.ptr(self.tree_boundary, ctypes.c_int))
        return self

    @property
    def num_leaves(self):
        return len(self.levels)


class Mesh:
    """Flattened tables for octlb_gpu_create (octlb_tables).

    Cell arrays are [block][ix][iy][iz] (the reference's block order)."""

    def __init__(self, n, levels, bounds, kinds=None, same_level=None, coarse_fine=None,
                 coarse_fine_bounds=None, tree_boundary=None, tree_boundary_spec=None,
                 link_cells=None, link_q=None, moving=None, wall_u=None, obstacle=None, periodic=0):
        self.n = int(n)
        self.levels = np.ascontiguousarray(levels, dtype=np.int32)
        nb = len(self.levels)
        self.bounds = np.ascontiguousarray(bounds, dtype=np.float64).reshape(nb, 6)
        shape = (nb, self.n, self.n, self.n)
        self.kinds = np.zeros(shape, np.uint8) if kinds is None else np.ascontiguousarray(kinds, np.uint8).reshape(shape)
        self.same_level = np.zeros((0, 3), np.int32) if same_level is None else np.ascontiguousarray(same_level, np.int32).reshape(-1, 3)
        self.coarse_fine = np.zeros((0, 8), np.int32) if coarse_fine is None else np.ascontiguousarray(coarse_fine, np.int32).reshape(-1, 8)
        self.coarse_fine_bounds = (np.zeros((len(self.coarse_fine), 30)) if coarse_fine_bounds is None
                                   else np.ascontiguousarray(coarse_fine_bounds, np.float64).reshape(-1, 30))
        self.tree_boundary = np.zeros((0, 2), np.int32) if tree_boundary is None else np.ascontiguousarray(tree_boundary, np.int32).reshape(-1, 2)
        self.tree_boundary_spec = (np.zeros((len(self.tree_boundary), 8)) if tree_boundary_spec is None
                                   else np.ascontiguousarray(tree_boundary_spec, np.float64).reshape(-1, 8))
        self.link_cells = np.zeros((0, 5), np.int32) if link_cells is None else np.ascontiguousarray(link_cells, np.int32).reshape(-1, 5)
        self.link_q = np.zeros(0) if link_q is None else np.ascontiguousarray(link_q, np.float64).reshape(-1)
        self.moving = None if moving is None else np.ascontiguousarray(moving, np.uint8).reshape(shape)
        self.wall_u = None if wall_u is None else np.ascontiguousarray(wall_u, np.float64).reshape(shape + (3,))
        self.obstacle = None if obstacle is None else np.ascontiguousarray(obstacle, np.uint8).reshape(shape)
        self.periodic = int(periodic)

    @classmethod
    def from_forest(cls, forest, n, **kw):
        return cls(n, forest.levels, forest.bounds, same_level=forest.same_level,
                   coarse_fine=forest.coarse_fine, coarse_fine_bounds=forest.coarse_fine_bounds,
                   tree_boundary=forest.tree_boundary, **kw)

    @property
    def n_blocks(self):
        return len(self.levels)

    def cells_per_level(self):
        out = {}
        for l in self.levels:
            out[int(l)] = out.get(int(l), 0) + self.n ** 3
        return out

    def lattice_updates_per_coarse_step(self):
        """sum over levels of cells x 2^level (TimeLoop recursion from level 0)."""
        return sum(c << l for l, c in self.cells_per_level().items())

    def c_tables(self):
        t = capi.Tables()
        t.n, t.n_blocks = self.n, self.n_blocks
        t.levels = capi.ptr(self.levels, ctypes.c_int)
        t.bounds = capi.ptr(self.bounds, ctypes.c_double)
        t.kinds = capi.ptr(self.kinds, ctypes.c_uint8)
        t.n_same_level, t.same_level = len(self.same_level), capi.ptr(self.same_level, ctypes.c_int)
        t.n_coarse_fine = len(self.coarse_fine)
        t.coarse_fine = capi.ptr(self.coarse_fine, ctypes.c_int)
        t.coarse_fine_bounds = capi.ptr(self.coarse_fine_bounds, ctypes.c_double)
        t.n_tree_boundary = len(self.tree_boundary)
        t.tree_boundary = capi.ptr(self.tree_boundary, ctypes.c_int)
        t.tree_boundary_spec = capi.ptr(self.tree_boundary_spec, ctypes.c_double)
        t.n_links = len(self.link_q)
        t.link_cells = capi.ptr(self.link_cells, ctypes.c_int)
        t.link_q = capi.ptr(self.link_q, ctypes.c_double)
        t.moving = capi.ptr(self.moving, ctypes.c_uint8)
        t.wall_u = capi.ptr(self.wall_u, ctypes.c_double)
        t.obstacle = capi.ptr(self.obstacle, ctypes.c_uint8)
        t.periodic = self.periodic
        return t


def plan(mesh, omega, precision=FP32, stream_mode=STREAM_ROTATE, drag=False):
    """Host-only dry run of the context build (octlb_gpu_plan): per level a
    dict of blocks, halo pages, open blocks, boundary-fill writes, coupler
    items, saved cells, link records, drag cells and slots."""
    L = capi.lib()
    p = capi.Params()
    p.omega, p.precision, p.stream_mode, p.drag = float(omega), int(precision), int(stream_mode), int(bool(drag))
    buf = (ctypes.c_longlong * 4096)()
    n = L.octlb_gpu_plan(ctypes.byref(mesh.c_tables()), ctypes.byref(p), buf, 4096)
    if n < 0:
        raise OctlbError(n, "plan failed")
    keys = ["blocks", "pages", "open", "fills", "prolong", "restrict", "saved", "links", "drag", "slots"]
    nl = buf[0]
    return [dict(zip(keys, [buf[1 + 10 * l + k] for k in range(10)])) for l in range(nl)]


_VTK_FIELDS = {"velocity": capi.VTK_VELOCITY, "density": capi.VTK_DENSITY, "pressure": capi.VTK_PRESSURE}


def vtk_write_block(path, bounds, fields):
    """One StructuredGrid .vts (octlb_vtk_write_block): fields is a list of
    (name, values [nx][ny][nz] or [nx][ny][nz][c]) on the cells of a block
    with the given bounds (x_min, y_min, z_min, x_max, y_max, z_max)."""
    L = capi.lib()
    arrs, names, comps = [], [], []
    shape = None
    for name, v in fields:
        v = np.asarray(v, np.float64)
        c = 1 if v.ndim == 3 else v.shape[3]
        shape = v.shape[:3] if shape is None else shape
        if v.shape[:3] != shape:
            raise ValueError("all fields take the block's cell shape")
        # file order: i (x) fastest, then j, then k
        arrs.append(np.ascontiguousarray(np.transpose(v.reshape(shape + (c,)), (2, 1, 0, 3))).reshape(-1))
        names.append(name.encode())
        comps.append(c)
    nx, ny, nz = shape
    b = np.ascontiguousarray(bounds, np.float64)
    data = (capi.F64P * len(arrs))(*[capi.ptr(a, ctypes.c_double) for a in arrs])
    rc = L.octlb_vtk_write_block(str(path).encode(), nx, ny, nz, capi.ptr(b, ctypes.c_double), len(arrs),
                                 (ctypes.c_char_p * len(names))(*names), (ctypes.c_int * len(comps))(*comps), data)
    if rc:
        raise OctlbError(rc, "vtk_write_block failed")


def vtk_write_index(output_dir, base_name, step, vts_relative_paths):
    """The .vtm of one timestep and its .pvd entry (octlb_vtk_write_index)."""
    L = capi.lib()
    p = [str(x).encode() for x in vts_relative_paths]
    rc = L.octlb_vtk_write_index(str(output_dir).encode(), str(base_name).encode(), int(step), len(p),
                                 (ctypes.c_char_p * max(len(p), 1))(*p))
    if rc:
        raise OctlbError(rc, "vtk_write_index failed")


FD_NO_SLIP, FD_MOVING_LID, FD_VELOCITY, FD_OUTFLOW, FD_PRESSURE = 0, 1, 2, 3, 4


def fd_inlet(kind, u=(0.0, 0.0, 0.0), u_peak=0.0, n_inplane=(1, 1), patch=(0.0, 1.0, 0.0, 1.0), ramp_end_t=0.0):
    """One face's inlet velocity field (octlb_fd_inlet): kind INLET_UNIFORM
    (velocity u), INLET_POISEUILLE (peak u_peak along direction u over
    n_inplane cells of the block's in-plane axes) or INLET_CHANNEL_POISEUILLE
    (the same over the physical patch (in0_lo, in0_hi, in1_lo, in1_hi))."""
    return {"kind": kind, "u": u, "u_peak": u_peak, "n_inplane": n_inplane, "patch": patch,
            "ramp_end_t": ramp_end_t}


def fd_inlets(inlets):
    """Six faces' inlet fields (dicts of fd_inlet, or None) as the C array."""
    arr = (capi.FdInlet * 6)()
    for f, d in enumerate(inlets):
        if d is None:
            continue
        arr[f].kind = int(d["kind"])
        arr[f].n_inplane[:] = [int(v) for v in d["n_inplane"]]
        arr[f].u[:] = [float(v) for v in d["u"]]
        arr[f].u_peak = float(d["u_peak"])
        arr[f].patch[:] = [float(v) for v in d["patch"]]
        arr[f].ramp_end_t = float(d["ramp_end_t"])
    return arr


def stamp_fd_kinds(mesh, types):
    """The mesh with its tree-boundary face slabs stamped by face type
    (octlb_fd_stamp_kinds, the reference's StampTreeBoundaryCells)."""
    t = np.ascontiguousarray(types, np.int32).reshape(6)
    kinds = np.zeros_like(mesh.kinds)
    rc = capi.lib().octlb_fd_stamp_kinds(ctypes.byref(mesh.c_tables()), capi.ptr(t, ctypes.c_int),
                                         capi.ptr(kinds, ctypes.c_uint8))
    if rc:
        raise OctlbError(rc, "stamp_fd_kinds failed")
    out = Mesh(mesh.n, mesh.levels, mesh.bounds, kinds=kinds, same_level=mesh.same_level,
               coarse_fine=mesh.coarse_fine, coarse_fine_bounds=mesh.coarse_fine_bounds,
               tree_boundary=mesh.tree_boundary, tree_boundary_spec=np.zeros_like(mesh.tree_boundary_spec),
               link_cells=mesh.link_cells, link_q=mesh.link_q, moving=mesh.moving, wall_u=mesh.wall_u,
               obstacle=mesh.obstacle, periodic=mesh.periodic)
    return out


def partition(mesh, nranks):
    """The reference's weighted partition (octlb_gpu_partition): owning rank
    of every leaf, contiguous runs of the forest order of equal 2^level
    weight."""
    owner = np.zeros(mesh.n_blocks, np.int32)
    rc = capi.lib().octlb_gpu_partition(ctypes.byref(mesh.c_tables()), int(nranks), capi.ptr(owner, ctypes.c_int))
    if rc:
        raise OctlbError(rc, "partition failed")
    return owner


def plan_part(mesh, omega, rank, owner, precision=FP32, stream_mode=STREAM_ROTATE, drag=False):
    """Host-only dry run of a rank context (octlb_gpu_plan_part): its
    exchange lists as an int64 array of (level, kind, peer, global cell)
    rows, kind 0 / 1 cells sent / received before a level step, 2 / 3 save
    rows sent / received after it."""
    L = capi.lib()
    p = capi.Params()
    p.omega, p.precision, p.stream_mode, p.drag = float(omega), int(precision), int(stream_mode), int(bool(drag))
    own = np.ascontiguousarray(owner, np.int32)
    nranks = int(own.max()) + 1
    n = L.octlb_gpu_plan_part(ctypes.byref(mesh.c_tables()), ctypes.byref(p), int(rank), nranks,
                              capi.ptr(own, ctypes.c_int), None, 0)
    if n < 0:
        raise OctlbError(n, "plan_part failed")
    out = np.zeros((max(n, 1), 4), np.int64)
    n = L.octlb_gpu_plan_part(ctypes.byref(mesh.c_tables()), ctypes.byref(p), int(rank), nranks,
                              capi.ptr(own, ctypes.c_int), out.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)),
                              len(out))
    return out[:n]


class Comm:
    """Transport between rank contexts (octlb_comm): ``Comm.local(n)`` for n
    rank contexts of this process (one host thread each), ``Comm.nccl(id, n,
    rank)`` for one process per GPU (``Comm.nccl_unique_id()`` on rank 0,
    shared by the caller's launcher)."""

    def __init__(self, handle, nranks):
        self._h, self.nranks = handle, nranks

    @classmethod
    def local(cls, nranks):
        h = capi.P()
        rc = capi.lib().octlb_comm_create_local(int(nranks), ctypes.byref(h))
        if rc:
            raise OctlbError(rc, "local comm")
        return cls(h, nranks)

    @staticmethod
    def nccl_unique_id():
        buf = (ctypes.c_ubyte * 128)()
        rc = capi.lib().octlb_comm_nccl_unique_id(buf)
        if rc:
            raise OctlbError(rc, "nccl unique id: " + capi.lib().octlb_comm_last_error().decode())
        return bytes(buf)

    @classmethod
    def nccl(cls, uid, nranks, rank):
        buf = (ctypes.c_ubyte * 128).from_buffer_copy(uid)
        h = capi.P()
        rc = capi.lib().octlb_comm_create_nccl(buf, int(nranks), int(rank), ctypes.byref(h))
        if rc:
            raise OctlbError(rc, "nccl comm: " + capi.lib().octlb_comm_last_error().decode())
        return cls(h, nranks)

    def close(self):
        if self._h:
            capi.lib().octlb_comm_destroy(self._h)
            self._h = None


class GpuLattice:
    """One octlb_gpu context (include/octlb_gpu.h).  With ``part=(rank,
    owner, comm)`` a rank context (octlb_gpu_create_part) stepping the leaves
    with owner == rank.  ``stream_order=ORDER_AA`` keeps one population
    buffer on a uniform periodic box (half the memory, the same results)."""

    def __init__(self, mesh, omega, precision=FP32, stream_mode=STREAM_ROTATE, drag=False,
                 init_pops=None, fp16_scale=None, part=None, coupler_mode=capi.COUPLER_REFERENCE,
                 omega_level=None, stream_order=capi.ORDER_AB):
        self._L = capi.lib()
        self.mesh = mesh
        self.omega = float(omega)
        self.precision = precision
        p = capi.Params()
        p.omega, p.precision, p.stream_mode, p.drag = float(omega), int(precision), int(stream_mode), int(bool(drag))
        if fp16_scale is not None:
            sc = np.broadcast_to(np.asarray(fp16_scale, dtype=np.float64), (32,))
            for i in range(32):
                p.fp16_scale[i] = float(sc[i])
        p.coupler_mode = int(coupler_mode)
        p.stream_order = int(stream_order)
        if omega_level is not None:
            for i, w in enumerate(omega_level):
                p.omega_level[i] = float(w)
        self._init = None if init_pops is None else np.ascontiguousarray(init_pops, np.float64)
        if self._init is not None:
            assert self._init.size == mesh.n_blocks * mesh.n ** 3 * Q
        h = capi.P()
        self.rank, self.owner = 0, None
        if part is None:
            rc = self._L.octlb_gpu_create(ctypes.byref(mesh.c_tables()), ctypes.byref(p),
                                          capi.ptr(self._init, ctypes.c_double), ctypes.byref(h))
        else:
            rank, owner, comm = part
            self.rank, self.owner = int(rank), np.ascontiguousarray(owner, np.int32)
            pt = capi.Partition(self.rank, comm.nranks, capi.ptr(self.owner, ctypes.c_int), comm._h)
            rc = self._L.octlb_gpu_create_part(ctypes.byref(mesh.c_tables()), ctypes.byref(p),
                                               capi.ptr(self._init, ctypes.c_double), ctypes.byref(pt),
                                               ctypes.byref(h))
        self._h = h
        if rc != 0:
            msg = self._L.octlb_gpu_last_error(h).decode() if h else "create failed"
            self.close()
            raise OctlbError(rc, msg)

    def _check(self, rc):
        if rc != 0:
            raise OctlbError(rc, self._L.octlb_gpu_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            self._L.octlb_gpu_destroy(self._h)
            self._h = None

    __del__ = close

    def set_stream(self, cuda_stream_ptr):
        """Run on the caller's cudaStream_t (an integer handle); 0 / None
        gives the context a private non-blocking stream again."""
        if not cuda_stream_ptr:
            raise ValueError("pass a non-default stream handle (the legacy default stream is not used)")
        self._check(self._L.octlb_gpu_set_stream(self._h, capi.P(cuda_stream_ptr)))

    def advance(self, n=1):
        self._check(self._L.octlb_gpu_advance(self._h, int(n)))

    def synchronize(self):
        self._check(self._L.octlb_gpu_synchronize(self._h))

    def _cells(self):
        return self.mesh.n_blocks * self.mesh.n ** 3

    def get_populations(self):
        out = np.zeros((self._cells(), Q))
        self._check(self._L.octlb_gpu_get_populations(self._h, capi.ptr(out, ctypes.c_double)))
        n = self.mesh.n
        return out.reshape(self.mesh.n_blocks, n, n, n, Q)

    def set_populations(self, pops):
        a = np.ascontiguousarray(pops, np.float64)
        assert a.size == self._cells() * Q
        self._check(self._L.octlb_gpu_set_populations(self._h, capi.ptr(a, ctypes.c_double)))

    def set_equilibrium(self, rho, u):
        """Equilibrium of per-cell fields (octlb_gpu_set_equilibrium): rho
        [n_blocks*n^3], u [n_blocks*n^3][3], float64 (ideally pinned)."""
        r = np.ascontiguousarray(rho, np.float64)
        v = np.ascontiguousarray(u, np.float64)
        assert r.size == self._cells() and v.size == 3 * self._cells()
        self._check(self._L.octlb_gpu_set_equilibrium(self._h, capi.ptr(r, ctypes.c_double),
                                                      capi.ptr(v, ctypes.c_double)))

    def get_fields(self, rho=None, u=None):
        """rho, u of every core cell; pass preallocated (ideally pinned)
        float64 arrays of n_blocks*n^3 and n_blocks*n^3*3 to fill in place."""
        rho = np.zeros(self._cells()) if rho is None else rho
        u = np.zeros((self._cells(), 3)) if u is None else u
        assert rho.dtype == np.float64 and u.dtype == np.float64 and rho.size == self._cells() and u.size == 3 * self._cells()
        assert rho.flags.c_contiguous and u.flags.c_contiguous
        self._check(self._L.octlb_gpu_get_fields(self._h, capi.ptr(rho, ctypes.c_double), capi.ptr(u, ctypes.c_double)))
        n = self.mesh.n
        return rho.reshape(self.mesh.n_blocks, n, n, n), u.reshape(self.mesh.n_blocks, n, n, n, 3)

    def force(self):
        out = np.zeros(3)
        self._check(self._L.octlb_gpu_force(self._h, capi.ptr(out, ctypes.c_double)))
        return out

    def force_sum(self):
        out = np.zeros(3)
        steps = ctypes.c_longlong(0)
        self._check(self._L.octlb_gpu_force_sum(self._h, capi.ptr(out, ctypes.c_double), ctypes.byref(steps)))
        return out, steps.value

    def force_reset(self):
        self._check(self._L.octlb_gpu_force_reset(self._h))

    def audit(self):
        out = np.zeros(4)
        self._check(self._L.octlb_gpu_audit(self._h, capi.ptr(out, ctypes.c_double)))
        return out

    def counters(self):
        c = np.zeros(32, np.int32)
        s = np.zeros(32, np.int32)
        nl = self._L.octlb_gpu_counters(self._h, capi.ptr(c, ctypes.c_int), capi.ptr(s, ctypes.c_int), 32)
        return c[:nl].tolist(), s[:nl].tolist()

    def max_level(self):
        return self._L.octlb_gpu_max_level(self._h)

    def step_stats(self):
        a, b = ctypes.c_longlong(0), ctypes.c_longlong(0)
        self._check(self._L.octlb_gpu_step_stats(self._h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def set_body_force(self, force=None):
        """Body force [n_blocks][n^3][3] (or None to remove it)."""
        f = None if force is None else np.ascontiguousarray(force, np.float64)
        if f is not None and f.size != self._cells() * 3:
            raise ValueError("body force must hold n_blocks * n^3 * 3 values")
        self._check(self._L.octlb_gpu_set_body_force(self._h, capi.ptr(f, ctypes.c_double)))

    def write_vtk(self, output_dir, base_name, step, fields=("velocity", "pressure"), rank=0, write_index=True):
        """One .vts per block of the current rho / u (octlb_gpu_write_vtk),
        plus the .vtm index and the .pvd entry of the step."""
        mask = 0
        for f in fields:
            mask |= _VTK_FIELDS[f]
        self._check(self._L.octlb_gpu_write_vtk(self._h, str(output_dir).encode(), str(base_name).encode(),
                                                int(step), int(rank), mask, 1 if write_index else 0))

    def set_fd_boundary(self, types, u_wall=None, rho_target=None, inlet_u=None, ramp_end_t=0.0, inlets=None):
        """The finite-difference domain conditions (octlb_gpu_set_fd_boundary):
        types per face (x-, x+, y-, y+, z-, z+), FD_VELOCITY or FD_PRESSURE;
        u_wall [6][3] (the y+ row is the lid), rho_target [6], inlet_u [6][3]
        (a nonzero row: that face's uniform inlet, ramped over ramp_end_t
        steps) -- or inlets, six inlet fields (fd_inlet(); None for a face
        without one; octlb_gpu_set_fd_boundary_inlets).  The mesh's kinds must
        be stamped (stamp_fd_kinds)."""
        t = np.ascontiguousarray(types, np.int32).reshape(6)
        u = np.zeros((6, 3)) if u_wall is None else np.ascontiguousarray(u_wall, np.float64).reshape(6, 3)
        r = np.ones(6) if rho_target is None else np.ascontiguousarray(rho_target, np.float64).reshape(6)
        if inlets is not None:
            arr = fd_inlets(inlets)
            self._check(self._L.octlb_gpu_set_fd_boundary_inlets(
                self._h, capi.ptr(t, ctypes.c_int), capi.ptr(u, ctypes.c_double), capi.ptr(r, ctypes.c_double), arr))
            return
        iu = None if inlet_u is None else np.ascontiguousarray(inlet_u, np.float64).reshape(6, 3)
        self._check(self._L.octlb_gpu_set_fd_boundary(self._h, capi.ptr(t, ctypes.c_int), capi.ptr(u, ctypes.c_double),
                                                      capi.ptr(r, ctypes.c_double),
                                                      capi.ptr(iu, ctypes.c_double), float(ramp_end_t)))

    def set_const_rho(self, on=True):
        """ConstRhoBGK (TimeLoop's use_const_rho_bgk): before the first
        advance; on a multi-level mesh the finest level's statistics set the
        average density every level collides at."""
        self._check(self._L.octlb_gpu_set_const_rho(self._h, 1 if on else 0))

    def average_rho(self):
        """TimeLoop::average_rho(): the density the next ConstRhoBGK collide uses."""
        out = np.zeros(1)
        self._check(self._L.octlb_gpu_average_rho(self._h, capi.ptr(out, ctypes.c_double)))
        return float(out[0])

    def adjoint(self, coarse_steps, window, checkpoint_interval=0, component=0, force_grad=True):
        """Run coarse_steps forward and the adjoint sweep back (octlb_gpu_adjoint).
        Returns (J, dJ/du_max, dJ/dtau, dJ/dF or None) with J = mean force
        component over the last `window` coarse steps."""
        p = capi.AdjParams(int(coarse_steps), int(window), int(checkpoint_interval), int(component))
        J = np.zeros(1)
        g = np.zeros(2)
        gF = np.zeros(self._cells() * 3) if force_grad else None
        self._check(self._L.octlb_gpu_adjoint(self._h, ctypes.byref(p), capi.ptr(J, ctypes.c_double),
                                              capi.ptr(g, ctypes.c_double), capi.ptr(gF, ctypes.c_double)))
        n = self.mesh.n
        return float(J[0]), float(g[0]), float(g[1]), (None if gF is None else gF.reshape(self.mesh.n_blocks, n ** 3, 3))


class GpuTimeLoop:
    """Reference TimeLoop interface (time_loop.h:47-121) over a GpuLattice."""

    def __init__(self, lattice):
        self.lattice = lattice
        self._snapshot = False

    def advance_one(self):
        self.lattice.advance(1)

    def max_level(self):
        return self.lattice.max_level()

    def counters(self):
        c, s = self.lattice.counters()
        return {"collide": c, "stream": s}

    def set_snapshot_post_collide(self, on):
        # The momentum-exchange force always reads the post-collide state the
        # step consumed; nothing extra is copied.
        self._snapshot = bool(on)

    def snapshot_post_collide(self):
        return self._snapshot
