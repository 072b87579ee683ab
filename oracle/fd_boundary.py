"""Restatement of the reference's post-stream InterpolatedVelocity / pressure
reconstruction of the domain boundary cells of one block
(ApplyInterpolatedVelocityBoundaryCells, src/solver/lbm/boundary/
interpolated_velocity.h:951-1037, with ApplyPlaneFdBoundary :571-636,
ApplyEdgeBoundary :687-752, ApplyCornerBoundary :638-685 and the
BoundaryLatticeView reads :213-445), in numpy.  TEST INFRASTRUCTURE ONLY: the
checker of a future GPU kernel, pinned against the reference build by
tests/test_fd_boundary_oracle.py.

The reference rewrites the boundary cells in place, walking (ix, iy, iz) with
z fastest.  A cell's stencil reads velocities, and, on edges and corners,
densities of the boundary neighbours one and two cells inward.  A neighbour is
already rewritten exactly when it comes earlier in that walk.  Plane cells read
only their own populations and velocities the pass does not change.  Edge
cells read plane-cell densities, and corners read edge-cell densities (blocks
of n >= 4).  So the walk is three phases, plane -> edge -> corner, each
choosing the rewritten or the original neighbour by that order rule.

Populations are the reference's shifted f - t_i, [n][n][n][19] in the
reference's D3Q19 order.  Velocity-Dirichlet cells take the prescribed
velocity; pressure cells the face's target density and the inward
neighbour's velocity.  Reads outside the block follow the view: a cell of the
overlap padding (within min(halo, 2) of the block) reads as rho = 1, u = 0;
one further out reads its mirror image inside, with the velocity components
normal to the crossed faces flipped.  On edges along y (x and z faces) the
reference pairs the x normal with the z axis and the z normal with the x axis
(ApplyEdgeBoundary's plane = 1 case); where the two normals differ in sign
that stencil reaches outside the block.  Both behaviours are restated as
they are."""
import numpy as np

# D3Q19 in the reference's order (descriptor/definition/common.h): rest, the
# nine negative-leading directions, then their opposites
C = np.array([(0, 0, 0), (-1, 0, 0), (0, -1, 0), (0, 0, -1), (-1, -1, 0), (-1, 1, 0), (-1, 0, -1), (-1, 0, 1),
              (0, -1, -1), (0, -1, 1), (1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 0), (1, -1, 0), (1, 0, 1),
              (1, 0, -1), (0, 1, 1), (0, 1, -1)], dtype=np.int64)
W = np.array([1 / 3] + [1 / 18] * 3 + [1 / 36] * 6 + [1 / 18] * 3 + [1 / 36] * 6)
INV_CS2 = 3.0
VELOCITY, PRESSURE = 5, 6  # BcKind::kVelocityDirichlet, kPressureDirichlet (bc_kind.h)


def _eq(rho, u):
    """Shifted second-order equilibrium (dynamics/lbm.h:50-64)."""
    cu = C @ u
    usq = float(u @ u)
    return rho * W * (1.0 + INV_CS2 * cu + INV_CS2 * INV_CS2 * 0.5 * cu * cu - INV_CS2 * 0.5 * usq) - W


def _fneq_from_pi(pi):
    """f_neq from the symmetric stress (xx, xy, xz, yy, yz, zz) (lbm.h:248-270)."""
    out = np.zeros(19)
    k = 0
    for a in range(3):
        for b in range(a, 3):
            q = C[:, a] * C[:, b] - (1.0 / INV_CS2 if a == b else 0.0)
            if a != b:
                q = q * 2.0
            out += q * pi[k]
            k += 1
    return out * W * INV_CS2 * INV_CS2 / 2.0


def _velocity_bm_rho(f, direction, orientation, u):
    """velocityBMRho: (2 sum_out f + sum_wall f + 1) / (1 + o u_d)."""
    wall = C[:, direction] == 0
    out = C[:, direction] == orientation
    return (2.0 * f[out].sum() + f[wall].sum() + 1.0) / (1.0 + orientation * u[direction])


class Block:
    """One block's kinds, prescribed boundary data and state for the pass."""

    def __init__(self, f_pre, kinds, omega, u_lid=(0.0, 0.0, 0.0), rho_target=None, halo=1, inlets=None, t=0.0,
                 origin=(0.0, 0.0, 0.0), cell_width=0.0):
        self.f_pre = np.asarray(f_pre, np.float64)
        self.kinds = np.asarray(kinds)
        self.n = self.kinds.shape[0]
        assert self.n >= 4 and self.kinds.shape == (self.n,) * 3
        self.omega = float(omega)
        self.u_lid = np.asarray(u_lid, np.float64)
        self.rho_target = np.ones(6) if rho_target is None else np.asarray(rho_target, np.float64)
        self.stencil = min(int(halo), 2)  # kInterpolatedVelocityOverlap = 2
        # face index (x-, x+, y-, y+, z-, z+) -> (u_const, ramp_end_t) of a
        # uniform inlet, or a dict (kind, u, u_peak, n_inplane, patch,
        # ramp_end_t) of any of the reference's inlet fields
        self.inlets = dict(inlets or {})
        self.t = float(t)
        self.origin = np.asarray(origin, np.float64)  # BlockLattice::phys_origin, phys_cell_width
        self.cell_width = float(cell_width)
        self.new = {}

    def inside(self, cell):
        return all(0 <= c < self.n for c in cell)

    def padding(self, cell):
        return (not self.inside(cell)) and self.stencil > 0 and all(
            -self.stencil <= c < self.n + self.stencil for c in cell)

    def mirror(self, cell):
        return tuple(-c if c < 0 else (2 * (self.n - 1) - c if c >= self.n else c) for c in cell)

    # --- the view's reads (interpolated_velocity.h:213-445) --------------
    def faces(self, x, y, z):
        n1 = self.n - 1
        return [(0, -1) if x == 0 else (0, 1) if x == n1 else None,
                (1, -1) if y == 0 else (1, 1) if y == n1 else None,
                (2, -1) if z == 0 else (2, 1) if z == n1 else None]

    def flat(self, x, y, z):
        fs = [f for f in self.faces(x, y, z) if f]
        return fs[0] if len(fs) == 1 else None

    @staticmethod
    def ramp(t, t_end):
        """PolynomialStartScale: 10 x^3 - 15 x^4 + 6 x^5, x = t / t_end in [0, 1]."""
        if t_end <= 0.0:
            return 1.0
        x = min(max(t / t_end, 0.0), 1.0)
        x2 = x * x
        x3 = x2 * x
        return x3 * (10.0 + x * (-15.0 + 6.0 * x))

    def prescribed_u(self, x, y, z):
        # PrescribedBoundaryU (interpolated_velocity.h:69-117): the inlet field
        # of the first face the cell touches that has one; else the lid's
        # velocity on the interior top-face cells
        n1 = self.n - 1
        for face, on in enumerate((x == 0, x == n1, y == 0, y == n1, z == 0, z == n1)):
            if on and face in self.inlets:
                spec = self.inlets[face]
                if isinstance(spec, tuple):
                    spec = {"kind": 1, "u": spec[0], "ramp_end_t": spec[1]}
                return self.inlet_velocity(spec, face, (x, y, z))
        if y == n1 and 0 < x < n1 and 0 < z < n1:
            return self.u_lid.copy()
        return np.zeros(3)

    def inlet_velocity(self, spec, face, cell):
        """The reference's inlet fields (inlet_velocity_field.h):
        UniformInletProfile (kind 1, :131-159), PoiseuilleInletProfile (2,
        block-local in-plane indices, :38-129) and ChannelPoiseuilleInletProfile
        (3, the physical position origin + (i + 1/2) cell_width on a patch,
        :163-269); in-plane axes y, z on x faces, x, z on y faces, x, y on z
        faces."""
        r = self.ramp(self.t, spec["ramp_end_t"])
        u = np.asarray(spec["u"], np.float64)
        if spec["kind"] == 1:
            return np.array([r * u[d] for d in range(3)])
        ax = face // 2
        a0, a1 = (1, 2) if ax == 0 else ((0, 2) if ax == 1 else (0, 1))
        if spec["kind"] == 2:
            c0 = (cell[a0] + 0.5) / spec["n_inplane"][0]
            c1 = (cell[a1] + 0.5) / spec["n_inplane"][1]
        else:
            lo0, hi0, lo1, hi1 = spec["patch"]
            pos = self.origin + (np.asarray(cell, np.float64) + 0.5) * self.cell_width
            c0 = min(max((pos[a0] - lo0) / (hi0 - lo0), 0.0), 1.0)
            c1 = min(max((pos[a1] - lo1) / (hi1 - lo1), 0.0), 1.0)
        mag = r * spec["u_peak"] * (4.0 * c0 * (1.0 - c0)) * (4.0 * c1 * (1.0 - c1))
        return np.array([mag * u[d] for d in range(3)])

    def pops(self, cell, reader):
        """The populations of cell as reader sees them in the in-place walk."""
        if cell in self.new and cell < reader:
            return self.new[cell]
        return self.f_pre[cell]

    def fluid_u(self, cell):
        f = self.f_pre[cell]
        rho = 1.0 + f.sum()
        return (C.T @ f) / rho

    def compute_u(self, cell):
        if not self.inside(cell):
            if self.padding(cell):
                return np.zeros(3)
            u = self.compute_u(self.mirror(cell))
            return np.array([-u[a] if not 0 <= cell[a] < self.n else u[a] for a in range(3)])
        k = self.kinds[cell]
        if k == VELOCITY:
            return self.prescribed_u(*cell)
        if k == PRESSURE:  # ExtrapolatedU: the inward neighbour's velocity
            fl = self.flat(*cell)
            if fl is None:  # a block-rim cell: u = 0 (interpolated_velocity.h:297-305)
                return np.zeros(3)
            d, o = fl
            nb = list(cell)
            nb[d] -= o
            return self.compute_u(tuple(nb))
        return self.fluid_u(cell)

    def compute_rho(self, cell, reader):
        if not self.inside(cell):
            return 1.0 if self.padding(cell) else self.compute_rho(self.mirror(cell), reader)
        k = self.kinds[cell]
        if k == PRESSURE:  # PrescribedRho (interpolated_velocity.h:320-330): 1 off a flat face
            fl = self.flat(*cell)
            return 1.0 if fl is None else self.rho_target[2 * fl[0] + (fl[1] > 0)]
        f = self.pops(cell, reader)
        if k == VELOCITY:
            fl = self.flat(*cell)
            if fl:
                return _velocity_bm_rho(f, fl[0], fl[1], self.prescribed_u(*cell))
        return 1.0 + f.sum()

    # --- the three stencils -------------------------------------------------
    def write(self, cell, rho, u, du):
        s = -rho / INV_CS2 / self.omega
        pi = np.array([2 * du[0][0], du[0][1] + du[1][0], du[0][2] + du[2][0], 2 * du[1][1],
                       du[1][2] + du[2][1], 2 * du[2][2]]) * s
        self.new[cell] = _eq(rho, u) + _fneq_from_pi(pi)

    def normal_grad(self, cell, axis, normal):
        c0 = np.array(cell)
        step = np.zeros(3, np.int64)
        step[axis] = -normal
        u0 = self.compute_u(tuple(c0))
        u1 = self.compute_u(tuple(c0 + step))
        u2 = self.compute_u(tuple(c0 + 2 * step))
        return -normal * (-3.0 * u0 + 4.0 * u1 - u2) / 2.0

    def central_grad(self, cell, axis):
        step = np.zeros(3, np.int64)
        step[axis] = 1
        c0 = np.array(cell)
        return (self.compute_u(tuple(c0 + step)) - self.compute_u(tuple(c0 - step))) / 2.0

    def plane(self, cell):
        d, o = self.flat(*cell)
        if self.kinds[cell] == PRESSURE:
            rho, u = self.rho_target[2 * d + (o > 0)], self.compute_u(cell)
        else:
            u = self.prescribed_u(*cell)
            rho = _velocity_bm_rho(self.f_pre[cell], d, o, u)
        du = [self.normal_grad(cell, a, o) if a == d else self.central_grad(cell, a) for a in range(3)]
        self.write(cell, rho, u, du)

    def edge(self, cell):
        fs = self.faces(*cell)
        nx_, ny_, nz_ = [f[1] if f else 0 for f in fs]
        # ApplyInterpolatedVelocityBoundaryCells' choice (interpolated_velocity.h:991-1012)
        if nx_ and ny_:
            plane, n1, n2 = 2, nx_, ny_
        elif nx_ and nz_:
            plane, n1, n2 = 1, nx_, nz_
        else:
            plane, n1, n2 = 0, ny_, nz_
        d1, d2 = (plane + 1) % 3, (plane + 2) % 3

        def rho_at(s1, s2):
            c = list(cell)
            c[d1] -= n1 * s1
            c[d2] -= n2 * s2
            return self.compute_rho(tuple(c), cell)

        rho = 2.0 / 3.0 * (rho_at(0, 1) + rho_at(1, 0)) - 1.0 / 6.0 * (rho_at(0, 2) + rho_at(2, 0))
        du = [None] * 3
        du[plane] = self.central_grad(cell, plane)
        du[d1] = self.normal_grad(cell, d1, n1)
        du[d2] = self.normal_grad(cell, d2, n2)
        self.write(cell, rho, self.compute_u(cell), du)

    def corner(self, cell):
        fs = self.faces(*cell)

        def rho_at(a, s):
            c = list(cell)
            c[a] -= fs[a][1] * s
            return self.compute_rho(tuple(c), cell)

        rho = 4.0 / 9.0 * (rho_at(2, 1) + rho_at(1, 1) + rho_at(0, 1)) - 1.0 / 9.0 * (
            rho_at(2, 2) + rho_at(1, 2) + rho_at(0, 2))
        du = [self.normal_grad(cell, a, fs[a][1]) for a in range(3)]
        self.write(cell, rho, self.compute_u(cell), du)


def reconstruct(f_pre, kinds, omega, u_lid=(0.0, 0.0, 0.0), rho_target=None, halo=1, inlets=None, t=0.0,
                origin=(0.0, 0.0, 0.0), cell_width=0.0):
    """The block's populations after the pass: boundary cells (velocity or
    pressure Dirichlet on the block's faces) rewritten in three phases, the
    others unchanged."""
    b = Block(f_pre, kinds, omega, u_lid, rho_target, halo, inlets, t, origin, cell_width)
    cells = [tuple(c) for c in np.argwhere(np.isin(b.kinds, (VELOCITY, PRESSURE)))]
    count = {c: sum(1 for f in b.faces(*c) if f) for c in cells}
    for want, fn in ((1, b.plane), (2, b.edge), (3, b.corner)):
        for c in cells:
            if count[c] == want:
                fn(c)
    out = b.f_pre.copy()
    for c, f in b.new.items():
        out[c] = f
    return out


def collide(f, kinds, omega, u_lid=(0.0, 0.0, 0.0), average_rho=None, stats=None):
    """The collide of a block with the FD domain conditions, OpenLB order
    (BcDispatcher::collide, bc_dispatcher.h:33-79): kBulk cells f <- (1 - omega)
    f + omega f_eq(rho, u) (lbm.h:395-403) at their own moments; velocity-
    Dirichlet cells the same at the prescribed velocity and the density of
    BoundaryCellStatisticRho (interpolated_velocity.h:815-884: velocityBMRho
    on plane cells, 1 + sum f on edges and corners); other kinds unchanged.
    Every cell reads only itself, so the order does not matter.

    average_rho (ConstRhoBGK): kBulk cells take ratio (f_eq + t) - t +
    (1 - omega)(f - f_eq), ratio = 1 + (1 - average_rho) / rho
    (block_lattice.h:134-151); stats (a list) gets rho + 1 - average_rho per
    kBulk cell and the raw boundary density per velocity-Dirichlet cell (the
    kFluidAndBoundary scope)."""
    b = Block(f, kinds, omega, u_lid)
    out = b.f_pre.copy()
    n = b.n
    for x in range(n):
        for y in range(n):
            for z in range(n):
                c = (x, y, z)
                k = b.kinds[c]
                g = b.f_pre[c]
                if k == 0:
                    rho = 1.0 + g.sum()
                    u = (C.T @ g) / rho
                elif k == VELOCITY:
                    u = b.prescribed_u(*c)
                    fl = b.flat(*c)
                    rho = _velocity_bm_rho(g, fl[0], fl[1], u) if fl else 1.0 + g.sum()
                else:
                    continue
                feq = _eq(rho, u)
                if k == 0 and average_rho is not None:
                    ratio = 1.0 + (1.0 - average_rho) / rho if rho > 1e-12 else 1.0
                    out[c] = ratio * (feq + W) - W + (1.0 - omega) * (g - feq)
                    if stats is not None:
                        stats.append(rho + (1.0 - average_rho))
                    continue
                if k == VELOCITY and average_rho is not None and stats is not None:
                    stats.append(rho)
                out[c] = g * (1.0 - omega) + omega * feq
    return out


def stream_padded(p):
    """The torus-rotate stream of a padded block ([n+2][n+2][n+2][19], halo 1):
    population i of padded cell s comes from cell s - (c_x (n+2)^2 + c_y (n+2)
    + c_z), wrapped over the block's linear index
    (OpenLbPaddedBlockStreamSourceLinear; block_lattice.cpp:554-575)."""
    m = p.shape[0]
    flat = p.reshape(-1, 19)
    out = np.empty_like(flat)
    for i in range(19):
        out[:, i] = np.roll(flat[:, i], int(C[i][0] * m * m + C[i][1] * m + C[i][2]))
    return out.reshape(p.shape)
