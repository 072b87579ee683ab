"""Parity of the sm_100a path (through the C ABI) with the CPU oracles.

Tolerances (plain FP32 path): max |rho_gpu - rho_ref| / max |rho_ref| and
max |u_gpu - u_ref| / max |u_ref| <= 1e-5 after N steps, against the
reference's own FP64 code (oracle/_ref) or its C restatement.  FP16-shifted
storage: <= 2e-3 on the same fields.
"""
import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu

TOL32 = 1e-5
TOL16 = 2e-3


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def fields_of(pops):
    return oracle.rho_u(pops)


def test_tgv_periodic_fp32_matches_oracle(ob, orc):
    from octlb_b200 import cases
    n, steps = 32, 200
    mesh, init, info = cases.tgv_periodic(n, u0=0.05, tau=0.55)
    lat = ob.GpuLattice(mesh, info["omega"], precision=ob.FP32, init_pops=init)
    lat.advance(steps)
    rho_g, u_g = lat.get_fields()
    blk = oracle.Block(orc, n)
    blk.set_core(init[0])
    blk.run_periodic(info["omega"], steps)
    rho_o, u_o = fields_of(blk.core())
    assert rel(rho_g[0], rho_o) <= TOL32
    assert rel(u_g[0], u_o) <= TOL32
    # post-collision populations = oracle state after one more collide
    blk.collide(info["omega"])
    assert rel(lat.get_populations()[0], blk.core()) <= 1e-4


def test_tgv_periodic_fp16_shifted(ob, orc):
    from octlb_b200 import cases
    n, steps = 32, 100
    mesh, init, info = cases.tgv_periodic(n, u0=0.05, tau=0.55)
    lat = ob.GpuLattice(mesh, info["omega"], precision=ob.FP16_SHIFTED, init_pops=init)
    lat.advance(steps)
    rho_g, u_g = lat.get_fields()
    blk = oracle.Block(orc, n)
    blk.set_core(init[0])
    blk.run_periodic(info["omega"], steps)
    rho_o, u_o = fields_of(blk.core())
    assert rel(rho_g[0], rho_o) <= TOL16
    assert rel(u_g[0], u_o) <= TOL16


def test_cavity_shell_matches_reference(ob, ref):
    """Solid shell + q = 1 link table: the reference's own half-way
    bounce-back (block_lattice.cpp:667-669) plus the moving-lid term."""
    from octlb_b200 import cases
    n, steps = 16, 300
    mesh, init, info = cases.cavity_shell(n, lid=0.1, tau=0.6)
    lat = ob.GpuLattice(mesh, info["omega"], stream_mode=ob.STREAM_LINKS, init_pops=init)
    lat.advance(steps)
    rho_g, u_g = lat.get_fields()
    m = n + 2
    blk = oracle.Block(ref, m)
    blk.set_kinds(mesh.kinds[0])
    blk.set_links(np.zeros((0, 4), np.int32), np.zeros(0))
    blk.set_core(init[0])
    blk.run_walls(info["omega"], steps, mesh.moving[0], mesh.wall_u[0])
    rho_r, u_r = fields_of(blk.core())
    fl = mesh.kinds[0] == ob.BULK
    assert rel(rho_g[0][fl], rho_r[fl]) <= TOL32
    assert rel(u_g[0][fl], u_r[fl]) <= TOL32
    assert np.abs(u_r[fl]).max() > 0.01  # the lid drives the flow


def test_links_bouzidi_random_state_one_step(ob, ref):
    """Random post-collide state, cut links with q on both branches, reflect
    kinds: one GPU step equals the reference's stream followed by collide."""
    rng = np.random.default_rng(7)
    n = 10
    kinds = np.zeros((n, n, n), np.uint8)
    kinds[6:, :, :] = ob.SOLID
    kinds[5, 2:4, :] = ob.BOUZIDI
    kinds[3, 3, 3] = ob.VELOCITY_DIRICHLET
    cells = []
    qs = []
    for y in range(n):
        for z in range(n):
            for i in (1, 4, 5, 6, 7):        # directions pulling from +x (solid side)
                if kinds[5, y, z] != ob.SOLID:
                    cells.append((0, 5, y, z, i))
                    qs.append(rng.uniform(0.05, 0.95))
    mesh = ob.Mesh(n, [0], [0, 0, 0, 1, 1, 1], kinds=kinds[None],
                   link_cells=np.array(cells), link_q=np.array(qs))
    pre = rng.standard_normal((1, n, n, n, 19)) * 1e-3
    omega = 1.3
    # GPU: state = C(pre); one step = stream + collide
    lat = ob.GpuLattice(mesh, omega, stream_mode=ob.STREAM_LINKS, init_pops=pre)
    g0 = lat.get_populations()[0]
    lat.advance(1)
    g1 = lat.get_populations()[0]
    blk = oracle.Block(ref, n)
    blk.set_kinds(kinds)
    blk.set_links(np.array(cells)[:, 1:], np.array(qs))
    blk.set_core(pre[0])
    blk.collide(omega)
    assert rel(g0, blk.core()) <= 1e-5
    blk.stream()
    blk.collide(omega)
    core = blk.core()
    # halo-adjacent cells read stale halo values on both sides (zeros at start)
    assert rel(g1, core) <= 1e-5


@pytest.mark.parametrize("band,n", [(0, 8), (8, 8), (16, 16)])
def test_cavity_forest_matches_reference(ob, ref, band, n):
    """Cavity forests (one level, or a refined band under the moving lid) with
    8^3 and 16^3 blocks, fields and counters against the reference TimeLoop."""
    from octlb_b200 import cases
    mesh, init, info = cases.cavity_forest(cells=32 if n == 8 else 64, n=n, lid=0.1, tau=0.6, band_cells=band)
    steps = 10
    lat = ob.GpuLattice(mesh, info["omega"], init_pops=init)
    lat.advance(steps)
    rho_g, u_g = lat.get_fields()
    sim = oracle.Sim(ref, mesh, info["omega"], init)
    sim.advance(steps)
    rho_r, u_r = fields_of(sim.core())
    assert rel(rho_g, rho_r) <= TOL32
    assert rel(u_g, u_r) <= TOL32
    c, s = lat.counters()
    cr, sr, _ = sim.counters()
    assert c == cr and s == sr


def test_audit_mass_conserved_periodic(ob):
    from octlb_b200 import cases
    mesh, init, info = cases.tgv_periodic(32, u0=0.05, tau=0.55)
    lat = ob.GpuLattice(mesh, info["omega"], init_pops=init)
    a0 = lat.audit()
    lat.advance(100)
    a1 = lat.audit()
    assert abs(a1[0] - a0[0]) / a0[0] < 1e-6
    assert np.all(np.abs(a1[1:] - a0[1:]) < 1e-6 * a0[0])


@pytest.mark.parametrize("prec", ["fp32", "fp16"])
def test_step_kernel_variants_bitwise_equal(ob, prec, monkeypatch):
    """The paired vector step, the pipelined bulk-copy step and the plain step
    kernel compute the same arithmetic on the same pulled values: identical
    populations."""
    from octlb_b200 import cases
    p = ob.FP32 if prec == "fp32" else ob.FP16_SHIFTED
    mesh, init, info = cases.tgv_periodic(64, u0=0.05, tau=0.55)
    outs = []
    for variant in ("pair", "bulk", "plain"):
        monkeypatch.setenv("OCTLB_STEP_KERNEL", variant)
        lat = ob.GpuLattice(mesh, info["omega"], precision=p, init_pops=init)
        lat.advance(25)
        outs.append(lat.get_populations())
        lat.close()
    assert np.array_equal(outs[0], outs[1]) and np.array_equal(outs[0], outs[2])


def small_cylinder(ob, n=8):
    from octlb_b200 import cases
    if n == 16:
        return cases.cylinder_forest(length=128, height=64, n=16, diameter=8.0, center=(32.0, 32.0),
                                     levels=2, u_max=0.05, re=40.0)
    return cases.cylinder_forest(length=128, height=32, n=8, diameter=8.0, center=(32.0, 16.0),
                                 levels=2, u_max=0.05, re=40.0)


@pytest.mark.parametrize("n", [8, 16])
def test_cylinder_two_levels_matches_reference_with_drag(ob, ref, n):
    """Two-level channel with an exact-circle Bouzidi cylinder, parabolic
    inlet, zero-gradient outlet, periodic z: fields and the momentum-exchange
    force per coarse step against the reference TimeLoop + MomentumExchangeDrag
    (8^3 and 16^3 blocks).  The force is a sum of ~10^3 link terms of the
    shifted populations; while the start-up wave reaches the cylinder it is a
    small difference of those (1e-4 against terms of ~1e-3), whose FP32
    rounding is ~1e-8 absolute, so the tolerance is 1e-5 of max(|F|, 1e-2)."""
    mesh, init, info = small_cylinder(ob, n)
    assert len(mesh.link_q) > 0 and len(mesh.coarse_fine) > 0
    lat = ob.GpuLattice(mesh, info["omega"], stream_mode=ob.STREAM_LINKS, drag=True, init_pops=init)
    sim = oracle.Sim(ref, mesh, info["omega"], init, link_mode=True)
    for step in range(12):
        lat.advance(1)
        sim.advance(1)
        fg, fr = lat.force(), sim.drag(mesh.obstacle)
        assert np.max(np.abs(fg - fr)) <= 1e-5 * max(np.max(np.abs(fr)), 1e-2), (step, fg, fr)
    rho_g, u_g = lat.get_fields()
    rho_r, u_r = fields_of(sim.core())
    fl = mesh.kinds == ob.BULK
    assert rel(rho_g[fl], rho_r[fl]) <= TOL32
    assert rel(u_g[fl], u_r[fl]) <= TOL32
    fs, nsteps = lat.force_sum()
    assert nsteps == 12 and np.all(np.isfinite(fs))


def test_cylinder_fp16_drag_close_to_fp32(ob):
    mesh, init, info = small_cylinder(ob)
    forces = {}
    for p in (ob.FP32, ob.FP16_SHIFTED):
        lat = ob.GpuLattice(mesh, info["omega"], precision=p, stream_mode=ob.STREAM_LINKS, drag=True,
                            init_pops=init)
        lat.advance(200)
        lat.force_reset()
        lat.advance(100)
        forces[p] = lat.force_sum()[0] / 100.0
        lat.close()
    f32, f16 = forces[ob.FP32], forces[ob.FP16_SHIFTED]
    assert abs(f16[0] - f32[0]) <= 1e-2 * abs(f32[0])


def test_amr_cavity_fp16_fields(ob, ref):
    from octlb_b200 import cases
    mesh, init, info = cases.cavity_forest(cells=32, n=8, lid=0.1, tau=0.6, band_cells=8)
    lat = ob.GpuLattice(mesh, info["omega"], precision=ob.FP16_SHIFTED, init_pops=init)
    lat.advance(10)
    rho_g, u_g = lat.get_fields()
    sim = oracle.Sim(ref, mesh, info["omega"], init)
    sim.advance(10)
    rho_r, u_r = fields_of(sim.core())
    assert rel(u_g, u_r) <= 5e-3
    assert rel(rho_g, rho_r) <= 5e-3


@pytest.mark.parametrize("case", ["cylinder_fp32", "cylinder_fp16", "cavity_band_fp16"])
def test_forest_map_step_bitwise_equals_plain(ob, case, monkeypatch):
    """On forest levels the slot-map step (one CTA per block, the block's
    padded-position -> slot map in shared memory, one or two cells per
    thread) and the one-cell-per-thread k_step give identical populations
    and forces: same pulls, same arithmetic."""
    from octlb_b200 import cases
    p = ob.FP16_SHIFTED if case.endswith("fp16") else ob.FP32
    if case.startswith("cylinder"):
        mesh, init, info = small_cylinder(ob)
        kw = dict(stream_mode=ob.STREAM_LINKS, drag=True)
    else:
        mesh, init, info = cases.cavity_forest(cells=32, n=8, lid=0.1, tau=0.6, band_cells=8)
        kw = {}
    res = []
    for variant, cells in (("map", "2"), ("map", "1"), ("plain", "2")):
        monkeypatch.setenv("OCTLB_STEP_KERNEL", variant)
        monkeypatch.setenv("OCTLB_MAP_CELLS", cells)
        lat = ob.GpuLattice(mesh, info["omega"], precision=p, init_pops=init, **kw)
        lat.advance(6)
        res.append((lat.get_populations(), lat.force() if kw else None))
        lat.close()
    for r in res[1:]:
        assert np.array_equal(res[0][0], r[0])
        if kw:
            assert np.array_equal(res[0][1], r[1])


@pytest.mark.parametrize("case", ["cylinder", "cavity_band"])
def test_graph_and_programmatic_launch_bitwise_equal(ob, case, monkeypatch):
    """advance_one captured as CUDA graphs (one per buffer parity), launched
    kernel by kernel, and either way with or without programmatic dependent
    launches gives the same populations, forces and counters."""
    from octlb_b200 import cases
    if case == "cylinder":
        mesh, init, info = small_cylinder(ob)
        kw = dict(stream_mode=ob.STREAM_LINKS, drag=True)
    else:
        mesh, init, info = cases.cavity_forest(cells=32, n=8, lid=0.1, tau=0.6, band_cells=8)
        kw = {}
    res = []
    for ng, npdl in (("0", "0"), ("1", "0"), ("0", "1"), ("1", "1")):
        monkeypatch.setenv("OCTLB_NO_GRAPH", ng)
        monkeypatch.setenv("OCTLB_NO_PDL", npdl)
        lat = ob.GpuLattice(mesh, info["omega"], init_pops=init, **kw)
        forces = []
        for _ in range(5):
            lat.advance(1)
            forces.append(lat.force() if kw else np.zeros(3))
        lat.advance(4)
        res.append((lat.get_populations(), np.array(forces), lat.counters(),
                    lat.force_sum() if kw else (np.zeros(3), 9)))
        lat.close()
    p0, f0, c0, s0 = res[0]
    for p1, f1, c1, s1 in res[1:]:
        assert np.array_equal(p0, p1) and np.array_equal(f0, f1) and c0 == c1
        assert np.array_equal(s0[0], s1[0]) and s0[1] == s1[1] == 9


def test_body_force_matches_reference(ob, ref):
    """A nonzero per-cell body force: GPU fields and MEM force per coarse step
    against the reference TimeLoop with the same forcing term added at its
    DomainBoundaryHandler::apply() hook (restated there)."""
    mesh, init, info = small_cylinder(ob)
    rng = np.random.default_rng(7)
    F = rng.normal(0.0, 1e-5, size=(mesh.n_blocks, mesh.n ** 3, 3))
    F[..., 0] += 2e-5
    lat = ob.GpuLattice(mesh, info["omega"], stream_mode=ob.STREAM_LINKS, drag=True, init_pops=init)
    lat.set_body_force(F)
    sim = oracle.Sim(ref, mesh, info["omega"], init, link_mode=True)
    sim.set_body_force(F)
    for step in range(10):
        lat.advance(1)
        sim.advance(1)
        fg, fr = lat.force(), sim.drag(mesh.obstacle)
        assert np.max(np.abs(fg - fr)) <= 1e-5 * max(np.max(np.abs(fr)), 1e-6), (step, fg, fr)
    rho_g, u_g = lat.get_fields()
    rho_r, u_r = fields_of(sim.core())
    fl = mesh.kinds == ob.BULK
    assert rel(rho_g[fl], rho_r[fl]) <= TOL32
    assert rel(u_g[fl], u_r[fl]) <= TOL32
    # removing the force restores the plain forward
    lat.set_body_force(None)
    lat.close()


def test_adjoint_and_body_force_argument_checks(ob):
    mesh, init, info = small_cylinder(ob)
    lat16 = ob.GpuLattice(mesh, info["omega"], precision=ob.FP16_SHIFTED, stream_mode=ob.STREAM_LINKS, drag=True,
                          init_pops=init)
    with pytest.raises(ob.OctlbError):
        lat16.adjoint(4, 2)                  # FP16 storage is not differentiated
    lat16.close()
    nodrag = ob.GpuLattice(mesh, info["omega"], stream_mode=ob.STREAM_LINKS, init_pops=init)
    with pytest.raises(ob.OctlbError):
        nodrag.adjoint(4, 2)                 # the objective needs the drag
    nodrag.close()
    lat = ob.GpuLattice(mesh, info["omega"], stream_mode=ob.STREAM_LINKS, drag=True, init_pops=init)
    for steps, window in ((0, 0), (4, 0), (4, 5)):
        with pytest.raises(ob.OctlbError):
            lat.adjoint(steps, window)
    bad = np.zeros((mesh.n_blocks, mesh.n ** 3, 3))
    bad[0, 0, 0] = np.nan
    with pytest.raises(ob.OctlbError):
        lat.set_body_force(bad)
    with pytest.raises(ValueError):
        lat.set_body_force(np.zeros(5))
    lat.close()


@pytest.mark.parametrize("prec,tol", [("fp32", TOL32), ("fp16", TOL16)])
def test_periodic_three_level_forest_matches_reference(ob, ref, prec, tol):
    """A fully periodic forest with interior hanging faces on two nested
    levels (32^3 base cells at level 2, the central half refined to level 3
    and its central quarter to level 4), started from a uniform moving state:
    fields against the reference TimeLoop, and the collide counters in its
    1:2:4 ratio (test_time_loop_levels.cpp:66-149).  (The reference does not
    keep this state uniform: the coarse blocks' ghost cells toward a finer
    neighbour are never filled and keep their initial rest values.)"""
    from octlb_b200 import C, Forest, Mesh
    f = Forest((1, 1, 1), (1, 1, 1), (0, 0, 0, 1, 1, 1)).refine_uniform(2)
    f.refine_box((0.25, 0.25, 0.25, 0.75, 0.75, 0.75), 3)
    f.refine_box((0.375, 0.375, 0.375, 0.625, 0.625, 0.625), 4)
    f.balance().build()
    n = 8
    mesh = Mesh.from_forest(f, n)
    assert sorted(set(mesh.levels.tolist())) == [2, 3, 4]
    rho0, u0 = 1.02, np.array([0.03, -0.02, 0.01])
    Cf = C.astype(np.float64)
    w = np.where(np.abs(Cf).sum(1) == 0, 1 / 3, np.where(np.abs(Cf).sum(1) == 1, 1 / 18, 1 / 36))
    cu = Cf @ u0
    feq = w * (rho0 * (1 + 3 * cu + 4.5 * cu * cu - 1.5 * u0 @ u0) - 1)
    init = np.broadcast_to(feq, (mesh.n_blocks, n, n, n, 19)).copy()
    omega, steps = 1.0 / 0.6, 3
    lat = ob.GpuLattice(mesh, omega, precision=ob.FP32 if prec == "fp32" else ob.FP16_SHIFTED, init_pops=init)
    sim = oracle.Sim(ref, mesh, omega, init)
    lat.advance(steps)
    sim.advance(steps)
    rho_g, u_g = lat.get_fields()
    c, s = lat.counters()
    lat.close()
    rho_r, u_r = fields_of(sim.core())
    cr, sr, _ = sim.counters()
    assert rel(rho_g, rho_r) <= tol
    assert rel(u_g, u_r) <= tol
    assert c == cr and s == sr
    assert c[2] == steps * 4 and c[3] == 2 * c[2] and c[4] == 4 * c[2]


def test_host_staging_reuse_across_calls(ob):
    """set/get_populations and get_fields stage through FP64 buffers the
    context keeps: calls of different sizes in any order give the values a
    fresh context gives."""
    from octlb_b200 import cases
    mesh, init, info = cases.cavity_forest(cells=32, n=8, lid=0.1, tau=0.6, band_cells=8)
    rng = np.random.default_rng(11)
    state = init + 1e-3 * rng.standard_normal(init.shape)
    lat = ob.GpuLattice(mesh, info["omega"], init_pops=init)
    lat.advance(2)
    rho1, u1 = (a.copy() for a in lat.get_fields())      # fields staging first
    pops = lat.get_populations().copy()                    # then the larger populations staging
    rho2, u2 = lat.get_fields()
    assert np.array_equal(rho1, rho2) and np.array_equal(u1, u2)
    rho_p, u_p = oracle.rho_u(pops)
    assert rel(rho_p, rho1) <= 1e-12 and rel(u_p, u1) <= 1e-10
    lat.set_populations(state)
    fresh = ob.GpuLattice(mesh, info["omega"], init_pops=state)
    assert np.array_equal(lat.get_populations(), fresh.get_populations())
    assert np.array_equal(lat.get_fields()[0], fresh.get_fields()[0])
    lat.close()
    fresh.close()
