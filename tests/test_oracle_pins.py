"""Pins of the CPU oracles (CPU only).

1. The C restatement (oracle/octlb_oracle.c) against the reference's own code
   compiled from its sources (oracle/_ref): identical to 1e-13 on the periodic
   rotate path and the per-cell link path (Bouzidi, reflect kinds, moving wall)
   and in the momentum-exchange force.
2. Both oracles against the reference's own unit-test known answers
   (tests/unit/solver/test_collision_bgk.cpp, test_bouzidi_link.cpp,
   test_drag_postprocessor.cpp).
3. The restatement against committed golden vectors made by the reference
   build (tests/golden/make_golden.py), so the pin holds where oracle/_ref is
   absent.
"""
import os

import numpy as np
import pytest

from oracle import oracle

HERE = os.path.dirname(os.path.abspath(__file__))

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
Q = 19
C = np.array([[0, 0, 0], [-1, 0, 0], [0, -1, 0], [0, 0, -1], [-1, -1, 0], [-1, 1, 0], [-1, 0, -1],
              [-1, 0, 1], [0, -1, -1], [0, -1, 1], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 1, 0],
              [1, -1, 0], [1, 0, 1], [1, 0, -1], [0, 1, 1], [0, 1, -1]])
OPP = [0, 10, 11, 12, 13, 14, 15, 16, 17, 18, 1, 2, 3, 4, 5, 6, 7, 8, 9]
W = np.array([1 / 3] + [1 / 18] * 3 + [1 / 36] * 6 + [1 / 18] * 3 + [1 / 36] * 6)


def both(orc, ref):
    return [(orc, "orc"), (ref, "ref")]


def link_case(L, steps=5):
    """Random padded state, solid half, Bouzidi / reflecting kinds, cut links,
    moving top layer; collide -> snapshot -> stream -> moving-wall term."""
    n = 6
    rng = np.random.default_rng(1)
    b = oracle.Block(L, n)
    b.set_padded(rng.standard_normal((n + 2, n + 2, n + 2, Q)) * 1e-3)
    kinds = np.zeros((n, n, n), np.uint8)
    kinds[0] = 1
    kinds[-1] = 1
    kinds[:, 0] = 1
    kinds[:, -1] = 1
    kinds[2, 3, :] = 4
    kinds[3, 2, 2] = 5
    b.set_kinds(kinds)
    b.set_links(np.array([[1, 3, 2, 10], [3, 3, 3, 1], [2, 2, 2, 5], [2, 4, 2, 2]]), np.array([0.3, 0.7, 0.5, 0.2]))
    mov = np.zeros((n, n, n), np.uint8)
    mov[:, -1, :] = 1
    uw = np.zeros((n, n, n, 3))
    uw[..., 0] = 0.1
    for _ in range(steps):
        b.collide(1.7)
        b.snapshot()
        b.stream()
        b.add_moving_wall(mov, uw)
    return b


def test_restatement_matches_reference_periodic(orc, ref):
    n = 6
    rng = np.random.default_rng(3)
    pad = rng.standard_normal((n + 2, n + 2, n + 2, Q)) * 1e-3
    outs = []
    for L, _ in both(orc, ref):
        b = oracle.Block(L, n)
        b.set_padded(pad)
        b.run_periodic(1.7, 7)
        outs.append(b.padded())
    assert np.max(np.abs(outs[0] - outs[1])) < 1e-13


def test_restatement_matches_reference_links(orc, ref):
    bo, br = link_case(orc), link_case(ref)
    assert np.max(np.abs(bo.padded() - br.padded())) < 1e-13
    assert np.max(np.abs(bo.drag() - br.drag())) < 1e-13


def test_restatement_matches_reference_rotate_nonperiodic(orc, ref):
    """Torus-rotate stream over the padded block (no link table, halo never
    filled): the reference's OpenLB-rotate path, block_lattice.cpp:554-577."""
    n = 5
    rng = np.random.default_rng(4)
    pad = rng.standard_normal((n + 2, n + 2, n + 2, Q)) * 1e-3
    kinds = (rng.random((n, n, n)) < 0.2).astype(np.uint8)
    outs = []
    for L, _ in both(orc, ref):
        b = oracle.Block(L, n)
        b.set_padded(pad)
        b.set_kinds(kinds)
        for _ in range(4):
            b.collide(1.2)
            b.stream()
        outs.append(b.padded())
    assert np.max(np.abs(outs[0] - outs[1])) < 1e-13


@pytest.mark.parametrize("which", ["orc", "ref"])
def test_kat_bgk_conserves_mass_and_momentum(orc, ref, which):
    """test_collision_bgk.cpp:52-81: 8^3 periodic, omega = 1.4, 100 steps."""
    L = orc if which == "orc" else ref
    b = oracle.Block(L, 8)
    b.initialize(1.0, (0.0, 0.0, 0.0))
    rng = np.random.default_rng(5)
    core = b.core() + rng.standard_normal((8, 8, 8, Q)) * 1e-3   # nontrivial state
    b.set_core(core)
    rho0, u0 = oracle.rho_u(b.core())
    m0, p0 = rho0.sum(), (rho0[..., None] * u0).sum((0, 1, 2))
    b.run_periodic(1.4, 100)
    rho1, u1 = oracle.rho_u(b.core())
    assert abs(rho1.sum() - m0) < 1e-10
    assert np.all(np.abs((rho1[..., None] * u1).sum((0, 1, 2)) - p0) < 1e-10)


@pytest.mark.parametrize("which", ["orc", "ref"])
def test_kat_sin_mode_decays(orc, ref, which):
    """test_collision_bgk.cpp:92-135: u_x = 0.05 sin(2 pi i / 8) damps to a
    spread below 1e-5 after 400 steps at omega = 1.4."""
    L = orc if which == "orc" else ref
    n = 8
    b = oracle.Block(L, n)
    ux = 0.05 * np.sin(2 * np.pi * np.arange(n) / n)
    u = np.zeros((n, n, n, 3))
    u[..., 0] = ux[:, None, None]
    cu = np.einsum("xyzd,qd->xyzq", u, C)
    usq = (u * u).sum(-1)[..., None]
    b.set_core(W * (1 + 3 * cu + 4.5 * cu * cu - 1.5 * usq) - W)
    s0 = np.ptp(oracle.rho_u(b.core())[1][..., 0])
    b.run_periodic(1.4, 400)
    s1 = np.ptp(oracle.rho_u(b.core())[1][..., 0])
    assert s0 > s1 and s1 < 1e-5


@pytest.mark.parametrize("which", ["orc", "ref"])
def test_kat_bouzidi_replaces_solid_pull(orc, ref, which):
    """test_bouzidi_link.cpp:105-155: the pulled value at a cut link equals
    BouzidiPostCollisionPull(f_bb, f_same, f_same, 0.35)."""
    L = orc if which == "orc" else ref
    n = 8
    b = oracle.Block(L, n)
    b.initialize(1.0, (0.0, 0.0, 0.0))
    kinds = np.zeros((n, n, n), np.uint8)
    kinds[n // 2:] = 1
    b.set_kinds(kinds)
    i, ipop, q = n // 2 - 1, 1, 0.35
    b.set_links(np.array([[i, 0, 0, ipop]]), np.array([q]))
    b.collide(1.0)
    core = b.core()
    core[i, 0, 0, 3] += 0.05
    b.set_core(core)
    f_bb, f_same = core[i, 0, 0, OPP[ipop]], core[i, 0, 0, ipop]
    pull = getattr(L, L._pre + "bouzidi_pull")
    expected = pull(f_bb, f_same, f_same, q)
    b.stream()
    assert abs(b.core()[i, 0, 0, ipop] - expected) < 1e-12
    # the formula's branches (bouzidi_pull.h:11-25)
    assert pull(0.3, 0.1, 0.2, 1.0) == 0.3 and pull(0.3, 0.1, 0.2, 0.0) == 0.3
    assert abs(pull(0.3, 0.1, 0.2, 0.25) - (0.5 * 0.3 + 0.5 * 0.2)) < 1e-15
    assert abs(pull(0.3, 0.1, 0.2, 0.75) - (0.3 / 1.5 + (1 - 1 / 1.5) * 0.1)) < 1e-15


@pytest.mark.parametrize("which", ["orc", "ref"])
def test_kat_drag_known_force(orc, ref, which):
    """test_drag_postprocessor.cpp:29-70: one +x link at rest gives
    F_x = -1/9; a +x free stream gives F_x < 0."""
    L = orc if which == "orc" else ref
    b = oracle.Block(L, 3, 1, 1)
    kinds = np.zeros((3, 1, 1), np.uint8)
    kinds[1:] = 1
    b.set_kinds(kinds)
    pad = b.padded()
    pad[1, 1, 1] = W
    b.set_padded(pad)
    f = b.drag()
    assert abs(f[0] + 1.0 / 9.0) < 1e-12 and abs(f[1]) < 1e-12 and abs(f[2]) < 1e-12
    U = 0.1
    cu = C[:, 0] * U
    pad[1, 1, 1] = W * (1 + 3 * cu + 4.5 * cu * cu - 1.5 * U * U)
    b.set_padded(pad)
    f = b.drag()
    assert f[0] < 0 and abs(f[1]) < 1e-12 and abs(f[2]) < 1e-12


def test_golden_vectors_restatement(orc):
    """Restatement against vectors the reference build produced
    (tests/golden/make_golden.py)."""
    path = os.path.join(GOLDEN, "block_paths.npz")
    g = np.load(path)
    n = int(g["periodic_n"])
    b = oracle.Block(orc, n)
    b.set_padded(g["periodic_in"])
    b.run_periodic(float(g["periodic_omega"]), int(g["periodic_steps"]))
    assert np.max(np.abs(b.padded() - g["periodic_out"])) < 1e-13
    b = link_case(orc)
    assert np.max(np.abs(b.padded() - g["links_out"])) < 1e-13
    assert np.max(np.abs(b.drag() - g["links_drag"])) < 1e-13


def test_golden_amr_cavity_reference_state(ref):
    """The reference's AMR TimeLoop on the committed two-level cavity
    reproduces the committed golden state (guards the oracle build)."""
    g = np.load(os.path.join(GOLDEN, "amr_cavity.npz"))
    import octlb_b200 as ob
    from octlb_b200 import cases
    mesh, init, info = cases.cavity_forest(cells=16, n=8, lid=0.1, tau=0.6, band_cells=8)
    assert np.array_equal(mesh.levels, g["levels"])
    sim = oracle.Sim(ref, mesh, info["omega"], init)
    sim.advance(int(g["steps"]))
    rho, u = oracle.rho_u(sim.core())
    assert np.max(np.abs(rho - g["rho"])) < 1e-12 and np.max(np.abs(u - g["u"])) < 1e-12


def test_threaded_restatement_reproduces_reference_tgv64_history(orc):
    """The C restatement's threaded periodic loop (the checker of the 256^3
    GPU test and of the bench's accuracy leg) reproduces the reference's own
    BlockLattice<double> run of the 64^3 Taylor-Green vortex over 1,000 steps
    (tests/golden/tgv64_reference.npz): kinetic energy and mass every 10
    steps, final fields on the sampled lattice, all to 1e-12."""
    from octlb_b200 import cases
    g = np.load(os.path.join(HERE, "golden", "tgv64_reference.npz"))
    n, every, steps = int(g["n"]), int(g["every"]), int(g["steps"])
    mesh, init, info = cases.tgv_periodic(n, u0=float(g["u0"]), tau=float(g["tau"]))
    b = oracle.Block(orc, n)
    b.set_core(init[0])
    ke = []
    for k in range(steps // every + 1):
        if k:
            b.run_periodic_mt(info["omega"], every)
        rho, u = b.fields()
        ke.append(0.5 * float(np.sum(rho * np.sum(u * u, axis=-1))))
    assert np.max(np.abs(np.array(ke) - g["ke"]) / g["ke"]) <= 1e-12
    sl = (slice(2, None, 4),) * 3
    assert np.max(np.abs(u[sl] - g["sample_u"])) <= 1e-12 * np.max(np.abs(g["sample_u"]))
    assert np.max(np.abs(rho[sl] - g["sample_rho"])) <= 1e-12


def test_threaded_restatement_is_the_serial_loop(orc):
    """run_periodic_mt only shares the serial loop's work: bitwise equal."""
    from octlb_b200 import cases
    mesh, init, info = cases.tgv_periodic(20, u0=0.05, tau=0.55)
    a = oracle.Block(orc, 20)
    a.set_core(init[0])
    a.run_periodic(info["omega"], 6)
    b = oracle.Block(orc, 20)
    b.set_core(init[0])
    b.run_periodic_mt(info["omega"], 6, 3)
    assert np.array_equal(a.padded(), b.padded())


def test_physical_mode_restatement_with_one_rate_is_the_reference_loop(ref):
    """The physical coupler mode's restated TimeLoop::advance (per-level
    rates, one LevelCoupler per level pair), given the same rate on every
    level, is the reference TimeLoop bit for bit: the restatement keeps the
    reference's phase order."""
    from octlb_b200 import cases
    mesh, init, info = cases.cavity_forest(cells=16, n=8, lid=0.1, tau=0.6, band_cells=8)
    a = oracle.Sim(ref, mesh, info["omega"], init)
    a.advance(3)
    b = oracle.Sim(ref, mesh, info["omega"], init)
    b.set_physical(np.full(int(mesh.levels.max()) + 1, info["omega"]))
    b.advance(3)
    assert np.array_equal(a.core(), b.core())
