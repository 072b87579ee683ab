"""Host-side checks (CPU only): the forest flattener's topology, the C ABI's
exported symbols and table validation, and the index helpers the kernels use."""
import ctypes
import itertools
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in ("octlb_gpu.h", "octlb_forest.h"):
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"\b(octlb_[a-z_0-9]+)\s*\(", src):
            names.add(m.group(1))
    return sorted(names)


def test_library_exports_every_declared_symbol(ob):
    L = ob.capi.lib()
    syms = declared_symbols()
    assert len(syms) >= 25
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing


def test_fastdiv_matches_integer_division(ob):
    L = ob.capi.lib()
    rng = np.random.default_rng(0)
    for d in [1, 2, 3, 7, 8, 10, 34, 64, 100, 488, 512, 1000, 4096, 5832, 16777216, 2 ** 31 - 1]:
        vals = list(rng.integers(0, 2 ** 32, 200)) + [0, 1, d - 1, d, d + 1, 2 ** 32 - 1]
        for v in vals:
            v = int(v) % (2 ** 32)
            assert L.octlb_gpu_debug_fastdiv(d, v) == v // d, (d, v)


def face_neighbors_bruteforce(levels, bounds, domain, periodic):
    """All (a, d, b) with leaf b touching face d of leaf a (positive area)."""
    out = []
    ext = np.array(domain[3:]) - np.array(domain[:3])
    for a in range(len(levels)):
        for d in range(6):
            ax, hi = d // 2, d & 1
            plane = bounds[a][3 + ax] if hi else bounds[a][ax]
            for b in range(len(levels)):
                if a == b and not periodic[ax]:
                    continue
                other = bounds[b][ax] if hi else bounds[b][3 + ax]
                shift = 0.0
                if abs(other - plane) > 1e-12:
                    if periodic[ax] and abs(abs(other - plane) - ext[ax]) < 1e-12:
                        shift = 1
                    else:
                        continue
                ok = True
                for t in range(3):
                    if t == ax:
                        continue
                    lo = max(bounds[a][t], bounds[b][t])
                    up = min(bounds[a][3 + t], bounds[b][3 + t])
                    if up - lo <= 1e-12:
                        ok = False
                if ok:
                    out.append((a, d, b))
    return out


@pytest.mark.parametrize("periodic", [(0, 0, 0), (0, 0, 1)])
def test_forest_faces_match_geometry(ob, periodic):
    dom = (0, 0, 0, 2, 1, 1)
    f = ob.Forest((2, 1, 1), periodic, dom).refine_uniform(1)
    f.refine_box((0.4, 0.4, 0.1, 0.6, 0.6, 0.3), 3).balance().build()
    lv, bd = f.levels, f.bounds
    # 2:1 balance across faces and leaves tile the domain
    vol = np.prod(bd[:, 3:] - bd[:, :3], axis=1).sum()
    assert abs(vol - 2.0) < 1e-12
    nb = face_neighbors_bruteforce(lv, bd, dom, periodic)
    for a, d, b in nb:
        assert abs(int(lv[a]) - int(lv[b])) <= 1
    same = {(a, d, b) for a, d, b in nb if lv[a] == lv[b]}
    assert set(map(tuple, f.same_level.tolist())) == same
    # every coarse-fine face: coarse side listed once per face, 4 fine leaves
    # one level finer touching that face, in Morton (id) order
    cf_expected = {}
    for a, d, b in nb:
        if lv[b] == lv[a] + 1:
            cf_expected.setdefault((a, d), []).append(b)
    got = {(int(r[0]), int(r[5])): list(r[1:5]) for r in f.coarse_fine}
    assert set(got) == set(cf_expected)
    for k, fines in got.items():
        assert sorted(cf_expected[k]) == fines
        assert fines == sorted(fines)
    assert np.all(np.diff(f.coarse_fine[:, 6]) >= 0)  # grouped by coarse level
    # tree-boundary faces are exactly the faces on the non-periodic domain boundary
    tb = {(int(a), int(d)) for a, d in f.tree_boundary}
    exp = set()
    for a in range(len(lv)):
        for d in range(6):
            ax = d // 2
            on = abs(bd[a][3 + ax] - dom[3 + ax]) < 1e-12 if d & 1 else abs(bd[a][ax] - dom[ax]) < 1e-12
            if on and not periodic[ax]:
                exp.add((a, d))
    assert tb == exp


def test_forest_uniform_has_only_same_level_faces(ob):
    """test_face_pair_list.cpp: uniform refinement -> no hanging faces; one
    root -> six tree-boundary faces and no same-level face on them."""
    f = ob.Forest().refine_uniform(2).balance().build()
    assert len(f.coarse_fine) == 0 and len(f.same_level) == 64 * 6 - 6 * 16
    g = ob.Forest().build()
    assert len(g.tree_boundary) == 6 and len(g.same_level) == 0
    assert sorted(int(d) for d in g.tree_boundary[:, 1]) == list(range(6))


def test_forest_center_refine_six_hanging_faces(ob):
    """One level-2 octant refined to level 3 inside a uniform level-2 forest:
    its six faces hang, each with four fine leaves."""
    f = ob.Forest().refine_uniform(2).refine_box((0.25, 0.25, 0.25, 0.5, 0.5, 0.5), 3).balance().build()
    assert len(f.coarse_fine) == 6
    for r in f.coarse_fine:
        assert len(set(r[1:5].tolist())) == 4 and r[6] == 2 and r[7] == 3


def make_tables_mesh(ob, **kw):
    n = 4
    return ob.Mesh(n, [0], [0, 0, 0, 1, 1, 1], **kw)


def test_create_rejects_bad_tables_without_device(ob):
    """Validation happens before any CUDA call, so these run on the CPU."""
    bad = [
        dict(kinds=np.full((1, 4, 4, 4), 9, np.uint8)),                       # BcKind out of range
        dict(same_level=np.array([[0, 7, 0]])),                               # dir out of range
        dict(link_cells=np.array([[0, 9, 0, 0, 1]]), link_q=np.array([0.5])),  # cell out of range
    ]
    for kw in bad:
        with pytest.raises(ob.OctlbError) as e:
            ob.GpuLattice(make_tables_mesh(ob, **kw), 1.5, stream_mode=ob.STREAM_LINKS)
        assert e.value.code == ob.capi.OCTLB_EINVAL
    with pytest.raises(ob.OctlbError):
        ob.GpuLattice(make_tables_mesh(ob), 2.5)                              # omega outside (0, 2)
    with pytest.raises(ob.OctlbError):
        ob.GpuLattice(ob.Mesh(1, [0], [0, 0, 0, 1, 1, 1]), 1.5)               # block edge below 2
    from octlb_b200 import cases
    odd_cf, _, _ = cases.cavity_forest(cells=6, n=3, band_cells=3)
    with pytest.raises(ob.OctlbError) as e:                                     # odd block edge with 2:1
        ob.GpuLattice(odd_cf, 1.5)                                              # coupling
    assert e.value.code == ob.capi.OCTLB_EINVAL and "coarse-fine" in str(e.value)
    # parameters out of their sets (the ABI's enumerations)
    for kw in (dict(precision=7), dict(stream_mode=5), dict(coupler_mode=3), dict(stream_order=2),
               dict(coupler_mode=ob.COUPLER_PHYSICAL, omega_level=[2.5]),
               dict(stream_order=ob.ORDER_AA),                                  # AA needs a periodic box
               dict(stream_order=ob.ORDER_AA, drag=True)):
        with pytest.raises(ob.OctlbError) as e:
            ob.GpuLattice(make_tables_mesh(ob), 1.5, **kw)
        assert e.value.code == ob.capi.OCTLB_EINVAL, kw
    with pytest.raises(ob.OctlbError) as e:
        ob.GpuLattice(make_tables_mesh(ob, periodic=1), 1.5, stream_order=ob.ORDER_AA, drag=True)
    assert e.value.code == ob.capi.OCTLB_EINVAL


def test_lattice_updates_per_coarse_step(ob):
    from octlb_b200 import cases
    mesh, _, _ = cases.cavity_forest(cells=32, n=8, band_cells=8)
    # TimeLoop recursion from level 0: a level-l leaf is stepped 2^l times
    exp = sum((8 ** 3) << int(l) for l in mesh.levels)
    assert mesh.lattice_updates_per_coarse_step() == exp


def test_cpp_adapter_compiles_links_and_reports_errors(ob, tmp_path):
    """include/octlb_gpu_time_loop.hpp (TimeLoop method names over the C ABI)
    compiles against the library; invalid tables raise std::runtime_error
    before any device work."""
    import subprocess
    src = tmp_path / "adapter.cpp"
    src.write_text(r'''
#include "octlb_gpu_time_loop.hpp"
#include <cstdio>
// the whole adapter surface compiles and links
double use(octlb::GpuTimeLoop& loop) {
  loop.advance_one();
  loop.write_vtk("out", "case", 1);
  return loop.average_rho() + loop.total_mass() + loop.force_on_fluid()[0] + loop.counters().collide.size();
}
// cavity3d's construction: ConstRhoBGK and the domain handler's face specs
void cavity(const octlb_tables& t, const octlb_params& p) {
  octlb::GpuDomainBc bc;
  for (int f = 0; f < 6; ++f) bc.types[f] = OCTLB_FD_VELOCITY;
  bc.u_wall[3 * 3] = 0.1;
  octlb::GpuTimeLoop cav(t, p, nullptr, true, &bc);
  cav.advance(5269);
}
int main() {
  octlb_tables t{};
  octlb_params p{};
  t.n = 1;  // block edge below 2: rejected by validation
  t.n_blocks = 1;
  int lv = 0; double bd[6] = {0,0,0,1,1,1}; unsigned char k[1] = {0};
  t.levels = &lv; t.bounds = bd; t.kinds = k;
  p.omega = 1.5;
  try {
    octlb::GpuTimeLoop loop(t, p);
    return 2;
  } catch (const std::runtime_error& e) {
    std::printf("%s\n", e.what());
  }
  try {  // face specs on invalid tables: refused before any device work
    octlb::GpuDomainBc bc;
    octlb::GpuTimeLoop loop(t, p, nullptr, false, &bc);
    return 3;
  } catch (const std::runtime_error& e) {
    std::printf("%s\n", e.what());
    return 0;
  }
}
''')
    exe = tmp_path / "adapter"
    lib_dir = os.path.join(ROOT, "octlb_b200")
    subprocess.run(["g++", "-std=c++17", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                    "-L", lib_dir, "-loctlb_b200", f"-Wl,-rpath,{lib_dir}"], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0 and ">= 2" in r.stdout


@pytest.mark.parametrize("name", ["tgv", "shell", "c1", "c2", "cyl", "c3"])
def test_plan_dry_run_all_configurations(ob, name):
    """octlb_gpu_plan flattens every benchmark configuration on the host with
    all kernel-derived indices bounds-checked, no device needed."""
    from octlb_b200 import cases
    cfg = {
        "tgv": (lambda: cases.tgv_periodic(32), ob.STREAM_ROTATE, False),
        "shell": (lambda: cases.cavity_shell(16), ob.STREAM_LINKS, False),
        "c1": (lambda: cases.cavity_forest(cells=32, n=8), ob.STREAM_ROTATE, False),
        "c2": (lambda: cases.cavity_forest(cells=64, n=8, lid=0.05, tau=0.56, band_cells=8), ob.STREAM_ROTATE, False),
        "cyl": (lambda: cases.cylinder_forest(length=128, height=32, n=8, diameter=8.0, center=(32.0, 16.0),
                                              levels=2, u_max=0.05, re=40.0), ob.STREAM_LINKS, True),
        "c3": (lambda: cases.cylinder_forest(), ob.STREAM_LINKS, True),
    }[name]
    mesh, init, info = cfg[0]()
    pl = ob.plan(mesh, info["omega"], stream_mode=cfg[1], drag=cfg[2])
    assert sum(d["blocks"] for d in pl) == mesh.n_blocks
    for l, d in enumerate(pl):
        if d["blocks"]:
            assert d["slots"] >= d["blocks"] * mesh.n ** 3
    if name in ("c2", "c3", "cyl"):
        assert sum(d["prolong"] for d in pl) > 0 and sum(d["restrict"] for d in pl) > 0
    if name in ("c3", "cyl"):
        assert sum(d["drag"] for d in pl) > 0 and sum(d["links"] for d in pl) > 0


@pytest.mark.parametrize("name", ["amr_cavity", "cylinder"])
def test_coupler_items_are_the_reference_plan(ob, ref, name):
    """The Lagrava plan (level_coupler.cpp:70-118, tested by the reference in
    test_lagrava_coupler.cpp:126-192): every coupling point's indices lie
    inside its blocks, the pairs are unique, and the GPU's prolongation /
    restriction items are exactly the plan's distinct fine / coarse targets
    per level (a later point writing the same cell wins)."""
    from octlb_b200 import cases
    from oracle import oracle
    if name == "amr_cavity":
        mesh, init, info = cases.cavity_forest(cells=32, n=8, lid=0.1, tau=0.6, band_cells=8)
        mode = ob.STREAM_ROTATE
    else:
        mesh, init, info = cases.cylinder_forest(length=128, height=32, n=8, diameter=8.0, center=(32.0, 16.0),
                                                 levels=2)
        mode = ob.STREAM_LINKS
    sim = oracle.Sim(ref, mesh, info["omega"], init, link_mode=mode == ob.STREAM_LINKS)
    plan = sim.plan()
    n = mesh.n
    assert len(plan) > 0
    assert np.all((plan[:, [1, 2, 3, 5, 6, 7]] >= 0) & (plan[:, [1, 2, 3, 5, 6, 7]] < n))
    assert np.all(mesh.levels[plan[:, 0]] == plan[:, 8]) and np.all(mesh.levels[plan[:, 4]] == plan[:, 9])
    assert np.all(plan[:, 9] == plan[:, 8] + 1)
    assert len({tuple(r) for r in plan[:, :8]}) == len(plan)
    stats = ob.plan(mesh, info["omega"], stream_mode=mode)
    for l, st in enumerate(stats):
        fine_targets = {tuple(r) for r in plan[plan[:, 8] == l][:, 4:8]}
        coarse_targets = {tuple(r) for r in plan[plan[:, 9] == l][:, 0:4]}
        assert st["prolong"] == len(fine_targets), (l, st, len(fine_targets))
        assert st["restrict"] == len(coarse_targets), (l, st, len(coarse_targets))
