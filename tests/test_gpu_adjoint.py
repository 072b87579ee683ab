"""Hand-written adjoint (octlb_gpu_adjoint) against FP64 central finite
differences of the reference's own TimeLoop (oracle/_ref), stored by
tests/golden/make_adjoint_reference.py:

* adjoint_c5_short.npz  24 advance_one calls, objective over the last 12;
* adjoint_c5.npz        the adjoint configuration: channel 128x32x32, two
                        levels, D = 8, Re = 40, 1,000 advance_one calls (4
                        finest steps each: 4,000 finest steps), drag averaged
                        over the last 250 calls (1,000 finest steps),
                        checkpoints every 16 calls (64 finest steps).

and against the exact derivatives of the same discrete FP64 map from the
tangent-linear reference (the reference's TimeLoop on forward-mode dual
numbers, tests/golden/make_tlm_reference.py): adjoint_c5_short_tlm.npz,
adjoint_c5_tlm.npz.

Gradients: inlet u_max, tau, and the per-cell body force along 8 seeded
N(0, 1e-6) directions.  Tolerance: 1e-4 relative.  The adjoint is wrapped in
a torch.autograd.Function here, in the test harness only.
"""
import os
import time

import numpy as np
import pytest

from octlb_b200.cases import adjoint_channel as case, adjoint_directions as directions  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))

pytestmark = pytest.mark.gpu
TOL = 1e-4


def lattice(ob, force=None):
    mesh, init, info = case()
    lat = ob.GpuLattice(mesh, info["omega"], precision=ob.FP32, stream_mode=ob.STREAM_LINKS, drag=True,
                        init_pops=init)
    if force is not None:
        lat.set_body_force(force)
    return mesh, lat


def check(ob, name, checkpoint):
    g = np.load(os.path.join(HERE, "golden", name))
    steps, window = int(g["steps"]), int(g["window"])
    mesh, lat = lattice(ob)
    J, du, dtau, gF = lat.adjoint(steps, window, checkpoint)
    lat.close()
    d = directions(mesh)
    gdir = np.array([np.sum(gF * d[k]) for k in range(len(d))])
    assert abs(J - g["J"]) <= 1e-4 * abs(g["J"])
    assert abs(du - g["dJ_du"]) <= TOL * abs(g["dJ_du"]), (du, float(g["dJ_du"]))
    assert abs(dtau - g["dJ_dtau"]) <= TOL * abs(g["dJ_dtau"]), (dtau, float(g["dJ_dtau"]))
    err = np.abs(gdir - g["dJ_dir"]) / np.abs(g["dJ_dir"])
    assert np.all(err <= TOL), err
    tname = os.path.join(HERE, "golden", name.replace(".npz", "_tlm.npz"))
    if os.path.exists(tname):  # the tangent-linear FP64 reference
        t = np.load(tname)
        assert int(t["steps"]) == steps and int(t["window"]) == window
        assert abs(du - t["dJ_du"]) <= TOL * abs(t["dJ_du"]), (du, float(t["dJ_du"]))
        assert abs(dtau - t["dJ_dtau"]) <= TOL * abs(t["dJ_dtau"]), (dtau, float(t["dJ_dtau"]))
        terr = np.abs(gdir - t["dJ_dir"]) / np.abs(t["dJ_dir"])
        assert np.all(terr <= TOL), terr
    return steps, window


def test_adjoint_short_horizon_matches_fp64_fd(ob):
    check(ob, "adjoint_c5_short.npz", 5)


def test_adjoint_checkpointing_does_not_change_the_gradient(ob):
    """Checkpoint spacing only trades memory for recomputation (results agree
    to the FP32 rounding of the adjoint's atomic accumulation order)."""
    mesh, init, info = case()
    out = []
    for k in (1, 7, 24):
        _, lat = lattice(ob)
        J, du, dtau, gF = lat.adjoint(24, 12, k)
        lat.close()
        out.append((J, du, dtau, gF))
    for J, du, dtau, gF in out[1:]:
        assert J == out[0][0]
        assert abs(du - out[0][1]) <= 1e-6 * abs(out[0][1])
        assert abs(dtau - out[0][2]) <= 1e-6 * abs(out[0][2])
        assert np.max(np.abs(gF - out[0][3])) <= 1e-5 * np.max(np.abs(out[0][3]))


def test_adjoint_leaves_the_forward_state(ob):
    """After the adjoint the context holds the forward's final state, as
    after advance(n), and the force accumulators of the forward."""
    _, a = lattice(ob)
    _, b = lattice(ob)
    a.adjoint(10, 4, 3, force_grad=False)
    b.advance(6)
    b.force_reset()
    b.advance(4)
    assert np.array_equal(a.get_populations(), b.get_populations())
    assert np.array_equal(a.force(), b.force())
    sa, sb = a.force_sum(), b.force_sum()
    assert np.array_equal(sa[0], sb[0]) and sa[1] == sb[1]


def test_body_force_zero_is_the_plain_forward(ob):
    mesh, a = lattice(ob)
    _, b = lattice(ob, np.zeros((mesh.n_blocks, mesh.n ** 3, 3)))
    a.advance(5)
    b.advance(5)
    assert np.array_equal(a.get_populations(), b.get_populations())


def test_adjoint_c5_matches_fp64_fd_and_cost(ob):
    """The full adjoint configuration against FP64 finite differences and the
    tangent-linear reference; then its cost: (forward + adjoint sweep) of the
    1,000 calls against the forward alone, both in steady state (the forward
    after a warm-up call, the sweep after a first call that captured its
    graphs; each the best of three timings), must stay within the north
    star's 3x."""
    check(ob, "adjoint_c5.npz", 16)
    g = np.load(os.path.join(HERE, "golden", "adjoint_c5.npz"))
    steps, window = int(g["steps"]), int(g["window"])
    _, lat = lattice(ob)
    lat.advance(3)  # warm-up (graph capture)
    lat.synchronize()
    t_fwd = float("inf")
    for _ in range(3):
        t0 = time.perf_counter()
        lat.advance(steps)
        lat.synchronize()
        t_fwd = min(t_fwd, time.perf_counter() - t0)
    lat.close()
    _, lat = lattice(ob)
    lat.adjoint(steps, window, 16)
    lat.synchronize()
    t_all = float("inf")
    for _ in range(3):
        t0 = time.perf_counter()
        lat.adjoint(steps, window, 16)
        lat.synchronize()
        t_all = min(t_all, time.perf_counter() - t0)
    lat.close()
    ratio = (t_all - t_fwd) / t_fwd
    print(f"adjoint cost: forward {t_fwd:.3f} s, forward + adjoint {t_all:.3f} s, adjoint / forward {ratio:.2f}")
    assert ratio <= 3.0, ratio


def test_torch_autograd_wrapper(ob):
    """torch.autograd.Function over the adjoint, the test harness's wrapper:
    backward of J(u_max, tau, F) returns the adjoint gradients."""
    torch = pytest.importorskip("torch")

    class AveragedDrag(torch.autograd.Function):
        @staticmethod
        def forward(ctx, u_max, tau, force):
            mesh, init, info = case(float(u_max), float(tau))
            lat = ob.GpuLattice(mesh, 1.0 / float(tau), precision=ob.FP32, stream_mode=ob.STREAM_LINKS, drag=True,
                                init_pops=init)
            lat.set_body_force(force.detach().cpu().numpy())
            J, du, dtau, gF = lat.adjoint(24, 12, 5)
            lat.close()
            ctx.save_for_backward(torch.tensor(du), torch.tensor(dtau), torch.from_numpy(gF))
            return torch.tensor(J, dtype=torch.float64)

        @staticmethod
        def backward(ctx, gJ):
            du, dtau, gF = ctx.saved_tensors
            return gJ * du, gJ * dtau, gJ * gF

    mesh, _, info = case()
    u = torch.tensor(0.05, dtype=torch.float64, requires_grad=True)
    tau = torch.tensor(info["tau"], dtype=torch.float64, requires_grad=True)
    F = torch.zeros((mesh.n_blocks, mesh.n ** 3, 3), dtype=torch.float64, requires_grad=True)
    J = AveragedDrag.apply(u, tau, F)
    J.backward()
    g = np.load(os.path.join(HERE, "golden", "adjoint_c5_short.npz"))
    assert abs(u.grad.item() - g["dJ_du"]) <= TOL * abs(g["dJ_du"])
    assert abs(tau.grad.item() - g["dJ_dtau"]) <= TOL * abs(g["dJ_dtau"])
    d = directions(mesh)
    assert abs(float((F.grad.numpy() * d[0]).sum()) - g["dJ_dir"][0]) <= TOL * abs(g["dJ_dir"][0])
