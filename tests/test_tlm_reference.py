"""The tangent-linear FP64 reference (the reference's own TimeLoop on
forward-mode dual numbers, oracle/ref_tlm.cpp) and the finite-difference
goldens pin each other: exact derivatives of the discrete map against central
differences of the plain reference build (tests/golden/make_tlm_reference.py,
make_adjoint_reference.py)."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from make_adjoint_reference import case, directions  # noqa: E402


def golden(name):
    path = os.path.join(HERE, "golden", name)
    if not os.path.exists(path):
        pytest.skip(f"{name} not generated")
    return np.load(path)


@pytest.mark.parametrize("tlm_name,fd_name", [("adjoint_c5_short_tlm.npz", "adjoint_c5_short.npz"),
                                              ("adjoint_c5_tlm.npz", "adjoint_c5.npz")])
def test_tlm_goldens_agree_with_finite_differences(tlm_name, fd_name):
    """Same objective value; u_max and tau derivatives within the central
    differences' O(h^2) truncation (h = 1e-4 relative).  The body-force
    differences are taken over a 1e-6 perturbation, so their rounding floor is
    absolute (~1e-10 on the 1,000-call horizon, 4e-5 relative for its smallest
    component): the bound is relative to the largest component."""
    t, f = golden(tlm_name), golden(fd_name)
    assert int(t["steps"]) == int(f["steps"]) and int(t["window"]) == int(f["window"])
    assert abs(t["J"] - f["J"]) <= 1e-12 * abs(f["J"])
    assert abs(t["dJ_du"] - f["dJ_du"]) <= 1e-6 * abs(f["dJ_du"])
    assert abs(t["dJ_dtau"] - f["dJ_dtau"]) <= 1e-5 * abs(f["dJ_dtau"])
    assert np.all(np.abs(t["dJ_dir"] - f["dJ_dir"]) <= 1e-5 * np.max(np.abs(f["dJ_dir"])))


def test_tlm_library_matches_central_differences(ref, tlm):
    """A short run of the tangent-linear library against central differences
    of the plain reference computed here: u_max, tau and one body-force
    direction (4 advance_one calls, objective over the last 2)."""
    from oracle import oracle
    steps, window, u0 = 4, 2, 0.05
    mesh, init, info = case(u0)
    tau = info["tau"]
    d0 = directions(mesh)[0]

    def J(u=u0, t=tau, sign=0.0):
        m, i, inf = case(u, t)
        s = oracle.Sim(ref, m, inf["omega"], i, link_mode=True)
        if sign:
            s.set_body_force(sign * d0)
        acc = 0.0
        for k in range(steps):
            s.advance(1)
            if k >= steps - window:
                acc += s.drag(m.obstacle)[0]
        return acc / window

    nd = tlm.tlm_dirs()
    om = 1.0 / tau
    om_seed, wall_seed = np.zeros(nd), np.zeros(nd)
    om_seed[1], wall_seed[0] = -om * om, 1.0 / u0
    dirs = np.zeros((nd,) + d0.shape)
    dirs[2] = d0
    s = oracle.Sim(tlm, mesh, om, init, link_mode=True, omega_seed=om_seed, wall_seed=wall_seed)
    s.set_body_force_tlm(None, dirs)
    Jt, dJ = 0.0, np.zeros(nd)
    for k in range(steps):
        s.advance(1)
        if k >= steps - window:
            f, df = s.drag_tlm(mesh.obstacle)
            Jt += f[0]
            dJ += df[0]
    Jt, dJ = Jt / window, dJ / window
    J0 = J()
    assert abs(Jt - J0) <= 1e-13 * abs(J0)  # the value part is the reference's own trajectory
    hu, ht = 1e-4 * u0, 1e-4 * tau
    fd_u = (J(u=u0 + hu) - J(u=u0 - hu)) / (2 * hu)
    fd_t = (J(t=tau + ht) - J(t=tau - ht)) / (2 * ht)
    fd_d = (J(sign=1.0) - J(sign=-1.0)) / 2.0
    assert abs(dJ[0] - fd_u) <= 1e-6 * abs(fd_u), (dJ[0], fd_u)
    assert abs(dJ[1] - fd_t) <= 1e-5 * abs(fd_t), (dJ[1], fd_t)
    assert abs(dJ[2] - fd_d) <= 1e-5 * abs(fd_d), (dJ[2], fd_d)
