"""The reference's cavity3d accuracy gate (tests/integration/
test_cavity3d_serial.cpp:56-82) on the example's own case: one 31^3 block
(RESOLUTION = 30), tau = 0.509, lid velocity 0.1, InterpolatedVelocity on
every face, ConstRhoBGK with the boundary cells in the statistics, run to
the converged 5,269 steps.  The centerline u / u_lid, sampled as the example
samples it, must lie within relative L2 0.02 of OpenLB's values
(tests/golden/cavity3d_centerline.json, read from the example's source by
tests/golden/make_cavity3d_centerline.py).

* CPU: the reference's own TimeLoop (oracle/_ref, FP64) through the restated
  sampling reproduces the fixture's FP64 profile and passes the gate
  (L2 3.5e-3).
* GPU: FP32 and FP16-shifted through the C ABI pass the gate, and their
  profiles lie within 2e-5 (FP32) and 5e-3 (FP16) of u_lid of the FP64 one.
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
GATE = 0.02


def fixture():
    with open(os.path.join(HERE, "golden", "cavity3d_centerline.json")) as f:
        return json.load(f)


def case(g):
    from octlb_b200 import cases
    return cases.cavity3d(g["resolution"], g["tau"], g["phys_length"], g["phys_velocity"], g["phys_viscosity"])


def test_reference_timeloop_passes_the_gate(ref):
    from octlb_b200 import cases
    g = fixture()
    mesh, init, info = case(g)
    assert abs(info["u_lid"] - 0.1) < 1e-12 and mesh.n == 31
    sim = oracle.Sim(ref, mesh, info["omega"], init)
    sim.set_fd_boundary([oracle.Sim.INTERPOLATED_VELOCITY] * 6, info["u_wall"], const_rho=True)
    sim.advance(g["steps"])
    _, u = oracle.rho_u(sim.core())
    prof = cases.cavity3d_centerline(u[0][..., 0], info, g["y_over_h"])
    l2 = cases.relative_l2(prof, g["openlb_u_over_lid"])
    print(f"cavity3d reference FP64: L2 vs OpenLB {l2:.3e}")
    assert np.max(np.abs(prof - np.array(g["reference_fp64_u_over_lid"]))) <= 1e-12
    assert l2 < GATE


@pytest.mark.gpu
@pytest.mark.parametrize("prec,tol", [("fp32", 2e-5), ("fp16", 5e-3)])
def test_gpu_passes_the_gate(ob, prec, tol):
    from octlb_b200 import cases
    g = fixture()
    mesh, init, info = case(g)
    lat = ob.GpuLattice(ob.stamp_fd_kinds(mesh, info["types"]), info["omega"],
                        precision=ob.FP32 if prec == "fp32" else ob.FP16_SHIFTED, init_pops=init)
    lat.set_const_rho(True)
    lat.set_fd_boundary(info["types"], info["u_wall"])
    lat.advance(g["steps"])
    _, u = lat.get_fields()
    avg = lat.average_rho()
    lat.close()
    prof = cases.cavity3d_centerline(u[0][..., 0], info, g["y_over_h"])
    l2 = cases.relative_l2(prof, g["openlb_u_over_lid"])
    dev = float(np.max(np.abs(prof - np.array(g["reference_fp64_u_over_lid"]))))
    print(f"cavity3d {prec}: L2 vs OpenLB {l2:.3e} (FP64 reference {g['reference_fp64_l2']:.3e}), "
          f"profile vs FP64 {dev:.2e}, average_rho {avg:.9f} ({g['reference_fp64_average_rho']:.9f})")
    assert l2 < GATE
    assert dev <= tol
