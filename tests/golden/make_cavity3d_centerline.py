"""The reference's cavity3d accuracy gate data, read from its example source:

  examples/cavity3d/cavity3d_case.h   kGhiaRe100_YOverH (the 17 sample heights
                                      y / H on the centerline x = z = L / 2),
                                      kOpenLbCavity3d_UOverLid (OpenLB's u / u_lid
                                      there after kOpenLbCavity3dConvergedSteps),
                                      kOpenLbCavity3dConvergedSteps
  src/solver/lbm/unit_converter/unit_converter.cpp
                                      OpenLbCavity3dDefaults (resolution, tau,
                                      L, U, nu, rho)

tests/integration/test_cavity3d_serial.cpp:56-82 runs the example to the
converged step count and requires the relative L2 of the sampled profile
against the OpenLB values to stay below 0.02.  The file also holds the
profile of the reference's own TimeLoop in FP64 (oracle/_ref: BlockLattice,
ConcreteDomainBoundaryHandler, ConstRhoBGK with the boundary cells in the
statistics, one 31^3 block at halo 1) after the same steps, sampled the same
way (octlb_b200.cases.cavity3d_centerline), with its L2.  Saved as
cavity3d_centerline.json; the tests and bench.py read that file.

  python tests/golden/make_cavity3d_centerline.py [reference root]   (about a minute)
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def array(text, name):
    m = re.search(name + r"\s*=\s*\{([^}]*)\}", text)
    if not m:
        raise SystemExit(f"{name} not found")
    return [float(v) for v in m.group(1).replace("\n", " ").split(",") if v.strip()]


def main():
    root = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    case = open(os.path.join(root, "examples", "cavity3d", "cavity3d_case.h")).read()
    conv = open(os.path.join(root, "src", "solver", "lbm", "unit_converter", "unit_converter.cpp")).read()
    steps = int(re.search(r"kOpenLbCavity3dConvergedSteps\s*=\s*(\d+)", case).group(1))
    m = re.search(r"OpenLbCavity3dDefaults\(\)\s*\{\s*return UnitConverter\(([^;]*)\);", conv, re.S)
    args = [float(re.sub(r"/\*.*?\*/", "", a).strip()) for a in m.group(1).split(",")]
    resolution, tau, length, velocity, nu, rho = args
    out = {
        "source": "examples/cavity3d/cavity3d_case.h, src/solver/lbm/unit_converter/unit_converter.cpp",
        "gate": "relative L2 of u / u_lid against openlb_u_over_lid < 0.02 "
                "(tests/integration/test_cavity3d_serial.cpp:56-82)",
        "steps": steps,
        "resolution": int(resolution),
        "tau": tau,
        "phys_length": length,
        "phys_velocity": velocity,
        "phys_viscosity": nu,
        "phys_density": rho,
        "y_over_h": array(case, "kGhiaRe100_YOverH"),
        "openlb_u_over_lid": array(case, "kOpenLbCavity3d_UOverLid"),
    }
    assert len(out["y_over_h"]) == len(out["openlb_u_over_lid"]) == 17
    # the reference's TimeLoop in FP64 on the same case
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from octlb_b200 import cases
    from oracle import oracle
    ref = oracle.load("ref")
    mesh, init, info = cases.cavity3d(out["resolution"], out["tau"], length, velocity, nu)
    sim = oracle.Sim(ref, mesh, info["omega"], init)
    sim.set_fd_boundary([oracle.Sim.INTERPOLATED_VELOCITY] * 6, info["u_wall"], const_rho=True)
    sim.advance(steps)
    _, u = oracle.rho_u(sim.core())
    prof = cases.cavity3d_centerline(u[0][..., 0], info, out["y_over_h"])
    out["reference_fp64_u_over_lid"] = [float(v) for v in prof]
    out["reference_fp64_l2"] = cases.relative_l2(prof, out["openlb_u_over_lid"])
    out["reference_fp64_average_rho"] = float(sim.average_rho())
    with open(os.path.join(HERE, "cavity3d_centerline.json"), "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")
    print(json.dumps(out)[:300])


if __name__ == "__main__":
    main()
