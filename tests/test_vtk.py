"""VTK output (src/solver/io/vtk_writer/): the library's .vts / .vtm / .pvd
files against the reference's own writer (compiled into oracle/_ref), byte
for byte for the same values, and the fields octlb_gpu_write_vtk writes
against octlb_gpu_get_fields."""
import base64
import ctypes
import os
import re
import struct
import subprocess

import numpy as np
import pytest

REF_VTK = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "ref_vtk")


@pytest.fixture(scope="module")
def ref_vtk():
    """The reference's writer as a program (oracle/_ref/ref_vtk, built with
    `make -C oracle ref REF=<reference tree>`)."""
    if not os.path.exists(REF_VTK):
        pytest.skip("oracle/_ref/ref_vtk not built")
    return REF_VTK


def ref_write_block(tool, path, bounds, fields):
    """The reference's WriteStructuredGridVts with the same (name, values
    [nx][ny][nz](, c)) fields as octlb_b200.vtk_write_block."""
    shape = np.asarray(fields[0][1]).shape[:3]
    blob = [struct.pack("<4i", *shape, len(fields)), np.asarray(bounds, "<f8").tobytes()]
    for name, v in fields:
        v = np.asarray(v, np.float64)
        c = 1 if v.ndim == 3 else v.shape[3]
        blob += [struct.pack("<i", len(name)), name.encode(), struct.pack("<i", c),
                 np.ascontiguousarray(np.transpose(v.reshape(shape + (c,)), (2, 1, 0, 3)), "<f8").tobytes()]
    inp = str(path) + ".in"
    with open(inp, "wb") as f:
        f.write(b"".join(blob))
    subprocess.run([tool, "block", str(path), inp], check=True)


def read_vts(path):
    """{name: values} of a .vts written by either writer (Float64 arrays,
    base64 of a UInt32 byte count + the values), "Points" included."""
    text = open(path).read()
    out = {}
    for m in re.finditer(r'<DataArray type="Float64"(?: Name="([^"]*)")? NumberOfComponents="(\d)" '
                         r'format="binary" encoding="base64">\n\s*([A-Za-z0-9+/=]+)\n', text):
        raw = base64.b64decode(m.group(3))
        nbytes = struct.unpack("<I", raw[:4])[0]
        assert nbytes == len(raw) - 4
        out[m.group(1) or "Points"] = np.frombuffer(raw[4:], "<f8").reshape(-1, int(m.group(2)))
    return out


def test_vts_bytes_equal_reference(ob, ref_vtk, tmp_path):
    rng = np.random.default_rng(1)
    for shape, bounds in (((4, 5, 6), (0.25, -1.0, 3.0, 1.5, 2.0, 3.75)), ((8, 8, 8), (0, 0, 0, 1, 1, 1)),
                          ((1, 1, 1), (0.1, 0.2, 0.3, 0.7, 0.9, 1.3))):
        fields = [("velocity", rng.standard_normal(shape + (3,)) * 0.05),
                  ("density", 1 + 0.01 * rng.standard_normal(shape)),
                  ("pressure", (1 + 0.01 * rng.standard_normal(shape)) / 3)]
        ob.vtk_write_block(tmp_path / "ours.vts", bounds, fields)
        ref_write_block(ref_vtk, tmp_path / "ref.vts", bounds, fields)
        assert (tmp_path / "ours.vts").read_bytes() == (tmp_path / "ref.vts").read_bytes(), shape
        got = read_vts(tmp_path / "ours.vts")
        for name, v in fields:
            v = np.asarray(v)
            c = 1 if v.ndim == 3 else v.shape[3]
            expect = np.transpose(v.reshape(shape + (c,)), (2, 1, 0, 3)).reshape(-1, c)
            assert np.array_equal(got[name], expect)
        # the reference's own decoder reads our payload back bit for bit
        payload = re.search(r'Name="density"[^>]*>\n\s*([A-Za-z0-9+/=]+)\n', open(tmp_path / "ours.vts").read())
        (tmp_path / "payload").write_text(payload.group(1))
        out = subprocess.run([ref_vtk, "decode", str(tmp_path / "payload")], check=True, capture_output=True, text=True)
        assert np.array_equal(np.array([float(x) for x in out.stdout.split()]), got["density"][:, 0])


def test_vtm_pvd_bytes_equal_reference(ob, ref_vtk, tmp_path):
    for step, files in ((0, ["c_r0_oct0_T00000.vts", "c_r0_oct1_T00000.vts"]),
                        (25, ["c_r0_oct0_T00025.vts", "c_r0_oct1_T00025.vts", "c_r0_oct2_T00025.vts"])):
        ob.vtk_write_index(tmp_path / "ours", "c", step, files)
        subprocess.run([ref_vtk, "index", str(tmp_path / "ref"), "c", str(step)] + files, check=True)
        tag = f"{step:05d}"
        assert (tmp_path / "ours" / f"c_T{tag}.vtm").read_bytes() == (tmp_path / "ref" / f"c_T{tag}.vtm").read_bytes()
        assert (tmp_path / "ours" / "c.pvd").read_bytes() == (tmp_path / "ref" / "c.pvd").read_bytes()
    assert open(tmp_path / "ours" / "c.pvd").read().count("<DataSet timestep=") == 2


def test_vtk_argument_checks(ob, tmp_path):
    with pytest.raises(ob.OctlbError):
        ob.vtk_write_block(tmp_path / "x.vts", (0, 0, 0, 1, 1, 1), [("v", np.zeros((2, 2, 2, 4)))])  # 4 components
    L = ob.capi.lib()
    b = np.zeros(6)
    assert L.octlb_vtk_write_block(str(tmp_path / "y.vts").encode(), 0, 2, 2, ob.capi.ptr(b, ctypes.c_double), 0,
                                   None, None, None) != 0                                   # nx = 0
    (tmp_path / "bad.pvd").write_text("not a series")
    with pytest.raises(ob.OctlbError):
        ob.vtk_write_index(tmp_path, "bad", 0, ["a.vts"])


@pytest.mark.gpu
def test_write_vtk_matches_fields_and_reference_writer(ob, ref_vtk, tmp_path):
    """octlb_gpu_write_vtk on a two-level cavity forest: one file per block
    with AmrVtkWriter's names, the values of get_fields (pressure = rho / 3),
    the bytes of the reference's writer fed with those values, the index."""
    from octlb_b200 import cases
    mesh, init, info = cases.cavity_forest(cells=32, n=8, lid=0.1, tau=0.6, band_cells=8)
    lat = ob.GpuLattice(mesh, info["omega"], init_pops=init)
    lat.advance(3)
    lat.write_vtk(tmp_path / "out", "cav", 3, fields=("velocity", "density", "pressure"))
    rho, u = lat.get_fields()
    lat.close()
    n = mesh.n
    for b in range(mesh.n_blocks):
        f = tmp_path / "out" / f"cav_r0_oct{b}_T00003.vts"
        got = read_vts(f)
        order = lambda v: np.transpose(v.reshape(n, n, n, -1), (2, 1, 0, 3)).reshape(-1, v.size // n ** 3)
        assert np.array_equal(got["velocity"], order(u[b]))
        assert np.array_equal(got["density"], order(rho[b]))
        assert np.array_equal(got["pressure"], order(rho[b] * (1.0 / 3.0)))
        if b in (0, mesh.n_blocks - 1):
            ref_write_block(ref_vtk, tmp_path / "ref.vts", mesh.bounds[b],
                            [("velocity", u[b]), ("density", rho[b]), ("pressure", rho[b] * (1.0 / 3.0))])
            assert f.read_bytes() == (tmp_path / "ref.vts").read_bytes()
    vtm = open(tmp_path / "out" / "cav_T00003.vtm").read()
    assert vtm.count("<Block index=") == mesh.n_blocks
    assert 'file="cav_r0_oct0_T00003.vts"' in vtm
    assert 'timestep="3"' in open(tmp_path / "out" / "cav.pvd").read()
