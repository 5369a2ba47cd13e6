"""The files around the step: the VTK image data of pmlib_output_mesh (checked
byte for byte against a .pvti the reference wrote, and field by field for the
.vti), the topology summary, and the particle restart file (Fortran unformatted
records).  Host code only: these tests run without a GPU."""
import os
import struct

import numpy as np

from pmlib3d_b200 import pmlib as P

HERE = os.path.dirname(os.path.abspath(__file__))


def test_pvti_matches_reference_file(tmp_path):
    patch = P.make_patch((-0.6875, -1.1875, -1.1875), (0.6875, 1.1875, 1.1875), (1 / 64,) * 3)
    patch.ncell[0], patch.ncell[1], patch.ncell[2] = 88, 152, 152
    icell = [(1, 1, 1), (1, 77, 1), (1, 1, 77), (1, 77, 77)]
    ncell = [(88, 76, 76)] * 4
    out = tmp_path / "out.pvti"
    assert P.output_pvti(str(out), "out", patch, icell, ncell) == 0
    assert out.read_bytes() == open(os.path.join(HERE, "golden", "poisson_out.pvti"), "rb").read()


def test_vti_fields(tmp_path):
    patch = P.make_patch((-1, -0.5, -0.75), (1, 0.5, 0.75), (0.125,) * 3, nghost=4)
    ierr, topo = P.pmlib_topology_cuboid(patch, 3)
    rng = np.random.default_rng(3)
    vort = rng.standard_normal(P.topo_shape(topo))
    vel = rng.standard_normal(P.topo_shape(topo))
    assert P.pmlib_output_mesh(str(tmp_path) + "/", "m", patch, topo, vort, vel) == 0
    data = (tmp_path / "m_P00000.vti").read_bytes()
    assert data.startswith(b'<?xml version="1.0"?><VTKFile type="ImageData" version="0.1" byte_order="LittleEndian">')
    head, raw = data.split(b'<AppendedData encoding="raw">_', 1)
    assert b'Name="vel" NumberOfComponents="3" format="appended" offset="' in head
    nx, ny, nz = topo.ncell
    nb = 3 * nx * ny * nz * 4
    g = [topo.nghost[0], topo.nghost[2], topo.nghost[4]]
    inner = lambda a: a[g[2]:g[2] + nz, g[1]:g[1] + ny, g[0]:g[0] + nx, :].astype(np.float32).ravel()
    assert struct.unpack("<i", raw[:4])[0] == nb
    assert np.array_equal(np.frombuffer(raw[4:4 + nb], "<f4"), inner(vort))
    assert struct.unpack("<i", raw[4 + nb:8 + nb])[0] == nb
    assert np.array_equal(np.frombuffer(raw[8 + nb:8 + 2 * nb], "<f4"), inner(vel))
    assert raw[8 + 2 * nb:] == b"</AppendedData></VTKFile>"
    # the second array's offset is the first one's bytes plus its 4-byte length
    assert f'offset="{nb + 4:10d}"'.encode() in head
    pv = (tmp_path / "m.pvti").read_text()
    assert f'WholeExtent="{0:8d}{nx:8d}{0:8d}{ny:8d}{0:8d}{nz:8d}"' in pv and 'Source="m_P00000.vti"' in pv


def test_topology_file(tmp_path):
    patch = P.make_patch((-1, -1, -0.5), (1, 1, 0.5), (0.125, 0.125, 0.0625), bound_cond=(1, 1, 0), nghost=4)
    ierr, topo = P.pmlib_topology_cuboid(patch, 3)
    tag = str(tmp_path / "topo")
    assert P.pmlib_output_topology(tag, patch, topo) == 0
    lines = open(tag + ".dat").read().splitlines()
    assert lines[4] == "# Patch type:              1"
    assert lines[5] == "# Minimum extend:            -1.00   -1.00   -0.50"
    assert lines[7] == "# Resolution:                1/   8"
    assert lines[8] == "# Number of mesh cells:         16      16      16"
    assert "#  Boundary conditions:       1   1   1   1   0   0" in lines
    assert "#  Neighbours:                0   0   0   0  -1  -1" in lines


def test_particle_restart_roundtrip(tmp_path):
    rng = np.random.default_rng(5)
    pos = rng.standard_normal((500, 3))
    vort = rng.standard_normal((500, 3)) * np.linspace(0, 2, 500)[:, None]
    tag = str(tmp_path / "part")
    assert P.output_particles(tag, 11, 0.25, pos, vort) == 0
    raw = open(tag + ".dat", "rb").read()
    # records: [4] itime [4], [8] time [8], [4] npart [4], then 500 x [48] (pos, vort) [48]
    assert struct.unpack("<iii", raw[:12]) == (4, 11, 4)
    assert struct.unpack("<idi", raw[12:28]) == (8, 0.25, 8)
    assert struct.unpack("<iii", raw[28:40]) == (4, 500, 4)
    assert len(raw) == 40 + 500 * 56
    rec = np.frombuffer(raw[40:], dtype=np.dtype([("a", "<i4"), ("v", "<f8", 6), ("b", "<i4")]))
    assert np.all(rec["a"] == 48) and np.all(rec["b"] == 48)
    assert np.array_equal(rec["v"][:, :3], pos) and np.array_equal(rec["v"][:, 3:], vort)
    trunc = 1.0
    ierr, p2, w2, it, tm = P.input_particles(tag + ".dat", trunc)
    keep = np.sqrt((vort ** 2).sum(1)) >= trunc
    assert ierr == 0 and it == 11 and tm == 0.25
    assert np.array_equal(p2, pos[keep]) and np.array_equal(w2, vort[keep])
    assert P.input_particles(tag + ".dat", 1e9)[0] == -1  # nothing above the truncation
