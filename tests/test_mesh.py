"""Lattice meshes in the reference's per-rank file layout (multiphaselb_b200.mesh):
write -> read round trips, fscanf-style parsing, the single-domain check, and
the non-box channel-with-cylinder geometry.  Host code only."""
import os

import numpy as np
import pytest

from multiphaselb_b200 import abi, cases, mesh


def same_mesh(a, b):
    assert a.lattice == b.lattice and a.nlocal == b.nlocal and a.nghosts == b.nghosts
    assert np.array_equal(a.points, b.points) and np.array_equal(a.nb, b.nb)
    assert a.patch_names == b.patch_names
    assert all(np.array_equal(p, q) for p, q in zip(a.patches, b.patches)) and len(a.patches) == len(b.patches)


@pytest.mark.parametrize("lattice,dims,per", [(abi.D2Q9, (12, 10), (True, False)),
                                              (abi.D3Q15, (5, 4, 6), (False, True, False))])
def test_box_round_trip(tmp_path, lattice, dims, per):
    nb, points, patches, names = cases.box_mesh(lattice, dims, per)
    m = mesh.LatticeMesh(lattice, points, nb, names, patches, len(nb))
    mesh.write_lattice_mesh(m, str(tmp_path), pid=2)
    got = mesh.read_lattice_mesh(str(tmp_path), pid=2)
    same_mesh(got, m)
    assert got.recv_ghosts and len(got.recv_ghosts[0]) == 0


def test_file_layout_and_whitespace(tmp_path):
    """The files hold what writeLatticeMesh prints; the reader, like fscanf,
    does not care how the whitespace falls."""
    m = mesh.channel_with_cylinder(10, 8, 4.5, 3.5, 1.6)
    mesh.write_lattice_mesh(m, str(tmp_path))
    d = tmp_path / "processor0" / "lattice"
    head = (d / "neighbours").read_text().splitlines()[0]
    assert head == f"{m.nlocal} 2 9"
    b = (d / "boundary").read_text().splitlines()
    assert b[0] == "3" and b[1] == "" and b[2] == "bottom" and b[3] == str(len(m.patches[0]))
    (d / "neighbours").write_text((d / "neighbours").read_text().replace("\n", "   \n\t"))
    same_mesh(mesh.read_lattice_mesh(str(tmp_path)), m)


def test_cylinder_geometry():
    nx, ny, cx, cy, r = 24, 16, 11.5, 6.5, 3.5
    m = mesh.channel_with_cylinder(nx, ny, cx, cy, r)
    pts = m.points
    inside = (pts[:, 0] - cx) ** 2 + (pts[:, 1] - cy) ** 2 < r * r
    assert not inside.any() and m.nlocal == nx * ny - int(np.sum(
        (np.arange(nx)[None, :] - cx) ** 2 + (np.arange(ny)[:, None] - cy) ** 2 < r * r))
    # every pull source is the node at x - c_k (x wraps), or -1 where that is solid or off the walls
    index = {(x, y): i for i, (x, y, _) in enumerate(pts.tolist())}
    for i, (x, y, _) in enumerate(pts.tolist()):
        for k, c in enumerate(cases.VEL[abi.D2Q9]):
            want = index.get(((x - c[0]) % nx, y - c[1]), -1)
            assert m.nb[i, k] == want
    cyl = set(m.patches[2].tolist())
    for i, (x, y, _) in enumerate(pts.tolist()):
        wall = y in (0, ny - 1)
        assert (i in cyl) == (not wall and bool((m.nb[i] == -1).any()))


def test_mesh_case_refuses_ghosts(tmp_path):
    m = mesh.channel_with_cylinder(10, 8, 4.5, 3.5, 1.6)
    m.nghosts = 2
    m.points = np.vstack([m.points, np.zeros((2, 3), dtype=np.int32)])
    with pytest.raises(ValueError):
        mesh.mesh_case(m, "x", {}, None, None, np.zeros(m.nlocal), np.zeros((m.nlocal, 3)), np.zeros(m.nlocal))


def test_cylinder_case_runs_through_the_file_format(tmp_path):
    """The cylinder test case written to files and read back is the same case."""
    from tests.helpers import small_cases
    c = small_cases()["cylinder_d2q9"]
    m = mesh.LatticeMesh(c.lattice, c.points, c.nb, c.patch_names, c.patches, c.n)
    mesh.write_lattice_mesh(m, str(tmp_path))
    back = mesh.read_lattice_mesh(str(tmp_path))
    c2 = mesh.mesh_case(back, c.name, c.eos, c.f, c.g, c.rho, c.U, c.T)
    assert np.array_equal(c2.nb, c.nb) and c2.dims == c.dims
    assert os.path.exists(tmp_path / "processor0" / "lattice" / "vtkCells")
