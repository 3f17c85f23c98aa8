"""Partitions against the reference's own partitioner.

oracle/_ref/latticeMeshPartition is the reference's latticeMeshPartition
application built from its sources (oracle/Makefile, target `partition`;
kmetis left out).  It reads a mesh in the reference's lattice/ layout and
writes processor<pid>/lattice/*; slabs.partition with the standard
decomposition must give every rank the same local numbering, neighbours,
points, ghost lists and boundary lists."""
import os
import subprocess

import numpy as np
import pytest

from multiphaselb_b200 import abi, mesh, slabs
from oracle import oracle as orc
from tests.helpers import small_cases

HERE = os.path.dirname(os.path.abspath(__file__))
PARTITIONER = os.path.join(HERE, "..", "oracle", "_ref", "latticeMeshPartition")


def partitioner():
    if not os.path.exists(PARTITIONER):
        if not orc.ref_tree_present():
            pytest.skip("reference partitioner not built and the reference tree is absent")
        orc.make("ref", "partition")
    return PARTITIONER


def write_case_mesh(case, root, ranks):
    """The undecomposed mesh as readBasicMesh reads it (lattice/points,
    neighbours, vtkCells, boundary) and the dictionaries the partitioner
    reads (lattice model, method and process count, and the time settings
    its mesh writer looks up)."""
    os.makedirs(os.path.join(root, "lattice"), exist_ok=True)
    os.makedirs(os.path.join(root, "properties"), exist_ok=True)
    pts = np.asarray(case.points, dtype=np.int64)
    with open(os.path.join(root, "lattice", "points"), "w") as fp:
        fp.write(f"{case.n}\n")
        fp.writelines(f"{x} {y} {z}\n" for x, y, z in pts.tolist())
    with open(os.path.join(root, "lattice", "neighbours"), "w") as fp:
        fp.writelines(" ".join(str(v) for v in row) + "\n" for row in np.asarray(case.nb).tolist())
    with open(os.path.join(root, "lattice", "vtkCells"), "w") as fp:
        fp.write(f"0 {4 if case.lattice == abi.D2Q9 else 8}\n")
    with open(os.path.join(root, "lattice", "boundary"), "w") as fp:
        fp.write(f"{len(case.patches)}\n\n")
        for name, p in zip(case.patch_names, case.patches):
            fp.write(f"{name}\n{len(p)}\n")
            fp.writelines(f"{v}\n" for v in np.asarray(p).tolist())
            fp.write("\n")
    with open(os.path.join(root, "properties", "latticeProperties"), "w") as fp:
        fp.write(f"LBModel {'D2Q9' if case.lattice == abi.D2Q9 else 'D3Q15'};\n")
    with open(os.path.join(root, "properties", "parallel"), "w") as fp:
        fp.write(f"method standard;\n\nnumProc {ranks};\n")
    with open(os.path.join(root, "properties", "simulation"), "w") as fp:
        fp.write("startTime 0;\nendTime 1;\nwriteInterval 1;\n")


# The walled D3Q15 boxes (four patches, fed with no vtkCells) are not here:
# the reference partitioner ends with SIGSEGV on them at every process
# count, one included; the cause lies in the reference and is not pursued.
@pytest.mark.parametrize("name,ranks", [("bubble_d2q9", 3), ("lid_d2q9", 2), ("column_d2q9", 4),
                                        ("bubble_d3q15", 3), ("outflow_d3q15", 5), ("cylinder_d2q9", 3),
                                        ("cylinder_d2q9", 7)])
def test_standard_partition_equals_reference_partitioner(tmp_path, name, ranks):
    exe = partitioner()
    case = small_cases()[name]
    root = str(tmp_path)
    write_case_mesh(case, root, ranks)
    p = subprocess.run([exe], cwd=root, capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    parts = slabs.partition(case, slabs.standard_owner(case.n, ranks))
    assert len(parts) == ranks
    for part in parts:
        m = mesh.read_lattice_mesh(root, pid=part.rank)
        nloc = len(part.own)
        assert (m.nlocal, m.nghosts) == (nloc, len(part.gidx) - nloc), part.rank
        assert np.array_equal(np.asarray(m.points), np.asarray(part.case.points)), part.rank
        assert np.array_equal(np.asarray(m.nb), np.asarray(part.case.nb)[:nloc]), part.rank
        for s in range(ranks):
            got_r = np.asarray(m.recv_ghosts[s]) if s < len(m.recv_ghosts) else np.zeros(0)
            got_s = np.asarray(m.send_ghosts[s]) if s < len(m.send_ghosts) else np.zeros(0)
            assert np.array_equal(got_r, part.recv[s]), (part.rank, s, "recv")
            assert np.array_equal(got_s, part.send[s]), (part.rank, s, "send")
        assert list(m.patch_names) == list(part.case.patch_names)
        for a, b in zip(m.patches, part.case.patches):
            assert np.array_equal(np.asarray(a), np.asarray(b)), part.rank
