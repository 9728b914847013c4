"""Host mesh layer (include/cfsa_mesh.h) against the oracle's std::map-based restatement of
src/Mesh/Mesh.cpp: face order, P2 edge numbering, boundary tags and geometry must be identical."""
import sys
from pathlib import Path

import numpy as np
import pytest

GOLD = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLD))


def compare_with_oracle(cf, po, m, direction=(1.0, 0.0, 0.0), coverage=1.0):
    m.setupBoundaryConditions(direction, coverage)
    o = po.Oracle(m.vertices(), m.tets(), direction=direction, coverage=coverage)
    om = o.mesh()
    p1, p2 = m.fluidBC()
    fv, ft, fg = m.faces()
    vol, gr = m.tetGeometry()
    assert np.array_equal(m.tetEdges(), om["tet_edges"])
    assert np.array_equal(p1, om["p1"])
    assert np.array_equal(p2, om["p2"])
    assert np.array_equal(fv, om["face_verts"])
    assert np.array_equal(ft, om["face_tets"])
    assert np.array_equal(fg, om["face_geom"])
    assert np.array_equal(vol, om["vol"])
    assert np.array_equal(gr, om["grads"])
    assert np.array_equal(m.edgeNodes(), om["edge_xyz"])
    return p1, p2


@pytest.mark.parametrize("rings,layers", [(1, 1), (2, 4), (3, 9), (5, 68)])
def test_cylinder_matches_oracle(cf, po, rings, layers):
    m = cf.Mesh.cylinder(30.0, 2.0, rings, layers)
    p1, p2 = compare_with_oracle(cf, po, m)
    assert (p1 == cf.FluidBCType.Inlet).sum() > 0 and (p1 == cf.FluidBCType.Outlet).sum() > 0


def test_structured_prism_matches_oracle(cf, po):
    m = cf.Mesh.structuredRectangularPrism(4.0, 1.0, 1.0, 8, 2, 3)
    compare_with_oracle(cf, po, m)


def test_shuffled_mesh_matches_oracle(cf, po):
    """Random vertex relabelling and tet order exercise the ordering rules (face order by sorted
    triple, first-encounter edge ids, last-write-wins tagging)."""
    base = cf.Mesh.cylinder(10.0, 1.0, 3, 6)
    xyz, tets = base.vertices(), base.tets()
    rng = np.random.default_rng(20261203)
    perm = rng.permutation(len(xyz))
    inv = np.empty_like(perm)
    inv[perm] = np.arange(len(perm))
    xyz2 = xyz[perm]
    tets2 = inv[tets][rng.permutation(len(tets))]
    m = cf.Mesh.fromArrays(xyz2, tets2)
    compare_with_oracle(cf, po, m, direction=(-1.0, 0.0, 0.0), coverage=2.0)


def test_generator_matches_independent_construction(cf):
    import gen_golden

    xyz, tets = gen_golden.cylinder_points(30.0, 2.0, 2, 4)
    m = cf.Mesh.cylinder(30.0, 2.0, 2, 4)
    np.testing.assert_allclose(m.vertices(), xyz, rtol=0, atol=1e-15)
    assert np.array_equal(m.tets(), tets)


def test_cylinder_is_conforming_and_positive(cf):
    m = cf.Mesh.cylinder(30.0, 2.0, 4, 20)
    nv, nt, ne, nf, nb = m.sizes
    vol, _ = m.tetGeometry()
    assert vol.min() > 0
    assert abs(vol.sum() - np.pi * 4 * 30) / (np.pi * 4 * 30) < 0.05  # polygonal disk
    # Euler characteristic of a solid ball: V - E + F - T = 1
    assert nv - ne + nf - nt == 1
    # boundary faces: 2 caps of 6*rings^2 triangles + 2 per lateral quad
    assert nb == 2 * 6 * 16 + 2 * (6 * 4) * 20
    fv, ft, _ = m.faces()
    assert np.all(ft[:, 0] >= 0)


def test_msh_round_trip(cf, tmp_path):
    m = cf.Mesh.cylinder(5.0, 1.0, 3, 5)
    path = tmp_path / "cyl.msh"
    m.writeMshFile(path)
    m2 = cf.Mesh.fromMshFile(path)
    assert np.array_equal(m.vertices(), m2.vertices())
    assert np.array_equal(m.tets(), m2.tets())
    assert np.array_equal(m.tetEdges(), m2.tetEdges())
    text = path.read_text().splitlines()
    assert text[0] == "$MeshFormat" and text[1].startswith("4.1")


def test_msh_reader_skips_other_element_types(cf, tmp_path):
    path = tmp_path / "mixed.msh"
    path.write_text(
        "$MeshFormat\n4.1 0 8\n$EndMeshFormat\n$Nodes\n1 4 10 13\n3 1 0 4\n10\n11\n12\n13\n"
        "0 0 0\n1 0 0\n0 1 0\n0 0 1\n$EndNodes\n$Elements\n2 2 1 2\n2 1 2 1\n1 10 11 12\n"
        "3 1 4 1\n2 10 11 12 13\n$EndElements\n")
    m = cf.Mesh.fromMshFile(path)
    assert m.sizes[:2] == (4, 1)
    assert np.array_equal(m.tets(), [[0, 1, 2, 3]])


def test_errors_are_reported(cf, tmp_path):
    with pytest.raises(cf.CfsaError):
        cf.Mesh.fromMshFile(tmp_path / "missing.msh")
    with pytest.raises(cf.CfsaError):
        cf.Mesh.fromArrays(np.zeros((4, 3)), [[0, 1, 2, 7]])
    with pytest.raises(cf.CfsaError):  # degenerate tet
        cf.Mesh.fromArrays(np.zeros((4, 3)), [[0, 1, 2, 3]])
    bad = tmp_path / "bad.msh"
    bad.write_text("$Nodes\n1 1 1 1\n3 1 0 1\n1\n0 0 0\n$EndNodes\n$Elements\n1 1 1 1\n3 1 4 1\n1 1 2 3 4\n$EndElements\n")
    with pytest.raises(cf.CfsaError):
        cf.Mesh.fromMshFile(bad)


def test_y_bifurcation_mesher(cf):
    """Procedural Y-bifurcation: positive tets, inlet tags on the x = 0 cap only, outlet tags at
    both daughter ends, wall elsewhere, P2 tags derived from P1 (Mesh.hpp:198-215 rule)."""
    import numpy as np

    m = cf.Mesh.yBifurcation(cell=0.3)
    nv, nt, ne, nf, nb = m.sizes
    assert nt > 50000 and nb > 0
    vol, _ = m.tetGeometry()
    assert vol.min() > 0.0
    x = m.vertices()
    p1, p2 = m.fluidBC()
    assert set(np.unique(p1)) == {0, 1, 2, 3}
    assert np.all(x[p1 == 1, 0] == 0.0)
    ang = np.deg2rad(35.0)
    for sg in (1.0, -1.0):
        end = np.array([15.0 + 12.0 * np.cos(ang), sg * 12.0 * np.sin(ang), 0.0])
        d = np.array([np.cos(ang), sg * np.sin(ang), 0.0])
        o = x[(p1 == 2) & (sg * x[:, 1] > 0)]
        assert len(o) > 20
        assert np.all(np.abs((o - end) @ d) <= 1.5 * 0.3 + 1e-12)
    # P2 rule: an edge node gets its endpoints' tag when both share the same non-internal tag
    edges_ok = np.isin(p2, [0, 1, 2, 3])
    assert edges_ok.all() and (p2 == 1).sum() > 0 and (p2 == 2).sum() > 0
