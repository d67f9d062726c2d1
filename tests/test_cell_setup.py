"""Mesh set-up from cells: the library's face table (thx_cell_faces, host)
and the geometric factors computed on the GPU (thx_cell_geometry), the
stand-in for the reference's MFEM cache set-up
(include/dgsem_cache_utilities.hpp:83-215, 470-639).  The device set-up must
give the same tables and factors as the host builders -- bit for bit those
of the Gmsh and MFEM readers' quadrilateral geometry (the same formulas), to
round-off those of the box builder -- and the constants of affine cells."""
import os

import numpy as np
import pytest

import theseus_b200 as T
from theseus_b200.cells import cell_faces, cell_mesh
from theseus_b200.gmsh import quad_mesh_from

HERE = os.path.dirname(os.path.abspath(__file__))


def box_cells(dim, n, lo, hi, periodic=True):
    """Lexicographic cells of a Cartesian box in the box builder's element
    order (x fastest) with periodic vertex ids."""
    n = list(n)
    h = [(hi[d] - lo[d]) / n[d] for d in range(dim)]
    corners, ids = [], []
    idx = np.stack(np.meshgrid(*[np.arange(k) for k in n[::-1]], indexing="ij"), -1).reshape(-1, dim)[:, ::-1]
    for cell in idx:
        cs, vs = [], []
        for v in range(1 << dim):
            off = [(v >> d) & 1 for d in range(dim)]
            cs.append([lo[d] + (cell[d] + off[d]) * h[d] for d in range(dim)])
            g = [(cell[d] + off[d]) % n[d] if periodic else cell[d] + off[d] for d in range(dim)]
            m = [n[d] if periodic else n[d] + 1 for d in range(dim)]
            vs.append(sum(g[d] * int(np.prod(m[:d])) for d in range(dim)))
        corners.append(cs)
        ids.append(vs)
    return np.array(corners), np.array(ids, np.int64)


@pytest.mark.parametrize("dim,n", [(2, (4, 3)), (3, (3, 4, 3))])
def test_face_table_matches_the_box_builder(dim, n):
    m = T.periodic_box(dim, 2, n, [0.0] * dim, [1.0] * dim, coords=False)
    _, ids = box_cells(dim, n, [0.0] * dim, [1.0] * dim)
    fe, fl, be, bl = cell_faces(dim, ids)
    assert len(be) == 0 and len(fe) == m.num_faces
    key = lambda E, L: sorted(map(tuple, np.concatenate([E, L], axis=1).tolist()))
    assert key(fe, fl) == key(m.face_elem, m.face_lface)


def test_face_table_matches_the_gmsh_reader():
    g = np.load(os.path.join(HERE, "golden", "ffs", "ffs_p3_100.npz"))
    nodes = {int(i): tuple(xy) for i, xy in zip(g["node_id"], g["node_xy"])}
    quads = [(0, *map(int, q)) for q in g["quads"]]
    names = [str(x) for x in g["line_names"]]
    lines = [(names[k], int(a), int(b)) for k, a, b in g["lines"]]
    bc = {k: "slip" for k in names}
    m = quad_mesh_from((nodes, quads, lines, {}), 2, bc)
    # the reader's oriented cells, as lexicographic vertex ids
    P = np.array([[nodes[v] for v in q[1:]] for q in quads])
    V = np.array([q[1:] for q in quads], np.int64)
    ids = np.zeros_like(V)
    for e in range(len(P)):
        c = P[e].mean(axis=0)
        o = np.argsort(np.arctan2(P[e, :, 1] - c[1], P[e, :, 0] - c[0]))
        o = np.roll(o, -int(np.argmin(P[e, o, 0] + P[e, o, 1])))
        ids[e] = V[e, o][[0, 1, 3, 2]]
    fe, fl, be, bl = cell_faces(2, ids)
    assert np.array_equal(fe, m.face_elem) and np.array_equal(fl, m.face_lface)
    assert np.array_equal(be, m.boundary.elem) and np.array_equal(bl, m.boundary.lface)


def test_face_table_rejects_misaligned_and_nonmanifold_cells():
    _, ids = box_cells(2, (3, 3), [0.0, 0.0], [1.0, 1.0])
    bad = ids.copy()
    bad[4] = bad[4][[1, 0, 3, 2]]                    # mirrored in x: + face meets + face
    with pytest.raises(T.THXError):
        cell_faces(2, bad)
    three = np.concatenate([ids, ids[:1]])
    with pytest.raises(T.THXError):
        cell_faces(2, three)
    _, two = box_cells(3, (3, 3, 2), [0.0] * 3, [1.0] * 3)   # two cells across a periodic direction
    with pytest.raises(T.THXError):
        cell_faces(3, two)


@pytest.mark.gpu
@pytest.mark.parametrize("dim,n", [(2, (4, 3)), (3, (3, 4, 3))])
def test_device_geometry_of_a_box(cuda, dim, n):
    lo, hi = [-1.0, 0.0, 0.5][:dim], [1.0, 3.0, 2.0][:dim]
    ref = T.periodic_box(dim, 3, n, lo, hi)
    corners, ids = box_cells(dim, n, lo, hi)
    m = cell_mesh(dim, 3, corners, ids)
    for k in ("jac", "metric"):
        np.testing.assert_allclose(getattr(m, k), getattr(ref, k), rtol=1e-15, atol=1e-15, err_msg=k)
    np.testing.assert_allclose(np.asarray(m.coords), np.asarray(ref.coords), rtol=0, atol=4e-15)
    # the same faces (possibly listed in another order) with the same normals and weights
    where = {tuple(r): f for f, r in enumerate(np.concatenate([ref.face_elem, ref.face_lface], 1).tolist())}
    perm = [where[tuple(r)] for r in np.concatenate([m.face_elem, m.face_lface], 1).tolist()]
    for k in ("face_normal", "face_wminus", "face_wplus"):
        np.testing.assert_allclose(getattr(m, k), getattr(ref, k)[perm], rtol=1e-15, atol=1e-15, err_msg=k)


@pytest.mark.gpu
def test_device_geometry_equals_the_gmsh_reader_bit_for_bit(cuda):
    g = np.load(os.path.join(HERE, "golden", "ffs", "ffs_p3_100.npz"))
    nodes = {int(i): tuple(xy) for i, xy in zip(g["node_id"], g["node_xy"])}
    quads = [(0, *map(int, q)) for q in g["quads"]]
    names = [str(x) for x in g["line_names"]]
    lines = [(names[k], int(a), int(b)) for k, a, b in g["lines"]]
    bc = {"left": ("supersonic-inflow", [1.4, 4.2, 0.0, 8.8]), "bottom": "slip", "top": "slip",
          "right": "supersonic-outflow"}
    host = quad_mesh_from((nodes, quads, lines, {}), 3, bc, refinements=1)
    dev = quad_mesh_from((nodes, quads, lines, {}), 3, bc, refinements=1, device="cuda")
    for k in ("jac", "metric", "face_elem", "face_lface", "face_normal", "face_wminus", "face_wplus"):
        assert np.array_equal(getattr(dev, k), getattr(host, k)), k
    assert np.array_equal(np.asarray(dev.coords), np.asarray(host.coords))
    hb, db = host.boundary, dev.boundary
    for k in ("elem", "lface", "normal", "weight", "bc"):
        assert np.array_equal(getattr(db, k), getattr(hb, k)), k


@pytest.mark.gpu
def test_device_geometry_of_affine_trilinear_cells(cuda):
    """Cells of x = A xi + s: constant J = det(A) h^3 and metric = adj(A h)."""
    A = np.array([[1.0, 0.25, 0.0], [0.0, 0.75, 0.125], [0.5, 0.0, 1.5]])
    corners, ids = box_cells(3, (3, 3, 3), [0.0] * 3, [1.0] * 3)
    corners = corners @ A.T + np.array([0.1, -0.2, 0.3])
    m = cell_mesh(3, 2, corners, ids, coords=False)
    h = 1.0 / 3.0
    J = np.linalg.det(A) * h ** 3
    adj = np.linalg.inv(A * h) * np.linalg.det(A * h)
    np.testing.assert_allclose(m.jac, J, rtol=1e-13)
    np.testing.assert_allclose(m.metric, np.broadcast_to(adj, m.metric.shape), rtol=1e-12, atol=1e-15)
    # each face's normal is the minus cell's adjugate row of the face direction
    d = m.face_lface[:, 0] // 2
    np.testing.assert_allclose(m.face_normal, np.broadcast_to(adj[d][:, None, :], m.face_normal.shape),
                               rtol=1e-12, atol=1e-15)
