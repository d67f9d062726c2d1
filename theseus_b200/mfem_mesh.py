"""MFEM native meshes ("MFEM mesh v1.0") of quadrilaterals -> the library's
geometry.

Stands in for the part of the reference's mesh set-up used by its 2-D MFEM
mesh cases (src/Simulation.cpp:314-356: mfem::Mesh(file), ser_ref_levels
uniform refinements): the topology of the elements and boundary sections,
vertex coordinates either from the vertices section or from a first-order
nodal grid function (the periodic meshes of the reference's test cases carry
an L2_T1_2D_P1 "nodes" function, one coordinate set per element), and uniform
refinement that splits every quadrilateral into four with the nodes
transferred as MFEM transfers a P1 grid function: a child's vertex is the
parent's bilinear interpolant at that point, summed over the parent's four
degrees of freedom in their lexicographic order with the weights 1, 1/2 or
1/4.  Straight-sided, axis-structured quadrilaterals only (the geometry is
built by theseus_b200.gmsh.quad_cells_mesh).  Boundary elements keep their
attribute; `boundary` maps an attribute to a condition.
"""
import numpy as np

from .gmsh import quad_cells_mesh


def _tokens(path):
    lines = []
    with open(path) as f:
        for line in f:
            s = line.split("#", 1)[0].strip()
            if s:
                lines.append(s)
    return lines


def read_mfem_mesh(path):
    """(dim, elements [(attr, geom, vertex ids)], boundary [(attr, geom,
    vertex ids)], number of vertices, corner coordinates per element (ne, 4, 2)
    in lexicographic degree-of-freedom order (0,0), (1,0), (0,1), (1,1))."""
    L = _tokens(path)
    if not L or not L[0].startswith("MFEM mesh v1."):
        raise ValueError("not an MFEM mesh v1.x file")
    i = 1
    dim = elems = bdr = nv = None
    vcoords = dof_coords = None
    while i < len(L):
        key = L[i]
        if key == "dimension":
            dim = int(L[i + 1]); i += 2
        elif key == "elements":
            n = int(L[i + 1])
            elems = [tuple(int(t) for t in L[i + 2 + k].split()) for k in range(n)]
            i += 2 + n
        elif key == "boundary":
            n = int(L[i + 1])
            bdr = [tuple(int(t) for t in L[i + 2 + k].split()) for k in range(n)]
            i += 2 + n
        elif key == "vertices":
            nv = int(L[i + 1]); i += 2
            if i < len(L) and L[i] != "nodes":
                sdim = int(L[i])
                vcoords = np.array([[float(t) for t in L[i + 1 + k].split()[:sdim]] for k in range(nv)])
                i += 1 + nv
        elif key == "nodes":
            fields = {}
            i += 1
            if L[i] != "FiniteElementSpace":
                raise ValueError("nodes: FiniteElementSpace expected")
            i += 1
            while ":" in L[i]:
                k, v = L[i].split(":", 1)
                fields[k.strip()] = v.strip()
                i += 1
            fec, vdim = fields["FiniteElementCollection"], int(fields["VDim"])
            if not (fec.startswith("L2_T") and fec.endswith("_2D_P1")) or vdim != 2:
                raise NotImplementedError(f"nodes in {fec} (VDim {vdim}): only L2 first-order 2-D nodes")
            ne = len(elems)
            vals = np.array([float(t) for s in L[i:i + 4 * ne * (1 if fields.get("Ordering", "0") == "1" else 2)]
                             for t in s.split()])
            if fields.get("Ordering", "0") == "1":   # byVDIM: per dof, x y
                dof_coords = vals[:8 * ne].reshape(ne, 4, 2)
            else:                                     # byNODES: all x, then all y
                dof_coords = np.stack([vals[:4 * ne], vals[4 * ne:8 * ne]], axis=1).reshape(2, ne, 4)
                dof_coords = np.moveaxis(dof_coords, 0, 2)
            i = len(L)
        else:
            raise ValueError(f"unexpected section '{key}'")
    if dim != 2 or any(e[1] != 3 for e in elems):
        raise NotImplementedError("2-D quadrilateral meshes only")
    ids = np.array([e[2:6] for e in elems], np.int64)
    if dof_coords is None:
        if vcoords is None:
            raise ValueError("no vertex coordinates")
        # vertex order v0 v1 v2 v3 (counter-clockwise) -> lexicographic dofs
        dof_coords = vcoords[ids[:, [0, 1, 3, 2]], :2]
    return dim, elems, bdr or [], nv, np.asarray(dof_coords, dtype=np.float64)


def refine(elems, bdr, nv, dofs):
    """One uniform refinement (mfem::Mesh::UniformRefinement of quadrilaterals
    with the nodes transferred by the P1 refinement operator).  Returns the
    same four items for the refined mesh; children of element e are 4e..4e+3."""
    edge_id = {}

    def mid(a, b):
        nonlocal nv
        k = (min(a, b), max(a, b))
        if k not in edge_id:
            edge_id[k] = nv
            nv += 1
        return edge_id[k]

    new_e, new_d = [], []
    for e, (attr, geom, v0, v1, v2, v3) in enumerate(elems):
        d = dofs[e]                                   # (0,0) (1,0) (0,1) (1,1)
        half = lambda p, q: 0.5 * d[p] + 0.5 * d[q]
        P = {(0, 0): d[0], (2, 0): d[1], (0, 2): d[2], (2, 2): d[3],
             (1, 0): half(0, 1), (1, 2): half(2, 3), (0, 1): half(0, 2), (2, 1): half(1, 3),
             (1, 1): ((0.25 * d[0] + 0.25 * d[1]) + 0.25 * d[2]) + 0.25 * d[3]}
        c = nv
        nv += 1
        V = {(0, 0): v0, (2, 0): v1, (2, 2): v2, (0, 2): v3, (1, 1): c,
             (1, 0): mid(v0, v1), (2, 1): mid(v1, v2), (1, 2): mid(v2, v3), (0, 1): mid(v3, v0)}
        for j in range(2):
            for i in range(2):
                new_e.append((attr, geom, V[(i, j)], V[(i + 1, j)], V[(i + 1, j + 1)], V[(i, j + 1)]))
                new_d.append([P[(i, j)], P[(i + 1, j)], P[(i, j + 1)], P[(i + 1, j + 1)]])
    new_b = []
    for attr, geom, a, b in bdr:
        m = edge_id[(min(a, b), max(a, b))]
        new_b += [(attr, geom, a, m), (attr, geom, m, b)]
    return new_e, new_b, nv, np.array(new_d)


def mfem_quad_mesh(path, order, refinements=0, boundary=None, coords=True, device=None):
    """Geometry of an MFEM quadrilateral mesh after `refinements` uniform
    refinements (the reference's ser_ref_levels), at polynomial order
    `order`.  boundary maps a boundary attribute to a condition (as in box());
    `device` computes the geometric factors on that GPU."""
    return mfem_quad_mesh_from(read_mfem_mesh(path), order, refinements, boundary, coords, device)


def mfem_quad_mesh_from(parsed, order, refinements=0, boundary=None, coords=True, device=None):
    """mfem_quad_mesh from read_mfem_mesh's result."""
    _, elems, bdr, nv, dofs = parsed
    for _ in range(refinements):
        elems, bdr, nv, dofs = refine(elems, bdr, nv, dofs)
    corners = dofs[:, [0, 1, 3, 2]]                  # lexicographic -> cyclic
    vids = np.array([e[2:6] for e in elems], np.int64)
    blines = {(min(a, b), max(a, b)): str(attr) for attr, _, a, b in bdr}
    if boundary is not None:
        boundary = {str(k): v for k, v in boundary.items()}
    return quad_cells_mesh(corners, vids, order, blines, boundary, coords, device=device)
