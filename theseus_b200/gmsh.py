"""Gmsh (format 2.2, ASCII) quadrilateral meshes -> the library's geometry.

Stands in for the part of MFEM's mesh set-up the reference uses for its
2-D Gmsh cases (src/Simulation.cpp mesh loading, include/
dgsem_cache_utilities.hpp:83-215, 355-440, 516-639): straight-sided
quadrilaterals with the bilinear map of their four vertices, geometric
factors at the LGL nodes, conforming faces (aligned by orienting every
element along the global axes), periodic identification from the file's
$Periodic section, and boundary faces named by the physical groups of the
boundary lines.  Structured (axis-aligned, rectangular-topology) meshes
only: each element must have a unique lower-left vertex and neighbours
across every face, which is what transfinite Gmsh meshes give, with at least
three elements across a periodic direction (faces are matched by their
identified vertex pairs).  A periodic
face takes its normal from its minus element's edge; where the file's two
periodic edges do not coincide to the last digit, the reference (MFEM) may
take it from either side.
"""
import numpy as np


def _sections(path):
    out, name, buf = {}, None, []
    with open(path) as f:
        for line in f:
            s = line.strip()
            if s.startswith("$End"):
                out[name] = buf
                name, buf = None, []
            elif s.startswith("$"):
                name, buf = s[1:], []
            elif name is not None:
                buf.append(s)
    return out


def read_gmsh(path):
    """Nodes {id: (x, y)}, quads [(tag, v0..v3)], boundary lines
    [(physical name, a, b)], periodic node map {slave: master}."""
    sec = _sections(path)
    if not sec["MeshFormat"][0].startswith("2.2"):
        raise ValueError("Gmsh format 2.2 ASCII expected")
    names = {}
    for s in sec.get("PhysicalNames", [])[1:]:
        dim, tag, name = s.split(maxsplit=2)
        names[(int(dim), int(tag))] = name.strip('"')
    nodes = {}
    for s in sec["Nodes"][1:]:
        t = s.split()
        nodes[int(t[0])] = (float(t[1]), float(t[2]))
    quads, lines = [], []
    for s in sec["Elements"][1:]:
        t = [int(x) for x in s.split()]
        etype, ntags = t[1], t[2]
        phys = t[3] if ntags > 0 else 0
        v = t[3 + ntags:]
        if etype == 3:
            quads.append((phys, *v[:4]))
        elif etype == 1:
            lines.append((names.get((1, phys), str(phys)), v[0], v[1]))
    periodic = {}
    p = sec.get("Periodic", [])
    i = 1 if p else 0
    for _ in range(int(p[0]) if p else 0):
        i += 1                                   # entity line
        if p[i].startswith("Affine"):
            i += 1
        n = int(p[i]); i += 1
        for k in range(n):
            a, b = (int(x) for x in p[i + k].split())
            periodic[a] = b
        i += n
    return nodes, quads, lines, periodic


def quad_mesh(path, order, boundary=None, coords=True, refinements=0, device=None):
    """Geometry of a Gmsh quadrilateral mesh at polynomial order `order`,
    after `refinements` uniform refinements (the reference's ser_ref_levels).
    boundary maps a physical line name to a condition (as in box()); lines
    identified by $Periodic are periodic.  Returns a theseus_b200.Mesh."""
    return quad_mesh_from(read_gmsh(path), order, boundary, coords, refinements, device)


def refine(nodes, quads, lines):
    """One uniform refinement of a first-order quadrilateral mesh without
    high-order nodes, as mfem::Mesh::UniformRefinement makes it: new vertices
    are averages of the old ones (mfem::Mesh::AverageVertices: the sum in
    the listed order, times 1/n), an edge's midpoint from its two ends, an
    element's centre from its four vertices in the element's order; each
    quadrilateral splits into four, each boundary line into two."""
    nodes = dict(nodes)
    nxt = max(nodes) + 1
    mids = {}

    def average(vs):
        n = len(vs)
        x, y = nodes[vs[0]]
        for v in vs[1:]:
            x, y = x + nodes[v][0], y + nodes[v][1]
        return (x * (1.0 / n), y * (1.0 / n))

    def mid(a, b):
        nonlocal nxt
        k = (min(a, b), max(a, b))
        if k not in mids:
            nodes[nxt] = average([a, b])
            mids[k] = nxt
            nxt += 1
        return mids[k]

    out = []
    for tag, v0, v1, v2, v3 in quads:
        c = nxt
        nodes[c] = average([v0, v1, v2, v3])
        nxt += 1
        m01, m12, m23, m30 = mid(v0, v1), mid(v1, v2), mid(v2, v3), mid(v3, v0)
        out += [(tag, v0, m01, c, m30), (tag, m01, v1, m12, c), (tag, c, m12, v2, m23), (tag, m30, c, m23, v3)]
    new_lines = []
    for name, a, b in lines:
        m = mids[(min(a, b), max(a, b))]
        new_lines += [(name, a, m), (name, m, b)]
    return nodes, out, new_lines


def quad_mesh_from(parsed, order, boundary=None, coords=True, refinements=0, device=None):
    """quad_mesh from read_gmsh's (nodes, quads, lines, periodic)."""
    nodes, quads, lines, periodic = parsed
    if refinements and periodic:
        raise NotImplementedError("refinement of periodic Gmsh meshes")
    for _ in range(refinements):
        nodes, quads, lines = refine(nodes, quads, lines)

    def canon(v):
        seen = set()
        while v in periodic and v not in seen:
            seen.add(v)
            v = periodic[v]
        return v

    corners = np.array([[nodes[v] for v in vs] for _, *vs in quads], dtype=np.float64).reshape(-1, 4, 2)
    vids = np.array([vs for _, *vs in quads], np.int64).reshape(-1, 4)
    blines = {(min(p, q), max(p, q)): name for name, p, q in lines}
    return quad_cells_mesh(corners, vids, order, blines, boundary, coords, canon, device)


def quad_cells_mesh(corners, vids, order, blines=None, boundary=None, coords=True, canon=None, device=None):
    """Geometry of straight-sided quadrilaterals: corners[e] are element e's
    four vertex positions in cyclic order, vids[e] their vertex ids (shared
    ids make a face interior; canon maps an id to its periodic
    representative), blines maps a sorted vertex-id pair of a boundary edge to
    the name of its condition in `boundary`.  With `device` (a CUDA device)
    the face table comes from the library and the geometric factors are
    computed on that GPU (theseus_b200.cells); the result is the same."""
    from . import Mesh, lgl, sizes
    from ._abi import BC_TYPES, Boundary
    canon = canon or (lambda v: v)
    blines = blines or {}
    N = order + 1
    x, w = lgl(N)
    ne = len(corners)
    nd, nfp, _ = sizes(2, order)
    V = np.zeros((ne, 4, 2))
    vid = np.zeros((ne, 4), np.int64)
    for e in range(ne):
        P, vs = corners[e], vids[e]
        # orient along the axes: v0 lower-left, v1 lower-right, v2 upper-right, v3 upper-left
        c = P.mean(axis=0)
        ang = np.arctan2(P[:, 1] - c[1], P[:, 0] - c[0])
        order_ = np.argsort(ang)                     # counter-clockwise from -pi
        k0 = int(np.argmin(P[order_, 0] + P[order_, 1]))
        order_ = np.roll(order_, -k0)
        V[e] = P[order_]
        vid[e] = [vs[j] for j in order_]
    if device is not None:
        from .cells import cell_mesh
        lex = [0, 1, 3, 2]                           # cyclic (ll, lr, ur, ul) -> lexicographic
        ids = np.array([[canon(int(v)) for v in row] for row in vid[:, lex]], np.int64)
        bfaces = {tuple(sorted((canon(int(p)), canon(int(q))))): n for (p, q), n in blines.items()}
        return cell_mesh(2, order, V[:, lex], ids, bfaces, boundary, coords, device)
    # bilinear map at the LGL nodes (node = i + N j, i along x)
    xi, eta = np.meshgrid(x, x, indexing="xy")       # [j][i]
    xi, eta = xi.ravel(), eta.ravel()
    X0, X1, X2, X3 = (V[:, k, None, :] for k in range(4))
    a, b = xi[None, :, None], eta[None, :, None]
    pos = (1 - a) * (1 - b) * X0 + a * (1 - b) * X1 + a * b * X2 + (1 - a) * b * X3
    dxi = (1 - b) * (X1 - X0) + b * (X2 - X3)
    deta = (1 - a) * (X3 - X0) + a * (X2 - X1)
    J = dxi[..., 0] * deta[..., 1] - deta[..., 0] * dxi[..., 1]
    metric = np.zeros((ne, nd, 2, 2))
    metric[:, :, 0, 0], metric[:, :, 0, 1] = deta[..., 1], -deta[..., 0]
    metric[:, :, 1, 0], metric[:, :, 1, 1] = -dxi[..., 1], dxi[..., 0]
    # faces: element local faces 0:x- (v0,v3), 1:x+ (v1,v2), 2:y- (v0,v1), 3:y+ (v3,v2)
    fv = {0: (0, 3), 1: (1, 2), 2: (0, 1), 3: (3, 2)}
    key = {}
    for e in range(ne):
        for lf, (p, q) in fv.items():
            k = (min(canon(vid[e, p]), canon(vid[e, q])), max(canon(vid[e, p]), canon(vid[e, q])))
            key.setdefault(k, []).append((e, lf))
    faces, bfaces = [], []
    for k, users in key.items():
        if len(users) == 2:
            (e1, l1), (e2, l2) = users
            if l1 % 2 == 0:                          # minus side: the element whose + face it is
                (e1, l1), (e2, l2) = (e2, l2), (e1, l1)
            if l2 != l1 - 1:
                raise ValueError("faces not aligned: the mesh is not axis-structured")
            faces.append((l1 // 2, e1, l1, e2, l2))
        elif len(users) == 1:
            e, lf = users[0]
            p, q = fv[lf]
            raw = (min(vid[e, p], vid[e, q]), max(vid[e, p], vid[e, q]))
            bfaces.append((lf // 2, e, lf, blines.get(raw, "")))
        else:
            raise ValueError("non-manifold face")
    faces.sort()
    bfaces.sort(key=lambda t: (t[0], t[1], t[2]))

    def trace(lf):
        i = np.arange(N)
        if lf == 0:
            return i * N
        if lf == 1:
            return N - 1 + i * N
        if lf == 2:
            return i
        return i + N * (N - 1)

    def normal(e, lf):
        """Outward normal (face-Jacobian scaled) at the face points of element e."""
        t = trace(lf)
        if lf // 2 == 0:                             # x faces: tangent d/deta
            d = deta[e, t]
            n = np.stack([d[:, 1], -d[:, 0]], axis=1)
        else:                                        # y faces: tangent d/dxi
            d = dxi[e, t]
            n = np.stack([-d[:, 1], d[:, 0]], axis=1)
        return n if lf % 2 == 1 else 0.0 - n

    nf = len(faces)
    fe = np.zeros((nf, 2), np.int32)
    fl = np.zeros((nf, 2), np.int32)
    fn = np.zeros((nf, nfp, 2))
    wm = np.zeros((nf, nfp))
    wp = np.zeros((nf, nfp))
    for f, (_, e1, l1, e2, l2) in enumerate(faces):
        fe[f] = (e1, e2)
        fl[f] = (l1, l2)
        fn[f] = normal(e1, l1)
        wm[f] = 1.0 / (w[0] * J[e1, trace(l1)])
        wp[f] = 1.0 / (w[0] * J[e2, trace(l2)])
    bdr = None
    if bfaces:
        boundary = boundary or {}
        names = sorted({t[3] for t in bfaces})
        missing = [n for n in names if n not in boundary]
        if missing:
            raise ValueError(f"boundary lines without a condition: {missing}")
        bcs, data, index = [], [], {}
        for n in names:
            spec = boundary[n]
            nm, payload = (spec, ()) if isinstance(spec, str) else (spec[0], tuple(np.ravel(spec[1:])))
            index[n] = len(bcs)
            bcs.append((BC_TYPES[nm], len(data)))
            data.extend(float(v) for v in payload)
        be = np.array([t[1] for t in bfaces], np.int32)
        bl = np.array([t[2] for t in bfaces], np.int32)
        bn = np.stack([normal(e, lf) for _, e, lf, _ in bfaces])
        bw = np.stack([1.0 / (w[0] * J[e, trace(lf)]) for _, e, lf, _ in bfaces])
        bi = np.array([index[t[3]] for t in bfaces], np.int32)
        bdr = Boundary(be, bl, bn, bw, bi, bcs, data)
    xyz = np.stack([pos[..., 0], pos[..., 1]]) if coords else None
    return Mesh(2, order, J, metric, fe, fl, fn, wm, wp, coords=xyz, shape=None, boundary=bdr)
