"""Meshes of straight-sided cells with the face table built by the library
(thx_cell_faces, host) and the geometric factors computed on the GPU
(thx_cell_geometry): the device-side stand-in for the reference's MFEM cache
set-up (include/dgsem_cache_utilities.hpp:83-215, 470-639).

Cells are given by their 2^dim vertices in lexicographic order of the
reference coordinates (x fastest), oriented along the mesh axes, and by the
vertex ids that decide which faces are shared (periodic partners carry one
id)."""
import ctypes as C

import numpy as np

_I = C.POINTER(C.c_int32)


def _lib():
    from . import library
    lib = library()
    if not getattr(lib, "_cells_bound", False):
        lib.thx_cell_faces.argtypes = [C.c_int, C.c_int, C.c_void_p, _I, _I, _I, _I, _I, _I]
        lib.thx_cell_geometry.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p,
                                          C.c_void_p, C.c_int, C.c_void_p, C.c_void_p] + [C.c_void_p] * 9
        lib._cells_bound = True
    return lib


def cell_faces(dim, vertex_ids):
    """(face_elem, face_lface, bdr_elem, bdr_lface) of conforming cells."""
    from . import _check
    ids = np.ascontiguousarray(vertex_ids, dtype=np.int64).reshape(-1, 1 << dim)
    ne = len(ids)
    fe = np.zeros((ne * dim, 2), np.int32)
    fl = np.zeros((ne * dim, 2), np.int32)
    be = np.zeros(2 * dim * ne, np.int32)
    bl = np.zeros(2 * dim * ne, np.int32)
    nf, nb = C.c_int32(), C.c_int32()
    p = lambda a: a.ctypes.data_as(_I)
    _check(_lib().thx_cell_faces(dim, ne, ids.ctypes.data_as(C.c_void_p), p(fe), p(fl), C.byref(nf), p(be),
                                 p(bl), C.byref(nb)), "thx_cell_faces")
    return fe[:nf.value].copy(), fl[:nf.value].copy(), be[:nb.value].copy(), bl[:nb.value].copy()


def cell_geometry(dim, order, corners, face_elem, face_lface, bdr_elem=None, bdr_lface=None, device="cuda",
                  coords=True, stream=None):
    """The geometric factors, computed on the GPU, as device tensors:
    dict(jac, metric, face_normal, face_wminus, face_wplus, bdr_normal,
    bdr_weight, coords)."""
    import torch
    from . import _check, _stream_ptr, sizes
    nd, nfp, _ = sizes(dim, order)
    dev = torch.device(device)
    c = torch.as_tensor(np.ascontiguousarray(corners, np.float64).reshape(-1, 1 << dim, dim), device=dev)
    ne = c.shape[0]
    fe = torch.as_tensor(np.ascontiguousarray(face_elem, np.int32), device=dev)
    fl = torch.as_tensor(np.ascontiguousarray(face_lface, np.int32), device=dev)
    nf = fe.shape[0]
    be = torch.as_tensor(np.ascontiguousarray(bdr_elem if bdr_elem is not None else [], np.int32), device=dev)
    bl = torch.as_tensor(np.ascontiguousarray(bdr_lface if bdr_lface is not None else [], np.int32), device=dev)
    nb = be.shape[0]
    z = lambda *s: torch.zeros(s, dtype=torch.float64, device=dev)
    out = dict(jac=z(ne, nd), metric=z(ne, nd, dim, dim), face_normal=z(nf, nfp, dim), face_wminus=z(nf, nfp),
               face_wplus=z(nf, nfp), bdr_normal=z(nb, nfp, dim), bdr_weight=z(nb, nfp),
               coords=z(dim, ne, nd) if coords else None)
    ptr = lambda t: C.c_void_p(t.data_ptr()) if t is not None and t.numel() else None
    _check(_lib().thx_cell_geometry(dim, order, ne, ptr(c), nf, ptr(fe), ptr(fl), nb, ptr(be), ptr(bl),
                                    ptr(out["jac"]), ptr(out["metric"]), ptr(out["face_normal"]),
                                    ptr(out["face_wminus"]), ptr(out["face_wplus"]), ptr(out["bdr_normal"]),
                                    ptr(out["bdr_weight"]), ptr(out["coords"]), _stream_ptr(stream)),
           "thx_cell_geometry")
    return out


def cell_mesh(dim, order, corners, vertex_ids, boundary_faces=None, boundary=None, coords=True, device="cuda"):
    """A theseus_b200.Mesh of straight-sided cells: face table from the
    library, geometric factors computed on the GPU (copied to the host arrays
    the Mesh holds).  boundary_faces maps a boundary face's sorted vertex ids
    (a tuple) to the name of its condition in `boundary` (as in box())."""
    from . import Mesh
    from ._abi import BC_TYPES, Boundary
    ids = np.ascontiguousarray(vertex_ids, dtype=np.int64).reshape(-1, 1 << dim)
    fe, fl, be, bl = cell_faces(dim, ids)
    g = cell_geometry(dim, order, corners, fe, fl, be, bl, device=device, coords=coords)
    host = {k: (v.cpu().numpy() if v is not None else None) for k, v in g.items()}
    bdr = None
    if len(be):
        boundary_faces = boundary_faces or {}
        boundary = boundary or {}
        names = []
        for e, lf in zip(be, bl):
            side, d = lf & 1, lf >> 1
            key = tuple(sorted(int(ids[e, v]) for v in range(1 << dim) if ((v >> d) & 1) == side))
            names.append(boundary_faces.get(key, ""))
        missing = sorted({n for n in names if n not in boundary})
        if missing:
            raise ValueError(f"boundary faces without a condition: {missing}")
        bcs, data, index = [], [], {}
        for n in sorted(set(names)):
            spec = boundary[n]
            nm, payload = (spec, ()) if isinstance(spec, str) else (spec[0], tuple(np.ravel(spec[1:])))
            index[n] = len(bcs)
            bcs.append((BC_TYPES[nm], len(data)))
            data.extend(float(v) for v in payload)
        bdr = Boundary(be, bl, host["bdr_normal"], host["bdr_weight"], np.array([index[n] for n in names], np.int32),
                       bcs, data)
    return Mesh(dim, order, host["jac"], host["metric"], fe, fl, host["face_normal"], host["face_wminus"],
                host["face_wplus"], coords=host["coords"], shape=None, boundary=bdr)
