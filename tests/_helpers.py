"""Shared test helpers: meshes for both sides, states, error norms."""
import numpy as np

import oracle as O
import theseus_b200 as T
from theseus_b200 import cases


def oracle_mesh(m):
    """The product mesh's arrays wrapped for the oracle (same inputs on both sides)."""
    return O.Mesh(m.dim, m.order, m.jac, m.metric, m.face_elem, m.face_lface, m.face_normal,
                  m.face_wminus, m.face_wplus, coords=m.coords, shape=m.shape,
                  boundary=getattr(m, "boundary", None))


def box(dim, order, n, lo=None, hi=None):
    lo = lo if lo is not None else [-1.0, -0.5, -0.75][:dim]
    hi = hi if hi is not None else [1.5, 1.0, 1.25][:dim]
    return T.periodic_box(dim, order, n, lo, hi)


def random_geometry(m, seed=0, amp=0.05):
    """Per-node perturbed geometric factors: the RHS stays a well-defined
    function of (u, geometry) and every node/face index is exercised."""
    rng = np.random.default_rng(seed)
    jac = m.jac * (1.0 + amp * rng.uniform(-1, 1, m.jac.shape))
    met = m.metric + amp * np.abs(m.metric).max() * rng.uniform(-1, 1, m.metric.shape)
    nrm = m.face_normal * (1.0 + amp * rng.uniform(-1, 1, m.face_normal.shape)) + \
        amp * np.abs(m.face_normal).max() * rng.uniform(-1, 1, m.face_normal.shape)
    wm = m.face_wminus * (1.0 + amp * rng.uniform(-1, 1, m.face_wminus.shape))
    wp = m.face_wplus * (1.0 + amp * rng.uniform(-1, 1, m.face_wplus.shape))
    bdr = getattr(m, "boundary", None)
    if bdr is not None:
        from theseus_b200._abi import Boundary
        # oblique boundary normals: every branch of the wall rotation runs
        bn = bdr.normal + amp * 4 * np.abs(bdr.normal).max() * rng.uniform(-1, 1, bdr.normal.shape)
        bw = bdr.weight * (1.0 + amp * rng.uniform(-1, 1, bdr.weight.shape))
        bdr = Boundary(bdr.elem, bdr.lface, bn, bw, bdr.bc,
                       [(b.type, b.data_index) for b in bdr.bcs[:bdr.num_bcs]], bdr.bc_data[:bdr.bc_data_len])
    return T.Mesh(m.dim, m.order, jac, met, m.face_elem, m.face_lface, nrm, wm, wp,
                  coords=m.coords, shape=m.shape, boundary=bdr)


def smooth_state(m, seed=0, amp=0.05):
    """Smooth periodic perturbation of a uniform flow plus small seeded noise."""
    rng = np.random.default_rng(seed)
    x = m.coords
    dim = m.dim
    phase = sum((k + 1) * 2.1 * x[k] for k in range(dim))
    rho = 1.0 + 0.2 * np.sin(phase) + amp * rng.uniform(-1, 1, x[0].shape)
    vel = [0.3 * np.cos(phase + k) + amp * rng.uniform(-1, 1, x[0].shape) for k in range(dim)]
    p = 1.0 + 0.2 * np.cos(phase) + amp * rng.uniform(-1, 1, x[0].shape)
    return cases.conserved(rho, vel, p, 1.4)


def rel_l2(a, b):
    """Relative L2 error per conserved variable (rows of shape (neq, ...))."""
    a = np.asarray(a, np.float64).reshape(a.shape[0], -1)
    b = np.asarray(b, np.float64).reshape(b.shape[0], -1)
    nb = np.sqrt((b ** 2).sum(axis=1))
    floor = 1e-12 * nb.max() if nb.max() > 0 else 1.0
    return np.sqrt(((a - b) ** 2).sum(axis=1)) / np.maximum(nb, floor)


def to_dev(x, dtype=None):
    import torch
    t = torch.as_tensor(np.ascontiguousarray(x), device="cuda")
    return t.to(dtype) if dtype is not None else t
