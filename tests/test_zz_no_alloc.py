"""GPU: the allocation-free Euler right-hand side, for hosts that cannot let a
library call cudaMalloc (their device memory belongs to their own pool, or
their time loop cannot absorb cudaMalloc's device-wide synchronisation).

thx_rhs_euler_noalloc takes device-resident geometry and keeps its scratch in
a static device array; this file checks it, through the C ABI, against the
handle-based thx_rhs on two consecutive calls (the array keeps the previous
call's contents, so the second call shows nothing stale leaks through), and
that a mesh too large for the array is refused.  It lives in a file of its own
so that a run stopping at the first failure has already run everything else.
"""
import ctypes as C

import numpy as np
import pytest

import theseus_b200 as T
from _helpers import box, smooth_state, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-12


def device_geometry(mesh):
    """thx_geometry whose pointers are device tensors (kept alive by the caller)."""
    import torch
    keep = {k: torch.as_tensor(getattr(mesh, k), device="cuda").contiguous()
            for k in ("jac", "metric", "face_elem", "face_lface", "face_normal", "face_wminus",
                      "face_wplus")}
    g = T.Geometry()
    g.dim, g.order = mesh.dim, mesh.order
    g.num_elements, g.num_faces = mesh.num_elements, mesh.num_faces
    D, I = C.POINTER(C.c_double), C.POINTER(C.c_int32)
    for k, t in keep.items():
        setattr(g, k, C.cast(C.c_void_p(t.data_ptr()), I if k.startswith("face_e") or
                             k == "face_lface" else D))
    return g, keep


def noalloc_rhs(g, cfg, u, du):
    import torch
    lib = T.library()
    lib.thx_rhs_euler_noalloc.argtypes = [C.POINTER(T.Geometry), C.POINTER(T.Config), C.c_void_p,
                                          C.c_void_p, C.c_void_p]
    return lib.thx_rhs_euler_noalloc(C.byref(g), C.byref(cfg), C.c_void_p(u.data_ptr()),
                                     C.c_void_p(du.data_ptr()),
                                     C.c_void_p(torch.cuda.current_stream().cuda_stream))


@pytest.mark.parametrize("dim,order,n,vol,surf", [(2, 3, (6, 5), "chandrashekar", "roe"),
                                                  (3, 4, (3, 2, 3), "ranocha", "hll")])
def test_noalloc_matches_handle_path(cuda, dim, order, n, vol, surf):
    import torch
    m = box(dim, order, n)
    cfg = T.make_config(volume_flux=vol, surface_flux=surf)
    op = T.EulerOperator(m, numerical_flux=vol, surface_flux=surf)
    g, keep = device_geometry(m)
    for seed in (1, 2):  # two calls in a row through the shared scratch array
        u = torch.as_tensor(smooth_state(m, seed=seed), device="cuda").contiguous()
        ref = torch.empty_like(u)
        op.Mult(u, ref)
        got = torch.full_like(u, float("nan"))
        assert noalloc_rhs(g, cfg, u, got) == 0
        torch.cuda.synchronize()
        err = rel_l2(got.cpu().numpy(), ref.cpu().numpy())
        assert err.max() <= TOL, (seed, err)


def test_noalloc_rejects_oversized_mesh(cuda):
    import torch
    m = T.periodic_box(3, 4, (16, 16, 16), [0.0] * 3, [1.0] * 3, coords=False)  # 12 MB of face fluxes
    cfg = T.make_config(volume_flux="ranocha", surface_flux="hll")
    g, keep = device_geometry(m)
    u = torch.ones(m.state_shape(), dtype=torch.float64, device="cuda")
    du = torch.empty_like(u)
    assert noalloc_rhs(g, cfg, u, du) == T._abi.THX_ERR_INVALID_ARGUMENT


def test_noalloc_rejects_viscous_config(cuda):
    import torch
    m = box(2, 3, (3, 3))
    g, keep = device_geometry(m)
    u = torch.ones(m.state_shape(), dtype=torch.float64, device="cuda")
    cfg = T.make_config(flow="ns")
    assert noalloc_rhs(g, cfg, u, torch.empty_like(u)) == T._abi.THX_ERR_UNSUPPORTED
