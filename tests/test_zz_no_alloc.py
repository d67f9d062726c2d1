"""GPU: the allocation-free Euler right-hand side, for hosts that cannot let a
library call cudaMalloc (their device memory belongs to their own pool, or
their time loop cannot absorb cudaMalloc's device-wide synchronisation).

thx_rhs_euler_noalloc takes device-resident geometry and keeps its scratch in
a static device array; this file checks it, through the C ABI, against the
handle-based thx_rhs on two consecutive calls (the array keeps the previous
call's contents, so the second call shows nothing stale leaks through), that
further calls leave the device's free memory unchanged, that the status word
reaches the caller (a non-positive state, an out-of-range face table entry,
which touches nothing outside the caller's arrays), and that a mesh too large
for the array is refused.  It lives in a file of its own
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


def noalloc_rhs(g, cfg, u, du, status=None):
    """status: a one-element int32 CUDA tensor receiving the call's status bits."""
    import torch
    lib = T.library()
    lib.thx_rhs_euler_noalloc.argtypes = [C.POINTER(T.Geometry), C.POINTER(T.Config), C.c_void_p,
                                          C.c_void_p, C.c_void_p, C.c_void_p]
    return lib.thx_rhs_euler_noalloc(C.byref(g), C.byref(cfg), C.c_void_p(u.data_ptr()),
                                     C.c_void_p(du.data_ptr()),
                                     C.c_void_p(status.data_ptr()) if status is not None else None,
                                     C.c_void_p(torch.cuda.current_stream().cuda_stream))


@pytest.mark.parametrize("dim,order,n,vol,surf", [(2, 3, (6, 5), "chandrashekar", "roe"),
                                                  (3, 4, (3, 2, 3), "ranocha", "hll")])
def test_noalloc_matches_handle_path(cuda, dim, order, n, vol, surf):
    import torch
    m = box(dim, order, n)
    cfg = T.make_config(volume_flux=vol, surface_flux=surf)
    op = T.EulerOperator(m, numerical_flux=vol, surface_flux=surf)
    g, keep = device_geometry(m)
    st = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    for seed in (1, 2):  # two calls in a row through the shared scratch array
        u = torch.as_tensor(smooth_state(m, seed=seed), device="cuda").contiguous()
        ref = torch.empty_like(u)
        op.Mult(u, ref)
        got = torch.full_like(u, float("nan"))
        assert noalloc_rhs(g, cfg, u, got, st) == 0
        torch.cuda.synchronize()
        err = rel_l2(got.cpu().numpy(), ref.cpu().numpy())
        assert err.max() <= TOL, (seed, err)
        assert int(st.item()) == 0


def test_noalloc_allocates_nothing(cuda):
    """After the first call (which looks the scratch array up), further calls
    leave the device's free memory exactly as it was."""
    import torch
    m = box(3, 3, (4, 3, 3))
    cfg = T.make_config(volume_flux="chandrashekar", surface_flux="roe")
    g, keep = device_geometry(m)
    u = torch.as_tensor(smooth_state(m, seed=3), device="cuda").contiguous()
    du = torch.empty_like(u)
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert noalloc_rhs(g, cfg, u, du, st) == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(5):
        assert noalloc_rhs(g, cfg, u, du, st) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    assert int(st.item()) == 0


def test_noalloc_reports_nonpositive_state(cuda):
    import torch
    m = box(2, 3, (4, 4))
    cfg = T.make_config(volume_flux="chandrashekar", surface_flux="llf")
    g, keep = device_geometry(m)
    u = torch.as_tensor(smooth_state(m, seed=4), device="cuda").contiguous()
    u[0, 5, 3] = -1.0  # negative density at one node
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert noalloc_rhs(g, cfg, u, torch.empty_like(u), st) == 0
    torch.cuda.synchronize()
    assert int(st.item()) & T._abi.STATUS_NONPOSITIVE


def test_noalloc_out_of_range_face_entry(cuda):
    """An out-of-range face_elem entry is reported, its face's fluxes are NaN,
    the elements away from it are unchanged, and nothing is written outside
    the caller's rate array (guard cells around it stay as they were)."""
    import torch
    m = box(2, 3, (5, 4))
    cfg = T.make_config(volume_flux="chandrashekar", surface_flux="roe")
    op = T.EulerOperator(m, numerical_flux="chandrashekar", surface_flux="roe")
    u = torch.as_tensor(smooth_state(m, seed=5), device="cuda").contiguous()
    ref = torch.empty_like(u)
    op.Mult(u, ref)
    bad = 7
    e_good, e_lost = int(m.face_elem[bad, 0]), int(m.face_elem[bad, 1])
    fe = m.face_elem.copy()
    fe[bad, 1] = m.num_elements + 1000  # out of range
    m.face_elem = fe
    g, keep = device_geometry(m)
    guard = 4096
    buf = torch.full((u.numel() + 2 * guard,), 12345.0, dtype=torch.float64, device="cuda")
    du = buf[guard:guard + u.numel()].view_as(u)
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert noalloc_rhs(g, cfg, u, du, st) == 0
    torch.cuda.synchronize()
    assert int(st.item()) & T._abi.STATUS_FACE_TABLE
    assert bool((buf[:guard] == 12345.0).all()) and bool((buf[guard + u.numel():] == 12345.0).all())
    got, r = du.cpu().numpy(), ref.cpu().numpy()
    assert np.isnan(got[:, e_good]).any()  # the valid side lifts the NaN fluxes
    # e_good lifts the NaN fluxes; e_lost no longer sees the face at all
    others = [e for e in range(m.num_elements) if e not in (e_good, e_lost)]
    assert np.abs(got[:, others] - r[:, others]).max() <= 1e-12 * np.abs(r).max()


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
