"""Boundary faces: the inviscid boundary conditions of the reference
(include/bc_kernels.hpp:138-279, include/Flow.hpp:54-170) on Cartesian boxes
whose non-periodic sides carry them.

CPU: the oracle's restatement against the reference's own boundary kernel
(oracle/_ref), the split of a periodic box into interior and boundary faces,
and free-stream preservation along slip walls.  GPU: the CUDA path against
the oracle, per condition and mixed, FP64 (1e-12 relative L2 per variable)."""
import numpy as np
import pytest

import oracle as O
import theseus_b200 as T
from theseus_b200 import cases
from _helpers import oracle_mesh, random_geometry, rel_l2, smooth_state

TOL = 1e-12
Q_EXT = {2: [1.1, 0.35, -0.05, 2.7], 3: [1.1, 0.35, -0.05, 0.1, 2.75]}   # exterior state


def spec(name, dim):
    if name in ("supersonic-inflow", "exterior-state"):
        return (name, *Q_EXT[dim])
    if name == "no-slip-adiabatic":          # wall velocity, wall heat flux
        return (name, *([0.2, -0.1, 0.05][:dim]), 0.03)
    if name == "no-slip-isothermal":         # wall velocity, wall temperature
        return (name, *([0.2, -0.1, 0.05][:dim]), 0.004)
    return name


def bmesh(dim, order, n, sides, periodic=None, seed=0, perturb=True):
    lo, hi = [-1.0, -0.5, -0.75][:dim], [1.5, 1.0, 1.25][:dim]
    if periodic is None:
        periodic = tuple(f"{'xyz'[d]}-" not in sides for d in range(dim))
    m = T.box(dim, order, n, lo, hi, periodic=periodic, boundary=sides)
    return random_geometry(m, seed=seed) if perturb else m


CONDITIONS = ["slip", "supersonic-inflow", "supersonic-outflow", "exterior-state", "symmetry",
              "no-slip-adiabatic"]


def test_box_split_covers_every_element_face_once():
    m = bmesh(3, 2, (3, 2, 4), {"x-": "slip", "x+": "slip", "z-": "symmetry", "z+": "slip"},
              perturb=False)
    b = m.boundary
    assert b.num_faces == 2 * 2 * 4 + 2 * 3 * 2
    seen = np.zeros((m.num_elements, 6), int)
    for f in range(m.num_faces):
        for s in range(2):
            seen[m.face_elem[f, s], m.face_lface[f, s]] += 1
    for e, lf in zip(b.elem, b.lface):
        seen[e, lf] += 1
    assert np.all(seen == 1)
    # outward normals: -axis on the low side, +axis on the high side
    d = b.lface // 2
    sgn = np.where(b.lface % 2 == 1, 1.0, -1.0)
    assert np.all(np.sign(b.normal[np.arange(b.num_faces), 0, d]) == sgn)
    # boundary faces are numbered direction by direction
    assert np.all(np.diff(d) >= 0)


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built here")
@pytest.mark.parametrize("dim,order,n", [(2, 3, (4, 3)), (3, 2, (3, 2, 3))])
@pytest.mark.parametrize("name", CONDITIONS)
def test_oracle_boundary_matches_reference(dim, order, n, name):
    sides = {"x-": spec(name, dim), "x+": spec(name, dim)}
    if dim == 3:
        sides.update({"z-": spec(name, dim), "z+": spec(name, dim)})
    m = bmesh(dim, order, n, sides, seed=order)
    u = smooth_state(m, seed=dim)
    cfg = T.make_config(flow="euler", volume_flux="chandrashekar", surface_flux="roe")
    om = oracle_mesh(m)
    a = O.rhs(om, cfg, u)
    b = O.ref_rhs(om, cfg, u)
    assert np.array_equal(a, b), np.abs(a - b).max()


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built here")
@pytest.mark.parametrize("surf", ["hll", "llf", "roe", "chandrashekar", "ranocha"])
def test_oracle_mixed_boundaries_match_reference(surf):
    sides = {"x-": spec("supersonic-inflow", 2), "x+": "supersonic-outflow", "y-": "slip",
             "y+": "symmetry"}
    m = bmesh(2, 4, (3, 4), sides, seed=7)
    u = smooth_state(m, seed=3)
    cfg = T.make_config(flow="euler", volume_flux="ranocha", surface_flux=surf)
    om = oracle_mesh(m)
    assert np.array_equal(O.rhs(om, cfg, u), O.ref_rhs(om, cfg, u))


NS_CONDITIONS = ["no-slip-adiabatic", "no-slip-isothermal", "exterior-state", "slip", "symmetry",
                 "supersonic-outflow"]


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built here")
@pytest.mark.parametrize("dim,order,n", [(2, 3, (4, 3)), (3, 2, (3, 2, 3))])
@pytest.mark.parametrize("name", NS_CONDITIONS)
def test_oracle_ns_boundary_matches_reference(dim, order, n, name):
    """Gradient jump (BR1 lift) and viscous boundary flux of each condition."""
    sides = {"x-": spec(name, dim), "x+": spec(name, dim)}
    if dim == 3:
        sides.update({"z-": spec(name, dim), "z+": spec(name, dim)})
    m = bmesh(dim, order, n, sides, seed=order + 5)
    u = smooth_state(m, seed=dim + 2)
    cfg = T.make_config(flow="ns", volume_flux="ranocha", surface_flux="hll", mu=0.01, Pr=0.72)
    om = oracle_mesh(m)
    a = O.rhs(om, cfg, u)
    b = O.ref_rhs(om, cfg, u)
    assert np.array_equal(a, b), np.abs(a - b).max()


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built here")
def test_oracle_ns_mixed_boundaries_match_reference():
    sides = {"x-": spec("exterior-state", 2), "x+": "supersonic-outflow",
             "y-": spec("no-slip-isothermal", 2), "y+": spec("no-slip-adiabatic", 2)}
    m = bmesh(2, 4, (3, 4), sides, seed=9)
    u = smooth_state(m, seed=4)
    cfg = T.make_config(flow="ns", volume_flux="chandrashekar", surface_flux="roe", mu=0.02,
                        Pr=0.71)
    om = oracle_mesh(m)
    assert np.array_equal(O.rhs(om, cfg, u), O.ref_rhs(om, cfg, u))


def test_free_stream_along_slip_walls():
    """A uniform flow parallel to slip walls is a steady state."""
    m = bmesh(2, 3, (4, 4), {"y-": "slip", "y+": "slip"}, perturb=False)
    rho = np.ones(m.coords[0].shape)
    u = cases.conserved(rho, [0.4 * rho, 0.0 * rho], 1.0 * rho, 1.4)
    cfg = T.make_config(flow="euler", volume_flux="chandrashekar", surface_flux="hll")
    du = O.rhs(oracle_mesh(m), cfg, u)
    assert np.abs(du).max() < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("dim,order,n", [(2, 3, (5, 4)), (3, 3, (3, 2, 3))])
@pytest.mark.parametrize("name", CONDITIONS)
def test_gpu_boundary_conditions(cuda, dim, order, n, name):
    import torch
    sides = {"x-": spec(name, dim), "x+": spec(name, dim), "y-": spec(name, dim), "y+": spec(name, dim)}
    m = bmesh(dim, order, n, sides, seed=order + dim)
    u = smooth_state(m, seed=1)
    kw = dict(numerical_flux="chandrashekar", surface_flux="roe")
    op = T.EulerOperator(m, **kw)
    ud = torch.as_tensor(u, device="cuda")
    du = torch.empty_like(ud)
    op.Mult(ud, du)
    cfg = T.make_config(flow="euler", volume_flux="chandrashekar", surface_flux="roe")
    ref = O.rhs(oracle_mesh(m), cfg, u)
    assert rel_l2(du.cpu().numpy(), ref).max() <= TOL


@pytest.mark.gpu
@pytest.mark.parametrize("surf", ["hll", "llf", "roe", "pirozzoli"])
def test_gpu_mixed_boundaries_and_blending(cuda, surf):
    import torch
    sides = {"x-": spec("supersonic-inflow", 3), "x+": "supersonic-outflow", "y-": "slip",
             "y+": "symmetry", "z-": spec("exterior-state", 3), "z+": "slip"}
    m = bmesh(3, 3, (3, 3, 2), sides, seed=11)
    u = cases.sedov(m.coords, width=0.2)
    kw = dict(numerical_flux="chandrashekar", surface_flux=surf, fv_flux="llf", blending=True)
    op = T.EulerOperator(m, **kw)
    ud = torch.as_tensor(u, device="cuda")
    du = torch.empty_like(ud)
    op.Mult(ud, du)
    cfg = T.make_config(flow="euler", volume_flux="chandrashekar", surface_flux=surf, fv_flux="llf",
                        blending=True)
    ref = O.rhs(oracle_mesh(m), cfg, u)
    assert rel_l2(du.cpu().numpy(), ref).max() <= TOL


@pytest.mark.gpu
@pytest.mark.parametrize("dim,order,n", [(2, 4, (4, 3)), (3, 3, (3, 2, 2))])
@pytest.mark.parametrize("name", NS_CONDITIONS)
def test_gpu_ns_boundary_conditions(cuda, dim, order, n, name):
    """BR1 boundary jump in the gradient kernel, primitive gradients at the
    boundary points, viscous boundary flux in the boundary kernel."""
    import torch
    sides = {"x-": spec(name, dim), "x+": spec(name, dim), "y-": spec(name, dim), "y+": spec(name, dim)}
    m = bmesh(dim, order, n, sides, seed=order + 2 * dim)
    u = smooth_state(m, seed=5)
    op = T.NSOperator(m, numerical_flux="ranocha", surface_flux="hll", mu=0.01, Pr=0.72)
    ud = torch.as_tensor(u, device="cuda")
    du = torch.empty_like(ud)
    op.Mult(ud, du)
    cfg = T.make_config(flow="ns", volume_flux="ranocha", surface_flux="hll", mu=0.01, Pr=0.72)
    ref = O.rhs(oracle_mesh(m), cfg, u)
    assert rel_l2(du.cpu().numpy(), ref).max() <= TOL


@pytest.mark.gpu
def test_gpu_ns_mixed_walls_sutherland(cuda):
    import torch
    sides = {"x-": spec("exterior-state", 2), "x+": "supersonic-outflow",
             "y-": spec("no-slip-isothermal", 2), "y+": spec("no-slip-adiabatic", 2)}
    m = bmesh(2, 5, (3, 4), sides, seed=13)
    u = smooth_state(m, seed=6)
    kw = dict(mu=0.02, Pr=0.71, sutherland=True)
    op = T.NSOperator(m, numerical_flux="chandrashekar", surface_flux="roe", **kw)
    ud = torch.as_tensor(u, device="cuda")
    du = torch.empty_like(ud)
    op.Mult(ud, du)
    cfg = T.make_config(flow="ns", volume_flux="chandrashekar", surface_flux="roe", **kw)
    ref = O.rhs(oracle_mesh(m), cfg, u)
    assert rel_l2(du.cpu().numpy(), ref).max() <= TOL


@pytest.mark.gpu
def test_gpu_boundaries_unsupported_forms_are_refused(cuda):
    m = bmesh(2, 3, (3, 3), {"x-": "slip", "x+": "slip"})
    with pytest.raises(T.THXError, match="unsupported"):
        T.NSOperator(m, numerical_flux="chandrashekar", surface_flux="roe", precision="fp32",
                     mu=0.01, Pr=0.72)


@pytest.mark.gpu
@pytest.mark.parametrize("blending", [False, True])
def test_gpu_fp32_mixed_boundaries_fp64_islands(cuda, blending):
    """FP32-mixed Euler on a mesh with boundary faces: every block of elements
    next to a boundary face is an FP64 island (with its faces, the boundary
    fluxes and, with blending, the blended blocks): those elements' rate
    equals the FP64 operator's bit for bit, the rest is FP32-accurate, and an
    SSP-RK3 run stays within FP32 round-off of FP64."""
    import torch
    sides = {"x-": spec("supersonic-inflow", 2), "x+": "supersonic-outflow",
             "y-": "slip", "y+": "symmetry"}
    m = bmesh(2, 3, (8, 6), sides, seed=5, perturb=False)
    u = smooth_state(m, seed=9)
    kw = dict(numerical_flux="chandrashekar", surface_flux="roe", blending=blending)
    off = [1.0, 0.3, 0.0, 2.5 + 0.045]
    op64 = T.EulerOperator(m, **kw)
    op32 = T.EulerOperator(m, precision="fp32", state_offset=off, **kw)
    ud = torch.as_tensor(u, device="cuda").contiguous()
    d64, d32 = torch.empty_like(ud), torch.empty_like(ud)
    op64.Mult(ud, d64)
    op32.Mult(ud, d32)
    epb = max(1, 256 // m.nd)
    blk = np.zeros((m.num_elements + epb - 1) // epb, bool)
    blk[np.asarray(m.boundary.elem) // epb] = True
    elems = np.repeat(blk, epb)[:m.num_elements]
    a64, a32 = d64.cpu().numpy(), d32.cpu().numpy()
    assert np.array_equal(a32[:, elems], a64[:, elems])
    assert rel_l2(a32, a64).max() <= 1e-5
    assert op32.read_status() == 0
    dt = 0.3 * op64.estimate_dt(ud, 1.0)
    ya, yb = ud.clone(), ud.clone()
    op64.rk3_steps(ya, dt, 20)
    op32.rk3_steps(yb, dt, 20)
    assert rel_l2(yb.cpu().numpy(), ya.cpu().numpy()).max() <= 1e-6
    assert op32.read_status() == 0


@pytest.mark.gpu
@pytest.mark.parametrize("flow", ["euler", "ns"])
def test_gpu_stability_estimate_with_boundaries(cuda, flow):
    """The boundary-point term of the stability estimate: interior wave
    speed, exterior state's speed and diffusivity (include/RHSOperator_impl.hpp:176-268)."""
    import torch
    sides = {"x-": spec("exterior-state", 2), "x+": "supersonic-outflow",
             "y-": spec("no-slip-isothermal", 2), "y+": spec("supersonic-inflow", 2)}
    m = bmesh(2, 3, (4, 3), sides, seed=21)
    u = smooth_state(m, seed=8)
    kw = dict(numerical_flux="chandrashekar", surface_flux="roe")
    phys = dict(mu=0.05, Pr=0.72) if flow == "ns" else {}
    op = (T.NSOperator if flow == "ns" else T.EulerOperator)(m, **kw, **phys)
    r = op.EstimateStability(torch.as_tensor(u, device="cuda"))
    cfg = T.make_config(flow=flow, volume_flux="chandrashekar", surface_flux="roe", **phys)
    _, ref = O.estimate_dt(oracle_mesh(m), cfg, u, 1.0)
    np.testing.assert_allclose(r, ref, rtol=1e-13, atol=0)


def test_oracle_stability_boundary_term_is_active():
    """An exterior state faster than the interior raises the surface rate."""
    sides = {"x-": ("exterior-state", 1.0, 5.0, 0.0, 30.0), "x+": "supersonic-outflow"}
    m = bmesh(2, 3, (4, 3), sides, perturb=False)
    u = smooth_state(m, seed=2)
    cfg = T.make_config(flow="euler", volume_flux="chandrashekar", surface_flux="roe")
    _, with_b = O.estimate_dt(oracle_mesh(m), cfg, u, 1.0)
    mp = bmesh(2, 3, (4, 3), {}, periodic=(True, True), perturb=False)
    _, periodic = O.estimate_dt(oracle_mesh(mp), cfg, u, 1.0)
    assert with_b[1] > periodic[1]
