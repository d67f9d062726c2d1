"""GPU parity: the sm_100a kernels, called through the C ABI, against the CPU
oracle on the same seeded inputs.  Bar: relative L2 <= 1e-12 per conserved
variable for the FP64 path (include/RHSOperator_impl.hpp:719-793 semantics)."""
import itertools

import numpy as np
import pytest

import oracle as O
import theseus_b200 as T
from theseus_b200 import cases
from _helpers import box, oracle_mesh, random_geometry, smooth_state, rel_l2, to_dev

pytestmark = pytest.mark.gpu

TOL = 1e-12
FLUXES = ["chandrashekar", "ranocha", "pirozzoli", "hll", "llf", "roe"]


def gpu_rhs(mesh, u, **kw):
    import torch
    op = (T.NSOperator if kw.pop("ns", False) else T.EulerOperator)(mesh, **kw)
    ud = to_dev(u, op.dtype)
    du = torch.empty_like(ud)
    op.Mult(ud, du)
    torch.cuda.synchronize()
    return du.double().cpu().numpy(), op


def oracle_rhs(mesh, u, ns=False, **kw):
    if "numerical_flux" in kw:
        kw["volume_flux"] = kw.pop("numerical_flux")
    cfg = T.make_config(flow="ns" if ns else "euler", **kw)
    return O.rhs(oracle_mesh(mesh), cfg, u, nthreads=4, want_alpha=True)


@pytest.mark.parametrize("dim,order,n", [(2, 3, (6, 5)), (2, 2, (4, 7)), (2, 5, (3, 4)),
                                         (3, 2, (3, 4, 2)), (3, 3, (2, 3, 3)), (3, 4, (3, 2, 3)),
                                         (3, 5, (2, 2, 3))])
def test_euler_orders(cuda, dim, order, n):
    m = box(dim, order, n)
    u = smooth_state(m, seed=order)
    kw = dict(numerical_flux="chandrashekar", surface_flux="roe")
    du, _ = gpu_rhs(m, u, **kw)
    ref, _, _ = oracle_rhs(m, u, **kw)
    assert rel_l2(du, ref).max() <= TOL


@pytest.mark.parametrize("vol,surf", list(itertools.product(FLUXES[:3] + ["hll"], FLUXES)))
def test_flux_pairings_2d(cuda, vol, surf):
    m = box(2, 3, (5, 4))
    u = smooth_state(m, seed=3)
    du, _ = gpu_rhs(m, u, numerical_flux=vol, surface_flux=surf)
    ref, _, _ = oracle_rhs(m, u, volume_flux=vol, surface_flux=surf)
    assert rel_l2(du, ref).max() <= TOL


@pytest.mark.parametrize("vol,surf", [("chandrashekar", "roe"), ("ranocha", "hll"),
                                      ("pirozzoli", "llf"), ("roe", "chandrashekar"),
                                      ("ranocha", "ranocha"), ("pirozzoli", "pirozzoli")])
def test_flux_pairings_3d(cuda, vol, surf):
    m = box(3, 3, (3, 2, 3))
    u = smooth_state(m, seed=5)
    du, _ = gpu_rhs(m, u, numerical_flux=vol, surface_flux=surf)
    ref, _, _ = oracle_rhs(m, u, volume_flux=vol, surface_flux=surf)
    assert rel_l2(du, ref).max() <= TOL


@pytest.mark.parametrize("dim,order,n,vol,surf", [(2, 3, (5, 4), "ranocha", "hll"),
                                                  (3, 4, (3, 3, 3), "ranocha", "hll"),
                                                  (3, 2, (2, 3, 4), "chandrashekar", "roe"),
                                                  (2, 5, (3, 3), "pirozzoli", "llf")])
def test_navier_stokes(cuda, dim, order, n, vol, surf):
    m = box(dim, order, n)
    u = smooth_state(m, seed=11)
    kw = dict(numerical_flux=vol, surface_flux=surf, mu=0.05, Pr=0.71)
    du, _ = gpu_rhs(m, u, ns=True, **kw)
    cfg = dict(volume_flux=vol, surface_flux=surf, mu=0.05, Pr=0.71)
    ref, _, _ = oracle_rhs(m, u, ns=True, **cfg)
    assert rel_l2(du, ref).max() <= TOL


def test_tgv_ns_p4(cuda):
    """The benchmark's physics (TGV, Ranocha/HLL, Re=1600) on a small mesh."""
    m = T.periodic_box(3, 4, (4, 4, 4), [0, 0, 0], [2 * np.pi] * 3)
    u = cases.taylor_green(m.coords, mach=0.1, noise=1e-6, seed=0)
    kw = dict(numerical_flux="ranocha", surface_flux="hll", mu=1.0 / 1600, Pr=0.71)
    du, _ = gpu_rhs(m, u, ns=True, **kw)
    ref, _, _ = oracle_rhs(m, u, ns=True, volume_flux="ranocha", surface_flux="hll",
                           mu=1.0 / 1600, Pr=0.71)
    assert rel_l2(du, ref).max() <= TOL


@pytest.mark.parametrize("layout", [0, 1])
@pytest.mark.parametrize("dim,order,n,ns", [(2, 3, (4, 5), False), (3, 3, (2, 3, 2), False),
                                            (3, 2, (3, 2, 2), True), (2, 4, (3, 4), True)])
def test_random_geometry(cuda, dim, order, n, ns, layout):
    m = random_geometry(box(dim, order, n), seed=dim * 10 + order)
    u = smooth_state(m, seed=7)
    kw = dict(numerical_flux="ranocha", surface_flux="roe", geometry_layout=layout)
    du, _ = gpu_rhs(m, u, ns=ns, **kw)
    ref, _, _ = oracle_rhs(m, u, ns=ns, volume_flux="ranocha", surface_flux="roe")
    assert rel_l2(du, ref).max() <= TOL


@pytest.mark.parametrize("dim,order,n,ns", [(2, 3, (8, 8), False), (3, 3, (4, 4, 4), False),
                                            (3, 2, (4, 4, 3), True)])
def test_blending(cuda, dim, order, n, ns):
    """Persson-Peraire indicator + subcell FV blend on a Sedov-type blast."""
    m = T.periodic_box(dim, order, n, [-1.0] * dim, [1.0] * dim)
    u = cases.sedov(m.coords, width=0.05)
    kw = dict(numerical_flux="chandrashekar", surface_flux="llf", fv_flux="llf", blending=True)
    du, op = gpu_rhs(m, u, ns=ns, **kw)
    a_gpu, e_gpu = op.blending_coefficients()
    ref, a_ref, e_ref = oracle_rhs(m, u, ns=ns, volume_flux="chandrashekar", surface_flux="llf",
                                   fv_flux="llf", blending=True)
    assert (a_ref > 0).sum() > 0 and (a_ref == 0).sum() > 0, "case must mix blended and DG elements"
    assert np.abs(e_gpu.cpu().numpy() - e_ref).max() <= 1e-10
    assert np.abs(a_gpu.cpu().numpy() - a_ref).max() <= 1e-10
    assert rel_l2(du, ref).max() <= TOL


def test_rk3_steps(cuda):
    import torch
    m = box(2, 3, (6, 6))
    u = cases.isentropic_vortex(m.coords, strength=2.0)
    op = T.EulerOperator(m, numerical_flux="chandrashekar", surface_flux="roe")
    dt = 0.01
    ud = to_dev(u)
    op.rk3_steps(ud, dt, 5)
    torch.cuda.synchronize()
    cfg = T.make_config(volume_flux="chandrashekar", surface_flux="roe")
    ref = O.rk3_steps(oracle_mesh(m), cfg, u, dt, 5, nthreads=4)
    assert rel_l2(ud.cpu().numpy(), ref).max() <= TOL


def test_estimate_dt(cuda):
    m = box(3, 3, (3, 3, 2))
    u = smooth_state(m, seed=2)
    op = T.NSOperator(m, numerical_flux="ranocha", surface_flux="hll", mu=0.01)
    rates = op.EstimateStability(to_dev(u))
    cfg = T.make_config(flow="ns", volume_flux="ranocha", surface_flux="hll", mu=0.01)
    _, ref = O.estimate_dt(oracle_mesh(m), cfg, u, 0.5)
    assert np.allclose(rates, ref, rtol=1e-13, atol=0)


def test_entropy_residual(cuda):
    """The GPU reproduces the oracle's discrete entropy-production residual."""
    m = box(2, 3, (5, 5))
    u = smooth_state(m, seed=9)
    du, _ = gpu_rhs(m, u, numerical_flux="chandrashekar", surface_flux="chandrashekar")
    cfg = T.make_config(volume_flux="chandrashekar", surface_flux="chandrashekar")
    om = oracle_mesh(m)
    ref = O.rhs(om, cfg, u, nthreads=2)
    rs_gpu = O.entropy_residual(om, cfg, u, du)
    rs_ref = O.entropy_residual(om, cfg, u, ref)
    scale = O.entropy_residual(om, cfg, u, np.abs(ref))
    assert rs_ref <= 1e-12 * abs(scale)          # dissipative surface flux: R_S <= 0
    assert abs(rs_gpu - rs_ref) <= 1e-11 * abs(scale)


def _tgv_offset(mach=0.1, gamma=1.4):
    return [1.0, 0.0, 0.0, 0.0, 1.0 / (gamma * mach * mach) / (gamma - 1.0)]


def field_errors(a, b, dim):
    """Relative L2 error of each conserved field -- density, the momentum
    vector, total energy -- of a against b (arrays shaped (neq, ...))."""
    a = np.asarray(a, np.float64).reshape(a.shape[0], -1)
    b = np.asarray(b, np.float64).reshape(b.shape[0], -1)
    groups = [[0], list(range(1, dim + 1)), [dim + 1]]
    return np.array([np.sqrt(((a[g] - b[g]) ** 2).sum() / (b[g] ** 2).sum()) for g in groups])


def test_fp32_mixed_rhs_error(cuda):
    """FP32-mixed RHS of a compressible smooth 3-D flow (all rates O(1)) with
    the mean state as the working-copy offset: single-precision accuracy."""
    m = T.periodic_box(3, 4, (3, 3, 3), [-1.0, -0.5, -0.75], [1.5, 1.0, 1.25])
    u = smooth_state(m, seed=4)
    off = [float(u[k].mean()) for k in range(5)]
    kw = dict(numerical_flux="ranocha", surface_flux="hll", mu=0.01, Pr=0.71)
    du32, _ = gpu_rhs(m, u, ns=True, precision="fp32", state_offset=off, **kw)
    ref, _, _ = oracle_rhs(m, u, ns=True, volume_flux="ranocha", surface_flux="hll", mu=0.01, Pr=0.71)
    err = rel_l2(du32, ref)
    assert err.max() <= 2e-5, err


def test_fp32_mixed_tgv_rhs_error(cuda):
    """Low-Mach Taylor-Green vortex with the freestream offset.  The momentum
    rates are O(1); the mass and energy rates are O(Ma^2) remainders of
    divergence-free transport, so their FP32 error is measured against the
    momentum-rate scale."""
    m = T.periodic_box(3, 4, (3, 3, 3), [0, 0, 0], [2 * np.pi] * 3)
    u = cases.taylor_green(m.coords, mach=0.1, noise=1e-6)
    kw = dict(numerical_flux="ranocha", surface_flux="hll", mu=1.0 / 1600, Pr=0.71)
    du32, _ = gpu_rhs(m, u, ns=True, precision="fp32", state_offset=_tgv_offset(), **kw)
    ref, _, _ = oracle_rhs(m, u, ns=True, volume_flux="ranocha", surface_flux="hll",
                           mu=1.0 / 1600, Pr=0.71)
    fe = field_errors(du32, ref, 3)
    assert fe[1] <= 2e-5, fe                      # momentum vector
    mom = np.sqrt((ref[1:4] ** 2).sum())
    assert np.sqrt(((du32[0] - ref[0]) ** 2).sum()) <= 1e-5 * mom
    assert np.sqrt(((du32[4] - ref[4]) ** 2).sum()) <= 1e-3 * mom


@pytest.mark.parametrize("vol,surf", [("ranocha", "hll"), ("chandrashekar", "roe"),
                                      ("pirozzoli", "llf"), ("chandrashekar", "chandrashekar")])
def test_fp32_mixed_solution_error(cuda, vol, surf):
    """Final-solution error of FP32-mixed SSP-RK3 against the FP64 path (TGV)."""
    import torch
    m = T.periodic_box(3, 4, (4, 4, 4), [0, 0, 0], [2 * np.pi] * 3)
    u = cases.taylor_green(m.coords, mach=0.1, noise=1e-6)
    kw = dict(numerical_flux=vol, surface_flux=surf, mu=1.0 / 1600, Pr=0.71)
    op64 = T.NSOperator(m, **kw)
    op32 = T.NSOperator(m, precision="fp32", state_offset=_tgv_offset(), **kw)
    dt = 0.5 * op64.estimate_dt(to_dev(u), 1.0)
    a, b = to_dev(u), to_dev(u)
    op64.rk3_steps(a, dt, 20)
    op32.rk3_steps(b, dt, 20)
    torch.cuda.synchronize()
    err = field_errors(b.cpu().numpy(), a.cpu().numpy(), 3)
    assert err.max() <= 1e-6, err


@pytest.mark.parametrize("dim,order,n,ns", [(3, 4, (3, 3, 3), True), (3, 4, (4, 3, 2), False),
                                            (2, 3, (7, 5), False), (3, 2, (3, 3, 3), True)])
def test_bulk_copy_staged_volume_kernel(cuda, dim, order, n, ns):
    """volume_staging=1: persistent CTAs stage the next element block's state
    by bulk copy while evaluating the current one.  Same result as the oracle
    (odd element counts exercise the ordinary-load fallback of a short last
    block); FP32-mixed within FP32 round-off of the unstaged FP32 kernel (the
    two are separate compilations, free to contract multiply-adds differently)."""
    import torch
    m = box(dim, order, n)
    u = smooth_state(m, seed=7)
    kw = dict(numerical_flux="ranocha", surface_flux="hll", ns=ns, mu=0.01, Pr=0.71)
    du, op = gpu_rhs(m, u, volume_staging=1, **kw)
    assert op.read_status() == 0
    ref, _, _ = oracle_rhs(m, u, volume_flux="ranocha", surface_flux="hll", ns=ns, mu=0.01, Pr=0.71)
    assert rel_l2(du, ref).max() <= TOL
    d32a, _ = gpu_rhs(m, u, precision="fp32", volume_staging=1, **kw)
    d32b, _ = gpu_rhs(m, u, precision="fp32", **dict(kw))
    assert rel_l2(d32a, d32b).max() <= 1e-6


def test_fp32_mixed_fp64_islands(cuda):
    """FP32-mixed Euler with blending evaluates every block of elements (EPB
    = 256 / nodes per element) holding a blended element, and its faces, in
    FP64 from the FP64 state: those elements' right-hand side equals the FP64
    operator's bit for bit, the rest differs by FP32 round-off, and an SSP-RK3
    run stays closer to FP64 than with the blended elements kept in FP32."""
    import torch
    m = box(3, 3, (6, 6, 6), [-1.0] * 3, [1.0] * 3)
    u = cases.sedov(m.coords, width=0.05)
    kw = dict(numerical_flux="chandrashekar", surface_flux="llf", fv_flux="llf", blending=True,
              alpha_max=0.5, alpha_min=0.001)
    off = [1.0, 0.0, 0.0, 0.0, 1e-5 / 0.4]
    op64 = T.EulerOperator(m, **kw)
    op32 = T.EulerOperator(m, precision="fp32", state_offset=off, **kw)
    op32f = T.EulerOperator(m, precision="fp32", state_offset=off, mixed_blended_fp32=True, **kw)
    ud = to_dev(u)
    d64, d32, d32f = (torch.empty_like(ud) for _ in range(3))
    op64.Mult(ud, d64)
    op32.Mult(ud, d32)
    op32f.Mult(ud, d32f)
    a32, _ = op32.blending_coefficients()
    epb = max(1, 256 // m.nd)
    blk = (a32.view(-1, epb) > 0).any(dim=1) if m.num_elements % epb == 0 else None
    assert blk is not None and int(blk.sum()) > 0
    elems = torch.repeat_interleave(blk, epb)
    assert torch.equal(d32[:, elems], d64[:, elems])
    assert not torch.equal(d32f[:, elems], d64[:, elems])
    assert op32.read_status() == 0
    dt = 0.5 * op64.estimate_dt(ud, 0.5)
    ys = [to_dev(u) for _ in range(3)]
    for op, y in zip((op64, op32, op32f), ys):
        op.rk3_steps(y, dt, 20)
    torch.cuda.synchronize()
    e_isl = field_errors(ys[1].cpu().numpy(), ys[0].cpu().numpy(), 3).max()
    e_f32 = field_errors(ys[2].cpu().numpy(), ys[0].cpu().numpy(), 3).max()
    assert e_isl < e_f32, (e_isl, e_f32)
    assert op32.read_status() == 0


def test_fp32_mixed_perturbation_form(cuda):
    """FP32-mixed with the Chandrashekar volume flux and a Roe (LLF, HLL) surface
    flux evaluates the fluxes as deviations from those of the working-copy
    offset: a uniform state equal to the offset has a right-hand side of
    exactly zero, and on a Mach-1.5 isentropic vortex the SSP-RK3 solution
    stays closer to FP64 than with the fluxes evaluated whole."""
    import torch
    gamma, ma = 1.4, 1.5
    v = ma * np.sqrt(gamma) / np.sqrt(2.0)
    off = [1.0, v, v, 1.0 / (gamma - 1.0) + v * v]
    m = box(2, 5, (8, 8), [-5.0, -5.0], [5.0, 5.0])
    for surf in ("roe", "llf", "hll"):
        kw = dict(numerical_flux="chandrashekar", surface_flux=surf)
        op = T.EulerOperator(m, precision="fp32", state_offset=off, **kw)
        u0 = np.broadcast_to(np.array(off)[:, None, None], m.state_shape()).copy()
        ud = to_dev(u0)
        du = torch.empty_like(ud)
        op.Mult(ud, du)
        assert float(du.abs().max()) == 0.0, surf
    u = cases.isentropic_vortex(m.coords, strength=2.0, u_inf=(v, v))
    kw = dict(numerical_flux="chandrashekar", surface_flux="roe")
    op64 = T.EulerOperator(m, **kw)
    opp = T.EulerOperator(m, precision="fp32", state_offset=off, **kw)
    opw = T.EulerOperator(m, precision="fp32", state_offset=off, mixed_flux_no_perturbation=True, **kw)
    dt = 0.3 * op64.estimate_dt(to_dev(u), 1.0)
    ys = [to_dev(u) for _ in range(3)]
    for op, y in zip((op64, opp, opw), ys):
        op.rk3_steps(y, dt, 50)
    torch.cuda.synchronize()
    e_p = field_errors(ys[1].cpu().numpy(), ys[0].cpu().numpy(), 2).max()
    e_w = field_errors(ys[2].cpu().numpy(), ys[0].cpu().numpy(), 2).max()
    assert e_p < 0.5 * e_w and e_p < 1e-6, (e_p, e_w)
    assert opp.read_status() == 0


def test_status_flag(cuda):
    m = box(2, 2, (3, 3))
    u = smooth_state(m, seed=1)
    u[0, 0, 0] = -1.0  # negative density at one node
    du, op = gpu_rhs(m, u, numerical_flux="ranocha", surface_flux="hll")
    assert op.read_status() & 1
    assert op.read_status() == 0


def test_fp32_mixed_positivity_checked_in_fp64(cuda):
    """FP32-mixed: the positivity test runs on the FP64 state (the working
    copy's narrowing and the RK stage epilogue).  A node whose FP64 pressure is
    -1e-9 (p = (gamma-1)(rho E - |m|^2/(2 rho))) sets the status flag, for a
    right-hand side and for an SSP-RK3 run; a positive state does not."""
    import torch
    m = box(2, 3, (3, 3))
    u = smooth_state(m, seed=1)
    rho, mx, my = 1.0, 3.0, 4.0
    ke = 0.5 * (mx * mx + my * my) / rho
    u[:, 4, 5] = [rho, mx, my, ke - 1e-9 / 0.4]  # p = -1e-9 in FP64
    kw = dict(numerical_flux="ranocha", surface_flux="hll")
    op = T.EulerOperator(m, precision="fp32", state_offset=[1.0, 0.0, 0.0, 2.5], **kw)
    ud = to_dev(u)
    op.Mult(ud, torch.empty_like(ud))
    assert op.read_status() & T.STATUS_NONPOSITIVE
    v = smooth_state(m, seed=1)
    vd = to_dev(v)
    op.rk3_steps(vd, 1e-4, 2)
    assert op.read_status() == 0
    vd = to_dev(u)
    op.rk3_steps(vd, 1e-4, 1)
    assert op.read_status() & T.STATUS_NONPOSITIVE


def test_fp32_mixed_ns_rhs_narrows_in_gradient_kernel(cuda):
    """FP32-mixed Navier-Stokes right-hand side: the gradient kernel narrows
    the FP64 state into the working copy (no separate pass).  The positivity
    test still runs on the FP64 state, and the rate matches the FP64 oracle
    to single precision at every order."""
    import torch
    m = box(2, 3, (3, 3))
    u = smooth_state(m, seed=1)
    rho, mx, my = 1.0, 3.0, 4.0
    ke = 0.5 * (mx * mx + my * my) / rho
    u[:, 4, 5] = [rho, mx, my, ke - 1e-9 / 0.4]  # p = -1e-9 in FP64
    kw = dict(numerical_flux="ranocha", surface_flux="hll", mu=0.01, Pr=0.71)
    op = T.NSOperator(m, precision="fp32", state_offset=[1.0, 0.0, 0.0, 2.5], **kw)
    ud = to_dev(u)
    op.Mult(ud, torch.empty_like(ud))
    assert op.read_status() & T.STATUS_NONPOSITIVE
    for order in (2, 3, 4, 5):
        mm = T.periodic_box(2, order, (3, 4), [-1.0, -0.5], [1.5, 1.0])
        v = smooth_state(mm, seed=order)
        off = [float(v[k].mean()) for k in range(4)]
        du32, _ = gpu_rhs(mm, v, ns=True, precision="fp32", state_offset=off, **kw)
        ref, _, _ = oracle_rhs(mm, v, ns=True, volume_flux="ranocha", surface_flux="hll", mu=0.01, Pr=0.71)
        assert rel_l2(du32, ref).max() <= 2e-5, order


@pytest.mark.parametrize("dim,order,n,ns", [(2, 3, (6, 5), False), (3, 4, (3, 2, 3), True),
                                            (3, 2, (4, 3, 2), False)])
def test_integral_measures_match_oracle(cuda, dim, order, n, ns):
    """IntegralMeasures (include/RHSOperator_impl.hpp:530-717) on random geometry."""
    m = random_geometry(box(dim, order, n), seed=order)
    u = smooth_state(m, seed=2)
    kw = dict(numerical_flux="ranocha", surface_flux="hll", mu=0.01, Pr=0.71)
    op = (T.NSOperator if ns else T.EulerOperator)(m, **kw)
    got = op.IntegralMeasures(to_dev(u))
    cfg = T.make_config(flow="ns" if ns else "euler", volume_flux="ranocha", surface_flux="hll",
                        mu=0.01, Pr=0.71)
    ref = O.integral_measures(oracle_mesh(m), cfg, u)
    for k in ref:
        assert abs(got[k] - ref[k]) <= 1e-14 * abs(ref[k]), (k, got[k], ref[k])
