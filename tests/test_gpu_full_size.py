"""GPU parity at the benchmark configurations' own sizes, against the oracle
on all host threads (include/RHSOperator_impl.hpp:719-793,
include/EulerOperator_impl.hpp:396-421, include/NSOperator_impl.hpp:161-192):

* the 2-D isentropic vortex exactly as benchmarked -- 32 x 32 quads, p=3,
  Chandrashekar volume / Roe surface flux, rho = 1, u = (1, 1), p = 1 with a
  vortex of strength 5 at the origin on the periodic [-5, 5]^2 -- one
  right-hand side with its global entropy residual, and 100 SSP-RK3 steps at
  the oracle's CFL-0.5 time step of the initial state;
* one right-hand side of the Navier-Stokes Taylor-Green vortex at 32^3, p=4
  (4.1 M nodes; Ranocha / HLL, Ma 0.1, Re 1600, Pr 0.71, seeded 1e-6 noise);
* one right-hand side of the LTE-gas Taylor-Green vortex at 24^3, p=4
  (1.7 M nodes; LTEEC fluxes, the 256 x 512 synthetic Helmholtz table).

Bar: relative L2 <= 1e-12 per conserved variable; the entropy residual
equal to the oracle's within 1e-12 of the sum of its terms' magnitudes, and
non-positive (the Roe surface flux dissipates entropy)."""
import numpy as np
import pytest

import oracle as O
import theseus_b200 as T
from theseus_b200 import cases
from _helpers import oracle_mesh, rel_l2, to_dev

pytestmark = pytest.mark.gpu

TOL = 1e-12


def entropy_terms_magnitude(m, u, du, gamma=1.4):
    """sum_e sum_i w_i J_i sum_k |v_k(U_i) dU_k/dt|: the scale of the global
    entropy residual (ideal-gas entropy variables, include/EOS.hpp:206-234)."""
    dim, N = m.dim, m.order + 1
    _, w = T.lgl(N)
    wq = np.ones(m.nd)
    a = np.arange(m.nd)
    wq = w[a % N] * w[(a // N) % N] * (w[a // (N * N)] if dim == 3 else 1.0)
    rho, mom, E = u[0], u[1:1 + dim], u[dim + 1]
    ke = 0.5 * (mom ** 2).sum(0) / rho
    p = (gamma - 1.0) * (E - ke)
    s = np.log(p) - gamma * np.log(rho)
    v = [(gamma - s) / (gamma - 1.0) - ke / p] + [mom[d] / p for d in range(dim)] + [-rho / p]
    tot = sum(np.abs(v[k] * du[k]) for k in range(dim + 2))
    return float((wq[None, :] * m.jac * tot).sum())


def test_vortex_2d_benchmark_case(cuda):
    import torch
    m = T.periodic_box(2, 3, (32, 32), [-5.0, -5.0], [5.0, 5.0])
    u = cases.isentropic_vortex(m.coords, strength=5.0)
    cfg = T.make_config(flow="euler", volume_flux="chandrashekar", surface_flux="roe")
    om = oracle_mesh(m)
    nth = O.max_threads()
    op = T.EulerOperator(m, numerical_flux="chandrashekar", surface_flux="roe")
    ud = to_dev(u, torch.float64)
    du = torch.empty_like(ud)
    op.Mult(ud, du)
    got = du.cpu().numpy()
    ref = O.rhs(om, cfg, u, nthreads=nth)
    assert rel_l2(got, ref).max() <= TOL
    # global entropy residual R_S = sum w J v . dU/dt
    rs_gpu = O.entropy_residual(om, cfg, u, got)
    rs_ref = O.entropy_residual(om, cfg, u, ref)
    scale = entropy_terms_magnitude(m, u, ref)
    assert abs(rs_gpu - rs_ref) <= 1e-12 * scale, (rs_gpu, rs_ref, scale)
    assert rs_ref <= 1e-12 * scale and rs_gpu <= 1e-12 * scale
    # 100 SSP-RK3 steps at the oracle's CFL-0.5 step of the initial state
    dt, _ = O.estimate_dt(om, cfg, u, 0.5)
    assert abs(op.estimate_dt(ud, 0.5) - dt) <= 1e-13 * dt
    op.rk3_steps(ud, dt, 100)
    y = ud.cpu().numpy()
    ref_y = O.rk3_steps(om, cfg, u, dt, 100, nthreads=nth)
    assert rel_l2(y, ref_y).max() <= TOL
    assert op.read_status() == 0


def test_ns_tgv_32cubed_rhs(cuda):
    import torch
    m = T.periodic_box(3, 4, (32, 32, 32), [0.0] * 3, [2 * np.pi] * 3)
    u = cases.taylor_green(m.coords, mach=0.1, noise=1e-6, seed=0)
    kw = dict(mu=1.0 / 1600, Pr=0.71)
    op = T.NSOperator(m, numerical_flux="ranocha", surface_flux="hll", **kw)
    ud = to_dev(u, torch.float64)
    du = torch.empty_like(ud)
    op.Mult(ud, du)
    got = du.cpu().numpy()
    del op, ud, du
    cfg = T.make_config(flow="ns", volume_flux="ranocha", surface_flux="hll", **kw)
    ref = O.rhs(oracle_mesh(m), cfg, u, nthreads=O.max_threads())
    assert rel_l2(got, ref).max() <= TOL


def test_lte_tgv_24cubed_rhs(cuda):
    import torch
    tab = T.HelmholtzTable.ideal_dissociating_gas(256, 512, (-6.0, 1.0), (2.3, 4.3), **O.IDG_O2)
    m = T.periodic_box(3, 4, (24, 24, 24), [0.0] * 3, [2 * np.pi] * 3)
    u = cases.lte_taylor_green(m.coords)
    op = T.NSOperator(m, numerical_flux="lteec", surface_flux="lteec", gas=tab, Pr=0.71)
    ud = to_dev(u, torch.float64)
    du = torch.empty_like(ud)
    op.Mult(ud, du)
    got = du.cpu().numpy()
    assert op.read_status() == 0
    del op, ud, du
    cfg = T.make_config(flow="ns", volume_flux="lteec", surface_flux="lteec", Pr=0.71)
    ot = O.LteTable(256, 512, (-6.0, 1.0), (2.3, 4.3))
    ref = O.rhs_lte(oracle_mesh(m), cfg, ot, u, nthreads=O.max_threads())
    assert rel_l2(got, ref).max() <= TOL
