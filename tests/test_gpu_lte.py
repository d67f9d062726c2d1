"""GPU parity of the LTE Helmholtz gas path (LTEEC volume and face fluxes,
Newton temperature recovery, LTE entropy variables and table transport),
through the C ABI, against the reference's golden right-hand sides and the
CPU oracle.  Bar: relative L2 <= 1e-12 per conserved variable, FP64
(include/LTEECFlux.hpp, include/LTEHelmholtzEOS.hpp,
include/LTEHelmholtzGasEOS.hpp semantics)."""
import os

import numpy as np
import pytest

import oracle as O
import theseus_b200 as T
from theseus_b200 import cases
from _helpers import oracle_mesh, rel_l2, to_dev

pytestmark = pytest.mark.gpu

TOL = 1e-12
GOLD = os.path.join(os.path.dirname(__file__), "golden")
IDG = dict(O.IDG_O2)


def product_table(nx, ny, log_rho=(-6.0, 1.0), log_T=(2.3, 4.3)):
    return T.HelmholtzTable.ideal_dissociating_gas(nx, ny, log_rho, log_T, **IDG)


def oracle_table(nx, ny, log_rho=(-6.0, 1.0), log_T=(2.3, 4.3)):
    return O.LteTable(nx, ny, log_rho, log_T)


def load_cfg(raw):
    import ctypes
    cfg = T.Config()
    b = raw.tobytes()
    ctypes.memmove(ctypes.addressof(cfg), b, min(len(b), ctypes.sizeof(cfg)))
    return cfg


def gpu_rhs_lte(mesh, u, table, ns=False, **kw):
    import torch
    op = (T.NSOperator if ns else T.EulerOperator)(mesh, numerical_flux="lteec",
                                                    surface_flux="lteec", gas=table, **kw)
    ud = to_dev(u, torch.float64)
    du = torch.empty_like(ud)
    op.Mult(ud, du)
    torch.cuda.synchronize()
    return du.cpu().numpy(), op


@pytest.mark.parametrize("name,ns", [("lte_euler_tgv_p2", False), ("lte_ns_tgv_p3", True)])
def test_lte_rhs_matches_reference_golden(cuda, name, ns):
    z = np.load(os.path.join(GOLD, name + ".npz"))
    spec = z["table"]
    tab = product_table(int(spec[0]), int(spec[1]), (spec[2], spec[3]), (spec[4], spec[5]))
    order = int(z["order"])
    m = T.periodic_box(3, order, tuple(int(v) for v in z["n"]), (0.0,) * 3, (2 * np.pi,) * 3)
    cfg = load_cfg(z["cfg"])
    du, op = gpu_rhs_lte(m, z["u"], tab, ns=ns, mu=cfg.mu, Pr=cfg.Pr)
    assert rel_l2(du, z["dudt"]).max() <= TOL
    assert op.read_status() == 0


@pytest.mark.parametrize("order,n,ns", [(4, (2, 3, 2), False), (4, (2, 2, 2), True),
                                        (3, (3, 2, 2), True), (5, (2, 2, 2), False)])
def test_lte_rhs_matches_oracle(cuda, order, n, ns):
    """Perturbed LTE Taylor-Green states (rho = 0.01, T around 3000 K, velocity
    noise) on a 96 x 160 table."""
    tab_p, tab_o = product_table(96, 160), oracle_table(96, 160)
    m = T.periodic_box(3, order, n, (0.0,) * 3, (2 * np.pi,) * 3)
    u = cases.lte_taylor_green(m.coords, dT=0.2)
    rng = np.random.default_rng(order)
    u[1:4] += 0.05 * u[0] * 300.0 * rng.uniform(-1, 1, u[1:4].shape)
    kw = dict(mu=2e-4, Pr=0.71)
    du, op = gpu_rhs_lte(m, u, tab_p, ns=ns, **kw)
    cfg = T.make_config(flow="ns" if ns else "euler", volume_flux="lteec", surface_flux="lteec", **kw)
    ref = O.rhs_lte(oracle_mesh(m), cfg, tab_o, u, nthreads=4)
    assert rel_l2(du, ref).max() <= TOL
    assert op.read_status() == 0


def test_lte_rk3_matches_composed_stages(cuda):
    """The fused SSP-RK3 stages equal three Mult calls combined on the host side
    in mfem::RK3SSPSolver's order."""
    import torch
    tab = product_table(64, 128)
    m = T.periodic_box(3, 3, (2, 2, 2), (0.0,) * 3, (2 * np.pi,) * 3)
    u0 = cases.lte_taylor_green(m.coords)
    op = T.NSOperator(m, numerical_flux="lteec", surface_flux="lteec", gas=tab, mu=1e-4, Pr=0.71)
    dt = 2e-6
    u = to_dev(u0, torch.float64)
    op.rk3_steps(u, dt, 1)
    x = to_dev(u0, torch.float64)
    k = torch.empty_like(x)
    op.Mult(x, k)
    y = x + dt * k
    op.Mult(y, k)
    y = 0.75 * x + 0.25 * (y + dt * k)
    op.Mult(y, k)
    ref = (1.0 / 3.0) * x + (2.0 / 3.0) * (y + dt * k)
    torch.cuda.synchronize()
    diff = (u - ref).abs().max().item()
    assert diff <= 1e-14 * ref.abs().max().item()
    assert op.read_status() == 0


def test_lte_recovery_failure_sets_status(cuda):
    """An internal energy below the table's range fails the recovery: the
    kernels flag it in the status word instead of trapping."""
    import torch
    tab = product_table(64, 128)
    m = T.periodic_box(3, 2, (2, 2, 2), (0.0,) * 3, (2 * np.pi,) * 3)
    u = cases.lte_taylor_green(m.coords)
    u[4, 3, 5] = u[0, 3, 5] * tab.e[0] * 0.5  # e below the energy grid
    op = T.EulerOperator(m, numerical_flux="lteec", surface_flux="lteec", gas=tab)
    ud = to_dev(u, torch.float64)
    du = torch.empty_like(ud)
    op.Mult(ud, du)
    assert op.read_status() & T.STATUS_EOS
    # the handle stays usable
    op.Mult(to_dev(cases.lte_taylor_green(m.coords), torch.float64), du)
    assert op.read_status() == 0


def test_lte_integral_measures_match_oracle(cuda):
    import torch
    tab_p, tab_o = product_table(64, 128), oracle_table(64, 128)
    m = T.periodic_box(3, 3, (2, 3, 2), (0.0,) * 3, (2 * np.pi,) * 3)
    u = cases.lte_taylor_green(m.coords, dT=0.2)
    op = T.EulerOperator(m, numerical_flux="lteec", surface_flux="lteec", gas=tab_p)
    got = op.IntegralMeasures(to_dev(u, torch.float64))
    cfg = T.make_config(volume_flux="lteec", surface_flux="lteec")
    ref = O.integral_measures(oracle_mesh(m), cfg, u, table=tab_o)
    for k in ref:
        assert abs(got[k] - ref[k]) <= 1e-14 * abs(ref[k]), (k, got[k], ref[k])
