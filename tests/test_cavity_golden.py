"""The reference's own lid-driven-cavity golden trajectories (numerical-flux
regression: 2-D Navier-Stokes, p=2, 16 x 16 quads on [0,2]^2, adiabatic
no-slip walls, lid at unit velocity, Ma 0.1 rest state, mu 0.02, Pr 0.72,
subcell blending on, dt = 1e-4, HLL and Roe), compared at cycles 10 and 20
with the reference's own tolerances (rtol 1e-10, atol 1e-12) — the oracle on
the CPU and the CUDA path on the GPU.  Fixtures: tests/golden/cavity/*.npz,
made by tests/golden/cavity/make_cavity_fixtures.py from the reference's NPZ
files.

A golden entry is a DG node of one visualisation subcell, identified by the
subcell centre (which element) and the node position (which node).

The same cavity at p=3 with Chandrashekar fluxes is also compared after 4000
steps against the reference's recorded solution
(TestCases/GoldenData/LidDrivenCavity/Cycle004000, extracted by
tests/golden/cavity/make_cavity_vtu_fixture.py) with its regression recipe's
tolerances (rtol = atol = 1e-12)."""
import os

import numpy as np
import pytest

import oracle as O
import theseus_b200 as T
from theseus_b200 import cases
from _helpers import oracle_mesh

HERE = os.path.dirname(os.path.abspath(__file__))
GAMMA, MA, H, NX = 1.4, 0.1, 0.125, 16
WALL = ("no-slip-adiabatic", 0.0, 0.0, 0.0)
LID = ("no-slip-adiabatic", 1.0, 0.0, 0.0)
PHYS = dict(mu=0.02, Pr=0.72, R_gas=287.05, gamma=GAMMA)


def cavity(order=2):
    m = T.box(2, order, (NX, NX), [0.0, 0.0], [2.0, 2.0], periodic=(False, False),
              boundary={"x-": WALL, "x+": WALL, "y-": WALL, "y+": LID})
    rho = np.ones(m.coords[0].shape)
    u0 = cases.conserved(rho, [0.0 * rho, 0.0 * rho], rho / (MA * MA * GAMMA), GAMMA)
    return m, u0


def fields(m, u):
    """Density, pressure and velocity at every golden entry's node."""
    rho = u[0]
    vel = u[1:3] / rho
    p = (GAMMA - 1.0) * (u[3] - 0.5 * (u[1] ** 2 + u[2] ** 2) / rho)
    return rho, p, vel


def compare(m, u, flux, cycle, name=None, tol=1e-10):
    g = np.load(os.path.join(HERE, "golden", "cavity", name or f"{flux}_{cycle}.npz"))
    c, pt = g["center"], g["point"]
    e = (np.floor(c[:, 0] / H) + NX * np.floor(c[:, 1] / H)).astype(int)
    x, y = m.coords[0][e], m.coords[1][e]                    # (entries, nodes)
    d2 = (x - pt[:, :1]) ** 2 + (y - pt[:, 1:2]) ** 2
    node = d2.argmin(axis=1)
    assert np.all(d2[np.arange(len(e)), node] < 1e-20), "golden node not found on the mesh"
    rho, p, vel = fields(m, u)
    got = {"density": rho[e, node], "pressure": p[e, node], "velocity": vel[:, e, node].T}
    for k, v in got.items():
        np.testing.assert_allclose(v, g[k], rtol=tol, atol=1e-12, err_msg=f"{flux} cycle {cycle} {k}")


def config(flux):
    return T.make_config(flow="ns", volume_flux=flux, surface_flux=flux, fv_flux=flux, blending=True,
                         **PHYS)


@pytest.mark.parametrize("flux", ["hll", "roe"])
def test_oracle_reproduces_reference_cavity_trajectory(flux):
    m, u = cavity()
    om = oracle_mesh(m)
    cfg = config(flux)
    u10 = O.rk3_steps(om, cfg, u, 1e-4, 10, nthreads=4)
    compare(m, u10, flux, 10)
    u20 = O.rk3_steps(om, cfg, u10, 1e-4, 10, nthreads=4)
    compare(m, u20, flux, 20)


@pytest.mark.gpu
@pytest.mark.parametrize("flux", ["hll", "roe"])
def test_gpu_reproduces_reference_cavity_trajectory(cuda, flux):
    import torch
    m, u = cavity()
    op = T.NSOperator(m, numerical_flux=flux, surface_flux=flux, fv_flux=flux, blending=True, **PHYS)
    ud = torch.as_tensor(u, device="cuda").contiguous()
    op.rk3_steps(ud, 1e-4, 10)
    compare(m, ud.cpu().numpy(), flux, 10)
    op.rk3_steps(ud, 1e-4, 10)
    compare(m, ud.cpu().numpy(), flux, 20)
    assert op.read_status() == 0


LONG = dict(name="ldc_p3_4000.npz", tol=1e-12)


def test_oracle_reproduces_reference_cavity_after_4000_steps():
    m, u = cavity(order=3)
    u4000 = O.rk3_steps(oracle_mesh(m), config("chandrashekar"), u, 1e-4, 4000, nthreads=O.max_threads())
    compare(m, u4000, "chandrashekar", 4000, **LONG)


@pytest.mark.gpu
def test_gpu_reproduces_reference_cavity_after_4000_steps(cuda):
    import torch
    m, u = cavity(order=3)
    f = "chandrashekar"
    op = T.NSOperator(m, numerical_flux=f, surface_flux=f, fv_flux=f, blending=True, **PHYS)
    ud = torch.as_tensor(u, device="cuda").contiguous()
    op.rk3_steps(ud, 1e-4, 4000)
    compare(m, ud.cpu().numpy(), f, 4000, **LONG)
    assert op.read_status() == 0
