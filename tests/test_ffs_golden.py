"""The reference's recorded Mach 3 forward-facing step after 100 cycles
(TestCases/GoldenData/ForwardFacingStep.tgz: its run of
TestCases/Euler/2D/ForwardFacingStep/config.json through
tests/recipes/regression/golden-step.sh -- the Gmsh mesh refined once,
p=3, Chandrashekar fluxes, subcell FV blending, supersonic inflow on the
left, supersonic outflow on the right, slip walls, fixed dt 1e-4, 100 cycles),
reproduced on the same mesh (read and refined by theseus_b200.gmsh) through
the oracle's loop (CPU) and the device time loop (GPU) within the recipe's
tolerances (atol 3e-13, rtol 1e-13).  The golden's blending coefficient is
the one of the last right-hand side (the third stage of the last cycle).
Fixture: tests/golden/ffs/ffs_p3_100.npz (the mesh and a subset of the
golden's elements: every blended one and every 32nd other one), made by
tests/golden/ffs/make_ffs_fixture.py."""
import os

import numpy as np
import pytest

import oracle as O
import theseus_b200 as T
from theseus_b200.gmsh import quad_mesh_from
from theseus_b200.timeloop import TimeLoop
from _helpers import oracle_mesh

HERE = os.path.dirname(os.path.abspath(__file__))
GAMMA = 1.4
# ForwardFacingStepLeftBCVector and ForwardFacingStepIC (x1 = 2.5), include/StateInit.hpp:805-819
INFLOW = [1.4, 1.4 * 3.0, 0.0, 1.0 / (1.4 - 1.0) + 0.5 * 1.4 * 3.0 * 3.0]
INITIAL = [1.4, 1.4 * 3.0, 0.0, 1.0 * 2.5 + 0.5 * 1.4 * 3.0 * 3.0]
BOUNDARY = {"left": ("supersonic-inflow", INFLOW), "bottom": "slip", "top": "slip",
            "right": "supersonic-outflow"}
LOOP = dict(t_final=3.0, max_cycles=100, output_dt=0.01)


def fixture():
    return np.load(os.path.join(HERE, "golden", "ffs", "ffs_p3_100.npz"))


def mesh_and_state(g):
    nodes = {int(i): tuple(xy) for i, xy in zip(g["node_id"], g["node_xy"])}
    quads = [(0, *map(int, q)) for q in g["quads"]]
    names = [str(n) for n in g["line_names"]]
    lines = [(names[k], int(a), int(b)) for k, a, b in g["lines"]]
    m = quad_mesh_from((nodes, quads, lines, {}), 3, BOUNDARY, refinements=1)
    u = np.empty((4,) + m.coords[0].shape)
    for k in range(4):
        u[k] = INITIAL[k]
    return m, u


def golden_index(m, g):
    x, y = m.coords
    centres = np.stack([x.mean(axis=1), y.mean(axis=1)], axis=1)
    index = {tuple(np.round(c, 9)): e for e, c in enumerate(centres)}
    e = np.array([index[tuple(np.round(c, 9))] for c in g["center"]])
    pt = g["point"]
    d2 = (x[e] - pt[:, :1]) ** 2 + (y[e] - pt[:, 1:2]) ** 2
    node = d2.argmin(axis=1)
    assert np.all(d2[np.arange(len(e)), node] < 1e-24)
    return e, node


def compare(m, u, alpha, g):
    e, node = golden_index(m, g)
    rho = u[0][e, node]
    vel = (u[1:3] / u[0])[:, e, node].T
    p = ((GAMMA - 1.0) * (u[3] - 0.5 * (u[1] ** 2 + u[2] ** 2) / u[0]))[e, node]
    for k, a in (("density", rho), ("pressure", p), ("velocity", vel)):
        np.testing.assert_allclose(a, g[k], rtol=1e-13, atol=3e-13, err_msg=k)
    np.testing.assert_allclose(alpha[e], g["blending"], rtol=0, atol=1e-12, err_msg="blending")
    assert np.count_nonzero(g["blending"]) > 0


def config():
    f = "chandrashekar"
    return T.make_config(flow="euler", volume_flux=f, surface_flux=f, fv_flux=f, blending=True, gamma=GAMMA)


def test_refined_gmsh_mesh():
    g = fixture()
    m, _ = mesh_and_state(g)
    assert m.num_elements == 4 * len(g["quads"]) == int(g["num_golden_elements"])
    assert m.boundary.num_faces == 2 * len(g["lines"]) and np.all(m.jac > 0)


def test_oracle_reproduces_reference_forward_facing_step():
    g = fixture()
    m, u = mesh_and_state(g)
    om, cfg, nt = oracle_mesh(m), config(), O.max_threads()
    v99, _, taken, cycles, _ = O.time_loop(om, cfg, u, 0.0, dt=1e-4, nthreads=nt, **dict(LOOP, max_cycles=99))
    # the last cycle by hand, keeping the state its third stage sees
    h = O.limit_time_step_to_events(1e-4, sum(taken), (3.0, 0.01))
    k1 = O.rhs(om, cfg, v99, nthreads=nt)
    y1 = v99 + h * k1
    k2 = O.rhs(om, cfg, y1, nthreads=nt)
    y2 = 0.75 * v99 + 0.25 * (y1 + h * k2)
    alpha, _ = O.blending(om, cfg, y2)
    v = O.rk3_steps(om, cfg, v99, h, 1, nthreads=nt)
    compare(m, v, alpha, g)


@pytest.mark.gpu
def test_gpu_time_loop_reproduces_reference_forward_facing_step(cuda):
    import torch
    g = fixture()
    m, u = mesh_and_state(g)
    f = "chandrashekar"
    op = T.EulerOperator(m, numerical_flux=f, surface_flux=f, fv_flux=f, blending=True, gamma=GAMMA)
    ud = torch.as_tensor(u, device="cuda").contiguous()
    loop = TimeLoop(dt=1e-4, **LOOP)
    op.run_time_loop(ud, loop, 100)
    assert loop.done == 1 and loop.cycle == 100
    alpha, _ = op.blending_coefficients()
    compare(m, ud.cpu().numpy(), alpha.cpu().numpy(), g)
    assert op.read_status() == 0
