"""The reference's recorded isentropic vortex after 500 cycles
(TestCases/GoldenData/IsentropicVortex/Cycle000500: its CPU run of
TestCases/Euler/2D/IsentropicVortex/config.json through
tests/recipes/regression/golden-vortex.sh -- IsentropicVortex.mesh refined
three times, p=3, Chandrashekar fluxes, blending compiled in, fixed dt 1e-3
shortened to land on the 0.01 output times, 500 cycles), reproduced on the
same mesh (read and refined by theseus_b200.mfem_mesh) through the oracle's
loop (CPU) and the device time loop (GPU), within the recipe's tolerances
(rtol = atol = 1e-13).  Fixture: tests/golden/vortex/vortex_p3_500.npz, made
by tests/golden/vortex/make_vortex_fixture.py."""
import math
import os

import numpy as np
import pytest

import oracle as O
import theseus_b200 as T
from theseus_b200.mfem_mesh import mfem_quad_mesh, mfem_quad_mesh_from
from theseus_b200.timeloop import TimeLoop
from _helpers import oracle_mesh

HERE = os.path.dirname(os.path.abspath(__file__))
R_GAS, GAMMA = 287.05, 1.4
RADIUS, MINF, BETA = 0.2, 0.5, 0.2
LOOP = dict(t_final=2.0, max_cycles=500, output_dt=0.01, output_cycles=1000)


def fixture():
    return np.load(os.path.join(HERE, "golden", "vortex", "vortex_p3_500.npz"))


def vortex(x, y):
    """IsentropicVortexIC (include/StateInit.hpp:392-437) at one point, in
    its order of operations (libm exp and pow)."""
    pres_inf = (1.0 / GAMMA) * (1.0 / MINF) * (1.0 / MINF)
    temp_inf = pres_inf / (1.0 * R_GAS)
    r2 = 0.0
    r2 += (x - 0.0) * (x - 0.0)
    r2 += (y - 0.0) * (y - 0.0)
    r2 /= RADIUS * RADIUS
    s1 = 1.0 / (GAMMA - 1.0)
    vx = 1.0 * (1 - BETA * (y - 0.0) / RADIUS * math.exp(-0.5 * r2))
    vy = 1.0 * BETA * (x - 0.0) / RADIUS * math.exp(-0.5 * r2)
    v2 = vx * vx + vy * vy
    cp = R_GAS * GAMMA * s1
    temp = temp_inf - 0.5 * (1.0 * BETA) * (1.0 * BETA) / cp * math.exp(-r2)
    den = 1.0 * math.pow(temp / temp_inf, s1)
    pres = den * R_GAS * temp
    energy = s1 * pres / den + 0.5 * v2
    return den, den * vx, den * vy, den * energy


def mesh_and_state(g):
    elems = [tuple(int(v) for v in e) for e in g["elements"]]
    m = mfem_quad_mesh_from((2, elems, [], int(g["num_vertices"]), g["dofs"]), 3, refinements=3)
    x, y = m.coords
    u = np.zeros((4,) + x.shape)
    for e in range(x.shape[0]):
        for n in range(x.shape[1]):
            u[:, e, n] = vortex(x[e, n], y[e, n])
    return m, u


def compare(m, u, g):
    x, y = m.coords
    centres = np.stack([x.mean(axis=1), y.mean(axis=1)], axis=1)
    index = {tuple(np.round(c, 6)): e for e, c in enumerate(centres)}
    e = np.array([index[tuple(np.round(c, 6))] for c in g["center"]])
    pt = g["point"]
    d2 = (x[e] - pt[:, :1]) ** 2 + (y[e] - pt[:, 1:2]) ** 2
    node = d2.argmin(axis=1)
    assert np.all(d2[np.arange(len(e)), node] < 1e-24)
    rho = u[0][e, node]
    vel = (u[1:3] / u[0])[:, e, node].T
    p = ((GAMMA - 1.0) * (u[3] - 0.5 * (u[1] ** 2 + u[2] ** 2) / u[0]))[e, node]
    for k, a in (("density", rho), ("pressure", p), ("velocity", vel)):
        np.testing.assert_allclose(a, g[k], rtol=1e-13, atol=1e-13, err_msg=k)


def config():
    f = "chandrashekar"
    return T.make_config(flow="euler", volume_flux=f, surface_flux=f, fv_flux=f, blending=True,
                         R_gas=R_GAS, gamma=GAMMA)


def test_refined_mfem_mesh_is_periodic_and_conforming():
    g = fixture()
    m, u = mesh_and_state(g)
    assert m.num_elements == 576 and m.num_faces == 1152 and m.boundary is None
    assert np.all(m.jac > 0)
    x, y = m.coords
    assert x.min() == -1.0 and x.max() == 1.0 and y.min() == -1.0 and y.max() == 1.0


def test_oracle_reproduces_reference_vortex():
    g = fixture()
    m, u = mesh_and_state(g)
    v, t, taken, cycles, outputs = O.time_loop(oracle_mesh(m), config(), u, 0.0, dt=1e-3,
                                               nthreads=O.max_threads(), **LOOP)
    assert cycles == 500 and abs(t - 0.5) < 1e-12 and outputs == 50
    assert min(taken) < 1e-3                          # steps shortened onto the output times
    compare(m, v, g)


@pytest.mark.gpu
def test_gpu_time_loop_reproduces_reference_vortex(cuda):
    import torch
    g = fixture()
    m, u = mesh_and_state(g)
    f = "chandrashekar"
    op = T.EulerOperator(m, numerical_flux=f, surface_flux=f, fv_flux=f, blending=True, R_gas=R_GAS,
                         gamma=GAMMA)
    ud = torch.as_tensor(u, device="cuda").contiguous()
    loop = TimeLoop(dt=1e-3, **LOOP)
    op.run_time_loop(ud, loop, 500)
    assert loop.done == 1 and loop.cycle == 500 and loop.outputs == 50
    compare(m, ud.cpu().numpy(), g)
    alpha, _ = op.blending_coefficients()
    assert np.array_equal(alpha.cpu().numpy(), np.zeros(m.num_elements)) and np.all(g["blending"] == 0.0)
    assert op.read_status() == 0


MESH = """MFEM mesh v1.0

dimension
2

elements
6
1 3 0 1 5 4
1 3 1 2 6 5
1 3 2 3 7 6
1 3 5 6 10 9
1 3 6 7 11 10
1 3 4 5 9 8

boundary
6
1 1 0 1
1 1 1 2
1 1 2 3
2 1 9 10
2 1 10 11
2 1 8 9

vertices
12
2
0 0
1 0
2 0
3 0
0 1
1 1
2 1
3 1
0 2
1 2
2 2
3 2
"""


def test_mfem_reader_refines_topology_and_boundary(tmp_path):
    """A 3 x 2 mesh with plain vertex coordinates (walls at y = 0 and 2,
    open x sides) refined once: 24 elements, boundary edges split in two
    and named by attribute; the x sides become boundary faces too and must
    be given a condition."""
    path = tmp_path / "m.mesh"
    path.write_text(MESH)
    with pytest.raises(ValueError, match="without a condition"):
        mfem_quad_mesh(str(path), 2, refinements=1, boundary={1: "slip", 2: "slip"})
    text = MESH.replace("boundary\n6\n", "boundary\n10\n")
    text = text.replace("2 1 8 9\n", "2 1 8 9\n3 1 0 4\n3 1 4 8\n3 1 3 7\n3 1 7 11\n")
    path.write_text(text)
    m = mfem_quad_mesh(str(path), 2, refinements=1, boundary={1: "slip", 2: "symmetry", 3: "slip"})
    assert m.num_elements == 24 and np.allclose(m.jac, 0.25)
    b = m.boundary
    assert b.num_faces == 2 * (6 + 4) and m.num_faces == 5 * 4 + 6 * 3
    assert np.allclose(b.normal[b.lface == 2][..., 1], -0.5) and np.allclose(b.normal[b.lface == 3][..., 1], 0.5)
    x, y = m.coords
    assert x.min() == 0.0 and x.max() == 3.0 and y.max() == 2.0
