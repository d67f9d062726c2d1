"""Variable-dt SSP-RK3 with the time step computed on the device
(thx_rk3_steps_cfl): dt = cfl / (max(advective, surface) + diffusive rate)
of each step's initial state, the reference's variable_dt loop
(src/Simulation.cpp:1150-1160, include/RHSOperator_impl.hpp:10-270).
It must equal the host loop estimate_dt + one fixed-dt step, step by step,
agree with the oracle's loop, and replay unchanged from a captured graph."""
import numpy as np
import pytest

import oracle as O
import theseus_b200 as T
from theseus_b200 import cases
from _helpers import box, oracle_mesh, rel_l2, smooth_state


def make(flow, precision="fp64"):
    m = box(2, 3, (6, 5))
    u = smooth_state(m, seed=3)
    kw = dict(numerical_flux="ranocha", surface_flux="hll", precision=precision)
    if flow == "ns":
        return m, u, T.NSOperator(m, mu=0.01, Pr=0.72, **kw)
    return m, u, T.EulerOperator(m, **kw)


@pytest.mark.gpu
@pytest.mark.parametrize("flow,precision", [("euler", "fp64"), ("ns", "fp64"), ("ns", "fp32")])
def test_device_cfl_steps_equal_host_loop(cuda, flow, precision):
    import torch
    m, u, op = make(flow, precision)
    a = torch.as_tensor(u, device="cuda").contiguous()
    b = a.clone()
    dts = op.rk3_steps_cfl(a, 0.4, 6)
    host = []
    for _ in range(6):
        torch.cuda.synchronize()
        dt = op.estimate_dt(b, 0.4)
        host.append(dt)
        op.rk3_steps(b, dt, 1)
    torch.cuda.synchronize()
    assert np.array_equal(dts.cpu().numpy(), np.array(host))
    assert torch.equal(a, b)
    assert op.read_status() == 0


@pytest.mark.gpu
def test_device_cfl_steps_match_oracle(cuda):
    import torch
    m, u, op = make("ns")
    a = torch.as_tensor(u, device="cuda").contiguous()
    op.rk3_steps_cfl(a, 0.4, 5)
    cfg = T.make_config(flow="ns", volume_flux="ranocha", surface_flux="hll", mu=0.01, Pr=0.72)
    om = oracle_mesh(m)
    v = u.copy()
    for _ in range(5):
        dt, _ = O.estimate_dt(om, cfg, v, 0.4)
        v = O.rk3_steps(om, cfg, v, dt, 1)
    assert rel_l2(a.cpu().numpy(), v).max() <= 1e-12


@pytest.mark.gpu
def test_device_cfl_steps_replay_from_a_captured_graph(cuda):
    import torch
    m, u, op = make("euler")
    ref = torch.as_tensor(u, device="cuda").contiguous()
    op.rk3_steps_cfl(ref, 0.4, 4)
    x = torch.as_tensor(u, device="cuda").contiguous()
    op.rk3_steps_cfl(x.clone(), 0.4, 1)        # first call allocates the stage buffer
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            op._dts = op.rk3_steps_cfl(x, 0.4, 2, stream=s)
    torch.cuda.synchronize()
    x.copy_(torch.as_tensor(u, device="cuda"))
    g.replay()
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(x, ref)
