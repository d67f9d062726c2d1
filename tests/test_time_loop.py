"""The reference's clocked time loop (src/Simulation.cpp:1150-1335 with
include/TimeStepControl.hpp and include/RunControl.hpp) as the library runs
it: the host bookkeeping (thx_time_loop_begin/end, the code the device loop
runs) against the oracle's restatement on scripted rate sequences, the
reference's own time-step-control and step-limit cases, and on the GPU the
device loop (thx_rk3_time_loop) against a host-driven loop of fixed steps and
against the oracle's loop."""
import math

import numpy as np
import pytest

import oracle as O
import theseus_b200 as T
from theseus_b200.timeloop import TimeLoop, limit_time_step_to_events, step_limit_reached, time_event_reached
from _helpers import box, oracle_mesh, rel_l2, smooth_state


# tests/time_step_control_tests.cpp and tests/checkpoint_config_tests.cpp:172-175
def test_fixed_step_is_unchanged_without_an_earlier_event():
    assert limit_time_step_to_events(0.1, 1.0, [2.0, math.inf]) == 0.1


def test_fixed_step_lands_on_the_next_time_based_event():
    assert abs(limit_time_step_to_events(0.1, 1.0, [1.04, 1.08]) - 0.04) <= 1e-14


def test_an_event_at_the_current_time_does_not_create_a_zero_step():
    assert limit_time_step_to_events(0.1, 1.0, [1.0, 1.2]) == 0.1


def test_event_detection_tolerates_roundoff_at_the_target_time():
    assert time_event_reached(0.3, 0.1 + 0.2)


def test_step_limit():
    assert not step_limit_reached(1, -1)
    assert not step_limit_reached(199, 200)
    assert step_limit_reached(200, 200) and step_limit_reached(201, 200)


def test_defaults_are_the_reference_runtime_defaults():
    L = TimeLoop()
    assert L.max_dt_growth == 1.2 and L.output_dt == 0.01 and L.refine_time == 2.0
    assert L.output_cycles == 100 and L.max_cycles == -1 and L.done == 0
    assert math.isinf(L.next_output) and math.isinf(L.next_checkpoint) and math.isinf(L.t_final)


def test_record_layout_matches_the_c_header(tmp_path):
    """The ctypes record and the C struct agree in size and field offsets."""
    import ctypes
    import os
    import subprocess
    from theseus_b200.timeloop import TimeLoopC
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    names = [n for n, _ in TimeLoopC._fields_]
    src = tmp_path / "layout.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "theseus_b200.h"\nint main(void) {\n'
                   '  printf("%zu", sizeof(thx_time_loop));\n' +
                   "".join(f'  printf(" %zu", offsetof(thx_time_loop, {n}));\n' for n in names) +
                   "  return 0;\n}\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(root, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert got[0] == ctypes.sizeof(TimeLoopC)
    assert got[1:] == [getattr(TimeLoopC, n).offset for n in names]


def test_record_fields_are_set_on_the_record():
    L = TimeLoop(t_final=1.0)
    L.dt = 0.25
    L.max_cycles = 3
    assert L.c.dt == 0.25 and L.c.max_cycles == 3 and "dt" not in L.__dict__
    assert [L.begin() for _ in range(1)] == [0.25]


def host_driver(loop, rates, cfl, step_state=0.0):
    """Drive the library's host bookkeeping with scripted total rates."""
    if cfl > 0 and loop.dt <= 0:
        loop.dt = cfl / rates(0)
    taken = []
    while not loop.done:
        h = loop.begin()
        taken.append(h)
        loop.end(h, rates(loop.cycle + 1) if cfl > 0 else 0.0, cfl)
    return taken


CASES = [
    # fixed step landing on outputs and the final time
    dict(cfl=0.0, dt=0.001, t_final=0.0375, max_cycles=-1, output_dt=0.01),
    # fixed step stopped by the cycle limit, output every 7 cycles as well
    dict(cfl=0.0, dt=0.003, t_final=2.0, max_cycles=40, output_dt=0.025, output_cycles=7),
    # variable step with the growth limit, refined outputs after refine_time
    dict(cfl=0.3, dt=None, t_final=0.9, max_cycles=-1, output_dt=0.05, refined_output_dt=0.02,
         refine_time=0.4),
    # variable step, no outputs
    dict(cfl=0.5, dt=None, t_final=0.31, max_cycles=-1, output_dt=None),
]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_host_bookkeeping_equals_the_oracle_loop(case):
    kw = dict(CASES[case])
    cfl, dt = kw.pop("cfl"), kw.pop("dt")
    rng = np.random.default_rng(case)
    table = 20.0 + 15.0 * rng.random(100000)

    def rates(cycle):
        return float(table[cycle])
    counter = {"n": 0}

    def total(_u):                                    # the oracle asks once per cycle, in order
        r = rates(counter["n"])
        counter["n"] += 1
        return r
    _, t, taken, cycles, outputs = O.time_loop_driver(0.0, lambda u, h: u, total, cfl, dt=dt, **kw)
    loop = TimeLoop(t_final=kw["t_final"], dt=dt, max_cycles=kw["max_cycles"], output_dt=kw["output_dt"],
                    refined_output_dt=kw.get("refined_output_dt"), refine_time=kw.get("refine_time", 2.0),
                    output_cycles=kw.get("output_cycles", 100))
    mine = host_driver(loop, rates, cfl)
    assert mine == taken
    assert loop.t == t and loop.cycle == cycles and loop.outputs == outputs and loop.done == 1
    assert loop.begin() == 0.0                        # a finished loop takes no further step


def test_checkpoint_events_land_like_outputs():
    L = TimeLoop(t_final=0.05, dt=0.004, checkpoint_dt=0.01)
    taken = host_driver(L, None, 0.0)
    assert L.checkpoints == 5 and abs(L.t - 0.05) <= 1e-15
    assert any(abs(h - 0.002) < 1e-12 for h in taken)  # 0.008 -> 0.010 is shortened


# ---------------------------------------------------------------------------
# GPU: the device loop

def make(flow="euler", precision="fp64"):
    m = box(2, 3, (6, 5))
    u = smooth_state(m, seed=5)
    kw = dict(numerical_flux="ranocha", surface_flux="hll", precision=precision)
    if flow == "ns":
        return m, u, T.NSOperator(m, mu=0.01, Pr=0.72, **kw)
    return m, u, T.EulerOperator(m, **kw)


@pytest.mark.gpu
@pytest.mark.parametrize("flow,cfl", [("euler", 0.0), ("euler", 0.3), ("ns", 0.3)])
def test_device_loop_equals_host_driven_loop(cuda, flow, cfl):
    """Bit for bit: the device loop and a host loop of fixed-step calls
    driven by the same bookkeeping on the host."""
    import torch
    m, u, op = make(flow)
    kw = dict(t_final=0.0123, max_cycles=-1, output_dt=0.002, dt=(None if cfl > 0 else 3e-4))
    a = torch.as_tensor(u, device="cuda").contiguous()
    b = a.clone()
    dev_loop = TimeLoop(**kw)
    dts = op.run_time_loop(a, dev_loop, 200, cfl=cfl)
    host = TimeLoop(**kw)
    if cfl > 0:
        r = op.EstimateStability(b)
        host.dt = cfl / (max(r[0], r[1]) + r[2])
    taken = []
    while not host.done:
        h = host.begin()
        taken.append(h)
        op.rk3_steps(b, h, 1)
        r = op.EstimateStability(b) if cfl > 0 else (0.0, 0.0, 0.0)
        host.end(h, max(r[0], r[1]) + r[2], cfl)
    torch.cuda.synchronize()
    d = dts.cpu().numpy()
    assert np.array_equal(d[:len(taken)], np.array(taken)) and np.all(d[len(taken):] == 0.0)
    assert torch.equal(a, b)                          # cycles after done left the state alone
    assert dev_loop.t == host.t and dev_loop.cycle == host.cycle and dev_loop.outputs == host.outputs
    assert dev_loop.done == 1 and op.read_status() == 0


@pytest.mark.gpu
def test_device_loop_matches_oracle_loop(cuda):
    import torch
    m, u, op = make("ns")
    a = torch.as_tensor(u, device="cuda").contiguous()
    loop = TimeLoop(t_final=0.01, output_dt=0.003)
    op.run_time_loop(a, loop, 100, cfl=0.4)
    cfg = T.make_config(flow="ns", volume_flux="ranocha", surface_flux="hll", mu=0.01, Pr=0.72)
    v, t, taken, cycles, outputs = O.time_loop(oracle_mesh(m), cfg, u, 0.4, 0.01, -1, output_dt=0.003)
    assert loop.cycle == cycles and loop.outputs == outputs
    assert abs(loop.t - t) <= 1e-15
    assert rel_l2(a.cpu().numpy(), v).max() <= 1e-12


@pytest.mark.gpu
def test_device_loop_replays_from_a_captured_graph(cuda):
    """The record lives on the device, so a captured chunk of cycles replays
    and continues the same loop."""
    import torch
    m, u, op = make("euler")
    ref = torch.as_tensor(u, device="cuda").contiguous()
    full = TimeLoop(t_final=1.0, output_dt=0.004, max_cycles=6)
    op.run_time_loop(ref, full, 6, cfl=0.3)
    x = torch.as_tensor(u, device="cuda").contiguous()
    op.run_time_loop(x.clone(), TimeLoop(t_final=1.0), 1, cfl=0.3)    # allocates the stage buffer
    rec = TimeLoop(t_final=1.0, output_dt=0.004, max_cycles=6).to_device("cuda")
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    start = rec.clone()
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            op._graph_dts = op.run_time_loop(x, rec, 2, cfl=0.3, stream=s)
    torch.cuda.synchronize()
    x.copy_(torch.as_tensor(u, device="cuda"))
    rec.copy_(start)
    for _ in range(3):
        g.replay()
    torch.cuda.synchronize()
    back = TimeLoop().load(rec)
    assert torch.equal(x, ref)
    assert back.t == full.t and back.cycle == 6 and back.done == 1 and back.outputs == full.outputs


@pytest.mark.gpu
def test_fp32_mixed_device_loop_tracks_fp64(cuda):
    import torch
    m, u, op64 = make("euler")
    _, _, op32 = make("euler", "fp32")
    a = torch.as_tensor(u, device="cuda").contiguous()
    b = a.clone()
    l64, l32 = TimeLoop(t_final=0.02, output_dt=0.005), TimeLoop(t_final=0.02, output_dt=0.005)
    op64.run_time_loop(a, l64, 100, cfl=0.3)
    op32.run_time_loop(b, l32, 100, cfl=0.3)
    assert l32.done == 1 and abs(l32.t - 0.02) <= 1e-15 and abs(l32.cycle - l64.cycle) <= 1
    assert rel_l2(b.cpu().numpy(), a.cpu().numpy()).max() <= 1e-5
