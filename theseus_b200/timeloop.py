"""The reference's clocked time loop (src/Simulation.cpp:1150-1335,
include/TimeStepControl.hpp, include/RunControl.hpp) as a thx_time_loop record.

TimeLoop holds the record on the host; RHSOperator.run_time_loop advances it
on the device (thx_rk3_time_loop), where each cycle takes the nominal step
shortened to the next event, one SSP-RK3 step, and -- with cfl > 0 -- the next
nominal step min(cfl / TotalRate, max_dt_growth * dt).  begin/end run the same
bookkeeping on the host record (no GPU), for hosts that drive the steps
themselves.
"""
import ctypes as C
import math

import numpy as np


class TimeLoopC(C.Structure):
    _fields_ = [("t", C.c_double), ("dt", C.c_double), ("t_final", C.c_double),
                ("max_dt_growth", C.c_double), ("next_output", C.c_double), ("output_dt", C.c_double),
                ("refined_output_dt", C.c_double), ("refine_time", C.c_double),
                ("next_checkpoint", C.c_double), ("checkpoint_dt", C.c_double), ("last_dt", C.c_double),
                ("cycle", C.c_int64), ("max_cycles", C.c_int64), ("output_cycles", C.c_int64),
                ("outputs", C.c_int64), ("checkpoints", C.c_int64), ("done", C.c_int32),
                ("reserved", C.c_int32)]


def _lib():
    from . import library
    lib = library()
    if not getattr(lib, "_time_bound", False):
        P = C.POINTER(TimeLoopC)
        lib.thx_time_loop_defaults.argtypes = [P]
        lib.thx_time_loop_defaults.restype = None
        lib.thx_time_event_reached.argtypes = [C.c_double, C.c_double]
        lib.thx_limit_time_step_to_events.argtypes = [C.c_double, C.c_double, C.POINTER(C.c_double), C.c_int]
        lib.thx_limit_time_step_to_events.restype = C.c_double
        lib.thx_step_limit_reached.argtypes = [C.c_int64, C.c_int64]
        lib.thx_time_loop_begin.argtypes = [P]
        lib.thx_time_loop_begin.restype = C.c_double
        lib.thx_time_loop_end.argtypes = [P, C.c_double, C.c_double, C.c_double]
        lib.thx_time_loop_end.restype = None
        lib.thx_rk3_time_loop.argtypes = [C.c_void_p, C.c_void_p, C.c_double, C.c_int, C.c_void_p,
                                          C.c_void_p, C.c_void_p]
        lib._time_bound = True
    return lib


def time_event_reached(t, event_time):
    """TimeEventReached (include/TimeStepControl.hpp:21-25)."""
    return bool(_lib().thx_time_event_reached(float(t), float(event_time)))


def limit_time_step_to_events(step, t, events):
    """LimitTimeStepToEvents (include/TimeStepControl.hpp:42-49)."""
    ev = (C.c_double * max(1, len(events)))(*[float(e) for e in events])
    return _lib().thx_limit_time_step_to_events(float(step), float(t), ev, len(events))


def step_limit_reached(cycle, max_cycles):
    """StepLimitReached (include/RunControl.hpp:11-14)."""
    return bool(_lib().thx_step_limit_reached(int(cycle), int(max_cycles)))


class TimeLoop:
    """A thx_time_loop record with the reference's runTime defaults.

    t_final: final_time; dt: the fixed step, or with cfl > 0 the first nominal
    step (None: cfl / TotalRate of the initial state); max_cycles: nsteps_max
    (None: no limit); output_dt: initial_save_dt, None when output is off
    (visualize false); checkpoint_dt: None when checkpoints are off."""

    def __init__(self, t_final=math.inf, dt=None, max_cycles=None, output_dt=None, refined_output_dt=None,
                 refine_time=2.0, output_cycles=100, checkpoint_dt=None, max_dt_growth=1.2, t=0.0):
        c = TimeLoopC()
        _lib().thx_time_loop_defaults(C.byref(c))
        c.t, c.t_final, c.max_dt_growth = float(t), float(t_final), float(max_dt_growth)
        c.dt = 0.0 if dt is None else float(dt)
        c.max_cycles = -1 if max_cycles is None else int(max_cycles)
        if output_dt is not None:
            c.output_dt = float(output_dt)
            c.refined_output_dt = float(output_dt if refined_output_dt is None else refined_output_dt)
            c.next_output = c.t + c.output_dt
        c.refine_time, c.output_cycles = float(refine_time), int(output_cycles)
        if checkpoint_dt is not None:
            c.checkpoint_dt = float(checkpoint_dt)
            c.next_checkpoint = c.t + c.checkpoint_dt
        self.c = c

    def __getattr__(self, name):
        c = self.__dict__.get("c")
        if c is not None and name in dict(TimeLoopC._fields_):
            return getattr(c, name)
        raise AttributeError(name)

    def __setattr__(self, name, value):
        if name != "c" and name in dict(TimeLoopC._fields_):
            setattr(self.c, name, value)       # a record field, not a Python attribute
        else:
            object.__setattr__(self, name, value)

    def begin(self):
        """The step of the next cycle (0 once done), on the host record."""
        return _lib().thx_time_loop_begin(C.byref(self.c))

    def end(self, dt_taken, total_rate=0.0, cfl=0.0):
        """Close a cycle on the host record (total_rate of the new state when cfl > 0)."""
        _lib().thx_time_loop_end(C.byref(self.c), float(dt_taken), float(total_rate), float(cfl))

    def to_device(self, device):
        """The record as a device byte tensor (what thx_rk3_time_loop advances)."""
        import torch
        raw = np.frombuffer(bytes(self.c), dtype=np.uint8).copy()
        return torch.from_numpy(raw).to(device)

    def load(self, dev):
        """Read a device record back into this object."""
        raw = dev.cpu().numpy().tobytes()
        self.c = TimeLoopC.from_buffer_copy(raw)
        return self
