"""Checkpoint interchange in the reference's restart format.

A state saved here restarts a reference run, and a reference checkpoint
restarts a run here: the per-rank state file is
``Cycle<c>/checkpoint_cycle_<c>.<rank:08d>.chk`` ("THESEUS_CHECKPOINT_RAW_V1\\n",
a uint64 count, the raw FP64 byNODES state vector) and the cycle's metadata
``Cycle<c>/checkpoint_cycle_<c>.json`` (src/Simulation.cpp:1477-1603,
include/CheckpointConfig.hpp).  Files are written and read by the library
(thx_checkpoint_*); this module mirrors CheckpointConfig and
CheckpointCompatibility and raises ValueError with the reference's messages.
"""
import ctypes as C
import json
import os
from dataclasses import dataclass

import numpy as np

from ._abi import THX_OK

THX_ERR_UNSUPPORTED = 2
THX_ERR_IO = 8


class CheckpointCompatibilityC(C.Structure):
    _fields_ = [("mpi_ranks", C.c_int32), ("order", C.c_int32), ("dimension", C.c_int32),
                ("num_equations", C.c_int32), ("real_bytes", C.c_int32), ("axisymmetric", C.c_int32),
                ("global_elements", C.c_int64), ("global_dofs", C.c_int64)]


@dataclass
class CheckpointCompatibility:
    """CheckpointCompatibility (include/CheckpointConfig.hpp:19-29)."""
    mpi_ranks: int
    order: int
    dimension: int
    num_equations: int
    real_bytes: int
    global_elements: int
    global_dofs: int
    axisymmetric: bool = False

    @classmethod
    def of_mesh(cls, mesh, mpi_ranks=1):
        """The record of a state on `mesh` (global_dofs = equations x nodes,
        the state-vector length)."""
        return cls(mpi_ranks, mesh.order, mesh.dim, mesh.neq, 8, mesh.num_elements,
                   mesh.neq * mesh.num_nodes, False)

    def _c(self):
        return CheckpointCompatibilityC(self.mpi_ranks, self.order, self.dimension, self.num_equations,
                                        self.real_bytes, 1 if self.axisymmetric else 0,
                                        self.global_elements, self.global_dofs)


def _lib():
    from . import library
    lib = library()
    if not getattr(lib, "_checkpoint_bound", False):
        P = C.POINTER(CheckpointCompatibilityC)
        lib.thx_checkpoint_metadata.argtypes = [C.c_double, C.c_int, P, C.c_char_p, C.c_size_t]
        lib.thx_checkpoint_validate.argtypes = [C.c_char_p, P, C.POINTER(C.c_int), C.c_char_p, C.c_size_t]
        lib.thx_checkpoint_save.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_double, P, C.c_void_p,
                                            C.c_int64, C.c_int, C.c_char_p, C.c_size_t]
        lib.thx_checkpoint_load.argtypes = [C.c_char_p, C.c_int, C.c_int, P, C.POINTER(C.c_double),
                                            C.c_void_p, C.c_int64, C.c_char_p, C.c_size_t]
        lib._checkpoint_bound = True
    return lib


def _raise(st, msg, what):
    text = msg.value.decode(errors="replace") or what
    if st == THX_ERR_IO:
        raise OSError(text)
    if st == THX_ERR_UNSUPPORTED:
        raise NotImplementedError(text)
    raise ValueError(text)


class CheckpointConfig:
    """CheckpointConfig (include/CheckpointConfig.hpp:31-92): the runTime
    checkpoint keys and the paths they name."""

    def __init__(self, load=False, save=False, cycle=0, interval=0.01, directory="Checkpoints"):
        self.load, self.save, self.cycle, self.interval = load, save, cycle, interval
        self.directory = directory

    @classmethod
    def from_runtime(cls, runtime, output_directory):
        r = dict(runtime)
        cfg = cls(bool(r.get("checkpoint_load", False)), bool(r.get("checkpoint_save", False)),
                  int(r.get("checkpoint_cycle", 0)), float(r.get("checkpoint_dt", 0.01)))
        folder = r.get("checkpoints_folder", "Checkpoints")
        if not folder:
            raise ValueError("runTime.checkpoints_folder must not be empty")
        cfg.directory = os.path.join(output_directory, folder)
        if (cfg.load or cfg.save) and cfg.interval <= 0.0:
            raise ValueError("runTime.checkpoint_dt must be greater than zero")
        if cfg.load and cfg.cycle <= 0:
            raise ValueError("runTime.checkpoint_cycle must be greater than zero when checkpoint_load is true")
        return cfg

    def cycle_directory(self, cycle):
        return os.path.join(self.directory, f"Cycle{cycle}")

    def metadata_file(self, cycle):
        return os.path.join(self.cycle_directory(cycle), f"checkpoint_cycle_{cycle}.json")

    def rank_file(self, cycle, rank):
        return os.path.join(self.cycle_directory(cycle), f"checkpoint_cycle_{cycle}.{rank:08d}.chk")

    @staticmethod
    def metadata(time, cycle, compat):
        """CheckpointConfig::Metadata as a dict (the library's JSON text parsed)."""
        buf = C.create_string_buffer(4096)
        c = compat._c()
        st = _lib().thx_checkpoint_metadata(float(time), int(cycle), C.byref(c), buf, len(buf))
        if st != THX_OK:
            raise ValueError("thx_checkpoint_metadata failed")
        return json.loads(buf.value.decode())

    @staticmethod
    def validate_metadata(metadata, expected):
        """CheckpointConfig::ValidateMetadata: True for current metadata, False
        for legacy (time and cycle only); ValueError when incompatible."""
        text = metadata if isinstance(metadata, str) else json.dumps(metadata)
        cur = C.c_int(0)
        msg = C.create_string_buffer(512)
        c = expected._c()
        st = _lib().thx_checkpoint_validate(text.encode(), C.byref(c), C.byref(cur), msg, len(msg))
        if st != THX_OK:
            _raise(st, msg, "invalid checkpoint metadata")
        return bool(cur.value)


def save_checkpoint(directory, cycle, state, time, compat, rank=0, write_metadata=True):
    """Simulation::SaveCheckpoint for one rank.  `state` is the FP64 L-vector
    (numpy array or CUDA tensor, copied to the host)."""
    if hasattr(state, "detach"):
        state = state.detach().cpu().numpy()
    a = np.ascontiguousarray(state, dtype=np.float64).reshape(-1)
    msg = C.create_string_buffer(512)
    c = compat._c()
    st = _lib().thx_checkpoint_save(os.fsencode(directory), int(cycle), int(rank), float(time), C.byref(c),
                                    a.ctypes.data_as(C.c_void_p), a.size, 1 if write_metadata else 0,
                                    msg, len(msg))
    if st != THX_OK:
        _raise(st, msg, "thx_checkpoint_save failed")


def load_checkpoint(directory, cycle, expected, rank=0, shape=None):
    """Simulation::LoadCheckpoint for one rank: (time, state) with the state
    as a host FP64 array of expected.global_dofs // expected.mpi_ranks entries
    (or `shape`)."""
    n = int(np.prod(shape)) if shape is not None else expected.global_dofs // max(1, expected.mpi_ranks)
    out = np.empty(n, dtype=np.float64)
    t = C.c_double(0.0)
    msg = C.create_string_buffer(512)
    c = expected._c()
    st = _lib().thx_checkpoint_load(os.fsencode(directory), int(cycle), int(rank), C.byref(c), C.byref(t),
                                    out.ctypes.data_as(C.c_void_p), n, msg, len(msg))
    if st != THX_OK:
        _raise(st, msg, "thx_checkpoint_load failed")
    return t.value, (out.reshape(shape) if shape is not None else out)
