"""Batched serving of many independent DGSEM cases on one GPU.

`BatchEngine` wraps the library's batch engine (C ABI `thx_engine_*`): cases of
any periodic mesh size, polynomial order and flow model are admitted while
others run, their states stay on the device, and every (dimension, order,
flow) group advances by persistent kernels launched from one CUDA graph of
`steps_per_launch` SSP-RK3 steps.

`serve()` is the continuous-batching loop: requests arrive on a schedule
(seconds from the start), are admitted as soon as the engine's memory budget
has room (first come, first served), advance together, and are fetched when
their steps are done.  It returns each case's final state and its
time-to-solution (arrival -> result on the host).

`SyntheticStream` draws the mixed 2-D workload used by the serving benchmark:
periodic square meshes of 8..64 elements per side, p = 2..5, freestream Mach
0.1..2, Reynolds 100..10^4 or inviscid with probability 0.5, an isentropic
vortex of strength 1..5, Poisson arrivals.
"""
import ctypes as C
import time
from dataclasses import dataclass, field

import numpy as np

from . import (library, _check, make_config, Geometry, periodic_box, THXError, FLOW_EULER,
               FLOW_NAVIER_STOKES, PRECISION_FP32_MIXED)
from . import cases as _cases

THX_ERR_BUSY = 7


class CaseDesc(C.Structure):
    _fields_ = [("flow_model", C.c_int32), ("nsteps", C.c_int32), ("dt", C.c_double),
                ("mu", C.c_double), ("Pr", C.c_double), ("state_offset", C.c_double * 5),
                ("geometry_key", C.c_int64)]


class EngineStats(C.Structure):
    _fields_ = [("active_cases", C.c_int32), ("groups", C.c_int32), ("bytes_in_use", C.c_int64),
                ("launches", C.c_int64), ("cases_done", C.c_int64), ("admit_lock_s", C.c_double),
                ("admit_setup_s", C.c_double), ("admit_copy_s", C.c_double),
                ("advance_s", C.c_double), ("fetch_copy_s", C.c_double),
                ("pool_reserved_bytes", C.c_int64), ("pool_used_bytes", C.c_int64),
                ("advance_calls", C.c_int64), ("advance_tables_s", C.c_double),
                ("advance_launch_s", C.c_double), ("table_bytes", C.c_int64),
                ("ring_wait_s", C.c_double), ("ring_copy_s", C.c_double)]


class EngineGroup(C.Structure):
    _fields_ = [("dim", C.c_int32), ("order", C.c_int32), ("navier_stokes", C.c_int32),
                ("active_cases", C.c_int32), ("tuned", C.c_int32), ("volume_grid", C.c_int32),
                ("face_grid", C.c_int32), ("gradient_grid", C.c_int32),
                ("elements_per_block", C.c_int32), ("best_cost_ms", C.c_double)]


def _bind(lib):
    if getattr(lib, "_engine_bound", False):
        return lib
    P = C.c_void_p
    lib.thx_engine_create.argtypes = [C.c_void_p, C.c_size_t, C.c_int, C.POINTER(P)]
    lib.thx_engine_destroy.argtypes = [P]
    lib.thx_engine_admit.argtypes = [P, C.POINTER(Geometry), C.POINTER(CaseDesc), C.c_void_p,
                                     C.POINTER(C.c_int64)]
    lib.thx_engine_advance.argtypes = [P]
    lib.thx_engine_poll.argtypes = [P, C.POINTER(C.c_int64), C.c_int, C.POINTER(C.c_int)]
    lib.thx_engine_fetch.argtypes = [P, C.c_int64, C.c_void_p]
    lib.thx_engine_get_stats.argtypes = [P, C.POINTER(EngineStats)]
    lib.thx_engine_groups.argtypes = [P, C.POINTER(EngineGroup), C.c_int, C.POINTER(C.c_int)]
    lib.thx_case_footprint.argtypes = [C.POINTER(Geometry), C.c_void_p, C.c_int,
                                       C.POINTER(C.c_size_t)]
    lib._engine_bound = True
    return lib


@dataclass
class Case:
    """One request: mesh, initial state (host FP64 L-vector), physics, steps."""
    mesh: object
    u0: np.ndarray
    nsteps: int
    dt: float
    viscous: bool = False
    mu: float = 0.0
    Pr: float = 0.72
    state_offset: tuple = (0.0, 0.0, 0.0, 0.0, 0.0)
    arrival: float = 0.0
    tag: dict = field(default_factory=dict)
    factory: object = None   # builds u0 on first use when u0 is None
    geometry_key: int = 0    # nonzero: cases with the same key share the device geometry

    def state(self):
        if self.u0 is None:
            self.u0 = self.factory()
        return self.u0

    def desc(self):
        off = (C.c_double * 5)(*[float(x) for x in self.state_offset])
        return CaseDesc(FLOW_NAVIER_STOKES if self.viscous else FLOW_EULER, int(self.nsteps),
                        float(self.dt), float(self.mu), float(self.Pr), off, int(self.geometry_key))


class BatchEngine:
    """Mirror of the C ABI batch engine.  `numerical_flux`, `surface_flux`,
    `precision` and the gas constants are shared by all cases."""

    def __init__(self, numerical_flux="chandrashekar", surface_flux="roe", precision="fp32",
                 hbm_budget=None, steps_per_launch=10, device=None, **physics):
        import torch
        if not torch.cuda.is_available():
            raise THXError("no CUDA device: the batch engine has no CPU fallback")
        self.lib = _bind(library())
        self.cfg = make_config(flow="euler", volume_flux=numerical_flux, surface_flux=surface_flux,
                               precision=precision, **physics)
        self.device = torch.device(device) if device is not None else torch.device(
            "cuda", torch.cuda.current_device())
        if hbm_budget is None:
            free, _ = torch.cuda.mem_get_info(self.device)
            hbm_budget = int(0.8 * free)
        self.steps_per_launch = int(steps_per_launch)
        h = C.c_void_p()
        with torch.cuda.device(self.device):
            _check(self.lib.thx_engine_create(C.byref(self.cfg), C.c_size_t(int(hbm_budget)),
                                              self.steps_per_launch, C.byref(h)), "thx_engine_create")
        self._h = h
        self.hbm_budget = int(hbm_budget)

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self.lib.thx_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def footprint(self, case):
        b = C.c_size_t()
        _check(self.lib.thx_case_footprint(C.byref(case.mesh.struct()), C.byref(self.cfg),
                                           FLOW_NAVIER_STOKES if case.viscous else FLOW_EULER,
                                           C.byref(b)), "thx_case_footprint")
        return b.value

    def admit(self, case):
        """Case id, or None when the memory budget has no room now."""
        u0 = np.ascontiguousarray(case.state(), np.float64)
        cid = C.c_int64()
        st = self.lib.thx_engine_admit(self._h, C.byref(case.mesh.struct()), C.byref(case.desc()),
                                       u0.ctypes.data, C.byref(cid))
        if st == THX_ERR_BUSY:
            return None
        _check(st, "thx_engine_admit")
        return cid.value

    def advance(self):
        _check(self.lib.thx_engine_advance(self._h), "thx_engine_advance")

    def poll(self, cap=4096):
        if getattr(self, "_ids", None) is None or len(self._ids) < cap:
            self._ids = (C.c_int64 * cap)()
        n = C.c_int()
        _check(self.lib.thx_engine_poll(self._h, self._ids, cap, C.byref(n)), "thx_engine_poll")
        return [self._ids[i] for i in range(n.value)]

    def fetch(self, cid, shape):
        out = np.empty(shape, np.float64)
        _check(self.lib.thx_engine_fetch(self._h, int(cid), out.ctypes.data), "thx_engine_fetch")
        return out

    def stats(self):
        s = EngineStats()
        _check(self.lib.thx_engine_get_stats(self._h, C.byref(s)), "thx_engine_get_stats")
        return {k: getattr(s, k) for k, _ in EngineStats._fields_}

    def groups(self):
        """Per batch group: dimension, order, flow model, active cases and the
        kernel grids the online tuner has chosen so far (tuned = 1 once the
        volume, face and gradient grids have all been searched)."""
        n = C.c_int()
        _check(self.lib.thx_engine_groups(self._h, None, 0, C.byref(n)), "thx_engine_groups")
        arr = (EngineGroup * max(1, n.value))()
        _check(self.lib.thx_engine_groups(self._h, arr, n.value, C.byref(n)), "thx_engine_groups")
        return [{k: getattr(arr[i], k) for k, _ in EngineGroup._fields_} for i in range(n.value)]


def serve(engine, requests, clock=time.perf_counter, idle_sleep=2e-4, on_result=None, host=None,
          admitters=1):
    """Continuous batching: requests (sorted by .arrival, seconds from start)
    are admitted as they arrive and the budget allows, advanced together, and
    fetched when done.  Returns (results, latencies, makespan): results[i] is
    the final state of requests[i] (None when on_result(i, state) consumed it),
    latencies[i] its arrival-to-result time.  host, if a dict, receives the
    host seconds spent admitting, advancing/polling and fetching.

    Admission (building the initial state, the library's set-up of the case)
    runs on a second host thread in arrival order, first come first served: a
    request that does not fit waits, and the ones behind it with it, until a
    result is fetched.  admitters > 1 spreads the set-up over more threads
    (request i on thread i mod admitters) and gives up the strict order.  The calling thread keeps the GPU
    fed: it advances the running groups and hands finished cases to two
    fetching threads."""
    import threading
    n = len(requests)
    results = [None] * n
    latency = np.zeros(n)
    running = {}               # engine id -> request index
    cv = threading.Condition()
    box = {"admitted": 0, "error": None, "admit_s": 0.0, "state_s": 0.0, "call_s": 0.0}
    t0 = clock()

    # initial states are built ahead of admission by a small thread pool
    # (numpy releases the interpreter lock in its array work)
    from concurrent.futures import ThreadPoolExecutor
    import os
    pool = ThreadPoolExecutor(max_workers=max(1, min(8, (os.cpu_count() or 2) - 2)))
    depth = 64
    admitters = max(1, int(admitters))
    lock = threading.Lock()

    def admitter(k):
        mine = list(range(k, n, admitters))
        futures = {}
        submitted = [0]

        def prefetch(upto):
            while submitted[0] < min(upto, len(mine)):
                j = mine[submitted[0]]
                futures[j] = pool.submit(requests[j].state)
                submitted[0] += 1
        try:
            for pos, i in enumerate(mine):
                r = requests[i]
                prefetch(pos + depth // admitters)
                wait = r.arrival - (clock() - t0)
                if wait > 0:
                    time.sleep(wait)
                ta = clock()
                futures.pop(i).result()
                tb = clock()
                call = 0.0
                while True:
                    tc = clock()
                    cid = engine.admit(r)
                    call += clock() - tc
                    if cid is not None:
                        break
                    with cv:               # no room: wait for a fetch
                        cv.wait(timeout=0.005)
                with cv:
                    running[cid] = i
                    box["admitted"] += 1
                with lock:
                    box["state_s"] += tb - ta
                    box["call_s"] += call
                    box["admit_s"] += clock() - ta
        except Exception as exc:           # surfaced by the serving thread
            box["error"] = exc

    import queue
    fetch_q = queue.Queue()
    queued = set()
    tf = {"s": 0.0, "finished": 0}

    def fetcher():
        try:
            while True:
                cid = fetch_q.get()
                if cid is None:
                    return
                with cv:
                    i = running[cid]
                r = requests[i]
                ta = clock()
                out = engine.fetch(cid, r.u0.shape)
                latency[i] = (clock() - t0) - r.arrival
                with cv:
                    running.pop(cid)
                    tf["finished"] += 1
                    tf["s"] += clock() - ta
                if on_result is None:
                    results[i] = out
                else:
                    on_result(i, out)
                    r.u0 = None if r.factory is not None else r.u0
                with cv:
                    cv.notify_all()
        except Exception as exc:
            box["error"] = exc

    ths = [threading.Thread(target=admitter, args=(k,), daemon=True) for k in range(admitters)]
    fetchers = [threading.Thread(target=fetcher, daemon=True) for _ in range(2)]
    for th in ths:
        th.start()
    for f in fetchers:
        f.start()
    t_adv = 0.0

    def stop():
        for _ in fetchers:
            fetch_q.put(None)
        for f in fetchers:
            f.join()
        for th in ths:
            th.join()
        pool.shutdown(wait=True)

    while True:
        with cv:
            if tf["finished"] >= n:
                break
            busy = len(running) > len(queued & running.keys())
        if box["error"] is not None:
            stop()
            raise box["error"]
        if not busy:
            time.sleep(idle_sleep)
            continue
        ta = clock()
        engine.advance()
        done = [cid for cid in engine.poll() if cid not in queued]
        t_adv += clock() - ta
        for cid in done:
            queued.add(cid)
            fetch_q.put(cid)
        if not done:
            time.sleep(idle_sleep)
    stop()
    if isinstance(host, dict):
        host.update(admit_s=box["admit_s"], admit_state_wait_s=box["state_s"],
                    admit_call_s=box["call_s"], advance_poll_s=t_adv, fetch_s=tf["s"])
    return results, latency, clock() - t0


class SyntheticStream:
    """Seeded mixed 2-D workload (isentropic vortices on periodic squares)."""

    def __init__(self, count, rate=2000.0, seed=0, sides=(8, 64), orders=(2, 5), mach=(0.1, 2.0),
                 reynolds=(100.0, 1e4), p_inviscid=0.5, strength=(1.0, 5.0), nsteps=200, cfl=0.4,
                 gamma=1.4):
        rng = np.random.default_rng(seed)
        self.params = []
        t = 0.0
        for i in range(count):
            t += rng.exponential(1.0 / rate)
            side = int(rng.integers(sides[0], sides[1] + 1))
            order = int(rng.integers(orders[0], orders[1] + 1))
            ma = float(rng.uniform(*mach))
            inviscid = bool(rng.random() < p_inviscid)
            re = float(rng.uniform(*reynolds))
            b = float(rng.uniform(*strength))
            self.params.append(dict(arrival=t, side=side, order=order, mach=ma, inviscid=inviscid,
                                    reynolds=re, strength=b))
        self.nsteps, self.cfl, self.gamma = nsteps, cfl, gamma
        self._meshes = {}

    def mesh(self, side, order):
        """Periodic [-5, 5]^2 mesh, shared by the cases that draw the same size."""
        key = (side, order)
        if key not in self._meshes:
            self._meshes[key] = periodic_box(2, order, (side, side), (-5.0, -5.0), (5.0, 5.0))
        return self._meshes[key]

    def case(self, i, lazy=False):
        """Case i: domain [-5, 5]^2, freestream (rho=1, p=1, speed Ma*c along the
        diagonal), vortex of the drawn strength; mu from Re on the unit length.
        lazy: the initial state is built at admission."""
        p = self.params[i]
        m = self.mesh(p["side"], p["order"])
        c = np.sqrt(self.gamma)
        v = p["mach"] * c / np.sqrt(2.0)

        def build():
            return _cases.isentropic_vortex(m.coords, gamma=self.gamma, strength=p["strength"],
                                            u_inf=(v, v))
        u0 = None if lazy else build()
        # fixed step: cfl * h / ((2p+1) lambda) with lambda = |u| + c bounded over
        # the vortex, and the diffusive limit h^2 / ((p+1)^4 nu)
        h = 10.0 / p["side"]
        lam = np.sqrt(2.0) * v + 0.5 * p["strength"] / np.pi + c
        dt = self.cfl * h / ((2 * p["order"] + 1) * lam)
        mu = 0.0 if p["inviscid"] else p["mach"] * c * 1.0 / p["reynolds"]
        if mu > 0:
            nu = mu * self.gamma / 0.72
            dt = min(dt, self.cfl * h * h / ((p["order"] + 1) ** 4 * nu))
        off = (1.0, v, v, 1.0 / (self.gamma - 1.0) + v * v, 0.0)
        return Case(mesh=m, u0=u0, nsteps=self.nsteps, dt=dt, viscous=not p["inviscid"], mu=mu,
                    Pr=0.72, state_offset=off, arrival=p["arrival"], tag=p, factory=build,
                    geometry_key=1 + 16 * p["side"] + p["order"])
