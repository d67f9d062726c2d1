"""TEST INFRASTRUCTURE ONLY: ctypes front end of the CPU oracle.

Loads oracle/libthx_oracle.so (the FP64 restatement of the reference's DGSEM
right-hand side, built by `make -C oracle`) and, when it was built here,
oracle/_ref/libthx_ref.so (the reference's own header kernels driven by
oracle/ref_harness.cpp).  Only tests, the smoke check and the benchmark's CPU
baseline import this module; the product never does.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from theseus_b200._abi import Config, Geometry, make_config, FLOW_NAVIER_STOKES  # noqa: F401

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libthx_oracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libthx_ref.so")
REF_NATIVE_PATH = os.path.join(HERE, "_ref", "libthx_ref_native.so")
REF_NATIVE_FLAGS = os.path.join(HERE, "_ref", "native_cpu_flags.txt")
REF_V4_PATH = os.path.join(HERE, "_ref", "libthx_ref_v4.so")
# instruction-set flags that -march=x86-64-v4 assumes beyond v3 (AVX-512 F/BW/CD/DQ/VL)
V4_FLAGS = {"avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl", "avx2", "fma", "bmi1",
            "bmi2", "movbe", "f16c"}

_lib = None
_ref = None
_ref_native = None

D = C.POINTER(C.c_double)
I32 = C.POINTER(C.c_int32)


def build(ref_include=None):
    """Compile the oracle and, given the reference's include directory, _ref."""
    subprocess.check_call(["make", "-s", "-C", HERE])
    if ref_include and os.path.isdir(ref_include):
        subprocess.check_call(["make", "-s", "-C", HERE, "ref", f"REF={ref_include}"])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = C.CDLL(LIB_PATH)
    return _lib


def ref_available():
    return os.path.exists(REF_PATH)


def ref():
    global _ref
    if _ref is None:
        _ref = C.CDLL(REF_PATH)
    return _ref


def _cpu_flags():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("flags"):
                return set(line.split(":", 1)[1].split())
    except OSError:
        pass
    return set()


def ref_native():
    """The optimised build of the reference kernels that this host can run
    (the timed CPU baseline): -O3 -march=native when this host has every
    instruction-set flag of the host that built it, else -O3 -march=x86-64-v4
    on an AVX-512 host, else None.  Sets ref_native.build to its flags."""
    global _ref_native
    if _ref_native is None:
        have = _cpu_flags()
        if os.path.exists(REF_NATIVE_PATH) and os.path.exists(REF_NATIVE_FLAGS):
            need = set(open(REF_NATIVE_FLAGS).read().split())
            if need and need <= have:
                _ref_native = C.CDLL(REF_NATIVE_PATH)
                ref_native.build = "g++ -O3 -march=native (the build host's CPU)"
        if _ref_native is None and os.path.exists(REF_V4_PATH) and V4_FLAGS <= have:
            _ref_native = C.CDLL(REF_V4_PATH)
            ref_native.build = "g++ -O3 -march=x86-64-v4"
    return _ref_native


ref_native.build = None


def _dp(a):
    return a.ctypes.data_as(D) if a is not None else None


def _ip(a):
    return a.ctypes.data_as(I32) if a is not None else None


def sizes(dim, order):
    N = order + 1
    return (N ** dim, N ** (dim - 1), dim + 2)


class Mesh:
    """Geometry arrays in the thx_geometry layout, kept alive for ctypes."""

    def __init__(self, dim, order, jac, metric, face_elem, face_lface, face_normal,
                 face_wminus, face_wplus, coords=None, shape=None, boundary=None):
        self.dim, self.order = dim, order
        self.jac = np.ascontiguousarray(jac, dtype=np.float64)
        self.metric = np.ascontiguousarray(metric, dtype=np.float64)
        self.face_elem = np.ascontiguousarray(face_elem, dtype=np.int32)
        self.face_lface = np.ascontiguousarray(face_lface, dtype=np.int32)
        self.face_normal = np.ascontiguousarray(face_normal, dtype=np.float64)
        self.face_wminus = np.ascontiguousarray(face_wminus, dtype=np.float64)
        self.face_wplus = np.ascontiguousarray(face_wplus, dtype=np.float64)
        self.coords = coords
        self.shape = shape
        self.boundary = boundary   # theseus_b200._abi.Boundary (a plain data record) or None
        self.num_elements = self.jac.shape[0]
        self.num_faces = self.face_elem.shape[0]
        self.nd, self.nfp, self.neq = sizes(dim, order)

    def struct(self):
        g = Geometry()
        g.dim, g.order = self.dim, self.order
        g.num_elements, g.num_faces = self.num_elements, self.num_faces
        g.jac, g.metric = _dp(self.jac), _dp(self.metric)
        g.face_elem, g.face_lface = _ip(self.face_elem), _ip(self.face_lface)
        g.face_normal = _dp(self.face_normal)
        g.face_wminus, g.face_wplus = _dp(self.face_wminus), _dp(self.face_wplus)
        if self.boundary is not None:
            self.boundary.fill(g)
        self._g = g
        return g

    def state_shape(self):
        return (self.neq, self.num_elements, self.nd)


def box_mesh(dim, order, n, lo, hi):
    """Periodic Cartesian box, restated in the oracle (independent of the product)."""
    nd, nfp, neq = sizes(dim, order)
    nn = list(n) + [1] * (3 - len(n))
    ne = int(np.prod(nn[:dim]))
    nf = dim * ne
    jac = np.zeros((ne, nd))
    metric = np.zeros((ne, nd, dim, dim))
    fe = np.zeros((nf, 2), np.int32)
    fl = np.zeros((nf, 2), np.int32)
    fn = np.zeros((nf, nfp, dim))
    wm = np.zeros((nf, nfp))
    wp = np.zeros((nf, nfp))
    coords = np.zeros((dim, ne, nd))
    n32 = np.array(nn, np.int32)
    lo = np.array(list(lo) + [0.0] * (3 - len(lo)))
    hi = np.array(list(hi) + [1.0] * (3 - len(hi)))
    st = lib().orc_box_geometry(dim, order, _ip(n32), _dp(lo), _dp(hi), _dp(jac), _dp(metric),
                                _ip(fe), _ip(fl), _dp(fn), _dp(wm), _dp(wp), _dp(coords))
    if st:
        raise RuntimeError(f"orc_box_geometry failed ({st})")
    return Mesh(dim, order, jac, metric, fe, fl, fn, wm, wp, coords=coords, shape=tuple(nn[:dim]))


def _check(st, what):
    if st:
        raise RuntimeError(f"{what} failed with status {st}")


def rhs(mesh, cfg, u, nthreads=1, want_alpha=False):
    u = np.ascontiguousarray(u, dtype=np.float64)
    du = np.zeros_like(u)
    alpha = np.zeros(mesh.num_elements) if want_alpha else None
    eta = np.zeros(mesh.num_elements) if want_alpha else None
    _check(lib().orc_rhs(C.byref(mesh.struct()), C.byref(cfg), _dp(u), _dp(du), int(nthreads),
                         _dp(alpha), _dp(eta)), "orc_rhs")
    if want_alpha:
        return du, alpha, eta
    return du


MEASURES = ("mass", "ke", "energy", "min_pressure", "max_pressure", "min_temperature",
            "max_temperature", "min_density", "max_density")


def integral_measures(mesh, cfg, u, table=None):
    """IntegralMeasures (include/RHSOperator_impl.hpp:530-717) of state u."""
    u = np.ascontiguousarray(u, dtype=np.float64)
    out = np.zeros(9)
    tab = C.byref(table.struct()) if table is not None else None
    _check(lib().orc_integral_measures(C.byref(mesh.struct()), C.byref(cfg), tab, _dp(u), _dp(out)),
           "orc_integral_measures")
    return dict(zip(MEASURES, out.tolist()))


def gradient(mesh, cfg, u, nthreads=1):
    u = np.ascontiguousarray(u, dtype=np.float64)
    g = np.zeros((mesh.dim,) + u.shape)
    _check(lib().orc_gradient(C.byref(mesh.struct()), C.byref(cfg), _dp(u), _dp(g), int(nthreads)),
           "orc_gradient")
    return g


def rk3_steps(mesh, cfg, u, dt, nsteps, nthreads=1):
    u = np.array(u, dtype=np.float64, copy=True)
    _check(lib().orc_rk3_steps(C.byref(mesh.struct()), C.byref(cfg), _dp(u), C.c_double(dt),
                               int(nsteps), int(nthreads)), "orc_rk3_steps")
    return u


def estimate_dt(mesh, cfg, u, cfl):
    u = np.ascontiguousarray(u, dtype=np.float64)
    dt = C.c_double()
    rates = np.zeros(3)
    _check(lib().orc_estimate_dt(C.byref(mesh.struct()), C.byref(cfg), _dp(u), C.c_double(cfl),
                                 C.byref(dt), _dp(rates)), "orc_estimate_dt")
    return dt.value, rates


def time_event_tolerance(t):
    """TimeEventTolerance (include/TimeStepControl.hpp:15-19)."""
    return 16.0 * np.finfo(np.float64).eps * max(1.0, abs(t))


def time_event_reached(t, event):
    """TimeEventReached (include/TimeStepControl.hpp:21-25)."""
    return t + time_event_tolerance(t) >= event


def limit_time_step_to_events(step, t, events):
    """LimitTimeStepToEvents / TimeToNextEvent (include/TimeStepControl.hpp:27-49)."""
    r, tol = np.inf, time_event_tolerance(t)
    for e in events:
        d = e - t
        if np.isfinite(e) and d > tol:
            r = min(r, d)
    return min(step, r)


def time_loop_driver(u, step, total_rate, cfl, t_final, max_cycles, output_dt=0.01,
                     refined_output_dt=None, refine_time=2.0, output_cycles=100, growth=1.2, dt=None):
    """The reference's clocked time loop (src/Simulation.cpp:1150-1160 initial
    dt = cfl / TotalRate; 1241-1304 per cycle: the nominal step shortened to
    land on the final time and the next output time, one step, the new
    nominal step min(cfl / TotalRate, growth * dt), done at
    t >= t_final - 1e-8 dt or max_cycles; 1321-1331 output events advance the
    next output time by initial_save_dt, refined_save_dt after refine_time).
    step(u, h) advances u by h; total_rate(u) is TotalRate; cfl <= 0 keeps
    the fixed step dt; output_dt None turns output off.  Returns (u, t,
    [step per cycle], cycles, output events)."""
    refined_output_dt = output_dt if refined_output_dt is None else refined_output_dt
    t = 0.0
    if cfl > 0 and not dt:
        dt = cfl / total_rate(u)
    next_out = t + output_dt if output_dt else np.inf
    taken, cycle, outputs, done = [], 0, 0, False
    while not done:
        h = limit_time_step_to_events(dt, t, (t_final, next_out))
        u = step(u, h)
        t += h
        cycle += 1
        taken.append(h)
        if cfl > 0:
            dt = min(cfl / total_rate(u), growth * dt)
        done = t >= t_final - 1e-8 * dt or (max_cycles > 0 and cycle >= max_cycles)
        if np.isfinite(next_out) and (done or time_event_reached(t, next_out) or cycle % output_cycles == 0):
            next_out += output_dt if t < refine_time else refined_output_dt
            outputs += 1
    return u, t, taken, cycle, outputs


def time_loop(mesh, cfg, u, cfl, t_final, max_cycles, nthreads=1, **kw):
    """time_loop_driver over the oracle's SSP-RK3 step and stability estimate."""
    def total(v):
        _, r = estimate_dt(mesh, cfg, v, 1.0)
        return max(r[0], r[1]) + r[2]
    u = np.array(u, dtype=np.float64, copy=True)
    return time_loop_driver(u, lambda v, h: rk3_steps(mesh, cfg, v, h, 1, nthreads), total, cfl, t_final,
                            max_cycles, **kw)


def blending(mesh, cfg, u):
    u = np.ascontiguousarray(u, dtype=np.float64)
    a = np.zeros(mesh.num_elements)
    e = np.zeros(mesh.num_elements)
    _check(lib().orc_blending(C.byref(mesh.struct()), C.byref(cfg), _dp(u), _dp(a), _dp(e)),
           "orc_blending")
    return a, e


def entropy_residual(mesh, cfg, u, du):
    out = C.c_double()
    _check(lib().orc_entropy_residual(C.byref(mesh.struct()), C.byref(cfg),
                                      _dp(np.ascontiguousarray(u, np.float64)),
                                      _dp(np.ascontiguousarray(du, np.float64)), C.byref(out)),
           "orc_entropy_residual")
    return out.value


def operators(order):
    N = order + 1
    Dm, Dh, Dh2 = np.zeros(N * N), np.zeros(N * N), np.zeros(N * N)
    _check(lib().orc_operators(order, _dp(Dm), _dp(Dh), _dp(Dh2)), "orc_operators")
    x, w = np.zeros(N), np.zeros(N)
    _check(lib().orc_lgl(N, _dp(x), _dp(w)), "orc_lgl")
    return x, w, Dm, Dh, Dh2


def subcell_metrics(mesh, cfg):
    dim, N, ne = mesh.dim, mesh.order + 1, mesh.num_elements
    Nz = N if dim > 2 else 1
    xi = np.zeros(((N + 1) * N * Nz) * dim * ne)
    eta = np.zeros((N * (N + 1) * Nz) * dim * ne)
    zeta = np.zeros((N * N * (N + 1)) * dim * ne) if dim > 2 else np.zeros(1)
    _check(lib().orc_subcell_metrics(C.byref(mesh.struct()), C.byref(cfg), _dp(xi), _dp(eta),
                                     _dp(zeta)), "orc_subcell_metrics")
    return xi, eta, zeta


def _point(fn, flux, cfg, dim, *arrs):
    arrs = [np.ascontiguousarray(a, np.float64) for a in arrs]
    F = np.zeros(dim + 2)
    _check(fn(int(flux), C.byref(cfg), int(dim), *[_dp(a) for a in arrs], _dp(F)), "pointwise flux")
    return F


def volume_flux(flux, cfg, dim, q1, q2, m1, m2, use_ref=False):
    L = ref() if use_ref else lib()
    fn = L.ref_volume_flux if use_ref else L.orc_volume_flux
    return _point(fn, flux, cfg, dim, q1, q2, m1, m2)


def face_flux(flux, cfg, dim, qm, qp, n, use_ref=False):
    L = ref() if use_ref else lib()
    fn = L.ref_face_flux if use_ref else L.orc_face_flux
    return _point(fn, flux, cfg, dim, qm, qp, n)


def entropy_vars(cfg, dim, q, use_ref=False):
    L = ref() if use_ref else lib()
    fn = L.ref_entropy_vars if use_ref else L.orc_entropy_vars
    w = np.zeros(dim + 2)
    _check(fn(C.byref(cfg), int(dim), _dp(np.ascontiguousarray(q, np.float64)), _dp(w)), "entropy")
    return w


def viscous_flux(cfg, dim, q, dprim, use_ref=False):
    L = ref() if use_ref else lib()
    fn = L.ref_viscous_flux if use_ref else L.orc_viscous_flux
    out = np.zeros((dim + 2) * dim)
    _check(fn(C.byref(cfg), int(dim), _dp(np.ascontiguousarray(q, np.float64)),
              _dp(np.ascontiguousarray(dprim, np.float64)), _dp(out)), "viscous")
    return out.reshape(dim + 2, dim)


def ref_rhs(mesh, cfg, u, alpha=None, native=False):
    """Full RHS through the reference's own point kernels (oracle/_ref; with
    native=True the -O3 -march=native build, which must be available)."""
    x, w, Dm, Dh, Dh2 = operators(mesh.order)
    u = np.ascontiguousarray(u, dtype=np.float64)
    du = np.zeros_like(u)
    xi = eta = zeta = None
    if alpha is not None:
        xi, eta, zeta = subcell_metrics(mesh, cfg)
        alpha = np.ascontiguousarray(alpha, np.float64)
    L = ref_native() if native else ref()
    _check(L.ref_rhs(C.byref(mesh.struct()), C.byref(cfg), _dp(Dm), _dp(Dh), _dp(Dh2), _dp(w),
                         _dp(alpha), _dp(xi), _dp(eta), _dp(zeta), _dp(u), _dp(du)), "ref_rhs")
    return du


def max_threads():
    return lib().orc_max_threads()


# ---- LTE Helmholtz gas ----------------------------------------------------
class LteTableStruct(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("rho_grid", D), ("T_grid", D),
                ("e_grid", D), ("planes", D), ("inverse", D)]


class IdgParams(C.Structure):
    _fields_ = [("R", C.c_double), ("rho_d", C.c_double), ("theta_d", C.c_double),
                ("mu0", C.c_double), ("T0", C.c_double), ("Pr", C.c_double)]


# Config 4's table: O2-like ideal dissociating gas on 256 x 512 log-spaced samples
IDG_O2 = dict(R=8.314462618 / 0.0319988, rho_d=1.5e5, theta_d=59500.0, mu0=1.9e-5, T0=273.15,
              Pr=0.71)
GRID_CONFIG4 = dict(nx=256, ny=512, log_rho=(-6.0, 1.0), log_T=(2.3, 4.3))


class LteTable:
    """Oracle-built LTE table (forward planes + inverse table), kept alive for ctypes."""

    def __init__(self, nx, ny, log_rho, log_T, params=None):
        p = IdgParams(**(params or IDG_O2))
        self.params = p
        self.nx, self.ny = nx, ny
        self.rho = np.zeros(nx)
        self.T = np.zeros(ny)
        self.planes = np.zeros((6, ny, nx))
        self.e = np.zeros(ny)
        self.inv = np.zeros((ny, nx))
        _check(lib().orc_lte_idg_table(C.byref(p), nx, ny, C.c_double(log_rho[0]), C.c_double(log_rho[1]),
                                       C.c_double(log_T[0]), C.c_double(log_T[1]), _dp(self.rho),
                                       _dp(self.T), _dp(self.planes)), "orc_lte_idg_table")
        _check(lib().orc_lte_inverse_table(nx, ny, _dp(self.rho), _dp(self.T), _dp(self.planes),
                                           _dp(self.e), _dp(self.inv)), "orc_lte_inverse_table")

    def struct(self):
        s = LteTableStruct(self.nx, self.ny, _dp(self.rho), _dp(self.T), _dp(self.e),
                           _dp(self.planes), _dp(self.inv))
        self._s = s
        return s


def lte_point(table, rho, T, use_ref=False):
    out = np.zeros(7)
    fn = ref().ref_lte_point if use_ref else lib().orc_lte_point
    _check(fn(C.byref(table.struct()), C.c_double(rho), C.c_double(T), _dp(out)), "lte_point")
    return out


def lte_temperature(table, rho, e, use_ref=False):
    T, st = C.c_double(), C.c_int()
    fn = ref().ref_lte_temperature if use_ref else lib().orc_lte_temperature
    fn(C.byref(table.struct()), C.c_double(rho), C.c_double(e), C.byref(T), C.byref(st))
    return T.value, st.value


def lte_flux(table, cfg, dim, face, q1, q2, d1, d2, use_ref=False):
    F = np.zeros(dim + 2)
    arrs = [np.ascontiguousarray(a, np.float64) for a in (q1, q2, d1, d2)]
    if use_ref:
        st = ref().ref_lte_flux(C.byref(table.struct()), C.byref(cfg), int(dim), int(face),
                                *[_dp(a) for a in arrs], _dp(F))
    else:
        st = lib().orc_lte_flux(C.byref(table.struct()), int(dim), int(face), *[_dp(a) for a in arrs], _dp(F))
    _check(st, "lte_flux")
    return F


def rhs_lte(mesh, cfg, table, u, nthreads=1, use_ref=False):
    u = np.ascontiguousarray(u, dtype=np.float64)
    du = np.zeros_like(u)
    if use_ref:
        x, w, Dm, Dh, Dh2 = operators(mesh.order)
        st = ref().ref_rhs_lte(C.byref(mesh.struct()), C.byref(cfg), C.byref(table.struct()), _dp(Dm),
                               _dp(Dh), _dp(Dh2), _dp(w), _dp(u), _dp(du))
    else:
        st = lib().orc_rhs_lte(C.byref(mesh.struct()), C.byref(cfg), C.byref(table.struct()), _dp(u),
                               _dp(du), int(nthreads))
    _check(st, "rhs_lte")
    return du
