"""theseus_b200 -- B200-native DGSEM right-hand side (sm_100a CUDA behind a C ABI).

Python mirror of the reference's operator interface:

    op = MakeRHSOperator({"flow_model": "navier-stokes", "numerical_flux": "ranocha",
                          "surface_flux": "hll"}, mesh)
    op.Mult(u, dudt)                 # RHSOperator<PhysicsT>::Mult (include/RHSOperator.hpp:100)
    op.EstimateStability(u)          # include/RHSOperator_impl.hpp:10-270
    op.rk3_steps(u, dt, nsteps)      # mfem::RK3SSPSolver::Step, fused on the device

States are torch CUDA tensors shaped (num_equations, num_elements, nodes_per_element)
holding the byNODES L-vector.  The shared library is loaded from this package
directory; if it is missing, or no CUDA device is visible, every compute call
raises -- there is no CPU fallback.
"""
import ctypes as C
import os

import numpy as np

from ._abi import (Config, Geometry, LteTable, IdgParams, make_config, flux_id,  # noqa: F401
                   FLUX, FLUX_NAMES, FLOW_EULER, FLOW_NAVIER_STOKES, PRECISION_FP64,
                   PRECISION_FP32_MIXED, THX_OK, THX_ERR_CUDA, THX_ERR_OUT_OF_MEMORY, STATUS_NONPOSITIVE, STATUS_NONFINITE,
                   STATUS_LAUNCH, STATUS_EOS)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtheseus_b200.so")

_lib = None

_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int32)


class THXError(RuntimeError):
    pass


def library():
    """Load libtheseus_b200.so (build it with theseus_b200/build.py)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise THXError(f"{LIB_PATH} is missing: run `python theseus_b200/build.py` "
                           "(the CUDA extension is required; there is no CPU fallback)")
        lib = C.CDLL(LIB_PATH)
        lib.thx_version.restype = C.c_char_p
        lib.thx_status_string.restype = C.c_char_p
        lib.thx_last_cuda_failure.restype = C.c_char_p
        lib.thx_create.argtypes = [C.POINTER(Geometry), C.POINTER(Config), C.POINTER(C.c_void_p)]
        lib.thx_create_lte.argtypes = [C.POINTER(Geometry), C.POINTER(Config), C.POINTER(LteTable),
                                       C.POINTER(C.c_void_p)]
        lib.thx_lte_idg_table.argtypes = [C.POINTER(IdgParams), C.c_int, C.c_int, C.c_double,
                                          C.c_double, C.c_double, C.c_double, _D, _D, _D]
        lib.thx_lte_inverse_table.argtypes = [C.c_int, C.c_int, _D, _D, _D, _D, _D]
        lib.thx_destroy.argtypes = [C.c_void_p]
        lib.thx_rhs.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        lib.thx_rk3_steps.argtypes = [C.c_void_p, C.c_void_p, C.c_double, C.c_int, C.c_void_p]
        lib.thx_rk3_steps_cfl.argtypes = [C.c_void_p, C.c_void_p, C.c_double, C.c_int, C.c_void_p,
                                          C.c_void_p]
        lib.thx_blending_coefficients.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        lib.thx_estimate_dt.argtypes = [C.c_void_p, C.c_void_p, C.c_double, _D, _D]
        lib.thx_read_status.argtypes = [C.c_void_p, C.POINTER(C.c_uint32), C.c_void_p]
        lib.thx_describe.argtypes = [C.c_void_p, C.c_char_p, C.c_size_t]
        lib.thx_rhs_profile.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, _D]
        lib.thx_integral_measures.argtypes = [C.c_void_p, C.c_void_p, _D]
        _lib = lib
    return _lib


def _check(st, what):
    if st != THX_OK:
        msg = library().thx_status_string(st).decode()
        if st in (THX_ERR_CUDA, THX_ERR_OUT_OF_MEMORY):
            detail = library().thx_last_cuda_failure().decode()
            if detail:
                msg += f" [{detail}]"
        raise THXError(f"{what}: {msg} (status {st})")


def sizes(dim, order):
    N = order + 1
    return N ** dim, N ** (dim - 1), dim + 2


class Mesh:
    """Geometric factors in the thx_geometry layout (host numpy arrays)."""

    def __init__(self, dim, order, jac, metric, face_elem, face_lface, face_normal, face_wminus,
                 face_wplus, coords=None, shape=None, boundary=None):
        self.dim, self.order = int(dim), int(order)
        self.jac = np.ascontiguousarray(jac, np.float64)
        self.metric = np.ascontiguousarray(metric, np.float64)
        self.face_elem = np.ascontiguousarray(face_elem, np.int32)
        self.face_lface = np.ascontiguousarray(face_lface, np.int32)
        self.face_normal = np.ascontiguousarray(face_normal, np.float64)
        self.face_wminus = np.ascontiguousarray(face_wminus, np.float64)
        self.face_wplus = np.ascontiguousarray(face_wplus, np.float64)
        self.coords = coords
        self.shape = shape
        self.boundary = boundary   # _abi.Boundary or None (periodic)
        self.num_elements = self.jac.shape[0]
        self.num_faces = self.face_elem.shape[0]
        self.nd, self.nfp, self.neq = sizes(self.dim, self.order)

    @property
    def num_nodes(self):
        return self.num_elements * self.nd

    def state_shape(self):
        return (self.neq, self.num_elements, self.nd)

    def struct(self):
        g = Geometry()
        g.dim, g.order, g.num_elements, g.num_faces = self.dim, self.order, self.num_elements, self.num_faces
        g.jac = self.jac.ctypes.data_as(_D)
        g.metric = self.metric.ctypes.data_as(_D)
        g.face_elem = self.face_elem.ctypes.data_as(_I)
        g.face_lface = self.face_lface.ctypes.data_as(_I)
        g.face_normal = self.face_normal.ctypes.data_as(_D)
        g.face_wminus = self.face_wminus.ctypes.data_as(_D)
        g.face_wplus = self.face_wplus.ctypes.data_as(_D)
        if self.boundary is not None:
            self.boundary.fill(g)
        self._g = g
        return g


def periodic_box(dim, order, n, lo, hi, coords=True):
    """Periodic Cartesian box mesh (host set-up in the library, no device work)."""
    lib = library()
    nd, nfp, neq = sizes(dim, order)
    n32 = np.array(list(n) + [1] * (3 - len(n)), np.int32)
    ne, nf = C.c_int32(), C.c_int32()
    _check(lib.thx_box_counts(dim, n32.ctypes.data_as(_I), C.byref(ne), C.byref(nf)), "thx_box_counts")
    ne, nf = ne.value, nf.value
    jac = np.zeros((ne, nd))
    metric = np.zeros((ne, nd, dim, dim))
    fe = np.zeros((nf, 2), np.int32)
    fl = np.zeros((nf, 2), np.int32)
    fn = np.zeros((nf, nfp, dim))
    wm = np.zeros((nf, nfp))
    wp = np.zeros((nf, nfp))
    xyz = np.zeros((dim, ne, nd)) if coords else None
    lo3 = np.array(list(lo) + [0.0] * (3 - len(lo)))
    hi3 = np.array(list(hi) + [1.0] * (3 - len(hi)))
    _check(lib.thx_box_geometry(dim, order, n32.ctypes.data_as(_I), lo3.ctypes.data_as(_D),
                                hi3.ctypes.data_as(_D), jac.ctypes.data_as(_D),
                                metric.ctypes.data_as(_D), fe.ctypes.data_as(_I),
                                fl.ctypes.data_as(_I), fn.ctypes.data_as(_D), wm.ctypes.data_as(_D),
                                wp.ctypes.data_as(_D),
                                xyz.ctypes.data_as(_D) if coords else None), "thx_box_geometry")
    return Mesh(dim, order, jac, metric, fe, fl, fn, wm, wp, coords=xyz, shape=tuple(n[:dim]))


def box(dim, order, n, lo, hi, periodic=None, boundary=None, coords=True):
    """Cartesian box mesh with periodic sides or boundary conditions.
    periodic: one flag per direction (default all periodic); boundary maps each
    side of a non-periodic direction ("x-", "x+", "y-", "y+", "z-", "z+") to
    a condition named as in the reference's runtime JSON ("slip",
    "supersonic-outflow", "symmetry", ("supersonic-inflow", q),
    ("exterior-state", q) with q the exterior conserved state,
    ("no-slip-adiabatic", v..., heat), ("no-slip-isothermal", v..., T))."""
    from ._abi import box_boundary
    m = periodic_box(dim, order, n, lo, hi, coords)
    periodic = tuple(periodic) if periodic is not None else (True,) * dim
    if all(periodic[:dim]):
        return m
    faces, bdr = box_boundary(dim, n, m.face_elem, m.face_lface, m.face_normal, m.face_wminus,
                              m.face_wplus, periodic, boundary or {})
    return Mesh(dim, order, m.jac, m.metric, *faces, coords=m.coords, shape=m.shape, boundary=bdr)


def lgl(np_):
    x, w = np.zeros(np_), np.zeros(np_)
    _check(library().thx_lgl(np_, x.ctypes.data_as(_D), w.ctypes.data_as(_D)), "thx_lgl")
    return x, w


class HelmholtzTable:
    """LTE Helmholtz gas table (include/LTEHelmholtzTable.hpp:13-35): host numpy
    arrays rho_grid[nx], T_grid[ny], planes[6][ny][nx] (H, H_rho, H_T, H_rhoT, mu,
    lambda), plus the energy grid and inverse table, which Build() derives when
    they are not given (include/LTEHelmholtzTableBuilder.hpp:131-218)."""

    def __init__(self, rho_grid, T_grid, planes, e_grid=None, inverse=None):
        self.rho = np.ascontiguousarray(rho_grid, np.float64)
        self.T = np.ascontiguousarray(T_grid, np.float64)
        self.nx, self.ny = self.rho.size, self.T.size
        self.planes = np.ascontiguousarray(planes, np.float64).reshape(6, self.ny, self.nx)
        self.e = None if e_grid is None else np.ascontiguousarray(e_grid, np.float64)
        self.inv = None if inverse is None else np.ascontiguousarray(inverse, np.float64).reshape(
            self.ny, self.nx)
        if self.e is None or self.inv is None:
            self.Build()

    def Build(self):
        self.e = np.zeros(self.ny)
        self.inv = np.zeros((self.ny, self.nx))
        _check(library().thx_lte_inverse_table(self.nx, self.ny, self.rho.ctypes.data_as(_D),
                                               self.T.ctypes.data_as(_D),
                                               self.planes.ctypes.data_as(_D),
                                               self.e.ctypes.data_as(_D),
                                               self.inv.ctypes.data_as(_D)), "thx_lte_inverse_table")
        return self

    @classmethod
    def ideal_dissociating_gas(cls, nx, ny, log_rho, log_T, R, rho_d, theta_d, mu0, T0, Pr):
        """Synthetic table of Lighthill's ideal dissociating gas on log-spaced grids."""
        p = IdgParams(R, rho_d, theta_d, mu0, T0, Pr)
        rho, T, planes = np.zeros(nx), np.zeros(ny), np.zeros((6, ny, nx))
        _check(library().thx_lte_idg_table(C.byref(p), nx, ny, float(log_rho[0]), float(log_rho[1]),
                                           float(log_T[0]), float(log_T[1]),
                                           rho.ctypes.data_as(_D), T.ctypes.data_as(_D),
                                           planes.ctypes.data_as(_D)), "thx_lte_idg_table")
        return cls(rho, T, planes)

    def struct(self):
        s = LteTable(self.nx, self.ny, self.rho.ctypes.data_as(_D), self.T.ctypes.data_as(_D),
                     self.e.ctypes.data_as(_D), self.planes.ctypes.data_as(_D),
                     self.inv.ctypes.data_as(_D))
        self._s = s
        return s


def _stream_ptr(stream):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


class RHSOperator:
    """Mirror of Theseus::RHSOperator<PhysicsT> (include/RHSOperator.hpp:119-188)
    whose Mult forwards to the sm_100a kernels through the C ABI."""

    flow = "euler"

    def __init__(self, mesh, numerical_flux="chandrashekar", surface_flux=None, fv_flux="llf",
                 blending=False, precision="fp64", device=None, gas=None, **physics):
        import torch
        if not torch.cuda.is_available():
            raise THXError("no CUDA device: the DGSEM operator has no CPU fallback")
        self.mesh = mesh
        self.cfg = make_config(flow=self.flow, volume_flux=numerical_flux,
                               surface_flux=surface_flux, fv_flux=fv_flux, blending=blending,
                               precision=precision, **physics)
        self.mixed = self.cfg.precision == PRECISION_FP32_MIXED
        # the ABI state is FP64 in both precisions (FP32-mixed narrows internally)
        self.dtype = torch.float64
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.gas = gas
        h = C.c_void_p()
        with torch.cuda.device(self.device):
            if gas is None:
                _check(library().thx_create(C.byref(mesh.struct()), C.byref(self.cfg), C.byref(h)),
                       "thx_create")
            else:
                if not isinstance(gas, HelmholtzTable):
                    raise THXError("gas must be a HelmholtzTable (or None for the ideal gas)")
                _check(library().thx_create_lte(C.byref(mesh.struct()), C.byref(self.cfg),
                                                C.byref(gas.struct()), C.byref(h)), "thx_create_lte")
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                library().thx_destroy(h)
            except Exception:
                pass
            self._h = None

    # -- shape helpers --------------------------------------------------
    @property
    def height(self):
        return self.mesh.neq * self.mesh.num_nodes

    def _check_state(self, t, dtype):
        import torch
        if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == dtype and t.is_contiguous()
                and t.numel() == self.height and t.device == self.device):
            raise THXError(f"expected a contiguous {dtype} CUDA tensor with {self.height} entries "
                           f"on {self.device}")

    # -- the reference interface ------------------------------------------
    def Mult(self, u, dudt, stream=None):
        """dudt = L(u)."""
        self._check_state(u, self.dtype)
        self._check_state(dudt, self.dtype)
        _check(library().thx_rhs(self._h, C.c_void_p(u.data_ptr()), C.c_void_p(dudt.data_ptr()),
                                 _stream_ptr(stream)), "thx_rhs")
        return dudt

    def EstimateStability(self, u):
        """(advective, surface, diffusive) rates (include/StabilityEstimate.hpp:38-54)."""
        import torch
        self._check_state(u, torch.float64)
        dt = C.c_double()
        rates = np.zeros(3)
        torch.cuda.current_stream().synchronize()
        _check(library().thx_estimate_dt(self._h, C.c_void_p(u.data_ptr()), 1.0, C.byref(dt),
                                         rates.ctypes.data_as(_D)), "thx_estimate_dt")
        return rates

    MEASURES = ("mass", "ke", "energy", "min_pressure", "max_pressure", "min_temperature",
                "max_temperature", "min_density", "max_density")

    def IntegralMeasures(self, u):
        """Integrals of rho, kinetic energy and rho E and the pressure,
        temperature and density extrema of a device FP64 state
        (RHSOperator::ComputeIntegralMeasures, include/RHSOperator_impl.hpp:530-717)."""
        import torch
        self._check_state(u, torch.float64)
        out = np.zeros(9)
        torch.cuda.current_stream().synchronize()
        _check(library().thx_integral_measures(self._h, C.c_void_p(u.data_ptr()),
                                               out.ctypes.data_as(_D)), "thx_integral_measures")
        return dict(zip(self.MEASURES, out.tolist()))

    def estimate_dt(self, u, cfl):
        r = self.EstimateStability(u)
        return cfl / (max(r[0], r[1]) + r[2])

    def rk3_steps(self, u, dt, nsteps, stream=None):
        """nsteps SSP-RK3 steps on the FP64 master state u, in place."""
        import torch
        self._check_state(u, torch.float64)
        _check(library().thx_rk3_steps(self._h, C.c_void_p(u.data_ptr()), float(dt), int(nsteps),
                                       _stream_ptr(stream)), "thx_rk3_steps")
        return u

    def rk3_steps_cfl(self, u, cfl, nsteps, stream=None):
        """nsteps SSP-RK3 steps with dt = cfl / TotalRate of each step's
        initial state, computed on the device (no host round trip per step).
        Returns the device tensor of the nsteps time steps taken."""
        import torch
        self._check_state(u, torch.float64)
        dts = torch.zeros(max(1, int(nsteps)), dtype=torch.float64, device=u.device)
        _check(library().thx_rk3_steps_cfl(self._h, C.c_void_p(u.data_ptr()), float(cfl), int(nsteps),
                                           C.c_void_p(dts.data_ptr()), _stream_ptr(stream)),
               "thx_rk3_steps_cfl")
        return dts[:int(nsteps)]

    def mult_host(self, states, rates, stream=None):
        """rates[i] = L(states[i]) for FP64 host tensors (thx_rhs_host): the
        transfers of neighbouring states overlap the evaluation when the host
        tensors are pinned.  Stream-ordered: synchronise before reading rates."""
        import torch
        n = len(states)
        if len(rates) != n:
            raise ValueError("states and rates differ in length")
        size = self.mesh.neq * self.mesh.num_nodes
        for t in list(states) + list(rates):
            if t.device.type != "cpu" or t.dtype != torch.float64 or not t.is_contiguous() or t.numel() != size:
                raise ValueError("host states and rates must be contiguous float64 CPU tensors of the mesh's size")
        ins = (C.c_void_p * max(1, n))(*[t.data_ptr() for t in states])
        outs = (C.c_void_p * max(1, n))(*[t.data_ptr() for t in rates])
        lib = library()
        if not getattr(lib, "_rhs_host_bound", False):
            lib.thx_rhs_host.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
            lib._rhs_host_bound = True
        _check(lib.thx_rhs_host(self._h, n, ins, outs, _stream_ptr(stream)), "thx_rhs_host")
        return rates

    def run_time_loop(self, u, loop, ncycles, cfl=0.0, stream=None):
        """ncycles cycles of the reference's clocked SSP-RK3 loop on u (FP64,
        in place): `loop` is a TimeLoop (copied to the device, advanced there
        and read back once at the end) or a device record from
        TimeLoop.to_device (left on the device).  cfl > 0 makes the step
        variable.  Returns the device tensor of the steps taken."""
        import torch
        from .timeloop import TimeLoop, _lib as _time_lib
        self._check_state(u, torch.float64)
        host = isinstance(loop, TimeLoop)
        dev = loop.to_device(u.device) if host else loop
        dts = torch.zeros(max(1, int(ncycles)), dtype=torch.float64, device=u.device)
        _check(_time_lib().thx_rk3_time_loop(self._h, C.c_void_p(u.data_ptr()), float(cfl), int(ncycles),
                                             C.c_void_p(dev.data_ptr()), C.c_void_p(dts.data_ptr()),
                                             _stream_ptr(stream)), "thx_rk3_time_loop")
        if host:
            loop.load(dev)
        return dts[:int(ncycles)]

    def blending_coefficients(self, stream=None):
        import torch
        a = torch.zeros(self.mesh.num_elements, dtype=torch.float64, device=self.device)
        e = torch.zeros_like(a)
        _check(library().thx_blending_coefficients(self._h, C.c_void_p(a.data_ptr()),
                                                   C.c_void_p(e.data_ptr()), _stream_ptr(stream)),
               "thx_blending_coefficients")
        return a, e

    def read_status(self, stream=None):
        v = C.c_uint32()
        _check(library().thx_read_status(self._h, C.byref(v), _stream_ptr(stream)), "thx_read_status")
        return v.value

    def profile(self, u, dudt, stream=None):
        """One Mult with per-kernel device times (ms): indicator, gradient, faces, volume."""
        self._check_state(u, self.dtype)
        self._check_state(dudt, self.dtype)
        ms = np.zeros(4)
        _check(library().thx_rhs_profile(self._h, C.c_void_p(u.data_ptr()),
                                         C.c_void_p(dudt.data_ptr()), _stream_ptr(stream),
                                         ms.ctypes.data_as(_D)), "thx_rhs_profile")
        return ms

    def describe(self):
        buf = C.create_string_buffer(1024)
        _check(library().thx_describe(self._h, buf, 1024), "thx_describe")
        return buf.value.decode()

    def NumFluxName(self):
        return FLUX_NAMES[self.cfg.volume_flux]

    def FlowModelName(self):
        return self.flow


class EulerOperator(RHSOperator):
    """Mirror of Theseus::EulerOperator (include/EulerOperator.hpp)."""
    flow = "euler"


class NSOperator(RHSOperator):
    """Mirror of Theseus::NSOperator (include/NSOperator.hpp)."""
    flow = "navier-stokes"


def MakeRHSOperator(runtime, mesh, device=None, table=None):
    """Selection by the reference's runtime JSON keys (include/SimFactory_impl.hpp:63-488):
    flow_model, numerical_flux, gas_model, gamma, Pr, R_gas, mu; plus the keys this library
    adds to decouple the volume and surface fluxes (surface_flux, fv_flux), blending and
    precision.  gas_model "lte"/"lte_helmholtz" needs `table` (a HelmholtzTable)."""
    flow = str(runtime.get("flow_model", "euler")).lower()
    viscous = flow.startswith(("visc", "nav", "cns", "ns"))
    gas = str(runtime.get("gas_model", "cpg")).lower()
    if gas in ("lte", "lte_helmholtz", "helmholtz"):
        if table is None:
            raise THXError("gas_model 'lte' needs a HelmholtzTable (table=...)")
        cls = NSOperator if viscous else EulerOperator
        phys = {k: runtime[k] for k in ("Pr", "mu") if k in runtime}
        return cls(mesh, numerical_flux=runtime.get("numerical_flux", "lteec"),
                   surface_flux=runtime.get("surface_flux", "lteec"), device=device, gas=table,
                   **phys)
    if gas not in ("", "cpg", "ideal", "ideal_gas"):
        raise THXError(f"gas_model '{gas}' is not built in this library")
    cls = NSOperator if viscous else EulerOperator
    phys = {k: runtime[k] for k in ("gamma", "Pr", "R_gas", "mu", "mu0") if k in runtime}
    if "alpha_max" in runtime:
        phys["alpha_max"] = runtime["alpha_max"]
    return cls(mesh, numerical_flux=runtime.get("numerical_flux", "chandrashekar"),
               surface_flux=runtime.get("surface_flux"), fv_flux=runtime.get("fv_flux", "llf"),
               blending=bool(runtime.get("blending", False)),
               precision=runtime.get("precision", "fp64"), device=device, **phys)
