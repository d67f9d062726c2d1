"""ctypes mirror of the structs and enums in include/theseus_b200.h.

Pure data definitions: importing this module loads no shared library.
"""
import ctypes as C

THX_OK = 0
THX_ERR_INVALID_ARGUMENT = 1
THX_ERR_UNSUPPORTED = 2
THX_ERR_CUDA = 3
THX_ERR_NO_DEVICE = 4
THX_ERR_OUT_OF_MEMORY = 5
THX_ERR_NUMERICS = 6

FLUX = {"chandrashekar": 0, "ranocha": 1, "pirozzoli": 2, "hll": 3, "llf": 4, "roe": 5,
        "lteec": 6}
FLUX_NAMES = {v: k for k, v in FLUX.items()}
FLOW_EULER = 0
FLOW_NAVIER_STOKES = 1
PRECISION_FP64 = 0
PRECISION_FP32_MIXED = 1


class Config(C.Structure):
    _fields_ = [
        ("flow_model", C.c_int32), ("volume_flux", C.c_int32), ("surface_flux", C.c_int32),
        ("fv_flux", C.c_int32), ("blending", C.c_int32), ("precision", C.c_int32),
        ("sutherland", C.c_int32), ("geometry_layout", C.c_int32),
        ("gamma", C.c_double), ("Pr", C.c_double), ("R_gas", C.c_double), ("mu", C.c_double),
        ("mu0", C.c_double), ("mu_bulk", C.c_double), ("T0", C.c_double), ("Ts", C.c_double),
        ("alpha_max", C.c_double), ("alpha_min", C.c_double), ("sharpness", C.c_double),
        ("modal_threshold", C.c_double), ("state_offset", C.c_double * 5),
        ("volume_staging", C.c_int32), ("mixed_blended_fp32", C.c_int32),
        ("mixed_flux_no_perturbation", C.c_int32),
    ]


class BC(C.Structure):
    _fields_ = [("type", C.c_int32), ("data_index", C.c_int32)]


# Boundary condition names of the reference's runtime JSON (src/Simulation.cpp:540-860)
# and their BCType numbers (include/bc_cache_utilities.hpp:11-23).
BC_TYPES = {"slip": 0, "supersonic-inflow": 1, "supersonic-outflow": 2, "exterior-state": 3,
            "symmetry": 4, "axis": 5, "no-slip-adiabatic": 6, "no-slip-isothermal": 7}


class Geometry(C.Structure):
    _fields_ = [
        ("dim", C.c_int32), ("order", C.c_int32), ("num_elements", C.c_int32),
        ("num_faces", C.c_int32),
        ("jac", C.POINTER(C.c_double)), ("metric", C.POINTER(C.c_double)),
        ("face_elem", C.POINTER(C.c_int32)), ("face_lface", C.POINTER(C.c_int32)),
        ("face_normal", C.POINTER(C.c_double)), ("face_wminus", C.POINTER(C.c_double)),
        ("face_wplus", C.POINTER(C.c_double)),
        ("num_bdr_faces", C.c_int32),
        ("bdr_elem", C.POINTER(C.c_int32)), ("bdr_lface", C.POINTER(C.c_int32)),
        ("bdr_normal", C.POINTER(C.c_double)), ("bdr_weight", C.POINTER(C.c_double)),
        ("bdr_bc", C.POINTER(C.c_int32)),
        ("num_bcs", C.c_int32), ("bcs", C.POINTER(BC)),
        ("bc_data_len", C.c_int32), ("bc_data", C.POINTER(C.c_double)),
    ]


class Boundary:
    """Boundary faces in the thx_geometry layout: elem[b], lface[b], outward
    normal[b][fp][dim], lift weight[b][fp], bc[b] (index into bcs), bcs as
    (type, data_index) pairs and the packed payloads bc_data."""

    def __init__(self, elem, lface, normal, weight, bc, bcs, bc_data):
        import numpy as np
        self.elem = np.ascontiguousarray(elem, np.int32)
        self.lface = np.ascontiguousarray(lface, np.int32)
        self.normal = np.ascontiguousarray(normal, np.float64)
        self.weight = np.ascontiguousarray(weight, np.float64)
        self.bc = np.ascontiguousarray(bc, np.int32)
        self.bcs = (BC * max(1, len(bcs)))(*[BC(int(t), int(i)) for t, i in bcs])
        self.num_bcs = len(bcs)
        self.bc_data = np.ascontiguousarray(bc_data if len(bc_data) else [0.0], np.float64)
        self.bc_data_len = len(bc_data)

    @property
    def num_faces(self):
        return int(self.elem.shape[0])

    def fill(self, g):
        D, I = C.POINTER(C.c_double), C.POINTER(C.c_int32)
        g.num_bdr_faces = self.num_faces
        g.bdr_elem = self.elem.ctypes.data_as(I)
        g.bdr_lface = self.lface.ctypes.data_as(I)
        g.bdr_normal = self.normal.ctypes.data_as(D)
        g.bdr_weight = self.weight.ctypes.data_as(D)
        g.bdr_bc = self.bc.ctypes.data_as(I)
        g.num_bcs = self.num_bcs
        g.bcs = C.cast(self.bcs, C.POINTER(BC))
        g.bc_data_len = self.bc_data_len
        g.bc_data = self.bc_data.ctypes.data_as(D)


def box_boundary(dim, n, face_elem, face_lface, face_normal, face_wminus, face_wplus, periodic,
                 boundary):
    """Split the wrap faces of a periodic box's non-periodic directions into
    boundary faces.  The box numbers faces direction by direction, element by
    element (x fastest), the face of element e in direction d joining it to
    its +d neighbour; the wrap faces are those of the last element layer.
    boundary maps a side ("x-", "x+", "y-", "y+", "z-", "z+") to a condition:
    a name of BC_TYPES, or (name, payload) with the exterior conserved state
    for "supersonic-inflow"/"exterior-state" and (velocity..., heat or
    temperature) for the no-slip walls.  Returns the kept interior faces'
    arrays and the Boundary; boundary faces are numbered direction by
    direction, so that a node's boundary faces are in direction order."""
    import numpy as np
    nn = list(n) + [1] * (3 - len(n))
    ne = int(np.prod(nn[:dim]))
    e = np.arange(ne)
    ix = [e % nn[0], (e // nn[0]) % nn[1], e // (nn[0] * nn[1])]
    keep = np.ones(dim * ne, bool)
    sides = {}
    for d in range(dim):
        if periodic[d]:
            continue
        for s in (f"{'xyz'[d]}-", f"{'xyz'[d]}+"):
            if s not in boundary:
                raise ValueError(f"side {s} is not periodic and has no boundary condition")
        keep[d * ne:(d + 1) * ne] &= ix[d] != nn[d] - 1
    bcs, data, side_bc = [], [], {}
    for side in sorted(boundary, key=lambda s: ("xyz".index(s[0]), s[1] == "+")):
        spec = boundary[side]
        name, payload = (spec, ()) if isinstance(spec, str) else (spec[0], tuple(np.ravel(spec[1:])))
        if name not in BC_TYPES:
            raise ValueError(f"unknown boundary condition {name!r}")
        side_bc[side] = len(bcs)
        bcs.append((BC_TYPES[name], len(data)))
        data.extend(float(x) for x in payload)
    elem, lface, normal, weight, bci = [], [], [], [], []
    for d in range(dim):
        if periodic[d]:
            continue
        wrap = np.nonzero(ix[d] == nn[d] - 1)[0] + d * ne      # face of the last layer
        lo_e = face_elem[wrap, 1]                               # first layer: its -d face
        hi_e = face_elem[wrap, 0]                               # last layer: its +d face
        for f, eb, lf, sgn, w, side in ((wrap, lo_e, 2 * d, -1.0, face_wplus, f"{'xyz'[d]}-"),
                                        (wrap, hi_e, 2 * d + 1, 1.0, face_wminus, f"{'xyz'[d]}+")):
            order_ = np.argsort(eb, kind="stable")
            elem.append(eb[order_])
            lface.append(np.full(len(f), lf, np.int32))
            normal.append(face_normal[f[order_]] if sgn > 0 else 0.0 - face_normal[f[order_]])
            weight.append(w[f[order_]])
            bci.append(np.full(len(f), side_bc[side], np.int32))
    bdr = Boundary(np.concatenate(elem), np.concatenate(lface), np.concatenate(normal),
                   np.concatenate(weight), np.concatenate(bci), bcs, data)
    return (face_elem[keep], face_lface[keep], face_normal[keep], face_wminus[keep],
            face_wplus[keep]), bdr


def flux_id(name_or_id):
    if isinstance(name_or_id, int):
        return name_or_id
    key = str(name_or_id).lower()
    # selection aliases of include/SimFactory_impl.hpp:75-128
    if key in ("", "chan") or key.startswith("chan"):
        return FLUX["chandrashekar"]
    if key in ("piflux",) or key.startswith("pi"):
        return FLUX["pirozzoli"]
    if key in ("lfr", "laxfriedrichs", "lax_friedrichs") or key.startswith("lax"):
        return FLUX["llf"]
    if key in ("lteecflux",):
        return FLUX["lteec"]
    if key not in FLUX:
        raise ValueError(f"unknown numerical flux '{name_or_id}'; supported: "
                         "Chandrashekar, Ranocha, Pirozzoli, LLF/LFR, HLL, Roe")
    return FLUX[key]


def make_config(flow="euler", volume_flux="chandrashekar", surface_flux=None, fv_flux="llf",
                blending=False, precision="fp64", gamma=1.4, Pr=0.72, R_gas=287.05, mu=0.02,
                mu0=1.716e-5, mu_bulk=2.0 / 3.0, T0=273.15, Ts=110.4, alpha_max=0.5,
                alpha_min=0.001, sharpness=9.21024, modal_threshold=0.0, sutherland=False,
                geometry_layout=0, state_offset=None, volume_staging=0, mixed_blended_fp32=False,
                mixed_flux_no_perturbation=False):
    cfg = Config()
    f = str(flow).lower()
    viscous = f.startswith(("visc", "nav", "cns", "ns"))
    cfg.flow_model = FLOW_NAVIER_STOKES if viscous else FLOW_EULER
    cfg.volume_flux = flux_id(volume_flux)
    cfg.surface_flux = flux_id(surface_flux if surface_flux is not None else volume_flux)
    cfg.fv_flux = flux_id(fv_flux)
    cfg.blending = 1 if blending else 0
    cfg.precision = PRECISION_FP32_MIXED if str(precision).lower() in ("fp32", "fp32_mixed", "mixed") else PRECISION_FP64
    cfg.sutherland = 1 if sutherland else 0
    cfg.geometry_layout = int(geometry_layout)
    cfg.gamma, cfg.Pr, cfg.R_gas, cfg.mu, cfg.mu0 = gamma, Pr, R_gas, mu, mu0
    cfg.mu_bulk, cfg.T0, cfg.Ts = mu_bulk, T0, Ts
    cfg.alpha_max, cfg.alpha_min, cfg.sharpness = alpha_max, alpha_min, sharpness
    cfg.modal_threshold = modal_threshold
    cfg.volume_staging = int(volume_staging)
    cfg.mixed_blended_fp32 = 1 if mixed_blended_fp32 else 0
    cfg.mixed_flux_no_perturbation = 1 if mixed_flux_no_perturbation else 0
    if state_offset is not None:
        for i, v in enumerate(state_offset):
            cfg.state_offset[i] = float(v)
    return cfg


class LteTable(C.Structure):
    """thx_lte_table: six-plane Helmholtz table (host pointers)."""
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("rho_grid", C.POINTER(C.c_double)),
                ("T_grid", C.POINTER(C.c_double)), ("e_grid", C.POINTER(C.c_double)),
                ("planes", C.POINTER(C.c_double)), ("inverse", C.POINTER(C.c_double))]


class IdgParams(C.Structure):
    """thx_idg_params: synthetic ideal-dissociating gas."""
    _fields_ = [("R", C.c_double), ("rho_d", C.c_double), ("theta_d", C.c_double),
                ("mu0", C.c_double), ("T0", C.c_double), ("Pr", C.c_double)]


STATUS_NONPOSITIVE = 1
STATUS_NONFINITE = 2
STATUS_LAUNCH = 4
STATUS_EOS = 8
STATUS_FACE_TABLE = 16
STATUS_TIMEOUT = 32
