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
    ]


class Geometry(C.Structure):
    _fields_ = [
        ("dim", C.c_int32), ("order", C.c_int32), ("num_elements", C.c_int32),
        ("num_faces", C.c_int32),
        ("jac", C.POINTER(C.c_double)), ("metric", C.POINTER(C.c_double)),
        ("face_elem", C.POINTER(C.c_int32)), ("face_lface", C.POINTER(C.c_int32)),
        ("face_normal", C.POINTER(C.c_double)), ("face_wminus", C.POINTER(C.c_double)),
        ("face_wplus", C.POINTER(C.c_double)),
    ]


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
                geometry_layout=0, state_offset=None):
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
