"""Synthetic workloads: initial states on periodic boxes, in the byNODES layout.

The reference's benchmark configurations name no public data set; these seeded
generators are the inputs.  Every function returns u[eq][elem][node] (float64)
given node coordinates coords[dim][elem][node].
"""
import numpy as np


def conserved(rho, vel, p, gamma):
    """Primitive -> conserved (include/EOS.hpp:288-305)."""
    dim = len(vel)
    out = np.empty((dim + 2,) + np.shape(rho))
    out[0] = rho
    ke = np.zeros_like(rho)
    for d in range(dim):
        out[1 + d] = rho * vel[d]
        ke = ke + vel[d] * vel[d]
    out[dim + 1] = p / (gamma - 1.0) + 0.5 * rho * ke
    return out


def isentropic_vortex(coords, gamma=1.4, strength=5.0, center=(0.0, 0.0), rho_inf=1.0,
                      u_inf=(1.0, 1.0), p_inf=1.0):
    """Shu's isentropic vortex on a uniform flow (published formula):
    du = -b/(2 pi) y' e^{(1-r^2)/2}, dv = b/(2 pi) x' e^{(1-r^2)/2},
    T = T_inf - (gamma-1) b^2/(8 gamma pi^2) e^{1-r^2}, rho ~ T^{1/(gamma-1)}."""
    x = coords[0] - center[0]
    y = coords[1] - center[1]
    r2 = x * x + y * y
    T_inf = p_inf / rho_inf
    f = np.exp(0.5 * (1.0 - r2))
    du = -strength / (2 * np.pi) * y * f
    dv = strength / (2 * np.pi) * x * f
    T = T_inf - (gamma - 1.0) * strength ** 2 / (8.0 * gamma * np.pi ** 2) * (f * f)
    rho = rho_inf * (T / T_inf) ** (1.0 / (gamma - 1.0))
    p = rho * T
    vel = [u_inf[0] + du, u_inf[1] + dv]
    if coords.shape[0] == 3:
        vel.append(np.zeros_like(rho))
    return conserved(rho, vel, p, gamma)


def taylor_green(coords, gamma=1.4, mach=0.1, noise=0.0, seed=0):
    """Taylor-Green vortex as include/StateInit.hpp:139-161, plus an optional
    seeded uniform velocity perturbation of amplitude `noise`."""
    x, y, z = coords[0], coords[1], coords[2]
    p0 = 1.0 / (gamma * mach * mach)
    rho = np.ones_like(x)
    u = np.sin(x) * np.cos(y) * np.cos(z)
    v = -np.cos(x) * np.sin(y) * np.cos(z)
    w = np.zeros_like(x)
    if noise:
        rng = np.random.default_rng(seed)
        u = u + noise * rng.uniform(-1, 1, size=x.shape)
        v = v + noise * rng.uniform(-1, 1, size=x.shape)
        w = w + noise * rng.uniform(-1, 1, size=x.shape)
    p = p0 + 1.0 / 16.0 * (np.cos(2 * x) + np.cos(2 * y)) * (np.cos(2 * z) + 2.0)
    return conserved(rho, [u, v, w], p, gamma)


def sedov(coords, gamma=1.4, rho0=1.0, p0=1e-5, energy=1.0, width=0.05):
    """Sedov-type blast: uniform rest state plus `energy` deposited as a
    normalised Gaussian of standard deviation `width` at the origin."""
    dim = coords.shape[0]
    r2 = sum(coords[d] ** 2 for d in range(dim))
    g = np.exp(-0.5 * r2 / width ** 2) / ((2 * np.pi) ** (dim / 2) * width ** dim)
    rho = rho0 * np.ones_like(r2)
    out = conserved(rho, [np.zeros_like(r2)] * dim, p0 * np.ones_like(r2), gamma)
    out[dim + 1] += energy * g
    return out


def perturbed_uniform(shape_eq_e_nd, dim, seed=0, amp=0.1, gamma=1.4):
    """Smooth-ish random state around rho=1, u=(0.3,-0.2,0.1), p=1 for parity tests."""
    rng = np.random.default_rng(seed)
    _, ne, nd = shape_eq_e_nd
    rho = 1.0 + amp * rng.uniform(-1, 1, (ne, nd))
    vel = [c + amp * rng.uniform(-1, 1, (ne, nd)) for c in (0.3, -0.2, 0.1)[:dim]]
    p = 1.0 + amp * rng.uniform(-1, 1, (ne, nd))
    return conserved(rho, vel, p, gamma)


# O2-like ideal dissociating gas of the LTE benchmark table (gas constant of
# the molecule, characteristic density, dissociation temperature).
IDG_O2 = dict(R=8.314462618 / 0.0319988, rho_d=1.5e5, theta_d=59500.0)


def idg_energy(rho, T, R, rho_d, theta_d):
    """Specific internal energy of the ideal dissociating gas, e = 3RT + alpha R theta_d,
    alpha^2/(1-alpha) = (rho_d/rho) exp(-theta_d/T)."""
    K = (rho_d / rho) * np.exp(-theta_d / T)
    alpha = 2.0 / (1.0 + np.sqrt(1.0 + 4.0 / K))
    return 3.0 * R * T + alpha * R * theta_d


def lte_taylor_green(coords, rho0=0.01, T0=3000.0, U0=300.0, dT=0.05, gas=None):
    """Taylor-Green velocity field (include/StateInit.hpp:139-161 shape) on a uniform
    density, with the temperature carrying the TGV pressure pattern:
    T = T0 (1 + dT/16 (cos 2x + cos 2y)(cos 2z + 2))."""
    g = gas or IDG_O2
    x, y, z = coords[0], coords[1], coords[2]
    u = U0 * np.sin(x) * np.cos(y) * np.cos(z)
    v = -U0 * np.cos(x) * np.sin(y) * np.cos(z)
    w = np.zeros_like(x)
    T = T0 * (1.0 + dT / 16.0 * (np.cos(2 * x) + np.cos(2 * y)) * (np.cos(2 * z) + 2.0))
    rho = rho0 * np.ones_like(x)
    e = idg_energy(rho, T, g["R"], g["rho_d"], g["theta_d"])
    out = np.empty((5,) + x.shape)
    out[0] = rho
    out[1], out[2], out[3] = rho * u, rho * v, rho * w
    out[4] = rho * e + 0.5 * rho * (u * u + v * v + w * w)
    return out
