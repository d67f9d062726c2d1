"""CPU: the oracle restatement against the reference.

Pins (i) the golden fixtures generated from the reference's own kernels
(tests/golden/make_golden.py), (ii) live comparisons with oracle/_ref when it
was built here, and (iii) the known-answer properties the reference's own tests
assert (tests/test_riemann_fluxes.cpp)."""
import glob
import os

import numpy as np
import pytest

import oracle as O
from theseus_b200._abi import Config, make_config
from theseus_b200 import cases

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def rel_l2(a, b):
    a = a.reshape(a.shape[0], -1)
    b = b.reshape(b.shape[0], -1)
    nb = np.sqrt((b ** 2).sum(1))
    return np.sqrt(((a - b) ** 2).sum(1)) / np.maximum(nb, 1e-12 * nb.max())


def load_cfg(raw):
    """Configuration bytes stored with a fixture; fields added later stay zero."""
    import ctypes
    cfg = Config()
    b = raw.tobytes()
    ctypes.memmove(ctypes.addressof(cfg), b, min(len(b), ctypes.sizeof(cfg)))
    return cfg


@pytest.mark.parametrize("path", sorted(p for p in glob.glob(os.path.join(GOLD, "*.npz"))
                                        if not p.endswith("pointwise.npz")
                                        and not os.path.basename(p).startswith("lte_")))
def test_oracle_matches_reference_golden(path):
    z = np.load(path)
    m = O.box_mesh(int(z["dim"]), int(z["order"]), tuple(z["n"]), tuple(z["lo"]), tuple(z["hi"]))
    cfg = load_cfg(z["cfg"])
    du, alpha, _ = O.rhs(m, cfg, z["u"], nthreads=2, want_alpha=True)
    if cfg.blending:
        assert np.array_equal(alpha, z["alpha"])
        assert (alpha > 0).any() and (alpha == 0).any()
    assert rel_l2(du, z["dudt"]).max() <= 1e-12


def test_pointwise_golden():
    z = np.load(os.path.join(GOLD, "pointwise.npz"))
    cfg = load_cfg(z["cfg"])
    for i in range(int(z["count"])):
        g = {k.split("_", 1)[1]: z[k] for k in z.files if k.startswith(f"{i}_")}
        dim = int(g["dim"])
        for f in range(6):
            v = O.volume_flux(f, cfg, dim, g["q1"], g["q2"], g["m1"], g["m2"])
            assert np.allclose(v, g["vol"][f], rtol=1e-14, atol=1e-14), (i, f)
            s = O.face_flux(f, cfg, dim, g["q1"], g["q2"], g["n"])
            assert np.allclose(s, g["face"][f], rtol=1e-13, atol=1e-14), (i, f)
        assert np.allclose(O.entropy_vars(cfg, dim, g["q1"]), g["ent"], rtol=1e-14, atol=1e-14)
        assert np.allclose(O.viscous_flux(cfg, dim, g["q1"], g["dprim"]), g["vis"], rtol=1e-14, atol=1e-15)


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built here")
@pytest.mark.parametrize("dim,flow,vol,surf,blend", [
    (2, "euler", "chandrashekar", "roe", False), (3, "ns", "ranocha", "hll", False),
    (3, "euler", "chandrashekar", "llf", True), (2, "ns", "pirozzoli", "chandrashekar", True)])
def test_oracle_matches_reference_live(dim, flow, vol, surf, blend):
    order = 3 if dim == 2 else 2
    m = O.box_mesh(dim, order, (5, 4, 3)[:dim], [-1.0] * dim, [1.5, 2.0, 1.0][:dim])
    cfg = make_config(flow=flow, volume_flux=vol, surface_flux=surf, blending=blend, mu=0.01)
    u = cases.perturbed_uniform(m.state_shape(), dim, seed=3, amp=0.3)
    du, al, _ = O.rhs(m, cfg, u, want_alpha=True)
    ref = O.ref_rhs(m, cfg, u, alpha=al if blend else None)
    assert rel_l2(du, ref).max() <= 1e-12


def _state2d(rho, u, v, p, g=1.4):
    return np.array([rho, rho * u, rho * v, p / (g - 1) + 0.5 * rho * (u * u + v * v)])


def test_tadmor_entropy_conservation():
    """ECFlux_Tadmor_2D (tests/test_riemann_fluxes.cpp:158-192,357-372), tol 1e-13."""
    cfg = make_config(Pr=0.72, R_gas=287.05, mu=0.02)
    qL = _state2d(1.0, 20.0, 3.0, 100000.0)
    qR = _state2d(1.000001, -10.0, -2.0, 90000.0)
    wL, wR = O.entropy_vars(cfg, 2, qL), O.entropy_vars(cfg, 2, qR)
    for flux in (0, 1):
        for d in range(2):
            met = np.zeros(2)
            met[d] = 1.0
            F = O.volume_flux(flux, cfg, 2, qL, qR, met, met)
            psi = qR[1 + d] - qL[1 + d]
            assert abs(F @ (wR - wL) - psi) <= 1e-13 * max(1.0, abs(psi)) * 1e3 or \
                abs(F @ (wR - wL) - psi) <= 1e-13


def test_roe_stationary_contact():
    """RoeFlux_ResolvesStationaryContact_2D (tests/test_riemann_fluxes.cpp:333-355)."""
    cfg = make_config()
    qL = _state2d(1.0, 0.0, 7.0, 100000.0)
    qR = _state2d(2.0, 0.0, 7.0, 100000.0)
    F = O.face_flux(5, cfg, 2, qL, qR, np.array([1.0, 0.0]))
    assert abs(F[0]) <= 1e-12 and abs(F[2]) <= 1e-12 and abs(F[3]) <= 1e-8
    assert abs(F[1] - 100000.0) <= 1e-8


@pytest.mark.parametrize("flux", range(6))
@pytest.mark.parametrize("dim", (2, 3))
def test_consistency_and_reversal(flux, dim):
    """RiemannFlux_Consistency / NormalReversal (tests/test_riemann_fluxes.cpp:195-250)."""
    cfg = make_config()
    rng = np.random.default_rng(flux + 10 * dim)
    q = cases.conserved(np.array(1.2), [np.array(x) for x in rng.uniform(-.5, .5, dim)],
                        np.array(0.9), 1.4).ravel()
    q2 = cases.conserved(np.array(0.8), [np.array(x) for x in rng.uniform(-.5, .5, dim)],
                         np.array(1.3), 1.4).ravel()
    n = rng.uniform(-1, 1, dim)
    # physical normal flux
    rho, m, E = q[0], q[1:1 + dim], q[-1]
    p = 0.4 * (E - 0.5 * (m @ m) / rho)
    un = (m @ n) / rho
    fn = np.concatenate([[m @ n], m * un + p * n, [(E + p) * un]])
    assert np.allclose(O.face_flux(flux, cfg, dim, q, q, n), fn, rtol=1e-13, atol=1e-13)
    assert np.allclose(O.volume_flux(flux, cfg, dim, q, q, n, n), fn, rtol=1e-13, atol=1e-13)
    a = O.face_flux(flux, cfg, dim, q, q2, n)
    b = O.face_flux(flux, cfg, dim, q2, q, -n)
    assert np.allclose(a, -b, rtol=1e-12, atol=1e-12)


def test_persson_indicator_analytic():
    """eta = 0 for fields of degree <= p-2; a pure top mode is flagged."""
    m = O.box_mesh(2, 4, (3, 3), [0.0, 0.0], [1.0, 1.0])
    cfg = make_config(blending=True)
    x, y = m.coords
    smooth = cases.conserved(np.ones_like(x), [0 * x, 0 * x], 1.0 + 0.1 * x + 0.05 * y * y, 1.4)
    a, e = O.blending(m, cfg, smooth)
    assert np.all(e < 1e-10) and np.all(a == 0)
    # rho*p alternating node to node: dominated by the highest mode
    osc = smooth.copy()
    osc[3] = 1.0 / 0.4 * (1.0 + 0.5 * (-1.0) ** np.arange(m.nd))[None, :]
    a, e = O.blending(m, cfg, osc)
    assert np.all(e > 0.5) and np.all(a == 0.5)


def test_rk3_conserves_and_threads_agree():
    m = O.box_mesh(2, 3, (5, 5), [-5.0, -5.0], [5.0, 5.0])
    cfg = make_config(volume_flux="chandrashekar", surface_flux="roe")
    u = cases.isentropic_vortex(m.coords)
    a = O.rk3_steps(m, cfg, u, 0.01, 3, nthreads=1)
    b = O.rk3_steps(m, cfg, u, 0.01, 3, nthreads=4)
    assert np.array_equal(a, b)
    x, w = O.operators(3)[:2]
    wq = np.outer(w, w).ravel()
    mass0 = (u[0] * wq * m.jac).sum()
    mass1 = (a[0] * wq * m.jac).sum()
    assert abs(mass1 - mass0) <= 1e-13 * abs(mass0)


# ---- LTE Helmholtz gas -----------------------------------------------------
def _table(spec):
    return O.LteTable(int(spec[0]), int(spec[1]), (spec[2], spec[3]), (spec[4], spec[5]))


@pytest.mark.parametrize("name", ["lte_euler_tgv_p2", "lte_ns_tgv_p3"])
def test_lte_rhs_matches_reference_golden(name):
    z = np.load(os.path.join(GOLD, name + ".npz"))
    tab = _table(z["table"])
    m = O.box_mesh(3, int(z["order"]), tuple(z["n"]), (0.0,) * 3, (2 * np.pi,) * 3)
    du = O.rhs_lte(m, load_cfg(z["cfg"]), tab, z["u"], nthreads=2)
    assert rel_l2(du, z["dudt"]).max() <= 1e-12


def test_lte_pointwise_golden():
    z = np.load(os.path.join(GOLD, "lte_pointwise.npz"))
    tab = _table(z["table"])
    for row in z["points"]:
        v = O.lte_point(tab, row[0], row[1])
        assert np.allclose(v, row[2:], rtol=1e-13, atol=0)
    for rho, e, T, st in z["recoveries"]:
        Tr, s = O.lte_temperature(tab, rho, e)
        assert s == st and abs(Tr - T) <= 1e-12 * T
    cfg = make_config(volume_flux="lteec", surface_flux="lteec")
    for row in z["fluxes"]:
        face = int(row[0])
        q1, q2, d1, d2, F = row[1:6], row[6:11], row[11:14], row[14:17], row[17:22]
        got = O.lte_flux(tab, cfg, 3, face, q1, q2, d1, d2)
        assert np.allclose(got, F, rtol=1e-12, atol=1e-12 * np.abs(F).max())


def test_lte_table_is_the_ideal_dissociating_gas():
    """Table planes reproduce p = rho R T (1+alpha), e = 3RT + alpha R theta_d, and the
    inverse table inverts e(rho, T) (include/LTEHelmholtzTableBuilder.hpp:131-218)."""
    tab = O.LteTable(32, 64, (-6.0, 1.0), (2.3, 4.3))
    R, rd, th = O.IDG_O2["R"], O.IDG_O2["rho_d"], O.IDG_O2["theta_d"]
    for i in (0, 7, 31):
        for j in (0, 20, 63):
            rho, T = tab.rho[i], tab.T[j]
            K = rd / rho * np.exp(-th / T)
            a = 2.0 / (1.0 + np.sqrt(1.0 + 4.0 / K))
            p = rho * rho * tab.planes[1, j, i]
            e = tab.planes[0, j, i] - T * tab.planes[2, j, i]
            assert abs(p - rho * R * T * (1 + a)) <= 1e-12 * p
            assert abs(e - (3 * R * T + a * R * th)) <= 1e-10 * abs(e)
    rng = np.random.default_rng(3)
    for _ in range(20):
        rho = 10 ** rng.uniform(-5.9, 0.9)
        T = 10 ** rng.uniform(2.31, 4.29)
        e = O.lte_point(tab, rho, T)[1]
        Tr, st = O.lte_temperature(tab, rho, e)
        assert st == 0 and abs(Tr - T) <= 1e-8 * T


def test_product_lte_tables_equal_oracle_tables():
    """The library's table builders (synthetic gas planes, energy grid and
    inverse table) reproduce the oracle's bit for bit."""
    import theseus_b200 as T
    for nx, ny, lr, lt in [(64, 128, (-6.0, 1.0), (2.3, 4.3)), (33, 47, (-4.0, 0.5), (2.5, 4.0))]:
        o = O.LteTable(nx, ny, lr, lt)
        p = T.HelmholtzTable.ideal_dissociating_gas(nx, ny, lr, lt, **O.IDG_O2)
        for a in ("rho", "T", "planes", "e", "inv"):
            assert np.array_equal(getattr(p, a), getattr(o, a)), a
        q = T.HelmholtzTable(o.rho, o.T, o.planes)  # inverse rebuilt from the forward planes
        assert np.array_equal(q.e, o.e) and np.array_equal(q.inv, o.inv)
