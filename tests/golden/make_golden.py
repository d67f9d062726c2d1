"""Generate tests/golden/*.npz from the reference's own kernels.

Runs here only (it needs oracle/_ref/libthx_ref.so, built by `make -C oracle ref`
from the reference headers).  Each fixture stores the mesh spec, the
configuration, the input state and the reference RHS; tests/test_oracle.py
checks the oracle restatement against them on any machine.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as O  # noqa: E402
from theseus_b200._abi import make_config  # noqa: E402
from theseus_b200 import cases  # noqa: E402

CASES = [
    # name, dim, order, n, lo, hi, cfg kwargs, state
    ("euler2d_chan_roe_vortex", 2, 3, (6, 5), (-5.0, -5.0), (5.0, 5.0),
     dict(volume_flux="chandrashekar", surface_flux="roe"), "vortex"),
    ("euler2d_ranocha_hll_p4", 2, 4, (4, 3), (-1.0, -0.5), (1.5, 1.0),
     dict(volume_flux="ranocha", surface_flux="hll"), "perturbed"),
    ("euler3d_pirozzoli_llf_p2", 3, 2, (3, 2, 3), (-1.0, -0.5, -0.75), (1.5, 1.0, 1.25),
     dict(volume_flux="pirozzoli", surface_flux="llf"), "perturbed"),
    ("ns3d_ranocha_hll_tgv_p3", 3, 3, (3, 3, 3), (0.0, 0.0, 0.0), (2 * np.pi,) * 3,
     dict(flow="ns", volume_flux="ranocha", surface_flux="hll", mu=1.0 / 160, Pr=0.71), "tgv"),
    ("ns2d_chan_chan_p3", 2, 3, (4, 4), (-1.0, -1.0), (1.0, 1.0),
     dict(flow="ns", volume_flux="chandrashekar", surface_flux="chandrashekar", mu=0.01), "perturbed"),
    ("euler2d_blend_sedov_p3", 2, 3, (8, 8), (-1.0, -1.0), (1.0, 1.0),
     dict(volume_flux="chandrashekar", surface_flux="llf", fv_flux="llf", blending=True), "sedov"),
    ("euler3d_blend_sedov_p2", 3, 2, (4, 4, 4), (-1.0, -1.0, -1.0), (1.0, 1.0, 1.0),
     dict(volume_flux="chandrashekar", surface_flux="llf", fv_flux="llf", blending=True), "sedov"),
]


def state(kind, m):
    if kind == "vortex":
        return cases.isentropic_vortex(m.coords, strength=5.0)
    if kind == "tgv":
        return cases.taylor_green(m.coords, mach=0.1, noise=1e-6, seed=0)
    if kind == "sedov":
        return cases.sedov(m.coords, width=0.05)
    return cases.perturbed_uniform(m.state_shape(), m.dim, seed=4, amp=0.2)


def main():
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libthx_ref.so missing: run `make -C oracle ref` first")
    for name, dim, order, n, lo, hi, kw, kind in CASES:
        m = O.box_mesh(dim, order, n, lo, hi)
        cfg = make_config(**kw)
        u = state(kind, m)
        alpha = None
        if kw.get("blending"):
            alpha, _ = O.blending(m, cfg, u)
        du = O.ref_rhs(m, cfg, u, alpha=alpha)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), dim=dim, order=order,
                            n=np.array(n), lo=np.array(lo), hi=np.array(hi),
                            cfg=np.frombuffer(bytes(cfg), dtype=np.uint8), u=u, dudt=du,
                            alpha=alpha if alpha is not None else np.zeros(0))
        print(name, du.shape)


if __name__ == "__main__":
    main()


def pointwise():
    """Reference pointwise fluxes, entropy variables and viscous fluxes."""
    rng = np.random.default_rng(2024)
    cfg = make_config(mu=0.013, Pr=0.71)
    rows = []
    for dim in (2, 3):
        for k in range(8):
            def st():
                rho = np.array(0.5 + rng.random())
                vel = [np.array(rng.uniform(-1, 1)) for _ in range(dim)]
                p = np.array(0.3 + rng.random())
                return cases.conserved(rho, vel, p, 1.4).ravel()
            q1, q2 = st(), st()
            if k == 0:
                q2 = q1 * (1 + 1e-7)  # log-mean series branch
            m1, m2, n = rng.uniform(-1, 1, dim), rng.uniform(-1, 1, dim), rng.uniform(-1, 1, dim)
            dprim = rng.uniform(-1, 1, dim * (dim + 2))
            vols = np.array([O.volume_flux(f, cfg, dim, q1, q2, m1, m2, use_ref=True) for f in range(6)])
            faces = np.array([O.face_flux(f, cfg, dim, q1, q2, n, use_ref=True) for f in range(6)])
            ent = O.entropy_vars(cfg, dim, q1, use_ref=True)
            vis = O.viscous_flux(cfg, dim, q1, dprim, use_ref=True)
            rows.append(dict(dim=dim, q1=q1, q2=q2, m1=m1, m2=m2, n=n, dprim=dprim, vol=vols,
                             face=faces, ent=ent, vis=vis))
    out = {}
    for i, r in enumerate(rows):
        for k, v in r.items():
            out[f"{i}_{k}"] = v
    out["count"] = len(rows)
    out["cfg"] = np.frombuffer(bytes(cfg), dtype=np.uint8)
    np.savez_compressed(os.path.join(HERE, "pointwise.npz"), **out)
    print("pointwise", len(rows))


def lte():
    """Reference LTE Helmholtz RHS (LTEEC, Euler and Navier-Stokes) on a 64x128
    synthetic ideal-dissociating-gas table rebuilt by the oracle from its
    parameters, plus reference point evaluations, recoveries and fluxes."""
    tab = O.LteTable(64, 128, (-6.0, 1.0), (2.3, 4.3))
    for name, flow, order, n in [("lte_euler_tgv_p2", "euler", 2, (3, 3, 2)),
                                 ("lte_ns_tgv_p3", "ns", 3, (2, 2, 2))]:
        m = O.box_mesh(3, order, n, (0.0,) * 3, (2 * np.pi,) * 3)
        cfg = make_config(flow=flow, volume_flux="lteec", surface_flux="lteec", mu=1e-4)
        u = cases.lte_taylor_green(m.coords)
        du = O.rhs_lte(m, cfg, tab, u, use_ref=True)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), order=order, n=np.array(n),
                            cfg=np.frombuffer(bytes(cfg), dtype=np.uint8), u=u, dudt=du,
                            table=np.array([64, 128, -6.0, 1.0, 2.3, 4.3]))
        print(name, du.shape)
    rng = np.random.default_rng(7)
    pts, recs, fl = [], [], []
    cfg = make_config(volume_flux="lteec", surface_flux="lteec")
    for k in range(12):
        rho = 10 ** rng.uniform(-5.5, 0.5)
        T = 10 ** rng.uniform(2.4, 4.2)
        v = O.lte_point(tab, rho, T, use_ref=True)
        pts.append([rho, T] + list(v))
        Tr, st = O.lte_temperature(tab, rho, v[1], use_ref=True)
        recs.append([rho, v[1], Tr, st])
    for k in range(8):
        def st():
            rho = 0.01 * (1 + 0.2 * rng.random())
            T = 3000.0 * (1 + 0.3 * rng.random())
            u = rng.uniform(-300, 300, 3)
            e = O.lte_point(tab, rho, T)[1]
            return np.array([rho, rho * u[0], rho * u[1], rho * u[2], rho * e + 0.5 * rho * (u @ u)])
        q1, q2 = st(), st()
        d1, d2 = rng.uniform(-1, 1, 3), rng.uniform(-1, 1, 3)
        for face in (0, 1):
            F = O.lte_flux(tab, cfg, 3, face, q1, q2, d1, d2, use_ref=True)
            fl.append(np.concatenate([[face], q1, q2, d1, d2, F]))
    np.savez_compressed(os.path.join(HERE, "lte_pointwise.npz"), points=np.array(pts),
                        recoveries=np.array(recs), fluxes=np.array(fl),
                        table=np.array([64, 128, -6.0, 1.0, 2.3, 4.3]))
    print("lte_pointwise", len(pts), len(fl))


if __name__ == "__main__":
    pointwise()
    lte()
