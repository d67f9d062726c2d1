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


if __name__ == "__main__":
    pointwise()
