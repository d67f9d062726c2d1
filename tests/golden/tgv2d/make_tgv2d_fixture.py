"""Extract the reference's 2-D Taylor-Green golden (TestCases/GoldenData/
TaylorGreenVortex2D/Cycle000100/proc00000{0,1}.vtu: the reference's CPU run of
TestCases/NavierStokes/2D/TaylorGreenVortex/config.json on its Gmsh mesh,
p=3, Chandrashekar fluxes, mu = 6.25e-4, Ma 0.08, blending compiled in,
dt=1e-4, 100 steps, two ranks) and the mesh it ran on
(TaylorGreenVortex2D.msh: 32 x 32 transfinite quads on [-pi,pi]^2, periodic)
into tests/golden/tgv2d/tgv2d_p3_100.npz: the mesh as node coordinates, quad
vertex ids and periodic node pairs, and per golden point the element centre,
the point, density, pressure and velocity.  Run from the repository root with
the reference tree at REF."""
import base64
import os
import re
import sys

import numpy as np

REF = os.environ.get("REF")
if not REF:
    sys.exit("set REF to the root of the reference tree")
OUT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(OUT, "..", "..", ".."))
from theseus_b200.gmsh import read_gmsh  # noqa: E402

NODES = 16


def arrays(path):
    text = open(path).read()
    out = {}
    for m in re.finditer(r'<DataArray([^>]*)>\s*([A-Za-z0-9+/=]+)\s*</DataArray>', text):
        attrs, blob = m.group(1), m.group(2)
        name = re.search(r'Name="([^"]*)"', attrs)
        name = name.group(1) if name else "Points"
        kind = re.search(r'type="([^"]*)"', attrs).group(1)
        ncomp = int(re.search(r'NumberOfComponents="(\d+)"', attrs).group(1)) \
            if "NumberOfComponents" in attrs else 1
        nbytes = int(np.frombuffer(base64.b64decode(blob[:8]), "<u4")[0])
        raw = base64.b64decode(blob[8:])[:nbytes]
        a = np.frombuffer(raw, {"Float64": "<f8", "Int32": "<i4", "UInt8": "u1"}[kind])
        out[name] = a.reshape(-1, ncomp) if ncomp > 1 else a
    return out


def main():
    src = os.path.join(REF, "TestCases", "GoldenData", "TaylorGreenVortex2D", "Cycle000100")
    parts = [arrays(os.path.join(src, f"proc00000{r}.vtu")) for r in (0, 1)]
    pts = np.concatenate([p["Points"][:, :2] for p in parts])
    centre = np.repeat(pts.reshape(-1, NODES, 2).mean(axis=1), NODES, axis=0)
    f = {k: np.concatenate([p[k] for p in parts]) for k in ("Density", "Pressure", "Velocity")}
    nodes, quads, lines, periodic = read_gmsh(os.path.join(
        REF, "TestCases", "NavierStokes", "2D", "TaylorGreenVortex", "TaylorGreenVortex2D.msh"))
    ids = np.array(sorted(nodes))
    np.savez_compressed(os.path.join(OUT, "tgv2d_p3_100.npz"),
                        node_id=ids, node_xy=np.array([nodes[i] for i in ids]),
                        quads=np.array([q[1:] for q in quads], np.int64),
                        periodic=np.array(sorted(periodic.items()), np.int64),
                        center=centre, point=pts, density=f["Density"], pressure=f["Pressure"],
                        velocity=f["Velocity"])
    print("wrote tgv2d_p3_100.npz:", len(quads), "quads,", pts.shape[0], "points")


if __name__ == "__main__":
    sys.exit(main())
