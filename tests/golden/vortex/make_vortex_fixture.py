"""Extract the reference's isentropic-vortex golden (TestCases/GoldenData/
IsentropicVortex/Cycle000500/proc00000{0,1}.vtu: the reference's CPU run of
TestCases/Euler/2D/IsentropicVortex/config.json -- p=3, Chandrashekar
fluxes, blending compiled in, variable dt with cfl 0.2, 500 steps, two
ranks -- on IsentropicVortex.mesh refined three times) and the base mesh it
ran on (3 x 3 periodic quads with first-order L2 nodes) into
tests/golden/vortex/vortex_p3_500.npz: the mesh as element vertex ids, the
vertex count and per-element corner coordinates, and per golden point the
element centre, the point, density, pressure, velocity and blending
coefficient.  Run from the repository root with the reference tree at REF."""
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
from theseus_b200.mfem_mesh import read_mfem_mesh  # noqa: E402

NODES = 16


def arrays(path):
    """The base64 (uint32 byte-count header) data arrays of a VTU piece."""
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
    src = os.path.join(REF, "TestCases", "GoldenData", "IsentropicVortex", "Cycle000500")
    parts = [arrays(os.path.join(src, f"proc00000{r}.vtu")) for r in (0, 1)]
    pts = np.concatenate([p["Points"][:, :2] for p in parts])
    centre = np.repeat(pts.reshape(-1, NODES, 2).mean(axis=1), NODES, axis=0)
    f = {k: np.concatenate([p[k] for p in parts]) for k in ("Density", "Pressure", "Velocity", "Blending Coeff")}
    _, elems, bdr, nv, dofs = read_mfem_mesh(os.path.join(
        REF, "TestCases", "Euler", "2D", "IsentropicVortex", "IsentropicVortex.mesh"))
    assert not bdr
    np.savez_compressed(os.path.join(OUT, "vortex_p3_500.npz"),
                        elements=np.array(elems, np.int64), num_vertices=nv, dofs=dofs,
                        center=centre, point=pts, density=f["Density"], pressure=f["Pressure"],
                        velocity=f["Velocity"], blending=f["Blending Coeff"])
    print("wrote vortex_p3_500.npz:", len(elems), "base quads,", pts.shape[0], "points")


if __name__ == "__main__":
    sys.exit(main())
