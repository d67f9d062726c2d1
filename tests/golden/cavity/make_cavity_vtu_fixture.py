"""Extract the reference's lid-driven-cavity golden solution after 4000 steps
(TestCases/GoldenData/LidDrivenCavity/Cycle004000/proc00000{0,1}.vtu: the
reference's CPU run of TestCases/NavierStokes/2D/LidDrivenCavity/config.json,
p=3, Chandrashekar fluxes, subcell blending compiled in, dt=1e-4, two ranks)
into tests/golden/cavity/ldc_p3_4000.npz.

The VTU files hold each element's own nodes as points (not merged), in
element blocks of (p+1)^2 points, with binary arrays written as base64 of a
uint32 byte count followed by the data.  Stored per point: the element
centre (mean of its block), the point, density, pressure, velocity and the
blending coefficient.  Run from the repository root with the reference tree
at REF."""
import base64
import os
import re
import sys

import numpy as np

REF = os.environ.get("REF")
if not REF:
    sys.exit("set REF to the root of the reference tree")
SRC = os.path.join(REF, "TestCases", "GoldenData", "LidDrivenCavity", "Cycle004000")
OUT = os.path.dirname(os.path.abspath(__file__))
NODES = 16  # (p+1)^2 at p = 3


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
        dt = {"Float64": "<f8", "Int32": "<i4", "UInt8": "u1"}[kind]
        a = np.frombuffer(raw, dt)
        out[name] = a.reshape(-1, ncomp) if ncomp > 1 else a
    return out


def main():
    parts = [arrays(os.path.join(SRC, f"proc00000{r}.vtu")) for r in (0, 1)]
    pts = np.concatenate([p["Points"][:, :2] for p in parts])
    centre = np.repeat(pts.reshape(-1, NODES, 2).mean(axis=1), NODES, axis=0)
    fields = {k: np.concatenate([p[k] for p in parts])
              for k in ("Density", "Pressure", "Velocity", "Blending Coeff")}
    np.savez_compressed(os.path.join(OUT, "ldc_p3_4000.npz"), center=centre, point=pts,
                        density=fields["Density"], pressure=fields["Pressure"],
                        velocity=fields["Velocity"], alpha=fields["Blending Coeff"])
    print("wrote ldc_p3_4000.npz", pts.shape[0], "points; max blending coefficient",
          float(fields["Blending Coeff"].max()))


if __name__ == "__main__":
    sys.exit(main())
