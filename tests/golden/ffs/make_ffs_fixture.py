"""Extract the reference's forward-facing-step golden (TestCases/GoldenData/
ForwardFacingStep.tgz, Cycle000100/proc00000{0,1}.vtu: the reference's run of
TestCases/Euler/2D/ForwardFacingStep/config.json through
tests/recipes/regression/golden-step.sh -- the Gmsh mesh refined once, p=3,
Chandrashekar fluxes, blending, supersonic inflow/outflow and slip walls,
fixed dt 1e-4, 100 cycles, two ranks) and its mesh into
tests/golden/ffs/ffs_p3_100.npz: the mesh as node ids and coordinates, quad
vertex ids and named boundary lines, and for a subset of the golden's
elements -- every element with a non-zero blending coefficient and every
32nd other one, in the file's element order -- the points, element centres,
density, pressure, velocity and blending coefficient.  Run from the
repository root with the reference tree at REF."""
import base64
import io
import os
import re
import sys
import tarfile

import numpy as np

REF = os.environ.get("REF")
if not REF:
    sys.exit("set REF to the root of the reference tree")
OUT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(OUT, "..", "..", ".."))
from theseus_b200.gmsh import read_gmsh  # noqa: E402

NODES = 16
STRIDE = 32


def arrays(text):
    """The base64 (uint32 byte-count header) data arrays of a VTU piece."""
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
    parts = []
    with tarfile.open(os.path.join(REF, "TestCases", "GoldenData", "ForwardFacingStep.tgz")) as tar:
        for r in (0, 1):
            f = tar.extractfile(f"ForwardFacingStep/Cycle000100/proc00000{r}.vtu")
            parts.append(arrays(io.TextIOWrapper(f).read()))
    pts = np.concatenate([p["Points"][:, :2] for p in parts]).reshape(-1, NODES, 2)
    f = {k: np.concatenate([p[k] for p in parts]) for k in ("Density", "Pressure", "Velocity", "Blending Coeff")}
    f = {k: v.reshape((-1, NODES) + v.shape[1:]) for k, v in f.items()}
    blended = f["Blending Coeff"].max(axis=1) > 0.0
    keep = blended | (np.arange(len(pts)) % STRIDE == 0)
    nodes, quads, lines, periodic = read_gmsh(os.path.join(
        REF, "TestCases", "Euler", "2D", "ForwardFacingStep", "ForwardFacingStep.msh"))
    assert not periodic
    ids = np.array(sorted(nodes))
    names = sorted({name for name, _, _ in lines})
    np.savez_compressed(os.path.join(OUT, "ffs_p3_100.npz"),
                        node_id=ids, node_xy=np.array([nodes[i] for i in ids]),
                        quads=np.array([q[1:] for q in quads], np.int64),
                        line_names=np.array(names),
                        lines=np.array([(names.index(n), a, b) for n, a, b in lines], np.int64),
                        num_golden_elements=len(pts),
                        center=np.repeat(pts[keep].mean(axis=1), NODES, axis=0),
                        point=pts[keep].reshape(-1, 2),
                        density=f["Density"][keep].reshape(-1), pressure=f["Pressure"][keep].reshape(-1),
                        velocity=f["Velocity"][keep].reshape(-1, 2),
                        blending=f["Blending Coeff"][keep].reshape(-1))
    print("wrote ffs_p3_100.npz:", len(quads), "quads,", int(keep.sum()), "of", len(pts), "golden elements,",
          int(blended.sum()), "blended")


if __name__ == "__main__":
    sys.exit(main())
