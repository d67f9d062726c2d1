"""Extract the lid-driven-cavity golden fields of the reference's
numerical-flux regression (TestCases/GoldenData/NumericalFluxes/
cpg-{hll,roe}-cavity-{000010,000020}.npz: the reference's CPU run, 2-D
Navier-Stokes, p=2, 16 x 16 quads on [0,2]^2, four adiabatic no-slip walls
with the lid at unit velocity, subcell blending, dt=1e-4) into the compact
fixtures tests/golden/cavity/{hll,roe}_{10,20}.npz.

Each golden entry is one DG node of one visualisation subcell: keys are the
subcell centre (x, y) and the node (x, y); fields are density, pressure and
velocity there.  Every other entry is kept (the file stays small; every
element and every node position is still represented).  Run from the
repository root with the reference tree at REF.
"""
import os
import sys

import numpy as np

REF = os.environ.get("REF")
if not REF:
    sys.exit("set REF to the root of the reference tree")
SRC = os.path.join(REF, "TestCases", "GoldenData", "NumericalFluxes")
OUT = os.path.dirname(os.path.abspath(__file__))


def main():
    for flux in ("hll", "roe"):
        for cycle in (10, 20):
            src = os.path.join(SRC, f"cpg-{flux}-cavity-{cycle:06d}.npz")
            with np.load(src, allow_pickle=False) as d:
                keep = slice(0, None, 2)
                c = d["coordinates"][keep]
                np.savez_compressed(os.path.join(OUT, f"{flux}_{cycle}.npz"),
                                    center=c[:, 0:2], point=c[:, 3:5],
                                    density=d["Density"][keep], pressure=d["Pressure"][keep],
                                    velocity=d["Velocity"][keep])
            print("wrote", f"{flux}_{cycle}.npz")


if __name__ == "__main__":
    sys.exit(main())
