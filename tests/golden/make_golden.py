"""Generates the golden fixtures in tests/golden/ from the REFERENCE's own code.

The reference (annemiekie/BlackTracer) ships no tests and no golden vectors,
so these fixtures are this build's: outputs of the reference's own integrator
and grid builder, compiled in place from the reference tree by
``make -C oracle ref`` (oracle/ref_harness.cpp), on seeded inputs.  They let
the tests check the CPU restatement and the GPU library where the reference
tree is absent (the GPU box).

    python tests/golden/make_golden.py      # needs oracle/_ref/libbtref.so
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import oracle  # noqa: E402
from parity import CAMERAS, oracle_camera, seeded_rays  # noqa: E402

# (name, maxlevel, startlevel, angle, camera)
GRIDS = [
    ("g_c1_l6u", 6, 6, True, "c1"),     # uniform (start == max): no T-vertices
    ("g_c2_l7s4", 7, 4, True, "c2"),    # adaptive, full sphere
    ("g_c2_l7s4h", 7, 4, False, "c2"),  # adaptive, half grid (equatorial symmetry)
    ("g_c5_l7s5", 7, 5, True, "c5"),
]


def main():
    oracle.build(with_ref=True)
    assert oracle.have_ref(), "reference harness not built"
    for idx, name in enumerate(sorted(CAMERAS)):
        cam, a = oracle_camera(oracle, name, ref=True)
        th, ph = seeded_rays(1500, seed=20261203 + idx)
        to, po, st, _ = oracle.integrate_rays(cam, a, th, ph, ref=True, nthreads=8)
        np.savez_compressed(os.path.join(HERE, f"rays_{name}.npz"), cam=cam, a=a,
                            theta=th, phi=ph, theta_out=to, phi_out=po, steps=st)
        print("rays", name, (st > 0).sum(), "integrated")
    for name, ml, sl, ang, camname in GRIDS:
        cam, a = oracle_camera(oracle, camname, ref=True)
        g = oracle.grid_build(ml, sl, ang, cam, a, tfix=1, ref=True)
        g0 = oracle.grid_build(ml, sl, ang, cam, a, tfix=0, ref=True)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), cam=cam, a=a,
                            maxlevel=ml, startlevel=sl, angle=ang,
                            theta=g["theta"], phi=g["phi"], exists=g["exists"],
                            steps=g["steps"], blevel=g["blevel"],
                            theta_raw=g0["theta"], phi_raw=g0["phi"])
        print("grid", name, g["N"], g["M"], int(g["exists"].sum()), "vertices")


if __name__ == "__main__":
    main()
