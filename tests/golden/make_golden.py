"""Generates the golden fixtures in tests/golden/ from the REFERENCE's own code.

The reference (annemiekie/BlackTracer) ships no tests and no golden vectors,
so these fixtures are this build's: outputs of the reference's own integrator
and grid builder, compiled in place from the reference tree by
``make -C oracle ref`` (oracle/ref_harness.cpp), on seeded inputs.  They let
the tests check the CPU restatement and the GPU library where the reference
tree is absent (the GPU box).

    python tests/golden/make_golden.py        # needs oracle/_ref/libbtref.so
    python tests/golden/make_golden.py cache  # only the cache-file and view fixtures
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


# Cache files written by the reference through cereal, and its perspective
# views.  The reference's perfect hash is seeded with the time, so a new
# generation writes different (equally valid) tables.
CACHE_GRID = ("ref_c2_l6s4", 6, 4, True, "c2")
CACHE_STARS = ("ref_stars_l6", 300, 6)
VIEWS = [  # (view angle, offset up, offset right, W, H)
    (np.pi / 2, 0.0, 0.0, 64, 32),
    (1.2, 0.3, 1.0, 96, 48),
    (0.7, -0.5, -2.0, 33, 17),
]


def cache_fixtures():
    oracle.build(with_ref=True)
    assert oracle.have_ref(), "reference harness not built"
    name, ml, sl, ang, camname = CACHE_GRID
    cam, a = oracle_camera(oracle, camname, ref=True)
    path = os.path.join(HERE, f"{name}.grid")
    n = oracle.ref_grid_file_write(path, ml, sl, ang, cam, a)
    d = oracle.ref_grid_file_decode(path)
    np.savez_compressed(os.path.join(HERE, f"{name}_decoded.npz"), cam=cam, a=a, maxlevel=ml,
                        startlevel=sl, angle=ang, entries=n,
                        **{k: d[k] for k in ("N", "M", "hash_width", "offset_width",
                                             "hash_table", "offset_table", "pos_tag",
                                             "dense")})
    print("grid file", name, n, "entries", os.path.getsize(path), "bytes")
    sname, nstars, tl = CACHE_STARS
    from parity import synthetic_stars
    stars = synthetic_stars(nstars, seed=77)
    pos, mg, tree = oracle.ref_star_tree(*stars, tl)
    spath = os.path.join(HERE, f"{sname}.star")
    oracle.ref_stars_file_write(spath, pos, mg, tree, tl)
    np.savez_compressed(os.path.join(HERE, f"{sname}.npz"), pos=pos, mag=mg, tree=tree,
                        tree_level=tl)
    print("star file", sname, nstars, "stars", os.path.getsize(spath), "bytes")
    views = {}
    for k, (ang_, up, right, W, H) in enumerate(VIEWS):
        views[f"view{k}"] = oracle.ref_view_camera(ang_, up, right, W, H)
        views[f"args{k}"] = np.array([ang_, up, right, W, H], np.float64)
    np.savez_compressed(os.path.join(HERE, "ref_views.npz"), **views)
    print("views", len(VIEWS))


if __name__ == "__main__":
    if sys.argv[1:] == ["cache"]:
        cache_fixtures()
    else:
        main()
        cache_fixtures()
