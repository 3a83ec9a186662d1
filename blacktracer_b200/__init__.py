"""B200-native BlackTracer hot path: Kerr geodesic grid integration and the
per-pixel map, behind the reference's own Grid / Camera / BlackHole /
StarProcessor / makeImage interfaces.

Compute runs in hand-written sm_100a CUDA (libblacktracer_b200.so, C ABI in
include/blacktracer.h).  This package is the Python host mirror of the
reference interfaces; device buffers are torch CUDA tensors.
"""
from ._lib import (BtError, PRECISION_FAST, PRECISION_MIXED, PRECISION_PLAIN,  # noqa: F401
                   RAY_CAPTURED,
                   RAY_ESCAPED, RAY_MAXSTEP, RAY_NONCONVERGED, lib)
from .host import (BlackHole, Camera, Grid, GridSet, IntegOpts, grid_dims,  # noqa: F401
                   integrate_rays, integrate_rays_host)

from .render import (Blend, Environment, Renderer, StarProcessor, Trails,  # noqa: F401
                     Viewer, psf_airy)
from .serve import Server  # noqa: F401
from .cache import (GridFile, psh_build, read_grid_file, read_star_file,  # noqa: F401
                    write_grid_file, write_star_file)

__all__ = ["Environment", "GridFile", "Trails", "Renderer", "Server", "StarProcessor", "Viewer",
           "BlackHole", "psh_build", "read_grid_file", "write_grid_file", "read_star_file",
           "write_star_file",
           "Camera", "Grid",
           "GridSet", "IntegOpts", "grid_dims", "integrate_rays",
           "integrate_rays_host", "BtError", "lib"]
