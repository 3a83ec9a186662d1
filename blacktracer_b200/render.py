"""Host mirror of the reference's map-side interfaces.

  Viewer(viewangle, offUp, offRight, pixw, pixh, sphere)   BT/Viewer.h:20-33
  StarProcessor (star list -> kd tree)                    BT/StarProcessor.h:34-64
  Distorter(grids, viewer, stars, cams) -> makeImage      BT/Distorter.h:166-176
plus the resident pieces the B200 design keeps in HBM: Environment (the
summed-area table of an environment map) and Renderer (per-resolution
scratch).  Device buffers are torch CUDA tensors; compute is the C ABI.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .host import Camera, Grid, _stream_ptr, _torch


class Viewer:
    """Camera-sky corner directions of the output pixels (BT/Viewer.h:20-33):
    the equirectangular sphere view (makeSphereView) or, with sphere=False,
    the perspective view of horizontal angle `viewangle` turned by offUp and
    offRight (makeCameraView).  viewMatrix is a ((pixh+1)*(pixw+1), 2)
    float32 CUDA tensor."""

    def __init__(self, viewangle, offUp, offRight, pixw, pixh, sphere=True, stream=None):
        torch = _torch()
        self.pixelwidth, self.pixelheight = int(pixw), int(pixh)
        self.viewAngleWide = float(viewangle)
        self.viewMatrix = torch.empty(((pixh + 1) * (pixw + 1), 2), dtype=torch.float32,
                                      device="cuda")
        if sphere:
            L.check(L.lib().bt_view_sphere(self.viewMatrix.data_ptr(), self.pixelwidth,
                                           self.pixelheight, _stream_ptr(stream)))
        else:
            self.viewAngleUp = self.pixelheight * self.viewAngleWide / self.pixelwidth
            L.check(L.lib().bt_view_camera(self.viewMatrix.data_ptr(), self.pixelwidth,
                                           self.pixelheight, self.viewAngleWide, float(offUp),
                                           float(offRight), _stream_ptr(stream)))


class Environment:
    """A resident environment map (BGR8, rows x cols, rows = cols/2)."""

    def __init__(self, bgr, stream=None):
        torch = _torch()
        if isinstance(bgr, np.ndarray):
            bgr = np.ascontiguousarray(bgr, dtype=np.uint8)
            rows, cols = bgr.shape[:2]
            ptr, on_dev = bgr.ctypes.data, 0
            self._keep = bgr
        else:
            bgr = bgr.contiguous()
            rows, cols = bgr.shape[:2]
            ptr, on_dev = bgr.data_ptr(), 1
            self._keep = bgr
        self.rows, self.cols = int(rows), int(cols)
        h = C.c_void_p()
        L.check(L.lib().bt_env_create(ptr, self.rows, self.cols, on_dev, C.byref(h),
                                      _stream_ptr(stream)))
        self._h = h

    def sat(self):
        """The summed-area table as a (rows, cols, 4) float32 CUDA tensor view."""
        torch = _torch()
        p = C.c_void_p()
        L.check(L.lib().bt_env_sat(self._h, C.byref(p), None, None))
        return _device_view(p.value, (self.rows, self.cols, 4), torch.float32)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None:
            try:
                L.lib().bt_env_destroy(h)
            except Exception:
                pass
            self._h = None


def _device_view(ptr, shape, dtype):
    """A torch tensor aliasing library-owned device memory (copy it if it must
    outlive the owner)."""
    torch = _torch()

    class _Arr:
        __cuda_array_interface__ = {
            "shape": tuple(shape), "typestr": {torch.float32: "<f4", torch.int32: "<i4",
                                               torch.uint8: "|u1"}[dtype],
            "data": (ptr, False), "version": 2, "strides": None}
    return torch.as_tensor(_Arr(), device="cuda")


def psf_airy(size=33, first_zero=4.0):
    """An Airy diffraction sprite (size, size, 3) uint8, RGB (bt_psf_airy)."""
    out = np.empty((size, size, 3), dtype=np.uint8)
    L.check(L.lib().bt_psf_airy(int(size), float(first_zero), out.ctypes.data))
    return out


class Blend:
    """Blending between two grids of neighbouring camera poses (bt_blend):
    prepare(grid_a, grid_b) finds the black hole's border in both; a frame
    rendered with grid2 / alpha / cam2 / blend then mixes them."""

    def __init__(self):
        h = C.c_void_p()
        L.check(L.lib().bt_blend_create(C.byref(h)))
        self._h = h

    def prepare(self, grid_a, grid_b, stream=None):
        pa, rows, cols, _ = grid_a.map_grid()
        pb, rows_b, cols_b, _ = grid_b.map_grid()
        if (rows, cols) != (rows_b, cols_b):
            raise ValueError("grids of different shapes")
        L.check(L.lib().bt_blend_prepare(self._h, pa, pb, rows, cols, _stream_ptr(stream)))

    def info(self):
        """(border as an (2 + 2*angles, 2) CUDA tensor view, angles, walks
        that reached the lattice edge); synchronises the device first."""
        torch = _torch()
        torch.cuda.synchronize()
        p = C.c_void_p()
        n = C.c_int32()
        e = C.c_uint32()
        L.check(L.lib().bt_blend_info(self._h, C.byref(p), C.byref(n), C.byref(e)))
        return _device_view(p.value, (2 + 2 * n.value, 2), torch.float32), n.value, e.value

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None:
            try:
                L.lib().bt_blend_destroy(h)
            except Exception:
                pass
            self._h = None


class StarProcessor:
    """BT/StarProcessor.h: a star list arranged in the reference's binary
    tree (starPos, starMag, binaryStarTree) and uploaded to the device."""

    def __init__(self, theta, phi, mag, bv, treeLevel=8, magnitudeCut=1000.0,
                 psf=None, stream=None):
        lib = L.lib()
        theta = np.ascontiguousarray(theta, dtype=np.float32)
        phi = np.ascontiguousarray(phi, dtype=np.float32)
        mag = np.ascontiguousarray(mag, dtype=np.float32)
        bv = np.ascontiguousarray(bv, dtype=np.float32)
        n = theta.size
        self.treeLevel = int(treeLevel)
        tsize = lib.bt_stars_tree_size(self.treeLevel)
        self.starPos = np.empty(2 * n, dtype=np.float32)
        self.starMag = np.empty(2 * n, dtype=np.float32)
        self.binaryStarTree = np.empty(tsize, dtype=np.int32)
        kept = C.c_int()
        L.check(lib.bt_stars_build_tree(theta.ctypes.data, phi.ctypes.data, mag.ctypes.data,
                                        bv.ctypes.data, n, self.treeLevel,
                                        float(magnitudeCut), self.starPos.ctypes.data,
                                        self.starMag.ctypes.data,
                                        self.binaryStarTree.ctypes.data, C.byref(kept)))
        self.starSize = kept.value
        self.starPos = self.starPos[: 2 * self.starSize].copy()
        self.starMag = self.starMag[: 2 * self.starSize].copy()
        self._upload(psf, stream)

    @classmethod
    def from_tree(cls, starPos, starMag, binaryStarTree, treeLevel, psf=None, stream=None):
        """A star set already arranged in the reference's tree (a StarProcessor
        of the reference, or a .star file)."""
        self = cls.__new__(cls)
        self.treeLevel = int(treeLevel)
        self.starPos = np.ascontiguousarray(starPos, dtype=np.float32)
        self.starMag = np.ascontiguousarray(starMag, dtype=np.float32)
        self.binaryStarTree = np.ascontiguousarray(binaryStarTree, dtype=np.int32)
        self.starSize = self.starPos.size // 2
        self._upload(psf, stream)
        return self

    @classmethod
    def load(cls, path, psf=None, stream=None):
        """A star cache file of the reference (BT/BlackTracer.cpp:326-331)."""
        from .cache import read_star_file
        pos, mag, tree, level = read_star_file(path)
        return cls.from_tree(pos, mag, tree, level, psf=psf, stream=stream)

    def save(self, path):
        """Writes the reference's star cache file (writeStars,
        BT/BlackTracer.cpp:40-46)."""
        from .cache import write_star_file
        write_star_file(path, self.starPos, self.starMag, self.binaryStarTree, self.treeLevel)

    def _upload(self, psf, stream):
        lib = L.lib()
        self.psf = None if psf is None else np.ascontiguousarray(psf, dtype=np.uint8)
        h = C.c_void_p()
        L.check(lib.bt_stars_create(self.starPos.ctypes.data, self.starMag.ctypes.data,
                                    self.starSize, self.binaryStarTree.ctypes.data,
                                    self.treeLevel,
                                    None if self.psf is None else self.psf.ctypes.data,
                                    0 if self.psf is None else self.psf.shape[0],
                                    C.byref(h), _stream_ptr(stream)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None:
            try:
                L.lib().bt_stars_destroy(h)
            except Exception:
                pass
            self._h = None


class Trails:
    """Star trails between consecutive frames rendered with this object
    (addTrails / makeGradField / clearArrays, BT/MakeImageKernel.cu:98-174,
    517-537, 618-629).  Made for one star set and one output size."""

    def __init__(self, n_stars, width, height, trailnum=30, max_hits=0):
        h = C.c_void_p()
        L.check(L.lib().bt_trails_create(int(n_stars), int(width), int(height), int(trailnum),
                                         int(max_hits), C.byref(h)))
        self._h = h
        self.width, self.height = int(width), int(height)

    def reset(self):
        """The next frame is a first frame again (no trails)."""
        L.check(L.lib().bt_trails_reset(self._h))

    def query(self, stream=None):
        """dict(frame, hits, dropped, walks_cut, trail: (H*W, 3) float32 CUDA
        view of the last frame's trail light); synchronises."""
        torch = _torch()
        i = L.bt_trails_info()
        L.check(L.lib().bt_trails_query(self._h, C.byref(i), _stream_ptr(stream)))
        return dict(frame=i.frame, hits=i.hits, dropped=i.dropped, walks_cut=i.walks_cut,
                    trail=_device_view(i.trail, (self.width * self.height, 3), torch.float32))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None:
            try:
                L.lib().bt_trails_destroy(h)
            except Exception:
                pass
            self._h = None


class Renderer:
    """Per-resolution device scratch + the frame call (makeImage, G = 1)."""

    def __init__(self, width, height):
        self.width, self.height = int(width), int(height)
        h = C.c_void_p()
        L.check(L.lib().bt_map_create(self.width, self.height, C.byref(h)))
        self._h = h

    def render(self, grid: Grid, viewer: Viewer, cam: Camera, env: Environment | None = None,
               stars: StarProcessor | None = None, lr=True, step=1, diffraction=False,
               hor=0.0, ver=0.0, out=None, stream=None, bb_table=0, psf_scale=False,
               grid2=None, cam2=None, alpha=0.0, blend=None, trails=None):
        """Returns (or fills) an (H, W, 4) uint8 BGRA CUDA tensor.  bb_table=1
        selects the 1024-entry FP32 blackbody table, psf_scale scales the
        diffraction footprint by sqrt(pixel magnification); grid2 / cam2 /
        alpha / blend (a prepared Blend) mix a second grid in; trails (a
        Trails) adds star trails from the previous frame rendered with it."""
        gp, rows, cols, _ = grid.map_grid()
        extra = {}
        if grid2 is not None:
            extra = dict(grid2=grid2.map_grid()[0], cam2=cam2.getParamArray(), alpha=alpha,
                         blend=blend)
        return self.render_raw(gp, rows, cols, grid.MAXLEVEL, viewer.viewMatrix,
                               cam.getParamArray(), env=env, stars=stars, lr=lr, step=step,
                               diffraction=diffraction, hor=hor, ver=ver, out=out,
                               stream=stream, bb_table=bb_table, psf_scale=psf_scale,
                               trails=trails, **extra)

    def render_raw(self, grid_ptr, grid_rows, grid_cols, grid_level, view, cam7, env=None,
                   stars=None, lr=True, step=1, diffraction=False, hor=0.0, ver=0.0,
                   out=None, stream=None, bb_table=0, psf_scale=False, grid2=None,
                   cam2=None, alpha=0.0, blend=None, trails=None):
        """The same from a raw float2 grid (device pointer) and 7 camera floats."""
        torch = _torch()
        if out is None:
            out = torch.empty((self.height, self.width, 4), dtype=torch.uint8, device="cuda")
        f = L.bt_frame()
        f.grid, f.grid_rows, f.grid_cols, f.grid_level = grid_ptr, grid_rows, grid_cols, grid_level
        f.view = view.data_ptr()
        f.hor, f.ver = hor, ver
        f.cam[:] = [float(x) for x in cam7]
        f.env = env._h if env is not None else None
        f.stars = stars._h if stars is not None else None
        f.map, f.star, f.lr = int(env is not None), int(stars is not None), int(bool(lr))
        f.step, f.diffraction = int(step), int(bool(diffraction))
        f.bb_table, f.psf_scale = int(bb_table), int(bool(psf_scale))
        if grid2 is not None:
            f.grid2, f.alpha, f.blend = grid2, float(alpha), blend._h
            f.cam2[:] = [float(x) for x in cam2]
        f.out = out.data_ptr()
        f.trails = trails._h if trails is not None else None
        L.check(L.lib().bt_map_render(self._h, C.byref(f), _stream_ptr(stream)))
        self._last = (f, env, stars, view)
        return out

    def census(self, stream=None):
        """Work of the last frame: dict(env_columns, env_pixels, star_pixels,
        star_candidates_ref, star_candidates) -- environment columns spanned
        (sum of pixNum + 1), and star candidates per pixel as the reference
        tests them (its starsToCheck) and as this build does after pruning."""
        last = getattr(self, "_last", None)
        if last is None:
            raise L.BtError(L.BT_ERR_STATE, "no frame rendered yet")
        c = L.bt_map_census_t()
        L.check(L.lib().bt_map_census(self._h, C.byref(last[0]), C.byref(c),
                                      _stream_ptr(stream)))
        return {k: int(getattr(c, k)) for k, _ in c._fields_}

    def scratch(self):
        """Device views of the frame's intermediates (thphi, gap, bh, area, light)."""
        torch = _torch()
        b = L.bt_map_buffers()
        L.check(L.lib().bt_map_scratch(self._h, C.byref(b)))
        W, H = self.width, self.height
        return dict(
            thphi=_device_view(b.thphi, ((H + 1) * (W + 1), 2), torch.float32),
            gap=_device_view(b.gap, ((H + 1) * (W + 1),), torch.int32),
            bh=_device_view(b.bh, (H * W,), torch.uint8),
            area=_device_view(b.area, (H * W,), torch.float32),
            light=_device_view(b.light, (H * W * 3,), torch.float32),
            light_diffracted=_device_view(b.light_diffracted, (H * W * 3,), torch.float32),
            env_img=_device_view(b.env_img, (H * W * 4,), torch.uint8))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None:
            try:
                L.lib().bt_map_destroy(h)
            except Exception:
                pass
            self._h = None
