"""CPU oracle for the BlackTracer hot path -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this package, and only as the checker.  The product
library never loads it.

Two back ends:

* ``_build/libbt_oracle.so`` -- the plain-C restatement (bt_oracle.c) of the
  reference algorithm (annemiekie/BlackTracer, BT/Metric.h, BT/Grid.h).
* ``_ref/libbtref.so`` -- the reference's own code compiled in place from the
  reference tree by ``make -C oracle ref`` (ref_harness.cpp).  It exists only
  where the reference tree was present at build time; everything here that
  needs it checks ``have_ref()``.

Arrays are numpy; camera parameters are 12 doubles in the field order of the
reference Camera (BT/Camera.h:8-11).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_ORC = os.path.join(_HERE, "_build", "libbt_oracle.so")
_REF = os.path.join(_HERE, "_ref", "libbtref.so")
_REF_MAP = os.path.join(_HERE, "_ref", "libbtref_map.so")

CAM_FIELDS = ("theta", "phi", "r", "speed", "br", "btheta", "bphi",
              "alpha", "w", "wbar", "Delta", "ro")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
_i8p = np.ctypeslib.ndpointer(dtype=np.int8, flags="C_CONTIGUOUS")


def reference_dir() -> str:
    """The reference tree the harness is compiled from: $BT_REFERENCE_DIR,
    else the default checkout location."""
    return os.environ.get("BT_REFERENCE_DIR", "/root/reference")


def have_reference_tree() -> bool:
    return os.path.isdir(os.path.join(reference_dir(), "BlackTracer2"))


def build(with_ref: bool | None = None) -> None:
    """Compile the restatement (and the reference harness when the reference
    tree is present)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    if with_ref is None:
        with_ref = have_reference_tree()
    if with_ref:
        subprocess.run(["make", "-s", "-C", _HERE, "ref", f"REF={reference_dir()}"],
                       check=True)


_orc = None
_ref = None


def _lib():
    global _orc
    if _orc is None:
        if not os.path.exists(_ORC):
            build(with_ref=False)
        lib = C.CDLL(_ORC)
        lib.orc_camera_static.argtypes = [C.c_double] * 5 + [_dp]
        lib.orc_camera_orbit.argtypes = [C.c_double] * 7 + [_dp]
        lib.orc_integrate_rays.argtypes = [_dp, C.c_double, _dp, _dp, C.c_size_t,
                                           _dp, _dp, _i32p, _u8p, C.c_int]
        lib.orc_integrate_rays_opts.argtypes = [
            _dp, C.c_double, _dp, _dp, C.c_size_t, _dp, _dp, _i32p, _u8p,
            C.c_double, C.c_double, C.c_double, C.c_int32, C.c_int]
        lib.orc_grid_build.argtypes = [C.c_int, C.c_int, C.c_int, _dp, C.c_double,
                                       C.c_int, _dp, _dp, _u8p, _i32p, _i8p, C.c_int]
        lib.orc_grid_build.restype = C.c_long
        lib.orc_grid_dims.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_int),
                                      C.POINTER(C.c_int)]
        _orc = lib
    return _orc


def have_ref() -> bool:
    return os.path.exists(_REF)


def _reflib():
    global _ref
    if _ref is None:
        if not have_ref():
            raise RuntimeError("reference harness not built (make -C oracle ref)")
        lib = C.CDLL(_REF)
        lib.btref_camera.argtypes = [C.c_int] + [C.c_double] * 7 + [_dp]
        lib.btref_integrate_rays.argtypes = [_dp, C.c_double, _dp, _dp, C.c_long,
                                             _dp, _dp, _i32p, C.c_int]
        lib.btref_grid_build.argtypes = [C.c_int, C.c_int, C.c_int, _dp, C.c_double,
                                         C.c_int, _dp, _dp, _u8p, _i32p, _i8p]
        lib.btref_grid_build.restype = C.c_long
        lib.btref_grid_time.argtypes = [C.c_int, C.c_int, C.c_int, _dp, C.c_double,
                                        C.POINTER(C.c_long)]
        lib.btref_grid_time.restype = C.c_double
        _ref = lib
    return _ref


# ---------------------------------------------------------------- cameras
def camera_static(a, theta, phi, r, speed, ref=False):
    """Camera(theta, phi, r, speed) -- BT/Camera.h:27-38."""
    out = np.zeros(12)
    if ref:
        _reflib().btref_camera(0, a, theta, phi, r, speed, 0.0, 0.0, out)
    else:
        _lib().orc_camera_static(a, theta, phi, r, speed, out)
    return out


def camera_orbit(a, theta, phi, r, br, btheta, bphi, ref=False):
    """Camera(theta, phi, r, br, btheta, bphi), Keplerian -- BT/Camera.h:40-52."""
    out = np.zeros(12)
    if ref:
        _reflib().btref_camera(1, a, theta, phi, r, br, btheta, bphi, out)
    else:
        _lib().orc_camera_orbit(a, theta, phi, r, br, btheta, bphi, out)
    return out


# ---------------------------------------------------------------- rays
def integrate_rays(cam, a, theta, phi, nthreads=0, ref=False, opts=None):
    """Grid::integration_wrapper (BT/Grid.h:514-556) on n rays.

    Returns (theta_out, phi_out, steps, status); status is None for ref=True.
    opts = (eps, h1, z_end, maxstp) selects a non-default tolerance
    (restatement only).
    """
    cam = np.ascontiguousarray(cam, dtype=np.float64)
    theta = np.ascontiguousarray(theta, dtype=np.float64)
    phi = np.ascontiguousarray(phi, dtype=np.float64)
    n = theta.size
    to = np.empty(n)
    po = np.empty(n)
    st = np.empty(n, dtype=np.int32)
    if ref:
        _reflib().btref_integrate_rays(cam, a, theta, phi, n, to, po, st,
                                       max(1, nthreads or os.cpu_count() or 1))
        return to, po, st, None
    status = np.empty(n, dtype=np.uint8)
    if opts is None:
        _lib().orc_integrate_rays(cam, a, theta, phi, n, to, po, st, status, nthreads)
    else:
        eps, h1, z_end, maxstp = opts
        _lib().orc_integrate_rays_opts(cam, a, theta, phi, n, to, po, st, status,
                                       eps, h1, z_end, int(maxstp), nthreads)
    return to, po, st, status


# ---------------------------------------------------------------- grid
def grid_dims(maxlevel, angle=True):
    N, M = C.c_int(), C.c_int()
    _lib().orc_grid_dims(maxlevel, 1 if angle else 0, C.byref(N), C.byref(M))
    return N.value, M.value


def grid_build(maxlevel, startlevel, angle, cam, a, tfix=1, ref=False, nthreads=0):
    """Adaptive grid (BT/Grid.h:605-624) on a dense lattice.

    tfix: 0 = raw traced values, 1 = canonical-order T-vertex fix,
          2 = (ref only) the reference's own unordered_map order.
    Returns dict(theta, phi, exists, steps, blevel, N, M, count).
    """
    N, M = grid_dims(maxlevel, angle)
    cam = np.ascontiguousarray(cam, dtype=np.float64)
    th = np.empty(N * M)
    ph = np.empty(N * M)
    ex = np.empty(N * M, dtype=np.uint8)
    st = np.empty(N * M, dtype=np.int32)
    bl = np.empty(N * M, dtype=np.int8)
    if ref:
        cnt = _reflib().btref_grid_build(maxlevel, startlevel, 1 if angle else 0, cam,
                                         a, tfix, th, ph, ex, st, bl)
    else:
        if tfix == 2:
            raise ValueError("tfix=2 (native unordered_map order) exists only in the reference")
        cnt = _lib().orc_grid_build(maxlevel, startlevel, 1 if angle else 0, cam, a,
                                    tfix, th, ph, ex, st, bl, nthreads)
    if cnt < 0:
        raise ValueError("bad grid arguments")
    shp = (N, M)
    return dict(theta=th.reshape(shp), phi=ph.reshape(shp), exists=ex.reshape(shp),
                steps=st.reshape(shp), blevel=bl.reshape(shp), N=N, M=M, count=int(cnt))


def ref_grid_time(maxlevel, startlevel, angle, cam, a):
    """Wall time of the reference Grid constructor (one thread, incl. hash)."""
    n = C.c_long()
    cam = np.ascontiguousarray(cam, dtype=np.float64)
    t = _reflib().btref_grid_time(maxlevel, startlevel, 1 if angle else 0, cam, a,
                                  C.byref(n))
    return t, n.value


# ---------------------------------------------------------------- map (reference kernels)
_refmap = None
_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_i32 = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def have_ref_map() -> bool:
    return os.path.exists(_REF_MAP)


def _refmaplib():
    global _refmap
    if _refmap is None:
        if not have_ref_map():
            raise RuntimeError("reference map harness not built (make -C oracle ref)")
        lib = C.CDLL(_REF_MAP)
        lib.btref_map_pixinterp.argtypes = [_f32p, C.c_int, C.c_int, C.c_void_p, C.c_int,
                                            C.c_int, C.c_int, C.c_float, C.c_float, _f32p,
                                            _i32]
        lib.btref_map_bh_area.argtypes = [_f32p, C.c_int, C.c_int, _u8p, _f32p]
        lib.btref_map_smooth.argtypes = [_f32p, _f32p, _u8p, _i32, C.c_int, C.c_int]
        lib.btref_map_sat.argtypes = [_u8p, C.c_int, C.c_int, _f32p]
        lib.btref_map_env.argtypes = [_f32p, _u8p, _u8p, C.c_int, C.c_int, C.c_int, C.c_int,
                                      _f32p, _f32p, _f32p, _f32p, C.c_int]
        lib.btref_map_stars.argtypes = [_f32p, _u8p, _f32p, _i32, C.c_int, _f32p, _f32p,
                                        C.c_int, C.c_int, C.c_int, C.c_int, _f32p, C.c_int,
                                        _f32p, _f32p, _u8p, C.c_void_p]
        lib.btref_map_compose.argtypes = [_u8p, _u8p, _u8p, C.c_int, C.c_int]
        lib.btref_map_pixinterp_blend.argtypes = [_f32p, C.c_int, C.c_int, _f32p, C.c_int,
                                                  C.c_int, C.c_int, C.c_float, C.c_float,
                                                  C.c_float, _f32p, _i32, _f32p]
        _refmap = lib
    return _refmap


def ref_star_tree(theta, phi, mag, bv, tree_level):
    """StarProcessor::makeTree of the reference (BT/StarProcessor.h:172-212)."""
    lib = _reflib()
    lib.btref_star_tree.argtypes = [_f32p, _f32p, _f32p, _f32p, C.c_int, C.c_int,
                                    _f32p, _f32p, _i32]
    f = lambda x: np.ascontiguousarray(x, dtype=np.float32)  # noqa: E731
    n = len(theta)
    pos = np.empty(2 * n, np.float32)
    mg = np.empty(2 * n, np.float32)
    tree = np.empty((1 << (tree_level + 1)) - 1, np.int32)
    lib.btref_star_tree(f(theta), f(phi), f(mag), f(bv), n, tree_level, pos, mg, tree)
    return pos, mg, tree


def ref_map_blend(grid_a, grid_b, grid_rows, grid_cols, gridlvl, view, width, height, alpha,
                  hor=0.0, ver=0.0):
    """The reference's Gr = 2 corner interpolation (findBhCenter,
    findBhBorders, smoothBorder x 4, pixInterpolation; BT/MakeImageKernel.cu
    :391-510) on two map grids stored one after the other, as the reference
    stores them.  Returns (thphi, gap, border).  Only for grids where every
    border walk ends inside the lattice (the reference's walk has no bound):
    check with the device's walk count first."""
    lib = _refmaplib()
    g = np.ascontiguousarray(np.concatenate([np.asarray(grid_a, np.float32).reshape(-1, 2),
                                             np.asarray(grid_b, np.float32).reshape(-1, 2)]))
    view = np.ascontiguousarray(view, dtype=np.float32)
    M, N = width, height
    thphi = np.zeros(((N + 1) * (M + 1), 2), np.float32)
    gap = np.zeros((N + 1) * (M + 1), np.int32)
    border = np.zeros((2 + 2 * 1000, 2), np.float32)
    lib.btref_map_pixinterp_blend(view, M, N, g, grid_cols, grid_rows, gridlvl, hor, ver, alpha,
                                  thphi, gap, border)
    return thphi, gap, border


def ref_map_frame(grid_f2, grid_rows, grid_cols, gridlvl, view, width, height, cam7,
                  bgr=None, stars=None, lr=True, step=1, hor=0.0, ver=0.0, want_cells=False):
    """One frame through the reference's own map kernels (host-compiled).

    grid_f2: (grid_rows*grid_cols, 2) float32 map grid; view: ((H+1)*(W+1), 2)
    float32; bgr: (rows, cols, 3) uint8 or None; stars: (pos, mag, tree,
    tree_level) or None.  Rows of the grid are padded with absent vertices
    above and below, which is what this build reads where the reference
    indexes outside the grid.  Returns a dict of the intermediates and the
    BGRA image."""
    lib = _refmaplib()
    M, N = width, height
    pad = 2 * grid_rows + 8
    g = np.full(((grid_rows + 2 * pad) * grid_cols, 2), -2.0, np.float32)
    g[pad * grid_cols:(pad + grid_rows) * grid_cols] = grid_f2
    gview = g[pad * grid_cols:]
    view = np.ascontiguousarray(view, dtype=np.float32)
    thphi = np.zeros(((N + 1) * (M + 1), 2), np.float32)
    gap = np.zeros((N + 1) * (M + 1), np.int32)
    # pass a pointer into the padded array: the harness indexes rows around it
    lib.btref_map_pixinterp(view, M, N, C.c_void_p(gview.ctypes.data), grid_cols, grid_rows,
                            gridlvl, hor, ver, thphi, gap)
    bh = np.zeros(N * M, np.uint8)
    area = np.zeros(N * M, np.float32)
    lib.btref_map_bh_area(thphi, M, N, bh, area)
    area_raw = area.copy()
    tmp = np.zeros(N * M, np.float32)
    lib.btref_map_smooth(area, tmp, bh, gap, M, N)
    cam7 = np.ascontiguousarray(cam7, dtype=np.float32)
    out = dict(thphi=thphi, gap=gap, bh=bh, area_raw=area_raw, area=area)
    img = None
    if bgr is not None:
        bgr = np.ascontiguousarray(bgr, dtype=np.uint8)
        rows, cols = bgr.shape[:2]
        sat = np.zeros(rows * cols * 4, np.float32)
        lib.btref_map_sat(bgr, rows, cols, sat)
        # zero rows around the table: what this build reads where the
        # reference indexes a row before or past it
        padded = np.zeros((rows + 4) * cols * 4, np.float32)
        padded[2 * cols * 4:(rows + 2) * cols * 4] = sat
        img = np.zeros(N * M * 4, np.uint8)
        lib.btref_map_env.argtypes = list(lib.btref_map_env.argtypes[:7]) + [C.c_void_p] + \
            list(lib.btref_map_env.argtypes[8:])
        lib.btref_map_env(thphi, img, bh, rows, cols, M, N,
                          C.c_void_p(padded.ctypes.data + 2 * cols * 16), cam7, area, view,
                          int(lr))
        out["sat"] = sat
        out["env"] = img.copy()
    if stars is not None:
        pos, mg, tree, tl = stars
        light = np.zeros(N * M * 3, np.float32)
        simg = np.zeros(N * M * 4, np.uint8)
        fw = 2 * step + 1
        cells = np.zeros(N * M * fw * fw * 3, np.float32) if want_cells else None
        lib.btref_map_stars(thphi, bh, np.ascontiguousarray(pos, np.float32),
                            np.ascontiguousarray(tree, np.int32), len(pos) // 2, cam7,
                            np.ascontiguousarray(mg, np.float32), tl, M, N, step, view,
                            int(lr), area, light, simg,
                            None if cells is None else C.c_void_p(cells.ctypes.data))
        if cells is not None:
            out["cells"] = cells
        out["light"] = light
        out["stars"] = simg.copy()
        if img is not None:
            comp = np.zeros(N * M * 4, np.uint8)
            lib.btref_map_compose(simg, img, comp, M, N)
            img = comp
        else:
            img = simg
    out["image"] = img
    return out


# ---------------------------------------------------------------- cache files, view (reference)
def _path(p) -> bytes:
    return os.fsencode(os.fspath(p))


def ref_grid_file_write(path, maxlevel, startlevel, angle, cam, a) -> int:
    """The reference's Grid constructor (with its perfect hash) written
    through cereal as the reference's app writes it.  Returns CamToCel's
    size."""
    lib = _reflib()
    lib.btref_grid_file_write.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, _dp,
                                          C.c_double]
    lib.btref_grid_file_write.restype = C.c_long
    cam = np.ascontiguousarray(cam, dtype=np.float64)
    return int(lib.btref_grid_file_write(_path(path), maxlevel, startlevel, 1 if angle else 0,
                                         cam, a))


def ref_grid_file_decode(path) -> dict:
    """A .grid file read through cereal into the reference's Grid: its
    tables, and every lattice vertex looked up with the reference's hash
    (dense (N*M, 2) float32, -2 where absent)."""
    lib = _reflib()
    ip = C.POINTER(C.c_int)
    lib.btref_grid_file_dims.argtypes = [C.c_char_p, ip, ip, ip, ip, ip]
    lib.btref_grid_file_decode.argtypes = [C.c_char_p, _f32p, _i32, _i32, _f32p]
    v = [C.c_int() for _ in range(5)]
    if lib.btref_grid_file_dims(_path(path), *[C.byref(x) for x in v]) != 0:
        raise FileNotFoundError(path)
    ml, N, M, hw, ow = (x.value for x in v)
    ht = np.empty(2 * hw * hw, np.float32)
    ot = np.empty(2 * ow * ow, np.int32)
    tag = np.empty(2 * hw * hw, np.int32)
    dense = np.empty(2 * N * M, np.float32)
    lib.btref_grid_file_decode(_path(path), ht, ot, tag, dense)
    return dict(MAXLEVEL=ml, N=N, M=M, hash_width=hw, offset_width=ow,
                hash_table=ht.reshape(-1, 2), offset_table=ot.reshape(-1, 2),
                pos_tag=tag.reshape(-1, 2), dense=dense.reshape(-1, 2))


def ref_psh_build(keys, values) -> dict:
    """The reference's PSHOffsetTable from keys (n, 2) and values (n, 2)
    (its offset search is seeded with the time: tables differ run to run)."""
    lib = _reflib()
    ip = C.POINTER(C.c_int)
    lib.btref_psh_build.argtypes = [_i32, _f32p, C.c_int, ip, ip, C.c_void_p, C.c_void_p,
                                    C.c_void_p, C.c_long, C.c_long]
    k = np.ascontiguousarray(keys, dtype=np.int32).reshape(-1)
    v = np.ascontiguousarray(values, dtype=np.float32).reshape(-1)
    hw, ow = C.c_int(), C.c_int()
    lib.btref_psh_build(k, v, len(k) // 2, C.byref(hw), C.byref(ow), None, None, None, 0, 0)
    return dict(hash_width=hw.value, offset_width=ow.value)


def ref_stars_file_write(path, pos, mag, tree, tree_level) -> None:
    lib = _reflib()
    lib.btref_stars_file_write.argtypes = [C.c_char_p, _f32p, _f32p, C.c_int, _i32, C.c_int]
    pos = np.ascontiguousarray(pos, np.float32)
    lib.btref_stars_file_write(_path(path), pos, np.ascontiguousarray(mag, np.float32),
                               pos.size // 2, np.ascontiguousarray(tree, np.int32), tree_level)


def ref_stars_file_read(path):
    """(pos, mag, tree, treeLevel) of a .star file read through cereal into
    the reference's StarProcessor."""
    lib = _reflib()
    ip = C.POINTER(C.c_int)
    lib.btref_stars_file_read.argtypes = [C.c_char_p, ip, ip, C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.c_int, C.c_int]
    n, lv = C.c_int(), C.c_int()
    if lib.btref_stars_file_read(_path(path), C.byref(n), C.byref(lv), None, None, None,
                                 -1, -1) != 0:
        raise FileNotFoundError(path)
    pos = np.empty(2 * n.value, np.float32)
    mag = np.empty(2 * n.value, np.float32)
    tree = np.empty((1 << (lv.value + 1)) - 1, np.int32)
    lib.btref_stars_file_read(_path(path), C.byref(n), C.byref(lv), pos.ctypes.data,
                              mag.ctypes.data, tree.ctypes.data, n.value, tree.size)
    return pos, mag, tree, lv.value


def ref_view_camera(view_angle, off_up, off_right, width, height):
    """Viewer(viewangle, offUp, offRight, W, H, sphere = false).viewMatrix
    (BT/Viewer.h:109-133) as ((H+1)*(W+1), 2) float32."""
    lib = _reflib()
    lib.btref_view_camera.argtypes = [C.c_double, C.c_double, C.c_double, C.c_int, C.c_int,
                                      _f32p]
    out = np.zeros(2 * (height + 1) * (width + 1), np.float32)
    lib.btref_view_camera(view_angle, off_up, off_right, width, height, out)
    return out.reshape(-1, 2)


# ---------------------------------------------------------------- trails (reference)
def ref_trail_cache(thphi, bh, area, cam7, stars, width, height, step, view, lr, trailnum=30):
    """The star caches and hit counts the reference's frame-0 star pass
    leaves (no line is drawn at frame 0).  stars = (pos, mag, tree, level).
    Returns (cache (n, trailnum, 2) int32, counts (n,) int32)."""
    lib = _refmaplib()
    pos, mg, tree, tl = stars
    n = len(pos) // 2
    lib.btref_trail_cache.argtypes = [C.c_void_p, _u8p, _f32p, _i32, C.c_int, _f32p, _f32p,
                                      C.c_int, C.c_int, C.c_int, C.c_int, _f32p, C.c_int,
                                      _f32p, C.c_int, _i32, _i32]
    M, N = width, height
    th = _trail_corners(thphi, M, N)
    cache = np.zeros(n * trailnum * 2, np.int32)
    cnt = np.zeros(n, np.int32)
    lib.btref_trail_cache(C.c_void_p(th.ctypes.data), np.ascontiguousarray(bh, np.uint8),
                          np.ascontiguousarray(pos, np.float32),
                          np.ascontiguousarray(tree, np.int32), n,
                          np.ascontiguousarray(cam7, np.float32),
                          np.ascontiguousarray(mg, np.float32), tl, M, N, step,
                          np.ascontiguousarray(view, np.float32), int(lr),
                          np.ascontiguousarray(area, np.float32), trailnum, cache, cnt)
    return cache.reshape(n, trailnum, 2), cnt


def _trail_corners(thphi, M, N):
    # makeGradField reads one element past the corner array: an absent corner
    th = np.full(((N + 1) * (M + 1) + 1) * 2, -2.0, np.float32)
    th[:(N + 1) * (M + 1) * 2] = np.asarray(thphi, np.float32).reshape(-1)
    return th


def ref_trail_frames(f0, f1, stars, width, height, step, view, lr, trailnum=30):
    """Frames 0 and 1 through the reference's trail code (clearArrays,
    makeGradField, distortStarMap with addTrails, sumStarLight).  f0, f1 =
    (thphi, bh, area, cam7).  Returns (trail of frame 1 (N*M, 3), light of
    frame 1 (N*M, 3)).  Run only where oracle.trails.plan says every walk
    ends."""
    lib = _refmaplib()
    pos, mg, tree, tl = stars
    n = len(pos) // 2
    M, N = width, height
    lib.btref_trail_frames.argtypes = ([C.c_void_p, _u8p, _f32p, _f32p] * 2 +
                                       [_f32p, _i32, C.c_int, _f32p, C.c_int, C.c_int, C.c_int,
                                        C.c_int, _f32p, C.c_int, C.c_int, _f32p, _f32p])
    keep = []
    args = []
    for (thphi, bh, area, cam7) in (f0, f1):
        th = _trail_corners(thphi, M, N)
        keep.append(th)
        args += [C.c_void_p(th.ctypes.data), np.ascontiguousarray(bh, np.uint8),
                 np.ascontiguousarray(area, np.float32), np.ascontiguousarray(cam7, np.float32)]
    trail = np.zeros(N * M * 3, np.float32)
    light = np.zeros(N * M * 3, np.float32)
    lib.btref_trail_frames(*args, np.ascontiguousarray(pos, np.float32),
                           np.ascontiguousarray(tree, np.int32), n,
                           np.ascontiguousarray(mg, np.float32), tl, M, N, step,
                           np.ascontiguousarray(view, np.float32), int(lr), trailnum, trail,
                           light)
    return trail.reshape(-1, 3), light.reshape(-1, 3)


def ref_map_diffraction(light, width, height, sprite):
    """The reference's addDiffraction run pixel by pixel in row-major order on
    a copy of `light` ((height*width*3,) float32 summed star light) with an
    (fs, fs, 3) uint8 sprite; returns the diffracted light (height*width*3,).
    The extra row the kernel can write past the image is dropped."""
    lib = _refmaplib()
    lib.btref_map_diffraction.argtypes = [_f32p, C.c_int, C.c_int, _u8p, C.c_int]
    M, N = width, height
    buf = np.zeros((N + 1) * M * 3, np.float32)
    buf[:N * M * 3] = np.asarray(light, np.float32).reshape(-1)
    sp = np.ascontiguousarray(sprite, dtype=np.uint8)
    lib.btref_map_diffraction(buf, M, N, sp, sp.shape[0])
    return buf[:N * M * 3].copy()


def ref_map_sat(bgr):
    """The summed-area table of the reference's driver (cudaPrep,
    BT/MakeImageKernel.cu:1312-1330) over a (rows, cols, 3) BGR8 image, as
    (rows*cols*4,) float32 (host threads over columns)."""
    lib = _refmaplib()
    bgr = np.ascontiguousarray(bgr, dtype=np.uint8)
    rows, cols = bgr.shape[:2]
    sat = np.zeros(rows * cols * 4, np.float32)
    lib.btref_map_sat(bgr, rows, cols, sat)
    return sat


def ref_map_frame_rows(grid_f2, grid_rows, grid_cols, gridlvl, view, width, height, cam7,
                       rows, sat=None, env_shape=None, stars=None, step=1, lr=True,
                       nthreads=0, area=None):
    """One frame through the reference's own map kernels on host threads
    (btref_map_frame_rows): corners, black-hole mask and smoothed solid angles
    of the whole frame, and the environment, star and composite colours of the
    listed rows.  sat = ref_map_sat(bgr) with env_shape = (rows, cols), or
    None; stars = (pos, mag, tree, level) or None; area: (H*W,) smoothed solid
    angles for the colour passes to use instead of the harness's own (the
    returned `area` is the harness's).  Returns dict(thphi, gap, bh, area,
    env, stars, image) with the row images as (len(rows), W, 4)."""
    lib = _refmaplib()
    M, N = width, height
    rows = np.ascontiguousarray(rows, dtype=np.int32)
    nr = rows.size
    pad = 2 * grid_rows + 8
    g = np.full(((grid_rows + 2 * pad) * grid_cols, 2), -2.0, np.float32)
    g[pad * grid_cols:(pad + grid_rows) * grid_cols] = np.asarray(grid_f2, np.float32).reshape(-1, 2)
    if sat is not None:
        er, ec = env_shape
        sp = np.zeros((er + 4) * ec * 4, np.float32)
        sp[2 * ec * 4:(er + 2) * ec * 4] = np.asarray(sat, np.float32).reshape(-1)
        sat_ptr = C.c_void_p(sp.ctypes.data + 2 * ec * 16)
    else:
        er = ec = 0
        sat_ptr = None
    if stars is not None:
        pos, mg, tree, tl = stars
        pos = np.ascontiguousarray(pos, np.float32)
        mg = np.ascontiguousarray(mg, np.float32)
        tree = np.ascontiguousarray(tree, np.int32)
        sptr = (pos.ctypes.data, tree.ctypes.data, len(pos) // 2, mg.ctypes.data, tl)
    else:
        sptr = (None, None, 0, None, 0)
    thphi = np.zeros(((N + 1) * (M + 1), 2), np.float32)
    gap = np.zeros((N + 1) * (M + 1), np.int32)
    bh = np.zeros(N * M, np.uint8)
    area_out = np.zeros(N * M, np.float32)
    area_keep = None if area is None else np.ascontiguousarray(area, np.float32).reshape(-1)
    env = np.zeros((nr, M, 4), np.uint8) if sat is not None else None
    simg = np.zeros((nr, M, 4), np.uint8) if stars is not None else None
    img = np.zeros((nr, M, 4), np.uint8) if (sat is not None and stars is not None) else None
    vp = C.c_void_p
    lib.btref_map_frame_rows.argtypes = [
        _f32p, C.c_int, C.c_int, vp, C.c_int, C.c_int, C.c_int, vp, C.c_int, C.c_int,
        vp, vp, C.c_int, vp, C.c_int, _f32p, C.c_int, C.c_int, _i32, C.c_int, C.c_int,
        _f32p, _i32, _u8p, _f32p, vp, vp, vp, vp]
    lib.btref_map_frame_rows.restype = C.c_int
    ptr = lambda a: None if a is None else C.c_void_p(a.ctypes.data)  # noqa: E731
    rc = lib.btref_map_frame_rows(
        np.ascontiguousarray(view, np.float32), M, N,
        C.c_void_p(g.ctypes.data + pad * grid_cols * 8), grid_cols, grid_rows, gridlvl,
        sat_ptr, er, ec, sptr[0], sptr[1], sptr[2], sptr[3], sptr[4],
        np.ascontiguousarray(cam7, np.float32), step, int(lr), rows, nr, nthreads,
        thphi, gap, bh, area_out,
        None if area is None else C.c_void_p(area_keep.ctypes.data), ptr(env), ptr(simg),
        ptr(img))
    if rc != 0:
        raise RuntimeError("reference frame rows failed (scratch reservation)")
    return dict(thphi=thphi, gap=gap, bh=bh, area=area_out, env=env, stars=simg, image=img)


def ref_map_time(grid_f2, grid_rows, grid_cols, gridlvl, view, width, height, cam7, sat,
                 env_rows, env_cols, stars, step=1, lr=True, row_stride=16, nthreads=0):
    """The reference's per-pixel map kernels timed on host threads
    (btref_map_time): corners and areas over the whole frame, environment and
    stars over every row_stride-th row.  stars = (pos, mag, tree, level); sat
    (env_rows*env_cols*4 float32).  Returns dict(secs per phase, rows sampled,
    frame_s = the phases scaled to the whole frame)."""
    lib = _refmaplib()
    M, N = width, height
    pos, mg, tree, tl = stars
    pad = 2 * grid_rows + 8
    g = np.full(((grid_rows + 2 * pad) * grid_cols, 2), -2.0, np.float32)
    g[pad * grid_cols:(pad + grid_rows) * grid_cols] = np.asarray(grid_f2, np.float32).reshape(-1, 2)
    s = np.zeros((env_rows + 4) * env_cols * 4, np.float32)
    s[2 * env_cols * 4:(env_rows + 2) * env_cols * 4] = np.asarray(sat, np.float32).reshape(-1)
    lib.btref_map_time.argtypes = [_f32p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                   C.c_void_p, C.c_int, C.c_int, _f32p, _i32, C.c_int, _f32p,
                                   C.c_int, _f32p, C.c_int, C.c_int, C.c_int, C.c_int,
                                   np.ctypeslib.ndpointer(dtype=np.float64)]
    lib.btref_map_time.restype = C.c_int
    secs = np.zeros(4, np.float64)
    nr = lib.btref_map_time(np.ascontiguousarray(view, np.float32), M, N,
                            C.c_void_p(g.ctypes.data + pad * grid_cols * 8), grid_cols, grid_rows,
                            gridlvl, C.c_void_p(s.ctypes.data + 2 * env_cols * 16), env_rows,
                            env_cols, np.ascontiguousarray(pos, np.float32),
                            np.ascontiguousarray(tree, np.int32), len(pos) // 2,
                            np.ascontiguousarray(mg, np.float32), tl,
                            np.ascontiguousarray(cam7, np.float32), step, int(lr), row_stride,
                            nthreads, secs)
    if nr <= 0:
        raise RuntimeError("reference map timing failed")
    frame = secs[0] + secs[1] + (secs[2] + secs[3]) * N / nr
    return dict(corners_s=float(secs[0]), area_s=float(secs[1]), env_rows_s=float(secs[2]),
                stars_rows_s=float(secs[3]), rows_sampled=int(nr), frame_s=float(frame))
