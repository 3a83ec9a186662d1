"""Host mirror of the reference's integration-side interfaces.

Same names, arguments and meaning as annemiekie/BlackTracer:
  BlackHole(afactor)                           BT/BlackHole.h:7-21
  Camera(theta, phi, r, speed)                 BT/Camera.h:27-38
  Camera(theta, phi, r, br, btheta, bphi)      BT/Camera.h:40-52
  Grid(maxLevelPrec, startLevel, angle, cam, bh)   BT/Grid.h:605-624
Like the reference, constructing a BlackHole sets the spin that later
Camera constructions use (metric::setAngVel, BT/Metric.h:51-54); every
constructor also takes an explicit ``a=`` instead.  All compute goes through
the C ABI (libblacktracer_b200.so); device buffers are torch CUDA tensors.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L

# Blocks of 256 threads per SM of the one-launch build (set_flow).
FLOW_BLOCKS_PER_SM = 2

_current_spin = 0.0  # metric::a after the last BlackHole / setA


def _torch():
    import torch
    return torch


def _stream_ptr(stream=None):
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


class BlackHole:
    """BT/BlackHole.h: holds the spin a/M and makes it the current spin."""

    def __init__(self, afactor: float):
        self.setA(afactor)

    def setA(self, afactor: float) -> None:
        global _current_spin
        self.a = float(afactor)
        _current_spin = self.a

    def getAngVel(self, mass: float) -> float:
        return mass * self.a


class Camera:
    """BT/Camera.h.  Camera(theta, phi, r, speed) or
    Camera(theta, phi, r, br, btheta, bphi) (Keplerian speed)."""

    FIELDS = ("theta", "phi", "r", "speed", "br", "btheta", "bphi",
              "alpha", "w", "wbar", "Delta", "ro")

    def __init__(self, theta, phi, r, *args, a: float | None = None):
        self.a = _current_spin if a is None else float(a)
        c = L.bt_camera()
        if len(args) == 1:
            L.check(L.lib().bt_camera_static(self.a, theta, phi, r, args[0], C.byref(c)))
        elif len(args) == 3:
            L.check(L.lib().bt_camera_orbit(self.a, theta, phi, r, *args, C.byref(c)))
        else:
            raise TypeError("Camera(theta, phi, r, speed) or "
                            "Camera(theta, phi, r, br, btheta, bphi)")
        self._c = c
        for f in self.FIELDS:
            setattr(self, f, getattr(c, f))

    @classmethod
    def from_array(cls, arr12, a: float) -> "Camera":
        """A camera from the 12 Camera fields (as the oracle returns them)."""
        obj = cls.__new__(cls)
        obj.a = float(a)
        c = L.bt_camera(*[float(x) for x in arr12])
        obj._c = c
        for f in cls.FIELDS:
            setattr(obj, f, getattr(c, f))
        return obj

    def as_array(self) -> np.ndarray:
        return np.array([getattr(self._c, f) for f in self.FIELDS], dtype=np.float64)

    def getParamArray(self) -> np.ndarray:
        """BT/Camera.h:67-78: {speed, alpha, w, wbar, br, btheta, bphi} as float32."""
        out = (C.c_float * 7)()
        L.check(L.lib().bt_camera_params(C.byref(self._c), out))
        return np.array(out[:], dtype=np.float32)


class IntegOpts:
    """bt_integ_opts; defaults are the reference constants (BT/Metric.h:311-314)."""

    def __init__(self, precision: str | int = "plain", **kw):
        o = L.bt_integ_opts()
        L.lib().bt_integ_opts_default(C.byref(o))
        if isinstance(precision, str):
            precision = {"plain": L.PRECISION_PLAIN, "mixed": L.PRECISION_MIXED,
                         "fast": L.PRECISION_FAST}[precision]
        o.precision = int(precision)
        for k, v in kw.items():
            setattr(o, k, v)
        self._o = o

    @property
    def ref(self):
        return C.byref(self._o)


def _opts(opts) -> IntegOpts:
    if opts is None:
        return IntegOpts()
    if isinstance(opts, IntegOpts):
        return opts
    if isinstance(opts, str):
        return IntegOpts(opts)
    raise TypeError("opts must be IntegOpts, 'plain', 'mixed', 'fast' or None")


def integrate_rays(cam: Camera, theta, phi, opts=None, a: float | None = None, stream=None):
    """Grid::integration_wrapper (BT/Grid.h:514-556) on torch CUDA tensors.

    Returns (theta_out, phi_out, steps, status) as new CUDA tensors."""
    torch = _torch()
    a = cam.a if a is None else a
    theta = theta.contiguous().to(torch.float64)
    phi = phi.contiguous().to(torch.float64)
    n = theta.numel()
    tho = torch.empty_like(theta)
    pho = torch.empty_like(phi)
    st = torch.empty(n, dtype=torch.int32, device=theta.device)
    ss = torch.empty(n, dtype=torch.uint8, device=theta.device)
    o = _opts(opts)
    L.check(L.lib().bt_integrate_rays(C.byref(cam._c), a, theta.data_ptr(), phi.data_ptr(), n,
                                      tho.data_ptr(), pho.data_ptr(), st.data_ptr(),
                                      ss.data_ptr(), o.ref, _stream_ptr(stream)))
    return tho, pho, st, ss


def integrate_rays_host(cam: Camera, theta: np.ndarray, phi: np.ndarray, opts=None,
                        a: float | None = None):
    """The same with host numpy arrays (copies inside the library)."""
    a = cam.a if a is None else a
    theta = np.ascontiguousarray(theta, dtype=np.float64)
    phi = np.ascontiguousarray(phi, dtype=np.float64)
    n = theta.size
    tho = np.empty(n)
    pho = np.empty(n)
    st = np.empty(n, dtype=np.int32)
    ss = np.empty(n, dtype=np.uint8)
    o = _opts(opts)
    L.check(L.lib().bt_integrate_rays_host(
        C.byref(cam._c), a, theta.ctypes.data, phi.ctypes.data, n, tho.ctypes.data,
        pho.ctypes.data, st.ctypes.data, ss.ctypes.data, o.ref, None))
    return tho, pho, st, ss


def grid_dims(maxlevel: int, angle: bool = True):
    N, M = C.c_int32(), C.c_int32()
    L.check(L.lib().bt_grid_dims(maxlevel, 1 if angle else 0, C.byref(N), C.byref(M)))
    return N.value, M.value


def _tune_dict(r) -> dict:
    return {"shape": (r.shape.threads, r.shape.blocks_per_sm, r.shape.refill),
            "flow": int(r.flow), "fp64_band": float(r.fp64_band),
            "band_met": bool(r.band_met), "band_p99_rad": float(r.band_p99_rad),
            "best_ms": float(r.best_ms), "level_ms": float(r.level_ms),
            "flow_ms": float(r.flow_ms), "candidates": int(r.candidates)}


class Grid:
    """BT/Grid.h:605: Grid(maxLevelPrec, startLevel, angle, camera, bh).

    The grid lives on the current CUDA device as a dense lattice.  Public
    fields mirror the reference: MAXLEVEL, STARTLVL, N, M, STARTN, STARTM,
    equafactor; ``dense()`` gives the lattice as CUDA tensors, ``CamToCel``,
    ``steps`` and ``blockLevels`` give host copies in the reference's shapes.
    """

    def __init__(self, maxLevelPrec: int, startLevel: int, angle: bool, camera: Camera,
                 bh: BlackHole | None = None, opts=None, stream=None, handle=None):
        self.MAXLEVEL = int(maxLevelPrec)
        self.STARTLVL = int(startLevel)
        self.equafactor = 1 if angle else 0
        self.N, self.M = grid_dims(self.MAXLEVEL, angle)
        self.STARTN, self.STARTM = grid_dims(self.STARTLVL, angle)
        self.cam = camera
        self.a = bh.a if bh is not None else camera.a
        self._own = handle is None
        if handle is None:
            h = C.c_void_p()
            L.check(L.lib().bt_grid_create(self.MAXLEVEL, self.equafactor, C.byref(h)))
            self._h = h
        else:
            self._h = handle
        self.opts = _opts(opts)
        self._stream = stream
        self.build()

    def build(self, camera: Camera | None = None, a: float | None = None):
        if camera is not None:
            self.cam = camera
        if a is not None:
            self.a = a
        L.check(L.lib().bt_grid_build(self._h, C.byref(self.cam._c), self.a, self.STARTLVL,
                                      self.opts.ref, _stream_ptr(self._stream)))
        self._info = None
        self._map = None

    def info(self) -> L.bt_grid_info:
        if self._info is None:
            inf = L.bt_grid_info()
            L.check(L.lib().bt_grid_query(self._h, C.byref(inf), _stream_ptr(self._stream)))
            self._info = inf
        return self._info

    @property
    def traced(self) -> int:
        return int(self.info().traced)

    def dense(self):
        """theta, phi (float64, -2 where absent), exists (u8), steps (i32),
        blevel (i8, -1 = none), status (u8) as (N, M) CUDA tensors."""
        torch = _torch()
        dev = torch.device("cuda", torch.cuda.current_device())
        shp = (self.N, self.M)
        out = dict(theta=torch.empty(shp, dtype=torch.float64, device=dev),
                   phi=torch.empty(shp, dtype=torch.float64, device=dev),
                   exists=torch.empty(shp, dtype=torch.uint8, device=dev),
                   steps=torch.empty(shp, dtype=torch.int32, device=dev),
                   blevel=torch.empty(shp, dtype=torch.int8, device=dev),
                   status=torch.empty(shp, dtype=torch.uint8, device=dev))
        L.check(L.lib().bt_grid_export_dense(
            self._h, *(out[k].data_ptr() for k in
                       ("theta", "phi", "exists", "steps", "blevel", "status")),
            _stream_ptr(self._stream)))
        self.info()
        return out

    def set_timing(self, on=True):
        """Record CUDA events around the ray-tracing launches (info().trace_ms)."""
        L.check(L.lib().bt_grid_set_timing(self._h, 1 if on else 0))

    def set_graph(self, on=True):
        """Capture later builds once into a CUDA graph and replay it."""
        L.check(L.lib().bt_grid_set_graph(self._h, 1 if on else 0))

    def set_flow(self, on=True, blocks_per_sm=FLOW_BLOCKS_PER_SM):
        """Run the refinement levels of later builds as one persistent launch
        (blocks checked as soon as their corners are traced; same grids) of
        `blocks_per_sm` blocks of 256 threads per SM."""
        L.check(L.lib().bt_grid_set_flow(self._h, blocks_per_sm if on else 0))

    def set_shape(self, threads=128, blocks_per_sm=0, refill=0):
        """Trace launch shape of later level builds (as GridSet.set_shape)."""
        s = L.bt_trace_shape(threads, blocks_per_sm, refill)
        L.check(L.lib().bt_grid_set_shape(self._h, C.byref(s)))

    def tune(self, p99_target=1e-6, repeats=2):
        """The full autotuner (bt_grid_tune) on this grid's camera and spin;
        keeps the fastest configuration, a mixed grid's options take the band
        chosen.  Returns a dict of the choice (as GridSet.tune)."""
        r = L.bt_tune_result()
        L.check(L.lib().bt_grid_tune(self._h, self.opts.ref, float(p99_target), int(repeats),
                                     C.byref(r), _stream_ptr(self._stream)))
        self._info, self._map = None, None
        if self.opts._o.precision == L.PRECISION_MIXED:
            self.opts._o.fp64_band = r.fp64_band
        return _tune_dict(r)

    def set_tfix_passes(self, passes: int):
        """Jacobi passes of the T-vertex fix per level of later builds (1..8;
        default 8).  A level still changing at its last pass is reported as
        not converged by info() (flag 1, BtError BT_ERR_NUMERIC)."""
        L.check(L.lib().bt_grid_set_tfix_passes(self._h, int(passes)))

    def set_tfix_launch(self, cooperative=True):
        """Diagnostic: the T-vertex fix of later builds as one cooperative
        launch per level (default) or a launch per pass."""
        L.check(L.lib().bt_grid_set_tfix_launch(self._h, 1 if cooperative else 0))

    def export(self, out=None, pinned=True, stream=None):
        """The grid as key-ordered lists (CamToCel, steps, blockLevels).

        Returns dict of numpy arrays vi, vj, theta, phi, steps, bi, bj, level
        (host copies).  `out` may pass preallocated arrays (reused).  `stream`
        (default: the grid's) runs the export; it must follow the build (an
        event), and the grid must not be built again before this returns."""
        torch = _torch()
        if out is None:
            inf = self.info()
            nv = nb = int(inf.traced) + 2 * self.M + 16
            mk = (lambda n, dt: torch.empty(n, dtype=dt, pin_memory=pinned))
            out = dict(vi=mk(nv, torch.int32), vj=mk(nv, torch.int32),
                       theta=mk(nv, torch.float64), phi=mk(nv, torch.float64),
                       steps=mk(nv, torch.int32), bi=mk(nb, torch.int32),
                       bj=mk(nb, torch.int32), level=mk(nb, torch.int8))
        e = L.bt_grid_export_t()
        for k in ("vi", "vj", "theta", "phi", "steps", "bi", "bj", "level"):
            setattr(e, k, out[k].data_ptr())
        e.cap_vertices = out["vi"].numel()
        e.cap_blocks = out["bi"].numel()
        st = stream if stream is not None else self._stream
        L.check(L.lib().bt_grid_export(self._h, C.byref(e), _stream_ptr(st)))
        torch.cuda.current_stream().synchronize() if st is None else st.synchronize()
        nv, nb = int(e.n_vertices), int(e.n_blocks)
        res = {k: out[k][:nv] for k in ("vi", "vj", "theta", "phi", "steps")}
        res.update({k: out[k][:nb] for k in ("bi", "bj", "level")})
        res["_buffers"] = out
        return res

    def map_grid(self):
        """(pointer, rows, cols, sym) of the float2 map grid (makeGrid);
        exported once per build."""
        if getattr(self, "_map", None) is not None:
            return self._map
        p = C.c_void_p()
        rows, cols, sym = C.c_int32(), C.c_int32(), C.c_int32()
        L.check(L.lib().bt_grid_map_export(self._h, C.byref(p), C.byref(rows), C.byref(cols),
                                           C.byref(sym), _stream_ptr(self._stream)))
        self._map = (p.value, rows.value, cols.value, sym.value)
        return self._map

    def save(self, path):
        """Writes the reference's grid cache file (write, BT/BlackTracer.cpp
        :26-33): MAXLEVEL, N, M and the vertices in a perfect spatial hash,
        which the reference loads in place of computing the grid."""
        import os
        L.check(L.lib().bt_grid_save(self._h, os.fsencode(os.fspath(path)),
                                     _stream_ptr(self._stream)))

    # --- reference-shaped host views (slow; for compatibility and tests) ---
    @property
    def CamToCel(self) -> dict:
        d = {k: v.cpu().numpy() for k, v in self.dense().items()}
        ii, jj = np.nonzero(d["exists"])
        keys = (ii.astype(np.uint64) << np.uint64(32)) | jj.astype(np.uint64)
        return {int(k): (float(t), float(p)) for k, t, p in
                zip(keys, d["theta"][ii, jj], d["phi"][ii, jj])}

    @property
    def steps(self) -> np.ndarray:
        return self.dense()["steps"].cpu().numpy().reshape(-1)

    @property
    def blockLevels(self) -> dict:
        bl = self.dense()["blevel"].cpu().numpy()
        ii, jj = np.nonzero(bl >= 0)
        keys = (ii.astype(np.uint64) << np.uint64(32)) | jj.astype(np.uint64)
        return {int(k): int(v) for k, v in zip(keys, bl[ii, jj])}

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and getattr(self, "_own", False):
            try:
                L.lib().bt_grid_destroy(h)
            except Exception:
                pass
            self._h = None


class GridSet:
    """A set of grids of one size built together (bt_batch): grid k for
    cameras[k] and spins[k].  The reference builds its grids one by one
    (BT/BlackTracer.cpp:220-262); here all levels of all grids share launches
    and one persistent ray-tracing queue.  ``grids[k]`` are Grid views of the
    members (query, export and map as any Grid; released with the set)."""

    def __init__(self, maxLevelPrec: int, startLevel: int, angle: bool, count: int,
                 opts=None, stream=None):
        self.MAXLEVEL = int(maxLevelPrec)
        self.STARTLVL = int(startLevel)
        self.equafactor = 1 if angle else 0
        self.count = int(count)
        self.opts = _opts(opts)
        self._stream = stream
        h = C.c_void_p()
        L.check(L.lib().bt_batch_create(self.MAXLEVEL, self.equafactor, self.count,
                                        C.byref(h)))
        self._h = h
        N, M = grid_dims(self.MAXLEVEL, angle)
        sN, sM = grid_dims(self.STARTLVL, angle)
        self.grids = []
        for k in range(self.count):
            g = Grid.__new__(Grid)
            g.MAXLEVEL, g.STARTLVL, g.equafactor = self.MAXLEVEL, self.STARTLVL, self.equafactor
            g.N, g.M, g.STARTN, g.STARTM = N, M, sN, sM
            g.cam, g.a, g.opts, g._stream = None, None, self.opts, stream
            g._own, g._info, g._map, g._set = False, None, None, self
            g._h = C.c_void_p(L.lib().bt_batch_grid(h, k))
            self.grids.append(g)
        self._info = None

    def _arrays(self, cameras, spins):
        if len(cameras) != self.count or len(spins) != self.count:
            raise ValueError(f"need {self.count} cameras and spins")
        cams = (L.bt_camera * self.count)(*[c._c for c in cameras])
        a = (C.c_double * self.count)(*[float(x) for x in spins])
        return cams, a

    def build(self, cameras, spins):
        cams, a = self._arrays(cameras, spins)
        L.check(L.lib().bt_batch_build(self._h, cams, a, self.STARTLVL, self.opts.ref,
                                       _stream_ptr(self._stream)))
        for g, c, s in zip(self.grids, cameras, spins):
            g.cam, g.a, g._info, g._map = c, float(s), None, None
        self._info = None

    def info(self) -> L.bt_batch_info:
        if self._info is None:
            inf = L.bt_batch_info()
            L.check(L.lib().bt_batch_query(self._h, C.byref(inf), _stream_ptr(self._stream)))
            self._info = inf
        return self._info

    @property
    def traced(self) -> int:
        return int(self.info().traced)

    def set_graph(self, on=True):
        L.check(L.lib().bt_batch_set_graph(self._h, 1 if on else 0))

    def set_timing(self, on=True):
        L.check(L.lib().bt_batch_set_timing(self._h, 1 if on else 0))

    def set_flow(self, on=True, blocks_per_sm=FLOW_BLOCKS_PER_SM):
        """Run the refinement levels of later builds as one persistent launch
        of `blocks_per_sm` blocks of 256 threads per SM."""
        L.check(L.lib().bt_batch_set_flow(self._h, blocks_per_sm if on else 0))

    def set_shape(self, threads=128, blocks_per_sm=0, refill=0):
        """Trace launch shape of level builds: threads per block, resident
        blocks per SM (0: as many as fit), idle lanes a warp refills at once
        (0: 8)."""
        s = L.bt_trace_shape(threads, blocks_per_sm, refill)
        L.check(L.lib().bt_batch_set_shape(self._h, C.byref(s)))

    def tune(self, cameras, spins, p99_target=1e-6, repeats=2):
        """The full autotuner (bt_batch_tune): for the mixed form the FP64
        band by accuracy against the plain form, then the fastest of the level
        builds (trace shape x refill size) and the one-launch builds; the set
        keeps it, and a mixed set's options take the chosen band.  Returns a
        dict of the choice."""
        cams, a = self._arrays(cameras, spins)
        r = L.bt_tune_result()
        L.check(L.lib().bt_batch_tune(self._h, cams, a, self.STARTLVL, self.opts.ref,
                                      float(p99_target), int(repeats), C.byref(r),
                                      _stream_ptr(self._stream)))
        for g in self.grids:
            g._info, g._map = None, None
        self._info = None
        if self.opts._o.precision == L.PRECISION_MIXED:
            self.opts._o.fp64_band = r.fp64_band
        return _tune_dict(r)

    def autotune(self, cameras, spins, repeats=2):
        """Times the candidate trace launch shapes on these cameras, keeps
        the fastest; returns ((threads, blocks_per_sm), ms per build)."""
        cams, a = self._arrays(cameras, spins)
        best = L.bt_trace_shape()
        ms = C.c_float()
        L.check(L.lib().bt_batch_autotune(self._h, cams, a, self.STARTLVL, self.opts.ref,
                                          int(repeats), C.byref(best), C.byref(ms),
                                          _stream_ptr(self._stream)))
        for g in self.grids:
            g._info, g._map = None, None
        self._info = None
        return (best.threads, best.blocks_per_sm), ms.value

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None:
            try:
                L.lib().bt_batch_destroy(h)
            except Exception:
                pass
            self._h = None
