"""Python mirror of the frame server (bt_server in include/blacktracer.h).

A worker thread inside the library renders submitted frame requests --
resolution, camera and spin each -- with continuous batching: admission by
HBM budget and in-flight slots, grids resident in a cache keyed by the exact
camera and spin and reused, missing grids built together as one grid set,
frames of different requests overlapping on their own streams.
"""
from __future__ import annotations

import ctypes as C

from . import _lib as L
from .host import Camera, _opts


class Server:
    def __init__(self, env=None, stars=None, maxlevel=11, startlevel=6, angle=True,
                 precision="fast", grid_cache_bytes=40 << 30, render_bytes=40 << 30,
                 max_inflight=16, max_build_batch=8, step=1, lr=True):
        cfg = L.bt_server_config()
        L.lib().bt_server_config_default(C.byref(cfg))
        cfg.maxlevel, cfg.startlevel = int(maxlevel), int(startlevel)
        cfg.angle = 1 if angle else 0
        cfg.precision = _opts(precision)._o.precision
        cfg.grid_cache_bytes, cfg.render_bytes = int(grid_cache_bytes), int(render_bytes)
        cfg.max_inflight, cfg.max_build_batch = int(max_inflight), int(max_build_batch)
        cfg.env = env._h if env is not None else None
        cfg.stars = stars._h if stars is not None else None
        cfg.step, cfg.lr = int(step), 1 if lr else 0
        self._keep = (env, stars)  # must outlive the server
        h = C.c_void_p()
        L.check(L.lib().bt_server_create(C.byref(cfg), C.byref(h)))
        self._h = h
        self._outs = {}

    def submit(self, rid: int, width: int, height: int, cam: Camera, a: float, out):
        """out: a (height, width, 4) uint8 tensor in pinned host or device
        memory, kept alive here until the request completes."""
        r = L.bt_request()
        r.id, r.width, r.height = int(rid), int(width), int(height)
        r.cam = cam._c
        r.a = float(a)
        r.out = out.data_ptr()
        self._outs[int(rid)] = out
        L.check(L.lib().bt_server_submit(self._h, C.byref(r)))

    def poll(self, cap=256, wait_ms=0):
        """Completed requests (dicts with id, status, grid_reused and the
        submit / admit / done times in seconds)."""
        buf = (L.bt_completion * cap)()
        n = C.c_int()
        L.check(L.lib().bt_server_poll(self._h, buf, cap, C.byref(n), int(wait_ms)))
        res = []
        for k in range(n.value):
            c = buf[k]
            self._outs.pop(int(c.id), None)
            res.append(dict(id=int(c.id), status=int(c.status), grid_reused=bool(c.grid_reused),
                            t_submit=c.t_submit, t_admit=c.t_admit, t_done=c.t_done))
        return res

    def stats(self) -> dict:
        st = L.bt_server_stats()
        L.check(L.lib().bt_server_stats_get(self._h, C.byref(st)))
        return {f: int(getattr(st, f)) for f, _ in st._fields_}

    def close(self):
        """Finishes every submitted request, then releases the server."""
        h = getattr(self, "_h", None)
        if h is not None:
            L.lib().bt_server_destroy(h)
            self._h = None
            self._outs.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
