"""The reference's cache files and its perfect spatial hash (PSH) of a grid.

* ``.grid`` -- Grid::serialize (BT/Grid.h:36-39): MAXLEVEL, N, M and the
  PSHOffsetTable of the grid's vertices (BT/PSHOffsetTable.h:44-48).
* ``.star`` -- StarProcessor::serialize (BT/StarProcessor.h:21-23).

Files are read and written by the library (cereal's binary archive layout,
without cereal); a loaded grid file becomes a device map grid
(:class:`GridFile`) that :class:`blacktracer_b200.Renderer` renders like a
built :class:`blacktracer_b200.Grid`.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _lib as L
from .host import _stream_ptr, _torch


def _path(p) -> bytes:
    return os.fsencode(os.fspath(p))


def psh_build(keys, values) -> dict:
    """PSHOffsetTable(elements, datapoints) (BT/PSHOffsetTable.h:350-370):
    keys (n, 2) int32 lattice (i, j), values (n, 2) float32.  Returns
    dict(hash_table (hw*hw, 2) float32, pos_tag (hw*hw, 2) int32,
    offset_table (ow*ow, 2) int32, hash_width, offset_width)."""
    k = np.ascontiguousarray(keys, dtype=np.int32).reshape(-1, 2)
    v = np.ascontiguousarray(values, dtype=np.float32).reshape(-1, 2)
    if len(k) != len(v):
        raise ValueError("keys and values differ in length")
    n = len(k)
    # room for the widths the first attempts use, so one call usually does
    hw, ow = int((1.1 * n) ** 0.5 * 1.2) + 8, int((n / 4) ** 0.5 * 1.5) + 16
    for _ in range(2):
        buf = dict(hash_table=np.empty((hw * hw, 2), np.float32),
                   pos_tag=np.empty((hw * hw, 2), np.int32),
                   offset_table=np.empty((ow * ow, 2), np.int32))
        t = L.bt_psh()
        _fill(t, buf)
        rc = L.lib().bt_psh_build(k.ctypes.data, v.ctypes.data, n, C.byref(t))
        if rc == L.BT_OK:
            hw, ow = t.hash_width, t.offset_width
            return dict(hash_table=buf["hash_table"][:hw * hw].copy(),
                        pos_tag=buf["pos_tag"][:hw * hw].copy(),
                        offset_table=buf["offset_table"][:ow * ow].copy(),
                        hash_width=hw, offset_width=ow)
        if rc != L.BT_ERR_ARG or t.hash_width <= 0:
            L.check(rc)
        hw, ow = t.hash_width, t.offset_width
    L.check(rc)


def _fill(t, d):
    t.hash_table = d["hash_table"].ctypes.data
    t.pos_tag = d["pos_tag"].ctypes.data
    t.offset_table = d["offset_table"].ctypes.data
    t.cap_hash = d["hash_table"].size
    t.cap_offset = d["offset_table"].size


def write_grid_file(path, maxlevel, N, M, psh: dict) -> None:
    """A .grid file from a PSH (as :func:`psh_build` returns it)."""
    t = L.bt_psh()
    d = {k: np.ascontiguousarray(psh[k]) for k in ("hash_table", "pos_tag", "offset_table")}
    _fill(t, d)
    t.hash_width, t.offset_width = int(psh["hash_width"]), int(psh["offset_width"])
    L.check(L.lib().bt_grid_file_write(_path(path), int(maxlevel), int(N), int(M), C.byref(t)))


def read_grid_file(path) -> dict:
    """A .grid file: dict(MAXLEVEL, N, M, hash_table, pos_tag, offset_table,
    hash_width, offset_width)."""
    ml, N, M = C.c_int32(), C.c_int32(), C.c_int32()
    t = L.bt_psh()
    rc = L.lib().bt_grid_file_read(_path(path), C.byref(ml), C.byref(N), C.byref(M),
                                   C.byref(t))
    if rc != L.BT_ERR_ARG or t.hash_width <= 0:
        L.check(rc)
    hw, ow = t.hash_width, t.offset_width
    out = dict(hash_table=np.empty((hw * hw, 2), np.float32),
               pos_tag=np.empty((hw * hw, 2), np.int32),
               offset_table=np.empty((ow * ow, 2), np.int32))
    _fill(t, out)
    L.check(L.lib().bt_grid_file_read(_path(path), C.byref(ml), C.byref(N), C.byref(M),
                                      C.byref(t)))
    out.update(MAXLEVEL=ml.value, N=N.value, M=M.value, hash_width=hw, offset_width=ow)
    return out


def write_star_file(path, starPos, starMag, binaryStarTree, treeLevel) -> None:
    pos = np.ascontiguousarray(starPos, dtype=np.float32)
    mag = np.ascontiguousarray(starMag, dtype=np.float32)
    tree = np.ascontiguousarray(binaryStarTree, dtype=np.int32)
    if pos.size != mag.size or pos.size % 2:
        raise ValueError("starPos and starMag must hold 2 floats per star")
    if tree.size != L.lib().bt_stars_tree_size(int(treeLevel)):
        raise ValueError("binaryStarTree does not match treeLevel")
    L.check(L.lib().bt_stars_file_write(_path(path), pos.ctypes.data, mag.ctypes.data,
                                        pos.size // 2, tree.ctypes.data, int(treeLevel)))


def read_star_file(path):
    """(starPos, starMag, binaryStarTree, treeLevel) of a .star file."""
    n, lv = C.c_int(), C.c_int()
    L.check(L.lib().bt_stars_file_info(_path(path), C.byref(n), C.byref(lv)))
    pos = np.empty(2 * n.value, np.float32)
    mag = np.empty(2 * n.value, np.float32)
    tree = np.empty(L.lib().bt_stars_tree_size(lv.value), np.int32)
    L.check(L.lib().bt_stars_file_read(_path(path), pos.ctypes.data, mag.ctypes.data,
                                       n.value, tree.ctypes.data, tree.size))
    return pos, mag, tree, lv.value


class GridFile:
    """A .grid file loaded into a device map grid: the reference's cached
    grid (BT/BlackTracer.cpp:236-242) expanded by makeGrid
    (BT/MakeImageKernel.cu:369-384) on the device.  Renders like a Grid:
    ``Renderer.render(GridFile(path), view, cam, ...)``."""

    def __init__(self, path, stream=None):
        torch = _torch()
        ml, rows, cols, sym = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
        L.check(L.lib().bt_grid_file_map_shape(_path(path), C.byref(ml), C.byref(rows),
                                               C.byref(cols), C.byref(sym)))
        self.MAXLEVEL, self.rows, self.cols, self.sym = ml.value, rows.value, cols.value, \
            sym.value
        self.grid = torch.empty((self.rows * self.cols, 2), dtype=torch.float32, device="cuda")
        L.check(L.lib().bt_grid_file_load_map(_path(path), self.grid.data_ptr(), self.rows,
                                              self.cols, _stream_ptr(stream)))

    def map_grid(self):
        """(pointer, rows, cols, sym), as Grid.map_grid."""
        return (self.grid.data_ptr(), self.rows, self.cols, self.sym)
