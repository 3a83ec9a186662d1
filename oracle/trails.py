"""Star-trail geometry of the reference, restated in numpy -- TEST
INFRASTRUCTURE ONLY (tests/ use it to decide where the reference's own trail
code may be run and which pixels to compare).

addTrails (BT/MakeImageKernel.cu:98-174) picks, for a star seen at pixel
(i, j), the position of the same star in the previous frame's cache whose
displacement best follows the celestial gradient (makeGradField :517-537),
then walks a line from there to (i, j).  That walk (:148-172) can step past
its target and then never ends; before the reference's code runs on a frame
pair, every walk it could take is simulated here.
"""
from __future__ import annotations

import numpy as np

F = np.float32


def grad_field(thphi, M, N):
    """makeGradField on an ((N+1)*(M+1), 2) corner array; the read one past
    the array (last row, last column) is absent."""
    M1, N1 = M + 1, N + 1
    th = np.asarray(thphi, np.float32).reshape(N1 * M1, 2)[:, 0]
    thp = np.concatenate([th, np.array([-2.0], np.float32)])
    g = np.zeros((N1 * M1, 2), np.float32)
    ii, jj = np.meshgrid(np.arange(N1), np.arange(M1), indexing="ij")
    up = th[np.minimum(N, ii + 1) * M1 + jj]
    down = th[np.maximum(0, ii - 1) * M1 + jj]
    left = th[ii * M1 + np.maximum(0, jj - 1)]
    right = thp[np.minimum(ii * M1 + np.minimum(M1, jj + 1), N1 * M1)]
    mid = th[ii * M1 + jj]
    xdir = np.where((up > 0) & (down > 0), F(.5) * (up - mid) - F(.5) * (down - mid), F(0))
    ydir = np.where((left > 0) & (right > 0), F(.5) * (right - mid) - F(.5) * (left - mid), F(0))
    sel = (mid > 0).ravel()
    g[sel, 0] = -ydir.ravel()[sel]
    g[sel, 1] = xdir.ravel()[sel]
    return g


def walk(px, py, i, j, cap=None):
    """The reference's line walk from (px, py) to (i, j) in float32, without
    its own bound.  Returns (pixels, ended, left_box): ended is False when it
    had not stopped after `cap` steps."""
    deltax, deltay = i - px, j - py
    sx = -1 if deltax < 0 else 1
    sy = -1 if deltay < 0 else 1
    deltaerr = F(abs(deltax)) if deltay == 0 else F(abs(F(deltax) / F(deltay)))
    error = F(0)
    x, y = px, py
    cap = cap or 8 * (abs(deltax) + abs(deltay) + 2)
    out, left = [], False
    xlo, xhi, ylo, yhi = min(px, i), max(px, i), min(py, j), max(py, j)
    for _ in range(cap):
        if y == j and x == i:
            return out, True, left
        if error < F(1):
            y += sy
            error = F(error + deltaerr)
        if error >= F(.5):
            x += sx
            error = F(error - F(1))
        if x < xlo or x > xhi or y < ylo or y > yhi:
            left = True
        out.append((x, y))
        d = F(F(x - i) * F(x - i) + F(y - j) * F(y - j))
        if d <= F(1):
            return out, True, left
    return out, False, left


def plan(cache0, n0, cache1, n1, grad, M, N, trailnum):
    """Frame 1's trails from the caches the reference's frame-0 runs leave
    (cache: (stars, trailnum, 2) pixel (i, j), n: hits per star).

    Returns dict(complete: every star's hits fit its cache; safe: every walk
    any candidate could start ends inside its box; writers: lines through
    each pixel under the selection computed here in float32 (acosf rounding
    may pick another candidate in rare ties))."""
    M1 = M + 1
    complete = bool((n0 <= trailnum).all() and (n1 <= trailnum).all())
    safe = True
    writers = np.zeros(N * M, np.int32)
    for q in np.nonzero(n1)[0]:
        prevs = cache0[q, :min(int(n0[q]), trailnum)]
        for (i, j) in cache1[q, :min(int(n1[q]), trailnum)]:
            i, j = int(i), int(j)
            angle, best, line = F(2 * np.pi), None, False
            for (px, py) in prevs:
                px, py = int(px), int(py)
                dx, dy = px - i, py - j
                if dx * dx <= 1 and dy * dy <= 1:
                    line = False
                    break
                dist = F(np.sqrt(F(dx * dx + dy * dy)))
                if dist > F(M) / F(25):
                    continue
                _, ended, left = walk(px, py, i, j)
                if not ended or left:
                    safe = False
                gr = grad[px * M1 + py]
                div = F(dist * F(np.sqrt(F(gr[0] * gr[0] + gr[1] * gr[1]))))
                with np.errstate(all="ignore"):
                    a1 = np.arccos(F(F(F(dx) * gr[0] + F(dy) * gr[1]) / div))
                    a2 = np.arccos(F(F(F(dx) * -gr[0] + F(dy) * -gr[1]) / div))
                a = np.fmin(a1, a2)
                if a > angle or a > F(np.pi) * F(.25):
                    continue
                if a < angle:
                    angle, best, line = a, (px, py), True
            if line:
                pix, _, _ = walk(best[0], best[1], i, j)
                for (x, y) in pix:
                    if 0 <= x < N and 0 <= y < M:
                        writers[x * M + y] += 1
    return dict(complete=complete, safe=safe, writers=writers)
