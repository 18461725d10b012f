"""CPU checker of the learned-closure kernels (test infrastructure only).

numpy restatement of the 3x3x3 convolution the closure network uses:
channels-last arrays [z][y][x][C], periodic in x and y, zero outside in z;
weights [COUT][27*CIN] with k = tap*CIN + ci and tap = (dx+1) + 3*(dy+1) +
9*(dz+1), so out[z,y,x,n] = bias[n] + sum_{tap,ci} x[z+dz, y+dy, x+dx, ci] *
w[n, tap*CIN+ci].  Forward, input gradient and weight gradient in FP64.
"""
from __future__ import annotations

import numpy as np


def _taps():
    for tap in range(27):
        yield tap, tap % 3 - 1, (tap // 3) % 3 - 1, tap // 9 - 1


def _shift(a, dx, dy, dz):
    """s[z,y,x] = a[z+dz, y+dy, x+dx] (periodic x, y; zero outside in z)."""
    nz = a.shape[0]
    s = np.roll(np.roll(a, -dy, axis=1), -dx, axis=2)
    out = np.zeros_like(s)
    lo, hi = max(0, -dz), min(nz, nz - dz)
    if hi > lo:
        out[lo:hi] = s[lo + dz:hi + dz]
    return out


def conv3d_fwd(x, w, b=None, relu=False):
    x = np.asarray(x, dtype=np.float64)
    w = np.asarray(w, dtype=np.float64)
    cin = x.shape[3]
    out = np.zeros(x.shape[:3] + (w.shape[0],))
    for tap, dx, dy, dz in _taps():
        out += _shift(x, dx, dy, dz) @ w[:, tap * cin:(tap + 1) * cin].T
    if b is not None:
        out += np.asarray(b, dtype=np.float64)
    return np.maximum(out, 0.0) if relu else out


def conv3d_dx(dy, w, cin):
    """Gradient of sum(out * dy) with respect to x (no activation)."""
    dy = np.asarray(dy, dtype=np.float64)
    w = np.asarray(w, dtype=np.float64)
    dx = np.zeros(dy.shape[:3] + (cin,))
    for tap, ddx, ddy, ddz in _taps():
        dx += _shift(dy, -ddx, -ddy, -ddz) @ w[:, tap * cin:(tap + 1) * cin]
    return dx


def conv3d_dw(x, dy):
    x = np.asarray(x, dtype=np.float64)
    dy = np.asarray(dy, dtype=np.float64)
    cin, cout = x.shape[3], dy.shape[3]
    dw = np.zeros((cout, 27 * cin))
    g = dy.reshape(-1, cout)
    for tap, dx, ddy, dz in _taps():
        dw[:, tap * cin:(tap + 1) * cin] = g.T @ _shift(x, dx, ddy, dz).reshape(-1, cin)
    return dw, g.sum(axis=0)
