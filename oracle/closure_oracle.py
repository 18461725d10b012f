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


# -- closure tendencies -------------------------------------------------------
# The tendencies the coarse run adds to its right-hand sides from the
# network's 12 outputs P (stress tau_xx, tau_yy, tau_zz, tau_xy, tau_xz,
# tau_yz; heat flux q_x, q_y, q_z; EMF eps_x, eps_y, eps_z, each times its
# scale): centred differences with the grid's metric factors, periodic in x
# and y, zero on the first and last z plane.  Output fields RU, RV, RW, TT,
# BX, BY, BZ.  (field, direction, sign) of every output channel; TT's terms
# are also divided by the cell's density.
TEND_TERMS = {
    0: [(0, 0, -1.0)], 1: [(1, 1, -1.0)], 2: [(2, 2, -1.0)],
    3: [(0, 1, -1.0), (1, 0, -1.0)], 4: [(0, 2, -1.0), (2, 0, -1.0)], 5: [(1, 2, -1.0), (2, 1, -1.0)],
    6: [(3, 0, -1.0)], 7: [(3, 1, -1.0)], 8: [(3, 2, -1.0)],
    9: [(5, 2, 1.0), (6, 1, -1.0)], 10: [(6, 0, 1.0), (4, 2, -1.0)], 11: [(4, 1, 1.0), (5, 0, -1.0)],
}


def _metric(ax, ay, az, d, shape):
    nz, ny, nx = shape
    if d == 0:
        return np.broadcast_to(np.asarray(ax)[None, None, :], shape)
    if d == 1:
        return np.broadcast_to(np.asarray(ay)[None, :, None], shape)
    return np.broadcast_to(np.asarray(az)[:, None, None], shape)


def _cdiff(a, d):
    """a[n+1] - a[n-1] along axis d of [z][y][x] (2 - d); periodic in x, y."""
    axis = 2 - d
    if d < 2:
        return np.roll(a, -1, axis=axis) - np.roll(a, 1, axis=axis)
    out = np.zeros_like(a)
    out[1:-1] = a[2:] - a[:-2]
    return out


def tendency_fwd(pred, osc, ax, ay, az, ro):
    """pred [z][y][x][>=12] (normalised outputs), osc[12] scales, ax[nx],
    ay[ny], az[nz] metric factors of the cells, ro [z][y][x] density.
    Returns [7][z][y][x]."""
    shape = pred.shape[:3]
    out = np.zeros((7,) + shape)
    for c, terms in TEND_TERMS.items():
        p = np.asarray(pred[..., c], dtype=np.float64) * float(osc[c])
        for f, d, s in terms:
            t = s * _cdiff(p, d) * _metric(ax, ay, az, d, shape)
            out[f] += t / ro if f == 3 else t
    out[:, 0] = 0.0
    out[:, -1] = 0.0
    return out


def tendency_adj(g, osc, ax, ay, az, ro):
    """Adjoint of tendency_fwd: g [7][z][y][x] -> dpred [z][y][x][16]."""
    shape = g.shape[1:]
    gi = np.array(g, dtype=np.float64)
    gi[:, 0] = 0.0
    gi[:, -1] = 0.0
    out = np.zeros(shape + (16,))
    for c, terms in TEND_TERMS.items():
        acc = np.zeros(shape)
        for f, d, s in terms:
            h = gi[f] * _metric(ax, ay, az, d, shape)
            if f == 3:
                h = h / ro
            # adjoint of a[n+1] - a[n-1]: h[m-1] - h[m+1]
            axis = 2 - d
            if d < 2:
                acc += s * (np.roll(h, 1, axis=axis) - np.roll(h, -1, axis=axis))
            else:
                t = np.zeros(shape)
                t[1:] += h[:-1]
                t[:-1] -= h[1:]
                acc += s * t
        out[..., c] = acc * float(osc[c])
    return out
