"""The CPU checker of the closure convolution: its input and weight gradients
are the exact adjoints of its forward pass (inner-product identities)."""
import numpy as np

from closure_oracle import conv3d_dw, conv3d_dx, conv3d_fwd


def test_adjoint_identities():
    rng = np.random.default_rng(0)
    for shape, cin, cout in (((4, 5, 6), 3, 2), ((3, 4, 8), 16, 32)):
        x = rng.standard_normal(shape + (cin,))
        w = rng.standard_normal((cout, 27 * cin))
        dy = rng.standard_normal(shape + (cout,))
        e = rng.standard_normal(x.shape)
        assert np.isclose(np.sum(conv3d_fwd(e, w) * dy), np.sum(e * conv3d_dx(dy, w, cin)), rtol=1e-12)
        ew = rng.standard_normal(w.shape)
        dw, db = conv3d_dw(x, dy)
        assert np.isclose(np.sum(conv3d_fwd(x, ew) * dy), np.sum(ew * dw), rtol=1e-12)
        assert np.allclose(db, dy.reshape(-1, cout).sum(axis=0))


def test_periodic_and_wall_padding():
    # a single nonzero voxel at x=0 reaches x=nx-1 (periodic) but not across the z ends
    x = np.zeros((3, 4, 8, 1))
    x[0, 0, 0, 0] = 1.0
    w = np.zeros((1, 27))
    w[0, 0] = 1.0     # tap (dx,dy,dz) = (-1,-1,-1): out[z,y,x] = x[z-1,y-1,x-1]
    out = conv3d_fwd(x, w)[..., 0]
    assert out[1, 1, 1] == 1.0 and out.sum() == 1.0
    w2 = np.zeros((1, 27))
    w2[0, 13 + 1] = 1.0   # tap (+1,0,0): out[z,y,x] = x[z,y,x+1]
    out2 = conv3d_fwd(x, w2)[..., 0]
    assert out2[0, 0, 7] == 1.0 and out2.sum() == 1.0


def test_tendency_adjoint_identity():
    from closure_oracle import tendency_adj, tendency_fwd
    rng = np.random.default_rng(3)
    nz, ny, nx = 6, 5, 8
    p = rng.standard_normal((nz, ny, nx, 16))
    osc = rng.uniform(0.5, 2.0, 12)
    ax, ay, az = rng.uniform(1, 2, nx), rng.uniform(1, 2, ny), rng.uniform(1, 2, nz)
    ro = rng.uniform(0.5, 1.5, (nz, ny, nx))
    g = rng.standard_normal((7, nz, ny, nx))
    t = tendency_fwd(p, osc, ax, ay, az, ro)
    assert not t[:, 0].any() and not t[:, -1].any()
    d = tendency_adj(g, osc, ax, ay, az, ro)
    assert not d[..., 12:].any()
    assert np.isclose(np.sum(t * g), np.sum(p * d), rtol=1e-12)
    # one stress component: RU's tendency is minus the x difference of tau_xx
    q = np.zeros_like(p)
    q[2, 2, 3, 0] = 1.0
    t = tendency_fwd(q, np.ones(12), np.ones(nx), np.ones(ny), np.ones(nz), np.ones((nz, ny, nx)))
    assert t[0, 2, 2, 2] == -1.0 and t[0, 2, 2, 4] == 1.0 and np.abs(t).sum() == 2.0
