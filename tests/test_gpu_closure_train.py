"""The learned closure end to end on the GPU: coarsening and targets against
numpy, network gradients against the CPU checker layer by layer, the
error-indicator fallback (bit-identical to the plain coarse step), and what a
trained network gains a priori over the method without it."""
import ctypes as C

import numpy as np
import pytest

from closure_oracle import conv3d_dw, conv3d_dx, conv3d_fwd, tendency_adj, tendency_fwd
from test_gpu_parity import _gpu_or_skip

pytestmark = pytest.mark.gpu


def _np(t):
    return t.double().cpu().numpy() if t.dtype != np.float64 else t


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def test_coarsen_against_numpy(mhd3d):
    _gpu_or_skip(mhd3d)
    torch = pytest.importorskip("torch")
    lib = mhd3d.gpu_lib()
    setup = mhd3d.make_setup(mhd3d.convection_config(16, 12, 8, ampt=0.05, seed=3))
    g = mhd3d.GpuSim(setup, mode=mhd3d.MODE_FAST)
    g.upload(setup.state)
    g.step(3)
    st = g.download()
    fac = 4
    nc = (4 + 2) * (3 + 2) * (2 + 2)
    cs = torch.zeros(8 * nc, dtype=torch.float64, device="cuda")
    tg = torch.zeros((2, 3, 4, 12), dtype=torch.float32, device="cuda")
    assert lib.mhd3d_coarsen(g.h, fac, _p(cs), _p(tg), None) == 0
    torch.cuda.synchronize()
    # numpy box filter of the interior, blocks of 4x4x4 (arrays [i, j, k] Fortran order)
    it = {f: st[f][1:-1, 1:-1, 1:-1] for f in mhd3d.FIELDS}

    def box(a):
        return a.reshape(4, fac, 3, fac, 2, fac).mean(axis=(1, 3, 5))
    ro, m = it["ro"], [it["ru"], it["rv"], it["rw"]]
    u = [x / ro for x in m]
    R, M, E = box(ro), [box(x) for x in m], box(ro * it["tt"])
    B = [box(it[f]) for f in ("bx", "by", "bz")]
    pairs = [(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]
    ref = [box(m[a] * u[b]) - M[a] * M[b] / R for a, b in pairs]
    ref += [box(m[a] * it["tt"]) - M[a] * E / R for a in range(3)]
    bx, by, bz = it["bx"], it["by"], it["bz"]
    X = [box(u[1] * bz - u[2] * by), box(u[2] * bx - u[0] * bz), box(u[0] * by - u[1] * bx)]
    V = [M[a] / R for a in range(3)]
    ref += [X[0] - (V[1] * B[2] - V[2] * B[1]), X[1] - (V[2] * B[0] - V[0] * B[2]), X[2] - (V[0] * B[1] - V[1] * B[0])]
    got = tg.double().cpu().numpy()   # [k][j][i][c]
    for c in range(12):
        r = np.transpose(ref[c], (2, 1, 0))
        assert np.abs(got[..., c] - r).max() <= 1e-6 * max(np.abs(r).max(), 1e-30), c
    csn = cs.cpu().numpy()
    sh = (6, 5, 4)
    ro_c = csn[4 * nc:5 * nc].reshape(sh, order="F")
    assert np.allclose(ro_c[1:-1, 1:-1, 1:-1], R, rtol=1e-13, atol=0)
    tt_c = csn[3 * nc:4 * nc].reshape(sh, order="F")
    assert np.allclose(tt_c[1:-1, 1:-1, 1:-1], E / R, rtol=1e-13, atol=0)
    g.close()


def test_network_gradients_layer_by_layer(mhd3d):
    """Each backward kernel against the checker on the GPU's own intermediates."""
    _gpu_or_skip(mhd3d)
    torch = pytest.importorskip("torch")
    import closure
    shape = (4, 3, 128)
    net = closure.ClosureNet(seed=5)
    rng = np.random.default_rng(1)
    f = np.zeros(shape + (16,))
    f[..., :8] = rng.standard_normal(shape + (8,))
    feat = torch.tensor(f, dtype=torch.bfloat16, device="cuda")
    tgt = torch.tensor(rng.standard_normal(shape + (12,)), dtype=torch.float32, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    acts, pred = net.forward(feat, shape, s)
    loss, dy3 = net.loss_and_grad(pred, tgt, s)
    torch.cuda.synchronize()
    W = [w.double().cpu().numpy() for w in net.w16]
    Bv = [b.double().cpu().numpy() for b in net.b]
    A = [a.double().cpu().numpy() for a in acts]
    P = pred.double().cpu().numpy()
    # forward of each layer on its (BF16) input
    for li in range(2):
        ref = conv3d_fwd(A[li], W[li], Bv[li], relu=True)
        assert np.abs(A[li + 1] - ref).max() <= 8e-3 * np.abs(ref).max()
    ref = conv3d_fwd(A[2], W[2], Bv[2])
    assert np.abs(P - ref).max() <= 2e-5 * np.abs(ref).max()
    # loss and its gradient
    t = tgt.double().cpu().numpy()
    d = P[..., :12] - t
    n = np.prod(shape) * 12
    assert abs(loss.item() - (d * d).sum() / n) <= 1e-9 * abs(loss.item())
    g3 = dy3.double().cpu().numpy()
    assert np.abs(g3[..., :12] - 2 * d / n).max() <= 8e-3 * np.abs(2 * d / n).max()
    assert not g3[..., 12:].any()
    # backward, layer by layer
    net.zero_grad()
    dy = dy3
    for li in (2, 1, 0):
        cin, cout, _ = closure.LAYERS[li]
        G = dy.double().cpu().numpy()
        assert mhd3d.gpu_lib().mhd3d_conv3d_wgrad(cin, cout, _p(acts[li]), _p(dy), _p(net.dw[li]), _p(net.db[li]),
                                                  shape[2], shape[1], shape[0], C.c_void_p(s)) == 0
        torch.cuda.synchronize()
        rdw, rdb = conv3d_dw(A[li], G)
        assert np.abs(net.dw[li].double().cpu().numpy() - rdw).max() <= 2e-5 * np.abs(rdw).max()
        assert np.abs(net.db[li].double().cpu().numpy() - rdb).max() <= 2e-5 * np.abs(rdb).max()
        if li == 0:
            break
        wt = torch.empty((cin, 27 * cout), dtype=torch.bfloat16, device="cuda")
        assert mhd3d.gpu_lib().mhd3d_conv3d_wtranspose(cin, cout, _p(net.w16[li]), _p(wt), C.c_void_p(s)) == 0
        dxf = torch.empty(shape + (cin,), dtype=torch.float32, device="cuda")
        assert mhd3d.gpu_lib().mhd3d_conv3d(cout, cin, _p(dy), _p(wt), None, _p(acts[li]), 0, None, _p(dxf),
                                            shape[2], shape[1], shape[0], _p(net.err), C.c_void_p(s)) == 0
        torch.cuda.synchronize()
        rdx = conv3d_dx(G, W[li], cin) * (A[li] > 0)
        assert np.abs(dxf.double().cpu().numpy() - rdx).max() <= 2e-5 * np.abs(rdx).max()
        dy = dxf.to(torch.bfloat16)
    assert int(net.err.item()) == 0


def test_tendency_loss_and_adjoint(mhd3d):
    """The closure tendencies, their weighted loss and the adjoint that turns
    the loss gradient into the last layer's dy, against the numpy checker."""
    _gpu_or_skip(mhd3d)
    torch = pytest.importorskip("torch")
    from test_gpu_parity import _random_state
    lib = mhd3d.gpu_lib()
    setup = mhd3d.make_setup(mhd3d.convection_config(32, 12, 10, ra=1e5, ta=1e4, seed=4))
    st = _random_state(mhd3d, setup, seed=5, amp=0.05)
    g = mhd3d.GpuSim(setup, mode=mhd3d.MODE_FP32)
    g.upload(st)
    p = g.params
    nz, ny, nx = p.npz, p.npy, p.npx
    rng = np.random.default_rng(2)
    pred = torch.tensor(rng.standard_normal((nz, ny, nx, 16)), dtype=torch.float32, device="cuda")
    osc = torch.tensor(rng.uniform(0.5, 2.0, 12), dtype=torch.float32, device="cuda")
    ax = p.hx * setup.grid["dxxdx"][1:-1]
    ay = p.hy * setup.grid["dyydy"][1:-1]
    az = p.hz * setup.grid["dzzdz"][1:-1]
    ro = np.transpose(st["ro"][1:-1, 1:-1, 1:-1], (2, 1, 0))
    s = torch.cuda.current_stream().cuda_stream
    tend = torch.empty((7, nz, ny, nx), dtype=torch.float32, device="cuda")
    flag = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert lib.mhd3d_closure_tendency(g.h, _p(pred), _p(osc), _p(tend), _p(flag), C.c_float(1e30), C.c_void_p(s)) == 0
    torch.cuda.synchronize()
    P, O = pred.double().cpu().numpy(), osc.double().cpu().numpy()
    ref = tendency_fwd(P, O, ax, ay, az, ro)
    assert np.abs(tend.double().cpu().numpy() - ref).max() <= 1e-5 * np.abs(ref).max()
    # loss and gradient against a target
    tgt = torch.tensor(rng.standard_normal((7, nz, ny, nx)), dtype=torch.float32, device="cuda")
    w = torch.tensor(rng.uniform(0.5, 2.0, 7), dtype=torch.float32, device="cuda")
    gr = torch.empty_like(tend)
    loss = torch.zeros(1, dtype=torch.float64, device="cuda")
    assert lib.mhd3d_closure_tendency_loss(_p(tend), _p(tgt), _p(w), nz * ny * nx, _p(gr), _p(loss), C.c_void_p(s)) == 0
    torch.cuda.synchronize()
    T, R, W = tend.double().cpu().numpy(), tgt.double().cpu().numpy(), w.double().cpu().numpy()
    n = 7 * nz * ny * nx
    d = T - R
    assert abs(loss.item() - (W[:, None, None, None] * d * d).sum() / n) <= 1e-9 * loss.item()
    G = gr.double().cpu().numpy()
    assert np.abs(G - 2 * W[:, None, None, None] * d / n).max() <= 1e-6 * np.abs(G).max()
    # adjoint (BF16 output)
    dy = torch.empty((nz, ny, nx, 16), dtype=torch.bfloat16, device="cuda")
    assert lib.mhd3d_closure_tendency_adjoint(g.h, _p(gr), _p(osc), _p(dy), C.c_void_p(s)) == 0
    torch.cuda.synchronize()
    radj = tendency_adj(G, O, ax, ay, az, ro)
    got = dy.double().cpu().numpy()
    assert np.abs(got - radj).max() <= 8e-3 * np.abs(radj).max()
    assert not got[..., 12:].any()
    # the same through the training helper
    import closure
    net = closure.ClosureNet(seed=0)
    net.out_scale = osc
    l2, dy2 = net.tendency_loss_and_grad(g, pred, tgt, w, s)
    torch.cuda.synchronize()
    assert abs(l2.item() - loss.item()) <= 1e-12 * loss.item()
    assert torch.equal(dy2, dy)
    g.close()


def _coarse_setup(mhd3d, npx=128):
    return mhd3d.make_setup(mhd3d.convection_config(npx, 16, 16, ra=1e5, ta=1e4, ampt=1e-2, seed=2))


@pytest.mark.parametrize("npx", [128, 96, 24])
def test_closure_fallback_is_the_plain_step(mhd3d, npx):
    _gpu_or_skip(mhd3d)
    pytest.importorskip("torch")
    import closure
    setup = _coarse_setup(mhd3d, npx)
    plain = mhd3d.GpuSim(setup, mode=mhd3d.MODE_FP32)
    plain.upload(setup.state)
    plain.step(12)
    ref = plain.download()
    g = mhd3d.GpuSim(setup, mode=mhd3d.MODE_FP32)
    g.upload(setup.state)
    net = closure.ClosureNet(seed=1)
    net.attach(g, trip=0.0)          # every evaluation trips: the plain coarse method runs
    g.step(12)
    got = g.download()
    s = g.closure_status()
    assert s["evals"] == 12 and s["trips"] == 12 and s["err"] == 0
    for f in mhd3d.FIELDS:
        assert np.array_equal(got[f], ref[f]), f
    # a closure that never trips changes the run and keeps it finite
    h = mhd3d.GpuSim(setup, mode=mhd3d.MODE_FP32)
    h.upload(setup.state)
    net.attach(h, trip=1e30)
    h.step(12)
    s = h.closure_status()
    assert s["evals"] == 12 and s["trips"] == 0 and s["err"] == 0
    got2 = h.download()
    assert all(np.isfinite(got2[f]).all() for f in mhd3d.FIELDS)
    assert any(not np.array_equal(got2[f], ref[f]) for f in mhd3d.FIELDS)


def test_closure_bias_is_a_per_plane_tendency(mhd3d):
    """With the network's outputs scaled to zero, the closure's tendency is its
    per-plane bias alone: a constant RU bias integrates to dt*b over one RK3
    step on the interior planes (the coupling through the right-hand side is
    second order in dt*b here), and a zero bias leaves the plain step."""
    _gpu_or_skip(mhd3d)
    torch = pytest.importorskip("torch")
    import closure
    setup = _coarse_setup(mhd3d, 64)
    npz = setup.params.npz
    plain = mhd3d.GpuSim(setup, mode=mhd3d.MODE_FP32)
    plain.upload(setup.state)
    r0 = plain.step(1)
    ref = plain.download()
    net = closure.ClosureNet(seed=1)
    net.out_scale = torch.zeros(12, device="cuda")
    g = mhd3d.GpuSim(setup, mode=mhd3d.MODE_FP32)
    g.upload(setup.state)
    net.attach(g, trip=1e30)
    g.closure_set_bias(np.zeros((7, npz), dtype=np.float32))
    g.step(1)
    same = g.download()
    for f in mhd3d.FIELDS:
        assert np.array_equal(same[f], ref[f]), f
    g.close()
    b = 1e-3
    bias = np.zeros((7, npz), dtype=np.float32)
    bias[0, 1:-1] = b
    h = mhd3d.GpuSim(setup, mode=mhd3d.MODE_FP32)
    h.upload(setup.state)
    net.attach(h, trip=1e30)
    h.closure_set_bias(torch.tensor(bias, device="cuda"))
    h.step(1)
    got = h.download()
    assert h.closure_status()["trips"] == 0
    d = (got["ru"] - ref["ru"])[1:-1, 1:-1, 4:-4] / (r0["dt"] * b)
    assert np.abs(d - 1.0).max() < 0.05, np.abs(d - 1.0).max()
    # without a network the bias stands alone: the same step, no evaluation
    e = mhd3d.GpuSim(setup, mode=mhd3d.MODE_FP32)
    e.upload(setup.state)
    e.closure_set_bias(bias)
    e.step(1)
    alone = e.download()
    for f in mhd3d.FIELDS:
        assert np.array_equal(alone[f], got[f]), f
    assert e.closure_status()["evals"] == 0
    # detaching the network from h leaves its bias alone as well
    h.upload(setup.state)
    net.detach(h)
    h.step(1)
    again = h.download()
    for f in mhd3d.FIELDS:
        assert np.array_equal(again[f], got[f]), f
    e.closure_set_bias(None)
    e.upload(setup.state)
    e.step(1)
    back = e.download()
    for f in mhd3d.FIELDS:
        assert np.array_equal(back[f], ref[f]), f
    e.close()
    h.closure_set_bias(None)
    h.close()
    plain.close()


def test_trained_network_gains_over_no_closure(mhd3d):
    """A priori: on held-out snapshots the trained closure's subgrid tendencies
    are closer to the filtered fine run's than no closure (zero) is."""
    _gpu_or_skip(mhd3d)
    torch = pytest.importorskip("torch")
    import closure
    fine_setup = mhd3d.make_setup(mhd3d.convection_config(512, 64, 64, ra=1e6, ta=1e4, ampt=5e-2, seed=9))
    coarse_setup = mhd3d.make_setup(mhd3d.convection_config(128, 16, 16, ra=1e6, ta=1e4, ampt=5e-2, seed=9))
    fine = mhd3d.GpuSim(fine_setup, mode=mhd3d.MODE_FAST)
    fine.upload(fine_setup.state)
    pc = closure.PairCollector(fine_setup, coarse_setup)
    ones = torch.ones(8, dtype=torch.float32, device="cuda")
    raw = []
    for _ in range(12):
        fine.step(25)
        raw.append(pc.snapshot(fine, ones))
    feats = torch.stack([f for f, _ in raw]).float()
    tgts = torch.stack([t for _, t in raw])
    net = closure.ClosureNet(seed=3)
    net.in_scale = (1.0 / feats[..., :8].reshape(-1, 8).std(dim=0).clamp_min(1e-12)).contiguous()
    net.out_scale = tgts.reshape(-1, 12).std(dim=0).clamp_min(1e-30).contiguous()
    data = [((f.float()[..., :16] * torch.cat([net.in_scale, torch.ones(8, device="cuda")])).to(torch.bfloat16),
             (t / net.out_scale).contiguous()) for f, t in raw]
    # train on the first ten snapshots; hold out the last (the collector's coarse state is the last one's)
    train, test = data[:10], data[11:]
    s = torch.cuda.current_stream().cuda_stream
    shape = pc.shape

    def mean_loss(sets):
        tot = 0.0
        for f, t in sets:
            _, p = net.forward(f, shape, s)
            loss, _ = net.loss_and_grad(p, t, s)
            tot += loss.item()
        return tot / len(sets)
    before = mean_loss(train)
    for it in range(150):
        f, t = train[it % len(train)]
        net.zero_grad()
        acts, p = net.forward(f, shape, s)
        _, dy = net.loss_and_grad(p, t, s)
        net.backward(acts, dy, shape, s)
        net.adam_step(2e-3, s)
    after = mean_loss(train)
    assert after < 0.8 * before, (before, after)
    # a priori gain on held-out snapshots, in tendency space
    errs = []
    for (f, t), (fr, tr) in zip(test, raw[11:]):
        _, p = net.forward(f, shape, s)
        ptrue = closure.pad_targets(tr, torch.ones(12, device="cuda"))
        true_t, _ = closure.tendencies(pc.coarse, ptrue, torch.ones(12, device="cuda"))
        pred_t, _ = closure.tendencies(pc.coarse, p, net.out_scale)
        num = ((pred_t - true_t) ** 2).sum().item()
        den = (true_t ** 2).sum().item()
        errs.append(num / den)
    gain = 1.0 - float(np.mean(errs))
    print("closure a-priori: loss", before, "->", after, "held-out tendency error ratio", errs, "gain", gain)
    assert gain > 0.0, errs
    assert int(net.err.item()) == 0
