"""Ensemble runs as the closure's training data: members of uneven grid sizes
(64x64x48, 96x96x64, 128x128x96, stepped together by the persistent ensemble
kernels) are box-filtered by 4 onto their own coarse grids (16, 24 and 32
wide, so the convolutions run on rows that are not multiples of 128), and one
network is trained on the pairs of all three grid sizes by the library's
forward, backward and Adam kernels.  On snapshots it was not trained on, its
subgrid terms are closer to the filtered runs' than no closure is."""
import numpy as np
import pytest

from test_gpu_parity import _gpu_or_skip

pytestmark = pytest.mark.gpu

GRIDS = [(64, 64, 48), (96, 96, 64), (128, 128, 96)]
PHYS = dict(ra=1e5, ta=1e4, contrast=3.0, ampt=5e-2)
FAC = 4


def test_ensemble_members_train_the_closure(mhd3d):
    _gpu_or_skip(mhd3d)
    torch = pytest.importorskip("torch")
    import closure
    setups = [mhd3d.make_setup(mhd3d.convection_config(*g, seed=11 + i, **PHYS)) for i, g in enumerate(GRIDS)]
    coarse = [mhd3d.make_setup(mhd3d.convection_config(g[0] // FAC, g[1] // FAC, g[2] // FAC, seed=11 + i, **PHYS))
              for i, g in enumerate(GRIDS)]
    ens = mhd3d.Ensemble(setups)
    for m, su in zip(ens.members, setups):
        m.upload(su.state)
    ep = closure.EnsemblePairs(ens, coarse, fac=FAC)
    ones = torch.ones(8, dtype=torch.float32, device="cuda")
    train, held = [], []
    ens.step(300)
    for snap in range(4):
        ens.step(60)
        (held if snap == 3 else train).extend(ep.snapshot(ones))
    r = ens.sync()
    assert (r["status"] == 0).all(), r
    assert {p[2] for p in train} == {(g[2] // FAC, g[1] // FAC, g[0] // FAC) for g in GRIDS}

    net = closure.ClosureNet(seed=4)
    feats = torch.cat([f[..., :8].reshape(-1, 8).float() for f, _, _ in train])
    tgts = torch.cat([t.reshape(-1, 12) for _, t, _ in train])
    net.in_scale = (1.0 / feats.std(dim=0).clamp_min(1e-12)).contiguous()
    net.out_scale = tgts.std(dim=0).clamp_min(1e-30).contiguous()
    pad = torch.cat([net.in_scale, torch.ones(8, device="cuda")])

    def prep(pairs):
        return [((f.float() * pad).to(torch.bfloat16), (t / net.out_scale).contiguous(), sh) for f, t, sh in pairs]

    data, test = prep(train), prep(held)
    s = torch.cuda.current_stream().cuda_stream

    def mse(pairs):
        tot, n = 0.0, 0
        for f, t, sh in pairs:
            _, p = net.forward(f, sh, s)
            tot += ((p[..., :12] - t) ** 2).sum().item()
            n += t.numel()
        return tot / n

    def zero_mse(pairs):
        return sum((t ** 2).sum().item() for _, t, _ in pairs) / sum(t.numel() for _, t, _ in pairs)

    before = mse(data)
    for it in range(600):
        f, t, sh = data[it % len(data)]
        net.zero_grad()
        acts, p = net.forward(f, sh, s)
        _, dy = net.loss_and_grad(p, t, s)
        net.backward(acts, dy, sh, s)
        net.adam_step(2e-3 * 0.5 * (1 + np.cos(np.pi * it / 600)), s)
    torch.cuda.synchronize()
    after = mse(data)
    assert int(net.err.item()) == 0
    assert after < 0.8 * before, (before, after)
    # held-out snapshots of every member: better than no closure
    assert mse(test) < zero_mse(test), (mse(test), zero_mse(test))
    ep.close()
    ens.close()
