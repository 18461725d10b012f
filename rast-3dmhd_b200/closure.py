"""Learned subgrid closure: training pairs from fine runs, training by the
library's own GPU kernels, and attachment to a coarse FP32 run.

The network is three 3x3x3 convolutions (16->32 ReLU, 32->32 ReLU, 32->16),
BF16 weights and activations with FP32 accumulation.  Inputs: the coarse
state's u, v, w, TT-<TT>, RO-<RO>, BX, BY-<BY>, BZ (8 channels, padded to 16),
scaled per channel.  Outputs: the 12 subgrid terms of a box filter by 4 --
stress tau_ij (6), heat flux q_i (3), EMF eps_i (3) -- divided by their scales.

Every arithmetic step runs in the library (libmhd3d_gpu.so): coarsening and
targets (mhd3d_coarsen), features, the tcgen05 convolutions and their input
gradients (mhd3d_conv3d, mhd3d_conv3d_wtranspose), FP32 weight gradients
(mhd3d_conv3d_wgrad), the loss and its gradient (mhd3d_closure_loss), Adam
(mhd3d_adam), the closure tendencies (mhd3d_closure_tendency) and, for
training on tendencies, their loss and adjoint (mhd3d_closure_tendency_loss,
mhd3d_closure_tendency_adjoint).  torch provides device memory and streams.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

import mhd3d

LAYERS = ((16, 32, True), (32, 32, True), (32, 16, False))


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _torch():
    import torch
    return torch


def _check(st, what):
    if st:
        raise mhd3d.Mhd3dError(st, what)


class ClosureNet:
    """FP32 master weights, BF16 copies, Adam state and gradient buffers on the GPU."""

    def __init__(self, seed: int = 0):
        torch = _torch()
        self.lib = mhd3d.gpu_lib()
        rng = np.random.default_rng(seed)
        self.w, self.b, self.w16, self.dw, self.db, self.m, self.v = [], [], [], [], [], [], []
        for li, (cin, cout, _) in enumerate(LAYERS):
            fan_in = 27 * (8 if li == 0 else cin)
            w = rng.standard_normal((cout, 27 * cin)) * np.sqrt(2.0 / fan_in)
            if li == 0:
                w.reshape(cout, 27, cin)[:, :, 8:] = 0.0   # padded input channels
            if li == len(LAYERS) - 1:
                w *= 0.1
                w[12:] = 0.0                               # padded output channels
            wt = torch.tensor(w, dtype=torch.float32, device="cuda")
            bt = torch.zeros(cout, dtype=torch.float32, device="cuda")
            self.w.append(wt)
            self.b.append(bt)
            self.w16.append(wt.to(torch.bfloat16))
            self.dw.append(torch.zeros_like(wt))
            self.db.append(torch.zeros_like(bt))
            self.m.append([torch.zeros_like(wt), torch.zeros_like(bt)])
            self.v.append([torch.zeros_like(wt), torch.zeros_like(bt)])
        self.t = 0
        self.in_scale = torch.ones(8, dtype=torch.float32, device="cuda")
        self.out_scale = torch.ones(12, dtype=torch.float32, device="cuda")
        self.err = torch.zeros(1, dtype=torch.int32, device="cuda")

    # -- passes ---------------------------------------------------------------
    def forward(self, feat, shape, stream):
        torch = _torch()
        nz, ny, nx = shape
        acts = [feat]
        pred = None
        for li, (cin, cout, relu) in enumerate(LAYERS):
            last = li == len(LAYERS) - 1
            y = None if last else torch.empty((nz, ny, nx, cout), dtype=torch.bfloat16, device="cuda")
            yf = torch.empty((nz, ny, nx, cout), dtype=torch.float32, device="cuda") if last else None
            _check(self.lib.mhd3d_conv3d(cin, cout, _p(acts[-1]), _p(self.w16[li]), _p(self.b[li]), None,
                                         1 if relu else 0, _p(y), _p(yf), nx, ny, nz, _p(self.err),
                                         C.c_void_p(stream)), "mhd3d_conv3d")
            if last:
                pred = yf
            else:
                acts.append(y)
        return acts, pred

    def backward(self, acts, dy, shape, stream):
        """Accumulate dW, db of every layer from dy of the last layer's output (BF16)."""
        torch = _torch()
        nz, ny, nx = shape
        for li in range(len(LAYERS) - 1, -1, -1):
            cin, cout, _ = LAYERS[li]
            _check(self.lib.mhd3d_conv3d_wgrad(cin, cout, _p(acts[li]), _p(dy), _p(self.dw[li]), _p(self.db[li]),
                                               nx, ny, nz, C.c_void_p(stream)), "mhd3d_conv3d_wgrad")
            if li == 0:
                break
            wt = torch.empty((cin, 27 * cout), dtype=torch.bfloat16, device="cuda")
            _check(self.lib.mhd3d_conv3d_wtranspose(cin, cout, _p(self.w16[li]), _p(wt), C.c_void_p(stream)),
                   "mhd3d_conv3d_wtranspose")
            dx = torch.empty((nz, ny, nx, cin), dtype=torch.bfloat16, device="cuda")
            # the input of layer li is the ReLU output of layer li-1: its mask
            _check(self.lib.mhd3d_conv3d(cout, cin, _p(dy), _p(wt), None, _p(acts[li]), 0, _p(dx), None, nx, ny, nz,
                                         _p(self.err), C.c_void_p(stream)), "mhd3d_conv3d (input gradient)")
            dy = dx

    def reset_optimizer(self):
        """Zero Adam's moments and step count (before training on a new loss)."""
        for mv in self.m + self.v:
            for t in mv:
                t.zero_()
        self.t = 0

    def zero_grad(self):
        for g in self.dw + self.db:
            g.zero_()

    def adam_step(self, lr, stream, b1=0.9, b2=0.999, eps=1e-8):
        self.t += 1
        for li in range(len(LAYERS)):
            _check(self.lib.mhd3d_adam(_p(self.w[li]), _p(self.dw[li]), _p(self.m[li][0]), _p(self.v[li][0]),
                                       self.w[li].numel(), lr, b1, b2, eps, self.t, _p(self.w16[li]),
                                       C.c_void_p(stream)), "mhd3d_adam")
            _check(self.lib.mhd3d_adam(_p(self.b[li]), _p(self.db[li]), _p(self.m[li][1]), _p(self.v[li][1]),
                                       self.b[li].numel(), lr, b1, b2, eps, self.t, None, C.c_void_p(stream)),
                   "mhd3d_adam")

    def loss_and_grad(self, pred, target, stream):
        torch = _torch()
        nvox = pred.shape[0] * pred.shape[1] * pred.shape[2]
        loss = torch.zeros(1, dtype=torch.float64, device="cuda")
        dy = torch.empty(pred.shape[:3] + (16,), dtype=torch.bfloat16, device="cuda")
        _check(self.lib.mhd3d_closure_loss(_p(pred), _p(target), nvox, _p(dy), _p(loss), C.c_void_p(stream)),
               "mhd3d_closure_loss")
        return loss, dy

    def tendency_loss_and_grad(self, sim, pred, target, weight, stream):
        """Loss of the closure tendencies of pred (for sim's current state)
        against target [7, nz, ny, nx] with per-field weights [7], and its
        gradient with respect to pred as the last layer's dy (BF16)."""
        torch = _torch()
        nz, ny, nx = pred.shape[:3]
        nvox = nz * ny * nx
        tend = torch.empty((7, nz, ny, nx), dtype=torch.float32, device="cuda")
        flag = torch.zeros(1, dtype=torch.int32, device="cuda")
        _check(self.lib.mhd3d_closure_tendency(sim.h, _p(pred), _p(self.out_scale), _p(tend), _p(flag),
                                               C.c_float(1e30), C.c_void_p(stream)), "mhd3d_closure_tendency")
        g = torch.empty_like(tend)
        loss = torch.zeros(1, dtype=torch.float64, device="cuda")
        _check(self.lib.mhd3d_closure_tendency_loss(_p(tend), _p(target), _p(weight), nvox, _p(g), _p(loss),
                                                    C.c_void_p(stream)), "mhd3d_closure_tendency_loss")
        dy = torch.empty((nz, ny, nx, 16), dtype=torch.bfloat16, device="cuda")
        _check(self.lib.mhd3d_closure_tendency_adjoint(sim.h, _p(g), _p(self.out_scale), _p(dy), C.c_void_p(stream)),
               "mhd3d_closure_tendency_adjoint")
        return loss, dy

    def attach(self, sim: mhd3d.GpuSim, trip: float = 1.0):
        st = self.lib.mhd3d_closure_set(sim.h, _p(self.w16[0]), _p(self.b[0]), _p(self.w16[1]), _p(self.b[1]),
                                        _p(self.w16[2]), _p(self.b[2]), _p(self.in_scale), _p(self.out_scale),
                                        C.c_float(trip))
        _check(st, "mhd3d_closure_set")

    def detach(self, sim: mhd3d.GpuSim):
        """Take the network off sim (a per-plane bias, if set, stays)."""
        _check(self.lib.mhd3d_closure_set(sim.h, None, None, None, None, None, None, None, None, C.c_float(0.0)),
               "mhd3d_closure_set")


class PairCollector:
    """Coarse features and subgrid targets from snapshots of a fine run."""

    def __init__(self, fine_setup, coarse_setup, fac: int = 4):
        torch = _torch()
        self.lib = mhd3d.gpu_lib()
        self.fac = fac
        self.coarse = mhd3d.GpuSim(coarse_setup, mode=mhd3d.MODE_FP32)
        cp = coarse_setup.params
        self.shape = (cp.npz, cp.npy, cp.npx)
        self.nf = 8 if cp.lmag else 5
        self.NC = (cp.npx + 2) * (cp.npy + 2) * (cp.npz + 2)
        self.cstate = torch.zeros(self.nf * self.NC, dtype=torch.float64, device="cuda")
        self.means = torch.zeros(3 * cp.npz, dtype=torch.float64, device="cuda")
        self.stream = torch.cuda.current_stream().cuda_stream

    def snapshot(self, fine: mhd3d.GpuSim, in_scale):
        """(features [nz,ny,nx,16] BF16, targets [nz,ny,nx,12] FP32) of fine's current state."""
        torch = _torch()
        nz, ny, nx = self.shape
        tg = torch.empty((nz, ny, nx, 12), dtype=torch.float32, device="cuda")
        _check(self.lib.mhd3d_coarsen(fine.h, self.fac, _p(self.cstate), _p(tg), C.c_void_p(self.stream)),
               "mhd3d_coarsen")
        torch.cuda.synchronize()
        self.load(self.cstate)
        feat = torch.empty((nz, ny, nx, 16), dtype=torch.bfloat16, device="cuda")
        _check(self.lib.mhd3d_closure_features(self.coarse.h, _p(in_scale), _p(feat), _p(self.means),
                                               C.c_void_p(self.stream)), "mhd3d_closure_features")
        torch.cuda.synchronize()
        return feat, tg

    def load(self, cstate):
        """Upload a filtered state (device, as mhd3d_coarsen writes it) into the coarse handle."""
        ptrs = [C.c_void_p(cstate.data_ptr() + 8 * self.NC * i) for i in range(self.nf)]
        ptrs += [None] * (8 - self.nf)
        _check(self.lib.mhd3d_upload(self.coarse.h, *ptrs), "mhd3d_upload")

    def coarse_state(self):
        """The last snapshot's coarse state as Fortran arrays (host)."""
        sh = (self.shape[2] + 2, self.shape[1] + 2, self.shape[0] + 2)
        a = self.cstate.cpu().numpy()
        out = {f: a[i * self.NC:(i + 1) * self.NC].reshape(sh, order="F").copy(order="F") for i, f in
               enumerate(mhd3d.FIELDS[:self.nf])}
        for f in mhd3d.FIELDS[self.nf:]:
            out[f] = None
        return out


class EnsemblePairs:
    """Training pairs from the members of an ensemble (grids of uneven sizes):
    one PairCollector a member, on that member's coarse grid (coarse_setups[i],
    the member's physics at 1/fac resolution)."""

    def __init__(self, ens: mhd3d.Ensemble, coarse_setups, fac: int = 4):
        self.members = ens.members
        self.collectors = [PairCollector(m.setup, cs, fac=fac) for m, cs in zip(ens.members, coarse_setups)]

    def snapshot(self, in_scale):
        """[(features, targets, shape)] of every member's current state."""
        return [pc.snapshot(m, in_scale) + (pc.shape,) for m, pc in zip(self.members, self.collectors)]

    def close(self):
        for pc in self.collectors:
            pc.coarse.close()


def tendencies(sim: mhd3d.GpuSim, pred, out_scale, trip: float = 1e30):
    """Closure tendencies [7, nz, ny, nx] (RU, RV, RW, TT, BX, BY, BZ) of pred for sim's state."""
    torch = _torch()
    lib = mhd3d.gpu_lib()
    nz, ny, nx = pred.shape[:3]
    out = torch.empty((7, nz, ny, nx), dtype=torch.float32, device="cuda")
    flag = torch.zeros(1, dtype=torch.int32, device="cuda")
    _check(lib.mhd3d_closure_tendency(sim.h, _p(pred), _p(out_scale), _p(out), _p(flag), C.c_float(trip),
                                      C.c_void_p(torch.cuda.current_stream().cuda_stream)), "mhd3d_closure_tendency")
    torch.cuda.synchronize()
    return out, int(flag.item())


def pad_targets(tg, out_scale):
    """Normalised targets [.., 12] -> the network's output layout [.., 16]."""
    torch = _torch()
    p = torch.zeros(tg.shape[:3] + (16,), dtype=torch.float32, device="cuda")
    p[..., :12] = tg / out_scale
    return p
