"""The learned-closure case a posteriori: fine FP64 runs, box-filtered training
pairs, a network trained on the GPU, and coarse FP32 runs with and without the
closure scored against the filtered fine run's mean profiles.

Pipeline (every arithmetic step in libmhd3d_gpu.so; torch holds device memory):

1. A training fine run (FP64, FMA mode) of the rotating MHD polytrope spins up
   to ``--spin`` (simulated time) and is then sampled ``--samples`` times over
   ``--window``: each sample is box-filtered by ``--fac`` into coarse features
   and the 12 subgrid terms (stress, heat flux, EMF).
2. The three-layer convolutional closure is trained on those pairs by the
   library's forward, backward and Adam kernels.
3. A second fine run of another seed (the held-out run) is spun up the same way; its
   filtered state at the start of the window starts two coarse FP32 runs,
   one plain and one with the closure attached, over the same window.  The
   filtered fine run's horizontal-mean profiles, averaged over the window's
   samples, are the reference for both.
4. Wall time of each run over the window (host clock around synchronous steps,
   sampling excluded) gives the wall-time ratio of the fine run to the coarse
   run with the closure.

With ``--resid-steps N`` the network trained on the filter commutator is
then fine-tuned on the coarse scheme's residual: at each sample the fine run
is advanced N more steps, and R = (B - A)/(tB - tA) - (F(A) + F(B))/2 of the
filtered states A, B and the coarse FP32 right-hand side F is what the
closure tendencies are fitted to (what the coarse method misses in total,
truncation error included, not only the subgrid terms).

Prints one JSON object: per-profile relative L2 errors of the time-averaged
profiles (plain coarse and closure coarse against filtered fine), the closure's
trip count, the a-priori tendency error on the held-out run's last pair, step
counts, DT and wall times.  A coarse run that stops (non-finite values or DT
collapse) reports its status and the simulated time it reached.

Usage: python closure_case.py [--fine 256 256 128] [--fac 4] [--spin 5.0]
       [--window 2.0] [--samples 16] [--iters 3000] [--out FILE]
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import os
import sys
import time

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import mhd3d  # noqa: E402
import closure  # noqa: E402


def _torch():
    import torch
    return torch


def config(nx, ny, nz, args, seed):
    return mhd3d.convection_config(nx, ny, nz, ra=args.ra, ta=args.ta, contrast=args.contrast, ampt=args.ampt,
                                   seed=seed)


def advance_to(sim, t_target, chunk, log=None, tag="", last=None):
    """Step until the simulated time reaches t_target, in chunks of at most
    chunk steps sized from the last DT so that the run stops within a step or
    two of the target.  Returns (steps, wall seconds, last step record); the
    record's status is non-zero when the run stopped (non-finite values or DT
    collapse)."""
    steps, wall = 0, 0.0
    r = last
    while True:
        n = chunk
        if r is not None and r["dt"] > 0:
            n = int(max(1, min(chunk, np.ceil((t_target - r["timt"]) / r["dt"]))))
        t0 = time.perf_counter()
        r = sim.step(n, check=False)
        wall += time.perf_counter() - t0
        steps += n
        if log is not None:
            log(f"{tag} t={r['timt']:.4f} dt={r['dt']:.3e} umach={r['umach']:.3e} steps={steps}")
        if r["status"] or r["timt"] >= t_target:
            return steps, wall, r


TEND_FIELDS = ((0, "fu"), (1, "fv"), (2, "fw"), (3, "ft"), (5, "ww1"), (6, "ww2"), (7, "ww3"))


def residual_target(pc, fine, nsteps):
    """The coarse scheme's residual at the collector's current filtered
    state A: advance the fine run nsteps to B, and return
    R = (B - A) / (tB - tA) - (F(A) + F(B)) / 2 for RU, RV, RW, TT, BX, BY, BZ
    as [7, nz, ny, nx] FP32 on the device, where F is the coarse FP32
    scheme's right-hand side (trapezoidal, so R is second order in tB - tA),
    together with the filtered state A itself (device, as mhd3d_coarsen
    writes it) and the fine run's step record at B."""
    torch = _torch()
    nz, ny, nx = pc.shape
    sh = (nx + 2, ny + 2, nz + 2)
    ta = pc.t_last
    ca = pc.cstate.clone()
    fa = pc.coarse.fluxes()
    t0 = time.perf_counter()
    r = fine.step(nsteps, check=False)
    r["wall"] = time.perf_counter() - t0
    if r["status"]:
        raise mhd3d.Mhd3dError(r["status"], "fine residual steps")
    pc.snapshot(fine, torch.ones(8, dtype=torch.float32, device="cuda"))
    pc.t_last = r["timt"]
    fb = pc.coarse.fluxes()
    a, b = ca.cpu().numpy(), pc.cstate.cpu().numpy()
    dt = r["timt"] - ta
    out = np.zeros((7, nz, ny, nx))
    for o, (fi, fn) in enumerate(TEND_FIELDS):
        if fi >= pc.nf:
            continue
        A = a[fi * pc.NC:(fi + 1) * pc.NC].reshape(sh, order="F")[1:-1, 1:-1, 1:-1]
        B = b[fi * pc.NC:(fi + 1) * pc.NC].reshape(sh, order="F")[1:-1, 1:-1, 1:-1]
        rr = (B - A) / dt - 0.5 * (fa[fn] + fb[fn])[1:-1, 1:-1, 1:-1]
        out[o] = np.transpose(rr, (2, 1, 0))
    out[:, 0] = 0.0
    out[:, -1] = 0.0
    return torch.tensor(out, dtype=torch.float32, device="cuda"), ca, r


def fine_phase(args, seed, collect, log):
    """Spin up a fine run, then sample the window.  Returns the filtered
    coarse state the coarse runs start from (at the window start, or
    ``--settle`` earlier), the sampled pairs (all of them if collect, else the
    last), the time-averaged filtered profiles and the window's cost."""
    torch = _torch()
    fnx, fny, fnz = args.fine
    fac = args.fac
    fs = mhd3d.make_setup(config(fnx, fny, fnz, args, seed))
    cs = mhd3d.make_setup(config(fnx // fac, fny // fac, fnz // fac, args, seed))
    fine = mhd3d.GpuSim(fs, mode=mhd3d.MODE_FAST)
    fine.upload(fs.state)
    pc = closure.PairCollector(fs, cs, fac=fac)
    ones = torch.ones(8, dtype=torch.float32, device="cuda")
    start, t_start = None, None
    if args.settle > 0:
        # the coarse runs start from the filtered state settle earlier and
        # settle before the window: a filtered state is not in balance on the
        # coarse grid, and its adjustment would otherwise fall in the window
        steps, _, r = advance_to(fine, args.spin - args.settle, args.chunk, log, f"fine{seed} spin")
        if r["status"]:
            raise mhd3d.Mhd3dError(r["status"], "fine spin-up")
        pc.snapshot(fine, ones)
        start, t_start = pc.coarse_state(), r["timt"]
        n, _, r = advance_to(fine, args.spin, args.chunk, log, f"fine{seed} spin", last=r)
        steps += n
    else:
        steps, _, r = advance_to(fine, args.spin, args.chunk, log, f"fine{seed} spin")
    if r["status"]:
        raise mhd3d.Mhd3dError(r["status"], "fine spin-up")
    t0 = r["timt"]
    pairs, profs, resid = [], [], []
    pair = pc.snapshot(fine, ones)
    pc.t_last = r["timt"]
    if start is None:
        start, t_start = pc.coarse_state(), t0
    profs.append(pc.coarse.profiles())
    if collect:
        pairs.append(pair)
    wsteps, wwall = 0, 0.0
    if args.resid_steps and collect:
        R, ca, r = residual_target(pc, fine, args.resid_steps)
        resid.append((R, ca))
        wsteps, wwall = args.resid_steps, r["wall"]
    dts, machs = [], []
    for s in range(1, args.samples + 1):
        n, w, r = advance_to(fine, t0 + args.window * s / args.samples, args.chunk, last=r)
        if r["status"]:
            raise mhd3d.Mhd3dError(r["status"], "fine window")
        wsteps += n
        wwall += w
        dts.append(r["dt"])
        machs.append(r["umach"])
        pair = pc.snapshot(fine, ones)
        pc.t_last = t_sample = r["timt"]
        profs.append(pc.coarse.profiles())
        if collect:
            pairs.append(pair)
        if args.resid_steps and (collect or s == args.samples):
            R, ca, r = residual_target(pc, fine, args.resid_steps)
            resid.append((R, ca))
            if collect:   # the held-out run's last target lies past its window
                wsteps += args.resid_steps
                wwall += r["wall"]
        log(f"fine{seed} sample {s} t={r['timt']:.4f} dt={r['dt']:.3e} umach={r['umach']:.3e}")
    if not collect:
        pairs = [pair]   # the last pair: its filtered state is resident in the collector
    fine.close()
    return {"start": start, "pairs": pairs, "resid": resid, "profiles": np.mean(profs, axis=0),
            "profiles_t": np.array(profs), "t0": t0, "t_start": t_start,
            "t1": t_sample,
            "steps": wsteps, "wall": wwall, "spin_steps": steps, "dt_mean": float(np.mean(dts)),
            "umach_max": float(np.max(machs)), "pc": pc, "coarse_setup": cs}


def train(pairs, args, log):
    torch = _torch()
    feats = torch.stack([f for f, _ in pairs]).float()
    tgts = torch.stack([t for _, t in pairs])
    net = closure.ClosureNet(seed=args.net_seed)
    net.in_scale = (1.0 / feats[..., :8].reshape(-1, 8).std(dim=0).clamp_min(1e-12)).contiguous()
    net.out_scale = tgts.reshape(-1, 12).std(dim=0).clamp_min(1e-30).contiguous()
    pad = torch.cat([net.in_scale, torch.ones(8, device="cuda")])
    data = [((f.float()[..., :16] * pad).to(torch.bfloat16), (t / net.out_scale).contiguous()) for f, t in pairs]
    s = torch.cuda.current_stream().cuda_stream
    shape = tuple(pairs[0][0].shape[:3])
    first = None
    t0 = time.perf_counter()
    for it in range(args.iters):
        f, t = data[it % len(data)]
        net.zero_grad()
        acts, p = net.forward(f, shape, s)
        loss, dy = net.loss_and_grad(p, t, s)
        net.backward(acts, dy, shape, s)
        lr = args.lr * 0.5 * (1.0 + np.cos(np.pi * it / args.iters))
        net.adam_step(lr, s)
        if it % 500 == 0 or it == args.iters - 1:
            lv = loss.item()
            first = lv if first is None else first
            log(f"train it={it} loss={lv:.4e} lr={lr:.2e}")
    torch.cuda.synchronize()
    return net, {"iters": args.iters, "pairs": len(pairs), "loss_first": first, "loss_last": loss.item(),
                 "seconds": time.perf_counter() - t0}, data


def train_residual(net, data, resid, pc, args, log):
    """Fine-tune on the coarse scheme's residual: the closure tendencies of
    the network's outputs are fitted to R by the tendency loss (fields
    weighted by 1 / mean R_f^2) and its adjoint."""
    torch = _torch()
    if args.bias:
        # the per-plane bias takes the horizontally uniform part of the
        # residual; the network is fitted to the rest
        resid = [(R - R.mean(dim=(2, 3), keepdim=True), ca) for R, ca in resid]
    msq = torch.stack([(R.double() ** 2).mean(dim=(1, 2, 3)) for R, _ in resid]).mean(dim=0)
    w = (1.0 / msq.clamp_min(1e-300)).float()
    w = (w * 7.0 / w.sum()).contiguous()
    s = torch.cuda.current_stream().cuda_stream
    shape = pc.shape
    net.reset_optimizer()
    t0 = time.perf_counter()
    first = None
    n = min(len(data), len(resid))
    for it in range(args.resid_iters):
        i = it % n
        (f, _), (R, ca) = data[i], resid[i]
        pc.load(ca)
        net.zero_grad()
        acts, p = net.forward(f, shape, s)
        loss, dy = net.tendency_loss_and_grad(pc.coarse, p, R, w, s)
        net.backward(acts, dy, shape, s)
        lr = args.resid_lr * 0.5 * (1.0 + np.cos(np.pi * it / args.resid_iters))
        net.adam_step(lr, s)
        if it % 500 == 0 or it == args.resid_iters - 1:
            lv = loss.item()
            first = lv if first is None else first
            log(f"residual it={it} loss={lv:.4e} lr={lr:.2e}")
    torch.cuda.synchronize()
    return {"iters": args.resid_iters, "pairs": n, "loss_first": first, "loss_last": loss.item(),
            "seconds": time.perf_counter() - t0, "weights": w.cpu().tolist()}, w


def residual_bias(resid):
    """The horizontally uniform part of the coarse scheme's residual, averaged
    over the training pairs: [7, NPZ] float32 on the device (RU, RV, RW, TT,
    BX, BY, BZ; zero on the wall planes, as the targets are).  A box filter
    on a stretched grid does not place the filtered mean profile where the
    coarse grid's own discrete balance has it; this is the steady forcing
    that mismatch leaves."""
    torch = _torch()
    return torch.stack([R.double().mean(dim=(2, 3)) for R, _ in resid]).mean(dim=0).float().contiguous()


def a_priori(net, heldout, log, bias=None):
    """Tendency error ratio |pred - true|^2 / |true|^2 on the held-out run's
    last pair, whose filtered state is resident in the collector's coarse
    handle (no closure gives 1); with a per-plane bias, also the residual
    error ratios of the bias alone and of the network plus the bias."""
    torch = _torch()
    pc = heldout["pc"]
    s = torch.cuda.current_stream().cuda_stream
    pad = torch.cat([net.in_scale, torch.ones(8, device="cuda")])
    ones12 = torch.ones(12, device="cuda")
    f, t = heldout["pairs"][-1]
    if heldout["resid"]:
        pc.load(heldout["resid"][-1][1])   # the pair's own filtered state
    _, p = net.forward((f.float()[..., :16] * pad).to(torch.bfloat16), pc.shape, s)
    true_t, _ = closure.tendencies(pc.coarse, closure.pad_targets(t, ones12), ones12)
    pred_t, _ = closure.tendencies(pc.coarse, p, net.out_scale)
    ratio = ((pred_t - true_t) ** 2).sum().item() / (true_t ** 2).sum().item()
    log(f"a priori tendency error ratio {ratio:.4f}")
    out = {"commutator_error_ratio": ratio}
    if heldout["resid"]:
        # against the coarse scheme's residual at the same state (weighted as in training)
        R, ca = heldout["resid"][-1]
        pc.load(ca)
        _, p = net.forward((f.float()[..., :16] * pad).to(torch.bfloat16), pc.shape, s)
        pred_t, _ = closure.tendencies(pc.coarse, p, net.out_scale)
        true_t, _ = closure.tendencies(pc.coarse, closure.pad_targets(t, ones12), ones12)
        w = heldout.get("resid_w")
        wv = (w if w is not None else torch.ones(7, device="cuda")).view(7, 1, 1, 1)
        den = (wv * R ** 2).sum().item()
        out["residual_error_ratio"] = (wv * (pred_t - R) ** 2).sum().item() / den
        out["commutator_vs_residual_ratio"] = (wv * (true_t - R) ** 2).sum().item() / den
        if bias is not None:
            bv = bias.view(7, -1, 1, 1)
            out["bias_residual_error_ratio"] = (wv * (bv - R) ** 2).sum().item() / den
            out["network_and_bias_residual_error_ratio"] = (wv * (pred_t + bv - R) ** 2).sum().item() / den
        log(f"a priori residual error ratio {out['residual_error_ratio']:.4f} "
            f"(exact commutator: {out['commutator_vs_residual_ratio']:.4f})")
    return out


TERMS = {"stress": range(0, 6), "heat": range(6, 9), "emf": range(9, 12)}


def term_gains(terms):
    """{group: gain} of a terms string: '+'-joined groups, each with an
    optional '@gain'; a group without one takes the next explicit gain to its
    right (so "stress+heat@0.5" scales both), 1 if none follows."""
    toks = terms.split("+")
    out, pending = {}, []
    for tok in toks:
        name, _, g = tok.partition("@")
        if name not in TERMS:
            raise ValueError(f"unknown closure term group {name!r}")
        pending.append(name)
        if g:
            out.update({n: float(g) for n in pending})
            pending = []
    out.update({n: 1.0 for n in pending})
    return out


def gain_grid(spec):
    """Candidate terms strings of a grid "stress+heat:0,0.25;emf:0,0.12": the
    cross product of one gain per ';'-separated set of groups."""
    sets = []
    for part in spec.split(";"):
        groups, _, gains = part.partition(":")
        sets.append((groups.split("+"), gains.split(",")))
    cands = [""]
    for groups, gains in sets:
        cands = [c + ("+" if c else "") + "+".join(f"{g}@{v}" for g in groups) for c in cands for v in gains]
    return cands


def with_bias(cands):
    """Every candidate terms string again with the per-plane bias ("|bias"),
    and the bias alone (every group at gain 0), without repeats."""
    zero = "+".join(f"{g}@0" for g in TERMS)
    return list(dict.fromkeys(cands + [c + "|bias" for c in cands] + [zero + "|bias"]))


def split_bias(terms):
    """(terms without a trailing "|bias", whether it had one)."""
    return (terms[:-len("|bias")], True) if terms.endswith("|bias") else (terms, False)


def bias_alone(terms, has_bias):
    """True when every term group's gain is zero and a bias is applied: the
    network adds nothing, so the coarse run attaches none."""
    gains = term_gains(terms)
    return has_bias and not any(gains.get(name, 0.0) for name in TERMS)


def eddy_factors(spec):
    """Candidate (viscosity, conduction, magnetic diffusivity) factors of
    "1,1.5:1.5:1,2": a bare number scales all three."""
    out = []
    for tok in spec.split(","):
        v = [float(x) for x in tok.split(":")]
        out.append(tuple(v * 3) if len(v) == 1 else tuple(v))
    return out


def eddy_setup(setup, factors):
    """The coarse run's set-up with its diffusion coefficients multiplied by
    (fv, ft, fm): viscosity 1/RE, conduction OCV/REPR and magnetic diffusivity
    1/RM, with RE, REPR and RM (the CFL limits' forms) divided to match.  The
    constant-coefficient eddy-diffusivity part of the closure: the coarse grid
    resolves less of the cascade that drains the resolved scales."""
    fv, ft, fm = factors
    if (fv, ft, fm) == (1.0, 1.0, 1.0):
        return setup
    p = mhd3d.Params.from_buffer_copy(setup.params)
    p.ore *= fv
    p.re /= fv
    p.repr /= ft
    p.orm *= fm
    p.rm /= fm
    return dataclasses.replace(setup, params=p)


def coarse_phase(heldout, net, args, log, tag, terms="stress+heat+emf", eddy=(1.0, 1.0, 1.0), bias=None):
    """A coarse FP32 run from the held-out run's filtered start over the window; with
    net, the closure is attached with only the named term groups applied,
    scaled by the gain after '@' (terms "stress+heat@0.5"), and with bias its
    per-plane bias tendency ([7, NPZ]); eddy multiplies the coarse run's
    diffusion coefficients (eddy_setup)."""
    g = mhd3d.GpuSim(eddy_setup(heldout["coarse_setup"], eddy), mode=mhd3d.MODE_FP32)
    g.upload(heldout["start"])
    terms, use_bias = split_bias(terms)
    if not use_bias:
        bias = None
    bias_only = False
    if net is not None:
        gains = term_gains(terms)
        # with every gain zero the network adds nothing: the bias stands alone
        # and no network is evaluated
        bias_only = bias_alone(terms, bias is not None)
        if not bias_only:
            keep = net.out_scale
            sc = net.out_scale.clone()
            for name, idx in TERMS.items():
                sc[list(idx)] *= gains.get(name, 0.0)
            net.out_scale = sc
            net.attach(g, trip=args.trip)
            net.out_scale = keep
        if bias is not None:
            g.closure_set_bias(bias)
    profs = [g.profiles()]
    steps, wall, dts = 1, 0.0, []
    status, t_end = 0, 0.0
    span = heldout["t1"] - heldout["t0"]
    lead = heldout["t0"] - (heldout.get("t_start") or heldout["t0"])
    t0 = time.perf_counter()
    r = g.step(1, check=False)
    wall += time.perf_counter() - t0
    tbase = r["timt"] - r["dt"]
    if lead > 0 and not r["status"]:
        # settle from the earlier filtered state up to the window (its steps
        # and wall time count); the window's first sample is taken there
        n, w, r = advance_to(g, tbase + lead, args.chunk, last=r)
        steps += n
        wall += w
        tbase += lead
        profs = [g.profiles()]
    if r["status"]:
        status, t_end = r["status"], r["timt"] - tbase
        log(f"{tag} stopped while settling: status {status}")
    for s in range(1, args.samples + 1 if not status else 1):
        n, w, r = advance_to(g, tbase + span * s / args.samples, args.chunk, last=r)
        steps += n
        wall += w
        if r["status"]:
            status, t_end = r["status"], r["timt"] - tbase
            log(f"{tag} stopped: status {status} at t0+{t_end:.4f}")
            break
        dts.append(r["dt"])
        profs.append(g.profiles())
        t_end = r["timt"] - tbase
        log(f"{tag} sample {s} t0+{t_end:.4f} dt={r['dt']:.3e} umach={r['umach']:.3e}")
    out = {"status": status, "t_reached": t_end, "steps": steps, "wall_s": wall,
           "dt_mean": float(np.mean(dts)) if dts else None, "samples": len(profs)}
    if net is not None:
        out["closure"] = dict(g.closure_status(), bias_only=bias_only)
    out["profiles"] = np.mean(profs, axis=0)
    out["profiles_t"] = np.array(profs)
    g.close()
    return out


WINDOW_KEYS = ("t0", "t1", "t_start", "steps", "wall", "spin_steps", "dt_mean", "umach_max")


def save_case(path, net, heldout, tr, apri, val=None, bias=None):
    """The trained network and what the coarse runs are scored on (and, with
    val, the training run's window for choosing a gain)."""
    d = {f"start_{f}": a for f, a in heldout["start"].items() if a is not None}
    if val is not None:
        d.update({f"val_start_{f}": a for f, a in val["start"].items() if a is not None})
        d["val_profiles"] = val["profiles"]
        d["val_meta"] = np.array(json.dumps({k: val[k] for k in WINDOW_KEYS}))
    for li in range(len(closure.LAYERS)):
        d[f"w{li}"] = net.w[li].cpu().numpy()
        d[f"b{li}"] = net.b[li].cpu().numpy()
    d["in_scale"] = net.in_scale.cpu().numpy()
    d["out_scale"] = net.out_scale.cpu().numpy()
    d["profiles"] = heldout["profiles"]
    if bias is not None:
        d["bias"] = bias.cpu().numpy()
    if "profiles_t" in heldout:
        d["profiles_t"] = heldout["profiles_t"]
    d["meta"] = np.array(json.dumps({k: heldout[k] for k in WINDOW_KEYS} | {"train": tr, "a_priori": apri}))
    np.savez(path, **d)


def load_case(path, args):
    torch = _torch()
    z = np.load(path)
    meta = json.loads(str(z["meta"]))
    net = closure.ClosureNet(seed=args.net_seed)
    for li in range(len(closure.LAYERS)):
        net.w[li] = torch.tensor(z[f"w{li}"], device="cuda")
        net.w16[li] = net.w[li].to(torch.bfloat16)
        net.b[li] = torch.tensor(z[f"b{li}"], device="cuda")
    net.in_scale = torch.tensor(z["in_scale"], device="cuda")
    net.out_scale = torch.tensor(z["out_scale"], device="cuda")
    fnx, fny, fnz = args.fine
    cs = mhd3d.make_setup(config(fnx // args.fac, fny // args.fac, fnz // args.fac, args, args.heldout_seed))
    start = {f: (z[f"start_{f}"] if f"start_{f}" in z else None) for f in mhd3d.FIELDS}
    heldout = {k: meta.get(k) for k in WINDOW_KEYS}
    heldout.update({"start": start, "profiles": z["profiles"], "coarse_setup": cs})
    if "profiles_t" in z:
        heldout["profiles_t"] = z["profiles_t"]
    if "bias" in z:
        heldout["bias"] = torch.tensor(z["bias"], device="cuda")
    val = None
    if "val_profiles" in z:
        val = json.loads(str(z["val_meta"]))
        val["start"] = {f: (z[f"val_start_{f}"] if f"val_start_{f}" in z else None) for f in mhd3d.FIELDS}
        val["profiles"] = z["val_profiles"]
        val["coarse_setup"] = mhd3d.make_setup(config(fnx // args.fac, fny // args.fac, fnz // args.fac, args,
                                                      args.train_seed))
    return net, heldout, meta["train"], meta["a_priori"], val


def rel_errors(got, ref):
    return {name: float(np.linalg.norm(got[i] - ref[i]) / max(np.linalg.norm(ref[i]), 1e-300))
            for i, name in enumerate(mhd3d.PROFILES)}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--fine", type=int, nargs=3, default=(256, 256, 128))
    ap.add_argument("--fac", type=int, default=4)
    ap.add_argument("--ra", type=float, default=1e6)
    ap.add_argument("--ta", type=float, default=1e6)
    ap.add_argument("--contrast", type=float, default=10.0)
    ap.add_argument("--ampt", type=float, default=5e-2)
    ap.add_argument("--spin", type=float, default=5.0)
    ap.add_argument("--window", type=float, default=2.0)
    ap.add_argument("--settle", type=float, default=0.0,
                    help="start the coarse runs from the filtered fine state this much simulated time before the "
                         "window (it counts in their steps and wall time); 0: at the window start")
    ap.add_argument("--samples", type=int, default=16)
    ap.add_argument("--chunk", type=int, default=400)
    ap.add_argument("--iters", type=int, default=3000)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--trip", type=float, default=1.0)
    ap.add_argument("--resid-steps", type=int, default=0,
                    help="fine steps between the two filtered states of a residual target; 0: commutator only")
    ap.add_argument("--resid-iters", type=int, default=3000)
    ap.add_argument("--resid-lr", type=float, default=1e-3)
    ap.add_argument("--train-seed", type=int, default=101)
    ap.add_argument("--heldout-seed", type=int, default=202)
    ap.add_argument("--net-seed", type=int, default=7)
    ap.add_argument("--variants", default="stress+heat+emf",
                    help="comma-separated closure runs, each a '+'-joined set of stress, heat, emf")
    ap.add_argument("--gains", default=None,
                    help="comma-separated closure gains tried on the training run's window; the best is scored on the held-out run")
    ap.add_argument("--gain-terms", default="stress+heat+emf")
    ap.add_argument("--gain-grid", default=None,
                    help="per-group gains tried on the training window, e.g. 'stress+heat:0,0.25;emf:0,0.12'")
    ap.add_argument("--eddy", default="1",
                    help="eddy-diffusivity factors tried on the training window with every gain candidate: "
                         "comma-separated, each 'f' or 'fv:ft:fm' (viscosity, conduction, magnetic diffusivity)")
    ap.add_argument("--bias", action="store_true",
                    help="fit the closure's per-plane bias tendency to the training run's horizontal-mean residual "
                         "and the network to the rest; try every gain candidate with and without the bias, and the "
                         "bias alone")
    ap.add_argument("--out", default=None)
    ap.add_argument("--save", default=None, help="write the trained network and the held-out run's window (.npz)")
    ap.add_argument("--load", default=None, help="skip the fine runs and training: read a --save file")
    args = ap.parse_args(argv)

    def log(msg):
        print(msg, file=sys.stderr, flush=True)

    val, bias = None, None
    if args.load:
        net, heldout, tr, apri, val = load_case(args.load, args)
        bias = heldout.pop("bias", None)
    else:
        trainer = fine_phase(args, args.train_seed, True, log)
        net, tr, data = train(trainer["pairs"], args, log)
        val = {k: trainer[k] for k in WINDOW_KEYS + ("start", "profiles", "coarse_setup")}
        w = None
        if args.resid_steps:
            bias = residual_bias(trainer["resid"])
            tr["residual"], w = train_residual(net, data, trainer["resid"], trainer["pc"], args, log)
        del trainer, data
        heldout = fine_phase(args, args.heldout_seed, False, log)
        heldout["resid_w"] = w
        apri = a_priori(net, heldout, log, bias if args.bias else None)
        if args.save:
            save_case(args.save, net, heldout, tr, apri, val, bias)
    chosen, chosen_eddy = None, (1.0, 1.0, 1.0)
    cands = gain_grid(args.gain_grid) if args.gain_grid else (
        [f"{args.gain_terms}@{gv}" for gv in args.gains.split(",")] if args.gains else [])
    if args.bias and bias is not None and cands:
        cands = with_bias(cands)
    eddies = eddy_factors(args.eddy)
    if (cands or len(eddies) > 1) and val is not None:
        # gains and eddy factors are chosen on the training run's own window, never on the held-out run's
        scores = {}
        best = None
        # with several eddy factors the plain coarse run (no network) competes as well
        pool = (cands + [None]) if len(eddies) > 1 else (cands or [None])
        for ed in eddies:
            for cand in pool:
                key = f"{cand}|eddy={':'.join(f'{x:g}' for x in ed)}"
                run = coarse_phase(val, net if cand else None, args, log, f"validate {key}", cand or "", ed, bias)
                err = rel_errors(run["profiles"], val["profiles"])
                sc = float(np.mean([err[n] for n in ("ke", "fconv", "me")])) if run["status"] == 0 else None
                scores[key] = sc
                log(f"{key}: status {run['status']} mean(ke, fconv, me) error {sc}")
                if sc is not None and (best is None or sc < best[0]):
                    best = (sc, cand, ed)
        plain_val = rel_errors(coarse_phase(val, None, args, log, "validate plain")["profiles"], val["profiles"])
        if best is not None:
            chosen, chosen_eddy = best[1], best[2]
        tr["gain_scores"] = scores
        tr["gain_plain_score"] = float(np.mean([plain_val[n] for n in ("ke", "fconv", "me")]))
        tr["gain_chosen"] = chosen
        tr["eddy_chosen"] = list(chosen_eddy)
    runs = [("plain", coarse_phase(heldout, None, args, log, "plain"))]
    variants = args.variants.split(",") if args.variants else []
    for v in variants:
        runs.append(("closure" if v == "stress+heat+emf" else f"closure[{v}]",
                     coarse_phase(heldout, net, args, log, f"closure[{v}]", v)))
    if chosen_eddy != (1.0, 1.0, 1.0):
        tag = f"eddy={':'.join(f'{x:g}' for x in chosen_eddy)}"
        runs.append((f"plain[{tag}]", coarse_phase(heldout, None, args, log, f"plain[{tag}]", "", chosen_eddy)))
        if chosen is not None:
            runs.append((f"closure[{chosen}|{tag}]",
                         coarse_phase(heldout, net, args, log, f"closure[{chosen}|{tag}]", chosen, chosen_eddy,
                                      bias)))
    elif chosen is not None:
        runs.append((f"closure[{chosen}]", coarse_phase(heldout, net, args, log, f"closure[{chosen}]", chosen,
                                                        bias=bias)))
    ref = heldout["profiles"]
    res = {
        "fine": list(args.fine), "fac": args.fac, "ra": args.ra, "ta": args.ta, "contrast": args.contrast,
        "window": [heldout["t0"], heldout["t1"]], "settle": heldout["t0"] - (heldout.get("t_start") or heldout["t0"]),
        "fine_window": {"steps": heldout["steps"], "wall_s": heldout["wall"], "dt_mean": heldout["dt_mean"],
                        "spin_steps": heldout["spin_steps"], "umach_max": heldout["umach_max"]},
        "train": tr, "a_priori": apri,
    }
    ke = mhd3d.PROFILES.index("ke")
    for name, run in runs:
        d = {k: v for k, v in run.items() if not k.startswith("profiles")}
        ref_t = heldout.get("profiles_t")
        if ref_t is not None and len(ref_t) == len(run["profiles_t"]):
            # the run's volume KE over the filtered fine run's, sample by sample
            d["ke_ratio_t"] = [float(a[ke].sum() / max(b[ke].sum(), 1e-300))
                               for a, b in zip(run["profiles_t"], ref_t)]
        d["profile_rel_err"] = rel_errors(run["profiles"], ref)
        d["profile_rel_bias"] = {n: float((run["profiles"][i] - ref[i]).sum() / max(abs(ref[i].sum()), 1e-300))
                                 for i, n in enumerate(mhd3d.PROFILES)}
        if run["wall_s"] > 0 and run["status"] == 0:
            d["wall_ratio_fine_over_coarse"] = heldout["wall"] / run["wall_s"]
        res[name] = d
    line = json.dumps(res)
    print(line)
    if args.out:
        with open(args.out, "w") as f:
            f.write(line + "\n")
    return res


if __name__ == "__main__":
    main()
