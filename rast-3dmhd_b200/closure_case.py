"""The learned-closure case a posteriori: fine FP64 runs, box-filtered training
pairs, a network trained on the GPU, and coarse FP32 runs with and without the
closure judged against the filtered fine run's mean profiles.

Pipeline (every arithmetic step in libmhd3d_gpu.so; torch holds device memory):

1. A training fine run (FP64, FMA mode) of the rotating MHD polytrope spins up
   to ``--spin`` (simulated time) and is then sampled ``--samples`` times over
   ``--window``: each sample is box-filtered by ``--fac`` into coarse features
   and the 12 subgrid terms (stress, heat flux, EMF).
2. The three-layer convolutional closure is trained on those pairs by the
   library's forward, backward and Adam kernels.
3. A second fine run of another seed (the judge) is spun up the same way; its
   filtered state at the start of the window starts two coarse FP32 runs,
   one plain and one with the closure attached, over the same window.  The
   filtered fine run's horizontal-mean profiles, averaged over the window's
   samples, are the reference for both.
4. Wall time of each run over the window (host clock around synchronous steps,
   sampling excluded) gives the wall-time ratio of the fine run to the coarse
   run with the closure.

Prints one JSON object: per-profile relative L2 errors of the time-averaged
profiles (plain coarse and closure coarse against filtered fine), the closure's
trip count, the a-priori tendency error on the judge run's last pair, step
counts, DT and wall times.  A coarse run that stops (non-finite values or DT
collapse) reports its status and the simulated time it reached.

Usage: python closure_case.py [--fine 256 256 128] [--fac 4] [--spin 5.0]
       [--window 2.0] [--samples 16] [--iters 3000] [--out FILE]
"""
from __future__ import annotations

import argparse
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


def fine_phase(args, seed, collect, log):
    """Spin up a fine run, then sample the window.  Returns the filtered
    coarse state at the window start, the sampled pairs (all of them if
    collect, else the last), the time-averaged filtered profiles and the
    window's cost."""
    torch = _torch()
    fnx, fny, fnz = args.fine
    fac = args.fac
    fs = mhd3d.make_setup(config(fnx, fny, fnz, args, seed))
    cs = mhd3d.make_setup(config(fnx // fac, fny // fac, fnz // fac, args, seed))
    fine = mhd3d.GpuSim(fs, mode=mhd3d.MODE_FAST)
    fine.upload(fs.state)
    pc = closure.PairCollector(fs, cs, fac=fac)
    ones = torch.ones(8, dtype=torch.float32, device="cuda")
    steps, _, r = advance_to(fine, args.spin, args.chunk, log, f"fine{seed} spin")
    if r["status"]:
        raise mhd3d.Mhd3dError(r["status"], "fine spin-up")
    t0 = r["timt"]
    pairs, profs = [], []
    pair = pc.snapshot(fine, ones)
    start = pc.coarse_state()
    profs.append(pc.coarse.profiles())
    if collect:
        pairs.append(pair)
    wsteps, wwall, dts, machs = 0, 0.0, [], []
    for s in range(1, args.samples + 1):
        n, w, r = advance_to(fine, t0 + args.window * s / args.samples, args.chunk, last=r)
        if r["status"]:
            raise mhd3d.Mhd3dError(r["status"], "fine window")
        wsteps += n
        wwall += w
        dts.append(r["dt"])
        machs.append(r["umach"])
        pair = pc.snapshot(fine, ones)
        profs.append(pc.coarse.profiles())
        if collect:
            pairs.append(pair)
        log(f"fine{seed} sample {s} t={r['timt']:.4f} dt={r['dt']:.3e} umach={r['umach']:.3e}")
    if not collect:
        pairs = [pair]   # the last pair: its filtered state is resident in the collector
    fine.close()
    return {"start": start, "pairs": pairs, "profiles": np.mean(profs, axis=0), "t0": t0, "t1": r["timt"],
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
                 "seconds": time.perf_counter() - t0}


def a_priori(net, judge, log):
    """Tendency error ratio |pred - true|^2 / |true|^2 on the judge run's
    last pair, whose filtered state is resident in the collector's coarse
    handle (no closure gives 1)."""
    torch = _torch()
    pc = judge["pc"]
    s = torch.cuda.current_stream().cuda_stream
    pad = torch.cat([net.in_scale, torch.ones(8, device="cuda")])
    ones12 = torch.ones(12, device="cuda")
    f, t = judge["pairs"][-1]
    _, p = net.forward((f.float()[..., :16] * pad).to(torch.bfloat16), pc.shape, s)
    true_t, _ = closure.tendencies(pc.coarse, closure.pad_targets(t, ones12), ones12)
    pred_t, _ = closure.tendencies(pc.coarse, p, net.out_scale)
    ratio = ((pred_t - true_t) ** 2).sum().item() / (true_t ** 2).sum().item()
    log(f"a priori tendency error ratio {ratio:.4f}")
    return ratio


TERMS = {"stress": range(0, 6), "heat": range(6, 9), "emf": range(9, 12)}


def coarse_phase(judge, net, args, log, tag, terms="stress+heat+emf"):
    """A coarse FP32 run from the judge's filtered start over the window; with
    net, the closure is attached with only the named term groups applied."""
    g = mhd3d.GpuSim(judge["coarse_setup"], mode=mhd3d.MODE_FP32)
    g.upload(judge["start"])
    if net is not None:
        keep = net.out_scale
        sc = net.out_scale.clone()
        for name, idx in TERMS.items():
            if name not in terms.split("+"):
                sc[list(idx)] = 0.0
        net.out_scale = sc
        net.attach(g, trip=args.trip)
        net.out_scale = keep
    profs = [g.profiles()]
    steps, wall, dts = 1, 0.0, []
    status, t_end = 0, 0.0
    span = judge["t1"] - judge["t0"]
    t0 = time.perf_counter()
    r = g.step(1, check=False)
    wall += time.perf_counter() - t0
    tbase = r["timt"] - r["dt"]
    for s in range(1, args.samples + 1):
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
        out["closure"] = g.closure_status()
    out["profiles"] = np.mean(profs, axis=0)
    g.close()
    return out


def save_case(path, net, judge, tr, apri):
    """The trained network and what the coarse runs are judged on."""
    d = {f"start_{f}": a for f, a in judge["start"].items() if a is not None}
    for li in range(len(closure.LAYERS)):
        d[f"w{li}"] = net.w[li].cpu().numpy()
        d[f"b{li}"] = net.b[li].cpu().numpy()
    d["in_scale"] = net.in_scale.cpu().numpy()
    d["out_scale"] = net.out_scale.cpu().numpy()
    d["profiles"] = judge["profiles"]
    d["meta"] = np.array(json.dumps({k: judge[k] for k in ("t0", "t1", "steps", "wall", "spin_steps", "dt_mean",
                                                            "umach_max")} | {"train": tr, "a_priori": apri}))
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
    cs = mhd3d.make_setup(config(fnx // args.fac, fny // args.fac, fnz // args.fac, args, args.judge_seed))
    start = {f: (z[f"start_{f}"] if f"start_{f}" in z else None) for f in mhd3d.FIELDS}
    judge = {k: meta[k] for k in ("t0", "t1", "steps", "wall", "spin_steps", "dt_mean", "umach_max")}
    judge.update({"start": start, "profiles": z["profiles"], "coarse_setup": cs})
    return net, judge, meta["train"], meta["a_priori"]


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
    ap.add_argument("--samples", type=int, default=16)
    ap.add_argument("--chunk", type=int, default=400)
    ap.add_argument("--iters", type=int, default=3000)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--trip", type=float, default=1.0)
    ap.add_argument("--train-seed", type=int, default=101)
    ap.add_argument("--judge-seed", type=int, default=202)
    ap.add_argument("--net-seed", type=int, default=7)
    ap.add_argument("--variants", default="stress+heat+emf",
                    help="comma-separated closure runs, each a '+'-joined set of stress, heat, emf")
    ap.add_argument("--out", default=None)
    ap.add_argument("--save", default=None, help="write the trained network and the judge run's window (.npz)")
    ap.add_argument("--load", default=None, help="skip the fine runs and training: read a --save file")
    args = ap.parse_args(argv)

    def log(msg):
        print(msg, file=sys.stderr, flush=True)

    if args.load:
        net, judge, tr, apri = load_case(args.load, args)
    else:
        trainer = fine_phase(args, args.train_seed, True, log)
        net, tr = train(trainer["pairs"], args, log)
        del trainer
        judge = fine_phase(args, args.judge_seed, False, log)
        apri = a_priori(net, judge, log)
        if args.save:
            save_case(args.save, net, judge, tr, apri)
    runs = [("plain", coarse_phase(judge, None, args, log, "plain"))]
    for v in args.variants.split(","):
        runs.append(("closure" if v == "stress+heat+emf" else f"closure[{v}]",
                     coarse_phase(judge, net, args, log, f"closure[{v}]", v)))
    ref = judge["profiles"]
    res = {
        "fine": list(args.fine), "fac": args.fac, "ra": args.ra, "ta": args.ta, "contrast": args.contrast,
        "window": [judge["t0"], judge["t1"]],
        "fine_window": {"steps": judge["steps"], "wall_s": judge["wall"], "dt_mean": judge["dt_mean"],
                        "spin_steps": judge["spin_steps"], "umach_max": judge["umach_max"]},
        "train": tr, "a_priori_tendency_error_ratio": apri,
    }
    for name, run in runs:
        d = {k: v for k, v in run.items() if k != "profiles"}
        d["profile_rel_err"] = rel_errors(run["profiles"], ref)
        d["profile_rel_bias"] = {n: float((run["profiles"][i] - ref[i]).sum() / max(abs(ref[i].sum()), 1e-300))
                                 for i, n in enumerate(mhd3d.PROFILES)}
        if run["wall_s"] > 0 and run["status"] == 0:
            d["wall_ratio_fine_over_coarse"] = judge["wall"] / run["wall_s"]
        res[name] = d
    line = json.dumps(res)
    print(line)
    if args.out:
        with open(args.out, "w") as f:
            f.write(line + "\n")
    return res


if __name__ == "__main__":
    main()
