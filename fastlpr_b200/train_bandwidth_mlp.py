"""Train the bandwidth-proposal network shipped in ``data/bandwidth_mlp.npz``.

    python -m fastlpr_b200.train_bandwidth_mlp --train 200000 --heldout 4096

Pipeline (all on one GPU):

1. seeded synthetic problems, generated on the device: x ~ U[0,1]^d
   (d = 1 or 2), y = sum of 1-8 sinusoids (plane waves in 2-D) with
   frequencies ~U[0.5, 6] cycles and random phases, plus Gaussian noise with
   sigma ~ logU[0.01, 0.5]; N ~ logU[1e4, 1e6]; order 0/1/2 in 1-D, 0/1 in
   2-D;
2. for each problem the full GCV sweep over the canonical 32 isotropic
   bandwidths (``learned.HGRID``) by this package's own GPU path (grid 1024
   in 1-D, 512^2 in 2-D), and the feature summary of ``learned.summarize``;
3. training with the package's BF16 tensor-core MLP kernels (Adam, MSE on
   the standardised fractional index of the GCV minimum);
4. evaluation on held-out problems: proposal + five-bandwidth refine (the
   window moves toward an edge minimum at most three times, else the full
   sweep runs), scored by the GCV ratio against the full sweep's minimum.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np
import torch

from . import api, learned

GRID_1D = 1024
GRID_2D = [512, 512]


def problem_spec(seed: int) -> dict:
    """Parameters of one seeded training problem (drawn on the host)."""
    rng = np.random.default_rng(seed)
    d = 1 if rng.random() < 0.5 else 2
    order = int(rng.choice([0, 1, 2], p=[0.2, 0.5, 0.3])) if d == 1 else \
        int(rng.choice([0, 1], p=[0.25, 0.75]))
    k = int(rng.integers(1, 9))
    return {
        "d": d, "order": order, "n": int(10 ** rng.uniform(4.0, 6.0)),
        "freq": rng.uniform(0.5, 6.0, k), "phase": rng.uniform(0.0, 2 * np.pi, k),
        "amp": rng.uniform(0.5, 1.5, k) / np.sqrt(k), "theta": rng.uniform(0.0, np.pi, k),
        "sigma": float(10 ** rng.uniform(-2.0, np.log10(0.5))), "seed": seed,
    }


def synthetic_problem(seed: int, device="cuda"):
    """(x (N, d), y (N,), d, order) of one seeded training problem, generated
    on the device (x ~ U[0,1]^d, y = sum of plane-wave sinusoids + noise)."""
    sp = problem_spec(seed)
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    n, d = sp["n"], sp["d"]
    x = torch.rand((n, d), generator=g, dtype=torch.float64, device=device)
    freq = torch.tensor(sp["freq"], device=device)
    phase = torch.tensor(sp["phase"], device=device)
    amp = torch.tensor(sp["amp"], device=device)
    if d == 1:
        proj = x[:, :1]
    else:
        th = torch.tensor(sp["theta"], device=device)
        proj = x[:, :1] * torch.cos(th) + x[:, 1:2] * torch.sin(th)
    y = (amp * torch.sin(2 * np.pi * freq * proj + phase)).sum(dim=1)
    y = y + sp["sigma"] * torch.randn(n, generator=g, dtype=torch.float64, device=device)
    return x.contiguous(), y.contiguous(), d, sp["order"]


def problem_curve(x: torch.Tensor, y: torch.Tensor, d: int, order: int):
    """(features (FEATURE_DIM,), GCV curve over HGRID) by the GPU path."""
    n = int(x.shape[0])
    stats = torch.cat([x.min(dim=0).values, x.max(dim=0).values]).contiguous()
    stream = torch.cuda.current_stream(x.device).cuda_stream
    feats = learned.dataset_features(x, y, stats, n, d, order, stream)
    h = np.column_stack([learned.HGRID] * d)
    opts = {"order": order, "N": GRID_1D if d == 1 else GRID_2D}
    res = api.cv_fastlpr_device(x, y, h, opts)
    return feats, np.asarray(res.gcv_yhat["gcv_m"], dtype=np.float64)


def generate(nprob: int, seed0: int, log_every: int = 5000):
    feats = np.zeros((nprob, learned.FEATURE_DIM), np.float32)
    curves = np.zeros((nprob, len(learned.HGRID)), np.float64)
    meta = np.zeros((nprob, 3), np.int64)  # d, order, n
    t0 = time.time()
    for i in range(nprob):
        x, y, d, order = synthetic_problem(seed0 + i)
        f, g = problem_curve(x, y, d, order)
        feats[i], curves[i], meta[i] = f, g, (d, order, x.shape[0])
        if log_every and (i + 1) % log_every == 0:
            print(f"  generated {i + 1}/{nprob} in {time.time() - t0:.0f} s", flush=True)
    return feats, curves, meta


def targets(curves: np.ndarray) -> np.ndarray:
    return np.array([learned.curve_target(g) for g in curves], np.float64)


def train(feats: np.ndarray, tgt: np.ndarray, epochs: int = 40, batch: int = 1024,
          lr: float = 1e-3, weight_decay: float = 1e-5, seed: int = 0, device="cuda"):
    fmean = feats.mean(axis=0)
    fstd = feats.std(axis=0)
    fstd = np.where(fstd > 1e-8, fstd, 1.0)
    net = learned.BandwidthMLP(device=device, fmean=fmean, fstd=fstd, seed=seed)
    X16 = net._inputs(feats)                       # standardised, BF16, on the device
    T = torch.tensor(((tgt - learned.T_CENTER) / learned.T_SCALE)[:, None], dtype=torch.float32,
                     device=device)
    n = feats.shape[0]
    rng = np.random.default_rng(seed)
    steps = epochs * max(n // batch, 1)
    step = 0
    for ep in range(epochs):
        perm = torch.tensor(rng.permutation(n), device=device)
        tot = torch.zeros(1, device=device)
        nb = 0
        for b0 in range(0, n - batch + 1, batch):
            idx = perm[b0:b0 + batch]
            cur_lr = lr * 0.5 * (1 + np.cos(np.pi * step / steps))
            tot += net.train_step(X16[idx].contiguous(), T[idx].contiguous(), cur_lr,
                                  weight_decay)
            nb += 1
            step += 1
        if ep == 0 or (ep + 1) % 5 == 0 or ep == epochs - 1:
            print(f"  epoch {ep + 1}/{epochs}: mse {float(tot.item()) / max(nb, 1):.4f}",
                  flush=True)
    return net


def search_on_curve(proposal: float, curve: np.ndarray, max_walks: int = 3):
    """The deployed learned search (cv_fastlpr, bandwidth_search='learned')
    replayed on a recorded GCV curve: (GCV of the choice, accepted, number
    of distinct bandwidths evaluated; the full sweep adds all of them)."""
    lh = np.log(learned.HGRID)
    nlist = len(learned.HGRID)
    window = learned.refine_window(proposal, lh)
    seen = set()
    for _ in range(max_walks + 1):
        seen.update(int(i) for i in window)
        gw = curve[window]
        pos = int(np.argmin(gw))
        if learned.accept_window(window, pos, nlist):
            return float(gw[pos]), True, len(seen)
        step = learned.REFINE - 1
        lo = int(window[0]) + (step if pos == len(window) - 1 else -step)
        lo = int(np.clip(lo, 0, nlist - learned.REFINE))
        nxt = np.arange(lo, lo + learned.REFINE)
        if np.array_equal(nxt, window):
            break
        window = nxt
    return float(np.min(curve)), False, len(seen) + nlist


def evaluate(net: learned.BandwidthMLP, feats: np.ndarray, curves: np.ndarray) -> dict:
    """Proposal + five-bandwidth refine (with window walks) against the full sweep."""
    if len(curves) == 0:
        return {"problems": 0}
    prop = net.predict(feats)
    ratio, accepted, first, nev, err = [], [], [], [], []
    for p, g in zip(prop, curves):
        chosen, ok, k = search_on_curve(p, g)
        ratio.append(chosen / np.min(g))
        accepted.append(ok)
        nev.append(k)
        first.append(search_on_curve(p, g, max_walks=0)[1])
        err.append(abs(p - learned.curve_target(g)))
    ratio, accepted = np.asarray(ratio), np.asarray(accepted)
    return {
        "problems": int(len(ratio)),
        "accepted_first_window": float(np.mean(first)),
        "accepted_after_walks": float(accepted.mean()),
        "within_1pct_fraction": float(np.mean(ratio <= 1.01)),
        "max_gcv_ratio": float(ratio.max()),
        "median_abs_index_error": float(np.median(err)),
        "mean_bandwidths_evaluated": float(np.mean(nev)),
    }


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--train", type=int, default=200000)
    ap.add_argument("--heldout", type=int, default=4096)
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--batch", type=int, default=1024)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default=learned.WEIGHTS_PATH)
    ap.add_argument("--summary", default=None, help="write the evaluation summary (JSON) here")
    args = ap.parse_args(argv)
    t0 = time.time()
    print(f"generating {args.train} training curves", flush=True)
    ftr, ctr, mtr = generate(args.train, seed0=1_000_000 + args.seed)
    t_gen = time.time() - t0
    print(f"generating {args.heldout} held-out curves", flush=True)
    fte, cte, mte = generate(args.heldout, seed0=9_000_000 + args.seed)
    t1 = time.time()
    net = train(ftr, targets(ctr), epochs=args.epochs, batch=args.batch, lr=args.lr,
                seed=args.seed)
    torch.cuda.synchronize()
    t_train = time.time() - t1
    summary = {
        "train_problems": args.train, "heldout_problems": args.heldout,
        "epochs": args.epochs, "batch": args.batch,
        "generation_s": round(t_gen, 1), "training_s": round(t_train, 1),
        "train_1d_fraction": float(np.mean(mtr[:, 0] == 1)),
        "heldout": evaluate(net, fte, cte),
        "heldout_2d_order1": evaluate(net, fte[(mte[:, 0] == 2) & (mte[:, 1] == 1)],
                                      cte[(mte[:, 0] == 2) & (mte[:, 1] == 1)]),
        "train_fit": evaluate(net, ftr[:4096], ctr[:4096]),
    }
    net.save(args.out, summary=json.dumps(summary))
    print(json.dumps(summary, indent=1))
    if args.summary:
        with open(args.summary, "w") as fh:
            json.dump(summary, fh, indent=1)


if __name__ == "__main__":
    main()
