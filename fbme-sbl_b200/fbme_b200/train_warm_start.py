"""Train and evaluate the learned warm start on one GPU.

    python -m fbme_b200.train_warm_start [--scenes 20000] [--epochs 6] [--eval 1024]

1. Training pairs: ``--scenes`` learned-distribution scenes (256x256 grid,
   128x128 prefix, K ~ U{100..400}, SNR ~ U[5, 25] dB, seeds 10^6 ...) solved
   by the plain Stable plan; the target is log(|x|^2 / (P/N) + 1e-3) of its
   polished reconstruction x (``--target`` moment / prior: posterior second
   moment / prior after ``--target-sweeps`` sweeps instead).
2. Training: minibatch Adam with cosine decay on the library's kernels.
3. Evaluation on ``--eval`` held-out seeds (2*10^6 ...): raw NMSE of plain
   FBME-Stable (auto sweep rule), of the plain plan with 1 sweep, and of the
   warm-started plan with 1 and 2 sweeps (with the plain fallback), and the
   fallback counts.
4. Writes the weights (``fbme_b200/weights/warm_start_256x256_128x128.npz``,
   with the evaluation numbers stored beside the parameters) and prints
   one JSON line.
"""

from __future__ import annotations

import argparse
import json
import time

import numpy as np
import torch

from . import scenes
from .engine import FBMEEngine
from .learned import DEFAULT_WEIGHTS, LearnedSBLPlan, WarmStartNet, plain_config, train, training_pairs

GRID, PREFIX = (256, 256), (128, 128)


def _nmse_batch(x_hat: np.ndarray, x_true: np.ndarray) -> np.ndarray:
    num = np.sum(np.abs(x_hat - x_true) ** 2, axis=1)
    den = np.sum(np.abs(x_true) ** 2, axis=1)
    return 10.0 * np.log10(num / den)


def evaluate(net: WarmStartNet, seeds, device, batch: int = 256) -> dict:
    """Raw NMSE on held-out scenes: plain FBME-Stable (auto sweep rule),
    the plain plan with 1 sweep (the warm plan's budget without the
    network) and the warm-started plan with 1 and 2 sweeps (fallback on)."""
    n = GRID[0] * GRID[1]
    plain = FBMEEngine(batch, GRID, PREFIX, plain_config(None), device)
    plain1 = FBMEEngine(batch, GRID, PREFIX, plain_config(1), device)
    example = torch.zeros(batch, *PREFIX, dtype=torch.complex64, device=device)
    warm = {s: LearnedSBLPlan(example, GRID, net=net, sweeps=s, warmup=1) for s in (1, 2)}
    res = {"plain": [], "plain1": [], "warm1": [], "warm2": [], "fallbacks1": 0, "fallbacks2": 0}
    seeds = list(seeds)
    for s0 in range(0, len(seeds), batch):
        chunk = seeds[s0:s0 + batch]
        ys = np.zeros((batch, PREFIX[0] * PREFIX[1]), np.complex64)
        xt = np.zeros((batch, n), np.complex128)
        for i, sd in enumerate(chunk):
            c = scenes.learned_scene(int(sd))
            ys[i] = c.y.reshape(-1)
            xt[i] = c.x.reshape(-1)
        y = torch.from_numpy(ys).to(device)
        for key, eng in (("plain", plain), ("plain1", plain1)):
            eng.run(y)
            xh = eng.result((batch,)).x.reshape(batch, -1).cpu().numpy()
            res[key] += list(_nmse_batch(xh, xt)[: len(chunk)])
        for s, lp in warm.items():
            r = lp.replay(y.view(batch, *PREFIX))
            xw = r.x.reshape(batch, -1).cpu().numpy()
            res[f"warm{s}"] += list(_nmse_batch(xw, xt)[: len(chunk)])
            res[f"fallbacks{s}"] += lp.fallbacks
    plain.close()
    plain1.close()
    out = {k: (float(np.mean(v)) if isinstance(v, list) else v) for k, v in res.items()}
    out["scenes"] = len(seeds)
    return out


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--scenes", type=int, default=20000)
    ap.add_argument("--epochs", type=int, default=6)
    ap.add_argument("--eval", type=int, default=1024)
    ap.add_argument("--target-sweeps", type=int, default=2)
    ap.add_argument("--target", choices=("polish", "moment", "prior"), default="polish")
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--out", default=str(DEFAULT_WEIGHTS))
    a = ap.parse_args()
    device = torch.device("cuda", 0)
    t0 = time.perf_counter()
    bp, tgt = training_pairs(range(1_000_000, 1_000_000 + a.scenes), device, target_sweeps=a.target_sweeps,
                             target=a.target)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    net = WarmStartNet(device, seed=0)
    losses = train(net, bp, tgt, GRID, epochs=a.epochs, batch=a.batch, lr=a.lr)
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    del bp, tgt
    ev = evaluate(net, range(2_000_000, 2_000_000 + a.eval), device)
    t3 = time.perf_counter()
    meta = dict(train_scenes=a.scenes, epochs=a.epochs, target_sweeps=a.target_sweeps, target=a.target, lr=a.lr,
                final_loss=losses[-1], **{f"eval_{k}": v for k, v in ev.items()})
    net.save(a.out, **meta)
    print(json.dumps({"losses": losses[:: max(1, len(losses) // 12)], "final_loss": losses[-1],
                      "pairs_s": t1 - t0, "train_s": t2 - t1, "eval_s": t3 - t2, **ev}), flush=True)


if __name__ == "__main__":
    main()
