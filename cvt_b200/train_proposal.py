"""Trains the learned plane proposal (cvt_b200/learn.py) at its full recipe and writes the
weights that the library ships (cvt_b200/weights/proposal.npz).

Recipe: 20,000 seeded procedural 512x384 pairs (scenes of 8-60 slanted planes, disparities
2-58 px), targets from plain random-init PatchMatch with both views (disparity range 0-64,
11x11 window, 8 iterations, LR-consistent pixels only), both views of every pair as training
maps (the right view through the mirrored pair), 30 epochs, batch 32, Adam with learning
rate 1e-3 (1e-4 for the last six epochs), L1 loss on disparity and normal.  Training runs on
the GPU through the library's own forward, backward and Adam kernels.

    python -m cvt_b200.train_proposal [--pairs 20000] [--epochs 30] [--batch 32]
        [--out cvt_b200/weights/proposal.npz] [--checkpoint PATH] [--log PATH]
"""
import argparse
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--pairs", type=int, default=20000)
    ap.add_argument("--width", type=int, default=512)
    ap.add_argument("--height", type=int, default=384)
    ap.add_argument("--dmax", type=float, default=64.0)
    ap.add_argument("--patch", type=int, default=5)
    ap.add_argument("--iterations", type=int, default=8)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--data-seed", type=int, default=100000)
    ap.add_argument("--out", default=os.path.join(HERE, "weights", "proposal.npz"))
    ap.add_argument("--checkpoint", default=None, help="also write the full training state (Adam moments) here")
    ap.add_argument("--log", default=None, help="write the training record (JSON) here")
    a = ap.parse_args()

    import torch

    from cvt_b200.learn import PlaneProposal, make_training_set

    torch.cuda.set_device(0)
    t0 = time.perf_counter()
    x, t = make_training_set(a.pairs, a.width, a.height, seed=a.data_seed, dmax=a.dmax, patch=a.patch,
                             iterations=a.iterations, log_every=max(a.pairs // 10, 1))
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    valid = float((t[..., 3] > 0).float().mean().item())
    pp = PlaneProposal(seed=a.seed)
    epoch_loss = []

    def on_epoch(e, net):
        epoch_loss.append(time.perf_counter())

    losses = pp.train(x, t, epochs=a.epochs, batch=a.batch, lr=a.lr, seed=a.seed, on_epoch=on_epoch)
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    ls = losses.cpu().numpy()
    per_epoch = len(ls) // max(a.epochs, 1)
    rec = {"pairs": a.pairs, "maps": int(x.shape[0]), "size": [a.width, a.height], "dmax": a.dmax,
           "target": {"patch_radius": a.patch, "iterations": a.iterations, "views": 2, "arith": "fused",
                      "valid_fraction": valid},
           "epochs": a.epochs, "batch": a.batch, "lr": a.lr, "steps": int(len(ls)), "data_s": round(t1 - t0, 1),
           "train_s": round(t2 - t1, 1), "ms_per_step": round(1e3 * (t2 - t1) / max(len(ls), 1), 3),
           "loss_per_epoch": [float(ls[i * per_epoch:(i + 1) * per_epoch].mean()) for i in range(a.epochs)]}
    os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
    pp.save(a.out, weights_only=True, recipe=json.dumps(rec))
    if a.checkpoint:
        pp.save(a.checkpoint)
    if a.log:
        with open(a.log, "w") as f:
            json.dump(rec, f, indent=1)
    print(json.dumps(rec))


if __name__ == "__main__":
    main()
