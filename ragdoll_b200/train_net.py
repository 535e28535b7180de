"""Trains the learned form's candidate network on the GPU and writes its weights.

    python -m ragdoll_b200.train_net --clips 200 --width 1280 --height 720 --frames 3 --out weights.f32

Training set: the full-search form's decisions (search range --range; --labels learned: the
learned form's own search with every candidate open) on `clips` seeded synthetic clips (gratings,
+-24 px global motion, 12 moving rectangles; one GOP each: an IDR picture and P pictures), QPs cycling through 22 / 26 / 30 / 34 -- every macroblock a sample (its two 24 x 24 luma
windows and its labels). Then `epochs` of Adam over shuffled batches. Prints one JSON line: sample
and label counts, loss per epoch and the time of each phase.
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path


def main(argv=None) -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--clips", type=int, default=200)
    ap.add_argument("--width", type=int, default=1280)
    ap.add_argument("--height", type=int, default=720)
    ap.add_argument("--frames", type=int, default=3)
    ap.add_argument("--range", type=int, default=32)
    ap.add_argument("--epochs", type=int, default=2)
    ap.add_argument("--batch", type=int, default=256)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--labels", default="fullsearch", choices=["fullsearch", "learned"],
                    help="decisions trained on: the full search's, or the learned form's search with every "
                         "candidate open")
    ap.add_argument("--out", required=True)
    args = ap.parse_args(argv)
    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
    import torch

    from ragdoll_b200.learned import CandidateNet, generate_training_set, train

    t0 = time.perf_counter()
    data = generate_training_set(args.clips, args.width, args.height, args.frames, search_range=args.range,
                                 labels=args.labels)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    net = CandidateNet(0, seed=args.seed)
    losses = train(net, data, epochs=args.epochs, batch=args.batch, lr=args.lr,
                   log=lambda m: print(m, file=sys.stderr, flush=True))
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    net.params().tofile(args.out)
    part = data[1].cpu()
    counts = {"samples": int(data[0].shape[0]), "partition_labels": int((part >= 0).sum()),
              "partition_histogram": [int((part == k).sum()) for k in range(4)],
              "intra4x4_block_labels": int((data[2] >= 0).sum()), "offset_labels": int(data[4].sum())}
    print(json.dumps({"train": {"labels": args.labels, "clips": args.clips, "size": f"{args.width}x{args.height}",
                                "frames": args.frames,
                                "search_range": args.range, "epochs": args.epochs, "batch": args.batch, **counts,
                                "loss_per_epoch": [round(x, 5) for x in losses],
                                "label_generation_s": round(t1 - t0, 1), "training_s": round(t2 - t1, 1)}}), flush=True)


if __name__ == "__main__":
    main()
