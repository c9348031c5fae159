"""Train the learned block preconditioner on the 1M-point workload's scene family and write its parameters.

    python blocklinearsystems.jl_b200/train_gnn.py [--scenes 48] [--steps 600] [--out PATH]

Scenes of 1,000 to 5,000 cameras with 100 points per camera (the 1M-point scene's density, window +-60, camera column
scales over four decades) are generated with their seeds, reduced by the plain mixed Schur path on the device, and the
network is trained on them with the device loss and Adam. The held-out evaluation (four more scenes) compares PCG to
1e-8 with the learned blocks against block-Jacobi. Writes the parameters (float32, .npy) and a JSON summary beside them.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import sys
import time
from pathlib import Path

import numpy as np
import torch

HERE = Path(__file__).resolve().parent


def load_package():
    if "blsgpu" in sys.modules:
        return sys.modules["blsgpu"]
    spec = importlib.util.spec_from_file_location("blsgpu", HERE / "__init__.py", submodule_search_locations=[str(HERE)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["blsgpu"] = mod
    spec.loader.exec_module(mod)
    return mod


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--scenes", type=int, default=48)
    ap.add_argument("--steps", type=int, default=600)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default=str(HERE / "gnn_pcg_params.npy"))
    args = ap.parse_args()
    bls = load_package()
    t0 = time.perf_counter()
    params, losses, systems = bls.gnn.train_on_scenes(args.scenes, steps=args.steps, lr=args.lr, seed=args.seed, log_every=100)
    t_train = time.perf_counter() - t0
    held = []
    for i in range(4):
        nc = 1500 + 1000 * i
        net, S, g = bls.gnn.scene_system(nc, 100 * nc, seed=90_000 + i)
        cmp_ = bls.gnn.pcg_comparison(net, S, g, params)
        cmp_["cameras"] = nc
        held.append(cmp_)
        print(json.dumps(cmp_))
    out = Path(args.out)
    np.save(out, params.cpu().numpy())
    summary = {"scenes": args.scenes, "steps": args.steps, "lr": args.lr, "seed": args.seed, "train_seconds": t_train,
               "loss_first": float(np.mean(losses[:20])), "loss_last": float(np.mean(losses[-20:])), "held_out": held}
    out.with_suffix(".json").write_text(json.dumps(summary, indent=1))
    print(json.dumps({k: v for k, v in summary.items() if k != "held_out"}))


if __name__ == "__main__":
    main()
