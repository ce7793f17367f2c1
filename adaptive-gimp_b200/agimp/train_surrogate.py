"""Train the snow return-map surrogate from plain runs and save it.

    python -m agimp.train_surrogate [--pairs 50000000] [--steps 3000] [--out PATH]

Records (trial state features, exactly projected state) pairs from plain
(SVD return map) runs of the 2D and 3D dynamic snow scenes, trains the MLP on
the GPU with the tensor-core forward/backward kernels, and writes the
parameters and the trained input range to an .npz file.
"""
from __future__ import annotations

import argparse
import json
import os
import time

DEFAULT_OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "surrogate_snow.npz")


def main(argv=None):
    import torch

    from . import scenes
    from .surrogate import MLP, evaluate, record_pairs, save, train, trained_range
    ap = argparse.ArgumentParser()
    ap.add_argument("--pairs", type=int, default=50_000_000)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--batch", type=int, default=65536)
    ap.add_argument("--out", default=DEFAULT_OUT)
    ap.add_argument("--seed", type=int, default=0)
    a = ap.parse_args(argv)
    t0 = time.time()
    half = a.pairs // 2
    Xs, Ts = [], []
    for k, cap in ((3, half), (2, a.pairs - half)):
        sc = scenes.make_config(k, seed=a.seed)
        X, T = record_pairs(sc, cap, stride=1, max_substeps=2000)
        Xs.append(X)
        Ts.append(T)
    X, T = torch.cat(Xs), torch.cat(Ts)
    n = X.shape[0]
    perm = torch.randperm(n, device=X.device)
    nval = max(n // 50, 1)
    Xv, Tv = X[perm[:nval]].contiguous(), T[perm[:nval]].contiguous()
    Xt, Tt = X[perm[nval:]].contiguous(), T[perm[nval:]].contiguous()
    t1 = time.time()
    mlp = MLP(seed=a.seed)
    hist = train(mlp, Xt, Tt, steps=a.steps, batch=a.batch, log_every=max(a.steps // 10, 1))
    t2 = time.time()
    mse, mx = evaluate(mlp, Xv, Tv)
    xmax = trained_range(Xt)
    os.makedirs(os.path.dirname(a.out), exist_ok=True)
    save(a.out, mlp, xmax, dict(val_mse=mse, val_max=mx, pairs=n))
    print(json.dumps(dict(pairs=n, record_s=t1 - t0, train_s=t2 - t1, val_mse=mse, val_max_abs=mx,
                          xmax=[float(v) for v in xmax], loss=hist)))


if __name__ == "__main__":
    main()
