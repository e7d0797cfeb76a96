"""Train the default learned con2prim seed and write cueva/data/c2p_seed.npz.

Training set (10 M pairs): snapshots of the 128x256 HLL/SSP2 and the
1024x2048 HLLC/SSP3 Kelvin-Helmholtz runs (every state of several time
levels) plus synthetic states from the seeded generator (seed 1234) for the
rest.  Training: minibatch Adam on the GPU (the library's kernels), batch
4096, cosine-decayed learning rate.

    python -m cueva.train_seed [--steps 20000] [--out path]
"""
import argparse
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT = os.path.join(HERE, "data", "c2p_seed.npz")


def kh_snapshots(cfg, levels, every):
    import torch
    from . import Cueva
    from .learned import snapshot_pairs
    g = Cueva(**cfg.solver_kwargs())
    g.kh_init(**cfg.kh_kwargs())
    g.upload()
    cons, prims = [], []
    for _ in range(levels):
        g.step(every)
        c, p = snapshot_pairs(g)
        cons.append(c)
        prims.append(p)
    g.close()
    return torch.cat(cons, 1), torch.cat(prims, 1)


def train_default(steps=20000, total=10_000_000, out=DEFAULT, seed=1234, log=print):
    import torch
    from .configs import C1, C2
    from .learned import LearnedSeed, synthetic_pairs
    t0 = time.time()
    c1 = kh_snapshots(C1, levels=10, every=20)
    c2 = kh_snapshots(C2, levels=2, every=5)
    nsyn = total - c1[0].shape[1] - c2[0].shape[1]
    syn = synthetic_pairs(nsyn, seed=seed)
    cons = torch.cat([c1[0], c2[0], syn[0]], 1).contiguous()
    prims = torch.cat([c1[1], c2[1], syn[1]], 1).contiguous()
    log(f"training set: {cons.shape[1]} pairs ({c1[0].shape[1]} + {c2[0].shape[1]} KH snapshot states)")
    net = LearnedSeed(seed=seed)
    net.fit_normalisation(cons, prims)
    loss0 = net.train(cons, prims, steps=10, batch=4096, lr=2e-3, seed=seed + 1)
    loss = net.train(cons, prims, steps=steps, batch=4096, lr=2e-3, seed=seed + 2)
    log(f"loss {loss0:.3e} -> {loss:.3e} after {steps} steps ({time.time() - t0:.1f} s)")
    os.makedirs(os.path.dirname(out), exist_ok=True)
    params = net.params()
    np.savez(out, params=params, loss=np.float32(loss), steps=np.int64(steps), pairs=np.int64(cons.shape[1]))
    return net


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--pairs", type=int, default=10_000_000)
    ap.add_argument("--out", default=DEFAULT)
    a = ap.parse_args()
    train_default(a.steps, a.pairs, a.out).close()


if __name__ == "__main__":
    main()
