"""Learned per-row Jacobi damping: training data from the solver itself,
training with the library's own MLP kernels, evaluation against fixed
damping.

    python -m thermofem_b200.learned train [--problems 200] [--out PATH]
    python -m thermofem_b200.learned evaluate [--size 256] [--model PATH]

Training data: for each training problem (3-D 7-point log-normal heat, side
uniform in [32, 64], seeds 5000..), for each level operator A_d of its AMG
hierarchy and each candidate damping w, the solver measures how much its
own cycle (the same aggregation hierarchy built on A_d, F-cycle) reduces the
error of each row: e <- e - M_w^{-1} A_d e from random e, twice, |e_i|
summed over a few vectors.  A row's target is the candidate with the
smallest remaining error.  Rows are subsampled per level.  The network
(tf_mlp) regresses the target from the row's features with minibatch
momentum SGD on the GPU (tf_mlp_backward / tf_mlp_sgd).
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np
import torch

from . import api as tf
from . import problems as P

CANDIDATES = (0.5, 0.6, 0.7, 0.8, 0.9, 1.0)
MODEL_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "damping_model.json")
AMG_BASE = dict(pre_sweeps=1, post_sweeps=1, coarse_rows=64, hierarchy_type="f64")


def level_operators(a: tf.DeviceCsr, ctx, cycle="f"):
    """The operators of a's AMG hierarchy (the last one is dropped when the
    coarse LU solves it exactly: no smoothing happens there)."""
    amg = tf.Amg(tf.amg_options(cycle=cycle, **AMG_BASE), ctx=ctx)
    amg.setup(a)
    ops = [amg.level_matrix(d) for d in range(amg.level_count())]
    if amg.coarse_solver() == "pivoted GPU LU" and len(ops) > 1:
        ops = ops[:-1]
    return ops


def row_targets(a: tf.DeviceCsr, ctx, seed: int, vectors: int = 4, sweeps: int = 2, cycle="f"):
    """Per-row best candidate damping of a's own cycle (see module doc)."""
    n = a.rows
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    e0 = [torch.rand(n, dtype=torch.float64, device="cuda", generator=gen) * 2 - 1 for _ in range(vectors)]
    remaining = []
    for w in CANDIDATES:
        amg = tf.Amg(tf.amg_options(jacobi_weight=w, cycle=cycle, **AMG_BASE), ctx=ctx)
        amg.setup(a)
        acc = torch.zeros(n, dtype=torch.float64, device="cuda")
        for e in e0:
            e = e.clone()
            for _ in range(sweeps):
                e = e - amg.apply(tf.spmv(a, e, ctx=ctx))
            acc += e.abs()
        remaining.append(acc)
        del amg
    best = torch.stack(remaining).argmin(dim=0)
    return torch.tensor(CANDIDATES, dtype=torch.float32, device="cuda")[best]


def training_set(count=200, side_min=32, side_max=64, seed=5000, rows_per_level=2048, ctx=None, log=None):
    """Features and targets (device tensors) from `count` training problems."""
    ctx = ctx or tf.default_context()
    feats, targs = [], []
    for k in range(count):
        u = P.uniform(seed + k, 1, 11)[0]
        m = side_min + min(int(u * (side_max - side_min + 1)), side_max - side_min)
        off, idx, val = P.heat3d(m, seed + k)
        a = tf.DeviceCsr.from_host(off, idx, val)
        for d, op in enumerate(level_operators(a, ctx)):
            f = tf.row_features(op, d, ctx=ctx)
            t = row_targets(op, ctx, seed=(seed + k) * 64 + d)
            g = torch.Generator(device="cuda")
            g.manual_seed((seed + k) * 64 + d)
            pick = torch.randperm(op.rows, device="cuda", generator=g)[:rows_per_level]
            feats.append(f[pick])
            targs.append(t[pick])
        if log:
            log(f"problem {k}: side {m}")
    return torch.cat(feats), torch.cat(targs)


def train(features, targets, epochs=40, batch=32768, lr=0.5, momentum=0.9, seed=1, ctx=None, log=None):
    """Minibatch momentum SGD with the library's kernels; returns the model."""
    ctx = ctx or tf.default_context()
    model = tf.Mlp(seed=seed, ctx=ctx)
    n = features.shape[0]
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    history = []
    for ep in range(epochs):
        perm = torch.randperm(n, device="cuda", generator=g)
        total = 0.0
        for s in range(0, n, batch):
            idx = perm[s:s + batch]
            x, t = features[idx].contiguous(), targets[idx].contiguous()
            total += model.backward(x, t) * x.shape[0]
            model.sgd(lr, momentum)
        history.append(total / n)
        if log:
            log(f"epoch {ep}: mse {history[-1]:.5f}")
    return model, history


def save(model: tf.Mlp, path=MODEL_PATH, meta=None):
    with open(path, "w") as f:
        json.dump({"omega_min": model.omega_min, "omega_max": model.omega_max,
                   "params": [float(v) for v in model.params()], "meta": meta or {}}, f, indent=1)


def load(path=MODEL_PATH, ctx=None) -> tf.Mlp:
    with open(path) as f:
        d = json.load(f)
    return tf.Mlp(omega_min=d["omega_min"], omega_max=d["omega_max"], ctx=ctx, params=np.array(d["params"]))


def evaluate(model: tf.Mlp, m=256, seed=9000, ctx=None, cycle="f"):
    """Held-out problem: PCG and BiCGStab with the cycle under fixed
    w = 2/3 and under the model; iterations, device time, true residual."""
    ctx = ctx or tf.default_context()
    off, idx, val = P.heat3d(m, seed)
    n = len(off) - 1
    a = tf.DeviceCsr.from_host(off, idx, val)
    b = torch.tensor(P.rhs_uniform(n, seed + 1), device="cuda")
    out = {}
    for kind, cls in (("pcg", tf.Cg), ("bicgstab", tf.BiCgStab)):
        for name, opts in (("fixed_2_3", dict(jacobi_weight=2 / 3)), ("learned", dict(damping_model=model))):
            s = cls(tf.solver_options(), "amg", tf.amg_options(cycle=cycle, hierarchy_type="f32", **opts), ctx=ctx)
            s.setup(a)
            x = torch.zeros(n, dtype=torch.float64, device="cuda")
            s.apply(b, x)  # warm-up (graph build)
            x.zero_()
            rep = s.apply(b, x)
            r = tf.residual(a, b, x, ctx=ctx)
            out[f"{kind}_{name}"] = {"iterations": rep["iterations"], "status": rep["status"],
                                     "ms": s.last_apply_ms,
                                     "true_relative_residual": float(torch.linalg.norm(r) / torch.linalg.norm(b))}
            del s
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("what", choices=["train", "evaluate"])
    ap.add_argument("--problems", type=int, default=200)
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--size", type=int, default=256)
    ap.add_argument("--model", default=MODEL_PATH)
    ap.add_argument("--out", default=MODEL_PATH)
    a = ap.parse_args()
    ctx = tf.Context(0)
    if a.what == "train":
        t0 = time.perf_counter()
        x, y = training_set(a.problems, ctx=ctx, log=print)
        t1 = time.perf_counter()
        model, hist = train(x, y, epochs=a.epochs, ctx=ctx, log=print)
        labels = {f"{w:.1f}": int((y == torch.tensor(w, dtype=torch.float32, device=y.device)).sum())
                  for w in CANDIDATES}
        save(model, a.out, {"problems": a.problems, "samples": int(x.shape[0]), "epochs": a.epochs,
                            "mse_first": hist[0], "mse_last": hist[-1], "target_counts": labels,
                            "data_s": t1 - t0, "train_s": time.perf_counter() - t1})
        print(json.dumps({"samples": int(x.shape[0]), "mse": [hist[0], hist[-1]], "targets": labels}))
    else:
        print(json.dumps(evaluate(load(a.model, ctx), a.size, ctx=ctx)))


if __name__ == "__main__":
    main()
