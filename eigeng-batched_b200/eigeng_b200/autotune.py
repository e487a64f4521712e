"""Autotuner of the solver's launch options (no counterpart in the
reference, whose launch parameters are fixed rules in
eigen_GPU_batch.hpp:23-102).

For each (precision, order n) it times, on this device, a solve of a
representative batch: first under each phase-1 kernel that applies
(reduce: the one-CTA forms or the cluster form, 32 < n <= 512; they differ
in rounding only), then, with the faster one, under every candidate
setting of the options that change speed but not results -- the apply
phase's CTAs per matrix (split), where that phase keeps its rows (zmem:
tensor or shared memory) and the QL phase's matrices per warp (ql_mpw) --
and keeps the fastest.  The table is
written as JSON and installed with eigen_GPU_batch_tune_set, after which
every solve of that (precision, n) whose options are automatic uses it
(including the groups of mixed-size batches).

    python -m eigeng_b200.autotune --sizes 32,64,128,256 --dtype f64 --out tune.json
"""
from __future__ import annotations

import argparse
import itertools
import json

import torch

from . import (REDUCE_AUTO, REDUCE_CLUSTER, REDUCE_CTA, ZMEM_AUTO, ZMEM_SHARED, eigen_GPU_batch_ex, tune_set,
               workspace)

QL_MPW = (0, 1, 2, 4, 8, 16, 32)
SPLITS = (0, 2, 4)
ZMEM = (ZMEM_AUTO, ZMEM_SHARED)


def candidates(n):
    """The settings tried for order n: every combination of the options
    that apply at that size (the apply phase's options only above n = 32)."""
    if n <= 32:
        return [dict(split=0, zmem=ZMEM_AUTO, ql_mpw=q) for q in QL_MPW]
    return [dict(split=s, zmem=z, ql_mpw=q) for s, z, q in itertools.product(SPLITS, ZMEM, QL_MPW)
            if s == 0 or s <= (n + 31) // 32]


def reduce_forms(n):
    """The phase-1 kernels tried for order n."""
    return [REDUCE_CTA, REDUCE_CLUSTER] if 32 < n <= 512 else [REDUCE_AUTO]


def default_batch(n):
    """Batch size that keeps a tuning solve near the throughput regime."""
    return max(256, min(16384, (1 << 24) // (n * n)))


def time_setting(base, n, setting, reps=3, dtype=torch.float64):
    """Median time in ms of `reps` solves of fresh copies of base."""
    L = base.shape[0]
    wk = workspace(L, n, n, dtype, base.device)
    w = torch.empty((L, n), dtype=dtype, device=base.device)
    info = torch.zeros(L, dtype=torch.int32, device=base.device)
    copies = [base.clone() for _ in range(reps + 1)]
    times = []
    for i, a in enumerate(copies):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        st = eigen_GPU_batch_ex(a, w, wk, n, info=info, split=setting["split"], zmem=setting["zmem"],
                                ql_mpw=setting["ql_mpw"])
        e1.record()
        if st != 0:
            return float("inf")
        torch.cuda.synchronize()
        if i > 0:  # the first one warms up
            times.append(e0.elapsed_time(e1))
    times.sort()
    return times[len(times) // 2]


def symmetric_batch(L, n, dtype, seed):
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    b = torch.rand((L, n, n), generator=g, dtype=torch.float64, device="cuda") * 2 - 1
    return (0.5 * (b + b.transpose(1, 2))).to(dtype).contiguous()


def tune(sizes, dtype=torch.float64, batch=None, reps=3, log=None):
    """Returns the table: a list of entries (dicts) for eigen_GPU_batch_tune_set,
    each with the measured times of the automatic and the chosen setting."""
    esize = 8 if dtype == torch.float64 else 4
    table = []
    for n in sizes:
        L = batch or default_batch(n)
        base = symmetric_batch(L, n, dtype, seed=n)
        plain = dict(split=0, zmem=ZMEM_AUTO, ql_mpw=0)
        tune_set([])
        auto_ms = time_setting(base, n, plain, reps, dtype)
        forms = []
        for red in reduce_forms(n):
            tune_set([dict(esize=esize, n=n, reduce=red, **plain)])
            forms.append((time_setting(base, n, plain, reps, dtype), red))
        red = min(forms)[1]
        tune_set([dict(esize=esize, n=n, reduce=red, **plain)])
        results = [(time_setting(base, n, c, reps, dtype), i, c) for i, c in enumerate(candidates(n))]
        tune_set([])
        best = min(results)
        e = dict(esize=esize, n=n, **best[2], reduce=red, ms=best[0], auto_ms=auto_ms, batch=L)
        auto = (auto_ms,)
        table.append(e)
        if log:
            log(f"n={n}: auto {auto[0]:.3f} ms, best {best[0]:.3f} ms with {best[2]}")
        del base
    return table


def save(table, path):
    with open(path, "w") as f:
        json.dump({"entries": table}, f, indent=1)


def load(path, install=True):
    with open(path) as f:
        table = json.load(f)["entries"]
    if install:
        tune_set(table)
    return table


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--sizes", default="32,64,96,128,160,200,256")
    ap.add_argument("--dtype", default="f64", choices=["f64", "f32"])
    ap.add_argument("--batch", type=int, default=0)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--out", default="eigen_tune.json")
    a = ap.parse_args()
    dt = torch.float64 if a.dtype == "f64" else torch.float32
    table = tune([int(x) for x in a.sizes.split(",")], dt, a.batch or None, a.reps, log=print)
    save(table, a.out)
    print("wrote", a.out)


if __name__ == "__main__":
    main()
