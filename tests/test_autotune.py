"""The autotuner (eigeng_b200/autotune.py) and the tuned-options table of
the library (eigen_GPU_batch_tune_set/_get).  CPU: the candidate grid and
the table file.  GPU: a tuning run installs a table whose options the
solves then use, and results are bit for bit those of the automatic
options (the tuned options change speed only)."""
import json
import os

import numpy as np
import pytest


def test_candidate_grid_covers_the_options():
    from eigeng_b200 import autotune as T
    small = T.candidates(32)
    assert {c["ql_mpw"] for c in small} == set(T.QL_MPW)
    assert all(c["split"] == 0 for c in small)
    big = T.candidates(256)
    assert {(c["split"], c["zmem"]) for c in big} >= {(0, 0), (0, 1), (2, 0), (4, 1)}
    assert len(big) == len(T.SPLITS) * len(T.ZMEM) * len(T.QL_MPW)
    assert all(c["split"] <= 2 for c in T.candidates(40) if c["split"])  # at most ceil(n/32) CTAs


def test_reduce_forms_by_order():
    from eigeng_b200 import autotune as T
    import eigeng_b200 as E
    assert T.reduce_forms(32) == [E.REDUCE_AUTO] and T.reduce_forms(1024) == [E.REDUCE_AUTO]
    assert T.reduce_forms(33) == T.reduce_forms(512) == [E.REDUCE_CTA, E.REDUCE_CLUSTER]


def test_table_round_trip(tmp_path):
    from eigeng_b200 import autotune as T
    table = [dict(esize=8, n=128, split=0, zmem=1, ql_mpw=8, ms=1.0, auto_ms=1.2, batch=256)]
    p = os.path.join(tmp_path, "t.json")
    T.save(table, p)
    assert json.load(open(p))["entries"] == table
    assert T.load(p, install=False) == table


@pytest.mark.gpu
def test_tuned_table_is_used_and_results_unchanged(oracle_mod):
    import torch
    import eigeng_b200 as E
    from eigeng_b200 import autotune as T
    table = T.tune([24, 72], torch.float64, batch=512, reps=1)
    E.tune_set(table)
    try:
        got = E.tune_get(8, 72)
        assert got is not None and got["ql_mpw"] == table[1]["ql_mpw"] and got["zmem"] == table[1]["zmem"]
        assert got["reduce"] == table[1]["reduce"] in (E.REDUCE_CTA, E.REDUCE_CLUSTER)
        assert E.tune_get(8, 73) is None
        for n, e in zip((24, 72), table):
            # the speed-only options change no bit: compare with the same
            # phase-1 kernel and the other options automatic
            a0 = oracle_mod.sym_uniform(40, n, seed=n)
            a1 = torch.from_numpy(a0.copy()).cuda()
            w1, i1 = E.solve(a1, n)
            E.tune_set([dict(esize=8, n=n, split=0, zmem=0, ql_mpw=0, reduce=e["reduce"])])
            a2 = torch.from_numpy(a0.copy()).cuda()
            w2, i2 = E.solve(a2, n)
            E.tune_set(table)
            torch.cuda.synchronize()
            assert torch.equal(w1, w2) and torch.equal(a1, a2)
    finally:
        E.tune_set([])
    with pytest.raises(E.EigenGError):
        E.tune_set([dict(esize=8, n=64, split=0, zmem=0, ql_mpw=3)])  # not a power of two
