"""The trace comparison of tests/chain_compare.py on oracle traces (CPU only).

An oracle chain compared with itself is exact; a copy with one planted change is classified by the kind of
the change: an accept decision flipped inside the ratio gap (tie class 1), a checkpoint decision flipped
across the 1e-5 threshold (tie class 2), or a different candidate pair (a fault).
"""
import numpy as np

import chain_compare as cc
import pyoracle as po
from rbm_pp_b200 import formats as fm


def _trace():
    p = fm.synthetic_problem(4, translations=True, alphar=1, nsample=4 * 8, seed=50)
    o = po.Oracle(p, nranks=4, nsample_per_rank=8, nthreads=2)
    o.set_params(p.br, p.Wr, p.slater, 0.0)
    o.set_trace(4096)
    o.seed(1000)
    o.make_sample(True)
    return o.events()


def test_identical_traces_are_exact():
    ev, tr = _trace()
    assert (ev[:, 4] > 100).all() and (ev[:, 4] <= 4096).all()
    recs = cc.compare_walkers(tr, ev, tr.copy(), ev.copy())
    assert cc.summary(recs) == {"exact": 4}


def test_planted_changes_are_classified():
    ev, tr = _trace()
    t2 = tr.copy()
    # walker 0: flip an accept decision (tie class 1)
    k0 = int(np.nonzero(t2[0, :, 0] == 0)[0][5])
    t2[0, k0, 5] = 1 - t2[0, k0, 5]
    t2[0, k0, 3] = t2[0, k0, 4] * (1 + (1e-12 if t2[0, k0, 5] == 0 else -1e-12))
    # walker 1: flip the first checkpoint decision, with its drift across the threshold (tie class 2)
    k1 = int(np.nonzero(t2[1, :, 0] == 1)[0][0])
    t2[1, k1, 5] = t2[1, k1, 5] + 7
    t2[1, k1, 2] = 2e-5 if tr[1, k1, 2] <= 1e-5 and tr[1, k1, 3] <= 1e-5 else 1e-9
    t2[1, k1, 3] = 1e-9
    # walker 2: another candidate pair (a fault)
    k2 = int(np.nonzero(t2[2, :, 0] == 0)[0][3])
    t2[2, k2, 1] = (t2[2, k2, 1] + 1) % 16
    recs = cc.compare_walkers(tr, ev, t2, ev)
    assert recs[0]["kind"] == "accept" and recs[0]["at"] == k0
    assert recs[0]["gap"] == cc.ratio_gap(tr[0, k0], t2[0, k0])
    assert recs[1]["kind"] == "checkpoint" and recs[1]["at"] == k1 and recs[1]["straddle"]
    assert recs[2]["kind"] == "draw" and recs[2]["at"] == k2
    assert recs[3]["kind"] == "exact"


def test_replay_decisions_follow_the_trace():
    ev, tr = _trace()
    dec = cc.replay_decisions(tr, ev, 32)
    for w in range(4):
        rows = [r for r in tr[w][:ev[w, 4]] if r[0] == 1]
        assert len(rows) == ev[w, 3]
        for k, r in enumerate(rows[:32]):
            assert dec[w, k, 0] == int(r[5]) and dec[w, k, 1] == 0
