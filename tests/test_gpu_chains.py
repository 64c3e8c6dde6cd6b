"""Chain parity of the device samplers with the oracle, decision by decision (make_sample.f90:4-240).

Both sides record every random decision of every walker (tests/chain_compare.py).  A walker is "exact"
when every decision and every drawn number agree.  The only allowed first differences are the two tie
classes: an accept test whose two ratios straddle the drawn u (class 1), and an Nfastup checkpoint whose two
drift measures straddle the 1e-5 threshold of make_sample.f90:120 (class 2).  The oracle carries the
reference's full 2N x 2N inverse with the skew rank-4 update of pfupdate_two.f90:113-224, the device the
N/2 x N/2 block inverse with a rank-2 update, so their drift measures differ: class 2 is the common one.
With the oracle's checkpoint decisions replayed on the device (rbmpp_set_replay) the chains must be
exact apart from class 1.
"""
import json
import os

import numpy as np
import pytest

import chain_compare as cc
import pyoracle as po
from rbm_pp_b200 import capi
from rbm_pp_b200 import formats as fm

pytestmark = pytest.mark.gpu

TRACE = 8192
FAULTS = ("type", "draw", "length")


def _threads():
    return max(1, min(8, os.cpu_count() or 1))


def _pair(L, trans, alphar, nw, ns, pseed, orbital="full", J2=0.5, spin_parity=1):
    p = fm.synthetic_problem(L, translations=trans, alphar=alphar, nsample=nw * ns, seed=pseed, orbital=orbital,
                             J2=J2, spin_parity=spin_parity)
    o = po.Oracle(p, nranks=nw, nsample_per_rank=ns, nthreads=_threads())
    g = capi.Context(p, n_walkers=nw, nsample_per_walker=ns)
    for c in (o, g):
        c.set_params(p.br, p.Wr, p.slater, 0.0)
        c.set_trace(TRACE)
    return p, o, g


def _sample(o, g, first):
    na_o = o.make_sample(first)
    na_g = g.make_sample(first)
    eo, to = o.events()
    eg, tg = g.events()
    recs = cc.compare_walkers(to, eo, tg, eg)
    return dict(na_o=na_o, na_g=na_g, eo=eo, eg=eg, to=to, tg=tg, recs=recs)


def _check_classes(recs):
    """Every walker is exact or parts at a tie.  The acceptance probabilities of the two sides differ by the
    fast-update error of each side's inverse, which the reference itself lets grow up to its recompute
    threshold, so their gap is reported, not bounded; a class-1 tie has u inside that gap by construction."""
    for r in recs:
        assert r["kind"] not in FAULTS, r
        if r["kind"] == "checkpoint":
            assert r["straddle"], r


def _exact_walkers_agree(res, o, g, L):
    """Walkers with identical decisions also agree in everything stored."""
    xo, psio, pfo = o.samples()
    xg, psig, pfg = g.samples()
    exact = [r["walker"] for r in res["recs"] if r["kind"] == "exact"]
    for w in exact:
        assert res["na_o"][w] == res["na_g"][w]
        assert np.array_equal(res["eo"][w], res["eg"][w])
        assert np.array_equal(xo[w], xg[w])
        assert o.nfastup()[w] == g.nfastup()[w]
    # stored amplitudes of every walker against a scratch evaluation of its configurations (1e-6: the
    # reference's own drift bound on fast-update products, make_sample.f90:120)
    scratch = g.eval_configs(xg.reshape(-1, L * L), want_h=False)["psi"]
    st = psig.reshape(-1, psig.shape[-1])
    assert float(np.abs(st[:, 0] - scratch[:, 0]).max() / np.abs(scratch[:, 0]).max()) < 1e-6
    return exact


def test_events_fire_and_match():
    """A global spin flip (make_sample.f90:135-158, p = 3e-4 per proposal) and a make_initial_x re-seed of a
    continued chain (:61, p = 0.05 per call) provably fire, with identical decisions on both sides."""
    L, nw, ns = 4, 16, 16
    p, o, g = _pair(L, True, 1, nw, ns, pseed=50)
    o.seed(1000)
    g.seed(1000)
    fired = np.zeros(5, dtype=np.int64)
    for first in (True, False):
        res = _sample(o, g, first)
        _check_classes(res["recs"])
        assert cc.summary(res["recs"]) == {"exact": nw}, cc.summary(res["recs"])
        assert np.array_equal(res["eo"], res["eg"])
        assert np.array_equal(res["na_o"], res["na_g"])
        _exact_walkers_agree(res, o, g, L)
        fired += res["eg"].sum(axis=0)
    assert fired[0] > 0 and fired[1] > 0, fired  # flips tried and accepted
    assert fired[2] > 0, fired  # re-seeds
    assert fired[3] > 0, fired  # checkpoints
    g.close()


@pytest.mark.parametrize("L,trans,alphar,nw,ns,kw", [
    (4, True, 1, 8, 8, dict(spin_parity=-1)),
    (6, False, 2, 6, 8, dict(orbital="sublattice2")),
    (6, True, 1, 4, 4, dict(J2=0.4)),
    (4, False, 2, 8, 8, dict(J2=0.6)),
])
def test_edge_case_chains(L, trans, alphar, nw, ns, kw):
    """spin_parity = -1 (spin_projection.f90:56-62), the 2-sublattice orbital map, J2 = 0.4 and 0.6."""
    p, o, g = _pair(L, trans, alphar, nw, ns, pseed=70 + L, **kw)
    o.seed(31)
    g.seed(31)
    res = _sample(o, g, True)
    _check_classes(res["recs"])
    exact = _exact_walkers_agree(res, o, g, L)
    assert len(exact) >= nw // 2, cc.summary(res["recs"])
    g.close()


def test_divergence_classes_over_seeds(capsys):
    """64 problem/stream seeds x 8 walkers of the 4x4 translation-symmetric problem: every walker is exact or
    parts at a tie; the rate of each class is reported."""
    L, nw, ns = 4, 8, 8
    tally = {}
    gaps = []
    for seed in range(64):
        p, o, g = _pair(L, True, 1, nw, ns, pseed=300 + seed)
        o.seed(5000 + seed)
        g.seed(5000 + seed)
        res = _sample(o, g, True)
        _check_classes(res["recs"])
        _exact_walkers_agree(res, o, g, L)
        for r in res["recs"]:
            tally[r["kind"]] = tally.get(r["kind"], 0) + 1
            gaps.append(r["max_ratio_gap"])
        g.close()
    total = sum(tally.values())
    with capsys.disabled():
        print("\nCHAIN_CLASSES_4x4 " + json.dumps(dict(walkers=total, classes=tally,
                                                       max_accept_prob_gap=float(max(gaps)),
                                                       median_accept_prob_gap=float(np.median(gaps)))))
    assert total == 64 * nw


def test_make_sample_10x10_translations(capsys):
    """The benched shape: 10x10, 100 translations (200 Pfaffian blocks of 50 x 50), alpha_r = 4, the
    compile-time 50-block sampler.  Natural run (both sides decide their own checkpoints), then the
    oracle's decisions replayed on the device: the replayed chains are exact apart from class-1 ties."""
    L, nw, ns = 10, _threads(), 1
    p, o, g = _pair(L, True, 4, nw, ns, pseed=5)
    o.seed(777)
    g.seed(777)
    res = _sample(o, g, True)
    _check_classes(res["recs"])
    natural = cc.summary(res["recs"])
    exact = _exact_walkers_agree(res, o, g, L)
    # every walker agrees decision by decision at least up to its first checkpoint
    for r in res["recs"]:
        if r["kind"] != "exact":
            assert r["at"] > 100, r
    # replay the oracle's recompute schedule on a fresh device context (same problem, same streams)
    g2 = capi.Context(p, n_walkers=nw, nsample_per_walker=ns)
    g2.set_params(p.br, p.Wr, p.slater, 0.0)
    g2.set_trace(TRACE)
    g2.set_replay(cc.replay_decisions(res["to"], res["eo"], 64))
    g2.seed(777)
    na2 = g2.make_sample(True)
    eg2, tg2 = g2.events()
    recs2 = cc.compare_walkers(res["to"], res["eo"], tg2, eg2)
    _check_classes(recs2)
    replay = cc.summary(recs2)
    xo = o.samples()[0]
    xg2 = g2.samples()[0]
    for r in recs2:
        assert r["kind"] in ("exact", "accept"), r
        if r["kind"] == "exact":
            w = r["walker"]
            assert np.array_equal(xo[w], xg2[w]) and res["na_o"][w] == na2[w]
    with capsys.disabled():
        print("\nCHAIN_CLASSES_10x10 " + json.dumps(dict(walkers=nw, natural=natural, replayed=replay,
                                                         exact_natural=len(exact),
                                                         natural_detail=res["recs"], replay_detail=recs2),
                                                    default=float))
    assert replay.get("exact", 0) >= nw - 1, replay
    g.close()
    g2.close()
