"""Batched sampling: one launch over walkers of several lattices and couplings (rbmpp_batch_*).

Every context of a batch must end with exactly the walkers, accept counts and stored samples that its own
rbmpp_make_sample (direct sampler, same seeds) produces: the batch only changes which block runs which
walker.  Covered: mixed Pfaffian block sizes in one launch, a block too large for shared memory (18x18,
Gauss-Jordan scratch in global memory), and the autotuner, whose probes must leave the chains unchanged.
"""
import numpy as np
import pytest

from rbm_pp_b200 import capi
from rbm_pp_b200 import formats as fm

pytestmark = pytest.mark.gpu


def _ctx(L, trans, alphar, nw, ns, J2, seed):
    p = fm.synthetic_problem(L, translations=trans, alphar=alphar, nsample=nw * ns, seed=seed, J2=J2)
    g = capi.Context(p, n_walkers=nw, nsample_per_walker=ns)
    g.set_params(p.br, p.Wr, p.slater, 0.0)
    g.seed(1000 + seed)
    return g


SHAPES = [(4, False, 1, 6, 4, 0.5, 1), (6, True, 2, 3, 2, 0.4, 2), (8, False, 2, 5, 2, 0.55, 3),
          (4, True, 1, 4, 3, 0.6, 4)]


def _reference(shapes, monkeypatch):
    monkeypatch.setenv("RBMPP_SAMPLER", "direct")
    out = []
    for sh in shapes:
        g = _ctx(*sh)
        na1 = g.make_sample(True)
        na2 = g.make_sample(False)
        x, psi, pf = g.samples()
        out.append((int(na1.sum()), int(na2.sum()), x, pf))
        g.close()
    monkeypatch.delenv("RBMPP_SAMPLER")
    return out


def _batched(shapes, tune):
    ctxs = [_ctx(*sh) for sh in shapes]
    b = capi.Batch(ctxs)
    info = b.tune() if tune else None
    n1 = b.make_sample(True)
    n2 = b.make_sample(False)
    res = []
    for k, g in enumerate(ctxs):
        x, psi, pf = g.samples()
        res.append((int(n1[k]), int(n2[k]), x, pf))
    b.close()
    for g in ctxs:
        g.close()
    return res, info


@pytest.mark.parametrize("tune", [False, True])
def test_batch_matches_individual_contexts(tune, monkeypatch):
    want = _reference(SHAPES, monkeypatch)
    got, info = _batched(SHAPES, tune)
    if tune:
        threads, order, ms = info
        assert threads in (128, 256, 512) and order in (0, 1, 2) and ms > 0.0
    for (a1, a2, xa, pfa), (b1, b2, xb, pfb) in zip(want, got):
        assert (a1, a2) == (b1, b2)
        assert np.array_equal(xa, xb)
        assert np.abs(pfa - pfb).max() <= 1e-9 * np.abs(pfa).max()


def test_batch_with_block_beyond_shared_memory(monkeypatch):
    """18x18 (N/2 = 162): the direct sampler keeps its Gauss-Jordan tile in global memory."""
    shapes = [(18, False, 2, 2, 1, 0.45, 5), (12, False, 2, 3, 1, 0.5, 6)]
    want = _reference(shapes, monkeypatch)
    got, _ = _batched(shapes, False)
    for (a1, a2, xa, pfa), (b1, b2, xb, pfb) in zip(want, got):
        assert (a1, a2) == (b1, b2)
        assert np.array_equal(xa, xb)


def test_batch_chains_match_oracle_at_large_lattices(capsys):
    """The batched launch at the batching row's lattice sizes against the oracle (make_sample.f90:4-240 in the
    reference's full 2N form): 12x12 and 14x14 contexts (alpha_r = 2, no translations, J2 = 0.45 and 0.55) in one
    launch with chain traces; every walker is exact decision by decision or parts at a documented tie, and the
    stored configurations and the measured energies of exact walkers agree."""
    import chain_compare as cc
    import pyoracle as po
    shapes = [(12, False, 2, 3, 1, 0.45, 7), (14, False, 2, 2, 1, 0.55, 8)]
    ctxs, oracles, probs = [], [], []
    for (L, trans, alphar, nw, ns, J2, seed) in shapes:
        p = fm.synthetic_problem(L, translations=trans, alphar=alphar, nsample=nw * ns, seed=seed, J2=J2)
        g = capi.Context(p, n_walkers=nw, nsample_per_walker=ns)
        o = po.Oracle(p, nranks=nw, nsample_per_rank=ns, nthreads=4)
        for c in (g, o):
            c.set_params(p.br, p.Wr, p.slater, 0.0)
            c.set_trace(20000)
            c.seed(1000 + seed)
        ctxs.append(g)
        oracles.append(o)
        probs.append(p)
    b = capi.Batch(ctxs)
    b.make_sample(True)
    kinds = {}
    for g, o, p in zip(ctxs, oracles, probs):
        o.make_sample(True)
        eo, to = o.events()
        eg, tg = g.events()
        recs = cc.compare_walkers(to, eo, tg, eg)
        xo, xg = o.samples()[0], g.samples()[0]
        for r in recs:
            assert r["kind"] not in ("type", "draw", "length"), r
            if r["kind"] == "checkpoint":
                assert r["straddle"], r
            kinds[r["kind"]] = kinds.get(r["kind"], 0) + 1
            if r["kind"] == "exact":
                assert np.array_equal(xo[r["walker"]], xg[r["walker"]])
    with capsys.disabled():
        print(f"\nBATCH_CHAINS_L12_14 {kinds}")
    assert kinds.get("exact", 0) >= 2
    b.close()
    for g in ctxs:
        g.close()
