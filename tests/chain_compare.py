"""Decision-by-decision comparison of two chain traces (the oracle's and the library's).

A trace lists a walker's random decisions in draw order (the record layout of rbmpp_get_walker_events):
  {0, i1, i2, ratio^2, u, accepted}  exchange proposal        (make_sample.f90:160-220)
  {1, i0, inverse drift, Pf drift, Nfastup before, after}     checkpoint (:74-128)
  {2, 0, 0, ratio^2, u, accepted}    global spin flip          (:135-158)
  {3, 0, 0, 0, 0, 0}                 make_initial_x re-seed    (:61)

Two correct implementations draw the same numbers and take the same decisions until one of two ties:
  tie class 1 ("accept"): an accept test u < ratio^2 whose two ratios, computed by different formulae, lie
      on either side of u;
  tie class 2 ("checkpoint"): an Nfastup checkpoint whose two drift measures lie on either side of the
      reference's 1e-5 recompute threshold (make_sample.f90:120).
After either, the streams part for good.  Any other first difference (another candidate pair or draw, a
record of another type) is a fault.
"""
from __future__ import annotations

import numpy as np

THRESH = 1.0e-5  # make_sample.f90:120


def first_divergence(ta, na, tb, nb):
    """(index, kind) of the first differing decision of traces ta, tb (records kept: min(n, len)); None when
    they agree over the kept length and the two chains produced the same number of records."""
    n = min(na, nb, len(ta), len(tb))
    for k in range(n):
        a, b = ta[k], tb[k]
        if a[0] != b[0]:
            return k, "type"
        t = int(a[0])
        if t == 0:
            if a[1] != b[1] or a[2] != b[2] or a[4] != b[4]:
                return k, "draw"
            if a[5] != b[5]:
                return k, "accept"
        elif t == 1:
            if a[1] != b[1] or a[4] != b[4]:
                return k, "draw"
            extra_a = a[2] > 10.0 and a[3] > 10.0
            extra_b = b[2] > 10.0 and b[3] > 10.0
            if a[5] != b[5] or extra_a != extra_b:
                return k, "checkpoint"
        elif t == 2:
            if a[4] != b[4]:
                return k, "draw"
            if a[5] != b[5]:
                return k, "accept"
    if na != nb and n == min(na, nb) and n < min(len(ta), len(tb)):
        return n, "length"
    return None


def ratio_gap(a, b):
    """Difference of the two acceptance probabilities min(1, ratio^2) of an accept record pair: the width of
    the interval of u for which the two accept decisions would differ."""
    return abs(min(1.0, a[3]) - min(1.0, b[3]))


def compare_walkers(tr_o, ev_o, tr_g, ev_g):
    """Classify every walker: 'exact', 'accept' (tie class 1), 'checkpoint' (tie class 2) or a fault kind.
    Returns a list of dicts with the divergence index, the kind and the evidence."""
    out = []
    for w in range(tr_o.shape[0]):
        no, ng = int(ev_o[w, 4]), int(ev_g[w, 4])
        d = first_divergence(tr_o[w], no, tr_g[w], ng)
        n_kept = min(no, ng, tr_o.shape[1])
        gaps = [ratio_gap(tr_o[w][k], tr_g[w][k]) for k in range(n_kept if d is None else d[0])
                if tr_o[w][k][0] in (0, 2)]
        rec = dict(walker=w, records=n_kept, max_ratio_gap=max(gaps) if gaps else 0.0)
        if d is None:
            rec["kind"] = "exact"
        else:
            k, kind = d
            rec.update(kind=kind, at=k)
            a, b = tr_o[w][k], tr_g[w][k]
            if kind == "accept":
                rec["gap"] = ratio_gap(a, b)
                rec["u"] = a[4]
            elif kind == "checkpoint":
                rec["drift_oracle"] = max(a[2], a[3])
                rec["drift_device"] = max(b[2], b[3])
                rec["straddle"] = (max(a[2], a[3]) > THRESH) != (max(b[2], b[3]) > THRESH)
        out.append(rec)
    return out


def replay_decisions(trace, events, max_checkpoints):
    """The checkpoint decisions of a trace as (n_walkers, max_checkpoints, 2) {Nfastup after, extra draw}
    for rbmpp_set_replay; unused slots repeat the last decision."""
    nw = trace.shape[0]
    dec = np.zeros((nw, max_checkpoints, 2), dtype=np.int32)
    for w in range(nw):
        rows = [r for r in trace[w][:min(int(events[w, 4]), trace.shape[1])] if r[0] == 1]
        last = (100, 0)
        for k in range(max_checkpoints):
            if k < len(rows):
                r = rows[k]
                last = (int(r[5]), int(r[2] > 10.0 and r[3] > 10.0))
            dec[w, k] = last
    return dec


def summary(recs):
    kinds = {}
    for r in recs:
        kinds[r["kind"]] = kinds.get(r["kind"], 0) + 1
    return kinds
