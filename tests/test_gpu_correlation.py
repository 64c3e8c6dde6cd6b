"""Parity of the correlation measurement (rbmpp_measure_correlation) with the oracle.

Chi_sp, Chi_vbs and the energy scalars of the same configurations agree within 1e-10, relative to each
array's largest entry (FP64).  Each walker's stream must advance by one draw per sample, antiparallel bond
and antiparallel site pair on both sides: checked on walker 0's next draws, and in lockstep with sampling
(sample, measure, sample again: the second chains are bit-identical only if every stream advanced alike).
"""
import numpy as np
import pytest

import pyoracle as po
from rbm_pp_b200 import capi
from rbm_pp_b200 import formats as fm

pytestmark = pytest.mark.gpu

RTOL = 1e-10


def _rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _random_configs(N, n, seed):
    rng = np.random.default_rng(seed)
    x = -np.ones((n, N), dtype=np.int32)
    for r in x:
        r[rng.choice(N, N // 2, replace=False)] = 1
    return x


def _pair(L, trans, alphar, nw, ns, seed):
    p = fm.synthetic_problem(L, translations=trans, alphar=alphar, nsample=nw * ns, seed=seed, J2=0.55)
    o = po.Oracle(p, nranks=nw, nsample_per_rank=ns, nthreads=4)
    g = capi.Context(p, n_walkers=nw, nsample_per_walker=ns)
    o.set_params(p.br, p.Wr, p.slater, 0.0)
    g.set_params(p.br, p.Wr, p.slater, 0.0)
    return o, g


def _compare(mo, mg):
    for k in ("Etot", "Etot2", "norm", "wf_av", "wf_sgn"):
        assert abs(mg[k] - mo[k]) <= RTOL * abs(mo[k]), k
    assert _rel(mg["chi_sp"], mo["chi_sp"]) < RTOL
    assert _rel(mg["chi_vbs"], mo["chi_vbs"]) < RTOL


@pytest.mark.parametrize("L,trans,alphar,nw,ns", [(4, False, 1, 4, 4), (4, True, 1, 2, 3), (6, True, 2, 2, 2),
                                                  (8, False, 2, 3, 2), (10, False, 2, 2, 1), (12, False, 1, 2, 1)])
def test_correlation_matches_oracle(L, trans, alphar, nw, ns):
    """The same configurations on both sides (uniform Sz = 0), the same RNG state before the measurement."""
    o, g = _pair(L, trans, alphar, nw, ns, seed=40 + L)
    x = _random_configs(L * L, nw * ns, seed=L)
    o.seed(2024)
    g.seed(2024)
    o.set_samples(x)
    g.set_samples(x)
    _compare(o.measure_correlation(), g.measure_correlation())
    # walker 0's stream advanced by the same number of amplitude draws
    assert np.array_equal(o.rank_grnd(0, 16), g.rank0_grnd(16))
    g.close()


def test_correlation_in_sampling_lockstep():
    """Sample, measure the correlations, sample again: every walker's stream advanced alike, so the
    second chains are bit-identical."""
    o, g = _pair(4, False, 1, 4, 4, seed=44)
    o.seed(2024)
    g.seed(2024)
    assert np.array_equal(o.make_sample(True), g.make_sample(True))
    assert np.array_equal(o.samples()[0], g.samples()[0])
    _compare(o.measure_correlation(), g.measure_correlation())
    assert np.array_equal(o.make_sample(False), g.make_sample(False))
    assert np.array_equal(o.samples()[0], g.samples()[0])
    g.close()


def test_correlation_energy_matches_measure_energy():
    """The correlation measurement's scalars equal the plain final-energy measurement's on the same samples."""
    L, nw, ns = 6, 3, 2
    p = fm.synthetic_problem(L, translations=True, alphar=1, nsample=nw * ns, seed=7, J2=0.5)
    g = capi.Context(p, n_walkers=nw, nsample_per_walker=ns)
    g.set_params(p.br, p.Wr, p.slater, 0.0)
    g.seed(11)
    g.make_sample(True)
    mc = g.measure_correlation()
    me = g.measure_energy()
    for k in ("Etot", "Etot2", "norm", "wf_av"):
        assert abs(mc[k] - me[k]) <= RTOL * abs(me[k]), k
    g.close()
