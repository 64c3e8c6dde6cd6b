"""Estimator parity with the oracle at the benched shape and on the reference's edge cases.

The benched shape is 10x10 with 100 translations (200 Pfaffian blocks of 50 x 50) and alpha_r = 4: the
compile-time 50-block estimator and correlation kernels.  The edge cases are spin_parity = -1
(spin_projection.f90:56-62), the 2-sublattice orbital map (several (i, j) pairs share one f, so dPf/df_k is
accumulated with atomics, slater.f90:140-167) and J2 in {0.40, 0.60}.  Amplitudes, local energies and O_k
agree within 1e-10 relative (FP64); the summed measurement within 1e-10 (scalars) and 1e-9 of the largest
entry (gvec, Ovec); correlations within 1e-10 of each array's largest entry.
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


def _configs(N, n, seed):
    rng = np.random.default_rng(seed)
    x = -np.ones((n, N), dtype=np.int32)
    for r in x:
        r[rng.choice(N, N // 2, replace=False)] = 1
    return x


def _pair(L, trans, alphar, nw, ns, seed, **kw):
    p = fm.synthetic_problem(L, translations=trans, alphar=alphar, nsample=nw * ns, seed=seed, **kw)
    o = po.Oracle(p, nranks=nw, nsample_per_rank=ns, nthreads=8)
    g = capi.Context(p, n_walkers=nw, nsample_per_walker=ns)
    o.set_params(p.br, p.Wr, p.slater, 0.0)
    g.set_params(p.br, p.Wr, p.slater, 0.0)
    return p, o, g


def _eval_match(o, g, x):
    ro = o.eval_configs(x, want_h=True, want_O=True)
    rg = g.eval_configs(x, want_h=True, want_O=True)
    assert _rel(rg["psi"], ro["psi"]) < RTOL
    for k in range(x.shape[0]):
        assert abs(rg["hpsi"][k] - ro["hpsi"][k]) <= RTOL * max(abs(ro["hpsi"][k]), abs(ro["psi"][k, 0]))
        # every O_k relative to its own configuration's largest derivative
        assert np.abs(rg["O"][k] - ro["O"][k].real).max() <= RTOL * np.abs(ro["O"][k]).max()
    return ro, rg


def _measure_match(o, g, x, want_S=False):
    o.seed(99)
    g.seed(99)
    o.set_samples(x)
    g.set_samples(x)
    mo = o.measure(want_S=want_S)
    mg = g.measure(want_S=want_S)
    for k in ("Etot", "Etot2", "norm", "wf_av"):
        assert abs(mg[k] - mo[k]) <= RTOL * abs(mo[k]), k
    assert _rel(mg["gvec"], mo["gvec"]) < 1e-9
    assert _rel(mg["Ovec"], mo["Ovec"]) < 1e-9
    if want_S:
        assert _rel(mg["S"], mo["S"]) < 1e-9


def test_eval_configs_10x10_translations():
    p, o, g = _pair(10, True, 4, 1, 16, seed=5)
    _eval_match(o, g, _configs(100, 16, seed=10))
    g.close()


def test_measure_10x10_translations():
    nw, ns = 4, 2
    p, o, g = _pair(10, True, 4, nw, ns, seed=6)
    _measure_match(o, g, _configs(100, nw * ns, seed=11))
    g.close()


def test_correlation_10x10_translations():
    nw, ns = 2, 1
    p, o, g = _pair(10, True, 4, nw, ns, seed=7)
    x = _configs(100, nw * ns, seed=12)
    o.seed(2024)
    g.seed(2024)
    o.set_samples(x)
    g.set_samples(x)
    mo = o.measure_correlation()
    mg = g.measure_correlation()
    for k in ("Etot", "Etot2", "norm", "wf_av", "wf_sgn"):
        assert abs(mg[k] - mo[k]) <= RTOL * abs(mo[k]), k
    assert _rel(mg["chi_sp"], mo["chi_sp"]) < RTOL
    assert _rel(mg["chi_vbs"], mo["chi_vbs"]) < RTOL
    assert np.array_equal(o.rank_grnd(0, 8), g.rank0_grnd(8))
    g.close()


@pytest.mark.parametrize("L,trans,alphar,kw", [
    (4, True, 1, dict(spin_parity=-1)),
    (6, True, 2, dict(spin_parity=-1)),
    (6, False, 2, dict(orbital="sublattice2")),
    (6, True, 1, dict(orbital="sublattice2")),
    (4, True, 2, dict(J2=0.4)),
    (6, False, 1, dict(J2=0.6)),
])
def test_edge_cases(L, trans, alphar, kw):
    nw, ns = 3, 4
    p, o, g = _pair(L, trans, alphar, nw, ns, seed=17 + L, **kw)
    _eval_match(o, g, _configs(L * L, 12, seed=L))
    _measure_match(o, g, _configs(L * L, nw * ns, seed=L + 1), want_S=True)
    g.close()


@pytest.mark.parametrize("L", [16, 18])
def test_estimator_large_blocks(L):
    """N/2 = 128 and 162: the estimator's Gauss-Jordan tiles no longer fit one block's shared memory and move to
    a global scratch slice per block, one block per SM looping over the configurations.  Amplitudes, local
    energies and O_k against the oracle at 1e-10; the summed measurement of stored samples too."""
    nw, ns = 2, 2
    p, o, g = _pair(L, False, 2, nw, ns, seed=130 + L)
    _eval_match(o, g, _configs(L * L, 6, seed=L))
    _measure_match(o, g, _configs(L * L, nw * ns, seed=L + 1))
    g.close()


@pytest.mark.parametrize("L,nw", [(16, 2), (18, 1)])
def test_correlation_large_blocks(L, nw):
    """The correlation measurement where its tiles and the N/2 x N/2 table of exchanged amplitudes no longer fit
    one block's shared memory (global scratch per block, one block per SM looping over the samples), against the
    oracle at 1e-10."""
    ns = 1
    p, o, g = _pair(L, False, 2, nw, ns, seed=150 + L)
    x = _configs(L * L, nw * ns, seed=L + 2)
    o.seed(2025)
    g.seed(2025)
    o.set_samples(x)
    g.set_samples(x)
    mo = o.measure_correlation()
    mg = g.measure_correlation()
    for k in ("Etot", "Etot2", "norm", "wf_av", "wf_sgn"):
        assert abs(mg[k] - mo[k]) <= RTOL * abs(mo[k]), k
    assert _rel(mg["chi_sp"], mo["chi_sp"]) < RTOL
    assert _rel(mg["chi_vbs"], mo["chi_vbs"]) < RTOL
    g.close()
