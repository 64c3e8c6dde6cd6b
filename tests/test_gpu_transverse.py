"""Transverse spin projection on the device: the full N x N skew form of the Pfaffian matrix (skew.cu) against
the oracle, which carries the reference's own 2N form with the transverse code's weights
(beta = -pi/2, pi/2, sqrt(2)-scaled: transverse_code/spin_projection.f90:30-38).

- amplitudes, local energies and O_k of given configurations within 1e-10 (calc_phys_quantity.f90:20-246);
- the summed measurement within 1e-10 / 1e-9 of the largest entry;
- Markov chains decision by decision (make_sample.f90:4-240): both sides carry the same matrix form here, so
  every walker must be exact or part at a documented tie;
- three SR iterations in lock step, with the transverse code's shift schedule
  (transverse_code/main.f90:451: 0.003 instead of 0.001);
- the identity O_b / psi = tanh(b) that this projection implies.
"""
import numpy as np
import pytest

import chain_compare as cc
import pyoracle as po
from rbm_pp_b200 import capi
from rbm_pp_b200 import formats as fm

pytestmark = pytest.mark.gpu

RTOL = 1e-10


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _configs(N, n, seed):
    rng = np.random.default_rng(seed)
    x = -np.ones((n, N), dtype=np.int32)
    for r in x:
        r[rng.choice(N, N // 2, replace=False)] = 1
    return x


def _pair(L, trans, alphar, nw, ns, seed, spin_parity=1, **kw):
    p = fm.synthetic_problem(L, translations=trans, alphar=alphar, nsample=nw * ns, seed=seed,
                             spin_parity=spin_parity, **kw)
    w = fm.spin_projection_weights(spin_parity, transverse=True)
    o = po.Oracle(p, nranks=nw, nsample_per_rank=ns, nthreads=8, sp_weights=w)
    g = capi.Context(p, n_walkers=nw, nsample_per_walker=ns, sp_weights=w)
    o.set_params(p.br, p.Wr, p.slater, 0.0)
    g.set_params(p.br, p.Wr, p.slater, 0.0)
    return p, o, g


@pytest.mark.parametrize("L,trans,alphar,kw", [
    (4, True, 1, dict()),
    (4, False, 2, dict(spin_parity=-1)),
    (6, True, 1, dict()),
    (6, False, 2, dict(orbital="sublattice2")),
])
def test_eval_configs_transverse(L, trans, alphar, kw):
    p, o, g = _pair(L, trans, alphar, 1, 8, seed=40 + L, **kw)
    x = _configs(L * L, 24, seed=L)
    ro = o.eval_configs(x, want_h=True, want_O=True)
    rg = g.eval_configs(x, want_h=True, want_O=True)
    assert _rel(rg["psi"], ro["psi"]) < RTOL
    for k in range(x.shape[0]):
        assert abs(rg["hpsi"][k] - ro["hpsi"][k]) <= RTOL * max(abs(ro["hpsi"][k]), abs(ro["psi"][k, 0]))
        assert np.abs(rg["O"][k] - ro["O"][k].real).max() <= RTOL * np.abs(ro["O"][k]).max(), k
    g.close()


def test_measure_transverse():
    nw, ns = 4, 4
    p, o, g = _pair(6, True, 1, nw, ns, seed=51)
    x = _configs(36, nw * ns, seed=52)
    for c in (o, g):
        c.seed(99)
        c.set_samples(x)
    mo = o.measure(want_S=True)
    mg = g.measure(want_S=True)
    for k in ("Etot", "Etot2", "norm", "wf_av"):
        assert abs(mg[k] - mo[k]) <= RTOL * abs(mo[k]), k
    assert _rel(mg["gvec"], mo["gvec"]) < 1e-9
    assert _rel(mg["Ovec"], mo["Ovec"]) < 1e-9
    assert _rel(mg["S"], mo["S"]) < 1e-9
    g.close()


@pytest.mark.parametrize("L,trans,alphar,nw,ns", [(4, True, 1, 8, 8), (6, False, 1, 4, 4)])
def test_chains_transverse(L, trans, alphar, nw, ns, capsys):
    p, o, g = _pair(L, trans, alphar, nw, ns, seed=60 + L)
    for c in (o, g):
        c.set_trace(8192)
        c.seed(2024)
    kinds = {}
    for first in (True, False):
        na_o = o.make_sample(first)
        na_g = g.make_sample(first)
        eo, to = o.events()
        eg, tg = g.events()
        recs = cc.compare_walkers(to, eo, tg, eg)
        for r in recs:
            assert r["kind"] not in ("type", "draw", "length"), r
            kinds[r["kind"]] = kinds.get(r["kind"], 0) + 1
        xo, xg = o.samples()[0], g.samples()[0]
        for r in recs:
            if r["kind"] == "exact":
                w = r["walker"]
                assert na_o[w] == na_g[w] and np.array_equal(xo[w], xg[w])
        # stored amplitudes against a scratch evaluation
        psig = g.samples()[1]
        scratch = g.eval_configs(xg.reshape(-1, L * L), want_h=False)["psi"]
        assert _rel(psig.reshape(-1, psig.shape[-1])[:, 0], scratch[:, 0]) < 1e-6
    with capsys.disabled():
        print(f"\nTRANSVERSE_CHAINS L={L}: {kinds}")
    assert kinds.get("exact", 0) >= nw  # most walkers over the two calls
    g.close()


def test_bias_derivative_is_tanh_b():
    """At beta = -/+pi/2 the two projection points give the same Pfaffian (B(-cs) = -D B(cs) D with
    D = diag(1 on up, -1 on down electrons)), so O_b / psi = tanh(b) on every configuration: the bias has no
    fluctuation, S_bb vanishes to rounding, and the reference's check i1 /= Nv_RBM (SR_pdposv.f90:32-33) then
    stops on the sign of that rounding.  The lock-step test below therefore runs without RBM units."""
    p, o, g = _pair(4, True, 1, 1, 8, seed=71)
    x = _configs(16, 64, seed=72)
    r = g.eval_configs(x, want_h=False, want_O=True)
    ob = r["O"][:, 0] / r["psi"][:, 0].real
    assert np.abs(ob - np.tanh(p.br[0])).max() <= 1e-12 * abs(np.tanh(p.br[0]))
    g.close()


def test_sr_lockstep_transverse():
    L, nw, ns = 4, 8, 16
    p, o, g = _pair(L, False, 0, nw, ns, seed=12345)
    loop = po.VMCLoop(o, p, iseed0=12345, shift_coef=0.003)
    g.seed(12345)
    br, Wr = capi.initial_params(g, p)
    g.set_params(br, Wr, p.slater, 0.0)
    for it in range(1, 4):
        rec = loop.iteration_step()
        sg = g.iteration(capi.SR_FP64, p.inp.delta_tau, p.inp.s_factor_scale, p.inp.s_cut, p.inp.s_factor0)
        assert np.array_equal(o.samples()[0], g.samples()[0]), it
        assert abs(sg.Etot - rec["Etot"]) <= 1e-9 * abs(rec["Etot"])
        bro, Wro, slo, sho = o.get_params()
        brg, Wrg, slg, shg = g.get_params()
        assert _rel(slg, slo) < 1e-8
        assert abs(shg - sho) <= 1e-9 * abs(sho) + 1e-300
    g.close()
