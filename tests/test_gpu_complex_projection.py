"""Complex amplitudes on the device against the oracle: complex momentum-projection weights para_mp_trans
(sym_info.txt; psi = sum_qp para_mp_trans(mp) ...,
sub.f90:47-50) on the device against the oracle.  psi, H psi and O_k become complex; O keeps a real and an
imaginary row per sample, the Ovec_Store columns of calc_phys_quantity.f90:227-228, so S = sum over both rows and
gvec, Ovec take the real parts of 2 conj(E) O and conj(psi) O (:225-226).

- amplitudes, local energies and O_k of given configurations within 1e-10;
- the summed measurement (scalars 1e-10; gvec, Ovec, S 1e-9 of the largest entry);
- Markov chains decision by decision: exact or parting at a documented tie;
- three SR iterations in lock step with the oracle, FP64 and split-BF16 with refinement;
and complex RBM units (alpha_c > 0: RBM.f90 thetac, 0.5^alpha_c prod cosh(thetac) in sub.f90:37-41, the (re, im)
parameter pairs of calc_phys_quantity.f90:115-160 and SR_pdposv.f90:385-413) the same way.
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


def _momentum(L, kx, ky):
    """para_mp_trans(mp) = exp(2 pi i (kx dx + ky dy) / L) for the translation mp = dx L + dy."""
    dx, dy = np.divmod(np.arange(L * L), L)
    return np.exp(2j * np.pi * (kx * dx + ky * dy) / L)


def _pair(L, alphar, nw, ns, seed, k=(1, 0), **kw):
    p = fm.synthetic_problem(L, translations=True, alphar=alphar, nsample=nw * ns, seed=seed, **kw)
    p.sym.para_mp = _momentum(L, *k)
    o = po.Oracle(p, nranks=nw, nsample_per_rank=ns, nthreads=8)
    g = capi.Context(p, n_walkers=nw, nsample_per_walker=ns)
    assert g.complex_weights
    o.set_params(p.br, p.Wr, p.slater, 0.0)
    g.set_params(p.br, p.Wr, p.slater, 0.0)
    return p, o, g


@pytest.mark.parametrize("L,alphar,k,kw", [(4, 1, (1, 0), dict()), (6, 2, (1, 2), dict(orbital="sublattice2")),
                                           (4, 2, (0, 1), dict(spin_parity=-1))])
def test_eval_configs_complex(L, alphar, k, kw):
    p, o, g = _pair(L, alphar, 1, 8, seed=80 + L, k=k, **kw)
    x = _configs(L * L, 24, seed=L + 1)
    ro = o.eval_configs(x, want_h=True, want_O=True)
    rg = g.eval_configs(x, want_h=True, want_O=True)
    assert np.abs(rg["psi"][:, 0].imag).max() > 1e-3 * np.abs(rg["psi"][:, 0]).max()  # genuinely complex
    assert _rel(rg["psi"], ro["psi"]) < RTOL
    # A momentum sector can nearly annihilate a configuration (|psi| ~ 1e-16 of the batch): its H psi is then
    # rounding noise, so each configuration is compared on the batch's scale.
    hscale = max(np.abs(ro["hpsi"]).max(), np.abs(ro["psi"][:, 0]).max())
    oscale = np.abs(ro["O"]).max()
    for j in range(x.shape[0]):
        assert abs(rg["hpsi"][j] - ro["hpsi"][j]) <= RTOL * max(abs(ro["hpsi"][j]), abs(ro["psi"][j, 0]),
                                                                 1e-3 * hscale), j
        assert np.abs(rg["O"][j] - ro["O"][j]).max() <= RTOL * max(np.abs(ro["O"][j]).max(), 1e-3 * oscale), j
    g.close()


def test_measure_complex():
    nw, ns = 4, 4
    p, o, g = _pair(6, 1, nw, ns, seed=91, k=(2, 1))
    x = _configs(36, nw * ns, seed=92)
    for c in (o, g):
        c.seed(99)
        c.set_samples(x)
    mo = o.measure(want_S=True)
    mg = g.measure(want_S=True)
    for key in ("Etot", "Etot2", "norm", "wf_av"):
        assert abs(mg[key] - mo[key]) <= RTOL * abs(mo[key]), key
    assert _rel(mg["gvec"], mo["gvec"]) < 1e-9
    assert _rel(mg["Ovec"], mo["Ovec"]) < 1e-9
    assert _rel(mg["S"], mo["S"]) < 1e-9
    g.close()


def test_chains_complex(capsys):
    L, nw, ns = 4, 8, 8
    p, o, g = _pair(L, 1, nw, ns, seed=93)
    for c in (o, g):
        c.set_trace(8192)
        c.seed(3030)
    kinds = {}
    for first in (True, False):
        o.make_sample(first)
        g.make_sample(first)
        eo, to = o.events()
        eg, tg = g.events()
        for r in cc.compare_walkers(to, eo, tg, eg):
            assert r["kind"] not in ("type", "draw", "length"), r
            if r["kind"] == "checkpoint":
                assert r["straddle"], r
            kinds[r["kind"]] = kinds.get(r["kind"], 0) + 1
    with capsys.disabled():
        print(f"\nCOMPLEX_CHAINS {kinds}")
    assert kinds.get("exact", 0) >= nw
    g.close()


@pytest.mark.parametrize("precision", [capi.SR_FP64, capi.SR_SPLIT_BF16])
def test_sr_lockstep_complex(precision):
    L, nw, ns = 4, 8, 16
    p, o, g = _pair(L, 1, nw, ns, seed=12345, k=(1, 1))
    loop = po.VMCLoop(o, p, iseed0=12345)
    g.seed(12345)
    br, Wr = capi.initial_params(g, p)
    g.set_params(br, Wr, p.slater, 0.0)
    for it in range(1, 4):
        rec = loop.iteration_step()
        sg = g.iteration(precision, p.inp.delta_tau, p.inp.s_factor_scale, p.inp.s_cut, p.inp.s_factor0)
        assert np.array_equal(o.samples()[0], g.samples()[0]), it
        assert abs(sg.Etot - rec["Etot"]) <= 1e-9 * abs(rec["Etot"])
        bro, Wro, slo, sho = o.get_params()
        brg, Wrg, slg, shg = g.get_params()
        assert _rel(slg, slo) < 1e-8 and _rel(Wrg, Wro) < 1e-8
        assert abs(shg - sho) <= 1e-9 * abs(sho) + 1e-300
    g.close()


# ---- complex RBM units (alpha_c > 0: RBM.f90 thetac, sub.f90:37-41, calc_phys_quantity.f90:115-160) ----

def _units_pair(L, trans, alphac, alphar, nw, ns, seed, **kw):
    p = fm.synthetic_problem(L, translations=trans, alphar=alphar, nsample=nw * ns, seed=seed, **kw)
    p.inp.alphac = alphac
    rng = np.random.default_rng(seed + 1)
    N = L * L
    p.bc = 0.05 * (rng.normal(size=alphac) + 1j * rng.normal(size=alphac))
    p.Wc = 0.05 * (rng.normal(size=(N, alphac)) + 1j * rng.normal(size=(N, alphac)))
    o = po.Oracle(p, nranks=nw, nsample_per_rank=ns, nthreads=8)
    g = capi.Context(p, n_walkers=nw, nsample_per_walker=ns)
    assert g.complex_weights
    o.set_params_c(p.bc, p.Wc)
    o.set_params(p.br, p.Wr, p.slater, 0.0)
    g.set_params(p.br, p.Wr, p.slater, 0.0, bc=p.bc, Wc=p.Wc)
    return p, o, g


@pytest.mark.parametrize("L,trans,alphac,alphar,kw", [(4, False, 1, 1, dict()), (4, True, 2, 1, dict()),
                                                      (6, True, 1, 0, dict(spin_parity=-1))])
def test_eval_configs_complex_units(L, trans, alphac, alphar, kw):
    p, o, g = _units_pair(L, trans, alphac, alphar, 1, 8, seed=100 + L, **kw)
    x = _configs(L * L, 24, seed=L + 7)
    ro = o.eval_configs(x, want_h=True, want_O=True)
    rg = g.eval_configs(x, want_h=True, want_O=True)
    assert _rel(rg["psi"], ro["psi"]) < RTOL
    hscale = max(np.abs(ro["hpsi"]).max(), np.abs(ro["psi"][:, 0]).max())
    oscale = np.abs(ro["O"]).max()
    for j in range(x.shape[0]):
        assert abs(rg["hpsi"][j] - ro["hpsi"][j]) <= RTOL * max(abs(ro["hpsi"][j]), abs(ro["psi"][j, 0]),
                                                                 1e-3 * hscale), j
        assert np.abs(rg["O"][j] - ro["O"][j]).max() <= RTOL * max(np.abs(ro["O"][j]).max(), 1e-3 * oscale), j
    g.close()


def test_chains_complex_units(capsys):
    L, nw, ns = 4, 8, 8
    p, o, g = _units_pair(L, True, 1, 1, nw, ns, seed=111)
    for c in (o, g):
        c.set_trace(8192)
        c.seed(4040)
    kinds = {}
    for first in (True, False):
        o.make_sample(first)
        g.make_sample(first)
        eo, to = o.events()
        eg, tg = g.events()
        for r in cc.compare_walkers(to, eo, tg, eg):
            assert r["kind"] not in ("type", "draw", "length"), r
            if r["kind"] == "checkpoint":
                assert r["straddle"], r
            kinds[r["kind"]] = kinds.get(r["kind"], 0) + 1
    with capsys.disabled():
        print(f"\nCOMPLEX_UNITS_CHAINS {kinds}")
    assert kinds.get("exact", 0) >= nw
    g.close()


@pytest.mark.parametrize("precision", [capi.SR_FP64, capi.SR_SPLIT_BF16])
def test_sr_lockstep_complex_units(precision):
    L, nw, ns = 4, 8, 16
    p, o, g = _units_pair(L, False, 1, 1, nw, ns, seed=12345)
    loop = po.VMCLoop(o, p, iseed0=12345)
    g.seed(12345)
    bc, Wc, br, Wr = capi.initial_params_c(g, p)
    g.set_params(br, Wr, p.slater, 0.0, bc=bc, Wc=Wc)
    for it in range(1, 4):
        rec = loop.iteration_step()
        sg = g.iteration(precision, p.inp.delta_tau, p.inp.s_factor_scale, p.inp.s_cut, p.inp.s_factor0)
        assert np.array_equal(o.samples()[0], g.samples()[0]), it
        assert abs(sg.Etot - rec["Etot"]) <= 1e-9 * abs(rec["Etot"])
        bro, Wro, slo, sho = o.get_params()
        brg, Wrg, slg, shg = g.get_params()
        bco, Wco = o.get_params_c()
        bcg, Wcg = g.get_params_c()
        assert _rel(slg, slo) < 1e-8 and _rel(Wrg, Wro) < 1e-8 and _rel(Wcg, Wco) < 1e-8 and _rel(bcg, bco) < 1e-8
        assert abs(shg - sho) <= 1e-9 * abs(sho) + 1e-300
    g.close()
