"""Failure detection: the reference's `stop` conditions become status codes, found on the host or by the
kernels, and a bounded device wait that runs out returns RBMPP_E_TIMEOUT with the context still usable.

No test here faults, traps or hangs a GPU.  Bad inputs are made on the host (a non-permutation W_map, an
out-of-range orbital index, a sublattice flag of 2, non-finite spin-projection weights, a transverse
projection beyond the skew form's size, a stored sample outside the Sz = 0 sector).  The timeout is made by a verification hook: walker 0 never issues one bulk
load, so the wait on it runs out after a short poll bound.
"""
import numpy as np
import pytest

from rbm_pp_b200 import capi
from rbm_pp_b200 import formats as fm

pytestmark = pytest.mark.gpu

E_ARG, E_CONFIG, E_TIMEOUT = 1, 2, 22


def _problem(L=4, trans=True, **kw):
    return fm.synthetic_problem(L, translations=trans, alphar=1, nsample=32, seed=9, **kw)


def _ctx(p, nw=4, ns=8, **kw):
    g = capi.Context(p, n_walkers=nw, nsample_per_walker=ns, **kw)
    g.set_params(p.br, p.Wr, p.slater, 0.0)
    return g


def _refused(p, msg, **kw):
    with pytest.raises(capi.RbmppError) as ei:
        capi.Context(p, n_walkers=1, nsample_per_walker=1, **kw)
    assert ei.value.code == E_ARG and msg in str(ei.value), str(ei.value)


def test_bad_tables_are_refused():
    p = _problem()
    W = p.sym.W_map.copy()
    W[1, 3] = W[0, 3]  # not a permutation (main.f90:117-121)
    p.sym.W_map = W
    _refused(p, "W_map wrong 2")
    p = _problem()
    W = p.sym.W_map.copy()
    W[2, 0] = 0
    p.sym.W_map = W
    _refused(p, "W_map wrong 1")
    p = _problem()
    o = p.orbital_idx.copy()
    o[3, 5] = p.n_slater + 1  # parameter.f90:96-99
    p.orbital_idx = o
    _refused(p, "error4")
    p = _problem()
    sb = np.zeros(16, dtype=np.int32)
    sb[7] = 2
    _refused(p, "neither 0 nor 1", subB=sb)
    spw = fm.spin_projection_weights(1, transverse=True)
    spw[1, 0] = np.nan
    _refused(_problem(), "non-finite value", sp_weights=spw)
    # the skew form (transverse projection) takes N <= 128
    _refused(_problem(L=12), "supports N <= 128", sp_weights=fm.spin_projection_weights(1, transverse=True))
    p = _problem()
    p.sym.para_mp = p.sym.para_mp.astype(np.complex128) + 0.5j
    _refused(p, "with the transverse (skew-form) projection", sp_weights=fm.spin_projection_weights(1, True))


def test_explicit_tables_equal_defaults():
    """subB and the spin-projection weights given explicitly, equal to the defaults, give bit-identical chains
    and measurements (spin_parity = -1, so the second weight is -1)."""
    p = _problem(spin_parity=-1)
    L = p.inp.L
    sb = np.array([(i // L + i % L) % 2 for i in range(L * L)], dtype=np.int32)
    spw = np.array([[np.cos(0.0), np.sin(0.0), 1.0], [np.cos(0.5 * np.pi), np.sin(0.5 * np.pi), -1.0]]).T
    out = []
    for kw in (dict(), dict(subB=sb, sp_weights=spw)):
        g = _ctx(p, **kw)
        g.seed(123)
        na = g.make_sample(True)
        x = g.samples()[0]
        m = g.measure(want_S=False)
        out.append((na, x, m))
        g.close()
    (na0, x0, m0), (na1, x1, m1) = out
    assert np.array_equal(na0, na1) and np.array_equal(x0, x1)
    for k in ("Etot", "Etot2", "norm", "wf_av"):
        assert m0[k] == m1[k], k
    assert np.array_equal(m0["gvec"], m1["gvec"]) and np.array_equal(m0["Ovec"], m1["Ovec"])


def test_corrupt_sample_is_refused_and_context_recovers():
    """A stored configuration outside the Sz = 0 sector (x_to_Ele_Idx_Ele_Cfg, interface_for_PP.f90:26-65)
    is refused with RBMPP_E_CONFIG; the context measures correct samples afterwards."""
    p = _problem()
    g = _ctx(p)
    g.seed(5)
    g.make_sample(True)
    x = g.samples()[0].copy()
    m_good = g.measure(want_S=False)
    bad = x.copy()
    bad[2, 3, :] = 1  # all spins up
    g.set_samples(bad)
    with pytest.raises(capi.RbmppError) as ei:
        g.measure(want_S=False)
    assert ei.value.code == E_CONFIG, str(ei.value)
    g.set_samples(x)
    m = g.measure(want_S=False)
    assert m["Etot"] == m_good["Etot"] and m["norm"] == m_good["norm"]
    g.close()


def test_bounded_wait_runs_out_and_context_recovers():
    """Walker 0 of the streaming sampler never issues its 5th bulk load; its consumers' bounded wait (4096
    polls) runs out, the CTA drains its copies in flight and returns ST_TIMEOUT, and make_sample reports
    RBMPP_E_TIMEOUT.  With the hooks off, the same context samples again, twice, and its stored amplitudes
    agree with a scratch evaluation (every walker's state was rebuilt from its configuration)."""
    p = _problem(L=6)
    g = _ctx(p, nw=4, ns=2)
    g.seed(77)
    g.debug_hook(2, 4096)
    g.debug_hook(1, 5)
    with pytest.raises(capi.RbmppError) as ei:
        g.make_sample(True)
    assert ei.value.code == E_TIMEOUT, str(ei.value)
    g.debug_hook(1, 0)
    g.debug_hook(2, 0)
    g.seed(78)
    na = g.make_sample(True)
    x, psi, _ = g.samples()
    scratch = g.eval_configs(x.reshape(-1, 36), want_h=False)["psi"]
    assert np.abs(psi.reshape(-1, psi.shape[-1])[:, 0] - scratch[:, 0]).max() <= 1e-6 * np.abs(scratch[:, 0]).max()
    assert (na > 0).all()
    g.make_sample(False)
    g.close()
